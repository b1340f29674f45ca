"""Mesh solve: reliability-guided propagation over GPU subset batches.

``Mesh`` mirrors the reference's Python ``Mesh.solve`` (python/src/py_mesh.rs
:215-291; Rust Mesh::solve / solve_impl, src/mesh.rs:599-857) for a mesh
whose nodes and elements the caller already has (mesh generation,
Mesh::new's refinement, is not part of this library).  The propagation runs
in the C++ driver of the library (gpv_mesh_solve): seed node, RG cascade or
layer-RG rounds, one GPU batch per graph colour, the two attempts of each
node solve.  The corrections stage (src/mesh.rs:766-790) is left to the
caller; the quality gate (:792-799) is applied to the propagated result.

``mesh_drive`` runs the same driver over any Python batch solver.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import _lib
from ._lib import DESC_DTYPE, PREC_MIXED, RESULT_DTYPE, GpvError, MeshParams, MeshStats, check, lib, ptr


def _mesh_params(radius, seed_coord, seed_warp, seed_tolerance, max_norm, max_iterations, subset_order, tolerance,
                 preconditioning, batch_factor, root_rel_eps, max_workers, precision, mask, progress, method="icgn",
                 texture="deformable"):
    if subset_order not in (1, 2):
        raise ValueError("subset_order must be 1 or 2 for a mesh (p_len = 6 * subset_order)")
    if preconditioning not in ("RG", "layer-RG"):
        raise ValueError(f"preconditioning must be 'RG' or 'layer-RG', got {preconditioning!r}")
    if batch_factor < 1:
        raise ValueError("layer_rg_batch_factor must be >= 1")
    m = MeshParams()
    m.seed_coord[0], m.seed_coord[1] = float(seed_coord[0]), float(seed_coord[1])
    w = [] if seed_warp is None else [float(v) for v in seed_warp]
    for k, v in enumerate(w[:12]):
        m.seed_warp[k] = v
    m.seed_tolerance, m.max_norm, m.tolerance, m.root_rel_eps = seed_tolerance, max_norm, tolerance, root_rel_eps
    m.max_iterations, m.subset_order, m.radius, m.precision = max_iterations, subset_order, radius, precision
    if method not in ("icgn", "fagn"):
        raise ValueError(f"method must be 'icgn' or 'fagn', got {method!r}")
    m.method = 1 if method == "fagn" else 0
    if texture not in ("deformable", "rigid"):  # check_texture (python/src/py_mesh.rs:954-961)
        raise ValueError(f"texture must be 'deformable' or 'rigid', got {texture!r}")
    m.texture = 1 if texture == "rigid" else 0
    m.layer_rg = int(preconditioning == "layer-RG")
    m.batch_factor = batch_factor
    # layer_rg_max_workers=None: the reference sizes rounds by its global
    # worker pool, one worker per logical CPU
    m.max_workers = int(max_workers) if max_workers is not None else (os.cpu_count() or 1)
    m.mask = mask.handle if mask is not None else None
    cb = None
    if progress is not None:
        def _cb(user, done, total):
            try:
                return 1 if progress(int(done), int(total)) else 0
            except Exception:
                return 1
        cb = _lib.PROGRESS_FN(_cb)
        m.progress = cb
    return m, cb


def _arrays(nodes, elements):
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elements = np.ascontiguousarray(elements, dtype=np.int64)
    if nodes.ndim != 2 or nodes.shape[1] != 2:
        raise ValueError("nodes must be (n, 2)")
    if elements.ndim != 2 or elements.shape[1] not in (3, 6):
        raise ValueError("elements must be (m, 3) or (m, 6)")
    return nodes, elements


class Cancelled(GpvError):
    """The progress observer stopped the solve (src/error.rs Cancelled)."""


def _finish(rc, what, out, rounds, st):
    if rc == -4:
        raise Cancelled(f"{what}: cancelled")
    check(rc, what)
    return dict(results=out, rounds=rounds, seed_node=int(st.seed_node),
                stats={k: int(getattr(st, k)) for k, _ in MeshStats._fields_})


def mesh_drive(nodes, elements, solver, *, radius, seed_coord, seed_warp=None, seed_tolerance=0.9, max_norm=1e-5,
               max_iterations=50, subset_order=1, tolerance=0.75, preconditioning="RG", layer_rg_batch_factor=4,
               layer_rg_root_rel_eps=0.02, layer_rg_max_workers=None, progress=None):
    """The library's mesh driver (gpv_mesh_drive) over `solver(desc, tolerance)
    -> RESULT_DTYPE array`.  Returns dict(results, rounds, seed_node, stats)."""
    nodes, elements = _arrays(nodes, elements)
    m, keep = _mesh_params(radius, seed_coord, seed_warp, seed_tolerance, max_norm, max_iterations, subset_order,
                           tolerance, preconditioning, layer_rg_batch_factor, layer_rg_root_rel_eps,
                           layer_rg_max_workers, PREC_MIXED, None, progress)

    failure = []

    def _solve(user, desc_p, n, tol, out_p):
        try:
            d = np.frombuffer((ct.c_char * (n * DESC_DTYPE.itemsize)).from_address(desc_p), dtype=DESC_DTYPE).copy()
            r = np.ascontiguousarray(solver(d, tol), dtype=RESULT_DTYPE)
            if r.shape != (n,):
                raise ValueError(f"solver returned {r.shape} results for {n} subsets")
            ct.memmove(out_p, r.ctypes.data, n * RESULT_DTYPE.itemsize)
            return 0
        except Exception as e:  # reported after the driver returns
            failure.append(e)
            return -1

    cb = _lib.BATCH_SOLVER_FN(_solve)
    out = np.zeros(len(nodes), RESULT_DTYPE)
    rounds = np.zeros(len(nodes), np.int32)
    st = MeshStats()
    rc = lib().gpv_mesh_drive(ptr(nodes), len(nodes), ptr(elements), len(elements), elements.shape[1], ct.byref(m),
                              cb, None, ptr(out), ptr(rounds), ct.byref(st))
    del keep
    if failure:
        raise failure[0]
    return _finish(rc, "gpv_mesh_drive", out, rounds, st)


class Mesh:
    """A mesh of subsets solved on the GPU (python/src/py_mesh.rs:84-380).

    nodes (n, 2) as (x, y); elements (m, 3) or (m, 6) node indices (6-node
    elements: corners then the mid-side nodes 01, 12, 20, src/mesh.rs:1744-1751).
    """

    def __init__(self, nodes, elements, f_img, g_img, mask=None):
        self.nodes, self.elements = _arrays(nodes, elements)
        self.f_img, self.g_img, self.mask = f_img, g_img, mask
        self.mesh_order = 2 if self.elements.shape[1] == 6 else 1
        self._sol = None

    def solve(self, local_mask, seed_coord, seed_warp=None, max_norm=1e-5, max_iterations=50, subset_order=1,
              tolerance=0.75, seed_tolerance=0.9, method="icgn", override_active=False, preconditioning="RG",
              masking="uniform", texture="deformable", layer_rg_batch_factor=4, layer_rg_root_rel_eps=0.02,
              layer_rg_max_workers=None, precision=PREC_MIXED, progress=None):
        """Mesh.solve (python/src/py_mesh.rs:215-291).  `local_mask` is a
        ``gpv.Mask("local", shape="circle", size=r)`` or the radius itself."""
        if masking != "uniform":
            raise NotImplementedError("only masking='uniform' runs on the GPU")
        radius = int(getattr(local_mask, "size", local_mask))
        m, keep = _mesh_params(radius, seed_coord, seed_warp, seed_tolerance, max_norm, max_iterations, subset_order,
                               tolerance, preconditioning, layer_rg_batch_factor, layer_rg_root_rel_eps,
                               layer_rg_max_workers, precision, self.mask, progress, method, texture)
        if texture == "rigid":
            self.f_img.build_grain()
        out = np.zeros(len(self.nodes), RESULT_DTYPE)
        rounds = np.zeros(len(self.nodes), np.int32)
        st = MeshStats()
        self._sol = None
        rc = lib().gpv_mesh_solve(self.f_img.ctx.handle, self.f_img.handle, self.g_img.handle, ptr(self.nodes),
                                  len(self.nodes), ptr(self.elements), len(self.elements), self.elements.shape[1],
                                  ct.byref(m), ptr(out), ptr(rounds), ct.byref(st))
        del keep
        sol = _finish(rc, "gpv_mesh_solve", out, rounds, st)
        sol["subset_order"] = subset_order
        if not override_active and sol["stats"]["n_bad"] > 0:
            raise GpvError(f"mesh unsolvable: {sol['stats']['n_bad']} subset(s) failed to reach quality_ok")
        self._sol = sol

    @property
    def solved(self) -> bool:
        return self._sol is not None

    def _r(self):
        if self._sol is None:
            raise GpvError("mesh not solved")
        return self._sol

    @property
    def results(self) -> np.ndarray:
        return self._r()["results"]

    @property
    def p(self) -> np.ndarray:
        r = self._r()
        return r["results"]["p"][:, :6 * r["subset_order"]].copy()

    @property
    def displacements(self) -> np.ndarray:
        return self._r()["results"]["p"][:, :2].copy()

    @property
    def c_zncc(self) -> np.ndarray:
        return np.fmax(self._r()["results"]["c_zncc"], 0.0)

    @property
    def quality_ok(self) -> np.ndarray:
        return self._r()["results"]["quality_ok"].astype(bool)

    @property
    def iterations(self) -> np.ndarray:
        return self._r()["results"]["iterations"].copy()

    @property
    def norms(self) -> np.ndarray:
        return self._r()["results"]["norm"].copy()

    @property
    def seed_node(self) -> int:
        return self._r()["seed_node"]

    @property
    def rounds(self) -> np.ndarray:
        return self._r()["rounds"]

    @property
    def stats(self) -> dict:
        return self._r()["stats"]
