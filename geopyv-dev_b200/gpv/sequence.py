"""Mesh sequences: Sequence::solve (src/sequence.rs:624-968) over gpv.Mesh.

Each image pair is a mesh solve on the GPU (``gpv.Mesh.solve``, the
reference's propagation); the pair loop, the reference-update fallback, the
override retry, sequential reference updates and the seed guidance between
pairs follow the reference.  Images are re-prefiltered in place
(``Image.update``) instead of being rebuilt per pair, and a sequential
reference update swaps the two images' roles, so the coefficients of the
previous target are reused as the new reference without another prefilter.

The mesh is the caller's (nodes, elements) for every pair -- the reference's
``sync`` reuse; generating a new mesh per pair (Mesh::new) and the ``tracked``
topology are not part of this library.

Seed guidance (deformation_preconditioning, src/sequence.rs:1062-1097): the
pair's displacement field is interpolated at the seed through the element
that holds it (element_locator, src/particle.rs:968-1018; local_coordinates,
shape_function and warp_increment, :135-330), strain terms clipped to
[-0.99, 0.99] as apply_warp_increment does (:1426-1434).
"""
from __future__ import annotations

import numpy as np

from ._lib import GpvError
from .mesh import Cancelled, Mesh


def _det3(a00, a01, a02, a10, a11, a12, a20, a21, a22):
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20)


def local_coordinates(coord, element_nodes):
    """Area coordinates (zeta, eta, theta) of coord in the element's corner triangle."""
    px, py = coord
    (n0x, n0y), (n1x, n1y), (n2x, n2y) = element_nodes[0], element_nodes[1], element_nodes[2]
    den = _det3(1.0, 1.0, 1.0, n0x, n1x, n2x, n0y, n1y, n2y)
    zeta = _det3(1.0, 1.0, 1.0, px, n1x, n2x, py, n1y, n2y) / den
    eta = _det3(1.0, 1.0, 1.0, px, n2x, n0x, py, n2y, n0y) / den
    return zeta, eta, 1.0 - zeta - eta, den


def shape_function(order, z, e, t):
    if order == 1:
        return np.array([z, e, t]), np.array([[1.0, 0.0, -1.0], [0.0, 1.0, -1.0]]), None
    n = np.array([z * (2 * z - 1), e * (2 * e - 1), t * (2 * t - 1), 4 * z * e, 4 * e * t, 4 * t * z])
    dn = np.array([[4 * z - 1, 0.0, 1 - 4 * t, 4 * e, -4 * e, 4 * (t - z)],
                   [0.0, 4 * e - 1, 1 - 4 * t, 4 * z, 4 * (t - e), -4 * z]])
    d2n = np.array([[4.0, 0, 4, 0, 0, -8], [0, 0, 4, 4, -4, -4], [0, 4, 4, 0, -8, 0]])
    return n, dn, d2n


def warp_increment(coord, element_nodes, element_disps, mesh_order):
    """[u, v, u_x, v_x, u_y, v_y (, second-order terms)] of the element field at coord."""
    x = np.asarray(element_nodes, dtype=np.float64)
    u = np.asarray(element_disps, dtype=np.float64)
    z, e, t, den = local_coordinates(coord, x)
    n, dn, d2n = shape_function(mesh_order, z, e, t)
    w = np.zeros(6 * mesh_order)
    w[:2] = n @ u
    jx, ju = dn @ x, dn @ u
    det = jx[0, 0] * jx[1, 1] - jx[0, 1] * jx[1, 0]
    inv = np.array([[jx[1, 1], -jx[0, 1]], [-jx[1, 0], jx[0, 0]]]) / det
    g = inv @ ju
    w[2:6] = g[0, 0], g[0, 1], g[1, 0], g[1, 1]
    if mesh_order == 2:
        dz = np.array([[x[1, 1] - x[2, 1], x[2, 1] - x[0, 1]], [x[2, 0] - x[1, 0], x[0, 0] - x[2, 0]]]) / den
        (d00, d01), (d10, d11) = dz
        kxi = np.array([[d00 * d00, 2 * d00 * d01, d01 * d01],
                        [d00 * d10, d00 * d11 + d01 * d10, d01 * d11],
                        [d10 * d10, 2 * d10 * d11, d11 * d11]])
        w[6:12] = (kxi @ (d2n @ u)).ravel()
    return w


def element_locator(coord, nodes, elements):
    """(element, adrift): the first element by centroid distance whose corner
    triangle holds coord, else the nearest centroid's with adrift = True."""
    c = nodes[elements[:, :3]].mean(axis=1)
    d = ((c[:, 0] - coord[0]) ** 2 + (c[:, 1] - coord[1]) ** 2)
    for idx in np.argsort(d, kind="stable"):
        z, e, t, _ = local_coordinates(coord, nodes[elements[idx, :3]])
        if z >= 0.0 and e >= 0.0 and t >= 0.0:
            return int(idx), False
    return int(np.argmin(d)), True


def deformation_preconditioning(nodes, elements, displacements, seed_coord, mesh_order, subset_order):
    """(seed displacement, seed warp of 6 * subset_order terms) for the next pair."""
    nodes = np.asarray(nodes, dtype=np.float64)
    elements = np.asarray(elements)
    idx, _ = element_locator(seed_coord, nodes, elements)
    el = elements[idx]
    w = warp_increment(seed_coord, nodes[el], np.asarray(displacements)[el], mesh_order)
    w[2:] = np.clip(w[2:], -0.99, 0.99)
    out = np.zeros(6 * subset_order)
    k = 6 * min(mesh_order, subset_order)
    out[:k] = w[:k]
    return w[:2].copy(), out


class Sequence:
    """Sequence of images solved pair by pair (python/src/py_sequence.rs).

    ``frames``: greyscale arrays (or RGB8 arrays with ``rgb=True``), all of
    one shape; ``nodes``, ``elements``: the mesh for every pair.
    """

    def __init__(self, frames, nodes, elements, border: int = 20, ctx=None, rgb: bool = False, mask=None):
        if len(frames) < 2:
            raise ValueError("a sequence needs at least two images")
        self.frames = frames
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.elements = np.ascontiguousarray(elements, dtype=np.int64)
        self.mesh_order = 2 if self.elements.shape[1] == 6 else 1
        self.border, self.ctx, self.rgb, self.mask = border, ctx, rgb, mask
        self.solution = None

    def _image(self, k, grain=False):
        from . import Image
        if self.rgb:
            return Image(image_rgb=self.frames[k], border=self.border, ctx=self.ctx, grain=grain)
        return Image(image_gs=self.frames[k], border=self.border, ctx=self.ctx, grain=grain)

    def _load(self, img, k):
        if self.rgb:
            img.update_rgb(self.frames[k])
        else:
            img.update(self.frames[k])

    def solve(self, local_mask, seed_coord, seed_warp=None, seed_tolerance=0.9, max_norm=1e-5, max_iterations=50,
              subset_order=1, tolerance=0.75, method="icgn", guide=True, sequential=False, override=False,
              preconditioning="RG", layer_rg_batch_factor=4, layer_rg_root_rel_eps=0.02, layer_rg_max_workers=None,
              precision=0, progress=None, texture="deformable"):
        """Sequence::solve (src/sequence.rs:624-968) with the options guide,
        sequential and override; returns and keeps a dict with one entry per
        solved pair (f_index, g_index, results, rounds, seed_coord) and the
        reference-update and override logs."""
        n_images = len(self.frames)
        n_pairs = n_images - 1
        warp_len = 6 * subset_order
        seed_coord = [float(seed_coord[0]), float(seed_coord[1])]
        sw = np.zeros(warp_len)
        if seed_warp is not None:
            v = np.asarray(seed_warp, dtype=np.float64).ravel()[:warp_len]
            sw[:len(v)] = v
        f_index, g_index = 0, 1
        # with the rigid texture both images keep grain maps: a sequential
        # update makes the target the next reference
        rigid = texture == "rigid"
        F, G = self._image(f_index, rigid), self._image(g_index, rigid and sequential)
        pairs, override_log = [], []
        reference_updates = [False] * n_pairs
        mesh_override = pending_ref_update = False
        unsolvable = False
        while True:
            mesh = Mesh(self.nodes, self.elements, F, G, mask=self.mask)
            kw = dict(seed_coord=tuple(seed_coord), seed_warp=list(sw), seed_tolerance=seed_tolerance,
                      max_norm=max_norm, max_iterations=max_iterations, subset_order=subset_order,
                      tolerance=0.0 if mesh_override else tolerance, method=method,
                      override_active=mesh_override, preconditioning=preconditioning,
                      layer_rg_batch_factor=layer_rg_batch_factor, layer_rg_root_rel_eps=layer_rg_root_rel_eps,
                      layer_rg_max_workers=layer_rg_max_workers, precision=precision, progress=progress,
                      texture=texture)
            try:
                mesh.solve(local_mask, **kw)
            except Cancelled:
                raise
            except GpvError:
                if f_index + 1 < g_index:  # non-consecutive pair failed: step the reference forward (:806-818)
                    f_index = g_index - 1
                    self._load(F, f_index)
                    pending_ref_update = True
                    if override:
                        mesh_override = True
                    continue
                unsolvable = True  # consecutive pair unsolvable: curtail the sequence (:819-838)
                break
            if mesh_override:  # (:859-865)
                if np.any(mesh.c_zncc < tolerance):
                    override_log.append(g_index)
                mesh_override = False
            if pending_ref_update:
                if len(pairs) < n_pairs:
                    reference_updates[len(pairs)] = True
                pending_ref_update = False
            pairs.append(dict(f_index=f_index, g_index=g_index, results=mesh.results.copy(),
                              rounds=mesh.rounds.copy(), seed_node=mesh.seed_node, seed_coord=tuple(seed_coord),
                              stats=mesh.stats))
            g_index += 1
            if g_index >= n_images:
                break
            displacements = mesh.displacements
            if sequential:  # the previous target becomes the reference: swap, then load the new target
                F, G = G, F
                f_index = g_index - 1
                reference_updates[g_index - 1] = True
            self._load(G, g_index)
            if guide:  # (:922-937)
                disp, new_warp = deformation_preconditioning(self.nodes, self.elements, displacements, seed_coord,
                                                             self.mesh_order, subset_order)
                seed_coord[0] += disp[0]
                seed_coord[1] += disp[1]
                n_copy = 6 * min(self.mesh_order, subset_order)
                sw[:n_copy] = new_warp[:n_copy]
                sw[n_copy:] = 0.0
        self.solution = dict(pairs=pairs, override_log=override_log, reference_updates=reference_updates,
                             all_converged=not unsolvable and g_index >= n_images, unsolvable=unsolvable)
        return self.solution
