"""Request loop (gpv_server_*): submit image pairs with subsets from any
thread, collect results, read p50/p99 latency and throughput.

Requests are admitted by device-memory footprint and served by worker
threads that each own a library context on the GPU; sessions keep the
reference coefficients and last results resident (see include/gpv.h).
"""
from __future__ import annotations

import ctypes as ct
import threading

import numpy as np

from . import _lib
from ._lib import DESC_DTYPE, PREC_MIXED, RESULT_DTYPE, GpvError, SolveParams, check, lib, ptr


class Ticket:
    """A submitted request: its id and the buffers the server writes into."""

    def __init__(self, rid, out, keep):
        self.id = rid
        self.out = out
        self._keep = keep
        self.latency_ms = None


class Server:
    def __init__(self, workers: int = 4, hbm_budget: int = 0, device: int = 0, executor=None,
                 reserve_subsets: int = 0, reserve_radius: int = 0, priority_workers: int = 0,
                 priority_subsets: int = 0):
        """executor(worker, request_dict, desc, out) -> int replaces the GPU solve
        (a stand-in for exercising the request loop without a GPU).
        reserve_subsets / reserve_radius size every worker's workspace up front.
        priority_workers > 0 opens a priority lane: workers 0..priority_workers-1
        (high-priority streams) serve the requests of at most priority_subsets
        subsets, the others the larger ones, all with one block per subset."""
        cfg = _lib.ServerConfig()
        cfg.hbm_budget, cfg.workers, cfg.device = hbm_budget, workers, device
        cfg.reserve_subsets, cfg.reserve_radius = reserve_subsets, reserve_radius
        cfg.priority_workers, cfg.priority_subsets = priority_workers, priority_subsets
        self._cb = None
        if executor is not None:
            def _exec(user, worker, req_p, desc_p, out_p):
                try:
                    req = _lib.Request.from_address(req_p)
                    n = int(req.n)
                    d = np.frombuffer((ct.c_char * (n * DESC_DTYPE.itemsize)).from_address(desc_p), dtype=DESC_DTYPE)
                    o = np.frombuffer((ct.c_char * (n * RESULT_DTYPE.itemsize)).from_address(out_p), dtype=RESULT_DTYPE)
                    info = dict(h=int(req.h), w=int(req.w), n=n, session=int(req.session), flags=int(req.flags),
                                f_px=req.f_px, g_px=req.g_px, dtype=int(req.dtype))
                    return int(executor(int(worker), info, d, o) or 0)
                except Exception:
                    return -1
            self._cb = _lib.EXECUTOR_FN(_exec)
            cfg.executor = self._cb
        h = ct.c_void_p()
        check(lib().gpv_server_create(ct.byref(cfg), ct.byref(h)), "gpv_server_create")
        self._h = h
        self._lock = threading.Lock()

    def prepare(self, shape, dtype, border: int = 20, timeout_ms: int = 120000) -> None:
        """Create every worker's cached image pair for requests of this shape and
        pixel type (gpv_server_prepare), so serving them allocates nothing."""
        check(lib().gpv_server_prepare(self._h, int(shape[0]), int(shape[1]), border,
                                       _lib.DTYPES[np.dtype(dtype)], timeout_ms), "gpv_server_prepare")

    def submit(self, f_px, g_px, desc, border: int = 20, max_norm=1e-5, max_iterations=50, tolerance=0.75,
               session: int = 0, reuse_reference: bool = False, seed_from_previous: bool = False,
               texture: str = "deformable") -> Ticket:
        g = np.ascontiguousarray(g_px)
        if g.dtype not in _lib.DTYPES:
            raise TypeError(f"unsupported pixel dtype {g.dtype}")
        f = None if f_px is None else np.ascontiguousarray(f_px, dtype=g.dtype)
        if f is not None and f.shape != g.shape:
            raise ValueError("reference and target shapes differ")
        d = np.ascontiguousarray(desc, dtype=DESC_DTYPE)
        out = np.zeros(d.size, RESULT_DTYPE)
        r = _lib.Request()
        r.f_px = None if f is None else f.ctypes.data
        r.g_px = g.ctypes.data
        r.dtype = _lib.DTYPES[g.dtype]
        r.border = border
        r.h, r.w = g.shape
        r.desc = d.ctypes.data
        r.n = d.size
        if texture not in ("deformable", "rigid"):
            raise ValueError(f"texture must be 'deformable' or 'rigid', got {texture!r}")
        r.params = SolveParams(max_norm=max_norm, tolerance=tolerance, max_iterations=max_iterations,
                               flags=_lib.SOLVE_RIGID_TEXTURE if texture == "rigid" else 0,
                               precision=PREC_MIXED, reserved=0, mask=None, history=None)
        r.session = session
        r.flags = (_lib.REQUEST_REUSE_REFERENCE if reuse_reference else 0) | \
            (_lib.REQUEST_SEED_FROM_PREVIOUS if seed_from_previous else 0)
        r.out = out.ctypes.data
        rid = ct.c_uint64()
        check(lib().gpv_server_submit(self._h, ct.byref(r), ct.byref(rid)), "gpv_server_submit")
        return Ticket(rid.value, out, (f, g, d))

    def wait(self, ticket: Ticket, timeout_ms: int = 60000) -> np.ndarray:
        st = ct.c_int32()
        lat = ct.c_double()
        check(lib().gpv_server_wait(self._h, ticket.id, timeout_ms, ct.byref(st), ct.byref(lat)), "gpv_server_wait")
        ticket.latency_ms = lat.value
        if st.value != 0:
            raise GpvError(f"request {ticket.id} failed ({st.value}): {_lib.last_error()}")
        return ticket.out

    def wait_raw(self, rid: int, timeout_ms: int = 0):
        """(rc, request status, latency) without raising -- for probing ids."""
        st = ct.c_int32()
        lat = ct.c_double()
        rc = lib().gpv_server_wait(self._h, rid, timeout_ms, ct.byref(st), ct.byref(lat))
        return rc, st.value, lat.value

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(lib().gpv_server_get_stats(self._h, ct.byref(s)), "gpv_server_get_stats")
        return {k: getattr(s, k) for k, _ in _lib.ServerStats._fields_}

    def reset_stats(self) -> None:
        check(lib().gpv_server_reset_stats(self._h), "gpv_server_reset_stats")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().gpv_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
