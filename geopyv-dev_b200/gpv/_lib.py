"""ctypes binding of libgpv_b200.so (the C ABI declared in include/gpv.h).

The library is built in-tree by ``geopyv-dev_b200/build.py``.  There is no
fallback: if the shared object is missing or cannot be loaded, importing the
package raises.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# GPV_LIB selects another build of the library (e.g. one compiled with
# different tuning macros); the default is the in-tree build.
LIB_PATH = os.environ.get("GPV_LIB") or os.path.join(HERE, "libgpv_b200.so")

# Record layouts of include/gpv.h
DESC_DTYPE = np.dtype([("coord", "<f8", (2,)), ("p0", "<f8", (12,)), ("order", "<i4"), ("radius", "<i4")])
RESULT_DTYPE = np.dtype([
    ("p", "<f8", (12,)), ("c_zncc", "<f8"), ("c_znssd", "<f8"), ("norm", "<f8"),
    ("eta_u", "<f8"), ("eta_v", "<f8"), ("f_m", "<f8"), ("delta_f", "<f8"), ("sssig", "<f8"),
    ("sigma", "<f8"), ("iterations", "<i4"), ("converged", "<i4"), ("quality_ok", "<i4"),
    ("status", "<i4"), ("n_px", "<i4"), ("has_eta", "<i4"), ("texture", "<i4"), ("reserved", "<i4"),
])
assert DESC_DTYPE.itemsize == 120 and RESULT_DTYPE.itemsize == 200


class SolveParams(ct.Structure):
    _fields_ = [("max_norm", ct.c_double), ("tolerance", ct.c_double), ("max_iterations", ct.c_int32),
                ("flags", ct.c_int32), ("precision", ct.c_int32), ("reserved", ct.c_int32),
                ("mask", ct.c_void_p), ("history", ct.c_void_p)]


# gpv_progress_fn / gpv_batch_solver_fn
PROGRESS_FN = ct.CFUNCTYPE(ct.c_int, ct.c_void_p, ct.c_int64, ct.c_int64)
BATCH_SOLVER_FN = ct.CFUNCTYPE(ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_double, ct.c_void_p)


class MeshParams(ct.Structure):
    _fields_ = [("seed_coord", ct.c_double * 2), ("seed_warp", ct.c_double * 12), ("seed_tolerance", ct.c_double),
                ("max_norm", ct.c_double), ("tolerance", ct.c_double), ("root_rel_eps", ct.c_double),
                ("max_iterations", ct.c_int32), ("subset_order", ct.c_int32), ("radius", ct.c_int32),
                ("precision", ct.c_int32), ("layer_rg", ct.c_int32), ("batch_factor", ct.c_int32),
                ("max_workers", ct.c_int32), ("method", ct.c_int32), ("texture", ct.c_int32),
                ("reserved", ct.c_int32), ("mask", ct.c_void_p),
                ("progress", PROGRESS_FN), ("progress_user", ct.c_void_p)]


class MeshStats(ct.Structure):
    _fields_ = [("n_bad", ct.c_int64), ("n_unreached", ct.c_int64), ("batches", ct.c_int64), ("solves", ct.c_int64),
                ("retries", ct.c_int64), ("rounds", ct.c_int64), ("seed_node", ct.c_int64)]


assert ct.sizeof(MeshParams) == 208 and ct.sizeof(MeshStats) == 56

EXECUTOR_FN = ct.CFUNCTYPE(ct.c_int, ct.c_void_p, ct.c_int32, ct.c_void_p, ct.c_void_p, ct.c_void_p)


class Request(ct.Structure):
    _fields_ = [("f_px", ct.c_void_p), ("g_px", ct.c_void_p), ("dtype", ct.c_int32), ("border", ct.c_int32),
                ("h", ct.c_int64), ("w", ct.c_int64), ("desc", ct.c_void_p), ("n", ct.c_int64),
                ("params", SolveParams), ("session", ct.c_uint64), ("flags", ct.c_uint32), ("reserved", ct.c_uint32),
                ("out", ct.c_void_p)]


class ServerConfig(ct.Structure):
    _fields_ = [("hbm_budget", ct.c_size_t), ("workers", ct.c_int32), ("device", ct.c_int32),
                ("executor", EXECUTOR_FN), ("executor_user", ct.c_void_p), ("reserve_subsets", ct.c_int64),
                ("reserve_radius", ct.c_int32), ("priority_workers", ct.c_int32), ("priority_subsets", ct.c_int64)]


class ServerStats(ct.Structure):
    _fields_ = [("submitted", ct.c_int64), ("completed", ct.c_int64), ("failed", ct.c_int64), ("queued", ct.c_int64),
                ("in_flight", ct.c_int64), ("subsets", ct.c_int64), ("p50_ms", ct.c_double), ("p99_ms", ct.c_double),
                ("mean_ms", ct.c_double), ("max_ms", ct.c_double), ("mean_queue_ms", ct.c_double),
                ("mean_service_ms", ct.c_double), ("subsets_per_s", ct.c_double),
                ("bytes_in_flight", ct.c_size_t), ("peak_bytes", ct.c_size_t), ("hbm_budget", ct.c_size_t)]


class Peaks(ct.Structure):
    _fields_ = [("fp32_scalar_tflops", ct.c_double), ("fp32_paired_tflops", ct.c_double),
                ("fp64_tflops", ct.c_double), ("smem_gbs", ct.c_double), ("sm_count", ct.c_int32),
                ("reserved", ct.c_int32)]


assert ct.sizeof(Peaks) == 40


class Tuning(ct.Structure):
    _fields_ = [("threads", ct.c_int32), ("layout", ct.c_int32), ("run_length", ct.c_int32),
                ("subsets_per_block", ct.c_int32), ("staging", ct.c_int32), ("reserved", ct.c_int32)]


assert ct.sizeof(Tuning) == 24

REQUEST_REUSE_REFERENCE, REQUEST_SEED_FROM_PREVIOUS = 1, 2
CONTEXT_HIGH_PRIORITY, CONTEXT_PER_SUBSET_BLOCKS = 1, 2

# enums
GPV_U8, GPV_U16, GPV_F32, GPV_F64 = 1, 2, 3, 4
PREC_MIXED, PREC_FP64 = 0, 1
SOLVE_ETA, SOLVE_HISTORY, SOLVE_FAGN, SOLVE_RIGID_TEXTURE, SOLVE_KAHAN = 1, 2, 4, 8, 16
IMAGE_KEEP_F64, IMAGE_GRAIN = 1, 2
STATUS = {0: "OK", 1: "EMPTY_MASK", 2: "FEATURELESS", 3: "SINGULAR_H", 4: "SINGULAR_WDELTA", 5: "NONFINITE",
          6: "TIMEOUT", 7: "CANCELLED", 8: "INVALID_SUBSET"}
DTYPES = {np.dtype(np.uint8): GPV_U8, np.dtype(np.uint16): GPV_U16, np.dtype(np.float32): GPV_F32,
          np.dtype(np.float64): GPV_F64}

# Every entry point of include/gpv.h: name -> (restype, argtypes)
P, I32, I64, U32, SZ, DBL = ct.c_void_p, ct.c_int32, ct.c_int64, ct.c_uint32, ct.c_size_t, ct.c_double
SIGNATURES = {
    "gpv_version": (ct.c_char_p, []),
    "gpv_abi_version": (ct.c_int, []),
    "gpv_last_error": (SZ, [ct.c_char_p, SZ]),
    "gpv_context_create": (ct.c_int, [ct.c_int, P]),
    "gpv_context_create_ex": (ct.c_int, [ct.c_int, ct.c_uint32, P]),
    "gpv_context_destroy": (ct.c_int, [P]),
    "gpv_context_stream": (P, [P]),
    "gpv_context_reserve": (ct.c_int, [P, I64, I32, I32]),
    "gpv_image_create": (ct.c_int, [P, P, I32, I64, I64, I32, U32, P]),
    "gpv_image_create_device": (ct.c_int, [P, P, I32, I64, I64, I32, U32, P]),
    "gpv_image_update_device": (ct.c_int, [P, P, I32]),
    "gpv_image_update": (ct.c_int, [P, P, I32]),
    "gpv_image_build_grain": (ct.c_int, [P]),
    "gpv_image_grain": (ct.c_int, [P, P, P, P]),
    "gpv_image_grain_sample": (ct.c_int, [P, P, I64, P]),
    "gpv_image_destroy": (ct.c_int, [P]),
    "gpv_image_shape": (ct.c_int, [P, P, P, P]),
    "gpv_image_coefficients_f32": (ct.c_int, [P, P]),
    "gpv_image_coefficients_f64": (ct.c_int, [P, P]),
    "gpv_image_eval": (ct.c_int, [P, P, I64, I32, P, P]),
    "gpv_image_create_rgb8": (ct.c_int, [P, P, I64, I64, I32, U32, P]),
    "gpv_image_update_rgb8": (ct.c_int, [P, P]),
    "gpv_image_update_rgb8_device": (ct.c_int, [P, P]),
    "gpv_image_grey": (ct.c_int, [P, P]),
    "gpv_mask_create": (ct.c_int, [P, P, I64, I64, P]),
    "gpv_mask_destroy": (ct.c_int, [P]),
    "gpv_solve_batch": (ct.c_int, [P, P, P, P, I64, P, P]),
    "gpv_solve_batch_device": (ct.c_int, [P, P, P, P, P, I64, P, P, P]),
    "gpv_probe_fp32_peak": (ct.c_int, [P, P]),
    "gpv_probe_peaks": (ct.c_int, [P, P]),
    "gpv_autotune": (ct.c_int, [P, P, P, P, I64, P, I32, P]),
    "gpv_context_tuning": (ct.c_int, [P, P, P]),
    "gpv_context_tuning_get": (ct.c_int, [P, P]),
    "gpv_batch_graph_create": (ct.c_int, [P, P, P, P, P, I64, P, P, P]),
    "gpv_batch_graph_launch": (ct.c_int, [P, P]),
    "gpv_batch_graph_destroy": (ct.c_int, [P]),
    "gpv_solve_batch_noalloc": (ct.c_int, [P, P, P, P, I64, I32, P, P, P]),
    "gpv_mesh_solve": (ct.c_int, [P, P, P, P, I64, P, I64, I32, P, P, P, P]),
    "gpv_sequence_create": (ct.c_int, [P, P, P, P, I64, P, I32, U32, P]),
    "gpv_server_create": (ct.c_int, [P, P]),
    "gpv_server_submit": (ct.c_int, [P, P, P]),
    "gpv_server_prepare": (ct.c_int, [P, I64, I64, I32, I32, I32]),
    "gpv_server_wait": (ct.c_int, [P, ct.c_uint64, I32, P, P]),
    "gpv_server_get_stats": (ct.c_int, [P, P]),
    "gpv_server_reset_stats": (ct.c_int, [P]),
    "gpv_server_destroy": (ct.c_int, [P]),
    "gpv_sequence_frame": (ct.c_int, [P, P, I32, P]),
    "gpv_sequence_results_device": (P, [P]),
    "gpv_sequence_frames": (I64, [P]),
    "gpv_sequence_destroy": (ct.c_int, [P]),
    "gpv_mesh_drive": (ct.c_int, [P, I64, P, I64, I32, P, BATCH_SOLVER_FN, P, P, P, P]),
}

_lib = None


def lib():
    """The loaded library (raises OSError when it is missing: no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with `python geopyv-dev_b200/build.py`")
        L = ct.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class GpvError(RuntimeError):
    """A failed library call (the message is gpv_last_error())."""


def last_error() -> str:
    buf = ct.create_string_buffer(1024)
    lib().gpv_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        raise GpvError(f"{what} failed ({rc}): {last_error()}")


def ptr(a) -> ct.c_void_p | None:
    if a is None:
        return None
    if isinstance(a, int):
        return ct.c_void_p(a)
    return ct.c_void_p(a.ctypes.data)
