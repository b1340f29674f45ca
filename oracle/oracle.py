"""ctypes binding of the CPU FP64 oracle (oracle/gpv_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against.
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product path never does.

Each wrapper names the reference function it restates (paths are within the
geopyv-dev crate).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgpvoracle.so")

# Record layouts shared with the library's C-ABI (gpv_subset_desc / result / params).
DESC_DTYPE = np.dtype([("coord", "<f8", (2,)), ("p0", "<f8", (12,)), ("order", "<i4"), ("radius", "<i4")])
RESULT_DTYPE = np.dtype([
    ("p", "<f8", (12,)), ("c_zncc", "<f8"), ("c_znssd", "<f8"), ("norm", "<f8"),
    ("eta_u", "<f8"), ("eta_v", "<f8"), ("f_m", "<f8"), ("delta_f", "<f8"), ("sssig", "<f8"),
    ("sigma", "<f8"), ("iterations", "<i4"), ("converged", "<i4"), ("quality_ok", "<i4"),
    ("status", "<i4"), ("n_px", "<i4"), ("has_eta", "<i4"), ("texture", "<i4"), ("reserved", "<i4"),
])
PARAMS_DTYPE = np.dtype([("max_norm", "<f8"), ("tolerance", "<f8"), ("max_iterations", "<i4"), ("flags", "<i4"),
                         ("s2", "<f8"), ("grain", "<u8"), ("gh", "<i8"), ("gw", "<i8")])

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ct.CDLL(_LIB_PATH)
        P = ct.c_void_p
        i64, dbl, i32 = ct.c_int64, ct.c_double, ct.c_int
        L.gpvo_fft.argtypes = [P, P, i64, i32, P, P]
        L.gpvo_get_c.argtypes = [P, i64, i64, i64, P, i32]
        L.gpvo_qt_poly.argtypes = [dbl, P]
        L.gpvo_qt_dpoly.argtypes = [dbl, P]
        L.gpvo_eval.argtypes = [P, i64, i64, i64, P, i64, P, P]
        L.gpvo_circle.argtypes = [i64, P]
        L.gpvo_circle.restype = i64
        L.gpvo_mask_update.argtypes = [P, i64, i64, P, P, i64, i64, P]
        L.gpvo_mask_update.restype = i64
        L.gpvo_apply_warp.argtypes = [P, P, i32, P, i64, P]
        L.gpvo_steepest_descent.argtypes = [P, P, P, i64, i32, P]
        L.gpvo_correlation_length.argtypes = [P, i64, i64, P]
        L.gpvo_correlation_length.restype = i32
        L.gpvo_gauss_kernel.argtypes = [i32, dbl, P]
        L.gpvo_gauss_kernel.restype = i32
        L.gpvo_grain_maps.argtypes = [P, i64, i64, dbl, P]
        L.gpvo_grain_template.argtypes = [P, dbl, P, dbl, P, i32, P, i64, P]
        L.gpvo_compose.argtypes = [P, P, i32, P]
        L.gpvo_compose.restype = i32
        L.gpvo_norm.argtypes = [P, i32, dbl]
        L.gpvo_norm.restype = dbl
        L.gpvo_znssd.argtypes = [P, P, i64, dbl, dbl, dbl, dbl]
        L.gpvo_znssd.restype = dbl
        L.gpvo_zn_slice.argtypes = [P, i64, P]
        L.gpvo_eta_component.argtypes = [P, i32, P, P, i64]
        L.gpvo_eta_component.restype = dbl
        L.gpvo_eta.argtypes = [P, i32, P, P, P, dbl, dbl, P, dbl, dbl, i64, P, P]
        L.gpvo_eta.restype = i32
        L.gpvo_solve_batch.argtypes = [P, P, i64, i64, i64, P, i64, P, P, P, P, i32]
        L.gpvo_ingest_rgb8.argtypes = [P, i64, i64, P]
        L.gpvo_subset_setup.argtypes = [P, i64, i64, i64, P, i64, P, P, P, P, P]
        L.gpvo_subset_setup.restype = i32
        L.gpvo_max_threads.restype = i32
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def _f8(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fft(x, inverse=False):
    """Complex DFT (rustfft 6.4.1 restated), unnormalised in both directions."""
    x = np.asarray(x, dtype=complex)
    re, im = _f8(x.real), _f8(x.imag)
    ro, io = np.empty_like(re), np.empty_like(im)
    lib().gpvo_fft(_p(re), _p(im), x.size, 1 if inverse else -1, _p(ro), _p(io))
    return ro + 1j * io


def get_c(image_gs, border=20, nthreads=0):
    """Image::from_array -> get_c (src/image.rs:83-86, :252-327)."""
    img = _f8(image_gs)
    h, w = img.shape
    out = np.empty((h + 2 * border, w + 2 * border))
    lib().gpvo_get_c(_p(img), h, w, border, _p(out), nthreads or lib().gpvo_max_threads())
    return out


def qt_poly(t):
    out = np.empty(6)
    lib().gpvo_qt_poly(float(t), _p(out))
    return out


def qt_dpoly(t):
    out = np.empty(6)
    lib().gpvo_qt_dpoly(float(t), _p(out))
    return out


def evaluate(coef, shape, border, xy, grad=False):
    """Image::eval / Image::eval_grad (src/image.rs:115-178) at points xy (n, 2) = (x=col, y=row)."""
    c = _f8(coef)
    xy = _f8(np.atleast_2d(xy))
    n = xy.shape[0]
    val = np.empty(n)
    g = np.empty((n, 2)) if grad else None
    lib().gpvo_eval(_p(c), shape[0], shape[1], border, _p(xy), n, _p(val), _p(g))
    return (val, g) if grad else val


def circle(radius):
    """LocalMask::circle (src/masks.rs:69-109): (n_px, 2) offsets [x, y]."""
    n = lib().gpvo_circle(radius, None)
    out = np.empty((n, 2))
    lib().gpvo_circle(radius, _p(out))
    return out


def mask_update(coords, size, centre, mask):
    """LocalMask::mask_update (src/masks.rs:199-263) for a circle template."""
    coords = _f8(coords)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    out = np.empty_like(coords)
    c = _f8(centre)
    n = lib().gpvo_mask_update(_p(coords), coords.shape[0], size, _p(c), _p(m), m.shape[0], m.shape[1], _p(out))
    return out[:n].copy()


def apply_warp(coord, p, xy):
    """apply_warp (src/subset.rs:252-300)."""
    xy = _f8(xy)
    p = _f8(p)
    out = np.empty_like(xy)
    lib().gpvo_apply_warp(_p(_f8(coord)), _p(p), p.size, _p(xy), xy.shape[0], _p(out))
    return out


def steepest_descent(coord, xy, grad, order):
    """steepest_descent (src/subset.rs:311-343)."""
    xy, grad = _f8(xy), _f8(grad)
    m = {0: 2, 1: 6, 2: 12}[order]
    out = np.empty((xy.shape[0], m))
    lib().gpvo_steepest_descent(_p(_f8(coord)), _p(xy), _p(grad), xy.shape[0], order, _p(out))
    return out


def compose(p, dp):
    """compose_icgn (src/subset.rs:487-611); None when W_delta is singular."""
    p, dp = _f8(p), _f8(dp)
    out = np.empty_like(p)
    ok = lib().gpvo_compose(_p(p), _p(dp), p.size, _p(out))
    return out if ok else None


def convergence_norm(dp, size):
    dp = _f8(dp)
    return lib().gpvo_norm(_p(dp), dp.size, float(size))


def znssd(f, g, f_m, g_m, df, dg):
    f, g = _f8(f), _f8(g)
    return lib().gpvo_znssd(_p(f), _p(g), f.size, f_m, g_m, df, dg)


def zn_slice(x):
    x = _f8(x)
    out = np.empty_like(x)
    lib().gpvo_zn_slice(_p(x), x.size, _p(out))
    return out


def eta_component(modes, grad_zn, e_centered):
    modes = _f8(modes)
    return lib().gpvo_eta_component(_p(modes), modes.shape[1], _p(_f8(grad_zn)), _p(_f8(e_centered)), modes.shape[0])


def omitted_mode_diagnostic(coord, order, f_coords, grad_f, f, f_m, df, g, g_m, dg):
    eu, ev = ct.c_double(), ct.c_double()
    fc = _f8(f_coords)
    ok = lib().gpvo_eta(_p(_f8(coord)), order, _p(fc), _p(_f8(grad_f)), _p(_f8(f)), f_m, df, _p(_f8(g)), g_m, dg,
                        fc.shape[0], ct.byref(eu), ct.byref(ev))
    return (eu.value, ev.value) if ok else None


def subset_setup(coef, shape, border, coord, radius, mask=None):
    """Subset::new (src/subset.rs:836-919): f, grad_f, (f_m, delta_f, sssig, sigma), status."""
    nmax = circle(radius).shape[0]
    f = np.empty(nmax)
    g = np.empty((nmax, 2))
    sc = np.empty(4)
    n = ct.c_int64()
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    st = lib().gpvo_subset_setup(_p(_f8(coef)), shape[0], shape[1], border, _p(_f8(coord)), radius, _p(m),
                                 _p(f), _p(g), _p(sc), ct.byref(n))
    k = n.value
    return f[:k].copy(), g[:k].copy(), sc, st


def solve_batch(coef_f, coef_g, shape, border, desc, max_norm=1e-5, max_iterations=50, tolerance=0.75,
                eta=False, mask=None, history=False, nthreads=0, method="icgn", grain=None):
    """Batched Subset::new + solve_icgn_result (src/subset.rs:836-919, 1117-1219),
    or solve_fagn_result (:1228-1334) with method="fagn".  grain = (maps, s2)
    from grain() fits the rigid-texture template (ICGN; order 1 and 2)."""
    desc = np.ascontiguousarray(desc, dtype=DESC_DTYPE)
    prm = np.zeros(1, PARAMS_DTYPE)
    flags = int(eta) | (4 if method == "fagn" else 0) | (8 if grain is not None else 0)
    prm["max_norm"], prm["tolerance"], prm["max_iterations"], prm["flags"] = max_norm, tolerance, max_iterations, flags
    if grain is not None and grain[0] is not None:
        maps = np.ascontiguousarray(grain[0], dtype=np.float64)
        prm["s2"], prm["grain"], prm["gh"], prm["gw"] = grain[1], maps.ctypes.data, maps.shape[1], maps.shape[2]
    out = np.zeros(desc.size, RESULT_DTYPE)
    hist = np.zeros((desc.size, max_iterations, 3)) if history else None
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    lib().gpvo_solve_batch(_p(_f8(coef_f)), _p(_f8(coef_g)), shape[0], shape[1], border, _p(desc), desc.size,
                           _p(prm), _p(m), _p(out), _p(hist), nthreads or lib().gpvo_max_threads())
    return (out, hist) if history else out


def correlation_length(image):
    """correlation_length (src/seam.rs:255-301): the speckle correlation length
    of a reference image (px), or None (too small / never falls to 0.5)."""
    a = _f8(image)
    ell = ct.c_double()
    rc = lib().gpvo_correlation_length(_p(a), a.shape[0], a.shape[1], ct.byref(ell))
    return ell.value if rc == 0 else None


def gauss_kernel(order, sigma=1.0):
    """kernel_with (src/texture.rs:49-68)."""
    k = np.empty(2 * int(np.ceil(4.0 * sigma)) + 1)
    lib().gpvo_gauss_kernel(order, float(sigma), _p(k))
    return k


def grain(image):
    """GrainMaps::build (src/texture.rs:99-115): (maps (3, h, w) = fxx, fyy,
    fxy scaled by the smoothing correction, s2), or (None, None) when the
    image has no measurable speckle."""
    a = _f8(image)
    ell = correlation_length(a)
    if ell is None:
        return None, None
    s2 = ell * ell / (2.0 * np.log(2.0))
    if not (np.isfinite(s2) and s2 > 0):
        return None, None
    corr = ((s2 / 2.0 + 1.0) / (s2 / 2.0)) ** 2
    maps = np.empty((3,) + a.shape)
    lib().gpvo_grain_maps(_p(a), a.shape[0], a.shape[1], corr, _p(maps))
    return maps, s2


def grain_maps(image, corr=1.0):
    """The three filtered maps (fxx, fyy, fxy) times corr (src/texture.rs:108-114)."""
    a = _f8(image)
    maps = np.empty((3,) + a.shape)
    lib().gpvo_grain_maps(_p(a), a.shape[0], a.shape[1], float(corr), _p(maps))
    return maps


def grain_template(f, f_m, h, s2, p, xy):
    """grain_template (src/texture.rs:213-244) with base = the subset mean."""
    f, h, p, xy = _f8(f), _f8(h), _f8(p), _f8(xy)
    out = np.empty_like(f)
    lib().gpvo_grain_template(_p(f), float(f_m), _p(h), float(s2), _p(p), p.size, _p(xy), f.size, _p(out))
    return out


def ingest_rgb8(rgb):
    """load_grayscale + gaussian_blur_5x5 (src/image.rs:450-534): (h, w, 3) uint8 -> (h, w) uint8."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    out = np.empty(rgb.shape[:2], np.uint8)
    lib().gpvo_ingest_rgb8(_p(rgb), rgb.shape[0], rgb.shape[1], _p(out))
    return out
