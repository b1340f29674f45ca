"""Seeded synthetic speckle pairs and subset layouts for the five benchmark
workloads (the generator model is stated in csrc/synth.c).

    C1  1024^2 u8, rigid (0.35, -0.20) px, r=25 on a 20 px grid, order 1
    C2  4096^2 u16 (12-bit, x16), 1% uniaxial strain + 0.5 deg rotation +
        1e-6 px^-1 quadratic, r=30 on a 10 px grid, order 2, p0 = field
        translation +- 0.3 px and field gradient (a neighbour preconditioner's
        seed; the displacement reaches ~30 px at the corners)
    C3  2048^2 u8, u = 2 tanh((y-1024)/40) + 0.2% background strain, 50k
        centres (coarse grid refined x4 within 150 px of the band), radii
        log-uniform in [15, 60], orders 1/2 70/30, p0 = field translation
        +- 0.3 px and field gradient
    C4  2048^2 u8 frames, simple shear rising linearly to 5% by frame 200,
        20k subsets r=25, seeded from the previous frame
    C5  Poisson request stream (see gpv.serve)
No public dataset is involved; every array is a function of its seed.
"""
from __future__ import annotations

import ctypes as ct
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "libgpvsynth.so")
_lib = None


class Field(ct.Structure):
    """gpv_field of synth.c: u = t0 + a00 dx + a01 dy + q0 dx^2 + q1 dx dy + q2 dy^2
    (+ band_amp tanh((y - band_y)/band_w)); v likewise with a10, a11, q3..q5."""
    _fields_ = [("xc", ct.c_double), ("yc", ct.c_double), ("t", ct.c_double * 2), ("a", ct.c_double * 4),
                ("q", ct.c_double * 6), ("band_amp", ct.c_double), ("band_y", ct.c_double), ("band_w", ct.c_double)]


def _L():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise OSError(f"{_LIB} is missing; build it with `python geopyv-dev_b200/build.py`")
        L = ct.CDLL(_LIB)
        P = ct.c_void_p
        L.gpv_synth_speckle.argtypes = [ct.c_int64, ct.c_int64, ct.c_uint64, ct.c_double, ct.c_double, P]
        L.gpv_synth_speckle.restype = ct.c_int64
        L.gpv_synth_quantize.argtypes = [P, ct.c_int64, ct.c_double, ct.c_uint64, ct.c_uint64, ct.c_double, ct.c_int, P]
        L.gpv_synth_warp.argtypes = [P, ct.c_int64, ct.c_int64, P, P]
        L.gpv_synth_field.argtypes = [P, P, ct.c_int64, P]
        _lib = L
    return _lib


def make_field(xc=0.0, yc=0.0, t=(0.0, 0.0), a=(0.0, 0.0, 0.0, 0.0), q=(0.0,) * 6, band=(0.0, 0.0, 0.0)) -> Field:
    f = Field()
    f.xc, f.yc = xc, yc
    f.t[:] = t
    f.a[:] = a
    f.q[:] = q
    f.band_amp, f.band_y, f.band_w = band
    return f


def speckle(h, w, seed, scale=1.0, coverage=0.6) -> np.ndarray:
    """Noise-free speckle intensity (FP64)."""
    out = np.empty((h, w))
    _L().gpv_synth_speckle(h, w, seed, coverage, scale, out.ctypes.data)
    return out


def quantize(img, seed, stream, sigma=2.0, dtype=np.uint8, maxval=None) -> np.ndarray:
    img = np.ascontiguousarray(img, dtype=np.float64)
    dt = np.dtype(dtype)
    if maxval is None:
        maxval = 255.0 if dt == np.uint8 else 4095.0
    out = np.empty(img.shape, dt)
    _L().gpv_synth_quantize(img.ctypes.data, img.size, sigma, seed, stream, maxval, 1 if dt == np.uint8 else 2,
                            out.ctypes.data)
    return out


def warp(ref, field: Field) -> np.ndarray:
    """Target intensity S_ref(X), x = X + u(X) (noise-free, FP64)."""
    ref = np.ascontiguousarray(ref, dtype=np.float64)
    out = np.empty_like(ref)
    _L().gpv_synth_warp(ref.ctypes.data, ref.shape[0], ref.shape[1], ct.byref(field), out.ctypes.data)
    return out


def displacement(field: Field, xy) -> np.ndarray:
    xy = np.ascontiguousarray(np.atleast_2d(xy), dtype=np.float64)
    out = np.empty_like(xy)
    _L().gpv_synth_field(ct.byref(field), xy.ctypes.data, xy.shape[0], out.ctypes.data)
    return out


def gradient(field: Field, xy) -> np.ndarray:
    """Analytic displacement gradient [du/dx, dv/dx, du/dy, dv/dy] at points (warp slots 2..5)."""
    xy = np.atleast_2d(np.asarray(xy, dtype=np.float64))
    dx, dy = xy[:, 0] - field.xc, xy[:, 1] - field.yc
    a, q = list(field.a), list(field.q)
    ux = a[0] + 2 * q[0] * dx + q[1] * dy
    uy = a[1] + q[1] * dx + 2 * q[2] * dy
    vx = a[2] + 2 * q[3] * dx + q[4] * dy
    vy = a[3] + q[4] * dx + 2 * q[5] * dy
    if field.band_w != 0.0:
        uy = uy + field.band_amp / field.band_w / np.cosh((xy[:, 1] - field.band_y) / field.band_w) ** 2
    return np.stack([ux, vx, uy, vy], 1)


def seeded_p0(field: Field, xy, rng, jitter=0.3) -> np.ndarray:
    """Initial warps as a neighbour-based preconditioner would give them: the
    field's translation perturbed by +-jitter px, and its gradient."""
    p0 = np.zeros((len(xy), 12))
    p0[:, :2] = displacement(field, xy) + rng.uniform(-jitter, jitter, (len(xy), 2))
    p0[:, 2:6] = gradient(field, xy)
    return p0


def pair(h, w, field: Field, seed, dtype=np.uint8, scale=1.0, sigma=2.0):
    """(reference, target) quantised images of one seeded speckle pair."""
    r0 = speckle(h, w, seed, scale)
    f = quantize(r0, seed, 11, sigma * scale, dtype)
    g = quantize(warp(r0, field), seed, 12, sigma * scale, dtype)
    return f, g


def grid(h, w, step, margin):
    ys = np.arange(margin, h - margin + 1e-9, step)
    xs = np.arange(margin, w - margin + 1e-9, step)
    X, Y = np.meshgrid(xs, ys)
    return np.stack([X.ravel(), Y.ravel()], 1).astype(np.float64)


# ----------------------------------------------------------------------------
# Workloads
# ----------------------------------------------------------------------------
def workload(config: int, scale_down: int = 1, seed_frame: int = 0):
    """Images, subset descriptors and truth for one workload.

    Returns dict(f, g, coords, radius, order, p0, truth_uv, field, name).  With
    scale_down > 1 the image side is divided by it (small cases for tests);
    radii and field shapes are kept.
    """
    seed = 1000 * config + seed_frame
    if config == 1:
        n = 1024 // scale_down
        fld = make_field(t=(0.35, -0.20))
        f, g = pair(n, n, fld, seed)
        r = 25
        xy = grid(n, n, 20, r + 3)
        order = np.ones(len(xy), np.int32)
        radius = np.full(len(xy), r, np.int32)
        p0 = np.zeros((len(xy), 12))
        name = f"C1 rigid {n}x{n} u8 r=25 grid20 order1"
    elif config == 2:
        n = 4096 // scale_down
        c = (n - 1) / 2.0
        th = math.radians(0.5)
        a = (0.01 + math.cos(th) - 1.0, -math.sin(th), math.sin(th), math.cos(th) - 1.0)
        fld = make_field(xc=c, yc=c, a=a, q=(1e-6, 0.0, 0.0, 0.0, 0.0, 1e-6))
        f, g = pair(n, n, fld, seed, dtype=np.uint16, scale=16.0)
        r = 30
        xy = grid(n, n, 10, r + 3 + 0.012 * n)
        order = np.full(len(xy), 2, np.int32)
        radius = np.full(len(xy), r, np.int32)
        p0 = seeded_p0(fld, xy, np.random.default_rng(seed))
        name = f"C2 affine+quadratic {n}x{n} u16 r=30 grid10 order2"
    elif config == 3:
        n = 2048 // scale_down
        c = (n - 1) / 2.0
        fld = make_field(xc=c, yc=c, a=(0.002, 0.0, 0.0, 0.002), band=(2.0, n / 2.0, 40.0))
        f, g = pair(n, n, fld, seed)
        rng = np.random.default_rng(seed)
        coarse = grid(n, n, 16, 64)
        near = np.abs(coarse[:, 1] - n / 2.0) <= 150
        fine = grid(n, n, 4, 64)
        fine = fine[np.abs(fine[:, 1] - n / 2.0) <= 150]
        xy = np.concatenate([coarse[~near], fine])
        target = 50000 // (scale_down * scale_down)
        if len(xy) > target:
            xy = xy[np.sort(rng.choice(len(xy), target, replace=False))]
        radius = np.exp(rng.uniform(math.log(15), math.log(60), len(xy))).round().astype(np.int32)
        order = np.where(rng.uniform(size=len(xy)) < 0.7, 1, 2).astype(np.int32)
        p0 = seeded_p0(fld, xy, rng)
        name = f"C3 shear band {n}x{n} u8 r=15..60 mixed order"
    elif config == 4:
        n = 2048 // scale_down
        c = (n - 1) / 2.0
        gam = 0.05 * seed_frame / 200.0
        fld = make_field(xc=c, yc=c, a=(0.0, gam, 0.0, 0.0))
        f, g = pair(n, n, fld, 1000 * config)
        r = 25
        xy = grid(n, n, 13, r + 3 + 0.05 * n / 2)
        target = 20000 // (scale_down * scale_down)
        if len(xy) > target:
            xy = xy[:target]
        order = np.ones(len(xy), np.int32)
        radius = np.full(len(xy), r, np.int32)
        p0 = np.zeros((len(xy), 12))
        name = f"C4 frame {seed_frame} simple shear {n}x{n} u8 r=25"
    else:
        raise ValueError("config must be 1..4 (config 5 is the serving stream)")
    truth = displacement(fld, xy)
    return dict(f=f, g=g, coords=xy, radius=radius, order=order, p0=p0, truth_uv=truth, field=fld, name=name)


def sequence_frames(frames, scale_down: int = 1, every: int = 1):
    """The incremental-sequence workload's frames 0, every, 2 every, ... below
    `frames` (simple shear rising linearly to 5% at frame 200): the reference
    speckle is rendered once and each target warps it, so the frames equal
    workload(4, scale_down, seed_frame=k)["g"].  Returns (frame-0 workload,
    list of target images)."""
    W0 = workload(4, scale_down, seed_frame=0)
    n = W0["f"].shape[0]
    c = (n - 1) / 2.0
    seed = 1000 * 4
    r0 = speckle(n, n, seed, 1.0)
    gs = []
    for k in range(0, frames, every):
        fld = make_field(xc=c, yc=c, a=(0.0, 0.05 * k / 200.0, 0.0, 0.0))
        gs.append(quantize(warp(r0, fld), seed, 12, 2.0, np.uint8))
    return W0, gs

