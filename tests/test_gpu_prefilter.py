"""GPU parity of the B-spline prefilter and interpolation against the oracle.

Reference: get_c (src/image.rs:252-327), Image::eval / eval_grad
(src/image.rs:115-178).  Tolerances: FP64 coefficients rtol 1e-8 of max|C|
(the reference's own Tier B, src/image.rs:21-23); FP32 coefficients 2e-7
of max|C| (FP32 storage); FP64 interpolation 1e-9 DN; FP32 interpolation
2e-4 DN (values are 0..255).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,border,dtype", [
    ((40, 57), 20, np.uint8),     # short lines: the all-residue (N < 89) path
    ((64, 50), 3, np.float64),    # minimum border
    ((40, 300), 20, np.uint8),    # long rows, short columns: the short-line path with 89-tap rows
    ((130, 100), 20, np.float64),  # fused kernel, FP64 pixels and FP64 coefficients (its largest staging)
    ((200, 300), 20, np.uint8),
    ((257, 129), 20, np.uint16),
    ((1024, 1024), 20, np.uint8),
])
def test_coefficients_match_oracle(oracle, gpv_mod, shape, border, dtype):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    hi = 255 if dtype != np.uint16 else 4095
    img = rng.integers(0, hi + 1, shape).astype(dtype)
    ref = oracle.get_c(img.astype(np.float64), border)
    im = gpv_mod.Image(image_gs=img, border=border, keep_f64=True)
    c64 = im.coef(f64=True)
    c32 = im.coef()
    scale = np.abs(ref).max()
    assert c64.shape == ref.shape
    assert np.abs(c64 - ref).max() <= 1e-8 * scale
    assert np.abs(c32.astype(np.float64) - ref).max() <= 2e-7 * scale


@pytest.mark.parametrize("shape,dtype", [((200, 300), np.uint8), ((257, 129), np.uint16), ((1024, 1024), np.uint8)])
def test_fp32_only_coefficients_match_oracle(oracle, gpv_mod, shape, dtype):
    """Images that keep FP32 coefficients only take the 57-tap filter
    (|m| <= 28): still within the FP32 bound of the oracle, and within a few
    FP32 roundings of the 89-tap coefficients of the same image."""
    rng = np.random.default_rng(shape[0] * 11 + shape[1])
    hi = 255 if dtype != np.uint16 else 4095
    img = rng.integers(0, hi + 1, shape).astype(dtype)
    ref = oracle.get_c(img.astype(np.float64), 20)
    c32 = gpv_mod.Image(image_gs=img, border=20).coef().astype(np.float64)
    c89 = gpv_mod.Image(image_gs=img, border=20, keep_f64=True).coef().astype(np.float64)
    scale = np.abs(ref).max()
    assert np.abs(c32 - ref).max() <= 2e-7 * scale
    assert np.abs(c32 - c89).max() <= 1e-7 * scale


def test_constant_image_gives_constant_coefficients(gpv_mod):
    # test_get_c_constant (src/image.rs:539-550): 20x25, border 5, value 77
    im = gpv_mod.Image(image_gs=np.full((20, 25), 77.0), border=5, keep_f64=True)
    c = im.coef(f64=True)
    assert c.shape == (30, 35)
    assert np.all(np.abs(c - 77.0) < 1e-8 * 77.0)


def test_interpolation_matches_oracle(oracle, gpv_mod):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (96, 120)).astype(np.uint8)
    border = 20
    ref_c = oracle.get_c(img.astype(np.float64), border)
    im = gpv_mod.Image(image_gs=img, border=border, keep_f64=True)
    xy = np.concatenate([
        rng.uniform(0, 119, (500, 2)) * [1, 95 / 119],
        [[0.0, 0.0], [119 - 1e-9, 95 - 1e-9], [-3.0, 40.0], [1e6, -1e6], [119.5, 10.25], [60.0, 95.7]],
    ])
    v_ref, g_ref = oracle.evaluate(ref_c, img.shape, border, xy, grad=True)
    v64, g64 = im.eval(xy, grad=True, precision=gpv_mod.PREC_FP64)
    v32, g32 = im.eval(xy, grad=True, precision=gpv_mod.PREC_MIXED)
    assert np.abs(v64 - v_ref).max() < 1e-9
    assert np.abs(g64 - g_ref).max() < 1e-9
    assert np.abs(v32 - v_ref).max() < 2e-4
    assert np.abs(g32 - g_ref).max() < 5e-4


def test_gradient_is_derivative_at_fractional_position(gpv_mod):
    # eval_grad_is_derivative_at_fractional_position (src/image.rs:634-647)
    r, c = np.mgrid[0:60, 0:60].astype(np.float64)
    a = 120.0 + 60.0 * np.sin(2 * np.pi * r / 7.0 + 0.3) * np.cos(2 * np.pi * c / 9.0)
    im = gpv_mod.Image(image_gs=a, border=8, keep_f64=True)
    h = 1e-5
    for x, y in [(30.0, 30.0), (30.25, 30.75), (30.5, 29.5), (31.9, 28.1)]:
        _, g = im.eval([[x, y]], grad=True, precision=gpv_mod.PREC_FP64)
        vals = im.eval([[x + h, y], [x - h, y], [x, y + h], [x, y - h]], precision=gpv_mod.PREC_FP64)
        fx, fy = (vals[0] - vals[1]) / (2 * h), (vals[2] - vals[3]) / (2 * h)
        assert abs(g[0, 0] - fx) < 1e-4 and abs(g[0, 1] - fy) < 1e-4


def test_far_out_of_range_query_saturates(gpv_mod):
    # test_bspline_eval_clamps_far_out_of_range_query (src/subset.rs:1834-1868)
    r, c = np.mgrid[0:8, 0:9].astype(np.float64)
    img = 100.0 + np.sin(c * 1.3) * 20.0 + np.cos(r * 0.8) * 10.0
    im = gpv_mod.Image(image_gs=img, border=5, keep_f64=True)
    for prec in (gpv_mod.PREC_FP64, gpv_mod.PREC_MIXED):
        far, edge = im.eval([[1_000_000.0, 0.0], [9.0 - 1e-9, 0.0]], precision=prec)
        assert np.isfinite(far) and abs(far) < 200.0
        assert abs(far - edge) < 1e-3
        _, g = im.eval([[1_000_000.0, -1_000_000.0]], grad=True, precision=prec)
        assert np.all(np.isfinite(g)) and np.all(np.abs(g) < 200.0)


@pytest.mark.parametrize("dtype,keep_f64,shape", [
    (np.uint16, False, (1000, 777)), (np.uint8, True, (1000, 777)), (np.float64, False, (1000, 777)),
    # heights whose quarter is a whole number of 32-row tiles but which do not
    # split into four equal parts (the chunk count must stay within the events)
    (np.uint8, False, (1025, 300)), (np.uint16, True, (257, 640)), (np.uint8, False, (2049, 200))])
def test_pinned_chunked_update_equals_pageable_update(gpv_mod, dtype, keep_f64, shape):
    """gpv_image_update from page-locked pixels uploads them in row chunks
    beside the row passes: the coefficients (and the pixel staging the grain
    statistics read) equal those of an update from pageable memory."""
    import ctypes as ct

    import torch
    from gpv import _lib
    rng = np.random.default_rng(17)
    hi = 4095 if dtype == np.uint16 else 255
    img = rng.integers(0, hi + 1, shape).astype(dtype)
    a = gpv_mod.Image(image_gs=np.zeros(shape, dtype), border=20, keep_f64=keep_f64)
    b = gpv_mod.Image(image_gs=np.zeros(shape, dtype), border=20, keep_f64=keep_f64)
    a.update(img)  # pageable
    pinned = torch.from_numpy(img.view(np.uint8).reshape(-1).copy()).pin_memory()
    _lib.check(_lib.lib().gpv_image_update(b.handle, ct.c_void_p(pinned.data_ptr()), _lib.DTYPES[np.dtype(dtype)]),
               "gpv_image_update (pinned)")
    assert np.array_equal(a.coef(), b.coef())
    if keep_f64:
        assert np.array_equal(a.coef(f64=True), b.coef(f64=True))
    a.build_grain()
    b.build_grain()
    ga, gb = a.grain(maps=True), b.grain(maps=True)
    assert ga["correlation_length"] == gb["correlation_length"]
    assert np.array_equal(ga["maps"], gb["maps"])
