"""The rigid-texture template in the oracle (src/texture.rs), on the CPU.

Restates the reference's texture tests against the oracle: the template's
identities (no correction for order 0, a zero warp or a rigid rotation;
order 2 with zero second-order terms equals order 1), the curvature maps of a
quadratic image, no speckle model for a flat or tiny image, and on rigid
speckles under shear the rigid template fitting better than the deformable
one (order 1) and equal to it at zero strain.  The correlation length from
direct lag sums is checked against numpy's FFT autocorrelation.
"""
import math

import numpy as np
import pytest

import texture_cases as TC


def _pixels(n=40, seed=3):
    rng = np.random.default_rng(seed)
    f = rng.uniform(50, 150, n)
    h = rng.normal(0, 5, (n, 3))
    xy = rng.integers(-10, 11, (n, 2)).astype(np.float64)
    return f, h, xy


def test_order0_and_zero_warp_return_f(oracle):
    """src/texture.rs:361-369."""
    f, h, xy = _pixels()
    for p in ([0.3, -0.2], [0.3, -0.2, 0, 0, 0, 0], [0.0] * 12):
        assert np.array_equal(oracle.grain_template(f, 21.0, h, 9.0, p, xy), f)


def test_rotation_gives_no_correction(oracle):
    """A rigid rotation has zero Green-Lagrange strain (src/texture.rs:343-357)."""
    f, h, xy = _pixels()
    for th in (0.01, 0.1, 0.5):
        p = [0.0, 0.0, math.cos(th) - 1.0, math.sin(th), -math.sin(th), math.cos(th) - 1.0]
        assert np.abs(oracle.grain_template(f, f.mean(), h, 9.0, p, xy) - f).max() < 1e-10


def test_order2_reduces_to_order1(oracle):
    """src/texture.rs:372-382."""
    f, h, xy = _pixels()
    p1 = [0.1, 0.2, 0.01, -0.02, 0.015, 0.03]
    p2 = p1 + [0.0] * 6
    a = oracle.grain_template(f, 21.0, h, 9.0, p1, xy)
    b = oracle.grain_template(f, 21.0, h, 9.0, p2, xy)
    assert np.abs(a - b).max() < 1e-12


def test_curvature_of_quadratic(oracle):
    """src/texture.rs:386-409: the filters give a quadratic's second
    derivatives, and the x derivative of x is 1."""
    a, b, c = 0.02, -0.03, 0.05
    y, x = np.mgrid[0:40, 0:40].astype(np.float64) - 20.0
    m = oracle.grain_maps(a * x * x + b * x * y + c * y * y, corr=1.0)
    for got, want in ((m[0, 20, 20], 2 * a), (m[1, 20, 20], 2 * c), (m[2, 20, 20], b)):
        assert abs(got - want) < 0.01 * abs(want)
    k0, k1 = oracle.gauss_kernel(0), oracle.gauss_kernel(1)
    assert k0.size == 9 and abs(k0.sum() - 1.0) < 1e-15
    ramp = np.tile(np.arange(40.0), (40, 1))
    assert abs(np.dot(k1, ramp[20, 16:25]) - 1.0) < 0.01


def test_flat_or_tiny_image_has_no_model(oracle):
    """src/texture.rs:413-419."""
    assert oracle.grain(np.full((64, 64), 128.0)) == (None, None)
    assert oracle.grain(np.full((10, 10), 128.0)) == (None, None)
    y, x = np.mgrid[0:14, 0:14].astype(np.float64)
    assert oracle.correlation_length(100.0 + 40.0 * np.sin(0.9 * x) * np.cos(0.7 * y)) is None  # 14 px < 16


def test_correlation_length_matches_the_fft(oracle):
    """The direct lag sums equal the |FFT|^2 autocorrelation of the reference."""
    f, _ = TC.shear_pair(0.0)
    side = min(512, *f.shape) & ~1
    half = side // 2
    cy, cx = f.shape[0] // 2, f.shape[1] // 2
    crop = f[cy - half:cy + half, cx - half:cx + half] - f[cy - half:cy + half, cx - half:cx + half].mean()
    F = np.fft.fft2(crop)
    ac = np.fft.ifft2(F * np.conj(F)).real
    prof = 0.5 * (ac[0, :half] + ac[:half, 0]) / ac[0, 0]
    k = int(np.argmax(prof < 0.5))
    want = k - 1 + (prof[k - 1] - 0.5) / (prof[k - 1] - prof[k])
    got = oracle.correlation_length(f)
    assert abs(got - want) < 1e-10 * want
    # blobs exp(-r^2 / S^2): half-height autocorrelation at about S sqrt(2 ln 2)
    assert 3.5 < got < 6.5


def _grid(oracle, gamma, order):
    import gpv
    f, g = TC.shear_pair(gamma)
    cf, cg = oracle.get_c(f, 8), oracle.get_c(g, 8)
    d = TC.grid_desc(gpv, gamma, order)
    maps, s2 = oracle.grain(f)
    kw = dict(max_norm=1e-6, max_iterations=100, tolerance=0.75)
    rd = oracle.solve_batch(cf, cg, f.shape, 8, d, **kw)
    rr = oracle.solve_batch(cf, cg, f.shape, 8, d, grain=(maps, s2), **kw)
    return rd, rr


@pytest.mark.parametrize("gamma", [0.02, 0.05, 0.1])
def test_rigid_icgn_helps_on_rigid_speckle_shear(oracle, gamma):
    """src/texture.rs:481-500, order 1."""
    rd, rr = _grid(oracle, gamma, 1)
    assert np.all(rr["texture"] == 1) and np.all(rd["texture"] == 0)
    assert np.all(rr["converged"] == 1)
    assert rr["c_znssd"].mean() < rd["c_znssd"].mean()
    assert np.abs(rr["p"][:, 4] - gamma).mean() < np.abs(rd["p"][:, 4] - gamma).mean()


@pytest.mark.parametrize("order", [1, 2])
def test_rigid_icgn_matches_deformable_at_zero_strain(oracle, order):
    """src/texture.rs:503-510."""
    rd, rr = _grid(oracle, 0.0, order)
    assert np.all(rd["converged"] == 1) and np.all(rr["converged"] == 1)
    assert abs(np.abs(rd["p"][:, 4]).mean() - np.abs(rr["p"][:, 4]).mean()) < 1e-6
    assert abs(rd["c_znssd"].mean() - rr["c_znssd"].mean()) < 1e-9


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("gamma", [0.0, 0.05, 0.1])
def test_rigid_fagn_helps_on_rigid_speckle_shear(oracle, order, gamma):
    """src/texture.rs:513-530: FAGN with the rigid template converges
    everywhere, matches the deformable fit at zero strain and fits better
    under shear at order 1."""
    import gpv
    f, g = TC.shear_pair(gamma)
    cf, cg = oracle.get_c(f, 8), oracle.get_c(g, 8)
    d = TC.grid_desc(gpv, gamma, order)
    maps, s2 = oracle.grain(f)
    kw = dict(max_norm=1e-6, max_iterations=100, tolerance=0.75, method="fagn")
    rd = oracle.solve_batch(cf, cg, f.shape, 8, d, **kw)
    rr = oracle.solve_batch(cf, cg, f.shape, 8, d, grain=(maps, s2), **kw)
    assert np.all(rr["converged"] == 1) and np.all(rr["texture"] == 1)
    ed, er = np.abs(rd["p"][:, 4] - gamma).mean(), np.abs(rr["p"][:, 4] - gamma).mean()
    if gamma == 0.0:
        assert abs(ed - er) < 1e-6 and abs(rd["c_znssd"].mean() - rr["c_znssd"].mean()) < 1e-9
    elif order == 1:
        assert rr["c_znssd"].mean() < rd["c_znssd"].mean() and er < ed
