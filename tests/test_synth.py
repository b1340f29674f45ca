"""The seeded synthetic speckle generator (test / benchmark inputs)."""
import numpy as np


def test_deterministic_and_bounded(gpv_mod):
    from gpv import synth
    a = synth.speckle(96, 80, seed=3)
    b = synth.speckle(96, 80, seed=3)
    c = synth.speckle(96, 80, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() >= 30.0 - 1e-9 and a.max() <= 200.0 + 1e-9
    # coverage: a good part of the image sits on blobs
    assert 0.3 < np.mean(a > 60.0) < 0.95
    q = synth.quantize(a, 3, 11)
    assert q.dtype == np.uint8 and abs(float(q.mean()) - float(a.mean())) < 0.5
    q16 = synth.quantize(a * 16, 3, 11, sigma=32.0, dtype=np.uint16)
    assert q16.dtype == np.uint16 and q16.max() <= 4095


def test_rigid_warp_is_the_shifted_interpolant(gpv_mod, oracle):
    """Target of a rigid shift = the reference's own B-spline at x - u."""
    from gpv import synth
    r0 = synth.speckle(64, 72, seed=9)
    fld = synth.make_field(t=(0.35, -0.2))
    g = synth.warp(r0, fld)
    C = oracle.get_c(r0, 20)
    yy, xx = np.mgrid[10:50, 10:60]
    xy = np.stack([xx.ravel() - 0.35, yy.ravel() + 0.2], 1).astype(float)
    v = oracle.evaluate(C, r0.shape, 20, xy)
    assert np.abs(v - g[10:50, 10:60].ravel()).max() < 1e-9


def test_field_and_gradient(gpv_mod):
    from gpv import synth
    fld = synth.make_field(xc=10.0, yc=20.0, t=(1.0, -2.0), a=(0.01, 0.02, 0.03, 0.04), q=(1e-3, 2e-3, 3e-3, 4e-3, 5e-3, 6e-3))
    xy = np.array([[13.0, 17.0], [0.0, 0.0]])
    h = 1e-6
    g = synth.gradient(fld, xy)
    for k, (ax, comp) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1)]):  # ux, vx, uy, vy
        e = np.zeros(2)
        e[ax] = h
        fd = (synth.displacement(fld, xy + e) - synth.displacement(fld, xy - e))[:, comp] / (2 * h)
        assert np.abs(fd - g[:, k]).max() < 1e-6


def test_workloads_have_their_shapes(gpv_mod):
    from gpv import synth
    W = synth.workload(1, scale_down=8)
    assert W["f"].shape == (128, 128) and W["f"].dtype == np.uint8
    assert np.all(W["radius"] == 25) and np.all(W["order"] == 1)
    W = synth.workload(3, scale_down=16)
    assert set(np.unique(W["order"])) <= {1, 2} and W["radius"].min() >= 15 and W["radius"].max() <= 60
    assert np.abs(W["p0"][:, :2] - W["truth_uv"]).max() <= 0.3 + 1e-12
