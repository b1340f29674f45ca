"""The rigid-texture template on the GPU against the oracle.

* Grain statistics: the device maps equal the oracle's (FP64 sums with the
  same rounding, stored as FP32) bit for bit; the correlation length, s2 and
  the smoothing correction agree to 1e-12 relative; updates rebuild them.
* Rigid solves (mixed precision) on the reference's rigid-blob shear pair
  (src/texture.rs:424-437): displacement within 1e-3 px and gradient terms
  within 1e-5 of the FP64 oracle's rigid solve, identical flags, texture = 1;
  better than the deformable template at order 1 (src/texture.rs:481-500);
  FAGN and the FP64 ICGN form with the rigid template against the oracle's
  (FP64 maps: the FP64 bars); the deformable template for order 0 and for an
  image without measurable speckle; maps refused for device-created images.
"""
import numpy as np
import pytest

import texture_cases as TC

pytestmark = pytest.mark.gpu


def test_grain_maps_equal_the_oracle(gpv_mod, oracle):
    from gpv import synth
    f, _ = TC.shear_pair(0.05)
    W = synth.workload(1, scale_down=4)
    for arr in (f, W["f"]):  # FP64 pixels and u8 pixels
        img = gpv_mod.Image(image_gs=arr, border=8, grain=True)
        got = img.grain(maps=True)
        ell = oracle.correlation_length(arr.astype(np.float64))
        maps, s2 = oracle.grain(arr.astype(np.float64))
        assert got["built"]
        assert abs(got["correlation_length"] - ell) < 1e-12 * ell
        assert abs(got["s2"] - s2) < 1e-12 * s2
        assert np.array_equal(got["maps"], maps.astype(np.float32))
    # an update rebuilds them; a flat image has none
    img = gpv_mod.Image(image_gs=f, border=8, grain=True)
    img.update(W["f"][:200, :200].astype(np.float64))
    assert abs(img.grain()["correlation_length"] - oracle.correlation_length(W["f"][:200, :200].astype(np.float64))) < 1e-9
    flat = gpv_mod.Image(image_gs=np.full((64, 64), 128.0), border=8, grain=True)
    assert not flat.grain()["built"]


def _solve_both(gpv_mod, oracle, gamma, order):
    f, g = TC.shear_pair(gamma)
    F = gpv_mod.Image(image_gs=f, border=8)
    G = gpv_mod.Image(image_gs=g, border=8)
    d = TC.grid_desc(gpv_mod, gamma, order)
    # max_norm 1e-5, the mixed form's bar in every parity test: at zero strain
    # its FP32 interpolation keeps second-order norms of these radius-15
    # subsets above 1e-6, with either template
    kw = dict(max_norm=1e-5, max_iterations=100, tolerance=0.75)
    gd = gpv_mod.solve_batch(F, G, d, **kw)
    gr = gpv_mod.solve_batch(F, G, d, texture="rigid", eta=True, **kw)
    maps, s2 = oracle.grain(f)
    cf, cg = oracle.get_c(f, 8), oracle.get_c(g, 8)
    od = oracle.solve_batch(cf, cg, f.shape, 8, d, **kw)
    orr = oracle.solve_batch(cf, cg, f.shape, 8, d, grain=(maps, s2), eta=True, **kw)
    return gd, gr, od, orr


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("gamma", [0.0, 0.05])
def test_rigid_solve_matches_the_oracle(gpv_mod, oracle, order, gamma):
    gd, gr, od, orr = _solve_both(gpv_mod, oracle, gamma, order)
    assert np.all(gr["texture"] == 1) and np.all(orr["texture"] == 1) and np.all(gd["texture"] == 0)
    for a, b in ((gr, orr), (gd, od)):
        ok = b["status"] == 0
        assert np.array_equal(a["status"], b["status"]) and np.array_equal(a["converged"], b["converged"])
        assert np.abs(a["p"][ok, :2] - b["p"][ok, :2]).max() <= 1e-3
        assert np.abs(a["p"][ok, 2:6] - b["p"][ok, 2:6]).max() <= 1e-5
        assert np.abs(a["c_zncc"][ok] - b["c_zncc"][ok]).max() < 1e-5
    assert np.abs(gr["eta_u"] - orr["eta_u"]).max() < 2e-3 and np.all(gr["has_eta"] == 1)
    if gamma > 0 and order == 1:  # src/texture.rs:481-500
        assert gr["c_znssd"].mean() < gd["c_znssd"].mean()
        assert np.abs(gr["p"][:, 4] - gamma).mean() < np.abs(gd["p"][:, 4] - gamma).mean()


@pytest.mark.parametrize("order", [1, 2])
def test_rigid_fagn_matches_the_oracle(gpv_mod, oracle, order):
    """FAGN with the rigid template (src/subset.rs:1228-1334), FP64 arithmetic:
    on FP64 coefficients (and FP64 grain maps) within 1e-8 px of the oracle,
    on FP32 coefficients and maps within the mixed bar."""
    gamma = 0.05
    f, g = TC.shear_pair(gamma)
    d = TC.grid_desc(gpv_mod, gamma, order)
    kw = dict(max_norm=1e-6, max_iterations=100, tolerance=0.75, method="fagn", texture="rigid")
    maps, s2 = oracle.grain(f)
    cf, cg = oracle.get_c(f, 8), oracle.get_c(g, 8)
    ref = oracle.solve_batch(cf, cg, f.shape, 8, d, grain=(maps, s2), eta=True,
                             **{k: v for k, v in kw.items() if k != "texture"})
    assert np.all(ref["texture"] == 1)
    for keep, prec, tol in ((True, gpv_mod.PREC_FP64, 1e-8), (False, gpv_mod.PREC_MIXED, 1e-3)):
        F = gpv_mod.Image(image_gs=f, border=8, keep_f64=keep)
        G = gpv_mod.Image(image_gs=g, border=8, keep_f64=keep)
        r = gpv_mod.solve_batch(F, G, d, precision=prec, eta=True, **kw)
        assert np.all(r["texture"] == 1)
        assert np.array_equal(r["converged"], ref["converged"]) and np.array_equal(r["status"], ref["status"])
        assert np.abs(r["p"][:, :2] - ref["p"][:, :2]).max() <= tol
        assert np.abs(r["p"][:, 2:6] - ref["p"][:, 2:6]).max() <= tol * 1e-2


@pytest.mark.parametrize("order", [1, 2])
def test_rigid_fp64_icgn_matches_the_oracle(gpv_mod, oracle, order):
    """The plain FP64 ICGN form with the rigid template: FP64 coefficients and
    FP64 grain maps (equal to the oracle's), displacement within 1e-9 px,
    gradients within 1e-11, identical iterations and flags -- the FP64 form's
    bar."""
    gamma = 0.05
    f, g = TC.shear_pair(gamma)
    d = TC.grid_desc(gpv_mod, gamma, order)
    kw = dict(max_norm=1e-6, max_iterations=100, tolerance=0.75)
    maps, s2 = oracle.grain(f)
    cf, cg = oracle.get_c(f, 8), oracle.get_c(g, 8)
    ref = oracle.solve_batch(cf, cg, f.shape, 8, d, grain=(maps, s2), eta=True, **kw)
    F = gpv_mod.Image(image_gs=f, border=8, keep_f64=True)
    G = gpv_mod.Image(image_gs=g, border=8, keep_f64=True)
    r = gpv_mod.solve_batch(F, G, d, precision=gpv_mod.PREC_FP64, texture="rigid", eta=True, **kw)
    assert np.all(r["texture"] == 1) and np.all(ref["texture"] == 1)
    assert np.array_equal(r["converged"], ref["converged"]) and np.array_equal(r["iterations"], ref["iterations"])
    assert np.abs(r["p"][:, :2] - ref["p"][:, :2]).max() < 1e-9
    assert np.abs(r["p"][:, 2:] - ref["p"][:, 2:]).max() < 1e-11
    assert np.abs(r["eta_u"] - ref["eta_u"]).max() < 1e-9


def test_rigid_falls_back_and_is_refused_where_unsupported(gpv_mod):
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F = gpv_mod.Image(image_gs=W["f"], border=20, keep_f64=True)
    G = gpv_mod.Image(image_gs=W["g"], border=20, keep_f64=True)
    d = gpv_mod.make_desc(W["coords"][:40], 25, 0, W["p0"][:40])
    r = gpv_mod.solve_batch(F, G, d, texture="rigid")  # order 0: deformable
    assert np.all(r["texture"] == 0) and np.mean(r["converged"]) > 0.9
    d1 = gpv_mod.make_desc(W["coords"][:40], 25, 1, W["p0"][:40])
    with pytest.raises(gpv_mod.GpvError):  # a device-created image has no staged pixels for the maps
        import torch
        dev = torch.from_numpy(np.ascontiguousarray(W["f"])).cuda()
        Fd = gpv_mod.Image.__new__(gpv_mod.Image)
        Fd.ctx, Fd.shape, Fd.dtype, Fd.border, Fd.keep_f64 = F.ctx, W["f"].shape, W["f"].dtype, 20, False
        h = gpv_mod.ct.c_void_p()
        gpv_mod.check(gpv_mod.lib().gpv_image_create_device(F.ctx.handle, gpv_mod.ct.c_void_p(dev.data_ptr()),
                                                             gpv_mod._lib.DTYPES[W["f"].dtype], W["f"].shape[0],
                                                             W["f"].shape[1], 20, 0, gpv_mod.ct.byref(h)), "create")
        Fd._h = h
        Fd.build_grain()
    with pytest.raises(ValueError):
        gpv_mod.solve_batch(F, G, d1, texture="grainy")
    # textured but too small to measure a correlation length (src/texture.rs:555-566):
    # the deformable template, texture 0, the deformable solve's result (the
    # rigid-capable kernel and the default deformable kernel round their FP32
    # sums differently: equal within the mixed-precision bar, same iterations)
    y, x = np.mgrid[0:14, 0:14].astype(np.float64)
    small = 100.0 + 40.0 * np.sin(0.9 * x) * np.cos(0.7 * y)
    R = gpv_mod.Image(image_gs=small, border=8)
    dr = gpv_mod.make_desc([[7.0, 7.0]], 3, 1)
    a = gpv_mod.solve_batch(R, R, dr, texture="rigid", tolerance=0.0, max_iterations=20)
    b = gpv_mod.solve_batch(R, R, dr, tolerance=0.0, max_iterations=20)
    assert not R.grain()["built"] and np.all(a["texture"] == 0)
    assert np.abs(a["p"] - b["p"]).max() < 1e-5 and np.array_equal(a["iterations"], b["iterations"])


def test_rigid_mesh_solve(gpv_mod, oracle):
    """Mesh.solve(texture="rigid") (python/src/py_mesh.rs:279-290) on the shear pair."""
    f, g = TC.shear_pair(0.05)
    F = gpv_mod.Image(image_gs=f, border=8)
    G = gpv_mod.Image(image_gs=g, border=8)
    xs = np.linspace(40, 160, 5)
    nodes = np.array([[x, y] for y in xs for x in xs])
    elements = []
    for j in range(4):
        for i in range(4):
            a, b, c, e = j * 5 + i, j * 5 + i + 1, (j + 1) * 5 + i, (j + 1) * 5 + i + 1
            elements += [[a, b, e], [a, e, c]]
    mesh = gpv_mod.Mesh(nodes, np.array(elements), F, G)
    mesh.solve(15, seed_coord=(100.3, 100.6), max_norm=1e-5, max_iterations=100, texture="rigid")
    res = mesh.results
    assert np.all(res["texture"] == 1) and np.all(res["converged"] == 1)
    assert np.abs(res["p"][:, 4] - 0.05).max() < 0.02


def test_rigid_residual_map_and_record(gpv_mod):
    """src/texture.rs:533-552: after a rigid solve the residual map uses the
    rigid template (well under half the deformable solve's rms) and the
    result records the texture."""
    f, g = TC.shear_pair(0.05)
    F = gpv_mod.Image(image_gs=f, border=8)
    G = gpv_mod.Image(image_gs=g, border=8)
    rms = []
    for tex in ("deformable", "rigid"):
        sub = gpv_mod.Subset([100.3, 100.6], gpv_mod.Mask("local", shape="circle", size=15), F, G, 1)
        sub.solve_icgn(max_norm=1e-5, max_iterations=100, tolerance=0.75, texture=tex)
        assert sub.texture == tex
        e = sub.residual_map()
        assert e.shape == (sub.n_px,) and sub.f_coords.shape == (sub.n_px, 2)
        rms.append(float(np.sqrt(np.mean(e * e))))
    assert rms[1] < 0.5 * rms[0]
    # the subset's reference values are the image's spline at its pixels
    assert np.abs(sub.f - F.eval(sub.f_coords)).max() == 0.0
