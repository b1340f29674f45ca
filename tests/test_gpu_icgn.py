"""GPU parity of the batched ICGN solve against the FP64 oracle.

Reference: Subset::new + solve_icgn_result (src/subset.rs:836-919,
1117-1219).  Both GPU forms are compared with the C oracle on the same
seeded synthetic speckle pairs:
  * FP64 form: displacement within 1e-9 px, gradients within 1e-11, ZNCC
    within 1e-10, identical iteration counts and flags;
  * mixed form (FP32 interpolation): displacement within 1e-3 px and
    strain terms within 1e-5 (the stated parity bar), ZNCC within 1e-5,
    identical converged / quality flags; iteration counts may differ by one
    on at most 2% of subsets (at least one) -- a borderline norm near max_norm.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BORDER = 20


def _images(gpv_mod, oracle, W):
    f = W["f"].astype(np.float64)
    g = W["g"].astype(np.float64)
    F = gpv_mod.Image(image_gs=W["f"], border=BORDER, keep_f64=True)
    G = gpv_mod.Image(image_gs=W["g"], border=BORDER, keep_f64=True)
    Cf, Cg = oracle.get_c(f, BORDER), oracle.get_c(g, BORDER)
    return F, G, Cf, Cg


def _desc(gpv_mod, W):
    return gpv_mod.make_desc(W["coords"], W["radius"], W["order"], W["p0"])


def _compare(res, ref, exact, label):
    ok = (ref["status"] == 0)
    assert np.array_equal(res["status"], ref["status"]), label
    assert np.array_equal(res["n_px"], ref["n_px"]), label
    dp = np.abs(res["p"] - ref["p"])
    if exact:
        assert dp[ok][:, :2].max() < 1e-9, label
        assert dp[ok][:, 2:].max() < 1e-11, label
        assert np.abs(res["c_zncc"] - ref["c_zncc"])[ok].max() < 1e-10, label
        assert np.array_equal(res["iterations"], ref["iterations"]), label
    else:
        assert dp[ok][:, :2].max() <= 1e-3, label
        assert dp[ok][:, 2:6].max() <= 1e-5, label
        assert np.abs(res["c_zncc"] - ref["c_zncc"])[ok].max() < 1e-5, label
        it_diff = np.abs(res["iterations"].astype(int) - ref["iterations"])
        assert it_diff.max() <= 1 and (it_diff > 0).sum() <= max(1, int(np.ceil(0.02 * len(it_diff)))), label
    assert np.array_equal(res["converged"], ref["converged"]), label
    assert np.array_equal(res["quality_ok"], ref["quality_ok"]), label


# (1, 1): the rigid 1024^2 workload at full size, every one of its 2,401 subsets
@pytest.mark.parametrize("config,scale", [(1, 1), (1, 4), (2, 16), (3, 8)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_oracle(oracle, gpv_mod, config, scale, precision):
    from gpv import synth
    W = synth.workload(config, scale_down=scale)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    d = _desc(gpv_mod, W)
    kw = dict(max_norm=1e-5, max_iterations=15 if config == 1 else 50, tolerance=0.75)
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, BORDER, d, **kw)
    prec = gpv_mod.PREC_FP64 if precision == "fp64" else gpv_mod.PREC_MIXED
    res = gpv_mod.solve_batch(F, G, d, precision=prec, **kw)
    _compare(res, ref, precision == "fp64", f"C{config} {precision}")
    # and the solve recovers the imposed field (noise-limited)
    good = ref["quality_ok"] == 1
    assert good.mean() > 0.9
    err = np.abs(res["p"][good, :2] - W["truth_uv"][good])
    assert np.median(err) < 0.05


@pytest.mark.parametrize("config,scale", [(2, 16), (3, 8)])
def test_compensated_sums_match_oracle(oracle, gpv_mod, config, scale):
    """The Kahan-compensated FP64 ZNSSD sums (GPV_SOLVE_KAHAN) meet the
    mixed-precision bar against the oracle like the default form."""
    from gpv import _lib, synth
    W = synth.workload(config, scale_down=scale)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    d = _desc(gpv_mod, W)
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, BORDER, d, max_norm=1e-5, max_iterations=50)
    prm = gpv_mod._params(1e-5, 50, 0.75, False, gpv_mod.PREC_MIXED, None, None)
    prm.flags |= _lib.SOLVE_KAHAN
    out = np.zeros(len(d), dtype=_lib.RESULT_DTYPE)
    _lib.check(_lib.lib().gpv_solve_batch(F.ctx.handle, F.handle, G.handle, _lib.ptr(d), len(d), _lib.ct.byref(prm),
                                          _lib.ptr(out)), "kahan solve")
    _compare(out, ref, False, f"C{config} kahan")


@pytest.mark.parametrize("order", [0, 1, 2])
def test_orders_and_history(oracle, gpv_mod, order):
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    n = 24
    d = gpv_mod.make_desc(W["coords"][:n], 25, order)
    d["coord"] += 0.37  # fractional centres
    kw = dict(max_norm=1e-5, max_iterations=20, tolerance=0.75)
    ref, rh = oracle.solve_batch(Cf, Cg, W["f"].shape, BORDER, d, history=True, eta=True, **kw)
    for prec, exact in ((gpv_mod.PREC_FP64, True), (gpv_mod.PREC_MIXED, False)):
        res, hist = gpv_mod.solve_batch(F, G, d, precision=prec, history=True, eta=True, **kw)
        _compare(res, ref, exact, f"order {order}")
        k = ref["iterations"].min()
        tol = 1e-9 if exact else 2e-5
        assert np.abs(hist[:, :k, 1] - rh[:, :k, 1]).max() < tol  # per-iteration ZNCC
        # eta (src/subset.rs:748-820) at the last sampled warp
        assert np.all(res["has_eta"] == 1)
        et = 1e-9 if exact else 2e-3
        assert np.abs(res["eta_u"] - ref["eta_u"]).max() < et
        assert np.abs(res["eta_v"] - ref["eta_v"]).max() < et


def test_border_subsets_clamp(oracle, gpv_mod):
    """Subsets that overhang the image sample the clamped spline (src/image.rs:129-132)."""
    from gpv import synth
    W = synth.workload(1, scale_down=8)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    n = W["f"].shape[0]
    xy = np.array([[3.2, 60.0], [n - 2.5, 40.0], [50.0, 1.0], [64.0, n - 1.5], [0.0, 0.0]])
    d = gpv_mod.make_desc(xy, 25, 1)
    kw = dict(max_norm=1e-5, max_iterations=15, tolerance=0.75)
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, BORDER, d, **kw)
    res = gpv_mod.solve_batch(F, G, d, precision=gpv_mod.PREC_FP64, **kw)
    _compare(res, ref, True, "border fp64")
    res = gpv_mod.solve_batch(F, G, d, precision=gpv_mod.PREC_MIXED, **kw)
    assert np.abs(res["p"][:, :2] - ref["p"][:, :2]).max() <= 1e-3


def test_global_mask(oracle, gpv_mod):
    """Global mask intersection (src/masks.rs:199-263), including an empty subset."""
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    h, w = W["f"].shape
    mask = np.ones((h, w), np.uint8)
    mask[:, 120:] = 0            # right part masked
    mask[40:70, 20:50] = 0       # a hole
    xy = np.array([[100.0, 100.0], [118.0, 60.0], [35.0, 55.0], [200.0, 200.0], [230.5, 230.5], [28.0, 230.0]])
    d = gpv_mod.make_desc(xy, 25, 1)
    gm = gpv_mod.Mask("global", binary=mask)
    kw = dict(max_norm=1e-5, max_iterations=15, tolerance=0.75)
    ref = oracle.solve_batch(Cf, Cg, (h, w), BORDER, d, mask=mask, **kw)
    assert ref["status"][3] == 1  # EMPTY_MASK
    for prec, exact in ((gpv_mod.PREC_FP64, True), (gpv_mod.PREC_MIXED, False)):
        res = gpv_mod.solve_batch(F, G, d, precision=prec, global_mask=gm, **kw)
        _compare(res, ref, exact, "mask")


def test_failure_statuses(oracle, gpv_mod):
    """Featureless subsets, invalid descriptors, convergence-gated quality."""
    flat = np.full((80, 80), 90, np.uint8)
    F = gpv_mod.Image(image_gs=flat, border=BORDER, keep_f64=True)
    d = gpv_mod.make_desc([[40.0, 40.0]], 10, 1)
    C = oracle.get_c(flat.astype(np.float64), BORDER)
    assert oracle.solve_batch(C, C, flat.shape, BORDER, d)["status"][0] == 2
    for prec in (gpv_mod.PREC_FP64, gpv_mod.PREC_MIXED):
        r = gpv_mod.solve_batch(F, F, d, precision=prec)
        assert r["status"][0] == 2 and r["quality_ok"][0] == 0  # FEATURELESS
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    d = gpv_mod.make_desc([[100.0, 100.0], [120.0, 120.0], [100.0, 120.0]], [25, 0, 25], [1, 1, 3])
    for prec in (gpv_mod.PREC_FP64, gpv_mod.PREC_MIXED):
        r = gpv_mod.solve_batch(F, G, d, precision=prec)
        assert list(r["status"]) == [0, 8, 8]
    # test_quality_ok_requires_convergence (src/subset.rs:2136-2167)
    d = gpv_mod.make_desc([[100.0, 100.0]], 25, 1)
    for prec in (gpv_mod.PREC_FP64, gpv_mod.PREC_MIXED):
        r = gpv_mod.solve_batch(F, G, d, precision=prec, max_norm=1e-8, max_iterations=1, tolerance=0.0)
        assert r["converged"][0] == 0 and r["quality_ok"][0] == 0 and r["iterations"][0] == 1
        # test_solved_false_below_tolerance (src/subset.rs:2104-2129)
        r = gpv_mod.solve_batch(F, G, d, precision=prec, max_norm=1e-3, tolerance=2.0)
        assert r["converged"][0] == 1 and r["quality_ok"][0] == 0
    # zero iterations: no history, ZNCC 0 / ZNSSD 4 (src/subset.rs:1190-1193)
    r = gpv_mod.solve_batch(F, G, d, max_iterations=0)
    assert r["iterations"][0] == 0 and r["c_zncc"][0] == 0.0 and r["c_znssd"][0] == 4.0


def test_subset_api(oracle, gpv_mod):
    """The Python mirror of Subset(...).solve() (geopyv_dev/__init__.py:338-385)."""
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    lm = gpv_mod.Mask("local", shape="circle", size=25)
    assert lm.n_px == 1961
    s = gpv_mod.Subset([128.43, 128.76], lm, F, G, subset_order=1)
    s.solve()  # defaults: max_norm 1e-3, max_iterations 50, tolerance 0.75
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, BORDER, gpv_mod.make_desc([[128.43, 128.76]], 25, 1),
                             max_norm=1e-3, max_iterations=50, tolerance=0.75)
    assert s.solved and s.converged == bool(ref["converged"][0])
    assert np.abs(s.p[:2] - ref["p"][0, :2]).max() < 1e-3
    assert s.n_px == 1961 and len(s.history) == s.iterations
    with pytest.raises(RuntimeError):
        gpv_mod.Subset([40.0, 40.0], gpv_mod.Mask("local", shape="circle", size=10),
                       gpv_mod.Image(image_gs=np.full((80, 80), 9.0)), gpv_mod.Image(image_gs=np.full((80, 80), 9.0))).solve()


def test_autotune_choices_do_not_change_results(oracle, gpv_mod):
    """Every launch shape the autotuner can pick gives the same solution."""
    from gpv import synth
    W = synth.workload(3, scale_down=8)
    F, G, Cf, Cg = _images(gpv_mod, oracle, W)
    d = _desc(gpv_mod, W)
    tuned = gpv_mod.autotune(F, G, d, sample_per_class=256)
    present = {0: np.any(d["radius"] <= 20), 1: np.any((d["radius"] > 20) & (d["radius"] <= 40)), 2: np.any(d["radius"] > 40)}
    for c in range(3):
        assert tuned[c] in ((64, 128, 256) if present[c] else (0,))
    choice = F.ctx.tuning()
    for c in range(3):
        if present[c]:  # an absent class keeps whatever the shared context held
            assert choice[c]["threads"] == tuned[c] and choice[c]["layout"] in (None, "compact", "tiles")
            assert choice[c]["run_length"] in (4, 8)
    import os
    res = {}
    for nt, k in (("128", "8"), ("256", "8"), ("64", "4"), ("128", "4")):
        os.environ["GPV_TILE_THREADS"] = nt
        os.environ["GPV_RUN_K"] = k
        try:
            ctx = gpv_mod.Context(0)  # a fresh context carries no tuned choice
            F2 = gpv_mod.Image(image_gs=W["f"], border=BORDER, ctx=ctx)
            G2 = gpv_mod.Image(image_gs=W["g"], border=BORDER, ctx=ctx)
            res[nt + "/" + k] = gpv_mod.solve_batch(F2, G2, d, max_norm=1e-5, max_iterations=50)
        finally:
            del os.environ["GPV_TILE_THREADS"]
            del os.environ["GPV_RUN_K"]
    base = res["128/8"]
    for key, r in res.items():
        assert np.array_equal(base["iterations"], r["iterations"]) or \
            (base["iterations"] != r["iterations"]).mean() < 0.02, key
        assert np.abs(base["p"] - r["p"]).max() < 1e-4, key


@pytest.mark.parametrize("layout", ["rows", "tiles"])
def test_template_layouts_match_the_oracle(gpv_mod, oracle, layout, monkeypatch):
    """The padded-row and 8 x 4 tile slot layouts of the tiled kernel (chosen
    with GPV_TILE_LAYOUT) solve every subset like its compact one."""
    from gpv import synth
    W = synth.workload(3, scale_down=8)
    d = gpv_mod.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    F = gpv_mod.Image(image_gs=W["f"], border=20)
    G = gpv_mod.Image(image_gs=W["g"], border=20)
    monkeypatch.setenv("GPV_SOLVE_KERNEL", "tile")
    base = gpv_mod.solve_batch(F, G, d)
    monkeypatch.setenv("GPV_TILE_LAYOUT", layout)
    got = gpv_mod.solve_batch(F, G, d)
    monkeypatch.delenv("GPV_TILE_LAYOUT")
    Cf = oracle.get_c(W["f"].astype(np.float64), 20)
    Cg = oracle.get_c(W["g"].astype(np.float64), 20)
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d)
    for a in (base, got):
        assert np.array_equal(a["status"], ref["status"]) and np.array_equal(a["converged"], ref["converged"])
        ok = a["status"] == 0
        assert np.abs(a["p"][ok, :2] - ref["p"][ok, :2]).max() <= 1e-3
        assert np.abs(a["p"][ok, 2:6] - ref["p"][ok, 2:6]).max() <= 1e-5
    assert np.array_equal(got["n_px"], base["n_px"])


def test_tune_cache_file_is_read_back(gpv_mod, tmp_path, monkeypatch):
    """A context reads GPV_TUNE_CACHE lines for its device: "name|class|threads"
    (layout unset) and "name|class|threads|layout"; later lines win, other
    devices' lines and malformed ones are ignored."""
    import torch
    name = torch.cuda.get_device_name(0)
    cache = tmp_path / "tune.txt"
    cache.write_text(f"{name}|0|128\nOther GPU|1|128|0\n{name}|1|128|0\n{name}|1|256|2\n{name}|2|999|0\n")
    monkeypatch.setenv("GPV_TUNE_CACHE", str(cache))
    ctx = gpv_mod.Context(0)
    try:
        got = [(t["threads"], t["layout"]) for t in ctx.tuning()]
        assert got == [(128, None), (256, "tiles"), (None, None)]
    finally:
        ctx.close()
