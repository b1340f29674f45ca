"""FAGN on the GPU (GPV_SOLVE_FAGN) against the oracle's FAGN
(src/subset.rs:1228-1334), on seeded synthetic pairs.

FP64 coefficients: warps within 1e-8, identical flags, iterations equal on
>= 98% of subsets.  FP32 coefficients (FP64 arithmetic): displacement within
1e-3 px, gradients within 1e-5, identical flags.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(config, scale):
    from gpv import synth
    W = synth.workload(config, scale_down=scale)
    if config == 3:  # keep it quick: every third subset
        for k in ("coords", "radius", "order", "p0", "truth_uv"):
            W[k] = W[k][::3]
    return W


@pytest.mark.parametrize("config,scale", [(1, 4), (3, 8), (2, 8)])
@pytest.mark.parametrize("precision", [1, 0], ids=["fp64", "mixed"])
def test_fagn_batch_matches_oracle(gpv_mod, oracle, config, scale, precision):
    W = _case(config, scale)
    d = gpv_mod.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    keep = precision == 1
    F = gpv_mod.Image(image_gs=W["f"], border=20, keep_f64=keep)
    G = gpv_mod.Image(image_gs=W["g"], border=20, keep_f64=keep)
    got = gpv_mod.solve_batch(F, G, d, max_norm=1e-5, eta=True, precision=precision, method="fagn")
    Cf = oracle.get_c(W["f"].astype(np.float64), 20)
    Cg = oracle.get_c(W["g"].astype(np.float64), 20)
    ref = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, eta=True, method="fagn")
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["converged"], ref["converged"])
    assert np.array_equal(got["quality_ok"], ref["quality_ok"])
    ok = (got["status"] == 0) & (got["iterations"] == ref["iterations"])
    assert ok.mean() >= 0.98
    if precision == 1:
        assert np.abs(got["p"][ok] - ref["p"][ok]).max() < 1e-8
        assert np.abs(got["eta_u"][ok] - ref["eta_u"][ok]).max() < 1e-8
    else:
        assert np.abs(got["p"][ok, :2] - ref["p"][ok, :2]).max() <= 1e-3
        assert np.abs(got["p"][ok, 2:6] - ref["p"][ok, 2:6]).max() <= 1e-5
    assert np.abs(got["c_zncc"][ok] - ref["c_zncc"][ok]).max() < 1e-5


def test_subset_fagn_api(gpv_mod):
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    F = gpv_mod.Image(image_gs=W["f"])
    G = gpv_mod.Image(image_gs=W["g"])
    m = gpv_mod.Mask("local", shape="circle", size=25)
    a = gpv_mod.Subset(W["coords"][0], m, F, G)
    a.solve(algorithm="fagn")
    b = gpv_mod.Subset(W["coords"][0], m, F, G)
    b.solve(algorithm="icgn")
    assert a.converged and b.converged
    assert abs(a.c_zncc - b.c_zncc) < 1e-4
    assert abs(a.p[0] - b.p[0]) < 5e-3 and abs(a.p[1] - b.p[1]) < 5e-3
    c = gpv_mod.Subset(W["coords"][0], m, F, G)
    c.solve_fagn(max_norm=1e-20, max_iterations=1)
    assert c.iterations == 1 and not c.converged


def test_mesh_fagn_matches_oracle(gpv_mod, oracle):
    import mesh_cases as MC
    import mesh_oracle as M
    f = MC.texture(100)
    g = MC.shift_uniform(f, 1.5)
    nodes, el = MC.grid_mesh()
    Cf = oracle.get_c(f, 15)
    Cg = oracle.get_c(g, 15)

    def solver(desc, tol):
        return oracle.solve_batch(Cf, Cg, f.shape, 15, desc, max_norm=1e-5, tolerance=tol, method="fagn")
    ref = M.solve_mesh(nodes, el, solver, desc_dtype=oracle.DESC_DTYPE, radius=8, seed_coord=(50.0, 50.0),
                       seed_tolerance=0.5, tolerance=0.5, preconditioning="layer-RG", max_workers=2)
    F = gpv_mod.Image(image_gs=f, border=15, keep_f64=True)
    G = gpv_mod.Image(image_gs=g, border=15, keep_f64=True)
    m = gpv_mod.Mesh(nodes, el, F, G)
    m.solve(8, seed_coord=(50.0, 50.0), seed_tolerance=0.5, tolerance=0.5, preconditioning="layer-RG",
            layer_rg_max_workers=2, method="fagn", precision=gpv_mod.PREC_FP64, override_active=True)
    rp = np.array([x["p"] for x in ref["results"]])
    assert m.seed_node == ref["seed_node"]
    assert np.array_equal(m.quality_ok, ref["quality_ok"])
    assert np.abs(m.results["p"] - rp).max() < 1e-7
