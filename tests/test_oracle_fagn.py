"""The oracle's FAGN restatement (src/subset.rs:1228-1334) against the
reference's own FAGN tests, restated on a seeded synthetic pair (the
reference's real-image goldens need images absent from its checkout):

* FAGN and ICGN agree: |dZNCC| < 1e-4 (tests/python/subset/test_subset.py:
  591-596) and the displacements closely (:598-605 bounds them by 1e-3 px on
  its real pair; with 2 DN noise here the two methods' fixed points --
  target-gradient vs reference-gradient weighted residuals -- sit up to
  ~2e-3 px apart, so the bound here is 5e-3 px);
* the oracle's FAGN equals an independent numpy restatement to 1e-9;
* first and second order converge, order 2 with ZNCC > 0.998 (:316-320 asks
  0.999 on its real pair; this pair's noise floor is 0.9989 for ICGN too);
* max_iterations is respected: one iteration at max_norm 1e-20 stops
  unconverged (:322-326).
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def pair(oracle):
    from gpv import synth
    W = synth.workload(1, scale_down=4)
    Cf = oracle.get_c(W["f"].astype(np.float64), 20)
    Cg = oracle.get_c(W["g"].astype(np.float64), 20)
    return W, Cf, Cg


def _desc(oracle, W, order, k=12):
    d = np.zeros(k, oracle.DESC_DTYPE)
    d["coord"] = W["coords"][:k]
    d["radius"], d["order"] = 25, order
    return d


@pytest.mark.parametrize("order", [1, 2])
def test_fagn_agrees_with_icgn(oracle, pair, order):
    W, Cf, Cg = pair
    d = _desc(oracle, W, order)
    ri = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-3, method="icgn")
    rf = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-3, method="fagn")
    assert np.all(rf["converged"] == 1) and np.all(rf["status"] == 0)
    assert np.abs(ri["c_zncc"] - rf["c_zncc"]).max() < 1e-4
    assert np.abs(ri["p"][:, :2] - rf["p"][:, :2]).max() < 5e-3
    if order == 2:  # :316-320 asks > 0.999 on its real pair; this pair's 2 DN noise caps ICGN at ~0.9989 too
        assert rf["c_zncc"].min() > 0.998
    # and both recover the imposed translation
    assert np.abs(rf["p"][:, :2] - W["truth_uv"][:len(d)]).max() < 0.02


def test_fagn_respects_max_iterations(oracle, pair):
    W, Cf, Cg = pair
    d = _desc(oracle, W, 1, 3)
    r = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-20, max_iterations=1, method="fagn")
    assert np.all(r["iterations"] == 1) and np.all(r["converged"] == 0)


def test_fagn_history_and_eta(oracle, pair):
    W, Cf, Cg = pair
    d = _desc(oracle, W, 1, 4)
    r, h = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, eta=True, history=True, method="fagn")
    for i in range(len(d)):
        k = int(r["iterations"][i])
        assert h[i, k - 1, 0] == r["norm"][i] and h[i, k - 1, 1] == r["c_zncc"][i]
    assert np.all(r["has_eta"] == 1) and np.all(np.isfinite(r["eta_u"]))


def _np_fagn(oracle, C, shape, coord, radius, order, max_norm, max_iterations, f, f_m, df):
    """Independent restatement: numpy arrays, the oracle's spline evaluator."""
    offs = oracle.circle(radius)
    fc = offs + np.asarray(coord)
    m = {0: 2, 1: 6, 2: 12}[order]
    p = np.zeros(m)
    n = len(fc)
    for it in range(1, max_iterations + 1):
        dx0, dy0 = offs[:, 0], offs[:, 1]
        u = p[0] + (p[2] * dx0 + p[4] * dy0 if m >= 6 else 0 * dx0)
        v = p[1] + (p[3] * dx0 + p[5] * dy0 if m >= 6 else 0 * dy0)
        if m == 12:
            u = u + 0.5 * p[6] * dx0 ** 2 + p[8] * dx0 * dy0 + 0.5 * p[10] * dy0 ** 2
            v = v + 0.5 * p[7] * dx0 ** 2 + p[9] * dx0 * dy0 + 0.5 * p[11] * dy0 ** 2
        gc = fc + np.stack([u, v], 1)
        g, grad = oracle.evaluate(C, shape, 20, gc, grad=True)
        gm = g.mean()
        dg = np.sqrt(((g - gm) ** 2).sum())
        dx = gc[:, 0] - (coord[0] + p[0])
        dy = gc[:, 1] - (coord[1] + p[1])
        gx, gy = grad[:, 0], grad[:, 1]
        cols = [gx, gy]
        if m >= 6:
            cols += [gx * dx, gy * dx, gx * dy, gy * dy]
        if m == 12:
            cols += [gx * 0.5 * dx * dx, gy * 0.5 * dx * dx, gx * dx * dy, gy * dx * dy, gx * 0.5 * dy * dy,
                     gy * 0.5 * dy * dy]
        sdi = np.stack(cols, 1)
        r = (f - f_m) * (dg / df) - (g - gm)
        dp = np.linalg.solve(sdi.T @ sdi, sdi.T @ r)
        p = p + dp
        nrm = oracle.convergence_norm(dp, np.sqrt(n))
        if nrm < max_norm:
            break
    return p, it


@pytest.mark.parametrize("order", [0, 1, 2])
def test_fagn_matches_numpy_restatement(oracle, pair, order):
    W, Cf, Cg = pair
    d = _desc(oracle, W, order, 3)
    r = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-6, method="fagn")
    for i in range(len(d)):
        coord = d["coord"][i]
        f = oracle.evaluate(Cf, W["f"].shape, 20, oracle.circle(25) + coord)
        fm = f.mean()
        df = np.sqrt(((f - fm) ** 2).sum())
        p, it = _np_fagn(oracle, Cg, W["f"].shape, coord, 25, order, 1e-6, 50, f, fm, df)
        m = len(p)
        assert it == r["iterations"][i]
        assert np.abs(p - r["p"][i, :m]).max() < 1e-9
