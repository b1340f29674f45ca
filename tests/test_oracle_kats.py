"""Pin the CPU oracle to the reference's own known answers.

Each case of tests/golden/reference_kats.json is a known-answer test of the
reference crate (file:line in the entry), run here against the C oracle.
"""
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))


def _quad_warp(q, x, y):
    # quad_warp (src/particle.rs:2624-2635)
    return [q[0] + q[2] * x + q[4] * y + 0.5 * q[6] * x * x + q[8] * x * y + 0.5 * q[10] * y * y,
            q[1] + q[3] * x + q[5] * y + 0.5 * q[7] * x * x + q[9] * x * y + 0.5 * q[11] * y * y]


def _qcqt(C, border, i, j):
    import np_oracle as N
    blk = C[i + border - 2:i + border + 4, j + border - 2:j + border + 4]
    return N.Q @ blk @ N.Q.T


@pytest.mark.parametrize("k", KATS, ids=[k["name"] for k in KATS])
def test_reference_kat(oracle, k):
    O = oracle
    fn = k["fn"]
    if fn == "norm":
        assert abs(O.convergence_norm(k["dp"], k["size"]) - k["expected"]) <= max(k["atol"], 0.0) + 0.0
    elif fn == "zn_slice":
        assert np.abs(O.zn_slice(k["x"]) - k["expected"]).max() <= k["atol"]
    elif fn == "eta_component":
        eta = O.eta_component(np.array(k["modes"]), k["grad_zn"], k["e_centered"])
        if k["expected"] == ">=0":
            assert eta >= 0.0
        else:
            assert abs(eta - k["expected"]) < k["atol"]
    elif fn == "eta_identical":
        f = np.array(k["f"])
        fm = f.mean()
        df = math.sqrt(np.sum((f - fm) ** 2))
        for order in (0, 1, 2):
            eu, ev = O.omitted_mode_diagnostic(k["coord"], order, k["f_coords"], k["grad_f"], f, fm, df, f, fm, df)
            assert abs(eu) < k["atol"] and abs(ev) < k["atol"]
        assert O.omitted_mode_diagnostic(k["coord"], 3, k["f_coords"], k["grad_f"], f, fm, df, f, fm, df) is None
    elif fn == "znssd_identical":
        f = np.array(k["f"])
        fm = f.mean()
        df = math.sqrt(np.sum((f - fm) ** 2))
        assert abs(O.znssd(f, f, fm, fm, df, df)) < k["atol"]
    elif fn == "znssd_range":
        f, g = np.array(k["f"]), np.array(k["g"])
        z = O.znssd(f, g, f.mean(), g.mean(), math.sqrt(np.sum((f - f.mean()) ** 2)), math.sqrt(np.sum((g - g.mean()) ** 2)))
        assert k["expected"][0] <= z <= k["expected"][1]
    elif fn == "compose":
        assert np.abs(O.compose(k["p"], k["dp"]) - k["expected"]).max() < k["atol"]
    elif fn == "compose_len":
        assert O.compose(k["p"], k["dp"]).size == k["expected"]
    elif fn == "warp_convention":
        q, c = k["q"], k["centre"]
        x = np.array(k["points"])
        for order in (1, 2):
            p = q[:6] if order == 1 else q
            g = O.apply_warp(c, p, x)
            for i in range(len(x)):
                dx, dy = x[i, 0] - c[0], x[i, 1] - c[1]
                want = _quad_warp(q, dx, dy) if order == 2 else [q[0] + q[2] * dx + q[4] * dy, q[1] + q[3] * dx + q[5] * dy]
                assert abs(g[i, 0] - x[i, 0] - want[0]) < 1e-12 and abs(g[i, 1] - x[i, 1] - want[1]) < 1e-12
        # SDI columns are warp derivatives (src/subset.rs:2241-2259)
        grad = np.array([[0.3, -0.7], [1.1, 0.2], [-0.4, 0.9], [0.6, 0.5]])
        sdi = O.steepest_descent(c, x, grad, 2)
        h = 1e-6
        for kk in range(12):
            pp = list(q)
            pp[kk] += h
            d = (O.apply_warp(c, pp, x) - O.apply_warp(c, q, x)) / h
            assert np.abs(sdi[:, kk] - (grad * d).sum(1)).max() < 1e-6
        for p in (q[:6], q):  # compose_zero_update_is_identity (src/subset.rs:2262-2269)
            assert np.abs(O.compose(p, [0.0] * len(p)) - p).max() < 1e-14
    elif fn == "compose_roundtrip1":
        c = [10.0, 10.0]
        x = np.array([[13.0, 7.0], [4.0, 15.0], [9.5, 9.5], [16.0, 2.0]])
        p = [0.1, -0.2, 0.02, 0.07, 0.03, -0.01]
        pn = O.compose(p, k["dp"])
        via = O.apply_warp(c, pn, O.apply_warp(c, k["dp"], x))
        assert np.abs(via - O.apply_warp(c, p, x)).max() < k["atol"]
        # order-2 composition with no quadratic terms is exactly affine (src/subset.rs:2308-2323)
        q = [0.1, -0.2, 0.02, 0.07, 0.03, -0.01] + [0.0] * 6
        dp = list(k["dp"]) + [0.0] * 6
        via = O.apply_warp(c, O.compose(q, dp), O.apply_warp(c, dp, x))
        assert np.abs(via - O.apply_warp(c, q, x)).max() < 1e-12
    elif fn == "compose_roundtrip2":
        inv = O.compose([0.0] * 12, k["dp"])

        def err(r):
            x = np.array([[0.6 * r, -0.8 * r]])
            back = O.apply_warp([0.0, 0.0], inv, O.apply_warp([0.0, 0.0], k["dp"], x))
            return float(np.hypot(*(back - x)[0]))
        for r in (8.0, 4.0, 2.0):
            assert err(r) / err(r / 2.0) > k["expected"]
    elif fn == "circle":
        c = O.circle(k["radius"])
        assert c.shape == (k["n_px"], 2)
        assert list(c[0]) == k["first"] and list(c[-1]) == k["last"]
    elif fn == "mask_zero":
        c = O.circle(2)
        assert O.mask_update(c, 2, [5.0, 5.0], np.zeros((20, 20), np.uint8)).shape[0] == 0
        assert O.mask_update(c, 2, [5.0, 5.0], np.ones((20, 20), np.uint8)).shape[0] == c.shape[0]
    elif fn == "get_c_constant":
        C = O.get_c(np.full(k["shape"], k["value"]), k["border"])
        assert C.shape == (k["shape"][0] + 2 * k["border"], k["shape"][1] + 2 * k["border"])
        assert np.all(np.abs(C - k["value"]) < k["rtol"] * k["value"])
        blk = _qcqt(C, k["border"], 5, 5)  # test_get_qcqt_constant (src/image.rs:554-566)
        assert abs(blk[0, 0] - k["value"]) < 1e-10 and np.abs(blk.ravel()[1:]).max() < 1e-10
    elif fn == "q_row_sums":
        import np_oracle as N
        assert np.abs(N.Q.sum(1) - k["expected"]).max() < k["atol"]
        for t in (0.0, 0.3, 0.999):  # oracle basis agrees with Q^T [1..t^5]
            assert np.abs(O.qt_poly(t) - N.qt_poly(t)).max() < 1e-15
            assert np.abs(O.qt_dpoly(t) - N.qt_dpoly(t)).max() < 1e-15
    elif fn == "qcqt_form":
        y, x = np.mgrid[0:k["shape"][0], 0:k["shape"][1]].astype(float)
        img = 60.0 + np.sin(x * 0.9) * 20.0 + np.cos(y * 0.7) * 15.0
        C = O.get_c(img, k["border"])
        pts = np.array(k["points"])
        v, g = O.evaluate(C, img.shape, k["border"], pts, grad=True)
        p = lambda t: np.array([1, t, t * t, t ** 3, t ** 4, t ** 5])
        d = lambda t: np.array([0, 1, 2 * t, 3 * t * t, 4 * t ** 3, 5 * t ** 4])
        for i, (px, py) in enumerate(pts):
            xf, yf = int(np.floor(px)), int(np.floor(py))
            blk = _qcqt(C, k["border"], yf, xf)
            assert abs(v[i] - p(py - yf) @ blk @ p(px - xf)) < k["atol"]
            assert abs(g[i, 0] - p(py - yf) @ blk @ d(px - xf)) < k["atol"]
            assert abs(g[i, 1] - d(py - yf) @ blk @ p(px - xf)) < k["atol"]
        assert np.array_equal(O.evaluate(C, img.shape, k["border"], pts), v)  # eval vs eval_grad bits
    elif fn == "grad_fd":
        r, c = np.mgrid[0:60, 0:60].astype(float)
        a = 120.0 + 60.0 * np.sin(2 * np.pi * r / 7.0 + 0.3) * np.cos(2 * np.pi * c / 9.0)
        C = O.get_c(a, k["border"])
        h = 1e-5
        for x, y in k["points"]:
            _, g = O.evaluate(C, a.shape, k["border"], [[x, y]], grad=True)
            vv = O.evaluate(C, a.shape, k["border"], [[x + h, y], [x - h, y], [x, y + h], [x, y - h]])
            assert abs(g[0, 0] - (vv[0] - vv[1]) / (2 * h)) < k["atol"]
            assert abs(g[0, 1] - (vv[2] - vv[3]) / (2 * h)) < k["atol"]
    elif fn == "const_eval":
        C = O.get_c(np.full(k["shape"], k["value"]), k["border"])
        v = O.evaluate(C, k["shape"], k["border"], k["points"])
        assert np.all(np.abs(v - k["value"]) < k["rtol"] * k["value"])
    elif fn == "clamp":
        r, c = np.mgrid[0:8, 0:9].astype(float)
        img = 100.0 + np.sin(c * 1.3) * 20.0 + np.cos(r * 0.8) * 10.0
        C = O.get_c(img, k["border"])
        far, edge = O.evaluate(C, img.shape, k["border"], [[1_000_000.0, 0.0], [9.0 - 1e-9, 0.0]])
        assert np.isfinite(far) and abs(far) < 200.0 and abs(far - edge) < k["atol"]
        _, g = O.evaluate(C, img.shape, k["border"], [[1_000_000.0, -1_000_000.0]], grad=True)
        assert np.all(np.isfinite(g)) and np.all(np.abs(g) < 200.0)
    elif fn.startswith("mesh_"):
        _mesh_kat(k)
    else:
        raise AssertionError(f"unknown KAT kind {fn}")


def _mesh_kat(k):
    import mesh_oracle as M
    fn = k["fn"]
    if fn == "mesh_connectivity":
        assert M.connectivity(k["elements"], k["order"], k["idx"], k["full"]) == k["expected"]
    elif fn == "mesh_adjacency":  # the per-node table equals the brute-force scan, both relations
        for elements, order, n in k["cases"]:
            full, edge = M.adjacency(elements, order, n)
            for i in range(n):
                assert full[i] == M.connectivity(elements, order, i, True)
                assert edge[i] == M.connectivity(elements, order, i, False)
    elif fn == "mesh_seed":
        assert M.find_seed_node(k["nodes"], k["coord"]) == k["expected"]
    elif fn == "mesh_project":
        p = [0.0] * 12
        for slot, v in k["p"].items():
            p[int(slot)] = v
        assert abs(M.project_warp(p, k["dx"], k["dy"])[k["slot"]] - k["expected"]) < k["atol"]
    elif fn == "mesh_project_quad":
        q = k["q"]

        def full(x, y):  # quad_warp (src/particle.rs:2624-2635), every slot
            u, v = _quad_warp(q, x, y)
            return [u, v, q[2] + q[6] * x + q[8] * y, q[3] + q[7] * x + q[9] * y, q[4] + q[8] * x + q[10] * y,
                    q[5] + q[9] * x + q[11] * y] + list(q[6:])
        (cx, cy), (dx, dy) = k["c"], k["d"]
        w = M.project_warp(full(cx, cy), dx, dy)
        assert np.abs(np.array(w) - full(cx + dx, cy + dy)).max() < k["atol"]
    elif fn == "mesh_affine_fit":
        (ux, uy, u0), (vx, vy, v0) = k["u"], k["v"]
        nodes = k["nodes"]
        p = [[ux * x + uy * y + u0, vx * x + vy * y + v0, 0, 0, 0, 0] for x, y in nodes]
        t = k["target"]
        fit = M.affine_field_fit(nodes, t, list(range(len(nodes))), p, 6)
        want = [ux * t[0] + uy * t[1] + u0, vx * t[0] + vy * t[1] + v0, ux, vx, uy, vy]
        assert np.abs(np.array(fit) - want).max() < k["atol"]
    elif fn == "mesh_affine_collinear":
        nodes = k["nodes"]
        assert M.affine_field_fit(nodes, k["target"], [0, 1, 2], [[0.0] * 6] * 3, 6) is None
    elif fn == "mesh_precondition":
        nodes, c, p, t = k["nodes"], k["c_zncc"], k["p"], k["target"]
        assert all(v == 0.0 for v in M.precondition_warp(nodes, t, [], c, p, 6))
        one = M.precondition_warp(nodes, t, [1], c, p, 6)
        assert abs(one[0] - 3.0) < k["atol"] and abs(one[1] - 4.0) < k["atol"]
    else:
        raise AssertionError(f"unknown KAT kind {fn}")


def test_oracle_fixture_unchanged(oracle):
    """The oracle still reproduces its committed small-case results."""
    import gpv  # noqa: F401
    z = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    d = z["desc"].view(oracle.DESC_DTYPE)
    # the fixture holds the 192-byte records written before the texture field
    legacy = np.dtype([(k, oracle.RESULT_DTYPE.fields[k][0]) for k in oracle.RESULT_DTYPE.names
                       if k not in ("texture", "reserved")])
    res0 = z["result"].view(legacy)
    Cf = oracle.get_c(z["f"].astype(np.float64), 20)
    Cg = oracle.get_c(z["g"].astype(np.float64), 20)
    res = oracle.solve_batch(Cf, Cg, z["f"].shape, 20, d, max_norm=1e-5, max_iterations=15, eta=True)
    assert np.array_equal(res["iterations"], res0["iterations"])
    assert np.abs(res["p"] - res0["p"]).max() < 1e-12
    assert np.abs(res["eta_u"] - res0["eta_u"]).max() < 1e-12
