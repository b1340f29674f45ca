"""Sequence host logic on the CPU: seed guidance between pairs
(deformation_preconditioning and the particle mesh path it uses) in the
library (gpv.sequence) and in the oracle's restatement, against the
reference's own tests (src/particle.rs:2083-2124, :2621-2673;
src/sequence.rs:1228-1300)."""
import numpy as np
import pytest

Q = [0.1, -0.2, 0.02, 0.07, 0.03, -0.01, 0.004, 0.008, 0.005, 0.009, 0.006, -0.003]  # src/particle.rs:2621


def quad_warp(x, y):  # src/particle.rs:2624-2635
    q = Q
    return [q[0] + q[2] * x + q[4] * y + 0.5 * q[6] * x * x + q[8] * x * y + 0.5 * q[10] * y * y,
            q[1] + q[3] * x + q[5] * y + 0.5 * q[7] * x * x + q[9] * x * y + 0.5 * q[11] * y * y,
            q[2] + q[6] * x + q[8] * y, q[3] + q[7] * x + q[9] * y, q[4] + q[8] * x + q[10] * y,
            q[5] + q[9] * x + q[11] * y] + q[6:]


def element():  # src/particle.rs:2637-2642
    c = [[1.0, 2.0], [9.0, 3.5], [3.0, 8.0]]

    def mid(a, b):
        return [(c[a][0] + c[b][0]) / 2.0, (c[a][1] + c[b][1]) / 2.0]
    return [c[0], c[1], c[2], mid(0, 1), mid(1, 2), mid(2, 0)]


def _impls():
    import sequence_oracle as SO
    from gpv import sequence as GS
    return [("oracle", SO), ("library", GS)]


@pytest.mark.parametrize("which", ["oracle", "library"])
def test_warp_increment_every_slot(which):
    M = dict(_impls())[which]
    nodes = element()
    d = [quad_warp(x, y)[:2] for x, y in nodes]
    w = M.warp_increment([4.0, 4.0], np.array(nodes) if which == "library" else nodes, d, 2)  # :2646-2654
    assert np.abs(np.array(w) - quad_warp(4.0, 4.0)).max() < 1e-12
    n3 = nodes[:3]

    def lin(x, y):
        return [Q[0] + Q[2] * x + Q[4] * y, Q[1] + Q[3] * x + Q[5] * y]
    w1 = M.warp_increment([4.0, 4.0], np.array(n3) if which == "library" else n3, [lin(x, y) for x, y in n3], 1)
    want = lin(4.0, 4.0) + Q[2:6]  # :2657-2668
    assert np.abs(np.array(w1) - want).max() < 1e-12


@pytest.mark.parametrize("which", ["oracle", "library"])
def test_element_locator(which):
    M = dict(_impls())[which]
    nodes = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]
    els = [[0, 1, 2], [1, 3, 2]]  # src/particle.rs:2083-2124
    if which == "library":
        nodes, els = np.array(nodes), np.array(els)
    assert M.element_locator([1 / 3, 1 / 3], nodes, els) == (0, False)
    assert M.element_locator([2 / 3, 2 / 3], nodes, els) == (1, False)
    assert M.element_locator([0.2, 0.2], nodes, els) == (0, False)
    assert M.element_locator([0.8, 0.8], nodes, els) == (1, False)
    assert M.element_locator([2.0, 2.0], nodes, els) == (1, True)
    assert M.element_locator([5.0, 5.0], nodes, els)[1] is True


@pytest.mark.parametrize("which", ["oracle", "library"])
def test_deformation_preconditioning(which):
    M = dict(_impls())[which]
    nodes = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]
    els = [[0, 1, 2], [1, 3, 2]]  # unit_square_solution, src/sequence.rs:1231-1263
    g = [0.1, 0.02, 0.03, -0.05]
    d = [[g[0] * x + g[2] * y, g[1] * x + g[3] * y] for x, y in nodes]
    _, warp = M.deformation_preconditioning(nodes, els, d, [0.4, 0.3], 1, 1)  # :1266-1281
    assert np.abs(np.array(warp[2:6]) - g).max() < 1e-12
    disp, _ = M.deformation_preconditioning(nodes, els, [[0.3, -0.2]] * 4, [0.333, 0.333], 1, 1)  # :1284-1290
    assert abs(disp[0] - 0.3) < 1e-8 and abs(disp[1] + 0.2) < 1e-8
    _, warp = M.deformation_preconditioning(nodes, els, [[0.5, 0.0]] * 4, [0.333, 0.333], 1, 1)  # :1293-1299
    assert np.abs(np.array(warp[2:])).max() < 1e-8
    # order-2 subsets get the order-1 mesh's six terms and zeros
    _, w12 = M.deformation_preconditioning(nodes, els, d, [0.4, 0.3], 1, 2)
    assert len(w12) == 12 and np.all(np.array(w12[6:]) == 0.0)
    # strain terms are clipped to [-0.99, 0.99] (src/particle.rs:1426-1434)
    big = [[3.0 * x, 0.0] for x, y in nodes]
    _, wc = M.deformation_preconditioning(nodes, els, big, [0.4, 0.3], 1, 1)
    assert wc[2] == 0.99


def test_library_and_oracle_guidance_agree_on_a_quadratic_mesh():
    import sequence_oracle as SO
    from gpv import sequence as GS
    rng = np.random.default_rng(2)
    nodes = element()
    d = [quad_warp(x, y)[:2] for x, y in nodes]
    els = [[0, 1, 2, 3, 4, 5]]
    for _ in range(5):
        c = [float(v) for v in rng.uniform(2, 5, 2)]
        a = GS.deformation_preconditioning(np.array(nodes), np.array(els), np.array(d), c, 2, 2)
        b = SO.deformation_preconditioning(nodes, els, d, c, 2, 2)
        assert np.abs(a[0] - b[0]).max() < 1e-12 and np.abs(np.array(a[1]) - b[1]).max() < 1e-12
