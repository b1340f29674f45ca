"""gpv.Sequence (Sequence::solve over GPU mesh solves) against the oracle's
restatement of the pair loop over the FP64 oracle: the same pairs solved
from the same references with the same seeds, reference updates and
override log, and per pair the mixed-precision parity bar (same flags,
displacement within 1e-3 px)."""
import numpy as np
import pytest

import mesh_cases as MC

pytestmark = pytest.mark.gpu


def _oracle(oracle, frames, nodes, el, **kw):
    import sequence_oracle as SO
    Cs = [oracle.get_c(np.asarray(f, dtype=np.float64), 15) for f in frames]

    def solver_for(Cf, Cg):
        def s(desc, tol):
            return oracle.solve_batch(Cf, Cg, frames[0].shape, 15, desc, max_norm=1e-5, tolerance=tol)
        return s
    return SO.solve_sequence(Cs, frames[0].shape, 15, nodes, el, solver_for, desc_dtype=oracle.DESC_DTYPE, **kw)


def _compare(got, ref):
    assert len(got["pairs"]) == len(ref["pairs"])
    assert got["reference_updates"] == ref["reference_updates"]
    assert got["override_log"] == ref["override_log"]
    assert got["unsolvable"] == ref["unsolvable"] and got["all_converged"] == ref["all_converged"]
    for a, b in zip(got["pairs"], ref["pairs"]):
        assert (a["f_index"], a["g_index"]) == (b["f_index"], b["g_index"])
        assert np.abs(np.array(a["seed_coord"]) - b["seed_coord"]).max() < 1e-3
        rb = np.array(b["sol"]["results"])
        ra = a["results"]
        assert np.array_equal(ra["quality_ok"], [x["quality_ok"] for x in rb])
        ok = ra["status"] == 0
        pb = np.array([x["p"] for x in rb])
        assert np.abs(ra["p"][ok, :2] - pb[ok, :2]).max() <= 1e-3


@pytest.mark.parametrize("sequential", [False, True])
def test_shift_sequence_matches_oracle(gpv_mod, oracle, sequential):
    f0 = MC.texture(100)
    frames = [f0] + [MC.shift_uniform(f0, 0.6 * k) for k in (1, 2, 3)]
    nodes, el = MC.grid_mesh()
    kw = dict(radius=8, seed_coord=(50.0, 50.0), seed_tolerance=0.5, tolerance=0.5, guide=True,
              sequential=sequential)
    ref = _oracle(oracle, frames, nodes, el, **kw)
    seq = gpv_mod.sequence.Sequence(frames, nodes, el, border=15)
    got = seq.solve(8, seed_coord=(50.0, 50.0), seed_tolerance=0.5, tolerance=0.5, guide=True, sequential=sequential)
    _compare(got, ref)
    assert got["all_converged"]
    last = got["pairs"][-1]["results"]["p"][:, 0]
    assert np.abs(last - (0.6 if sequential else 1.8)).max() < 0.05


@pytest.mark.parametrize("override", [False, True])
def test_reference_update_fallback(gpv_mod, oracle, override):
    """Frame 2 shares little with frame 0 and more with frame 1: the pair
    (0, 2) fails the quality gate and the reference steps to frame 1; the
    pair (1, 2) then fails too and curtails the sequence, unless the
    override retry (tolerance 0, no gate) lets it through and logs it."""
    a = MC.texture(100)
    b = np.rot90(MC.texture(100)).copy()
    frames = [a, 0.75 * a + 0.25 * b, 0.1 * a + 0.9 * b]
    nodes, el = MC.grid_mesh(n_side=7, start=25.0, step=8.33)
    kw = dict(radius=10, seed_coord=(50.0, 50.0), seed_tolerance=0.3, tolerance=0.5, guide=False, override=override)
    ref = _oracle(oracle, frames, nodes, el, **kw)
    seq = gpv_mod.sequence.Sequence(frames, nodes, el, border=15)
    got = seq.solve(10, seed_coord=(50.0, 50.0), seed_tolerance=0.3, tolerance=0.5, guide=False, override=override)
    _compare(got, ref)
    if override:
        assert [(p["f_index"], p["g_index"]) for p in got["pairs"]] == [(0, 1), (1, 2)]
        assert got["reference_updates"] == [False, True] and got["override_log"] == [2]
    else:
        assert [(p["f_index"], p["g_index"]) for p in got["pairs"]] == [(0, 1)] and got["unsolvable"]


@pytest.mark.parametrize("sequential", [False, True])
def test_rigid_texture_sequence_matches_oracle(gpv_mod, oracle, sequential):
    """Sequence.solve(texture="rigid") on rigid blobs under growing shear: each
    pair fits the rigid template of its reference frame (grain maps follow
    the images through in-place updates and the sequential swap), against the
    oracle's loop over its rigid solve."""
    import sequence_oracle as SO
    import texture_cases as TC
    frames = [TC.shear_pair(0.0)[0]] + [TC.shear_pair(g)[1] for g in (0.02, 0.04)]
    xs = np.linspace(60.0, 140.0, 5)
    nodes = np.array([[x, y] for y in xs for x in xs])
    el = []
    for j in range(4):
        for i in range(4):
            a, b, c, e = j * 5 + i, j * 5 + i + 1, (j + 1) * 5 + i, (j + 1) * 5 + i + 1
            el += [[a, b, e], [a, e, c]]
    el = np.array(el)
    Cs = [oracle.get_c(f, 15) for f in frames]
    grains = [oracle.grain(f) for f in frames]

    def solver_for(Cf, Cg):
        k = next(i for i, c in enumerate(Cs) if c is Cf)
        def s(desc, tol):
            return oracle.solve_batch(Cf, Cg, frames[0].shape, 15, desc, max_norm=1e-5, tolerance=tol,
                                      grain=grains[k])
        return s
    kw = dict(radius=15, seed_coord=(100.0, 100.0), seed_tolerance=0.5, tolerance=0.5, guide=True,
              sequential=sequential)
    ref = SO.solve_sequence(Cs, frames[0].shape, 15, nodes, el, solver_for, desc_dtype=oracle.DESC_DTYPE, **kw)
    seq = gpv_mod.sequence.Sequence(frames, nodes, el, border=15)
    got = seq.solve(15, seed_coord=(100.0, 100.0), seed_tolerance=0.5, tolerance=0.5, guide=True,
                    sequential=sequential, texture="rigid")
    _compare(got, ref)
    assert got["all_converged"]
    for pr in got["pairs"]:
        assert np.all(pr["results"]["texture"] == 1)


def test_rigid_texture_from_colour_pixels(gpv_mod, oracle):
    """Grain maps of a colour-ingested reference come from its device-made
    grey image: the same maps as from those grey pixels directly."""
    import texture_cases as TC
    f, _ = TC.shear_pair(0.0)
    grey = np.clip(np.round(f), 0, 255).astype(np.uint8)
    rgb = np.repeat(grey[:, :, None], 3, axis=2)
    Fc = gpv_mod.Image(image_rgb=rgb, border=8, grain=True)
    Fg = gpv_mod.Image(image_gs=gpv_mod.Image(image_rgb=rgb, border=8).image_gs, border=8, grain=True)
    a, b = Fc.grain(maps=True), Fg.grain(maps=True)
    assert a["built"] and np.array_equal(a["maps"], b["maps"]) and a["s2"] == b["s2"]
