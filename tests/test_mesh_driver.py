"""The library's mesh driver (gpv_mesh_drive) against the oracle's restatement.

On the CPU the C++ driver runs over the FP64 oracle's batch solve (a solver
callback), and oracle/mesh_oracle.py -- the restatement of the reference's
propagation -- runs over the same solver: seed node, rounds, every flag and
every warp must agree exactly.  Also the reference's own mesh-level tests
(src/mesh.rs:3014-3203): progress + cancellation, layer-RG determinism,
layer-RG within Tier C of serial RG, proper colouring.
"""
import numpy as np
import pytest

import mesh_cases as MC

RADIUS = 6


@pytest.fixture(scope="module")
def band_images():
    f = MC.texture(100)
    return f, MC.shift_band(f, 50, 1.5, -1.5)


@pytest.fixture(scope="module")
def uniform_images():
    f = MC.texture(100)
    return f, MC.shift_uniform(f, 1.5)


def _both(oracle, imgs, nodes, elements, **kw):
    import gpv
    import mesh_oracle as M
    solver = MC.oracle_solver(oracle, imgs[0], imgs[1], 15)
    ours = gpv.mesh_drive(nodes, elements, solver, **kw)
    kw2 = dict(kw)
    kw2["batch_factor"] = kw2.pop("layer_rg_batch_factor", 4)
    kw2["root_rel_eps"] = kw2.pop("layer_rg_root_rel_eps", 0.02)
    kw2["max_workers"] = kw2.pop("layer_rg_max_workers", 1)
    ref = M.solve_mesh(nodes, elements, solver, desc_dtype=oracle.DESC_DTYPE, **kw2)
    return ours, ref


def _assert_same(ours, ref):
    assert ours["seed_node"] == ref["seed_node"]
    assert np.array_equal(ours["rounds"], ref["rounds"])
    r = ours["results"]
    for k in ("status", "quality_ok", "converged", "iterations"):
        assert np.array_equal(r[k], [x[k] for x in ref["results"]]), k
    p_ref = np.array([x["p"] for x in ref["results"]])
    assert np.array_equal(r["p"], p_ref)
    assert np.array_equal(r["c_zncc"], [x["c_zncc"] for x in ref["results"]])
    for k in ("batches", "solves", "retries", "rounds", "n_bad", "n_unreached"):
        assert ours["stats"][k] == ref["stats"][k], k


CASES = [
    dict(preconditioning="RG"),
    dict(preconditioning="layer-RG", layer_rg_batch_factor=4, layer_rg_root_rel_eps=0.02, layer_rg_max_workers=2),
    dict(preconditioning="layer-RG", layer_rg_batch_factor=1, layer_rg_root_rel_eps=0.0, layer_rg_max_workers=1),
]


@pytest.mark.parametrize("case", CASES, ids=["RG", "layerRG_bf4_w2", "layerRG_bf1"])
def test_driver_matches_oracle_restatement_band(oracle, band_images, case):
    nodes, el = MC.grid_mesh()
    ours, ref = _both(oracle, band_images, nodes, el, radius=RADIUS, seed_coord=(50.0, 30.0), seed_tolerance=0.5,
                      tolerance=0.5, subset_order=1, **case)
    _assert_same(ours, ref)
    assert ours["stats"]["n_unreached"] == 0


@pytest.mark.parametrize("subset_order", [1, 2])
@pytest.mark.parametrize("prec", ["RG", "layer-RG"])
def test_driver_matches_oracle_restatement_order2_mesh(oracle, uniform_images, subset_order, prec):
    nodes, el = MC.to_order2(*MC.grid_mesh(n_side=6, step=12.0))
    ours, ref = _both(oracle, uniform_images, nodes, el, radius=8, seed_coord=(50.0, 50.0), seed_tolerance=0.5,
                      tolerance=0.5, subset_order=subset_order, preconditioning=prec, layer_rg_max_workers=2,
                      seed_warp=[1.4, 0.0])
    _assert_same(ours, ref)
    if subset_order == 2:  # the quadratic fit (>= 6 trusted neighbours) is exercised
        assert ours["stats"]["solves"] > 0


def test_rounds_are_a_proper_colouring(oracle, band_images):
    """No two nodes solved in one batch share an element (src/mesh.rs:3177-3203)."""
    import gpv
    nodes, el = MC.grid_mesh()
    solver = MC.oracle_solver(oracle, *band_images, 15)
    out = gpv.mesh_drive(nodes, el, solver, radius=RADIUS, seed_coord=(50.0, 30.0), seed_tolerance=0.5,
                         tolerance=0.5, preconditioning="layer-RG", layer_rg_max_workers=4)
    rounds = out["rounds"]
    for row in el:
        for a in row:
            for b in row:
                if a != b:
                    assert rounds[a] != rounds[b]
    # every solver call but the seed's and the retries covers one round
    assert out["stats"]["rounds"] == rounds.max() + 1


def test_layer_rg_is_deterministic(oracle, uniform_images):
    """src/mesh.rs:3140-3156: byte-identical p / c_zncc / iterations run to run."""
    import gpv
    nodes, el = MC.grid_mesh()
    solver = MC.oracle_solver(oracle, *uniform_images, 15)
    runs = [gpv.mesh_drive(nodes, el, solver, radius=8, seed_coord=(50.0, 50.0), seed_tolerance=0.5, tolerance=0.5,
                           preconditioning="layer-RG", layer_rg_max_workers=2)["results"] for _ in range(3)]
    for r in runs[1:]:
        assert r.tobytes() == runs[0].tobytes()


@pytest.mark.parametrize("bf,eps", [(4, 0.02), (1, 0.0)])
def test_layer_rg_within_tier_c_of_rg(oracle, uniform_images, bf, eps):
    """src/mesh.rs:3113-3136, 3159-3174: same seed node and quality flags,
    displacement within 1e-5 * max(|u|, |v|, 1), c_zncc within 1e-5."""
    import gpv
    nodes, el = MC.grid_mesh()
    solver = MC.oracle_solver(oracle, *uniform_images, 15)
    kw = dict(radius=8, seed_coord=(50.0, 50.0), seed_tolerance=0.5, tolerance=0.5)
    a = gpv.mesh_drive(nodes, el, solver, preconditioning="RG", **kw)
    b = gpv.mesh_drive(nodes, el, solver, preconditioning="layer-RG", layer_rg_batch_factor=bf,
                       layer_rg_root_rel_eps=eps, layer_rg_max_workers=2, **kw)
    assert a["seed_node"] == b["seed_node"]
    ra, rb = a["results"], b["results"]
    assert np.array_equal(ra["quality_ok"], rb["quality_ok"])
    scale = np.maximum(np.abs(ra["p"][:, :2]).max(axis=1), 1.0)
    assert np.all(np.abs(ra["p"][:, :2] - rb["p"][:, :2]).max(axis=1) <= 1e-5 * scale)
    assert np.abs(np.fmax(ra["c_zncc"], 0) - np.fmax(rb["c_zncc"], 0)).max() <= 1e-5
    # the uniform 1.5 px shift is recovered everywhere
    assert np.abs(ra["p"][:, 0] - 1.5).max() < 0.05 and np.abs(ra["p"][:, 1]).max() < 0.05


def test_progress_reports_every_node_and_cancels(oracle, band_images):
    """src/mesh.rs:3014-3035: n node reports when not cancelled; cancelling
    after 5 stops with Cancelled after exactly 5 reports."""
    import gpv
    nodes, el = MC.grid_mesh()
    solver = MC.oracle_solver(oracle, *band_images, 15)
    kw = dict(radius=RADIUS, seed_coord=(50.0, 30.0), seed_tolerance=0.5, tolerance=0.5)
    seen = []
    full = gpv.mesh_drive(nodes, el, solver, progress=lambda d, t: seen.append((d, t)) and False, **kw)
    assert len(seen) == len(nodes) and seen[-1] == (len(nodes), len(nodes))
    plain = gpv.mesh_drive(nodes, el, solver, **kw)
    assert np.array_equal(full["results"]["p"], plain["results"]["p"])
    count = []

    def stop_after_5(done, total):
        count.append(done)
        return done >= 5
    with pytest.raises(gpv.Cancelled):
        gpv.mesh_drive(nodes, el, solver, progress=stop_after_5, **kw)
    assert count == [1, 2, 3, 4, 5]


def test_featureless_node_fails_the_mesh(oracle):
    """A node whose subset Subset::new rejects ends the solve with an error
    naming the node (src/mesh.rs:575-592 `?`)."""
    import gpv
    f = MC.texture(100)
    f[:, :40] = 100.0  # flat left part: nodes at x <= 27.5 see no texture
    g = f.copy()
    nodes, el = MC.grid_mesh()
    solver = MC.oracle_solver(oracle, f, g, 15)
    with pytest.raises(gpv.GpvError, match="mesh node [0-9]+: featureless subset"):
        gpv.mesh_drive(nodes, el, solver, radius=RADIUS, seed_coord=(60.0, 60.0), tolerance=0.5)


def test_unreached_nodes_are_reported(oracle, uniform_images):
    """Nodes outside the seed's connected component are never solved."""
    import gpv
    nodes, el = MC.grid_mesh(n_side=4, step=15.0)
    nodes = np.vstack([nodes, [[70.0, 70.0], [75.0, 70.0], [70.0, 75.0]]])
    el = np.vstack([el, [[16, 17, 18]]])
    solver = MC.oracle_solver(oracle, *uniform_images, 15)
    out = gpv.mesh_drive(nodes, el, solver, radius=8, seed_coord=(20.0, 20.0), tolerance=0.5, seed_tolerance=0.5)
    assert out["stats"]["n_unreached"] == 3
    assert np.all(out["rounds"][16:] == -1) and np.all(out["results"]["status"][16:] == 8)
    assert np.all(out["rounds"][:16] >= 0)


def test_driver_argument_checks(gpv_mod):
    import gpv
    nodes, el = MC.grid_mesh(n_side=3)

    def never(desc, tol):
        raise AssertionError("solver must not be called")
    kw = dict(radius=6, seed_coord=(20.0, 20.0))
    with pytest.raises(gpv.GpvError, match="outside"):
        gpv.mesh_drive(nodes, el + 100, never, **kw)
    with pytest.raises(ValueError):
        gpv.mesh_drive(nodes, el[:, :2], never, **kw)
    with pytest.raises(ValueError):
        gpv.mesh_drive(nodes, el, never, subset_order=0, **kw)
    with pytest.raises(ValueError):
        gpv.mesh_drive(nodes, el, never, preconditioning="BFS", **kw)
    with pytest.raises(gpv.GpvError, match="radius"):
        gpv.mesh_drive(nodes, el, never, radius=0, seed_coord=(20.0, 20.0))
