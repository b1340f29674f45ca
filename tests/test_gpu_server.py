"""The request loop on the GPU: every request's result is the same whether it
is served alone or in a mix, and a session's frames match the frame tracker.

Requests are seeded speckle pairs of several sizes and pixel types under
random affine fields, with subsets of mixed radius and order and initial
warps from the field (a coarse upstream estimate) -- the shapes of the
serving stream at a reduced scale.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _request(rng, size, dtype, n, seed):
    import math

    import gpv
    from gpv import synth
    c = (size - 1) / 2.0
    th = math.radians(rng.uniform(-1, 1))
    e = rng.uniform(-0.02, 0.02, 2)
    a = ((1 + e[0]) * math.cos(th) - 1.0, -math.sin(th), math.sin(th), (1 + e[1]) * math.cos(th) - 1.0)
    fld = synth.make_field(xc=c, yc=c, t=tuple(rng.uniform(-5, 5, 2)), a=a)
    scale = 16.0 if dtype == np.uint16 else 1.0
    f, g = synth.pair(size, size, fld, seed, dtype=dtype, scale=scale)
    radius = rng.integers(15, 41, n).astype(np.int32)
    margin = 45 + 0.03 * size + 6
    xy = rng.uniform(margin, size - margin, (n, 2))
    order = rng.integers(1, 3, n).astype(np.int32)
    p0 = synth.seeded_p0(fld, xy, rng)
    return f, g, gpv.make_desc(xy, radius, order, p0)


def test_results_alone_equal_results_in_the_mix(gpv_mod, oracle):
    rng = np.random.default_rng(5)
    reqs = []
    for k, (size, dt) in enumerate([(256, np.uint8), (512, np.uint16), (1024, np.uint8), (256, np.uint16),
                                    (512, np.uint8), (1024, np.uint16), (256, np.uint8), (512, np.uint8)]):
        n = int(np.exp(rng.uniform(np.log(50), np.log(3000))))
        reqs.append(_request(rng, size, dt, n, 500 + k))
    srv = gpv_mod.Server(workers=3)
    tickets = [srv.submit(f, g, d) for f, g, d in reqs]
    mixed = [srv.wait(t, 120000).copy() for t in tickets]
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["p99_ms"] > 0
    srv.close()
    for k, ((f, g, d), got) in enumerate(zip(reqs, mixed)):
        ctx = gpv_mod.Context(0)
        alone = gpv_mod.solve_batch(gpv_mod.Image(image_gs=f, ctx=ctx), gpv_mod.Image(image_gs=g, ctx=ctx), d)
        assert alone.tobytes() == got.tobytes()
        assert np.mean(got["converged"]) > 0.95
        # served results against the FP64 oracle on a sample of each request
        # (the mixed-precision bar: 1e-3 px, 1e-5 strain, identical flags)
        pick = np.random.default_rng(k).choice(len(d), min(len(d), 60), replace=False)
        Cf = oracle.get_c(f.astype(np.float64), 20)
        Cg = oracle.get_c(g.astype(np.float64), 20)
        ref = oracle.solve_batch(Cf, Cg, f.shape, 20, d[pick], max_norm=1e-5, max_iterations=50, tolerance=0.75)
        sub = got[pick]
        assert np.array_equal(sub["status"], ref["status"])
        assert np.array_equal(sub["converged"], ref["converged"])
        assert np.array_equal(sub["quality_ok"], ref["quality_ok"])
        ok = ref["status"] == 0
        assert np.abs(sub["p"][ok, :2] - ref["p"][ok, :2]).max() <= 1e-3
        assert np.abs(sub["p"][ok, 2:6] - ref["p"][ok, 2:6]).max() <= 1e-5


def test_per_subset_blocks_give_the_persistent_bytes(gpv_mod):
    """One block per subset (any stream priority) returns the bytes of the
    persistent grid on a batch with every order and radius class, invalid
    subsets and the eta diagnostic."""
    rng = np.random.default_rng(17)
    f, g, d = _request(rng, 1024, np.uint8, 3000, 77)
    d["radius"] = rng.integers(8, 61, len(d))
    d["order"] = rng.integers(0, 3, len(d))
    d["radius"][:3] = 0
    d["order"][3:6] = 5
    got = {}
    for name, kw in (("persistent", {}), ("per_subset", dict(per_subset_blocks=True)),
                     ("priority", dict(per_subset_blocks=True, high_priority=True))):
        ctx = gpv_mod.Context(0, **kw)
        F, G = gpv_mod.Image(image_gs=f, ctx=ctx), gpv_mod.Image(image_gs=g, ctx=ctx)
        got[name] = gpv_mod.solve_batch(F, G, d, eta=True).copy()
        if name == "per_subset":  # a second batch on the same context reuses the freed slots
            again = gpv_mod.solve_batch(F, G, d[::-1].copy(), eta=True)
            assert again[::-1].tobytes() == got[name].tobytes()
    assert got["per_subset"].tobytes() == got["persistent"].tobytes()
    assert got["priority"].tobytes() == got["persistent"].tobytes()
    assert np.all(got["persistent"]["status"][:6] == 8)
    assert np.mean(got["persistent"]["converged"][6:]) > 0.9


def test_priority_lane_results_equal_results_alone(gpv_mod):
    rng = np.random.default_rng(23)
    reqs = []
    for k, (size, dt) in enumerate([(1024, np.uint8), (256, np.uint8), (512, np.uint16), (256, np.uint16),
                                    (1024, np.uint16), (512, np.uint8)]):
        n = [4000, 80, 300, 120, 3500, 200][k]
        reqs.append(_request(rng, size, dt, n, 700 + k))
    srv = gpv_mod.Server(workers=4, priority_workers=2, priority_subsets=500)
    tickets = [srv.submit(f, g, d) for f, g, d in reqs]
    mixed = [srv.wait(t, 120000).copy() for t in tickets]
    assert srv.stats()["failed"] == 0
    srv.close()
    for (f, g, d), got in zip(reqs, mixed):
        ctx = gpv_mod.Context(0)
        alone = gpv_mod.solve_batch(gpv_mod.Image(image_gs=f, ctx=ctx), gpv_mod.Image(image_gs=g, ctx=ctx), d)
        assert alone.tobytes() == got.tobytes()


def test_rigid_texture_requests_equal_solves_alone(gpv_mod):
    """A served request with the rigid texture (the worker builds the
    reference's grain maps) returns the bytes of the same solve alone."""
    rng = np.random.default_rng(31)
    reqs = [_request(rng, 512, np.uint8, 300, 810), _request(rng, 256, np.uint16, 120, 811)]
    srv = gpv_mod.Server(workers=2)
    got = [srv.wait(srv.submit(f, g, d, texture="rigid"), 120000).copy() for f, g, d in reqs]
    srv.close()
    for (f, g, d), r in zip(reqs, got):
        ctx = gpv_mod.Context(0)
        alone = gpv_mod.solve_batch(gpv_mod.Image(image_gs=f, ctx=ctx), gpv_mod.Image(image_gs=g, ctx=ctx), d,
                                    texture="rigid")
        assert alone.tobytes() == r.tobytes()
        assert np.all(r["texture"] == 1)


def test_session_frames_match_the_frame_tracker(gpv_mod):
    from gpv import synth
    Ws = [synth.workload(4, scale_down=4, seed_frame=k) for k in (0, 6, 12, 18, 24)]
    W0 = Ws[0]
    desc = gpv_mod.make_desc(W0["coords"], W0["radius"], W0["order"], W0["p0"])
    srv = gpv_mod.Server(workers=2)
    served = []
    for k, W in enumerate(Ws):
        t = srv.submit(W0["f"] if k == 0 else None, W["g"], desc, session=7, reuse_reference=k > 0,
                       seed_from_previous=k > 0)
        served.append(srv.wait(t, 60000).copy())
    srv.close()
    ctx = gpv_mod.Context(0)  # untuned, like the server's worker contexts
    F = gpv_mod.Image(image_gs=W0["f"], ctx=ctx)
    G = gpv_mod.Image(image_gs=W0["f"], ctx=ctx)
    seq = gpv_mod.SubsetSequence(F, G, desc, np.uint8)
    for W, got in zip(Ws, served):
        assert seq.frame(W["g"]).tobytes() == got.tobytes()
    seq.close()


def test_poisson_stream_reports_latency(gpv_mod):
    """A short Poisson stream (100 req/s for 1 s) of 256^2..1024^2 requests."""
    import time
    rng = np.random.default_rng(9)
    pool = [_request(rng, s, dt, 2000, 900 + k) for k, (s, dt) in
            enumerate([(256, np.uint8), (512, np.uint8), (1024, np.uint16)])]
    srv = gpv_mod.Server(workers=4)
    t0 = time.perf_counter()
    tickets = []
    t_next = 0.0
    while t_next < 1.0:
        while time.perf_counter() - t0 < t_next:
            time.sleep(0.0005)
        f, g, d = pool[rng.integers(len(pool))]
        n = int(np.exp(rng.uniform(np.log(100), np.log(2000))))
        tickets.append(srv.submit(f, g, d[:n]))
        t_next += rng.exponential(1 / 100.0)
    for t in tickets:
        srv.wait(t, 120000)
    st = srv.stats()
    assert st["completed"] == len(tickets) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] < 5000
    srv.close()
