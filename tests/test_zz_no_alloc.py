"""The allocation-free solve entry point (gpv_solve_batch_noalloc).

It exists for callers that may not allocate device memory while solving --
their device memory is owned by another framework's pooling allocator, or
their loop cannot take the device-wide synchronisation an allocation implies.
All its working memory is one static device array; these tests call it
through the C ABI and compare it with the regular device entry point
(gpv_solve_batch_device) on the same device inputs, twice in a row (the
second call reuses the array left by the first), check both calls against
the FP64 oracle on the same pixels, and check that device memory does not
move during a call.  Same tolerance as the other mixed-precision parity
tests: displacement 1e-3 px, gradient terms 1e-5, identical convergence /
quality flags (iteration counts within one on at most 2% of subsets against
the oracle).
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_batch(gpv_mod, W, max_radius):
    import torch
    from gpv import _lib
    ctx = gpv_mod.Context(0)
    F = gpv_mod.Image(image_gs=W["f"], border=20, ctx=ctx)
    G = gpv_mod.Image(image_gs=W["g"], border=20, ctx=ctx)
    d = gpv_mod.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    d_dev = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    ctx.reserve(len(d), max_radius, 50)
    return ctx, F, G, d, d_dev


def _run(fn, ctx, F, G, d_dev, n, prm, extra, stream, out):
    args = [ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr())]
    from gpv import _lib
    if fn == "noalloc":
        rc = _lib.lib().gpv_solve_batch_noalloc(*args, n, extra, ct.byref(prm), ct.c_void_p(out.data_ptr()),
                                                ct.c_void_p(stream.cuda_stream))
    else:
        rc = _lib.lib().gpv_solve_batch_device(*args, None, n, ct.byref(prm), ct.c_void_p(out.data_ptr()),
                                               ct.c_void_p(stream.cuda_stream))
    _lib.check(rc, fn)
    stream.synchronize()
    return np.frombuffer(out.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()


def _same(a, b):
    assert np.array_equal(a["status"], b["status"])
    assert np.array_equal(a["converged"], b["converged"])
    assert np.array_equal(a["quality_ok"], b["quality_ok"])
    ok = a["status"] == 0
    assert np.abs(a["p"][ok, :2] - b["p"][ok, :2]).max() <= 1e-3
    assert np.abs(a["p"][ok, 2:6] - b["p"][ok, 2:6]).max() <= 1e-5
    assert np.abs(a["c_zncc"][ok] - b["c_zncc"][ok]).max() < 1e-5


def _oracle_same(res, ref):
    assert np.array_equal(res["status"], ref["status"])
    assert np.array_equal(res["n_px"], ref["n_px"])
    assert np.array_equal(res["converged"], ref["converged"])
    assert np.array_equal(res["quality_ok"], ref["quality_ok"])
    ok = ref["status"] == 0
    assert np.abs(res["p"][ok, :2] - ref["p"][ok, :2]).max() <= 1e-3
    assert np.abs(res["p"][ok, 2:6] - ref["p"][ok, 2:6]).max() <= 1e-5
    assert np.abs(res["c_zncc"][ok] - ref["c_zncc"][ok]).max() < 1e-5
    it_diff = np.abs(res["iterations"].astype(int) - ref["iterations"])
    assert it_diff.max() <= 1 and (it_diff > 0).sum() <= max(1, int(np.ceil(0.02 * len(it_diff))))


@pytest.mark.parametrize("config,scale", [(1, 4), (3, 8)])
def test_noalloc_matches_device_entry_point(gpv_mod, oracle, config, scale):
    import torch
    from gpv import _lib, synth
    W = synth.workload(config, scale_down=scale)
    if config == 3:  # keep radii within the static limit
        keep = W["radius"] <= 32
        for k in ("coords", "radius", "order", "p0", "truth_uv"):
            W[k] = W[k][keep]
    ctx, F, G, d, d_dev = _device_batch(gpv_mod, W, 32)
    n = len(d)
    prm = _lib.SolveParams(max_norm=1e-5, tolerance=0.75, max_iterations=50, flags=0, precision=_lib.PREC_MIXED,
                           reserved=0, mask=None, history=None)
    s = torch.cuda.Stream()
    out = torch.zeros(n * 200, dtype=torch.uint8, device="cuda")  # caller-owned output
    ref = _run("device", ctx, F, G, d_dev, n, prm, None, s, out)
    first = _run("noalloc", ctx, F, G, d_dev, n, prm, 32, s, out)   # first call does the one-time set-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    second = _run("noalloc", ctx, F, G, d_dev, n, prm, 32, s, out)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, "device memory changed during a no-allocation call"
    _same(first, ref)
    _same(second, ref)
    assert np.array_equal(first["iterations"], second["iterations"])
    assert np.array_equal(first["p"], second["p"])
    # and against the FP64 oracle on the same pixels
    Cf = oracle.get_c(W["f"].astype(np.float64), 20)
    Cg = oracle.get_c(W["g"].astype(np.float64), 20)
    want = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, max_iterations=50, tolerance=0.75)
    _oracle_same(first, want)
    _oracle_same(second, want)


def test_noalloc_limits(gpv_mod):
    import torch
    from gpv import _lib, synth
    W = synth.workload(1, scale_down=8)
    ctx, F, G, d, d_dev = _device_batch(gpv_mod, W, 32)
    prm = _lib.SolveParams(max_norm=1e-5, tolerance=0.75, max_iterations=50, flags=0, precision=_lib.PREC_MIXED,
                           reserved=0, mask=None, history=None)
    s = torch.cuda.Stream()
    out = torch.zeros(len(d) * 200, dtype=torch.uint8, device="cuda")
    rc = _lib.lib().gpv_solve_batch_noalloc(ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), len(d), 40,
                                            ct.byref(prm), ct.c_void_p(out.data_ptr()), ct.c_void_p(s.cuda_stream))
    assert rc == -1 and "max_radius 40" in _lib.last_error()
    # subsets above the stated max_radius come back flagged, not solved
    res = _run("noalloc", ctx, F, G, d_dev, len(d), prm, 20, s, out)
    assert np.all(res["status"] == 8)
