"""A device batch captured as a CUDA graph (gpv_batch_graph_*).

The uneven batch of the shear-band workload (radii 15..60, first and second
order mixed) is solved once through gpv_solve_batch_device and captured;
replays must return the same bytes as eager calls on the same device
buffers, also after the target image is re-prefiltered in place, and a
replay after the context's workspace moved must be refused.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(gpv_mod, scale):
    import torch
    from gpv import synth
    W = synth.workload(3, scale_down=scale)
    ctx = gpv_mod.Context(0)
    F = gpv_mod.Image(image_gs=W["f"], border=20, ctx=ctx)
    G = gpv_mod.Image(image_gs=W["g"], border=20, ctx=ctx)
    d = gpv_mod.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    ctx.reserve(len(d), int(d["radius"].max()), 50)
    d_dev = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    order = np.argsort(-(3 * d["radius"].astype(np.int64) + d["order"]), kind="stable").astype(np.int32)
    o_dev = torch.from_numpy(order).cuda()
    return W, ctx, F, G, d, d_dev, o_dev


def _eager(gpv_mod, ctx, F, G, d_dev, o_dev, n, prm, out):
    import torch
    from gpv import _lib
    _lib.check(_lib.lib().gpv_solve_batch_device(ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()),
                                                 ct.c_void_p(o_dev.data_ptr()), n, ct.byref(prm),
                                                 ct.c_void_p(out.data_ptr()), None), "solve")
    torch.cuda.synchronize()
    return out.cpu().numpy().tobytes()


def test_graph_replays_equal_eager_solves(gpv_mod):
    import torch
    from gpv import _lib
    W, ctx, F, G, d, d_dev, o_dev = _setup(gpv_mod, 4)
    n = len(d)
    prm = gpv_mod._params(1e-5, 50, 0.75, False, gpv_mod.PREC_MIXED, None, None)
    out = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    eager = _eager(gpv_mod, ctx, F, G, d_dev, o_dev, n, prm, out)
    bg = ct.c_void_p()
    _lib.check(_lib.lib().gpv_batch_graph_create(ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()),
                                                 ct.c_void_p(o_dev.data_ptr()), n, ct.byref(prm),
                                                 ct.c_void_p(out.data_ptr()), ct.byref(bg)), "graph create")
    try:
        for _ in range(2):
            out.zero_()
            _lib.check(_lib.lib().gpv_batch_graph_launch(bg, None), "graph launch")
            torch.cuda.synchronize()
            assert out.cpu().numpy().tobytes() == eager
        res = np.frombuffer(eager, dtype=_lib.RESULT_DTYPE)
        assert np.mean(res["converged"]) > 0.95 and set(np.unique(d["order"])) == {1, 2}
        # a new target, prefiltered in place: the replay follows the buffers' contents
        G.update(W["f"])
        _lib.check(_lib.lib().gpv_batch_graph_launch(bg, None), "graph launch")
        torch.cuda.synchronize()
        replay = out.cpu().numpy().tobytes()
        assert replay == _eager(gpv_mod, ctx, F, G, d_dev, o_dev, n, prm, out)
        moved = np.frombuffer(replay, dtype=_lib.RESULT_DTYPE)
        assert np.abs(moved["p"][moved["converged"] == 1, :2]).max() < 0.05  # f against itself
        # a larger radius than reserved grows the context's tables: the graph is refused
        gpv_mod.solve_batch(F, G, gpv_mod.make_desc([[256.0, 256.0]], int(d["radius"].max()) + 40, 1))
        assert _lib.lib().gpv_batch_graph_launch(bg, None) == -1
    finally:
        _lib.lib().gpv_batch_graph_destroy(bg)
