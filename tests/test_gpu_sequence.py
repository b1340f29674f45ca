"""Frame-to-frame tracking (gpv_sequence_*) against the oracle's frame loop.

The tracked workload at 1/4 scale: 512^2 u8 speckle under simple shear that
grows frame by frame, 1,250 subsets of radius 25, reference fixed at frame 0.
The oracle loop restates the tracker's rule -- every subset starts from its
own last converged warp (src/sequence.rs:624-968 is the per-pair loop this
replaces) -- over the FP64 oracle.  Mixed precision: displacement within
1e-3 px, gradients within 1e-5, identical flags, every frame.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FRAMES = [0, 6, 12, 18, 24, 30, 36, 42]


@pytest.fixture(scope="module")
def frames():
    from gpv import synth
    W = [synth.workload(4, scale_down=4, seed_frame=k) for k in FRAMES]
    return W


def _oracle_frames(oracle, frames):
    W0 = frames[0]
    d = np.zeros(len(W0["coords"]), oracle.DESC_DTYPE)
    d["coord"], d["radius"], d["order"] = W0["coords"], W0["radius"], W0["order"]
    Cf = oracle.get_c(W0["f"].astype(np.float64), 20)
    out = []
    for W in frames:
        Cg = oracle.get_c(W["g"].astype(np.float64), 20)
        r = oracle.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, max_iterations=50)
        ok = (r["status"] == 0) & (r["converged"] == 1)
        d["p0"][ok] = r["p"][ok]
        out.append(r)
    return out


def _gpu_frames(gpv, frames, graph=True, device=False):
    import torch
    W0 = frames[0]
    ctx = gpv.Context(0)
    F = gpv.Image(image_gs=W0["f"], border=20, ctx=ctx)
    G = gpv.Image(image_gs=W0["f"], border=20, ctx=ctx)
    desc = gpv.make_desc(W0["coords"], W0["radius"], W0["order"], W0["p0"])
    seq = gpv.SubsetSequence(F, G, desc, np.uint8, graph=graph)
    out = []
    for W in frames:
        if device:
            t = torch.from_numpy(W["g"].copy()).cuda()
            torch.cuda.synchronize()
            out.append(seq.frame(device_ptr=t.data_ptr()))
        else:
            out.append(seq.frame(W["g"]))
    assert seq.frames == len(frames)
    seq.close()
    return out


def test_tracking_matches_oracle_frame_loop(gpv_mod, oracle, frames):
    ref = _oracle_frames(oracle, frames)
    got = _gpu_frames(gpv_mod, frames)
    for k, (a, b) in enumerate(zip(got, ref)):
        assert np.array_equal(a["status"], b["status"]), k
        assert np.array_equal(a["converged"], b["converged"]), k
        assert np.array_equal(a["quality_ok"], b["quality_ok"]), k
        ok = a["status"] == 0
        assert np.abs(a["p"][ok, :2] - b["p"][ok, :2]).max() <= 1e-3, k
        assert np.abs(a["p"][ok, 2:6] - b["p"][ok, 2:6]).max() <= 1e-5, k
    # the last frame recovers the imposed shear
    from gpv import synth
    W = frames[-1]
    truth = synth.displacement(W["field"], W["coords"])
    last = got[-1]
    good = last["converged"] == 1
    assert good.mean() > 0.99
    assert np.abs(last["p"][good, :2] - truth[good]).max() < 0.05


def test_graph_replay_equals_eager_launches(gpv_mod, frames):
    a = _gpu_frames(gpv_mod, frames, graph=True)
    b = _gpu_frames(gpv_mod, frames, graph=False)
    for x, y in zip(a, b):
        assert x.tobytes() == y.tobytes()


def test_device_pixels_equal_host_pixels(gpv_mod, frames):
    a = _gpu_frames(gpv_mod, frames[:4], device=True)
    b = _gpu_frames(gpv_mod, frames[:4])
    for x, y in zip(a, b):
        assert x.tobytes() == y.tobytes()


def test_sequence_argument_checks(gpv_mod, frames):
    W0 = frames[0]
    F = gpv_mod.Image(image_gs=W0["f"], border=20)
    G = gpv_mod.Image(image_gs=W0["f"], border=20)
    desc = gpv_mod.make_desc(W0["coords"][:10], 25, 1)
    seq = gpv_mod.SubsetSequence(F, G, desc, np.uint8)
    with pytest.raises(ValueError):
        seq.frame(np.zeros((10, 10), np.uint8))
    with pytest.raises(gpv_mod.GpvError):
        gpv_mod.SubsetSequence(F, G, desc, np.uint8, precision=gpv_mod.PREC_FP64)  # no FP64 coefficients
