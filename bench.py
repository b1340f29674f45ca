#!/usr/bin/env python
"""Benchmark: ICGN subsets/s on the second-order-at-scale workload.

Workload (one step = one image pair through the whole hot path):
    4096 x 4096 uint16 (12-bit) seeded speckle pair under 1% uniaxial strain,
    0.5 deg rotation and 1e-6 px^-1 quadratic terms; circular subsets r = 30
    on a 10 px grid (~150k subsets), 12-parameter (second-order) ICGN,
    max_norm 1e-5, 50 iterations, FP32 interpolation / FP64 reductions.
    step = prefilter(f) + prefilter(g) + batched ICGN solve of every subset.

value : subsets/s with pixels, descriptors and outputs resident in HBM
        (gpv_image_update_device + gpv_solve_batch_device), device-timed.
e2e   : the same through the host C ABI (gpv_image_update from pinned host
        pixels x2, gpv_solve_batch with host descriptors in / results out),
        device-timed on the library stream; H2D / D2H bytes counted.
roofline: the ICGN kernel against a live-measured FP32 FMA peak (algorithmic
        work = 42 tap FMAs per target sample + 90 per reference sample).
cpu_baseline: the FP64 C oracle (restatement of the reference's Rust solver)
        on a bounded sample of the same subsets, all host threads.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): every rank solves its own replica of the workload
(replicas only: the path has no exchange step); value = all ranks' subsets
/ max over ranks of the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "geopyv-dev_b200"))
# as the gpv package does on import, before anything initialises CUDA: enough
# hardware work queues for the serving leg's concurrent worker streams
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

# ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-size
# second-order solve launch, by kernel (captured separately, not in this run)
ICGN_C2_DRAM_BYTES = {"icgn_tile<2,128>": 977.85e6, "icgn_runs<2,128,4>": 1136.39e6}

METRIC = "ICGN subsets/s at <=1e-3 px vs FP64 oracle; p50/p99 served solve latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--scale-down", type=int, default=1)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mesh", action="store_true", help="skip the mesh-propagation leg")
    ap.add_argument("--no-sequence", action="store_true", help="skip the frame-tracking leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch (graph) leg")
    ap.add_argument("--no-rigid", action="store_true", help="skip the rigid-texture leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 form on the full batch")
    ap.add_argument("--no-c1", action="store_true", help="skip the first-order 1024^2 workload at full size")
    ap.add_argument("--no-precision-ab", action="store_true", help="skip the precision-form comparison")
    ap.add_argument("--sequence-frames", type=int, default=200, help="frames of the sequence leg")
    ap.add_argument("--serving-seconds", type=float, default=10.0)
    return ap.parse_args()


# ---------------------------------------------------------------------------
def _backend():
    """NCCL on GPUs; gloo when GPV_BENCH_BACKEND=gloo or no GPU is visible
    (the CPU tests of the multi-rank path)."""
    import torch
    if os.environ.get("GPV_BENCH_BACKEND") == "gloo" or not torch.cuda.is_available():
        return "gloo"
    return "nccl"


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if _backend() == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The largest of the ranks' values (device timing: the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if _backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, steps, t_ms_local, world):
    """Whole-job throughput of replicas: every rank's units over the slowest
    rank's timed region."""
    t_max = max_over_ranks(t_ms_local, world)
    return world * units_per_rank * steps / (t_max * 1e-3), t_max


class ClockSampler:
    """SM clock and clock-event reasons during the timed region, read through
    NVML every 10 ms (nvidia-smi every 200 ms when NVML is unavailable).
    Reads only; changes no setting."""

    NAMES = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
             0x80: "hw_power_brake_slowdown"}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm_mhz, reason bits)
        self.smax = None
        self.stop_ev = threading.Event()

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = self.device
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if self.device < len(ids) and ids[self.device].isdigit():
                idx = int(ids[self.device])
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def start(self):
        try:
            nv, h = self._handle()
            self.nvml = (nv, h)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self.stop_ev.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(get_reasons(h))))
                    except Exception:
                        pass
                    self.stop_ev.wait(0.01)
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_ev.set()
            self.t.join(timeout=2)
            sm = [c for c, _ in self.samples]
            bits = 0
            for _, b in self.samples:
                bits |= b
            reasons = sorted(n for k, n in self.NAMES.items() if bits & k)
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, 10 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------
def load_workload(args):
    from gpv import synth
    t = time.time()
    W = synth.workload(args.config, scale_down=args.scale_down)
    W["gen_s"] = time.time() - t
    return W


def common_config(W, args, world):
    """The workload's `config` object, the same in both arms."""
    h, w = W["f"].shape
    l2_bytes = 2 * 4 * (h + 40) * (w + 40) + 2 * W["f"].dtype.itemsize * h * w
    orders = np.unique(W["order"])
    return {"workload": W["name"], "subsets": int(len(W["coords"])), "image": [int(h), int(w)],
            "pixel_dtype": str(W["f"].dtype), "radius": int(np.max(W["radius"])),
            "order": int(orders[0]) if len(orders) == 1 else "mixed", "max_norm": 1e-5,
            "max_iterations": 15 if args.config == 1 else 50,
            "step": "prefilter(f)+prefilter(g)+batched ICGN solve of every subset",
            "l2": (("inputs larger than L2" if l2_bytes > 126e6 else "inputs SMALLER than L2 (profiling case)") +
                   f": 2 x {h + 40}x{w + 40} FP32 coefficients + 2 x {h}x{w} pixels ({l2_bytes / 1e6:.0f} MB)"
                   " rewritten each step"),
            "parallelism": f"replicas x{world}"}


def measured_hbm_gbs():
    """(GB/s, source): the HBM copy bandwidth measured on this pool
    (MEASURED_PEAKS.json), else the pool's earlier measurement (fallback)."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), \
            "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "6,650 GB/s copy rate measured earlier on this pool (of fallback: MEASURED_PEAKS.json absent)"


def algorithmic_flop(res):
    """2 x (42 FMA per target sample x iterations + 90 FMA per reference sample)."""
    n = res["n_px"].astype(np.float64)
    it = res["iterations"].astype(np.float64)
    return 2.0 * (42.0 * float(np.sum(n * it)) + 90.0 * float(np.sum(n)))


def cpu_baseline(W, args, nthreads=None, seconds=None, rng_seed=7):
    """Oracle (FP64 C restatement) on a bounded sample: subsets/s of the full step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import gpv
    O.build()
    nthreads = nthreads or O.lib().gpvo_max_threads()
    seconds = seconds or args.cpu_seconds
    d = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    n = len(d)
    rng = np.random.default_rng(rng_seed)
    perm = rng.permutation(n)
    f64 = W["f"].astype(np.float64)
    t0 = time.perf_counter()
    Cf = O.get_c(f64, 20, nthreads)
    t_pref1 = time.perf_counter() - t0
    Cg = O.get_c(W["g"].astype(np.float64), 20, nthreads)
    # calibrate, then size the sample to ~seconds of solving
    k = min(n, max(32, 4 * nthreads))
    t0 = time.perf_counter()
    O.solve_batch(Cf, Cg, W["f"].shape, 20, d[perm[:k]], max_norm=1e-5, max_iterations=50, nthreads=nthreads)
    per = (time.perf_counter() - t0) / k
    s = int(min(n - k, max(64, seconds / max(per, 1e-9))))
    sample = perm[k:k + s] if s > 0 else perm[:k]  # a small batch: time it whole
    t0 = time.perf_counter()
    ref = O.solve_batch(Cf, Cg, W["f"].shape, 20, d[sample], max_norm=1e-5, max_iterations=50, nthreads=nthreads)
    t_solve = time.perf_counter() - t0
    per = t_solve / len(sample)
    t_step = 2 * t_pref1 + per * n  # prefilter both images + every subset
    return dict(value=n / t_step, cores=int(nthreads), per_subset_s=per, prefilter_s=t_pref1,
                sample_idx=sample, sample_res=ref, n=n, solve_s=t_solve)


# ---------------------------------------------------------------------------
def grid_mesh(coords):
    """Two triangles per cell of a structured node grid (row-major coords)."""
    xs = np.unique(coords[:, 0])
    ys = np.unique(coords[:, 1])
    nx = len(xs)
    el = []
    for r in range(len(ys) - 1):
        for c in range(nx - 1):
            a, b, d, e = r * nx + c, r * nx + c + 1, (r + 1) * nx + c, (r + 1) * nx + c + 1
            el.append((a, b, d))
            el.append((b, e, d))
    return np.array(el, dtype=np.int64)


def mesh_leg(W, F, G, args, cpu=True):
    """Mesh propagation (gpv_mesh_solve, layer-RG) over the workload's image
    pair: a 20 px structured triangular mesh, second-order subsets of the
    workload's radius, rounds sized for 64 workers.  CPU rate: the oracle's
    restatement of the propagation over the FP64 oracle, on a sub-mesh."""
    import gpv
    from gpv import synth
    h, w = W["f"].shape
    r = int(W["radius"].max())
    margin = r + 3 + 0.012 * h
    nodes = synth.grid(h, w, 20, margin)
    el = grid_mesh(nodes)
    c = nodes[np.argmin(np.sum((nodes - [(w - 1) / 2.0, (h - 1) / 2.0]) ** 2, axis=1))]
    seed_warp = np.zeros(12)
    seed_warp[:2] = synth.displacement(W["field"], [c])[0]
    kw = dict(seed_coord=tuple(c), seed_warp=list(seed_warp), subset_order=2, preconditioning="layer-RG",
              layer_rg_max_workers=64, max_norm=1e-5, max_iterations=50)
    m = gpv.Mesh(nodes, el, F, G)
    m.solve(r, override_active=True, **kw)  # warm-up (tables, workspace)
    t0 = time.perf_counter()
    m.solve(r, override_active=True, **kw)
    t = time.perf_counter() - t0
    truth = synth.displacement(W["field"], nodes)
    out = {"nodes": int(len(nodes)), "elements": int(len(el)), "radius": r, "order": 2,
           "preconditioning": "layer-RG, batch_factor 4, root_rel_eps 0.02, max_workers 64",
           "ms": 1e3 * t, "nodes_per_s": len(nodes) / t, "batches": m.stats["batches"],
           "subset_solves": m.stats["solves"], "quality_ok_frac": float(m.quality_ok.mean()),
           "max_err_vs_field_px_quality_ok": float(np.abs(m.displacements - truth)[m.quality_ok].max()),
           "not_quality_ok": int((~m.quality_ok).sum()),
           "timing": "host wall clock around the synchronous C-ABI call (host driver + every batch)"}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import mesh_oracle as MO
        import oracle as O
        half = 30 * 20  # a 61 x 61-node sub-mesh around the seed
        sub = np.all(np.abs(nodes - c) <= half + 1e-9, axis=1)
        idx = np.nonzero(sub)[0]
        remap = -np.ones(len(nodes), np.int64)
        remap[idx] = np.arange(len(idx))
        sel = np.all(sub[el], axis=1)
        sel_el = remap[el[sel]]
        Cf = O.get_c(W["f"].astype(np.float64), 20)
        Cg = O.get_c(W["g"].astype(np.float64), 20)

        def solver(d, tol):
            return O.solve_batch(Cf, Cg, W["f"].shape, 20, d, max_norm=1e-5, max_iterations=50, tolerance=tol)
        t0 = time.perf_counter()
        ref = MO.solve_mesh(nodes[idx], sel_el, solver, desc_dtype=O.DESC_DTYPE, radius=r, seed_coord=tuple(c),
                            seed_warp=list(seed_warp), subset_order=2, preconditioning="layer-RG", max_workers=64)
        tc = time.perf_counter() - t0
        ms = gpv.Mesh(nodes[idx], sel_el, F, G)
        ms.solve(r, override_active=True, **kw)
        rp = np.array([x["p"][:2] for x in ref["results"]])
        out["cpu_oracle"] = {"nodes": int(len(idx)), "s": tc, "nodes_per_s": len(idx) / tc,
                             "cores": int(O.lib().gpvo_max_threads()),
                             "max_disp_diff_vs_gpu_px": float(np.abs(ms.displacements - rp).max()),
                             "same_rounds": bool(np.array_equal(ms.rounds, ref["rounds"])),
                             "what": "oracle/mesh_oracle.py over the FP64 C oracle (one OpenMP batch per colour)"}
    return out


# ---------------------------------------------------------------------------
def uneven_leg(device, steps=10):
    """The uneven batch in one launch: the shear-band workload (2048^2 u8,
    50k subsets from a mesh refined x4 near the band, radii 15..60
    log-uniform, 70/30 first/second order) solved through the device C ABI,
    eagerly and as a replayed CUDA graph (gpv_batch_graph_*); CUDA events on
    the library stream around `steps` solves, inputs resident."""
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib, synth
    W = synth.workload(3)
    ctx = gpv.Context(device)
    F = gpv.Image(image_gs=W["f"], border=20, ctx=ctx)
    G = gpv.Image(image_gs=W["g"], border=20, ctx=ctx)
    desc = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    n = len(desc)
    ctx.reserve(n, int(desc["radius"].max()), 50)
    order = np.argsort(-(3 * desc["radius"].astype(np.int64) + desc["order"]), kind="stable").astype(np.int32)
    d_dev = torch.from_numpy(desc.view(np.uint8).copy()).cuda(device)
    o_dev = torch.from_numpy(order).cuda(device)
    out_dev = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{device}")
    prm = gpv._params(1e-5, 50, 0.75, False, gpv.PREC_MIXED, None, None)
    L = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)
    args = (ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), ct.c_void_p(o_dev.data_ptr()), n,
            ct.byref(prm), ct.c_void_p(out_dev.data_ptr()))

    def timed(step):
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_eager = timed(lambda: _lib.check(L.gpv_solve_batch_device(*args, None), "solve"))
    res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    bg = ct.c_void_p()
    _lib.check(L.gpv_batch_graph_create(*args, ct.byref(bg)), "graph")
    ms_graph = timed(lambda: _lib.check(L.gpv_batch_graph_launch(bg, None), "graph launch"))
    res_g = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    L.gpv_batch_graph_destroy(bg)
    ok = res["converged"] == 1
    err = np.abs(res["p"][ok, :2] - W["truth_uv"][ok])
    samples = float(np.sum(res["n_px"].astype(np.float64) * res["iterations"]))
    return {"workload": W["name"], "subsets": n, "radius": [int(desc["radius"].min()), int(desc["radius"].max())],
            "order2_frac": float(np.mean(desc["order"] == 2)), "steps": steps,
            "ms_eager": ms_eager, "subsets_per_s_eager": n / (ms_eager * 1e-3),
            "ms_graph": ms_graph, "subsets_per_s_graph": n / (ms_graph * 1e-3),
            "samples_per_s_graph": samples / (ms_graph * 1e-3),
            "graph_equals_eager": bool(res.tobytes() == res_g.tobytes()),
            "converged_frac": float(ok.mean()), "iterations_mean": float(res["iterations"].mean()),
            "median_err_vs_field_px": float(np.median(err)) if ok.any() else None,
            "timing": "CUDA events on the library stream; device-resident images, descriptors, work order, results; "
                      "one launch = order partition + one persistent kernel per (order, radius class) segment"}


# ---------------------------------------------------------------------------
def fp64_leg(W, device, mixed_solve_ms, steps=3):
    """The plain one-subset-per-block FP64 form (icgn_fp64: FP64 coefficients,
    interpolation, sums and solve) on the headline batch, device-resident,
    CUDA events around `steps` solves; beside it the mixed form's solve time
    of the same batch from the headline timing."""
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib
    ctx = gpv.Context(device)
    F = gpv.Image(image_gs=W["f"], border=20, ctx=ctx, keep_f64=True)
    G = gpv.Image(image_gs=W["g"], border=20, ctx=ctx, keep_f64=True)
    desc = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    n = len(desc)
    ctx.reserve(n, int(desc["radius"].max()), 50)
    d_dev = torch.from_numpy(desc.view(np.uint8).copy()).cuda(device)
    out_dev = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{device}")
    prm = gpv._params(1e-5, 50, 0.75, False, gpv.PREC_FP64, None, None)
    L = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)
    args = (ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), None, n, ct.byref(prm),
            ct.c_void_p(out_dev.data_ptr()), None)
    _lib.check(L.gpv_solve_batch_device(*args), "fp64 solve")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        _lib.check(L.gpv_solve_batch_device(*args), "fp64 solve")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    return {"kernel": "icgn_fp64 (one block of 256 threads per subset, FP64 throughout)", "subsets": n,
            "solve_ms": ms, "fp64_plain_subsets_per_s": n / (ms * 1e-3),
            "mixed_solve_ms": mixed_solve_ms, "mixed_over_fp64": ms / mixed_solve_ms,
            "iterations_mean": float(res["iterations"].mean()), "converged_frac": float(res["converged"].mean()),
            "timing": "CUDA events on the library stream, device-resident inputs, solve only (both forms)"}


def precision_leg(ctx, F, G, desc, sample_idx, sample_ref, steps=3):
    """The headline batch solved by three precision forms, device-resident,
    each timed with CUDA events and compared with the same oracle sample:
    the tiled kernel (FP32 sums over at most 8 pixels then FP64; Gauss-Jordan
    inverse of the scaled Hessian), the run-layout kernel (FP32 sums over each
    run then FP64; Cholesky factor, substitution solve) and the run-layout
    kernel with Kahan-compensated FP64 ZNSSD sums (GPV_SOLVE_KAHAN)."""
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib
    n = len(desc)
    d_dev = torch.from_numpy(desc.view(np.uint8).copy()).cuda()
    out_dev = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    L = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)
    forms = {"tile_chunked_fp32_gauss_jordan": ("tile", 0), "runs_fp32_per_run_cholesky": ("runs", 0),
             "runs_kahan_fp64_cholesky": ("runs", _lib.SOLVE_KAHAN)}
    out = {}
    saved = os.environ.get("GPV_SOLVE_KERNEL")
    try:
        for name, (kern, flags) in forms.items():
            os.environ["GPV_SOLVE_KERNEL"] = kern
            prm = _lib.SolveParams(max_norm=1e-5, tolerance=0.75, max_iterations=50, flags=flags,
                                   precision=gpv.PREC_MIXED, reserved=0, mask=None, history=None)
            args = (ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), None, n, ct.byref(prm),
                    ct.c_void_p(out_dev.data_ptr()), None)
            _lib.check(L.gpv_solve_batch_device(*args), name)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                _lib.check(L.gpv_solve_batch_device(*args), name)
            e1.record(stream)
            torch.cuda.synchronize()
            res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
            entry = {"solve_ms": e0.elapsed_time(e1) / steps, "iterations_mean": float(res["iterations"].mean())}
            if sample_idx is not None:
                ok = (sample_ref["status"] == 0) & (sample_ref["converged"] == 1)
                r = res[sample_idx]
                entry.update({
                    "max_disp_err_px": float(np.abs(r["p"][ok, :2] - sample_ref["p"][ok, :2]).max()),
                    "max_strain_err": float(np.abs(r["p"][ok, 2:6] - sample_ref["p"][ok, 2:6]).max()),
                    "flag_agreement": float(np.mean((r["converged"] == sample_ref["converged"]) &
                                                    (r["quality_ok"] == sample_ref["quality_ok"]))),
                    "iteration_agreement": float(np.mean(r["iterations"] == sample_ref["iterations"]))})
            out[name] = entry
    finally:
        if saved is None:
            os.environ.pop("GPV_SOLVE_KERNEL", None)
        else:
            os.environ["GPV_SOLVE_KERNEL"] = saved
    out["oracle_sample"] = int(len(sample_idx)) if sample_idx is not None else 0
    out["timing"] = "CUDA events on the library stream, device-resident inputs, solve only"
    return out


def c1_leg(device, steps=10):
    """The first-order workload at full size (1024^2 u8, rigid (0.35, -0.20)
    px, r = 25 on a 20 px grid, 15 iterations): steps of prefilter(f) +
    prefilter(g) + solve through the device C ABI (CUDA events), and every
    subset compared with the FP64 oracle."""
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib, synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = synth.workload(1)
    ctx = gpv.Context(device)
    F = gpv.Image(image_gs=W["f"], border=20, ctx=ctx)
    G = gpv.Image(image_gs=W["g"], border=20, ctx=ctx)
    desc = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    n = len(desc)
    ctx.reserve(n, 25, 15)
    f_dev = torch.from_numpy(W["f"].copy()).cuda(device)
    g_dev = torch.from_numpy(W["g"].copy()).cuda(device)
    d_dev = torch.from_numpy(desc.view(np.uint8).copy()).cuda(device)
    out_dev = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{device}")
    prm = gpv._params(1e-5, 15, 0.75, False, gpv.PREC_MIXED, None, None)
    L = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        _lib.check(L.gpv_image_update_device(F.handle, ct.c_void_p(f_dev.data_ptr()), _lib.GPV_U8), "update f")
        _lib.check(L.gpv_image_update_device(G.handle, ct.c_void_p(g_dev.data_ptr()), _lib.GPV_U8), "update g")
        _lib.check(L.gpv_solve_batch_device(ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), None, n,
                                            ct.byref(prm), ct.c_void_p(out_dev.data_ptr()), None), "solve")
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    O.build()
    t0 = time.perf_counter()
    Cf, Cg = O.get_c(W["f"].astype(np.float64), 20), O.get_c(W["g"].astype(np.float64), 20)
    ref = O.solve_batch(Cf, Cg, W["f"].shape, 20, desc, max_norm=1e-5, max_iterations=15)
    tc = time.perf_counter() - t0
    ok = (ref["status"] == 0) & (ref["converged"] == 1)
    return {"workload": W["name"], "subsets": n, "steps": steps, "ms_per_step": ms, "subsets_per_s": n / (ms * 1e-3),
            "iterations_mean": float(res["iterations"].mean()),
            "accuracy": {"oracle_subsets": n, "max_disp_err_px": float(np.abs(res["p"][ok, :2] - ref["p"][ok, :2]).max()),
                         "max_strain_err": float(np.abs(res["p"][ok, 2:6] - ref["p"][ok, 2:6]).max()),
                         "flag_agreement": float(np.mean((res["converged"] == ref["converged"]) &
                                                         (res["quality_ok"] == ref["quality_ok"]))),
                         "iteration_agreement": float(np.mean(res["iterations"] == ref["iterations"])),
                         "max_err_vs_imposed_px": float(np.abs(res["p"][ok, :2] - W["truth_uv"][ok]).max())},
            "cpu_oracle_step_s": tc, "cpu_oracle_cores": int(O.lib().gpvo_max_threads()),
            "timing": "CUDA events on the library stream; step = prefilter(f) + prefilter(g) + solve, device pixels"}


# ---------------------------------------------------------------------------
def rigid_leg(W, device, steps=5):
    """The headline batch with the rigid-texture template (src/texture.rs): the
    reference's grain maps built on the device from its pixels, then the
    same subsets solved with the per-iteration template, beside the
    deformable solve on the same images; CUDA events on the library stream,
    inputs resident."""
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib
    ctx = gpv.Context(device)
    F = gpv.Image(image_gs=W["f"], border=20, ctx=ctx, grain=True)
    G = gpv.Image(image_gs=W["g"], border=20, ctx=ctx)
    desc = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    desc1 = desc.copy()  # the same subsets at first order
    desc1["order"] = 1
    desc1["p0"][:, 6:] = 0.0
    n = len(desc)
    ctx.reserve(n, int(desc["radius"].max()), 50)
    order = np.argsort(-(3 * desc["radius"].astype(np.int64) + desc["order"]), kind="stable").astype(np.int32)
    o_dev = torch.from_numpy(order).cuda(device)
    out_dev = torch.zeros(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{device}")
    L = _lib.lib()
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    for label, dsc in (("", desc), ("_order1", desc1)):
        d_dev = torch.from_numpy(dsc.view(np.uint8).copy()).cuda(device)
        for tex in ("deformable", "rigid"):
            prm = gpv._params(1e-5, 50, 0.75, False, gpv.PREC_MIXED, None, None, "icgn", tex)
            args = (ctx.handle, F.handle, G.handle, ct.c_void_p(d_dev.data_ptr()), ct.c_void_p(o_dev.data_ptr()), n,
                    ct.byref(prm), ct.c_void_p(out_dev.data_ptr()), None)
            for _ in range(2):
                _lib.check(L.gpv_solve_batch_device(*args), "solve")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                _lib.check(L.gpv_solve_batch_device(*args), "solve")
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
            out[tex + label] = dict(ms=ms, subsets_per_s=n / (ms * 1e-3),
                                    iterations_mean=float(res["iterations"].mean()),
                                    converged_frac=float(res["converged"].mean()),
                                    texture_frac=float(res["texture"].mean()))
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    F.update(W["f"])  # prefilter + grain statistics and maps of a 4096^2 reference
    t1.record(stream)
    torch.cuda.synchronize()
    gr = F.grain()
    return {"workload": W["name"], "subsets": n, "correlation_length_px": gr["correlation_length"],
            "update_with_grain_ms": t0.elapsed_time(t1),
            "update_with_grain": "host pixels of the reference: upload + prefilter + correlation length + maps", **out,
            "timing": "CUDA events on the library stream; the rigid template's extra work is one template pass "
                      "and its sums per iteration at second order, closed-form sums from fixed grain moments "
                      "at first order (*_order1: the same subsets solved at first order)"}


# ---------------------------------------------------------------------------
def sequence_leg(ctx, n_frames=200, frame_step=1):
    """Frame-to-frame tracking (gpv_sequence_*) on the incremental-sequence
    workload: 2048^2 u8 frames under simple shear rising linearly to 5% at
    frame 200 (every frame by default), 20,000 subsets of radius 25,
    reference fixed at frame 0.  Per frame: pinned host pixels -> device,
    in-place prefilter, seeding from the last converged warps, batched solve;
    results stay on the device.  Timed with CUDA events on the library stream
    over frames 1..n-1, once as CUDA-graph replay and once as eager launches."""
    import torch

    import gpv
    from gpv import synth
    t0 = time.perf_counter()
    W0, frames = synth.sequence_frames(n_frames, 1, frame_step)
    gen_s = time.perf_counter() - t0
    n_frames = len(frames)
    pins = [torch.from_numpy(g).pin_memory() for g in frames]
    desc = gpv.make_desc(W0["coords"], W0["radius"], W0["order"], W0["p0"])
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {"workload": W0["name"].replace("frame 0 ", "") + f", {n_frames} frames, shear +{0.05 * frame_step / 200:.5f}/frame",
           "subsets": int(len(desc)), "frames_timed": n_frames - 1, "frame_generation_s": gen_s}
    for graph in (True, False):
        F = gpv.Image(image_gs=W0["f"], border=20, ctx=ctx)
        G = gpv.Image(image_gs=W0["f"], border=20, ctx=ctx)
        seq = gpv.SubsetSequence(F, G, desc, np.uint8, graph=graph)
        seq.frame(pins[0].numpy(), download=False)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(1, n_frames):
            _lib_frame(seq, pins[k])
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / (n_frames - 1)
        key = "graph" if graph else "eager"
        out[f"ms_per_frame_{key}"] = ms
        out[f"subsets_per_s_{key}"] = len(desc) / (ms * 1e-3)
        if graph:
            from gpv import _lib
            res = np.zeros(len(desc), _lib.RESULT_DTYPE)
            torch.cuda.synchronize()
            import ctypes as ct
            _lib.check(_lib.lib().gpv_sequence_frame(seq._h, ct.c_void_p(pins[-1].data_ptr()), 0,
                                                     res.ctypes.data_as(ct.c_void_p)), "frame")
            c = (W0["f"].shape[0] - 1) / 2.0
            last = synth.make_field(xc=c, yc=c, a=(0.0, 0.05 * frame_step * (n_frames - 1) / 200.0, 0.0, 0.0))
            truth = synth.displacement(last, W0["coords"])
            good = res["converged"] == 1
            out["converged_frac_last_frame"] = float(good.mean())
            out["max_err_vs_field_px_last_frame"] = float(np.abs(res["p"][good, :2] - truth[good]).max())
        seq.close()
    out["timing"] = "CUDA events on the library stream; per frame: H2D of pinned pixels + prefilter + seeding + solve"
    return out


def _lib_frame(seq, pinned):
    import ctypes as ct

    from gpv import _lib
    _lib.check(_lib.lib().gpv_sequence_frame(seq._h, ct.c_void_p(pinned.data_ptr()), 0, None), "gpv_sequence_frame")


# ---------------------------------------------------------------------------
def serving_leg(seconds=10.0, rate=200.0, seed=55, configs=None):
    """The serving stream: Poisson arrivals at `rate` req/s for `seconds`,
    each request a seeded speckle pair of side 512..4096 (u8 or u16) under a
    random affine field (|strain| <= 2%, |rotation| <= 1 deg, |t| <= 5 px),
    100..100k subsets (log-uniform) of radius 15..50 and mixed order, initial
    warps from the field +-0.3 px (a coarse upstream estimate).  Pixels and
    subsets come from a pre-generated pool (one pair per size and pixel type,
    pinned host memory); latency is submit -> results in host memory.
    Each server configuration in `configs` (name -> Server keywords) serves
    the same arrival sequence; the first one is the headline."""
    import math

    import torch

    import gpv
    from gpv import synth
    rng = np.random.default_rng(seed)
    pool = []
    for size in (512, 1024, 2048, 4096):
        for dt in (np.uint8, np.uint16):
            c = (size - 1) / 2.0
            th = math.radians(rng.uniform(-1, 1))
            e = rng.uniform(-0.02, 0.02, 2)
            a = ((1 + e[0]) * math.cos(th) - 1.0, -math.sin(th), math.sin(th), (1 + e[1]) * math.cos(th) - 1.0)
            fld = synth.make_field(xc=c, yc=c, t=tuple(rng.uniform(-5, 5, 2)), a=a)
            f, g = synth.pair(size, size, fld, 7000 + size + (1 if dt == np.uint16 else 0), dtype=dt,
                              scale=16.0 if dt == np.uint16 else 1.0)
            fp = torch.from_numpy(f.view(np.uint8 if dt == np.uint8 else np.int16).copy()).pin_memory()
            gp = torch.from_numpy(g.view(np.uint8 if dt == np.uint8 else np.int16).copy()).pin_memory()
            margin = 60 + 0.027 * size  # radius 50 + the largest |u| of the field + 5 px
            m = 100000
            xy = rng.uniform(margin, size - margin, (m, 2))
            radius = rng.integers(15, 51, m).astype(np.int32)
            order = rng.integers(1, 3, m).astype(np.int32)
            desc = gpv.make_desc(xy, radius, order, synth.seeded_p0(fld, xy, rng))
            pool.append((fp.numpy().view(dt), gp.numpy().view(dt), desc, (fp, gp)))
    # the arrival sequence: (time, pool entry, subset count, first subset)
    arrivals = []
    t_next = 0.0
    while t_next < seconds:
        k = int(rng.integers(len(pool)))
        n = int(math.exp(rng.uniform(math.log(100), math.log(100000))))
        arrivals.append((t_next, k, n, int(rng.integers(0, 100000 - n + 1))))
        t_next += rng.exponential(1.0 / rate)
    if configs is None:
        configs = {"priority_lane": dict(workers=8, priority_workers=4, priority_subsets=20000),
                   "arrival_order": dict(workers=8)}
    results = {}
    for name, kw in configs.items():
        srv = gpv.Server(reserve_subsets=100000, reserve_radius=50, **kw)
        # every worker's image pair for every shape and pixel type (no allocation while serving)
        for f, _, _, _ in pool:
            srv.prepare(f.shape, f.dtype)
        # warm-up: kernels, tables, autotune-free launch paths
        for f, g, d, _ in pool:
            for t in [srv.submit(f, g, d[:n]) for n in (100, 30000) for _ in range(kw["workers"])]:
                srv.wait(t, 120000)
        srv.reset_stats()
        t0 = time.perf_counter()
        tickets = []
        for t_at, k, n, start in arrivals:
            while time.perf_counter() - t0 < t_at:
                time.sleep(0.0002)
            f, g, d, _ = pool[k]
            tickets.append((n, srv.submit(f, g, d[start:start + n])))
        lat = []
        conv = []
        for n, t in tickets:
            out = srv.wait(t, 600000)
            lat.append((n, t.latency_ms))
            conv.append(float(np.mean(out["converged"])))
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        ln = np.array([x[1] for x in lat])
        ns = np.array([x[0] for x in lat])
        mid = (ns >= 5000) & (ns <= 20000)
        big = ns > 20000
        results[name] = {
            "server": kw, "requests": len(tickets), "arrival_rate_per_s": rate, "seconds_of_arrivals": seconds,
            "p50_ms": float(np.percentile(ln, 50)), "p99_ms": float(np.percentile(ln, 99)),
            "p99_ms_5k_20k_subsets": float(np.percentile(ln[mid], 99)) if mid.any() else None,
            "p50_ms_5k_20k_subsets": float(np.percentile(ln[mid], 50)) if mid.any() else None,
            "requests_5k_20k_subsets": int(mid.sum()),
            "p99_ms_over_20k_subsets": float(np.percentile(ln[big], 99)) if big.any() else None,
            "subsets_per_s": float(ns.sum() / wall), "subsets": int(ns.sum()), "wall_s": wall,
            "mean_converged_frac": float(np.mean(conv)), "peak_admitted_bytes": int(st["peak_bytes"]),
            "mean_queue_ms": st["mean_queue_ms"], "mean_service_ms": st["mean_service_ms"],
            "hbm_budget_bytes": int(st["hbm_budget"])}
    head = dict(results[next(iter(configs))])
    head["configs"] = {k: v for k, v in results.items()}
    head["latency"] = "submit -> results in host memory; pinned host pixels; per request: H2D, prefilter x2, solve, D2H"
    return head


# ---------------------------------------------------------------------------
def run_reference(args, world, rank):
    """--impl reference: the FP64 C restatement of the reference's CPU solver
    (the Rust crate cannot be built here) on the box's host cores.  Every
    timed step is a full step of the workload -- the oracle's prefilter of
    both images and the solve of every subset, all host threads -- timed by
    the host clock; warm-up steps solve a bounded sample.  A single-core rate
    on a bounded sample follows the timed steps."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    import gpv
    O.build()
    W = load_workload(args)
    nthreads = O.lib().gpvo_max_threads()
    d = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    n = len(d)
    max_it = 15 if args.config == 1 else 50
    f64, g64 = W["f"].astype(np.float64), W["g"].astype(np.float64)
    rng = np.random.default_rng(100)

    def solve(Cf, Cg, dd, threads):
        return O.solve_batch(Cf, Cg, W["f"].shape, 20, dd, max_norm=1e-5, max_iterations=max_it, nthreads=threads)

    for _ in range(args.warmup):  # bounded: prefilter + 2% of the subsets
        Cf, Cg = O.get_c(f64, 20, nthreads), O.get_c(g64, 20, nthreads)
        solve(Cf, Cg, d[rng.choice(n, max(64, n // 50), replace=False)], nthreads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        Cf, Cg = O.get_c(f64, 20, nthreads), O.get_c(g64, 20, nthreads)
        ref = solve(Cf, Cg, d, nthreads)
        times.append(time.perf_counter() - t0)
    v = n * args.steps / float(np.sum(times))
    # one host thread on a bounded sample (~seconds), solve only
    k = min(n, 64)
    t0 = time.perf_counter()
    solve(Cf, Cg, d[:k], 1)
    per = (time.perf_counter() - t0) / k
    ks = int(min(n, max(k, args.cpu_seconds / 3.0 / max(per, 1e-9))))
    pick = rng.choice(n, ks, replace=False)
    t0 = time.perf_counter()
    solve(Cf, Cg, d[pick], 1)
    t1 = time.perf_counter() - t0
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "subsets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": common_config(W, args, world),
        "cpu_baseline": {"value": v, "unit": "subsets/s", "cores": int(nthreads), "kind": "port",
                         "sample": f"every step whole: oracle prefilter of both images + all {n} subsets (FP64 C "
                                   "restatement of src/image.rs / src/subset.rs, OpenMP); warm-up steps: prefilter "
                                   "+ 2% of the subsets"},
        "single_core": {"subsets_per_s": ks / t1, "cores": 1, "sample": f"{ks} random subsets, solve only, "
                                                                          f"{t1:.1f} s"},
        "step_ms": [1e3 * t for t in times],
        "converged_frac": float(np.mean(ref["converged"])),
        "timing": "host clock (time.perf_counter) around each full step",
        "e2e": {"value": v, "unit": "subsets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import ctypes as ct

    import torch

    import gpv
    from gpv import _lib
    torch.cuda.set_device(local)
    W = load_workload(args)
    h, w = W["f"].shape
    n = len(W["coords"])
    L = _lib.lib()
    ctx = gpv.Context(local)
    prec = gpv.PREC_FP64 if args.precision == "fp64" else gpv.PREC_MIXED
    keep64 = prec == gpv.PREC_FP64
    desc = gpv.make_desc(W["coords"], W["radius"], W["order"], W["p0"])
    max_r = int(W["radius"].max())
    ctx.reserve(n, max_r, 50)
    # images from device-resident pixels
    px_dtype = W["f"].dtype
    tdt = torch.uint8 if px_dtype == np.uint8 else torch.int16
    f_dev = torch.from_numpy(W["f"].view(np.uint8 if px_dtype == np.uint8 else np.int16).copy()).cuda()
    g_dev = torch.from_numpy(W["g"].view(np.uint8 if px_dtype == np.uint8 else np.int16).copy()).cuda()
    dcode = _lib.DTYPES[px_dtype]
    F = gpv.Image(image_gs=W["f"], border=20, keep_f64=keep64, ctx=ctx)
    G = gpv.Image(image_gs=W["g"], border=20, keep_f64=keep64, ctx=ctx)
    desc_dev = torch.from_numpy(desc.view(np.uint8).copy()).cuda()
    key = 3 * desc["radius"].astype(np.int64) + desc["order"]
    order = np.argsort(-key, kind="stable").astype(np.int32)
    order_dev = torch.from_numpy(order).cuda()
    out_dev = torch.empty(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    prm = _lib.SolveParams(max_norm=1e-5, tolerance=0.75, max_iterations=50, flags=0, precision=prec,
                           reserved=0, mask=None, history=None)
    stream = torch.cuda.Stream()  # a real stream: the C ABI maps NULL to the context stream
    torch.cuda.set_stream(stream)
    sptr = ct.c_void_p(stream.cuda_stream)
    # 2 images x (row pass + column pass), then the solve: the mixed form is
    # count_orders + scatter_orders + one tile kernel per order; FP64 one kernel
    launches_per_step = 4 + (5 if prec == gpv.PREC_MIXED else 1)
    # the prefilter runs on the library's context stream, the solve on torch's
    # current stream; events order the two
    ctx_stream = torch.cuda.ExternalStream(ctx.stream)

    def full_step(es0=None, es1=None):
        ev = torch.cuda.Event()
        ev.record(stream)
        ctx_stream.wait_event(ev)
        _lib.check(L.gpv_image_update_device(F.handle, ct.c_void_p(f_dev.data_ptr()), dcode), "update f")
        _lib.check(L.gpv_image_update_device(G.handle, ct.c_void_p(g_dev.data_ptr()), dcode), "update g")
        ev2 = torch.cuda.Event()
        ev2.record(ctx_stream)
        stream.wait_event(ev2)
        if es0 is not None:
            es0.record(stream)
        _lib.check(L.gpv_solve_batch_device(ctx.handle, F.handle, G.handle, ct.c_void_p(desc_dev.data_ptr()),
                                            ct.c_void_p(order_dev.data_ptr()), n, ct.byref(prm),
                                            ct.c_void_p(out_dev.data_ptr()), sptr), "solve")
        if es1 is not None:
            es1.record(stream)

    tuned = [0, 0, 0]
    if prec == gpv.PREC_MIXED and not os.environ.get("GPV_TILE_THREADS"):
        tuned = gpv.autotune(F, G, desc, sample_per_class=2048)
    layouts = [t["layout"] for t in ctx.tuning()]
    runk = [t["run_length"] for t in ctx.tuning()]
    runs = os.environ.get("GPV_SOLVE_KERNEL", "runs")[:1] != "t"
    cls = 0 if max_r <= 20 else (1 if max_r <= 40 else 2)
    if prec != gpv.PREC_MIXED:
        kernel_name = "icgn_fp64"
    elif runs:
        kernel_name = f"icgn_runs<{2 if args.config == 2 else 'mixed'},{tuned[cls] or 128},{runk[cls] or 4}>"
    else:
        kernel_name = f"icgn_tile<{2 if args.config == 2 else 'mixed'},{tuned[cls] or 128}>"
    peaks = _lib.Peaks()
    _lib.check(L.gpv_probe_peaks(ctx.handle, ct.byref(peaks)), "probe")
    fp32_peak = max(peaks.fp32_scalar_tflops, peaks.fp32_paired_tflops)
    for _ in range(args.warmup):
        full_step()
    torch.cuda.synchronize()
    res = np.frombuffer(out_dev.cpu().numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    solve_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e0.record(stream)
    for k in range(args.steps):
        full_step(*solve_ev[k])
    e1.record(stream)
    torch.cuda.synchronize()
    cl = clocks.stop()
    barrier(world)
    t_ms = e0.elapsed_time(e1)
    solve_ms = [a.elapsed_time(b) for a, b in solve_ev]
    value, t_max = replica_rate(n, args.steps, t_ms, world)

    # ---- e2e through the host C ABI (pinned host buffers) ----
    f_pin = torch.from_numpy(W["f"].view(np.uint8 if px_dtype == np.uint8 else np.int16).copy()).pin_memory()
    g_pin = torch.from_numpy(W["g"].view(np.uint8 if px_dtype == np.uint8 else np.int16).copy()).pin_memory()
    d_pin = torch.from_numpy(desc.view(np.uint8).copy()).pin_memory()
    o_pin = torch.empty(n * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()

    def e2e_step():
        _lib.check(L.gpv_image_update(F.handle, ct.c_void_p(f_pin.data_ptr()), dcode), "update f (host)")
        _lib.check(L.gpv_image_update(G.handle, ct.c_void_p(g_pin.data_ptr()), dcode), "update g (host)")
        _lib.check(L.gpv_solve_batch(ctx.handle, F.handle, G.handle, ct.c_void_p(d_pin.data_ptr()), n,
                                     ct.byref(prm), ct.c_void_p(o_pin.data_ptr())), "solve (host)")

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    lat = []
    a0.record(ctx_stream)
    for _ in range(args.steps):
        t = time.perf_counter()
        e2e_step()
        lat.append(time.perf_counter() - t)
    a1.record(ctx_stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(a0.elapsed_time(a1), world)
    e2e_value = world * n * args.steps / (e2e_ms * 1e-3)
    res_h = np.frombuffer(o_pin.numpy().tobytes(), dtype=_lib.RESULT_DTYPE).copy()
    h2d = W["f"].nbytes + W["g"].nbytes + desc.nbytes
    d2h = res_h.nbytes

    if rank != 0:
        return
    # ---- accuracy on the CPU-baseline sample + CPU baseline ----
    cpu = None
    acc = {}
    if not args.no_cpu_baseline:
        cpu = cpu_baseline(W, args)
        idx = cpu["sample_idx"]
        ref = cpu["sample_res"]
        ok = (ref["status"] == 0) & (ref["converged"] == 1)
        dpx = np.abs(res["p"][idx, :2] - ref["p"][:, :2])[ok]
        dstr = np.abs(res["p"][idx, 2:6] - ref["p"][:, 2:6])[ok]
        acc = {"oracle_sample": int(len(idx)), "converged_in_sample": int(ok.sum()),
               "max_disp_err_px": float(dpx.max()) if ok.any() else None,
               "max_strain_err": float(dstr.max()) if ok.any() else None,
               "flag_agreement": float(np.mean((res["converged"][idx] == ref["converged"]) &
                                               (res["quality_ok"][idx] == ref["quality_ok"]))),
               "iteration_agreement": float(np.mean(res["iterations"][idx] == ref["iterations"]))}
    mesh = None
    if not args.no_mesh and args.config == 2:
        mesh = mesh_leg(W, F, G, args, cpu=not args.no_cpu_baseline)
    seq = None
    if not args.no_sequence and args.config == 2 and args.scale_down == 1:
        seq = sequence_leg(ctx, n_frames=args.sequence_frames)
    uneven = None
    if not args.no_uneven and args.config == 2 and args.scale_down == 1:
        uneven = uneven_leg(local)
    rigid = None
    if not args.no_rigid and args.config == 2 and args.scale_down == 1 and prec == gpv.PREC_MIXED:
        rigid = rigid_leg(W, local)
    prec_ab = None
    if not args.no_precision_ab and args.config == 2 and prec == gpv.PREC_MIXED:
        prec_ab = precision_leg(ctx, F, G, desc, cpu["sample_idx"] if cpu else None, cpu["sample_res"] if cpu else None)
    fp64 = None
    if not args.no_fp64 and args.config == 2 and prec == gpv.PREC_MIXED:
        fp64 = fp64_leg(W, local, float(np.mean(solve_ms)))
    c1 = None
    if not args.no_c1 and args.config == 2 and args.scale_down == 1:
        c1 = c1_leg(local)
    serving = None
    if not args.no_serving and args.config == 2 and args.scale_down == 1:
        serving = serving_leg(seconds=args.serving_seconds)
    flop = algorithmic_flop(res)
    solve_avg_ms = float(np.mean(solve_ms))
    achieved = flop / (solve_avg_ms * 1e-3) / 1e12
    # DRAM bytes (read + write) of one solve launch from an ncu capture of the
    # same command at full size (not measured in this run; null elsewhere)
    traffic = None
    if args.config == 2 and args.scale_down == 1 and prec == gpv.PREC_MIXED:
        traffic = ICGN_C2_DRAM_BYTES.get(kernel_name)
    samples = float(np.sum(res["n_px"].astype(np.float64) * (res["iterations"] + 1)))
    # roofline time = the slower of the tap FMAs at the FP32 peak and the
    # coefficient-window bytes at the measured HBM bandwidth
    coef_bytes = float(np.sum((res["iterations"].astype(np.float64) + 1.0) *
                              (2.0 * desc["radius"].astype(np.float64) + 6.0) ** 2 * 4.0))
    hbm_gbs, hbm_source = measured_hbm_gbs()
    t_fma = flop / (fp32_peak * 1e12) if fp32_peak else 0.0
    t_bytes = coef_bytes / (hbm_gbs * 1e9)
    line = {
        "metric": METRIC, "value": value, "unit": "subsets/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec == gpv.PREC_MIXED else "f64", "data": "synthetic",
        "config": common_config(W, args, world),
        "precision": args.precision,
        "tuning": {"threads_per_block": {"r<=20": tuned[0], "r21-40": tuned[1], "r>40": tuned[2]},
                   "tile_layout": {"r<=20": layouts[0], "r21-40": layouts[1], "r>40": layouts[2]},
                   "run_length": {"r<=20": runk[0], "r21-40": runk[1], "r>40": runk[2]},
                   "kernel": kernel_name},
        "solve_ms": solve_avg_ms, "prefilter_ms": t_max / args.steps - solve_avg_ms,
        "samples_per_s": world * samples * args.steps / (t_max * 1e-3),
        "iterations_mean": float(np.mean(res["iterations"])),
        "converged_frac": float(np.mean(res["converged"])),
        "accuracy": acc,
        "roofline": {"bound": "fp32" if t_fma >= t_bytes else "hbm", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None, "traffic": traffic,
                     "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-size "
                                        f"{kernel_name} launch, captured separately (profiles/)"
                                        if traffic else "not captured for this configuration"),
                     "kernel": kernel_name,
                     "peak_scalar": peaks.fp32_scalar_tflops, "peak_paired": peaks.fp32_paired_tflops,
                     "peak_source": "measured live (gpv_probe_peaks): the larger of register-only FFMA and paired "
                                    "FFMA2 chains (of measured)",
                     "fp64_peak_tflops": peaks.fp64_tflops, "smem_peak_gbs": peaks.smem_gbs,
                     "work": "2 x (42 FMA per target sample x iterations + 90 FMA per reference sample)",
                     "t_fma_ms": 1e3 * t_fma, "t_bytes_ms": 1e3 * t_bytes,
                     "roofline_frac": max(t_fma, t_bytes) / (solve_avg_ms * 1e-3),
                     "hbm": {"algorithmic_bytes": coef_bytes, "achieved_gbs": coef_bytes / (solve_avg_ms * 1e-3) / 1e9,
                             "peak_gbs": hbm_gbs, "frac": coef_bytes / (solve_avg_ms * 1e-3) / 1e9 / hbm_gbs,
                             "peak_source": hbm_source,
                             "bytes": "(2r+6)^2 x 4 B coefficient window per subset per iteration and per setup"}},
        "e2e": {"value": e2e_value, "unit": "subsets/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "latency_ms": {"p50": 1e3 * float(np.percentile(lat, 50)), "p99": 1e3 * float(np.percentile(lat, 99))}},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": cl,
    }
    if mesh is not None:
        line["mesh"] = mesh
    if seq is not None:
        line["sequence"] = seq
    if uneven is not None:
        line["uneven_batch"] = uneven
    if rigid is not None:
        line["rigid_texture"] = rigid
    if prec_ab is not None:
        line["precision_forms"] = prec_ab
    if fp64 is not None:
        line["fp64_plain"] = fp64
        line["fp64_plain_subsets_per_s"] = fp64["fp64_plain_subsets_per_s"]
        line["mixed_over_fp64"] = fp64["mixed_over_fp64"]
    if c1 is not None:
        line["c1"] = c1
    if serving is not None:
        line["serving"] = serving
        line["p50_ms"] = serving["p50_ms"]
        line["p99_ms"] = serving["p99_ms"]
        line["p99_ms_5k_20k_subsets"] = serving["p99_ms_5k_20k_subsets"]
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": "subsets/s", "cores": cpu["cores"], "kind": "port",
                                "sample": f"{len(cpu['sample_idx'])} random subsets of the same batch solved by the FP64 C "
                                          f"oracle in {cpu['solve_s']:.1f} s + oracle prefilter of both images "
                                          f"({2 * cpu['prefilter_s']:.1f} s), scaled to the full step"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
