"""Benchmark of the fused batched TV-L1 flow path: 80^3 frame pairs per second.

Workload (one step): a synthetic cine sequence of T = 35 frames of 80^3 voxels; all 34 forward
and 34 backward consecutive pairs (68 independent solves, the reference's default solver
configuration: 3 levels x 15 warps x 300 iterations) run as ONE batched solve (one CUDA graph),
followed by the bidirectional propagation of the two end masks (t = 0 and t = 12) through the
flows. The sequence stands in for the reference's 80^3 x 35-frame cine MRI data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f16-flow32|f32|...] [--impl reference]

Before warm-up the iterate-kernel variant of each pyramid level is autotuned on the plan's own
state. Beside the headline line's contract keys it reports the plain GPU form (the reference's
per-operator structure on this package's kernels, one 80^3 pair, full schedule) for the ratio the
metric asks for, `latency` (p50/p99 of the 68-pair sequence from the timed steps, and of one 80^3
pair solved alone), `fp32_storage` (the same sequence solve with every field stored in FP32),
`persistent_form` (the same pair solves with the persistent iteration loop: one cooperative
launch per warp and level, its graph size, and a bitwise check against the headline flows) and
`compute_metrics` (the workload's own end-mask Dice / Hausdorff, warping.py:245-270). The
reference arm (--impl reference) adds `reference_gpu`: the reference's own CUDA extension on one
pair of the sequence. Further workloads, one JSON line each, on one GPU:

    python bench.py --workload uneven    # 64 pairs, dims per axis on {40, ..., 128}
    python bench.py --workload mixed     # the sequence + 16 x 128^3, 16-bit storage modes, EPE vs FP64 GPU oracle
    python bench.py --workload serving   # Poisson request streams through the continuous-batching server
    python bench.py --workload latency   # p50/p99 of one 80^3 pair alone and of the 68-pair sequence

Multi-GPU: one process per GPU (torchrun); every rank solves its own sequence (replicas, weak
scaling, no collective on the data path); NCCL is used only for the barrier and the max-over-ranks
timing. Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

T_FRAMES = 35
SHAPE = (80, 80, 80)
MASK_T0, MASK_T1 = 0, 12
METRIC = "80^3 TV-L1 flow pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    # default: the mixed-precision form that meets mean EPE <= 0.05 against the FP64 oracle
    # (FP16 dual field / tensor / linearisation, FP32 flow, FP32 arithmetic)
    ap.add_argument("--storage", default="f16-flow32", choices=["f32", "bf16", "f16", "bf16-flow32", "f16-flow32"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain-form", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-latency", action="store_true", help="skip the single-pair latency reps")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-storage sequence solve")
    ap.add_argument("--no-persistent", action="store_true", help="skip the persistent-loop sequence solve")
    ap.add_argument("--frames", type=int, default=T_FRAMES)
    ap.add_argument("--workload", default="sequence", choices=["sequence", "uneven", "mixed", "serving", "latency"],
                    help="sequence: 35-frame 80^3 cine sequence (the headline line); uneven: 64 pairs of "
                         "mixed sizes; mixed: the sequence plus 16 pairs of 128^3 with EPE against the FP64 "
                         "oracle; serving: Poisson request stream through the continuous-batching server")
    ap.add_argument("--rates", default="0.1,1,10,50", help="serving: arrival rates (requests/s)")
    ap.add_argument("--reps", type=int, default=50, help="latency: repetitions of the single-pair solve")
    ap.add_argument("--requests", type=int, default=6, help="serving: requests per rate")
    ap.add_argument("--max-active", type=int, default=0, help="serving: cap on admitted requests (0: the HBM budget alone)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"svs_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per voxel-iteration of the iterate kernel from the committed ncu summary
    (profiles/iterate_kernel_traffic.txt, line 'bytes_per_voxel_iteration <storage> <value>')."""
    path = os.path.join(ROOT, "profiles", "iterate_kernel_traffic.txt")
    out = {}
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) == 3 and parts[0] == "bytes_per_voxel_iteration":
                out[parts[1]] = float(parts[2])
    except OSError:
        pass
    return out


# ------------------------------------------------------------------------ CPU baselines
def sequence_pair(frames: int):
    """The first forward pair (fixed frame 1, moving frame 0) of the benchmark's cine sequence,
    generated on the host (bitwise the frames the GPU arm generates on the device)."""
    from singleventriclesegmentation_b200 import synthetic
    seq = synthetic.cine_sequence(T=frames, shape=SHAPE, seed=0, device="cpu", first=2)
    a, b = synthetic.sequence_pairs(frames, "forward")[0]
    return seq[a], seq[b]


def oracle_sample(threads: int, pair=None):
    """One bounded sample of the workload on the host with the oracle (C++/OpenMP restatement of
    the reference's path): one 80^3 pair through the full 3-level pyramid with 1 warp of K
    iterations per level. Returns (seconds, extrapolated seconds per full pair, description)."""
    from oracle import oracle as o
    from singleventriclesegmentation_b200 import synthetic
    o.build()
    o.set_threads(threads)
    if pair is None:
        I0, I1, _ = synthetic.frame_pair(SHAPE, seed=0)
    else:
        I0, I1 = pair
    # calibrate the iteration count so that the sample is about 15 s of host work: two probes
    # separate the fixed cost (blur, pyramid, linearisation) from the per-iteration cost
    times = []
    for probe in (4, 36):
        t0 = time.perf_counter()
        o.tvl1_compute(I0, I1, o.SolverParams(max_warps=1, max_outer_iterations=probe), dtype=np.float32)
        times.append(time.perf_counter() - t0)
    per_it = max((times[1] - times[0]) / 32, 1e-6)
    k = int(min(4500, max(36, 15.0 / per_it)))
    P = o.SolverParams(max_warps=1, max_outer_iterations=k)
    t0 = time.perf_counter()
    o.tvl1_compute(I0, I1, P, dtype=np.float32)
    dt = time.perf_counter() - t0
    full = dt * (15 * 300) / (1 * k)
    src = "one 80^3 pair" if pair is None else "the sequence's first forward pair (80^3)"
    desc = (f"{src}, full 3-level pyramid with 1 warp x {k} iterations per level "
            f"(= {k}/4500 of the iterations), extrapolated linearly to 15 x 300")
    return dt, full, desc


def reference_gpu_rate(frames: int):
    """The reference's own CUDA extension (its sources built for sm_100a by oracle/build_ref.sh),
    driven by its solver loop (tvl13d.py:122-255, restated call by call in oracle/ref_driver.py)
    on the sequence's first pair with the full schedule, serial as its processor runs it; timed
    with CUDA events. Returns a dict, or {"unavailable": why}."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        from oracle import ref_driver
        from oracle.oracle import SolverParams
        of = ref_driver.load_reference_module()
    except Exception as e:  # extension not built or not loadable here
        return {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    dev = torch.device("cuda", 0)
    I0, I1 = (torch.from_numpy(x).to(dev) for x in sequence_pair(frames))
    ref_driver.tvl1_compute(of, I0, I1, SolverParams(max_warps=1, max_outer_iterations=3))  # warm-up
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(st)
    ref_driver.tvl1_compute(of, I0, I1, SolverParams())
    e1.record(st)
    torch.cuda.synchronize(dev)
    sec = e0.elapsed_time(e1) / 1000.0
    return {"value": 1.0 / sec, "unit": "pairs/s", "seconds_per_pair": sec,
            "form": "the reference's CUDA extension (built for sm_100a with -maxrregcount=80; the stock build "
                    "returns zero flows on B200) under its own per-operator solver loop, FP32, one 80^3 pair of "
                    "the sequence, full 3 x 15 x 300 schedule"}


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pair = sequence_pair(args.frames)
    for _ in range(args.warmup):
        oracle_sample(threads, pair)
    samples = []
    desc = ""
    for _ in range(args.steps):
        dt, full, desc = oracle_sample(threads, pair)
        samples.append(full)
    per_pair = statistics.mean(samples)
    value = 1.0 / per_pair
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_pair * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(args, "f32"),
        "sample": ("each step times a bounded sample of the workload on the host: " + desc +
                   "; value = 1 / (extrapolated seconds per pair), the rate the 68-pair sequence runs at"),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu_rate(args.frames),
        "note": ("the reference has no CPU implementation of the solver (processor.py:33-34 requires "
                 "CUDA); this arm is the oracle's C++/OpenMP restatement of its kernels on all host threads; "
                 "reference_gpu times the reference's own CUDA extension on the same pair"),
    }
    print(json.dumps(line), flush=True)


def config_dict(args, storage):
    return {"workload": f"cine sequence T={args.frames} of 80^3, {2 * (args.frames - 1)} pairs (fwd+bwd) "
                        f"in one batched solve + 2-mask bidirectional propagation",
            "solver": "3 levels x 15 warps x 300 iterations, conf/flow.yaml defaults",
            "pairs_per_step_per_gpu": 2 * (args.frames - 1), "volume": "80x80x80",
            "storage": storage, "l2": "inputs larger than L2 (state ~6 GB per step)",
            "parallelism": f"replicas x{args.gpus}"}


# ------------------------------------------------------------------------ shared helpers
def tune_plan(plan, storage: str, levels: int = 3, per_class: bool = False):
    """Pick the fastest iterate-kernel variant per pyramid level on the plan's own state (TMA
    and split-role forms); with per_class also per size class of each level."""
    from singleventriclesegmentation_b200 import _lib, autotune
    n = int(_lib.lib().svs_tvl1_num_tiles())
    cands = [t for t in range(1, n + 1) if _lib.tile_info(t)["form"] != "plain"]
    return autotune.tune(plan, storage, levels, candidates=cands, use_cache=False, iters=12, per_class=per_class)


def iterate_roofline(plan, storage: str, level_voxels: int, stream, dev):
    """The dominant kernel (fused iteration, level 0) timed alone on the live state with CUDA
    events: (ms per launch, algorithmic bytes per launch)."""
    import torch
    n_it = 30
    plan.bench_iterations(0, 3)
    torch.cuda.synchronize(dev)
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    plan.bench_iterations(0, n_it)
    e5.record(stream)
    torch.cuda.synchronize(dev)
    it_ms = e4.elapsed_time(e5) / n_it
    # bytes per voxel-iteration: read u 3, p 9, D 6, rc 1, gw 3; write u 3, p 9
    ub = 2 if storage in ("bf16", "f16") else 4
    fb = 4 if storage == "f32" else 2
    return it_ms, level_voxels * (6 * ub + 28 * fb)


def plain_form_rate(dev, seq_dev):
    """The plain GPU form (the reference's per-operator structure, tvl13d.py:122-255, on this
    package's per-operator kernels, FP32) on one 80^3 pair of the sequence with the full
    schedule: pairs/s, timed with CUDA events."""
    import torch
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    s = TVL13DOpticalFlow(3, 15, 300, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                          "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev)
    I0, I1 = seq_dev[1], seq_dev[0]
    z = lambda: (torch.zeros(SHAPE + (3,), device=dev), torch.zeros(SHAPE + (3, 3), device=dev))
    warm = TVL13DOpticalFlow(3, 1, 3, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                             "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev)
    warm.compute_unfused(I0, I1, *z())
    torch.cuda.synchronize(dev)
    u, p = z()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.compute_unfused(I0, I1, u, p)
    e1.record(st)
    torch.cuda.synchronize(dev)
    sec = e0.elapsed_time(e1) / 1000.0
    return {"value": 1.0 / sec, "unit": "pairs/s", "seconds_per_pair": sec,
            "form": "TVL13DOpticalFlow.compute_unfused: per-operator kernels, FP32, one 80^3 pair, full "
                    "3 x 15 x 300 schedule"}


def pair_latency(dev, seq, storage: str, reps: int = 20):
    """Latency of one 80^3 pair alone (the sequence's first forward pair) through
    TVL13DOpticalFlow.compute: p50/p99 over `reps` repetitions, each timed with CUDA events around
    the call and a synchronisation."""
    import torch
    st = torch.cuda.current_stream(dev)
    I0, I1 = torch.from_numpy(seq[1]).to(dev), torch.from_numpy(seq[0]).to(dev)
    solver = _solver(dev, storage)
    for _ in range(3):
        solver.compute(I0, I1)
    torch.cuda.synchronize(dev)
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        solver.compute(I0, I1)
        e1.record(st)
        torch.cuda.synchronize(dev)
        out.append(e0.elapsed_time(e1) / 1000.0)
    a = np.array(out)
    return {"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99)), "reps": reps,
            "storage": storage}


def fp32_storage_rate(dev, d_seq, pairs, args):
    """The same sequence solve with every iteration field stored in FP32 (the plain FP32 form of
    the fused path): pairs/s over 3 timed solves after autotuning, and the level-0 iterate
    kernel's roofline fraction (136 algorithmic bytes per voxel-iteration)."""
    import torch
    solver = _solver(dev, "f32")
    n = len(pairs)
    plan = solver.plan_for([SHAPE] * n)
    if not args.no_autotune:
        tune_plan(plan, "f32")
    flows = [torch.empty(SHAPE + (3,), device=dev) for _ in range(n)]
    I0s, I1s = [d_seq[a] for a, b in pairs], [d_seq[b] for a, b in pairs]
    ms, clocks = _timed_solves(plan, I0s, I1s, flows, 3, 2, dev)
    st = torch.cuda.current_stream(dev)
    it_ms, alg = iterate_roofline(plan, "f32", n * int(np.prod(SHAPE)), st, dev)
    peak, kind = measured_peaks()
    out = {"value": n / (ms / 1000.0), "unit": "pairs/s", "ms_per_step": ms, "steps": 3,
           "what": "the 68 pair solves alone (no mask propagation), FP32 storage of every field",
           "level_tiles": plan.level_tiles()[:3], "launch_ms": it_ms,
           "roofline_frac": alg / (it_ms / 1000.0) / 1e9 / peak, "peak_kind": kind, "clocks": clocks}
    plan.close()
    solver._plans.clear()
    return out


def persistent_form_rate(dev, d_seq, pairs, storage, ref_host):
    """The same 68 pair solves with the persistent iteration loop (svs_tvl1_plan_set_persistent:
    every iteration of a warp at a level in one cooperative launch), on the automatic variants
    (each of which has the persistent form at these sizes): pairs/s over 2 timed solves, the
    graph's kernel nodes, and whether the flows are bitwise those of the headline run (ref_host,
    pinned host copies of its flows)."""
    import torch
    solver = _solver(dev, storage)
    n = len(pairs)
    plan = solver.plan_for([SHAPE] * n)
    plan.set_persistent(True)
    outs = torch.empty((n,) + SHAPE + (3,), dtype=torch.float32, device=dev)
    I0s, I1s = [d_seq[a] for a, b in pairs], [d_seq[b] for a, b in pairs]
    ms, clocks = _timed_solves(plan, I0s, I1s, [outs[i] for i in range(n)], 2, 1, dev)
    plan.check()
    out = {"value": n / (ms / 1000.0), "unit": "pairs/s", "ms_per_step": ms, "steps": 2,
           "what": "the 68 pair solves alone (no mask propagation), persistent iteration loop",
           "graph_kernels_per_solve": plan.graph_kernels, "levels_persistent": plan.level_persistent(3),
           "level_tiles": plan.level_tiles()[:3],
           "bitwise_equal_to_headline_flows": bool(torch.equal(outs.cpu(), ref_host)), "clocks": clocks}
    plan.close()
    solver._plans.clear()
    return out


# ----------------------------------------------------------------- further workloads (1 GPU)
def _solver(dev, storage):
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    return TVL13DOpticalFlow(3, 15, 300, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                             "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev, storage=storage)


def _timed_solves(plan, I0s, I1s, outs, steps, warmup, dev):
    import torch
    for _ in range(warmup):
        plan.solve(I0s, I1s, outs)
    torch.cuda.synchronize(dev)
    st = torch.cuda.current_stream(dev)
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        plan.solve(I0s, I1s, outs)
    e1.record(st)
    torch.cuda.synchronize(dev)
    info = clocks.stop()
    plan.check()
    return e0.elapsed_time(e1) / steps, info


def run_uneven(args):
    """64 frame pairs with volume dims drawn per axis from {40, 48, ..., 128}, blob and sine
    displacement recipe scaled to each volume, all in one batched solve (one CUDA graph), iterate
    variants autotuned per level."""
    import torch
    from singleventriclesegmentation_b200 import synthetic
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(3)
    dims = [tuple(int(v) for v in rng.choice(np.arange(40, 129, 8), size=3)) for _ in range(64)]
    I0s, I1s = [], []
    for i, d in enumerate(dims):
        a, b, _ = synthetic.frame_pair(d, seed=100 + i, device="cuda")
        I0s.append(torch.from_numpy(a).to(dev))
        I1s.append(torch.from_numpy(b).to(dev))
    outs = [torch.empty(d + (3,), device=dev) for d in dims]
    solver = _solver(dev, args.storage)
    plan = solver.plan_for(dims)
    tiles = None if args.no_autotune else tune_plan(plan, args.storage, per_class=True)
    ms, clocks = _timed_solves(plan, I0s, I1s, outs, args.steps, args.warmup, dev)
    vox = sum(int(np.prod(d)) for d in dims)
    it_ms, alg = iterate_roofline(plan, args.storage, vox, torch.cuda.current_stream(dev), dev)
    peak, kind = measured_peaks()
    print(json.dumps({
        "metric": "uneven-size TV-L1 flow pairs/s", "value": len(dims) / (ms / 1000.0), "unit": "pairs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "equivalent_80cube_pairs_per_s": vox / 512000.0 / (ms / 1000.0),
        "dtype": f"f32 math, {args.storage} storage", "data": "synthetic",
        "config": {"workload": "64 pairs, dims per axis uniform on {40,48,...,128} (seed 3), one batched solve",
                   "total_voxels": vox, "storage": args.storage, "level_tiles": plan.level_tiles()[:3],
                   "class_tiles": {str(l): {str(w): t for w, t in c.items()}
                                   for l, c in getattr(plan, "class_tiles", {}).items()}},
        "roofline": {"bound": "hbm", "achieved": alg / (it_ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (it_ms / 1000.0) / 1e9 / peak, "peak_kind": kind, "launch_ms": it_ms},
        "clocks": clocks}), flush=True)


def fp64_gpu_reference(dev, I0, I1):
    """The reference's algorithm in double precision on the GPU (the per-operator plain form on
    float64 tensors), default configuration: the FP64 oracle for large volumes."""
    import torch
    s = _solver(dev, "f32")
    z = tuple(I0.shape)
    u0 = torch.zeros(z + (3,), dtype=torch.float64, device=dev)
    p0 = torch.zeros(z + (3, 3), dtype=torch.float64, device=dev)
    u, _ = s.compute_unfused(I0.double(), I1.double(), u0, p0)
    return u.cpu().numpy()


def run_mixed(args):
    """The 35-frame 80^3 sequence (68 pairs) plus 16 pairs of 128^3 in one batched solve, in the
    16-bit storage modes; end-point error against the FP64 GPU oracle (the per-operator solver in
    double) on a subset (two forward and two backward 80^3 pairs, four 128^3 pairs) and Dice of
    the mask warped with each flow against the mask warped with the oracle's flow."""
    import torch
    from singleventriclesegmentation_b200 import synthetic
    from singleventriclesegmentation_b200.warping import Warp, dice
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    T = T_FRAMES
    seq = torch.from_numpy(synthetic.cine_sequence(T=T, shape=SHAPE, seed=0, device="cuda")).to(dev)
    pairs = synthetic.sequence_pairs(T, "forward") + synthetic.sequence_pairs(T, "backward")
    I0s = [seq[a] for a, b in pairs]
    I1s = [seq[b] for a, b in pairs]
    big = [synthetic.frame_pair((128, 128, 128), seed=200 + i, device="cuda") for i in range(16)]
    I0s += [torch.from_numpy(a).to(dev) for a, b, _ in big]
    I1s += [torch.from_numpy(b).to(dev) for a, b, _ in big]
    dims = [tuple(t.shape) for t in I0s]
    n80 = len(pairs)
    subset = [0, 20, n80 - 1, n80 - 21, n80, n80 + 5, n80 + 10, n80 + 15]
    t0 = time.perf_counter()
    ref = {i: fp64_gpu_reference(dev, I0s[i], I1s[i]) for i in subset}
    oracle_s = time.perf_counter() - t0
    warp = Warp("CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1))
    out = []
    for storage in ["bf16", "f16", "bf16-flow32", "f16-flow32"]:
        outs = [torch.empty(d + (3,), device=dev) for d in dims]
        solver = _solver(dev, storage)
        plan = solver.plan_for(dims)
        if not args.no_autotune:
            tune_plan(plan, storage, per_class=True)   # the 80^3 and the 128^3 pairs are two size classes
        ms, clocks = _timed_solves(plan, I0s, I1s, outs, args.steps, args.warmup, dev)
        epe, dices = {}, {}
        for i in subset:
            u = outs[i].cpu().numpy().astype(np.float64)
            e = np.sqrt(((u - ref[i]) ** 2).sum(-1))
            key = "x".join(map(str, dims[i])) + f"#{i}"
            epe[key] = {"mean": float(e.mean()), "p99": float(np.percentile(e, 99)), "max": float(e.max())}
            m = torch.from_numpy(synthetic.ellipsoid_mask(dims[i], (15, 12, 10))).to(dev)[None, None]
            w_ours = warp(m, outs[i][None]) > 0.5
            w_ref = warp(m, torch.from_numpy(ref[i].astype(np.float32)).to(dev)[None]) > 0.5
            dices[key] = dice(w_ours[0, 0].float(), w_ref[0, 0].float())
        vox = sum(int(np.prod(d)) for d in dims)
        out.append({"storage": storage, "pairs_per_s": len(dims) / (ms / 1000.0), "ms_per_step": ms,
                    "equivalent_80cube_pairs_per_s": vox / 512000.0 / (ms / 1000.0), "epe_vs_fp64_oracle": epe,
                    "warped_mask_dice_vs_fp64_oracle": dices, "level_tiles": plan.level_tiles()[:3],
                    "class_tiles": {str(l): {str(w): t for w, t in c.items()}
                                    for l, c in getattr(plan, "class_tiles", {}).items()},
                    "clocks": clocks})
        plan.close()
        solver._plans.clear()
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "mixed-precision TV-L1 flow, 68 x 80^3 + 16 x 128^3 pairs",
                      "unit": "pairs/s", "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
                      "oracle": "FP64 on the GPU: the reference's per-operator algorithm on float64 tensors "
                                "(TVL13DOpticalFlow.compute_unfused, svs_*_f64 kernels), default configuration",
                      "oracle_seconds": oracle_s,
                      "results": out}), flush=True)


def run_serving(args):
    """Poisson request streams (one request = a cine sequence with T uniform in 12..35 and dims per
    axis uniform on {64, 72, ..., 128}) through the continuous-batching server (bf16-flow32 storage
    unless --storage is given): p50/p99 latency from submit to flows and masks on the host, and
    throughput, per arrival rate."""
    import torch
    from singleventriclesegmentation_b200 import synthetic
    from singleventriclesegmentation_b200.serving import FlowServer
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    storage = args.storage if args.storage != "f16-flow32" else "bf16-flow32"
    results = []
    for rate in [float(r) for r in args.rates.split(",")]:
        reqs = []
        rng = np.random.default_rng(int(rate * 1000) + 1)
        t = 0.0
        for _ in range(args.requests):
            t += rng.exponential(1.0 / rate)
            T = int(rng.integers(12, 36))
            dims = tuple(int(v) for v in rng.choice(np.arange(64, 129, 8), size=3))
            reqs.append((t, T, dims))
        data = []
        for j, (_, T, dims) in enumerate(reqs):
            frames = torch.from_numpy(synthetic.cine_sequence(T=T, shape=dims, seed=j, device="cuda")).pin_memory()
            masks = torch.from_numpy(np.stack([synthetic.ellipsoid_mask(dims, (15, 12, 10)),
                                               synthetic.ellipsoid_mask(dims, (13, 12, 10))])).pin_memory()
            data.append((frames, masks, (0, min(12, T - 1))))
        server = FlowServer(budget_bytes=100 << 30, storage=storage, device=dev, max_active=args.max_active or None)
        t0 = time.perf_counter()
        futs = []
        for (ta, _, _), (frames, masks, mt) in zip(reqs, data):
            delay = ta - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            futs.append(server.submit(frames, masks, mt))
        for f in futs:
            f.result()
        server.close()
        st = server.stats()
        pairs = sum(2 * (T - 1) for _, T, _ in reqs)
        eq80 = sum(2 * (T - 1) * int(np.prod(d)) for _, T, d in reqs) / 512000.0
        span = st["completed"] / st["throughput_seq_per_s"] if st["throughput_seq_per_s"] else float("nan")
        results.append({"rate_per_s": rate, "requests": len(reqs), "p50_s": st["p50_s"], "p99_s": st["p99_s"],
                        "mean_s": st["mean_s"], "throughput_seq_per_s": st["throughput_seq_per_s"],
                        "throughput_pairs_per_s": pairs / span,
                        "throughput_80cube_equiv_pairs_per_s": eq80 / span, "max_concurrent": st["max_concurrent"],
                        "batches": st["batches"], "mixed_batches": st["mixed_batches"],
                        "sizes": [[T] + list(d) for _, T, d in reqs]})
    print(json.dumps({"metric": "serving: per-sequence latency p50/p99 and throughput", "unit": "s",
                      "storage": storage, "data": "synthetic", "budget_bytes": 100 << 30,
                      "max_active": args.max_active,
                      "results": results}), flush=True)


def run_latency(args):
    """Latency: one 80^3 pair (the blob / sine-displacement pair, default configuration) solved
    alone through TVL13DOpticalFlow.compute, --reps times, and the 68-pair sequence solve plus mask
    propagation, max(5, reps // 5) times; each repetition timed with CUDA events around the call
    and a synchronisation; p50/p99/mean in seconds."""
    import torch
    from singleventriclesegmentation_b200 import synthetic
    from singleventriclesegmentation_b200.warping import Warp, propagate_batched
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    st = torch.cuda.current_stream(dev)

    def timed(fn, reps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            torch.cuda.synchronize(dev)
            out.append(e0.elapsed_time(e1) / 1000.0)
        a = np.array(out)
        return {"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99)),
                "mean_s": float(a.mean()), "reps": reps}

    I0, I1, _ = synthetic.frame_pair(SHAPE, seed=0, device="cuda")
    I0, I1 = torch.from_numpy(I0).to(dev), torch.from_numpy(I1).to(dev)
    solver = _solver(dev, args.storage)
    pair = timed(lambda: solver.compute(I0, I1), args.reps, 3)

    T = T_FRAMES
    seq = torch.from_numpy(synthetic.cine_sequence(T=T, shape=SHAPE, seed=0, device="cuda")).to(dev)
    pairs = synthetic.sequence_pairs(T, "forward") + synthetic.sequence_pairs(T, "backward")
    masks = torch.from_numpy(np.stack([synthetic.ellipsoid_mask(SHAPE, (15, 12, 10)),
                                       synthetic.ellipsoid_mask(SHAPE, (13, 12, 10))])[:, None]).to(dev)
    flows = torch.empty((len(pairs),) + SHAPE + (3,), device=dev)
    plan = solver.plan_for([SHAPE] * len(pairs))
    warp = Warp("CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1))
    fwd_idx = list(range(MASK_T0, MASK_T1))
    bwd_idx = [(T - 1) + (T - 1 - t) for t in range(MASK_T1, MASK_T0, -1)]

    def sequence():
        plan.solve([seq[a] for a, b in pairs], [seq[b] for a, b in pairs], [flows[i] for i in range(len(pairs))])
        propagate_batched(warp, masks, torch.stack([flows[fwd_idx], flows[bwd_idx]], dim=1))

    seq_lat = timed(sequence, max(5, args.reps // 5), 2)
    print(json.dumps({"metric": "latency p50/p99", "unit": "s", "storage": args.storage, "data": "synthetic",
                      "pair_80cube": pair, "sequence_35x80cube_68pairs_with_masks": seq_lat}), flush=True)


# ------------------------------------------------------------------------------ our arm
def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload != "sequence":
        {"uneven": run_uneven, "mixed": run_mixed, "serving": run_serving, "latency": run_latency}[args.workload](args)
        return
    import torch
    import torch.distributed as dist
    from singleventriclesegmentation_b200 import _lib, synthetic
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    from singleventriclesegmentation_b200.warping import Warp, propagate_batched

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    # ----- data: one synthetic cine sequence (host, pinned) and its pair list
    T = args.frames
    seq = synthetic.cine_sequence(T=T, shape=SHAPE, seed=0, device=str(dev))
    m0 = synthetic.ellipsoid_mask(SHAPE, (15, 12, 10))
    m1 = synthetic.ellipsoid_mask(SHAPE, (13, 12, 10))
    pairs = synthetic.sequence_pairs(T, "forward") + synthetic.sequence_pairs(T, "backward")
    host_seq = torch.from_numpy(seq).pin_memory()
    host_masks = torch.from_numpy(np.stack([m0, m1])[:, None]).pin_memory()
    n_pairs = len(pairs)
    host_flows = torch.empty((n_pairs,) + SHAPE + (3,), dtype=torch.float32).pin_memory()
    nsteps = MASK_T1 - MASK_T0
    host_chain = torch.empty((nsteps + 1, 2, 1) + SHAPE, dtype=torch.float32).pin_memory()

    solver = TVL13DOpticalFlow(3, 15, 300, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                               "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev, storage=args.storage)
    warp = Warp("CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1))
    d_seq = host_seq.to(dev)
    d_masks = host_masks.to(dev)
    flows = torch.empty((n_pairs,) + SHAPE + (3,), dtype=torch.float32, device=dev)
    plan = solver.plan_for([SHAPE] * n_pairs)
    if not args.no_autotune:
        tune_plan(plan, args.storage)
    fwd_idx = list(range(MASK_T0, MASK_T1))                       # forward pairs t -> t+1
    bwd_idx = [(T - 1) + (T - 1 - t) for t in range(MASK_T1, MASK_T0, -1)]  # backward pairs t -> t-1

    def step(seq_dev, masks_dev):
        I0s = [seq_dev[a] for a, b in pairs]
        I1s = [seq_dev[b] for a, b in pairs]
        plan.solve(I0s, I1s, [flows[i] for i in range(n_pairs)])
        f = torch.stack([flows[fwd_idx], flows[bwd_idx]], dim=1)   # [steps, 2, Z,Y,X,3]
        return propagate_batched(warp, masks_dev, f)

    stream = torch.cuda.current_stream(dev)
    # warm-up (includes graph capture on the first call)
    for _ in range(args.warmup):
        chain = step(d_seq, d_masks)
    torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = ClockSampler(local)
    # ----- device-resident timed region (an event between steps gives the per-sequence latency)
    launches0 = _lib.launch_count()
    barrier()
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for i in range(args.steps):
        chain = step(d_seq, d_masks)
        ev[i + 1].record(stream)
    barrier()
    clock_info = clocks.stop()
    e0, e1 = ev[0], ev[-1]
    ms = max_over_ranks(e0.elapsed_time(e1))
    step_s = np.array([ev[i].elapsed_time(ev[i + 1]) / 1000.0 for i in range(args.steps)])
    launches = _lib.launch_count() - launches0
    value = world * n_pairs * args.steps / (ms / 1000.0)

    # ----- end to end through the public API with host buffers
    barrier()
    h2d = host_seq.numel() * 4 + host_masks.numel() * 4
    d2h = host_flows.numel() * 4 + host_chain.numel() * 4
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        s_dev = host_seq.to(dev, non_blocking=True)
        m_dev = host_masks.to(dev, non_blocking=True)
        chain = step(s_dev, m_dev)
        host_flows.copy_(flows, non_blocking=True)
        host_chain.copy_(chain, non_blocking=True)
    e3.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    e2e_value = world * n_pairs * args.steps / (ms_e2e / 1000.0)

    # ----- the dominant kernel (fused iteration, level 0) timed alone on the live state
    vox0 = n_pairs * int(np.prod(SHAPE))
    it_ms, alg_bytes = iterate_roofline(plan, args.storage, vox0, stream, dev)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (it_ms / 1000.0) / 1e9
    traffic_pv = profiled_traffic().get(args.storage)

    # the workload's own end metrics (warping.py:245-270): each propagated end mask against the
    # mask given at that end (two different synthetic annotations, so these are not parity values)
    from singleventriclesegmentation_b200.warping import dice, hausdorff
    fm = (chain[-1, 0, 0] > 0.5).float()
    bm = (chain[-1, 1, 0] > 0.5).float()
    mask_metrics = {"dice_fwd": dice(fm, d_masks[1, 0]), "hd_fwd": hausdorff(fm, d_masks[1, 0]),
                    "dice_bwd": dice(bm, d_masks[0, 0]), "hd_bwd": hausdorff(bm, d_masks[0, 0]),
                    "what": "propagated end mask vs the mask given at that end (t=12 and t=0 annotations)"}

    latency = None
    if rank == 0 and world == 1 and not args.no_latency:
        latency = {"sequence_68pairs_with_masks": {"p50_s": float(np.percentile(step_s, 50)),
                                                   "p99_s": float(np.percentile(step_s, 99)),
                                                   "reps": int(args.steps),
                                                   "from": "the timed steps above (events between steps)"},
                   "pair_80cube": pair_latency(dev, seq, args.storage, reps=20)}

    fp32 = None
    if rank == 0 and world == 1 and not args.no_fp32:
        fp32 = fp32_storage_rate(dev, d_seq, pairs, args)

    persistent = None
    if rank == 0 and world == 1 and not args.no_persistent:
        persistent = persistent_form_rate(dev, d_seq, pairs, args.storage, host_flows)

    plain = None
    if rank == 0 and world == 1 and not args.no_plain_form:
        plain = plain_form_rate(dev, d_seq)
        plain["speedup_of_value"] = value / plain["value"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        dt, full, desc = oracle_sample(threads)
        cpu = {"value": 1.0 / full, "unit": "pairs/s", "cores": threads, "kind": "port", "sample": desc,
               "sample_seconds": dt}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == "f32" else f"f32 math, {args.storage} storage",
            "level_tiles": plan.level_tiles()[:3],
            "data": "synthetic", "config": config_dict(args, args.storage),
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None if traffic_pv is None else traffic_pv * vox0,
                         "kernel": "iterate kernel (fused primal-dual iteration, variant %d), level 0"
                                   % plan.level_tiles()[0],
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": it_ms},
            "cpu_baseline": cpu, "plain_gpu_form": plain, "clocks": clock_info, "latency": latency,
            "fp32_storage": fp32, "persistent_form": persistent, "compute_metrics": mask_metrics,
            "graph_kernels_per_solve": plan.graph_kernels,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
