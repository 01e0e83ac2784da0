"""Benchmark of the fused batched TV-L1 flow path: 80^3 frame pairs per second.

Workload (one step): a synthetic cine sequence of T = 35 frames of 80^3 voxels; all 34 forward
and 34 backward consecutive pairs (68 independent solves, the reference's default solver
configuration: 3 levels x 15 warps x 300 iterations) run as ONE batched solve (one CUDA graph),
followed by the bidirectional propagation of the two end masks (t = 0 and t = 12) through the
flows. The sequence stands in for the reference's 80^3 x 35-frame cine MRI data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--storage f16-flow32|f32|...] [--impl reference]

Multi-GPU: one process per GPU (torchrun); every rank solves its own sequence (replicas, weak
scaling, no collective on the data path); NCCL is used only for the barrier and the max-over-ranks
timing. Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
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
    ap.add_argument("--frames", type=int, default=T_FRAMES)
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
def oracle_sample(threads: int):
    """One bounded sample of the workload on the host with the oracle (C++/OpenMP restatement of
    the reference's path): one 80^3 pair through the full 3-level pyramid with 1 warp of K
    iterations per level. Returns (seconds, extrapolated seconds per full pair, description)."""
    from oracle import oracle as o
    from singleventriclesegmentation_b200 import synthetic
    o.build()
    o.set_threads(threads)
    I0, I1, _ = synthetic.frame_pair(SHAPE, seed=0)
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
    desc = (f"one 80^3 pair, full 3-level pyramid with 1 warp x {k} iterations per level "
            f"(= {k}/4500 of the iterations), extrapolated linearly to 15 x 300")
    return dt, full, desc


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_sample(threads)
    samples = []
    desc = ""
    for _ in range(args.steps):
        dt, full, desc = oracle_sample(threads)
        samples.append(full)
    per_pair = statistics.mean(samples)
    value = 1.0 / per_pair
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_pair * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(args, "f32"),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference has no CPU implementation of the solver (processor.py:33-34 requires "
                 "CUDA); this arm is the oracle's C++/OpenMP restatement of its kernels on all host threads"),
    }
    print(json.dumps(line), flush=True)


def config_dict(args, storage):
    return {"workload": f"cine sequence T={args.frames} of 80^3, {2 * (args.frames - 1)} pairs (fwd+bwd) "
                        f"in one batched solve + 2-mask bidirectional propagation",
            "solver": "3 levels x 15 warps x 300 iterations, conf/flow.yaml defaults",
            "pairs_per_step_per_gpu": 2 * (args.frames - 1), "volume": "80x80x80",
            "storage": storage, "l2": "inputs larger than L2 (state ~6 GB per step)",
            "parallelism": f"replicas x{args.gpus}"}


# ------------------------------------------------------------------------------ our arm
def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
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
    # ----- device-resident timed region
    launches0 = _lib.launch_count()
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        chain = step(d_seq, d_masks)
    e1.record(stream)
    barrier()
    clock_info = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
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
    ub = 2 if args.storage in ("bf16", "f16") else 4
    fb = 4 if args.storage == "f32" else 2
    bpv = 6 * ub + 28 * fb
    vox0 = n_pairs * int(np.prod(SHAPE))
    alg_bytes = vox0 * bpv
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (it_ms / 1000.0) / 1e9
    traffic_pv = profiled_traffic().get(args.storage)

    # parity summary of this run (masks): Dice/HD of the propagated end masks
    from singleventriclesegmentation_b200.warping import dice, hausdorff
    fm = (chain[-1, 0, 0] > 0.5).float()
    bm = (chain[-1, 1, 0] > 0.5).float()
    mask_metrics = {"dice_fwd": dice(fm, d_masks[1, 0]), "hd_fwd": hausdorff(fm, d_masks[1, 0]),
                    "dice_bwd": dice(bm, d_masks[0, 0]), "hd_bwd": hausdorff(bm, d_masks[0, 0])}

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
                         "kernel": "iterate_kernel (fused primal-dual iteration), level 0",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": it_ms},
            "cpu_baseline": cpu, "clocks": clock_info, "masks": mask_metrics,
            "graph_kernels_per_solve": plan.graph_kernels,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
