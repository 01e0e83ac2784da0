"""A continuous-batching request loop for whole cine sequences.

Each request is one sequence [T, Z, Y, X] (any size; optional end masks). The server admits
requests while their device state fits a fixed HBM budget (and at most max_active at once),
gives each admitted request its own
CUDA stream and a solver plan (pyramids, dual state and the captured graph stay on the device
for the whole sequence), and starts the next waiting request as soon as an earlier one finishes
and its memory is released, while the others keep running: the work of all admitted requests
overlaps on the device. A request's result is its forward and backward flows (and propagated
masks), copied back to pinned host memory; its latency runs from submit() to that copy being
complete.

Every request is solved by its own plan with the same kernels on the same data, so its result is
the same alone and in any mix (tests/test_gpu_serving.py checks it bitwise).

    server = FlowServer(budget_bytes=40 << 30)
    fut = server.submit(frames)          # frames: [T,Z,Y,X] float32 (host or device)
    flows_fwd, flows_bwd, masks = fut.result()
    server.close(); server.stats()       # p50 / p99 latency, throughput
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Tuple

import numpy as np
import torch

from .tvl13d import SolverPlan, TVL13DOpticalFlow
from .warping import Warp, propagate_batched


@dataclass
class _Request:
    rid: int
    frames: torch.Tensor
    masks: Optional[torch.Tensor]
    mask_t: Tuple[int, int]
    future: cf.Future
    t_submit: float
    bytes_needed: int = 0
    # filled at admission
    plan: Optional[SolverPlan] = None
    stream: Optional[torch.cuda.Stream] = None
    done_event: Optional[torch.cuda.Event] = None
    out: Dict[str, torch.Tensor] = field(default_factory=dict)
    t_admit: float = 0.0


def _pairs(T: int):
    fwd = [(t + 1, t) for t in range(T - 1)]
    bwd = [(T - 2 - j, T - 1 - j) for j in range(T - 1)]
    return fwd + bwd


class FlowServer:
    """Admission by HBM budget, one stream per admitted request, results on the host."""

    def __init__(self, budget_bytes: int = 40 << 30, storage: str = "f16-flow32", device=None,
                 solver_args: Optional[dict] = None, poll_s: float = 0.002, max_active: int = 2):
        """max_active caps the requests on the device at once (memory permitting): one batched
        sequence already fills the GPU, so more overlap adds latency to every request without
        adding throughput; two keep the device busy across one request's host-side set-up."""
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.budget = int(budget_bytes)
        self.max_active = max(1, int(max_active))
        self.storage = storage
        args = dict(num_scales=3, max_warps=15, max_outer_iterations=300, weight_matching=1.0, weight_tv=0.025,
                    primaldual_algorithm_type=2, primaldual_algorithm_params=(0.5, 0.5, 0.25, 1.0),
                    use_anisotropic_diff=True, anisotropic_diff_params=(5.0, 0.5), use_gaussian_blur=True,
                    gaussian_blur_sigma=1.0, interpolation_type="CUBIC_HERMITESPLINE", boundary_type="MIRROR",
                    length_type="numDofs", length=(1, 1, 1))
        args.update(solver_args or {})
        self.solver = TVL13DOpticalFlow(device=self.device, storage=storage, max_cached_plans=0, **args)
        self.warp = Warp(args["interpolation_type"], args["boundary_type"], args["length_type"], args["length"])
        self._waiting: Deque[_Request] = collections.deque()
        self._active: List[_Request] = []
        self._idle_plans: Dict[tuple, List[SolverPlan]] = collections.defaultdict(list)
        self._in_use = 0
        self._lock = threading.Lock()
        self._wake = threading.Event()
        self._stop = False
        self._next_id = 0
        self._poll = poll_s
        self.latencies: List[float] = []
        self.completed = 0
        self._t0: Optional[float] = None
        self._t_last = 0.0
        self.max_concurrent = 0
        self._thread = threading.Thread(target=self._loop, name="svs-flow-server", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------------ public API
    def submit(self, frames: torch.Tensor, masks: Optional[torch.Tensor] = None,
               mask_t: Tuple[int, int] = (0, 0)) -> cf.Future:
        """Queue one sequence. frames [T,Z,Y,X] float32; masks [2,Z,Y,X] (at mask_t[0] and
        mask_t[1]) are propagated forward from the first and backward from the second."""
        if frames.dim() != 4 or frames.shape[0] < 2:
            raise ValueError("frames must be [T,Z,Y,X] with T >= 2")
        fut: cf.Future = cf.Future()
        with self._lock:
            rid = self._next_id
            self._next_id += 1
            now = time.perf_counter()
            if self._t0 is None:
                self._t0 = now
            req = _Request(rid, frames, masks, mask_t, fut, now)
            req.bytes_needed = self._estimate(frames.shape)
            if req.bytes_needed > self.budget:
                fut.set_exception(MemoryError(f"request needs {req.bytes_needed} B of device state; budget is {self.budget} B"))
                return fut
            self._waiting.append(req)
        self._wake.set()
        return fut

    def close(self, wait: bool = True) -> None:
        if wait:
            while True:
                with self._lock:
                    if not self._waiting and not self._active:
                        break
                time.sleep(self._poll)
        self._stop = True
        self._wake.set()
        self._thread.join()
        for plans in self._idle_plans.values():
            for p in plans:
                p.close()
        self._idle_plans.clear()

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        span = (self._t_last - self._t0) if self._t0 is not None else 0.0
        return {"completed": self.completed, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "throughput_seq_per_s": self.completed / span if span > 0 else 0.0,
                "max_concurrent": self.max_concurrent}

    # ---------------------------------------------------------------- internals
    def _estimate(self, shape) -> int:
        """Device bytes of one request's plan (state of all its pairs) plus its buffers."""
        T, nz, ny, nx = (int(v) for v in shape)
        ub = 2 if self.storage in ("bf16", "f16") else 4
        fb = 4 if self.storage == "f32" else 2
        per_voxel = 20 + 6 * ub + 28 * fb + 10 * 4 + 12  # float images/gradients, state, io buffers
        vox = 0
        z, y, x = nz, ny, nx
        for _ in range(self.solver.num_scales):
            pitch = (x + 7) // 8 * 8
            vox += z * y * pitch
            z, y, x = (z + 1) // 2, (y + 1) // 2, (x + 1) // 2
        return 2 * (T - 1) * vox * per_voxel + T * nz * ny * nx * 4 * 6

    def _key(self, frames: torch.Tensor) -> tuple:
        T, nz, ny, nx = frames.shape
        return (T, nz, ny, nx)

    def _admit(self, req: _Request) -> None:
        T, nz, ny, nx = (int(v) for v in req.frames.shape)
        key = self._key(req.frames)
        idle = self._idle_plans.get(key)
        plan = idle.pop() if idle else SolverPlan(self.solver.params(), [(nz, ny, nx)] * (2 * (T - 1)), self.device)
        req.plan = plan
        req.stream = torch.cuda.Stream(self.device)
        req.t_admit = time.perf_counter()
        self._in_use += req.bytes_needed
        with torch.cuda.stream(req.stream):
            frames = req.frames.to(self.device, non_blocking=True).float().contiguous()
            pairs = _pairs(T)
            flows = torch.empty((len(pairs), nz, ny, nx, 3), dtype=torch.float32, device=self.device)
            plan.solve([frames[a] for a, b in pairs], [frames[b] for a, b in pairs],
                       [flows[i] for i in range(len(pairs))], stream=req.stream.cuda_stream)
            out = {"flows": torch.empty(flows.shape, dtype=torch.float32, pin_memory=True)}
            out["flows"].copy_(flows, non_blocking=True)
            if req.masks is not None:
                t0, t1 = req.mask_t
                fwd_idx = list(range(t0, t1))
                bwd_idx = [(T - 1) + (T - 1 - t) for t in range(t1, t0, -1)]
                if fwd_idx:
                    m = req.masks.to(self.device, non_blocking=True).float().reshape(2, 1, nz, ny, nx).contiguous()
                    f = torch.stack([flows[fwd_idx], flows[bwd_idx]], dim=1)
                    chain = propagate_batched(self.warp, m, f)
                    out["masks"] = torch.empty(chain.shape, dtype=torch.float32, pin_memory=True)
                    out["masks"].copy_(chain, non_blocking=True)
            out["_device"] = (frames, flows)  # kept alive until the request's stream is done
            req.out = out
            req.done_event = torch.cuda.Event()
            req.done_event.record(req.stream)
        self._active.append(req)
        self.max_concurrent = max(self.max_concurrent, len(self._active))

    def _finish(self, req: _Request) -> None:
        now = time.perf_counter()
        self._in_use -= req.bytes_needed
        key = self._key(req.frames)
        self._idle_plans[key].append(req.plan)
        self.latencies.append(now - req.t_submit)
        self.completed += 1
        self._t_last = now
        T = req.frames.shape[0]
        flows = req.out["flows"]
        req.future.set_result((flows[: T - 1], flows[T - 1:], req.out.get("masks")))

    def _release_idle(self, need: int) -> None:
        """Free cached plans (LRU order is not tracked: any idle plan) until `need` fits."""
        for key in list(self._idle_plans):
            while self._idle_plans[key] and self._in_use + self._idle_bytes() + need > self.budget:
                self._idle_plans[key].pop().close()

    def _idle_bytes(self) -> int:
        return sum(p.device_bytes for plans in self._idle_plans.values() for p in plans)

    def _loop(self) -> None:
        torch.cuda.set_device(self.device)
        while not self._stop:
            progressed = False
            # completions first: they free memory for admissions
            for req in list(self._active):
                if req.done_event.query():
                    self._active.remove(req)
                    try:
                        self._finish(req)
                    except Exception as e:  # pragma: no cover - surfaced to the caller
                        req.future.set_exception(e)
                    progressed = True
            with self._lock:
                while self._waiting and len(self._active) < self.max_active:
                    req = self._waiting[0]
                    if self._in_use + req.bytes_needed > self.budget:
                        break
                    self._release_idle(req.bytes_needed)
                    self._waiting.popleft()
                    try:
                        self._admit(req)
                    except Exception as e:
                        self._in_use -= req.bytes_needed if req.plan is not None else 0
                        req.future.set_exception(e)
                    progressed = True
            if not progressed:
                self._wake.wait(self._poll)
                self._wake.clear()


def poisson_requests(rate: float, duration_s: float, seed: int = 0, t_range=(12, 35), dim_range=(64, 128),
                     dim_step: int = 8):
    """Arrival times and sizes of a Poisson request stream (the serving configuration: T uniform
    in 12-35, dims per axis uniform in 64-128)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration_s:
            return out
        T = int(rng.integers(t_range[0], t_range[1] + 1))
        dims = tuple(int(v) for v in rng.choice(np.arange(dim_range[0], dim_range[1] + 1, dim_step), size=3))
        out.append((t, T, dims))
