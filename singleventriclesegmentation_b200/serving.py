"""A continuous-batching request loop for cine sequences, batched at the granularity of frame
pairs.

Each request is one sequence [T, Z, Y, X] (any size; optional end masks). The server admits
requests while their device buffers (frames, flows, mask chains) and the solver plans fit a fixed
HBM budget, and queues the 2(T-1) frame pairs of every admitted request. A batch takes pairs from
the head of that queue, from as many requests as fit, up to a voxel target that fills the GPU,
and runs as one batched solve on one of two plans that are re-targeted to each batch without
allocating (svs_tvl1_plan_retarget): while one batch runs, the next is formed and launched on the
other plan, so pairs of requests that arrived while others were on the GPU join the next batch
and their work overlaps on the device. When the last pair of a request is done, its masks are
propagated on the device and its flows and masks are copied to pinned host memory; its latency
runs from submit() to that copy being complete. Pyramids, dual state and the captured solve
graphs stay on the device in the plans.

Every pair of a batch is solved by the same kernels on the same data whatever else is in the
batch (the iterate-kernel variants a batch's sizes may select all give bitwise the same result),
so a request's result is the same alone and in any mix (tests/test_gpu_serving.py checks it
bitwise).

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
    dims: Tuple[int, int, int] = (0, 0, 0)
    pairs: List[Tuple[int, int]] = field(default_factory=list)
    frames_dev: Optional[torch.Tensor] = None
    frames_ready: Optional[torch.cuda.Event] = None
    flows_dev: Optional[torch.Tensor] = None
    done: int = 0
    out: Dict[str, torch.Tensor] = field(default_factory=dict)
    final_event: Optional[torch.cuda.Event] = None
    t_admit: float = 0.0


@dataclass
class _Slot:
    """One of the server's plans with the batch it is running."""
    plan: Optional[SolverPlan] = None
    stream: Optional[torch.cuda.Stream] = None
    event: Optional[torch.cuda.Event] = None
    batch: List[Tuple[_Request, int]] = field(default_factory=list)


def _pairs(T: int):
    fwd = [(t + 1, t) for t in range(T - 1)]
    bwd = [(T - 2 - j, T - 1 - j) for j in range(T - 1)]
    return fwd + bwd


def state_bytes_per_voxel(storage: str, levels: int = 3) -> float:
    """Device bytes of a plan per level-0 voxel (the arena layout of svs_tvl1_plan_create: images,
    linearisation, tensor, ping-pong flow and dual field per level, raw frames and outputs at
    level 0), with the pyramid's 1 + 1/8 + ... factor."""
    ub = 2 if storage in ("bf16", "f16") else 4
    sb = 4 if storage == "f32" else 2
    per_level = 2 * 4 + 16 + 6 * sb + sb + 3 * sb + 2 * 3 * ub + 2 * 9 * sb
    level0_extra = 2 * 4 + 2 * 12 + 36
    pyr = sum(0.125 ** l for l in range(levels))
    return per_level * pyr + level0_extra


class FlowServer:
    """Admission by HBM budget, pair-granularity batches on two re-targeted plans, results on the
    host."""

    def __init__(self, budget_bytes: int = 40 << 30, storage: str = "f16-flow32", device=None,
                 solver_args: Optional[dict] = None, poll_s: float = 0.002, max_active: Optional[int] = None,
                 batch_voxels: int = 68 * 80 ** 3, max_batch_pairs: int = 160, num_plans: int = 2):
        """batch_voxels: the level-0 voxels a batch aims at (the default is the 68-pair 80^3
        sequence, which fills a B200); max_batch_pairs caps its pair count; max_active optionally
        caps the admitted requests (None: the budget alone decides)."""
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.budget = int(budget_bytes)
        self.max_active = None if max_active is None else max(1, int(max_active))
        self.storage = storage
        self.batch_voxels = int(batch_voxels)
        self.max_batch_pairs = int(max_batch_pairs)
        args = dict(num_scales=3, max_warps=15, max_outer_iterations=300, weight_matching=1.0, weight_tv=0.025,
                    primaldual_algorithm_type=2, primaldual_algorithm_params=(0.5, 0.5, 0.25, 1.0),
                    use_anisotropic_diff=True, anisotropic_diff_params=(5.0, 0.5), use_gaussian_blur=True,
                    gaussian_blur_sigma=1.0, interpolation_type="CUBIC_HERMITESPLINE", boundary_type="MIRROR",
                    length_type="numDofs", length=(1, 1, 1))
        args.update(solver_args or {})
        self.solver_args = args
        self.solver = TVL13DOpticalFlow(device=self.device, storage=storage, max_cached_plans=0, **args)
        self.warp = Warp(args["interpolation_type"], args["boundary_type"], args["length_type"], args["length"])
        # each plan holds one batch: at most batch_voxels of level-0 voxels (plus one pair over
        # the target, a batch never being empty) with 25% for pitch rounding and per-pair slack
        self.arena_bytes = int(1.25 * state_bytes_per_voxel(storage, args["num_scales"]) * self.batch_voxels) + (64 << 20)
        self._slots = [_Slot() for _ in range(max(1, int(num_plans)))]
        self._waiting: Deque[_Request] = collections.deque()
        self._active: List[_Request] = []
        self._finishing: List[_Request] = []
        self._pairq: Deque[Tuple[_Request, int]] = collections.deque()
        self._copy_stream = torch.cuda.Stream(self.device)
        self._final_stream = torch.cuda.Stream(self.device)
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
        self.batches = 0
        self.mixed_batches = 0   # batches holding pairs of more than one request
        self._error: Optional[BaseException] = None
        self._thread = threading.Thread(target=self._loop, name="svs-flow-server", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------------ public API
    def plan_bytes(self) -> int:
        """Device bytes the server's plans take out of the budget."""
        return len(self._slots) * self.arena_bytes

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
            req.bytes_needed = self._estimate(frames.shape, masks is not None, mask_t)
            if req.bytes_needed > self.budget - self.plan_bytes():
                fut.set_exception(MemoryError(
                    f"request needs {req.bytes_needed} B of device buffers; the budget leaves "
                    f"{self.budget - self.plan_bytes()} B beside the plans"))
                return fut
            self._waiting.append(req)
        self._wake.set()
        return fut

    def close(self, wait: bool = True) -> None:
        if wait:
            while True:
                with self._lock:
                    if not self._waiting and not self._active and not self._finishing:
                        break
                if self._error is not None or not self._thread.is_alive():
                    break
                time.sleep(self._poll)
        self._stop = True
        self._wake.set()
        self._thread.join()
        for sl in self._slots:
            if sl.plan is not None:
                sl.plan.close()
                sl.plan = None

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        span = (self._t_last - self._t0) if self._t0 is not None else 0.0
        return {"completed": self.completed, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
                "throughput_seq_per_s": self.completed / span if span > 0 else 0.0,
                "max_concurrent": self.max_concurrent, "batches": self.batches,
                "mixed_batches": self.mixed_batches}

    # ---------------------------------------------------------------- internals
    def _estimate(self, shape, with_masks: bool = False, mask_t=(0, 0)) -> int:
        """Device bytes of one request's buffers: frames, flows, and the two mask chains."""
        T, nz, ny, nx = (int(v) for v in shape)
        vox = nz * ny * nx
        steps = max(0, mask_t[1] - mask_t[0])
        return T * vox * 4 + 2 * (T - 1) * vox * 12 + ((steps + 1) * 2 * vox * 4 + 2 * vox * 4 if with_masks else 0)

    def _admit(self, req: _Request) -> None:
        T, nz, ny, nx = (int(v) for v in req.frames.shape)
        req.dims = (nz, ny, nx)
        req.pairs = _pairs(T)
        req.t_admit = time.perf_counter()
        self._in_use += req.bytes_needed
        with torch.cuda.stream(self._copy_stream):
            req.frames_dev = req.frames.to(self.device, non_blocking=True).float().contiguous()
            req.flows_dev = torch.empty((len(req.pairs), nz, ny, nx, 3), dtype=torch.float32, device=self.device)
            req.frames_ready = torch.cuda.Event()
            req.frames_ready.record(self._copy_stream)
        for i in range(len(req.pairs)):
            self._pairq.append((req, i))
        self._active.append(req)
        self.max_concurrent = max(self.max_concurrent, len(self._active))

    def _launch(self, sl: _Slot) -> None:
        """Form the next batch from the head of the pair queue and run it on slot `sl`."""
        batch: List[Tuple[_Request, int]] = []
        vox = 0
        while self._pairq and len(batch) < self.max_batch_pairs:
            req, i = self._pairq[0]
            v = req.dims[0] * req.dims[1] * req.dims[2]
            if batch and vox + v > self.batch_voxels:
                break
            self._pairq.popleft()
            batch.append((req, i))
            vox += v
        batch.sort(key=lambda ri: (ri[0].dims, ri[0].rid, ri[1]))  # equal sizes next to each other
        dims = [req.dims for req, _ in batch]
        if sl.stream is None:
            sl.stream = torch.cuda.Stream(self.device)
        if sl.plan is None:
            sl.plan = SolverPlan.reserve(self.solver.params(), self.max_batch_pairs, self.arena_bytes, self.device)
        try:
            sl.plan.retarget(dims, stream=sl.stream.cuda_stream)
        except Exception as e:  # one pair larger than a plan holds: this slot's plan grows
            if getattr(e, "status", None) != 2:
                raise
            need = int(1.25 * state_bytes_per_voxel(self.storage, self.solver.num_scales) *
                       sum(d[0] * d[1] * d[2] for d in dims)) + (64 << 20)
            sl.plan.close()
            sl.plan = SolverPlan.reserve(self.solver.params(), self.max_batch_pairs, need, self.device)
            sl.plan.retarget(dims, stream=sl.stream.cuda_stream)
        with torch.cuda.stream(sl.stream):
            for req in {id(r): r for r, _ in batch}.values():
                sl.stream.wait_event(req.frames_ready)
            I0s = [req.frames_dev[req.pairs[i][0]] for req, i in batch]
            I1s = [req.frames_dev[req.pairs[i][1]] for req, i in batch]
            outs = [req.flows_dev[i] for req, i in batch]
            sl.plan.solve(I0s, I1s, outs, stream=sl.stream.cuda_stream)
            sl.event = torch.cuda.Event()
            sl.event.record(sl.stream)
        sl.batch = batch
        self.batches += 1
        if len({req.rid for req, _ in batch}) > 1:
            self.mixed_batches += 1

    def _finalize(self, req: _Request) -> None:
        """All pairs of `req` are solved: masks on the device, then flows and masks to the host."""
        T, nz, ny, nx = req.frames.shape[0], *req.dims
        s = self._final_stream
        with torch.cuda.stream(s):
            out = {"flows": torch.empty(req.flows_dev.shape, dtype=torch.float32, pin_memory=True)}
            out["flows"].copy_(req.flows_dev, non_blocking=True)
            if req.masks is not None:
                t0, t1 = req.mask_t
                fwd_idx = list(range(t0, t1))
                bwd_idx = [(T - 1) + (T - 1 - t) for t in range(t1, t0, -1)]
                if fwd_idx:
                    m = req.masks.to(self.device, non_blocking=True).float().reshape(2, 1, nz, ny, nx).contiguous()
                    f = torch.stack([req.flows_dev[fwd_idx], req.flows_dev[bwd_idx]], dim=1)
                    chain = propagate_batched(self.warp, m, f)
                    out["masks"] = torch.empty(chain.shape, dtype=torch.float32, pin_memory=True)
                    out["masks"].copy_(chain, non_blocking=True)
            out["_device"] = (req.frames_dev, req.flows_dev)  # kept alive until the copies are done
            req.out = out
            req.final_event = torch.cuda.Event()
            req.final_event.record(s)
        self._finishing.append(req)

    def _complete(self, req: _Request) -> None:
        now = time.perf_counter()
        self._in_use -= req.bytes_needed
        self.latencies.append(now - req.t_submit)
        self.completed += 1
        self._t_last = now
        T = req.frames.shape[0]
        flows = req.out["flows"]
        req.out.pop("_device", None)
        req.frames_dev = req.flows_dev = None
        req.future.set_result((flows[: T - 1], flows[T - 1:], req.out.get("masks")))

    def _fail_all(self, e: BaseException) -> None:
        self._error = e
        with self._lock:
            reqs = list(self._waiting) + self._active + self._finishing
            self._waiting.clear()
            self._active.clear()
            self._finishing.clear()
            self._pairq.clear()
        for req in reqs:
            if not req.future.done():
                req.future.set_exception(e)

    def _loop(self) -> None:
        torch.cuda.set_device(self.device)
        while not self._stop:
            try:
                progressed = False
                # finished batches: count their pairs; a request whose pairs are all done is finalized
                for sl in self._slots:
                    if sl.batch and sl.event.query():
                        for req, _ in sl.batch:
                            req.done += 1
                            if req.done == len(req.pairs):
                                with self._lock:
                                    self._active.remove(req)
                                self._finalize(req)
                        sl.batch = []
                        progressed = True
                # host copies complete: results out, memory back
                for req in list(self._finishing):
                    if req.final_event.query():
                        with self._lock:
                            self._finishing.remove(req)
                        self._complete(req)
                        progressed = True
                # admissions: the budget (and the optional cap) decides
                with self._lock:
                    while self._waiting and (self.max_active is None or len(self._active) < self.max_active):
                        req = self._waiting[0]
                        if self._in_use + req.bytes_needed + self.plan_bytes() > self.budget:
                            break
                        self._waiting.popleft()
                        self._admit(req)
                        progressed = True
                # an idle plan takes the next batch
                for sl in self._slots:
                    if not sl.batch and self._pairq:
                        self._launch(sl)
                        progressed = True
                if not progressed:
                    self._wake.wait(self._poll)
                    self._wake.clear()
            except BaseException as e:  # surfaced to every waiting caller
                self._fail_all(e)
                return


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
