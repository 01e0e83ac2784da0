"""Per-sequence flow driver: the pair loop of svs/modules/flow/processor.py:95-121 as one batched
solve, plus the reference's flow file layout.

The reference solves the pairs of a patient one after another, median-filters each flow on the
host and stores them as `(T-1, 3, X, Y, Z)` float32 in `{name}_{mode}_flow.npy`
(processor.py:107-120; read back by svs/modules/datasets.py:279-291). Because the warm start is
overwritten when num_scales > 1 (tvl13d.py:150, 158), the pairs are independent and run here as
one batch; the median filter runs on the device inside the solve.
"""
from __future__ import annotations

import os
from concurrent.futures import Future, ThreadPoolExecutor
from typing import List, Sequence, Tuple

import numpy as np
import torch

from .flow_utils import compute_timepoints

# svs/modules/datasets.py:24-37
XYZT_TO_TZYX = (3, 2, 1, 0)
T3XYZ_TO_TZYX3 = (0, 4, 3, 2, 1)


def pair_indices(tdia: int, tsys: int, mode: str) -> List[Tuple[int, int]]:
    """(fixed, moving) frame indices of a patient's pairs, processor.py:104, 110-112:
    I0 = img[times[j+1]], I1 = img[times[j]] over compute_timepoints' time list."""
    *_, times = compute_timepoints(tdia, tsys, None, None, mode)
    return [(times[j + 1], times[j]) for j in range(len(times) - 1)]


def process_sequence(img: torch.Tensor, tdia: int, tsys: int, mode: str, solver,
                     median_kernel: int = 3) -> torch.Tensor:
    """Flows of one patient in the reference's output layout.

    img: [T, Z, Y, X] float32 CUDA tensor (the reference transposes its NIfTI xyzt volume to
    tzyx, processor.py:103). solver: a TVL13DOpticalFlow. Returns us [T'-1, 3, X, Y, Z] on the
    device, where T' is the number of time points between tdia and tsys (inclusive), with each
    flow median-filtered (processor.py:116-118) when median_kernel > 1.
    """
    pairs = pair_indices(tdia, tsys, mode)
    old = solver.median_kernel
    solver.median_kernel = median_kernel if median_kernel and median_kernel > 1 else 0
    try:
        us = solver.compute_batch([img[a] for a, b in pairs], [img[b] for a, b in pairs])
    finally:
        solver.median_kernel = old
    return torch.stack([u.permute(3, 2, 1, 0) for u in us])  # (3, x, y, z) per pair


def flow_path(out_dir: str, name: str, mode: str) -> str:
    return os.path.join(out_dir, f"{name}_{mode}_flow.npy")


def save_flow(out_dir: str, name: str, mode: str, us: torch.Tensor) -> str:
    """np.save of (T-1, 3, X, Y, Z) float32, processor.py:120."""
    os.makedirs(out_dir, exist_ok=True)
    path = flow_path(out_dir, name, mode)
    np.save(path, us.detach().float().cpu().numpy())
    return path


class FlowWriter:
    """Asynchronous flow-file output. A submitted flow array is copied device -> pinned host on a
    copy stream of its own (after an event that marks the end of the solve that produced it) and
    written as `{name}_{mode}_flow.npy` by a writer thread, so that the next patient's solve on the
    compute stream overlaps both the copy and the file write. Files are the bytes save_flow
    writes (processor.py:120)."""

    def __init__(self, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(self.device)
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.futures: List[Future] = []

    def submit(self, out_dir: str, name: str, mode: str, us: torch.Tensor) -> Future:
        """Queue `us` ([T-1, 3, X, Y, Z] float32 on the device, produced on the current stream)."""
        src = us.detach().float()
        solved = torch.cuda.Event()
        solved.record(torch.cuda.current_stream(self.device))
        host = torch.empty(src.shape, dtype=torch.float32, pin_memory=True)
        copied = torch.cuda.Event()
        with torch.cuda.stream(self.stream):
            self.stream.wait_event(solved)
            host.copy_(src, non_blocking=True)
            copied.record(self.stream)
        src.record_stream(self.stream)  # the device buffer stays allocated until the copy is done
        os.makedirs(out_dir, exist_ok=True)
        path = flow_path(out_dir, name, mode)

        def write() -> str:
            copied.synchronize()
            np.save(path, host.numpy())
            return path

        fut = self.pool.submit(write)
        self.futures.append(fut)
        return fut

    def close(self) -> List[str]:
        """Wait for every queued file; returns their paths in submission order."""
        paths = [f.result() for f in self.futures]
        self.futures.clear()
        self.pool.shutdown(wait=True)
        return paths


def process_patients(patients: Sequence[Tuple[str, torch.Tensor, int, int]], solver, out_dir: str,
                     modes: Sequence[str] = ("forward", "backward"), median_kernel: int = 3) -> List[str]:
    """The processor's patient loop (processor.py:95-121 per patient and direction) with the flow
    files written asynchronously: patients are (name, img [T,Z,Y,X] on the device, tdia, tsys);
    each patient's pairs run as one batched solve, and its flows go to disk through a FlowWriter
    while the next one is solved. Returns the written paths."""
    writer = FlowWriter(solver.device)
    try:
        for name, img, tdia, tsys in patients:
            for mode in modes:
                writer.submit(out_dir, name, mode, process_sequence(img, tdia, tsys, mode, solver, median_kernel))
    finally:
        paths = writer.close()
    return paths


def load_flow(out_dir: str, name: str, mode: str) -> np.ndarray:
    """datasets.py:279-291: the (t, 3, x, y, z) array as saved."""
    return np.load(flow_path(out_dir, name, mode))


def flows_for_warping(flow_t3xyz: np.ndarray, device=None) -> torch.Tensor:
    """warping.py:161-203 prepare_data: (t, 3, x, y, z) -> (t, z, y, x, 3) float tensor."""
    return torch.from_numpy(np.ascontiguousarray(flow_t3xyz.transpose(T3XYZ_TO_TZYX3))).float().to(device)
