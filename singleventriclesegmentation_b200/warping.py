"""Mask propagation and its metrics: svs/modules/flow/warping.py:35-65 (Warp), :205-243
(_propagate) and :245-270 (_compute_metrics), on the device.

Dice and the symmetric Hausdorff distance restate monai's compute_dice and
compute_hausdorff_distance as the reference calls them (include_background=False on a single
channel keeps that channel): Dice = 2|A and B| / (|A| + |B|) (NaN if both are empty); surface
voxels = mask minus its 6-neighbour erosion (zero border); HD = max of the two directed max-min
Euclidean distances between the surface voxel sets, in voxel units.
"""
from __future__ import annotations

from typing import Tuple

import torch

from . import opticalFlow
from .flow_utils import get_interpolation_type, get_mesh_length


class Warp:
    """warping.py:35-65: warps [B,C,Z,Y,X] volumes by [B,Z,Y,X,3] flows (WarpingCNN3D)."""

    def __init__(self, interpolation_type: str, boundary_type: str, mesh_length_type: str,
                 lenghts: Tuple[int, int, int]):
        self.interpolation, self.boundary = get_interpolation_type(interpolation_type, boundary_type)
        self.mesh_length_type = mesh_length_type
        self.LZ, self.LY, self.LX = lenghts

    def __call__(self, x: torch.Tensor, u: torch.Tensor) -> torch.Tensor:
        NZ, NY, NX = x.shape[2:]
        LZ, LY, LX = get_mesh_length(self.mesh_length_type, NZ, NY, NX, self.LZ, self.LY, self.LX)
        mesh_info = opticalFlow.MeshInfo3D(NZ, NY, NX, LZ, LY, LX)
        op = opticalFlow.WarpingCNN3D(mesh_info, self.interpolation, self.boundary)
        return op.forward(x.contiguous(), u.contiguous())


def propagate(warp: Warp, initial_mask: torch.Tensor, final_mask: torch.Tensor,
              forward_flow: torch.Tensor, backward_flow: torch.Tensor):
    """warping.py:205-243: chain the float masks through the flows both ways, reverse the
    backward chain, then threshold at 0.5. Masks [1,1,Z,Y,X]; flows [T-1,Z,Y,X,3]."""
    assert forward_flow.shape[0] == backward_flow.shape[0], "Forward and backward flow have different timesteps"
    fwd = [initial_mask]
    bwd = [final_mask]
    for t in range(forward_flow.shape[0]):
        fwd.append(warp(fwd[-1], forward_flow[t].unsqueeze(0)))
        bwd.append(warp(bwd[-1], backward_flow[t].unsqueeze(0)))
    bwd.reverse()
    fwd = torch.where(torch.cat(fwd, dim=0) > 0.5, 1.0, 0.0)
    bwd = torch.where(torch.cat(bwd, dim=0) > 0.5, 1.0, 0.0)
    return fwd, bwd


def propagate_batched(warp: Warp, masks: torch.Tensor, flows: torch.Tensor) -> torch.Tensor:
    """Many independent chains at once: masks [K,1,Z,Y,X] are warped step by step with flows
    [T-1,K,Z,Y,X,3] (chain k uses flows[:, k]); one batched launch per step instead of one per
    chain. Returns the float chains [T,K,1,Z,Y,X] (not thresholded)."""
    out = [masks]
    for t in range(flows.shape[0]):
        out.append(warp(out[-1], flows[t]))
    return torch.stack(out, 0)


def dice(pred: torch.Tensor, gt: torch.Tensor) -> float:
    a = pred > 0.5
    b = gt > 0.5
    s = a.sum() + b.sum()
    if int(s) == 0:
        return float("nan")
    return float(2.0 * (a & b).sum().double() / s.double())


def surface_voxels(mask: torch.Tensor) -> torch.Tensor:
    """Coordinates [K,3] of the mask voxels that have a 6-neighbour outside the mask."""
    m = (mask > 0.5)
    p = torch.nn.functional.pad(m.float()[None, None], (1, 1, 1, 1, 1, 1))[0, 0] > 0.5
    inner = (p[:-2, 1:-1, 1:-1] & p[2:, 1:-1, 1:-1] & p[1:-1, :-2, 1:-1] & p[1:-1, 2:, 1:-1]
             & p[1:-1, 1:-1, :-2] & p[1:-1, 1:-1, 2:])
    return torch.nonzero(m & ~inner).double()


def _directed(a: torch.Tensor, b: torch.Tensor, chunk: int = 4096) -> float:
    worst = 0.0
    for i in range(0, a.shape[0], chunk):
        d = torch.cdist(a[i:i + chunk], b).min(dim=1).values
        worst = max(worst, float(d.max()))
    return worst


def hausdorff(pred: torch.Tensor, gt: torch.Tensor) -> float:
    a = surface_voxels(pred)
    b = surface_voxels(gt)
    if a.shape[0] == 0 and b.shape[0] == 0:
        return float("nan")
    if a.shape[0] == 0 or b.shape[0] == 0:
        return float("inf")
    return max(_directed(a, b), _directed(b, a))


def compute_metrics(forward_masks: torch.Tensor, backward_masks: torch.Tensor):
    """warping.py:245-270: (dice_bwd, dice_fwd, hd_bwd, hd_fwd) between the propagated end masks
    and the given end masks. Masks [T,1,Z,Y,X] (or [T,Z,Y,X])."""
    fm = forward_masks.reshape(forward_masks.shape[0], *forward_masks.shape[-3:])
    bm = backward_masks.reshape(backward_masks.shape[0], *backward_masks.shape[-3:])
    initial_gt, initial_pred = fm[0], bm[0]
    final_gt, final_pred = bm[-1], fm[-1]
    return (dice(initial_pred, initial_gt), dice(final_pred, final_gt),
            hausdorff(initial_pred, initial_gt), hausdorff(final_pred, final_gt))
