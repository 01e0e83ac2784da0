"""Device versions of the reference's flow helpers (svs/utils/flow_utils.py).

get_interpolation_type, get_mesh_length and compute_timepoints keep the reference's semantics;
apply_gaussian_blur3d and apply_median_filter run on the GPU through libsvsflow (the reference
used cuDNN conv3d and a host round trip through scipy).
"""
from __future__ import annotations

from typing import Tuple

import numpy as np
import torch

from . import _lib
from . import opticalFlow
from ._lib import check, ptr, stream_ptr


def get_interpolation_type(inter_type_str: str, bound_type_str: str):
    """flow_utils.py:11-45."""
    inter = {"NEAREST": opticalFlow.InterpolationType.INTERPOLATE_NEAREST,
             "LINEAR": opticalFlow.InterpolationType.INTERPOLATE_LINEAR,
             "CUBIC_HERMITESPLINE": opticalFlow.InterpolationType.INTERPOLATE_CUBIC_HERMITESPLINE}
    bdry = {"NEAREST": opticalFlow.BoundaryType.BOUNDARY_NEAREST,
            "MIRROR": opticalFlow.BoundaryType.BOUNDARY_MIRROR,
            "REFLECT": opticalFlow.BoundaryType.BOUNDARY_REFLECT}
    if inter_type_str not in inter:
        raise Exception("Wrong interpolation type")
    if bound_type_str not in bdry:
        raise Exception("wrong boundary type")
    return inter[inter_type_str], bdry[bound_type_str]


def get_mesh_length(length_type: str, nz: int, ny: int, nx: int, lz, ly, lx):
    """flow_utils.py:48-71: numDofs -> (N-1) per axis, fixed -> the given lengths."""
    if length_type == "numDofs":
        return nz - 1, ny - 1, nx - 1
    if length_type == "fixed":
        return lz, ly, lx
    raise Exception("Wrong length type")


def gaussian_kernel1d(sigma: float) -> torch.Tensor:
    """flow_utils.py:74-91 (same torch CPU operations, float32)."""
    ks = int(sigma * 5)
    if ks % 2 == 0:
        ks += 1
    ts = torch.linspace(-ks // 2, ks // 2 + 1, ks)
    gauss = torch.exp((-(ts / sigma) ** 2 / 2))
    return gauss / gauss.sum()


def gaussian_kernel3d(sigma: float) -> torch.Tensor:
    """The 3D product kernel normalised again, flow_utils.py:106-107 (float32, CPU)."""
    k = gaussian_kernel1d(sigma)
    k3 = torch.einsum("i,j,k->ijk", k, k, k)
    return (k3 / k3.sum()).contiguous()


def apply_gaussian_blur3d(vol: torch.Tensor, sigma: float) -> torch.Tensor:
    """Zero-padded 3D blur with the reference kernel (flow_utils.py:94-112), on the GPU."""
    if vol.device.type != "cuda" or vol.dtype not in (torch.float32, torch.float64) or vol.dim() != 3:
        raise RuntimeError("apply_gaussian_blur3d: expected a 3D float32 or float64 CUDA tensor")
    vol = vol.contiguous()
    f64 = vol.dtype == torch.float64
    # the kernel is built in float32 as the reference builds it, then taken to the volume's type
    w = np.ascontiguousarray(gaussian_kernel3d(sigma).numpy().astype(np.float64 if f64 else np.float32))
    r = w.shape[0] // 2
    out = torch.empty_like(vol)
    nz, ny, nx = vol.shape
    fn = _lib.lib().svs_gauss_blur3d_f64 if f64 else _lib.lib().svs_gauss_blur3d
    with torch.cuda.device(vol.device):
        check(fn(ptr(vol), nz, ny, nx, w.ctypes.data, r, ptr(out), stream_ptr(vol.device)))
    return out


def apply_median_filter(u: torch.Tensor, ks: int, device: torch.device = None) -> torch.Tensor:
    """ks^3 median per component with scipy's 'reflect' boundary (flow_utils.py:115-132), computed
    on the GPU; the result is returned on `device` (default: u's device)."""
    if u.device.type != "cuda":
        raise RuntimeError("apply_median_filter: expected a CUDA tensor")
    x = u.detach()
    x = (x if x.dtype == torch.float64 else x.float()).contiguous()
    nz, ny, nx = x.shape[:3]
    C = 1 if x.dim() == 3 else int(np.prod(x.shape[3:]))
    out = torch.empty_like(x)
    fn = _lib.lib().svs_median3d_f64 if x.dtype == torch.float64 else _lib.lib().svs_median3d
    with torch.cuda.device(x.device):
        check(fn(ptr(x), nz, ny, nx, C, int(ks), ptr(out), stream_ptr(x.device)))
    return out if device is None else out.to(device)


def compute_timepoints(dia_ts: int, sys_ts: int, seg_dia, seg_sys, mode) -> Tuple:
    """flow_utils.py:135-169: (init, final) time points, their masks, and the time list (reversed
    for the backward direction)."""
    if sys_ts < dia_ts:
        timepoints = (sys_ts, dia_ts)
        segmentations = (seg_sys, seg_dia)
    else:
        timepoints = (dia_ts, sys_ts)
        segmentations = (seg_dia, seg_sys)
    times = np.arange(timepoints[0], timepoints[1] + 1, 1)
    if str(mode) == "backward" or getattr(mode, "value", None) == "backward":
        times = np.flip(times)
    return timepoints, segmentations, times.tolist()
