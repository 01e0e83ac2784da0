"""Preprocessing resample of a cine MRI to the flow path's grid, svs/preprocessing/prolongation.py:
each patient's 4D image (z, y, x, t) is resampled in space to nz x ny x nx (80^3 by default,
conf/preprocessing.yaml) with Prolongation3D (LINEAR, MIRROR; the time frames as the components
of one vector field, prolongation.py:83), the two segmentations with Prolongation3D.forward and
rounded (prolongation.py:81-82), and the time axis zero-padded to pad_time frames
(time_pading, prolongation.py:15-22). NIfTI reading and writing stay with the caller.
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch
import torch.nn.functional as F

from . import opticalFlow
from .flow_utils import get_interpolation_type, get_mesh_length


def time_pading(maxt: int, img: torch.Tensor) -> torch.Tensor:
    """Zero-pad the last (time) axis of a [z, y, x, t] tensor to maxt frames (prolongation.py:15-22)."""
    diff_t = maxt - img.shape[-1]
    return F.pad(img, [0, diff_t, 0, 0, 0, 0, 0, 0])


def resample_patient(img_zyxt: torch.Tensor, seg_dia_zyx: Optional[torch.Tensor] = None,
                     seg_sys_zyx: Optional[torch.Tensor] = None, shape: Tuple[int, int, int] = (80, 80, 80),
                     pad_time: int = 35, interpolation: str = "LINEAR", boundary: str = "MIRROR",
                     length_type: str = "numDofs", lengths: Tuple[float, float, float] = (1, 1, 1)):
    """The per-patient body of prolongation.py:67-85 on CUDA tensors.

    img_zyxt: [nz, ny, nx, nt] float; seg_*: [nz, ny, nx] masks (optional). shape = (nz, ny, nx)
    of the target grid; lengths = (lz, ly, lx) when length_type is "fixed" (both meshes take the
    configuration's length type and lengths, prolongation.py:72-73 and :45-46). Returns
    (img [NZ, NY, NX, pad_time], seg_dia, seg_sys, factors) with factors = (x, y, z, t)
    prolongation factors as the reference stores them (prolongation.py:117-120)."""
    interp, bdry = get_interpolation_type(interpolation, boundary)
    nz, ny, nx, nt = (int(v) for v in img_zyxt.shape)
    NZ, NY, NX = (int(v) for v in shape)
    lz, ly, lx = get_mesh_length(length_type, nz, ny, nx, *lengths)
    LZ, LY, LX = get_mesh_length(length_type, NZ, NY, NX, *lengths)
    old = opticalFlow.MeshInfo3D(nz, ny, nx, lz, ly, lx)
    new = opticalFlow.MeshInfo3D(NZ, NY, NX, LZ, LY, LX)
    op = opticalFlow.Prolongation3D(old, new, interp, bdry)
    seg_dia = op.forward(seg_dia_zyx.float().contiguous()).round() if seg_dia_zyx is not None else None
    seg_sys = op.forward(seg_sys_zyx.float().contiguous()).round() if seg_sys_zyx is not None else None
    img = time_pading(pad_time, op.forwardVectorField(img_zyxt.float().contiguous()))
    factors = (NX / nx, NY / ny, NZ / nz, pad_time / nt)
    return img, seg_dia, seg_sys, factors
