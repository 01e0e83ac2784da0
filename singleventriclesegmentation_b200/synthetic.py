"""Seeded synthetic inputs with the shapes and value ranges of the reference's data.

The reference works on cine MRI volumes resampled to 80^3 and padded to 35 frames
(conf/preprocessing.yaml prolongation nx/ny/nz = 80, pad_time = 35); those datasets are not
available here, so these generators stand in for them:

  blobs_volume      sum of random 3D Gaussian blobs clipped to [0, 1]
  sine_displacement u_d(x) = A sin(2 pi x_d / N_d + phi_d) per axis
  warp_volume       tricubic Catmull-Rom warp with the MIRROR fold (float64, torch; CPU or GPU)
  frame_pair        (I0, I1, true displacement) for one pair
  cine_sequence     T frames: frame t = I0 warped by a sin(2 pi t / T) v(x), v smooth, |v| <= 3
  ellipsoid_mask    binary ellipsoid, semi-axes (x, y, z) voxels, centred
Everything is generated in float64 from numpy.random.default_rng(seed) and returned as float32.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np
import torch


def blobs_volume(shape: Sequence[int], rng: np.random.Generator, n_blobs: int = 40,
                 sigma_range=(3.0, 10.0), amp_range=(0.2, 1.0)) -> np.ndarray:
    """I = clip(sum_k a_k exp(-|x - c_k|^2 / (2 s_k^2)), 0, 1); sigma scaled with the volume
    size relative to 80^3."""
    nz, ny, nx = shape
    scale = (nz * ny * nx) ** (1.0 / 3.0) / 80.0
    c = rng.uniform(0.0, 1.0, size=(n_blobs, 3)) * np.array([nz, ny, nx], dtype=np.float64)
    s = rng.uniform(*sigma_range, size=n_blobs) * scale
    a = rng.uniform(*amp_range, size=n_blobs)
    z = np.arange(nz, dtype=np.float64)[:, None, None]
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    x = np.arange(nx, dtype=np.float64)[None, None, :]
    vol = np.zeros((nz, ny, nx), dtype=np.float64)
    for k in range(n_blobs):
        d2 = (z - c[k, 0]) ** 2 + (y - c[k, 1]) ** 2 + (x - c[k, 2]) ** 2
        vol += a[k] * np.exp(-d2 / (2.0 * s[k] ** 2))
    return np.clip(vol, 0.0, 1.0)


def sine_displacement(shape: Sequence[int], rng: np.random.Generator, amplitude: float = 2.0) -> np.ndarray:
    """u [Z,Y,X,3] (components x, y, z) with u_d = A sin(2 pi x_d / N_d + phi_d)."""
    nz, ny, nx = shape
    phi = rng.uniform(0.0, 2.0 * math.pi, size=3)
    z = np.arange(nz, dtype=np.float64)[:, None, None]
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    x = np.arange(nx, dtype=np.float64)[None, None, :]
    u = np.zeros((nz, ny, nx, 3), dtype=np.float64)
    u[..., 0] = amplitude * np.sin(2 * math.pi * x / nx + phi[0])
    u[..., 1] = amplitude * np.sin(2 * math.pi * y / ny + phi[1])
    u[..., 2] = amplitude * np.sin(2 * math.pi * z / nz + phi[2])
    return u


def smooth_field(shape: Sequence[int], rng: np.random.Generator, max_amp: float = 3.0, n_modes: int = 4) -> np.ndarray:
    """A smooth random vector field [Z,Y,X,3] (sum of low-frequency sinusoids per component),
    normalised so that its largest component magnitude is max_amp."""
    nz, ny, nx = shape
    z = np.arange(nz, dtype=np.float64)[:, None, None] / nz
    y = np.arange(ny, dtype=np.float64)[None, :, None] / ny
    x = np.arange(nx, dtype=np.float64)[None, None, :] / nx
    v = np.zeros((nz, ny, nx, 3), dtype=np.float64)
    for c in range(3):
        for _ in range(n_modes):
            k = rng.uniform(0.3, 1.5, size=3)
            ph = rng.uniform(0, 2 * math.pi)
            v[..., c] += rng.uniform(0.5, 1.0) * np.sin(2 * math.pi * (k[0] * z + k[1] * y + k[2] * x) + ph)
    return v * (max_amp / np.abs(v).max())


def _fold_mirror(i: torch.Tensor, n: int) -> torch.Tensor:
    i = torch.where(i < 0, -i - 1, i)
    i = torch.where(i > n - 1, 2 * n - 1 - i, i)
    return i.clamp(0, n - 1)


def _cr_weights(w: torch.Tensor) -> List[torch.Tensor]:
    w2, w3 = w * w, w * w * w
    return [-w3 / 2 + w2 - w / 2, 1.5 * w3 - 2.5 * w2 + 1, -1.5 * w3 + 2 * w2 + w / 2, w3 / 2 - w2 / 2]


def warp_volume(vol: np.ndarray, disp: np.ndarray, device: str = "cpu") -> np.ndarray:
    """vol(x + disp(x)), tricubic Catmull-Rom with the MIRROR fold, in float64."""
    v = torch.as_tensor(vol, dtype=torch.float64, device=device)
    d = torch.as_tensor(disp, dtype=torch.float64, device=device)
    nz, ny, nx = v.shape
    zz, yy, xx = torch.meshgrid(torch.arange(nz, device=device, dtype=torch.float64),
                                torch.arange(ny, device=device, dtype=torch.float64),
                                torch.arange(nx, device=device, dtype=torch.float64), indexing="ij")
    cx, cy, cz = xx + d[..., 0], yy + d[..., 1], zz + d[..., 2]
    fx, fy, fz = torch.floor(cx), torch.floor(cy), torch.floor(cz)
    Wx, Wy, Wz = _cr_weights(cx - fx), _cr_weights(cy - fy), _cr_weights(cz - fz)
    fx, fy, fz = fx.long(), fy.long(), fz.long()
    flat = v.reshape(-1)
    out = torch.zeros_like(v)
    for a in range(4):
        iz = _fold_mirror(fz + a - 1, nz)
        for b in range(4):
            iy = _fold_mirror(fy + b - 1, ny)
            wzy = Wz[a] * Wy[b]
            base = (iz * ny + iy) * nx
            for c in range(4):
                ix = _fold_mirror(fx + c - 1, nx)
                out += wzy * Wx[c] * flat[base + ix]
    return out.cpu().numpy()


def frame_pair(shape=(80, 80, 80), seed: int = 0, amplitude: float = 2.0, noise: float = 0.01,
               device: str = "cpu") -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(I0, I1, u_true) float32: I1 = I0 warped by the sine displacement plus N(0, noise^2)."""
    rng = np.random.default_rng(seed)
    I0 = blobs_volume(shape, rng)
    u = sine_displacement(shape, rng, amplitude)
    I1 = warp_volume(I0, u, device) + rng.normal(0.0, noise, size=tuple(shape))
    return I0.astype(np.float32), I1.astype(np.float32), u.astype(np.float32)


def cine_sequence(T: int = 35, shape=(80, 80, 80), seed: int = 0, amplitude: float = 1.0,
                  max_disp: float = 3.0, noise: float = 0.01, device: str = "cpu",
                  first: int = None) -> np.ndarray:
    """[T,Z,Y,X] float32: frame t = I0 warped by amplitude sin(2 pi t / T) v(x), plus noise.
    With `first`, only frames 0 .. first-1 are made (bitwise those of the whole sequence)."""
    rng = np.random.default_rng(seed)
    I0 = blobs_volume(shape, rng)
    v = smooth_field(shape, rng, max_disp)
    n = T if first is None else min(T, first)
    frames = np.empty((n,) + tuple(shape), dtype=np.float32)
    for t in range(n):
        a = amplitude * math.sin(2 * math.pi * t / T)
        f = I0 if a == 0.0 else warp_volume(I0, a * v, device)
        frames[t] = (f + rng.normal(0.0, noise, size=tuple(shape))).astype(np.float32)
    return frames


def ellipsoid_mask(shape=(80, 80, 80), semi_axes=(15, 12, 10), center=None) -> np.ndarray:
    """Binary float32 mask [Z,Y,X]; semi_axes are (x, y, z) in voxels; centred by default."""
    nz, ny, nx = shape
    cz, cy, cx = center if center is not None else ((nz - 1) / 2, (ny - 1) / 2, (nx - 1) / 2)
    ax, ay, az = semi_axes
    z = np.arange(nz)[:, None, None]
    y = np.arange(ny)[None, :, None]
    x = np.arange(nx)[None, None, :]
    r = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 + ((z - cz) / az) ** 2
    return (r <= 1.0).astype(np.float32)


def sequence_pairs(T: int, mode: str = "forward") -> List[Tuple[int, int]]:
    """(fixed, moving) frame indices of the consecutive pairs of a sequence, as the reference's
    processor builds them (processor.py:104, 110-112): I0 = img[times[j+1]], I1 = img[times[j]]."""
    times = list(range(T))
    if mode == "backward":
        times = times[::-1]
    return [(times[j + 1], times[j]) for j in range(T - 1)]
