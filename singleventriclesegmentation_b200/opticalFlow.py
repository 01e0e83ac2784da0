"""Drop-in replacement of the reference's pybind module ``opticalFlow_cuda_ext.opticalFlow``
(svs/src/bindings.cpp:16-192, 3D subset) on top of libsvsflow.so.

Same class names, constructor arguments, method names, argument meanings and tensor layouts as the
reference. Differences a caller can observe:
  * tensors must be float32 or float64 CUDA tensors, all of one type within a call (the
    reference's dispatch took the first tensor's type and reinterpreted the others);
  * kernels run on torch's current CUDA stream (the reference used the legacy default stream);
  * launch errors raise (the reference ignored them, svs/src/cudaDebug.cuh:15-27).
Argument errors raise RuntimeError, as the reference's TORCH_CHECK / CHECK_INPUT did.
"""
from __future__ import annotations

import enum

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr


# --------------------------------------------------------------------------------- enums
class BoundaryType(enum.IntEnum):
    """svs/src/boundary.cuh:13-21 (bound with export_values, bindings.cpp:51-55)."""
    BOUNDARY_NEAREST = 0
    BOUNDARY_MIRROR = 1
    BOUNDARY_REFLECT = 2


class InterpolationType(enum.IntEnum):
    """svs/src/coreDefines.h:94-100 (bound with export_values, bindings.cpp:99-104)."""
    INTERPOLATE_NEAREST = 0
    INTERPOLATE_LINEAR = 1
    INTERPOLATE_CUBIC_HERMITESPLINE = 2


BOUNDARY_NEAREST = BoundaryType.BOUNDARY_NEAREST
BOUNDARY_MIRROR = BoundaryType.BOUNDARY_MIRROR
BOUNDARY_REFLECT = BoundaryType.BOUNDARY_REFLECT
INTERPOLATE_NEAREST = InterpolationType.INTERPOLATE_NEAREST
INTERPOLATE_LINEAR = InterpolationType.INTERPOLATE_LINEAR
INTERPOLATE_CUBIC_HERMITESPLINE = InterpolationType.INTERPOLATE_CUBIC_HERMITESPLINE


# ---------------------------------------------------------------------------------- mesh
class MeshInfo3D:
    """svs/src/coreDefines.h:62-90: node counts, lengths and spacings h = L/(N-1) (float32)."""

    def __init__(self, NZ: int, NY: int, NX: int, LZ: float, LY: float, LX: float):
        self._N = (int(NZ), int(NY), int(NX))
        self._L = tuple(float(np.float32(v)) for v in (LZ, LY, LX))
        with np.errstate(divide="ignore", invalid="ignore"):
            self._h = tuple(float(np.float32(np.float32(L) / np.float32(N - 1)))
                            for N, L in zip(self._N, self._L))

    def getNZ(self): return self._N[0]
    def getNY(self): return self._N[1]
    def getNX(self): return self._N[2]
    def getLZ(self): return self._L[0]
    def getLY(self): return self._L[1]
    def getLX(self): return self._L[2]
    def gethZ(self): return self._h[0]
    def gethY(self): return self._h[1]
    def gethX(self): return self._h[2]

    def h(self):
        return self._h

    def __repr__(self):
        return f"MeshInfo3D(N={self._N}, L={self._L})"


# ------------------------------------------------------------------------------- helpers
def _op(name: str, t: torch.Tensor):
    """The entry point for the tensor's value type: float32 -> name, float64 -> name_f64 (the
    reference dispatched both, AT_DISPATCH_FLOATING_TYPES)."""
    return getattr(_lib.lib(), name + ("_f64" if t.dtype == torch.float64 else ""))


def _check_input(t: torch.Tensor, name: str) -> None:
    """CHECK_INPUT of coreDefines.h:10-12, plus the float32 / float64 requirement."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.device.type != "cuda":
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if t.dtype not in (torch.float32, torch.float64):
        raise RuntimeError(f"{name} must be float32 or float64 (got {t.dtype})")


def _check_dim(t: torch.Tensor, d: int) -> None:
    if t.dim() != d:
        raise RuntimeError(f"Expected {d}d tensor")


def _same_device(*ts):
    dev = ts[0].device
    for t in ts[1:]:
        if t.device != dev:
            raise RuntimeError("all tensors must be on the same CUDA device")
        if t.dtype != ts[0].dtype:
            raise RuntimeError("all tensors must have the same dtype")
    return dev


# ------------------------------------------------------------------------------- Nabla3D
class Nabla3D_CD:
    """Central-difference gradient and its adjoint (svs/src/differentialOps.h:74-98)."""

    def __init__(self, meshInfo: MeshInfo3D, boundary: BoundaryType):
        self._mesh = meshInfo
        self._bdry = int(boundary)

    def _fwd(self, b, C):
        nz, ny, nx = b.shape[:3]
        out = torch.empty(tuple(b.shape) + (3,), dtype=b.dtype, device=b.device)
        hz, hy, hx = self._mesh.h()
        with torch.cuda.device(b.device):
            check(_op("svs_nabla3d_forward", b)(ptr(b), nz, ny, nx, C, hz, hy, hx, self._bdry,
                                                 ptr(out), stream_ptr(b.device)))
        return out

    def _bwd(self, p, C):
        nz, ny, nx = p.shape[:3]
        out = torch.empty(tuple(p.shape[:-1]), dtype=p.dtype, device=p.device)
        hz, hy, hx = self._mesh.h()
        with torch.cuda.device(p.device):
            check(_op("svs_nabla3d_backward", p)(ptr(p), nz, ny, nx, C, hz, hy, hx, self._bdry,
                                                  ptr(out), stream_ptr(p.device)))
        return out

    def forward(self, b: torch.Tensor) -> torch.Tensor:
        _check_input(b, "b")
        _check_dim(b, 3)
        return self._fwd(b, 1)

    def backward(self, b: torch.Tensor) -> torch.Tensor:
        _check_input(b, "b")
        _check_dim(b, 4)
        if b.shape[3] != 3:
            raise RuntimeError("Expected a [NZ,NY,NX,3] tensor")
        return self._bwd(b, 1)

    def forwardVectorField(self, b: torch.Tensor) -> torch.Tensor:
        _check_input(b, "b")
        _check_dim(b, 4)
        return self._fwd(b, b.shape[3])

    def backwardVectorField(self, b: torch.Tensor) -> torch.Tensor:
        _check_input(b, "b")
        _check_dim(b, 5)
        if b.shape[4] != 3:
            raise RuntimeError("Expected a [NZ,NY,NX,C,3] tensor")
        return self._bwd(b, b.shape[3])


# ------------------------------------------------------------------- AnisotropicNabla3D
class AnisotropicNabla3D:
    """Anisotropic tensor s n n^T + t1 t1^T (svs/src/anisotropicDifferentialOps.h:47-84)."""

    def __init__(self, meshInfo: MeshInfo3D, alpha: float, beta: float):
        self._mesh = meshInfo
        self._alpha = float(alpha)
        self._beta = float(beta)

    def computeTangentVecs(self, NablaInputImage: torch.Tensor):
        g = NablaInputImage
        _check_input(g, "NablaInputImage")
        _check_dim(g, 4)
        sh = tuple(g.shape[:3])
        s = torch.empty(sh, dtype=g.dtype, device=g.device)
        n, t1, t2 = (torch.empty(sh + (3,), dtype=g.dtype, device=g.device) for _ in range(3))
        with torch.cuda.device(g.device):
            check(_op("svs_aniso3d_tangents", g)(ptr(g), int(np.prod(sh)), self._alpha, self._beta,
                                                  ptr(s), ptr(n), ptr(t1), ptr(t2), stream_ptr(g.device)))
        return [s, n, t1, t2]

    def forwardVectorField(self, b, scalars, normals, tangents1, tangents2):
        for t, nm in ((b, "b"), (scalars, "scalars"), (normals, "normals"), (tangents1, "tangents1"),
                      (tangents2, "tangents2")):
            _check_input(t, nm)
        _check_dim(b, 5)
        nvox = int(np.prod(b.shape[:3]))
        if scalars.numel() < nvox or normals.numel() < 3 * nvox or tangents1.numel() < 3 * nvox:
            raise RuntimeError("tangent fields are smaller than the input field")
        _same_device(b, scalars, normals, tangents1, tangents2)
        out = torch.empty_like(b)
        with torch.cuda.device(b.device):
            check(_op("svs_aniso3d_apply", b)(ptr(b), nvox, ptr(scalars), ptr(normals), ptr(tangents1),
                                               ptr(tangents2), ptr(out), stream_ptr(b.device)))
        return out

    # The reference's backward is the same kernel (anisotropicDifferentialOps.h:437-444): D is
    # symmetric, so it is its own adjoint.
    backwardVectorField = forwardVectorField


# ----------------------------------------------------------------------------- Warping3D
class Warping3D:
    """u(x + phi(x)) and its gradients (svs/src/warpingOps.h:87-116)."""

    def __init__(self, meshInfo: MeshInfo3D, interpolation: InterpolationType, boundary: BoundaryType):
        self._mesh = meshInfo
        self._interp = int(interpolation)
        self._bdry = int(boundary)

    def _warp(self, u, phi, C):
        nz, ny, nx = u.shape[:3]
        if tuple(phi.shape) != (nz, ny, nx, 3):
            raise RuntimeError("phi must have shape [NZ,NY,NX,3] matching u")
        _same_device(u, phi)
        out = torch.empty_like(u)
        hz, hy, hx = self._mesh.h()
        with torch.cuda.device(u.device):
            check(_op("svs_warp3d", u)(ptr(u), nz, ny, nx, C, ptr(phi), hz, hy, hx, self._interp,
                                        self._bdry, ptr(out), stream_ptr(u.device)))
        return out

    def forward(self, u: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_input(phi, "phi")
        _check_dim(u, 3)
        _check_dim(phi, 4)
        return self._warp(u, phi, 1)

    def forwardVectorField(self, u: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_input(phi, "phi")
        _check_dim(u, 4)
        _check_dim(phi, 4)
        return self._warp(u, phi, u.shape[3])

    def backward(self, u: torch.Tensor, phi: torch.Tensor, forward_out: torch.Tensor):
        for t, nm in ((u, "u"), (phi, "phi"), (forward_out, "forward_out")):
            _check_input(t, nm)
        _check_dim(u, 3)
        _check_dim(phi, 4)
        _check_dim(forward_out, 3)
        nz, ny, nx = u.shape
        if tuple(phi.shape) != (nz, ny, nx, 3) or tuple(forward_out.shape) != (nz, ny, nx):
            raise RuntimeError("phi / grad shapes do not match u")
        _same_device(u, phi, forward_out)
        gu = torch.empty_like(u)
        gp = torch.empty_like(phi)
        hz, hy, hx = self._mesh.h()
        with torch.cuda.device(u.device):
            check(_op("svs_warp3d_backward", u)(ptr(u), nz, ny, nx, ptr(phi), ptr(forward_out), hz, hy,
                                                 hx, self._interp, self._bdry, ptr(gu), ptr(gp),
                                                 stream_ptr(u.device)))
        return [gu, gp]


class WarpingCNN3D:
    """Batched volume warp (svs/src/warpingOpsCNN.h:20-42)."""

    def __init__(self, meshInfo: MeshInfo3D, interpolation: InterpolationType, boundary: BoundaryType):
        self._mesh = meshInfo
        self._interp = int(interpolation)
        self._bdry = int(boundary)

    def forward(self, u: torch.Tensor, phi: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_input(phi, "phi")
        _check_dim(u, 5)
        _check_dim(phi, 5)
        B, C, nz, ny, nx = u.shape
        if tuple(phi.shape) != (B, nz, ny, nx, 3):
            raise RuntimeError("phi must have shape [B,NZ,NY,NX,3] matching u")
        _same_device(u, phi)
        out = torch.empty_like(u)
        hz, hy, hx = self._mesh.h()
        with torch.cuda.device(u.device):
            check(_op("svs_warp_cnn3d", u)(ptr(u), B, C, nz, ny, nx, ptr(phi), hz, hy, hx, self._interp,
                                            self._bdry, ptr(out), stream_ptr(u.device)))
        return out


# ------------------------------------------------------------------------- Prolongation3D
class Prolongation3D:
    """Resampling between meshes (svs/src/prolongationOps.h:79-107)."""

    def __init__(self, meshInfo: MeshInfo3D, meshInfoProlongated: MeshInfo3D,
                 interpolation: InterpolationType, boundary: BoundaryType):
        self._src = meshInfo
        self._dst = meshInfoProlongated
        self._interp = int(interpolation)
        self._bdry = int(boundary)

    def _run(self, u, tail):
        nz, ny, nx = u.shape[:3]
        C = int(np.prod(tail)) if tail else 1
        d = self._dst
        tz, ty, tx = d.getNZ(), d.getNY(), d.getNX()
        out = torch.empty((tz, ty, tx) + tuple(tail), dtype=u.dtype, device=u.device)
        s = self._src
        with torch.cuda.device(u.device):
            check(_op("svs_prolongate3d", u)(ptr(u), nz, ny, nx, C, s.getLZ(), s.getLY(), s.getLX(),
                                              tz, ty, tx, d.getLZ(), d.getLY(), d.getLX(), self._interp,
                                              self._bdry, ptr(out), stream_ptr(u.device)))
        return out

    def forward(self, u: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_dim(u, 3)
        return self._run(u, ())

    def forwardVectorField(self, u: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_dim(u, 4)
        return self._run(u, (u.shape[3],))

    def forwardMatrixField(self, u: torch.Tensor) -> torch.Tensor:
        _check_input(u, "u")
        _check_dim(u, 5)
        return self._run(u, (u.shape[3], u.shape[4]))


# -------------------------------------------------------------------------------- proxes
def _mesh_voxels(mesh: MeshInfo3D) -> int:
    return mesh.getNZ() * mesh.getNY() * mesh.getNX()


def TVL1OF3D_proxPrimal(primalVariable: torch.Tensor, primalStepSize_tau: float,
                        primalFctWeight_Matching: float, rho: torch.Tensor,
                        I1_warped_grad: torch.Tensor, meshInfo: MeshInfo3D) -> torch.Tensor:
    """L1 data-term shrinkage (svs/src/opticalFlowOps.h:111-120, opticalFlowOps.cu:123-175)."""
    _check_input(primalVariable, "primalVariable")
    _check_input(rho, "rho")
    _check_input(I1_warped_grad, "I1_warped_grad")
    _check_dim(primalVariable, 4)
    n = _mesh_voxels(meshInfo)
    if primalVariable.numel() != 3 * n or rho.numel() != n or I1_warped_grad.numel() != 3 * n:
        raise RuntimeError("proxPrimal: tensor sizes do not match the mesh")
    _same_device(primalVariable, rho, I1_warped_grad)
    out = torch.empty_like(primalVariable)
    dev = primalVariable.device
    with torch.cuda.device(dev):
        check(_op("svs_tvl1_prox_primal", primalVariable)(ptr(primalVariable), n, float(primalStepSize_tau),
                                              float(primalFctWeight_Matching), ptr(rho), ptr(I1_warped_grad),
                                              ptr(out), stream_ptr(dev)))
    return out


def TVL1OF3D_proxDual(dualVariable: torch.Tensor, dualStepSize_sigma: float, dualFctWeight_TV: float,
                      meshInfo: MeshInfo3D) -> torch.Tensor:
    """Projection onto the ball of radius weight_tv per flow component
    (svs/src/opticalFlowOps.h:123-129, opticalFlowOps.cu:179-208); sigma is unused."""
    _check_input(dualVariable, "dualVariable")
    _check_dim(dualVariable, 5)
    n = _mesh_voxels(meshInfo)
    if dualVariable.numel() != 9 * n:
        raise RuntimeError("proxDual: tensor size does not match the mesh")
    out = torch.empty_like(dualVariable)
    dev = dualVariable.device
    with torch.cuda.device(dev):
        check(_op("svs_tvl1_prox_dual", dualVariable)(ptr(dualVariable), n, float(dualStepSize_sigma),
                                            float(dualFctWeight_TV), ptr(out), stream_ptr(dev)))
    return out


__all__ = [
    "BoundaryType", "InterpolationType", "MeshInfo3D", "Nabla3D_CD", "AnisotropicNabla3D",
    "Warping3D", "WarpingCNN3D", "Prolongation3D", "TVL1OF3D_proxPrimal", "TVL1OF3D_proxDual",
    "BOUNDARY_NEAREST", "BOUNDARY_MIRROR", "BOUNDARY_REFLECT", "INTERPOLATE_NEAREST",
    "INTERPOLATE_LINEAR", "INTERPOLATE_CUBIC_HERMITESPLINE",
]
