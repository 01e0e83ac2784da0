"""Oracle: ctypes front end of the CPU restatement in ``svs_oracle.cpp``.

TEST INFRASTRUCTURE ONLY. The parity tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it as the checker; the product package never imports it.

Every function works on C-contiguous numpy arrays in the reference's layouts (scalar fields
[Z,Y,X], vector fields [Z,Y,X,3], matrix fields [Z,Y,X,3,3], CNN volumes [B,C,Z,Y,X]) and in
float32 or float64 (the dtype of the first array argument selects the instantiation).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "svs_oracle.cpp")
_LIB = os.path.join(_HERE, "libsvs_oracle.so")

BOUNDARY = {"NEAREST": 0, "MIRROR": 1, "REFLECT": 2}
INTERP = {"NEAREST": 0, "LINEAR": 1, "CUBIC_HERMITESPLINE": 2}


def build(force: bool = False) -> str:
    """Compile the oracle shared library next to its source (gcc, OpenMP, no FMA contraction)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp",
               "-fPIC", "-shared", "-o", _LIB + ".tmp", _SRC]
        subprocess.run(cmd, check=True)
        os.replace(_LIB + ".tmp", _LIB)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB)
        _lib.svso_dice.restype = ctypes.c_double
        _lib.svso_hausdorff.restype = ctypes.c_double
        _lib.svso_num_threads.restype = ctypes.c_int
    return _lib


def set_threads(n: int) -> None:
    lib().svso_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().svso_num_threads())


class _Params(ctypes.Structure):
    _fields_ = [
        ("num_scales", ctypes.c_int), ("max_warps", ctypes.c_int), ("max_iters", ctypes.c_int),
        ("weight_matching", ctypes.c_float), ("weight_tv", ctypes.c_float),
        ("pd_type", ctypes.c_int),
        ("sigma", ctypes.c_double), ("tau", ctypes.c_double), ("theta", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("use_aniso", ctypes.c_int), ("alpha", ctypes.c_float), ("beta", ctypes.c_float),
        ("use_blur", ctypes.c_int), ("blur_sigma", ctypes.c_float),
        ("interp", ctypes.c_int), ("bdry", ctypes.c_int),
        ("length_type", ctypes.c_int),
        ("len_z", ctypes.c_float), ("len_y", ctypes.c_float), ("len_x", ctypes.c_float),
    ]


@dataclass
class SolverParams:
    """Solver parameters with the defaults of the reference's conf/flow.yaml:17-57."""
    num_scales: int = 3
    max_warps: int = 15
    max_outer_iterations: int = 300
    weight_matching: float = 1.0
    weight_tv: float = 0.025
    primaldual_algorithm_type: int = 2
    primaldual_algorithm_params: tuple = (0.5, 0.5, 0.25, 1.0)
    use_anisotropic_diff: bool = True
    anisotropic_diff_params: tuple = (5.0, 0.5)
    use_gaussian_blur: bool = True
    gaussian_blur_sigma: float = 1.0
    interpolation_type: str = "CUBIC_HERMITESPLINE"
    boundary_type: str = "MIRROR"
    length_type: str = "numDofs"
    length: tuple = (1, 1, 1)  # (lx, ly, lz)

    def to_c(self) -> _Params:
        s, t, th, g = self.primaldual_algorithm_params
        lx, ly, lz = self.length
        return _Params(self.num_scales, self.max_warps, self.max_outer_iterations,
                       self.weight_matching, self.weight_tv, self.primaldual_algorithm_type,
                       s, t, th, g, int(self.use_anisotropic_diff),
                       self.anisotropic_diff_params[0], self.anisotropic_diff_params[1],
                       int(self.use_gaussian_blur), self.gaussian_blur_sigma,
                       INTERP[self.interpolation_type], BOUNDARY[self.boundary_type],
                       0 if self.length_type == "numDofs" else 1, lz, ly, lx)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(a: np.ndarray) -> str:
    if a.dtype == np.float32:
        return "f32"
    if a.dtype == np.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {a.dtype}")


def _c(a, dtype=None):
    a = np.asarray(a) if dtype is None else np.asarray(a, dtype=dtype)
    return np.ascontiguousarray(a)


def _f(x):
    return ctypes.c_float(float(x))


def mesh_spacing(n: int, length: float) -> float:
    """h = L / (N - 1) in float32, coreDefines.h:72-75."""
    return float(np.float32(np.float32(length) / np.float32(n - 1)))


# ------------------------------------------------------------------ operators
def nabla_forward(b, h=(1.0, 1.0, 1.0), bdry="MIRROR"):
    """Scalar gradient [Z,Y,X] -> [Z,Y,X,3] (differentialOps.cu:540-655). h = (hz, hy, hx)."""
    b = _c(b)
    out = np.empty(b.shape + (3,), b.dtype)
    getattr(lib(), "svso_nabla_fwd_vf_" + _sfx(b))(_p(b), *b.shape, 1, *map(_f, h),
                                                   BOUNDARY[bdry], _p(out))
    return out


def nabla_forward_vf(b, h=(1.0, 1.0, 1.0), bdry="MIRROR"):
    """Per-component gradient [Z,Y,X,C] -> [Z,Y,X,C,3] (differentialOps.cu:782-907)."""
    b = _c(b)
    out = np.empty(b.shape + (3,), b.dtype)
    getattr(lib(), "svso_nabla_fwd_vf_" + _sfx(b))(_p(b), *b.shape[:3], b.shape[3], *map(_f, h),
                                                   BOUNDARY[bdry], _p(out))
    return out


def nabla_backward(p, h=(1.0, 1.0, 1.0), bdry="MIRROR"):
    """Scalar adjoint [Z,Y,X,3] -> [Z,Y,X] (differentialOps.cu:658-779)."""
    p = _c(p)
    out = np.empty(p.shape[:3], p.dtype)
    getattr(lib(), "svso_nabla_bwd_vf_" + _sfx(p))(_p(p), *p.shape[:3], 1, *map(_f, h),
                                                   BOUNDARY[bdry], _p(out))
    return out


def nabla_backward_vf(p, h=(1.0, 1.0, 1.0), bdry="MIRROR"):
    """Matrix-field adjoint [Z,Y,X,C,3] -> [Z,Y,X,C] (differentialOps.cu:909-1039)."""
    p = _c(p)
    out = np.empty(p.shape[:4], p.dtype)
    getattr(lib(), "svso_nabla_bwd_vf_" + _sfx(p))(_p(p), *p.shape[:3], p.shape[3], *map(_f, h),
                                                   BOUNDARY[bdry], _p(out))
    return out


def aniso_tangents(g, alpha, beta):
    """(s, n, t1, t2) from an image gradient (anisotropicDifferentialOps.cu:89-141)."""
    g = _c(g)
    sh = g.shape[:3]
    s = np.empty(sh, g.dtype)
    n, t1, t2 = (np.empty(sh + (3,), g.dtype) for _ in range(3))
    getattr(lib(), "svso_aniso_tangents_" + _sfx(g))(_p(g), ctypes.c_size_t(int(np.prod(sh))),
                                                     _f(alpha), _f(beta), _p(s), _p(n), _p(t1),
                                                     _p(t2))
    return s, n, t1, t2


def aniso_apply(b, s, n, t1):
    """D b for a [Z,Y,X,3,3] field (anisotropicDifferentialOps.cu:143-175)."""
    b, s, n, t1 = _c(b), _c(s, b.dtype), _c(n, b.dtype), _c(t1, b.dtype)
    out = np.empty_like(b)
    getattr(lib(), "svso_aniso_apply_" + _sfx(b))(_p(b), ctypes.c_size_t(int(np.prod(b.shape[:3]))),
                                                  _p(s), _p(n), _p(t1), _p(out))
    return out


def prox_primal(pv, tau, lam, rho, g):
    """opticalFlowOps.cu:123-175."""
    pv = _c(pv)
    rho, g = _c(rho, pv.dtype), _c(g, pv.dtype)
    out = np.empty_like(pv)
    getattr(lib(), "svso_prox_primal_" + _sfx(pv))(_p(pv), ctypes.c_size_t(int(np.prod(pv.shape[:3]))),
                                                   _f(tau), _f(lam), _p(rho), _p(g), _p(out))
    return out


def prox_dual(dv, weight_tv):
    """opticalFlowOps.cu:179-208."""
    dv = _c(dv)
    out = np.empty_like(dv)
    getattr(lib(), "svso_prox_dual_" + _sfx(dv))(_p(dv), ctypes.c_size_t(int(np.prod(dv.shape[:3]))),
                                                 _f(weight_tv), _p(out))
    return out


def warp(u, phi, h=(1.0, 1.0, 1.0), interp="CUBIC_HERMITESPLINE", bdry="MIRROR"):
    """u(x + phi(x)) for a scalar [Z,Y,X] or C-component [Z,Y,X,C] field (warpingOps.cu)."""
    u = _c(u)
    phi = _c(phi, u.dtype)
    C = 1 if u.ndim == 3 else u.shape[3]
    out = np.empty_like(u)
    getattr(lib(), "svso_warp_" + _sfx(u))(_p(u), *u.shape[:3], C, _p(phi), *map(_f, h),
                                           INTERP[interp], BOUNDARY[bdry], _p(out))
    return out


def warp_backward(u, phi, grad_out, h=(1.0, 1.0, 1.0), interp="CUBIC_HERMITESPLINE", bdry="MIRROR"):
    """Warping3D.backward: (grad_u [Z,Y,X], grad_phi [Z,Y,X,3]) (warpingOps.cu:598-630)."""
    u = _c(u)
    phi, g = _c(phi, u.dtype), _c(grad_out, u.dtype)
    gu = np.empty_like(u)
    gp = np.empty(u.shape + (3,), u.dtype)
    getattr(lib(), "svso_warp_backward_" + _sfx(u))(_p(u), *u.shape, _p(phi), _p(g), *map(_f, h),
                                                    INTERP[interp], BOUNDARY[bdry], _p(gu), _p(gp))
    return gu, gp


def prolongate(u, src_len, dst_shape, dst_len, interp="CUBIC_HERMITESPLINE", bdry="MIRROR"):
    """Resample a field between meshes (prolongationOps.cu:533-625).

    u: [Z,Y,X] / [Z,Y,X,3] / [Z,Y,X,3,3]; src_len, dst_len: (LZ, LY, LX); dst_shape: (NZ,NY,NX).
    """
    u = _c(u)
    tail = u.shape[3:]
    C = int(np.prod(tail)) if tail else 1
    out = np.empty(tuple(dst_shape) + tail, u.dtype)
    getattr(lib(), "svso_prolongate_" + _sfx(u))(_p(u), *u.shape[:3], C, *map(_f, src_len),
                                                 *dst_shape, *map(_f, dst_len), INTERP[interp],
                                                 BOUNDARY[bdry], _p(out))
    return out


def warp_cnn(m, phi, h=(1.0, 1.0, 1.0), interp="CUBIC_HERMITESPLINE", bdry="MIRROR"):
    """Batched warp m [B,C,Z,Y,X] by phi [B,Z,Y,X,3] (warpingOpsCNN.cu:97-128)."""
    m = _c(m)
    phi = _c(phi, m.dtype)
    out = np.empty_like(m)
    getattr(lib(), "svso_warp_cnn_" + _sfx(m))(_p(m), *m.shape, _p(phi), *map(_f, h),
                                               INTERP[interp], BOUNDARY[bdry], _p(out))
    return out


def gaussian_kernel3d(sigma: float) -> np.ndarray:
    """The reference's blur kernel (svs/utils/flow_utils.py:74-91, :106-107), float32 [k,k,k].

    Restated with the same torch CPU operations: ks = int(5 sigma) made odd, taps
    linspace(-ks//2, ks//2+1, ks), g = exp(-(t/sigma)^2/2) normalised, outer product normalised.
    """
    import torch
    ks = int(sigma * 5)
    if ks % 2 == 0:
        ks += 1
    ts = torch.linspace(-ks // 2, ks // 2 + 1, ks)
    gauss = torch.exp((-(ts / sigma) ** 2 / 2))
    k = gauss / gauss.sum()
    k3 = torch.einsum("i,j,k->ijk", k, k, k)
    k3 = k3 / k3.sum()
    return np.ascontiguousarray(k3.numpy().astype(np.float32))


def blur(vol, sigma: float = 1.0):
    """Zero-padded 3D convolution with the reference blur kernel (flow_utils.py:94-112)."""
    vol = _c(vol)
    w = gaussian_kernel3d(sigma)
    out = np.empty_like(vol)
    getattr(lib(), "svso_conv3d_" + _sfx(vol))(_p(vol), *vol.shape, _p(w), w.shape[0] // 2, _p(out))
    return out


def median_filter(u, ks: int = 3):
    """scipy.ndimage.median_filter(u, size=(ks,ks,ks,1)) with mode 'reflect' (flow_utils.py:131)."""
    u = _c(u)
    C = 1 if u.ndim == 3 else u.shape[3]
    out = np.empty_like(u)
    getattr(lib(), "svso_median3_" + _sfx(u))(_p(u), *u.shape[:3], C, int(ks), _p(out))
    return out


def tvl1_compute(I0, I1, params: SolverParams | None = None, u=None, p=None, dtype=np.float32):
    """Full coarse-to-fine TV-L1 solve of one frame pair (svs/modules/flow/tvl13d.py:122-162).

    Returns (u [Z,Y,X,3], p [Z,Y,X,3,3]) in `dtype`.
    """
    params = params or SolverParams()
    I0, I1 = _c(I0, dtype), _c(I1, dtype)
    nz, ny, nx = I0.shape
    w = gaussian_kernel3d(params.gaussian_blur_sigma) if params.use_gaussian_blur else None
    u_out = np.empty((nz, ny, nx, 3), dtype)
    p_out = np.empty((nz, ny, nx, 3, 3), dtype)
    u_in = None if u is None else _c(u, dtype)
    p_in = None if p is None else _c(p, dtype)
    cp = params.to_c()
    rc = getattr(lib(), "svso_tvl1_compute_" + _sfx(I0))(
        ctypes.byref(cp), _p(I0), _p(I1), nz, ny, nx,
        None if w is None else _p(w), 0 if w is None else w.shape[0] // 2,
        None if u_in is None else _p(u_in), None if p_in is None else _p(p_in),
        _p(u_out), _p(p_out))
    if rc != 0:
        raise ValueError("oracle: invalid sizes for the pyramid (every level needs N >= 3 per axis)")
    return u_out, p_out


def dice(a, b) -> float:
    a = _c(a, np.uint8)
    b = _c(b, np.uint8)
    return float(lib().svso_dice(_p(a), _p(b), ctypes.c_size_t(a.size)))


def hausdorff(a, b) -> float:
    a = _c(a, np.uint8)
    b = _c(b, np.uint8)
    return float(lib().svso_hausdorff(_p(a), _p(b), *a.shape[-3:]))


def propagate_masks(initial_mask, final_mask, forward_flow, backward_flow,
                    interp="CUBIC_HERMITESPLINE", bdry="MIRROR"):
    """svs/modules/flow/warping.py:205-243: chained float-mask warps both ways, then > 0.5.

    masks: [Z,Y,X]; flows: [T-1,Z,Y,X,3]. Returns (forward [T,Z,Y,X], backward [T,Z,Y,X]) float.
    """
    m_f = [np.asarray(initial_mask, np.float32)]
    m_b = [np.asarray(final_mask, np.float32)]
    for t in range(forward_flow.shape[0]):
        m_f.append(warp_cnn(m_f[-1][None, None], forward_flow[t][None], interp=interp, bdry=bdry)[0, 0])
        m_b.append(warp_cnn(m_b[-1][None, None], backward_flow[t][None], interp=interp, bdry=bdry)[0, 0])
    m_b.reverse()
    fwd = np.where(np.stack(m_f) > 0.5, 1.0, 0.0).astype(np.float32)
    bwd = np.where(np.stack(m_b) > 0.5, 1.0, 0.0).astype(np.float32)
    return fwd, bwd


def pyramid_shapes(shape, num_scales):
    """Level sizes with ceil halving (tvl13d.py:91-99)."""
    out = [tuple(shape)]
    for _ in range(1, num_scales):
        out.append(tuple(int(math.ceil(0.5 * n)) for n in out[-1]))
    return out
