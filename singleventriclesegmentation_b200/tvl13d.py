"""TVL13DOpticalFlow: drop-in for svs/modules/flow/tvl13d.py backed by the fused batched solver.

The constructor takes the reference's arguments (tvl13d.py:14-31). `compute(I0, I1, u, p)`
returns (u, p) like the reference (tvl13d.py:122-162) but runs one fused solve (one CUDA graph)
instead of ~25 launches and 3 host syncs per iteration. `compute_batch` solves many independent
pairs (any mix of volume sizes) in one graph. `generate_pyramid` and `step` keep the reference's
per-operator structure on this package's operators (the "plain" form; it is the unfused
baseline and a drop-in for code that calls those methods).
"""
from __future__ import annotations

import collections
import ctypes
import math
from typing import Literal, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from . import opticalFlow
from ._lib import PairDesc, TVL1Params, check, ptr, stream_ptr
from .flow_utils import apply_gaussian_blur3d, get_interpolation_type, get_mesh_length


class SolverPlan:
    """Owns one svs_plan: device state and the captured CUDA graph for a fixed list of sizes."""

    def __init__(self, params: TVL1Params, dims: Sequence[Tuple[int, int, int]], device: torch.device):
        self.dims = [tuple(int(v) for v in d) for d in dims]
        self.device = device
        self.params = params
        arr = (ctypes.c_int * (3 * len(self.dims)))(*[v for d in self.dims for v in d])
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            check(_lib.lib().svs_tvl1_plan_create(ctypes.byref(params), len(self.dims), arr,
                                                  ctypes.byref(handle)))
        self._h = handle

    @classmethod
    def reserve(cls, params: TVL1Params, max_pairs: int, arena_bytes: int, device: torch.device) -> "SolverPlan":
        """A plan with room for up to max_pairs pairs and arena_bytes of device state, to be
        retarget()ed to each batch (svs_tvl1_plan_create_reserve)."""
        self = cls.__new__(cls)
        self.device = device
        self.params = params
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            check(_lib.lib().svs_tvl1_plan_create_reserve(ctypes.byref(params), int(max_pairs), int(arena_bytes),
                                                          ctypes.byref(handle)))
        self._h = handle
        side = 3 << (params.num_scales - 1)
        self.dims = [(side, side, side)] * int(max_pairs)
        self.capacity = int(max_pairs)
        return self

    @property
    def device_bytes(self) -> int:
        return int(_lib.lib().svs_tvl1_plan_device_bytes(self._h))

    def set_tile(self, tile_id: int) -> None:
        check(_lib.lib().svs_tvl1_plan_set_tile(self._h, int(tile_id)))

    def set_level_tile(self, level: int, tile_id: int) -> None:
        check(_lib.lib().svs_tvl1_plan_set_level_tile(self._h, int(level), int(tile_id)))

    def solve(self, I0s, I1s, u_outs, p_outs=None, u_inits=None, p_inits=None, stream=None):
        n = len(self.dims)
        descs = (PairDesc * n)()
        for i in range(n):
            nz, ny, nx = self.dims[i]
            descs[i].nz, descs[i].ny, descs[i].nx = nz, ny, nx
            descs[i].I0 = ptr(I0s[i])
            descs[i].I1 = ptr(I1s[i])
            descs[i].u_out = ptr(u_outs[i])
            descs[i].p_out = ptr(p_outs[i]) if p_outs is not None and p_outs[i] is not None else None
            descs[i].u_init = ptr(u_inits[i]) if u_inits is not None and u_inits[i] is not None else None
            descs[i].p_init = ptr(p_inits[i]) if p_inits is not None and p_inits[i] is not None else None
        s = stream if stream is not None else stream_ptr(self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().svs_tvl1_solve_batch(self._h, descs, n, s))

    def bench_iterations(self, level: int, count: int, stream=None) -> None:
        s = stream if stream is not None else stream_ptr(self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().svs_tvl1_bench_iterations(self._h, int(level), int(count), s))

    def check(self) -> None:
        """Raise if a bounded pipeline wait inside an iterate kernel gave up (synchronizes)."""
        with torch.cuda.device(self.device):
            check(_lib.lib().svs_tvl1_plan_check(self._h))

    def set_stall_test(self, level: int = -1, cta: int = -1, plane: int = -1, wait_us: int = 0) -> None:
        """Test hook of the bounded pipeline waits: at `level`, CTA `cta` never issues the copies
        of its staged plane number `plane`, and waits give up after wait_us (0 = 2 s); the next
        check() then raises with SVS_ERR_TIMEOUT. No arguments switch the stall off."""
        check(_lib.lib().svs_tvl1_plan_set_stall_test(self._h, int(level), int(cta), int(plane), int(wait_us)))

    def retarget(self, dims: Sequence[Tuple[int, int, int]], stream=None) -> None:
        """Take another batch (at most as many pairs as at creation, state within the arena)
        without allocating; synchronizes `stream`."""
        dims = [tuple(int(v) for v in d) for d in dims]
        arr = (ctypes.c_int * (3 * len(dims)))(*[v for d in dims for v in d])
        s = stream if stream is not None else stream_ptr(self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().svs_tvl1_plan_retarget(self._h, len(dims), arr, s))
        self.dims = dims

    def set_persistent(self, on: bool = True) -> None:
        """Run each warp's iterations of a level in one cooperative launch (grid barrier between
        iterations) where the level's variant has that form; the result is bitwise unchanged."""
        check(_lib.lib().svs_tvl1_plan_set_persistent(self._h, int(bool(on))))

    def level_persistent(self, levels: int = 3):
        """Per level, whether the captured solve runs the persistent loop (after a solve)."""
        return [bool(_lib.lib().svs_tvl1_plan_level_persistent(self._h, l)) for l in range(levels)]

    def level_tiles(self):
        return [int(_lib.lib().svs_tvl1_plan_level_tile(self._h, l)) for l in range(8)]

    def pair_tiles(self, level: int):
        """Variant each pair runs at `level` (its group's or the level's; after a solve)."""
        return [int(_lib.lib().svs_tvl1_plan_pair_tile_used(self._h, int(level), i)) for i in range(len(self.dims))]

    def level_ctas(self, level: int) -> int:
        """CTAs of one iterate launch at `level` (all variant groups; 0 before the first solve)."""
        return int(_lib.lib().svs_tvl1_plan_level_ctas(self._h, int(level)))

    def set_level_chunks(self, level: int, chunks: int) -> None:
        """z chunks per column tile at a level (0 = automatic)."""
        check(_lib.lib().svs_tvl1_plan_set_level_chunks(self._h, int(level), int(chunks)))

    def set_pair_tile(self, level: int, pair: int, tile_id: int) -> None:
        check(_lib.lib().svs_tvl1_plan_set_pair_tile(self._h, int(level), int(pair), int(tile_id)))

    def set_residuals(self, record: bool = True, stop_tol: float = 0.0) -> None:
        """Log the per-warp RMS change of each pair's flow (FP64 reduction) and, with stop_tol > 0,
        skip the remaining warps of a level once a pair's change falls below stop_tol."""
        with torch.cuda.device(self.device):
            check(_lib.lib().svs_tvl1_plan_set_residuals(self._h, int(bool(record)), float(stop_tol)))
        self._res_shape = (len(self.dims), self.params.num_scales, max(1, self.params.max_warps))

    def residuals(self) -> np.ndarray:
        """[pairs, levels, warps] log of the last solve (level 0 = finest, -1 = warp skipped)."""
        shape = getattr(self, "_res_shape", None)
        if shape is None:
            raise RuntimeError("residuals are not recorded (call set_residuals first)")
        out = np.empty(shape, dtype=np.float32)
        check(_lib.lib().svs_tvl1_plan_get_residuals(self._h, out.ctypes.data, out.size))
        return out

    @property
    def graph_kernels(self) -> int:
        return int(_lib.lib().svs_tvl1_plan_graph_kernels(self._h))

    def close(self):
        if self._h:
            _lib.lib().svs_tvl1_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TVL13DOpticalFlow:
    def __init__(
        self,
        num_scales: int,
        max_warps: int,
        max_outer_iterations: int,
        weight_matching: float,
        weight_tv: float,
        primaldual_algorithm_type: Literal[1, 2],
        primaldual_algorithm_params: Tuple[float, float, float, float],
        use_anisotropic_diff: bool,
        anisotropic_diff_params: Tuple[float, float],
        use_gaussian_blur: bool,
        gaussian_blur_sigma: float,
        interpolation_type: Literal["NEAREST", "LINEAR", "CUBIC_HERMITESPLINE"],
        boundary_type: Literal["NEAREST", "MIRROR", "REFLECT"],
        length_type: Literal["numDofs", "fixed"],
        length: Tuple[int, int, int],
        device: torch.device,
        storage: str = "f32",
        median_kernel: int = 0,
        max_cached_plans: int = 4,
    ):
        """Same arguments as tvl13d.py:14-31; `storage` selects f32 / bf16 / f16 storage of the
        iteration state (arithmetic stays float32); `median_kernel` > 1 applies the processor's
        median post-filter (processor.py:116-117) inside the solve."""
        self.num_scales = num_scales
        self.max_warps = max_warps
        self.max_outer_iterations = max_outer_iterations
        self.weight_matching = weight_matching
        self.weight_tv = weight_tv
        self.primaldual_algorithm_type = primaldual_algorithm_type
        self.sigma, self.tau, self.theta, self.gamma = primaldual_algorithm_params
        self.use_anisotropic_diff = use_anisotropic_diff
        self.anisotropic_diff_alpha, self.anistropic_diff_beta = anisotropic_diff_params
        self.use_gaussian_blur = use_gaussian_blur
        self.gaussian_blur_sigma = gaussian_blur_sigma
        self.length_type = length_type
        self.length_x, self.length_y, self.length_z = length
        self.interpolation_type, self.boundary_type = get_interpolation_type(interpolation_type, boundary_type)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.storage = storage
        self.median_kernel = int(median_kernel)
        self._plans: "collections.OrderedDict[tuple, SolverPlan]" = collections.OrderedDict()
        self._max_plans = max_cached_plans
        self.tile_id = 0

    # ------------------------------------------------------------------ fused solver
    def params(self) -> TVL1Params:
        p = TVL1Params()
        p.num_scales = self.num_scales
        p.max_warps = self.max_warps
        p.max_outer_iterations = self.max_outer_iterations
        p.weight_matching = self.weight_matching
        p.weight_tv = self.weight_tv
        p.primaldual_algorithm_type = self.primaldual_algorithm_type
        p.sigma, p.tau, p.theta, p.gamma = self.sigma, self.tau, self.theta, self.gamma
        p.use_anisotropic_diff = int(bool(self.use_anisotropic_diff))
        p.alpha, p.beta = self.anisotropic_diff_alpha, self.anistropic_diff_beta
        p.use_gaussian_blur = int(bool(self.use_gaussian_blur))
        p.gaussian_blur_sigma = self.gaussian_blur_sigma
        p.interpolation = int(self.interpolation_type)
        p.boundary = int(self.boundary_type)
        p.length_type = 0 if self.length_type == "numDofs" else 1
        p.length_z, p.length_y, p.length_x = self.length_z, self.length_y, self.length_x
        p.median_kernel = self.median_kernel
        p.storage = _lib.STORAGE[self.storage]
        return p

    def plan_for(self, dims: Sequence[Tuple[int, int, int]]) -> SolverPlan:
        key = tuple(tuple(d) for d in dims)
        plan = self._plans.get(key)
        if plan is None:
            plan = SolverPlan(self.params(), dims, self.device)
            if self.tile_id:
                plan.set_tile(self.tile_id)
            self._plans[key] = plan
            while len(self._plans) > self._max_plans:
                _, old = self._plans.popitem(last=False)
                old.close()
        else:
            self._plans.move_to_end(key)
        return plan

    @staticmethod
    def _frame(t: torch.Tensor, name: str) -> torch.Tensor:
        if t.device.type != "cuda" or t.dim() != 3:
            raise RuntimeError(f"{name} must be a 3D CUDA tensor")
        return t.float().contiguous()

    def compute(self, I0: torch.Tensor, I1: torch.Tensor, u: Optional[torch.Tensor] = None,
                p: Optional[torch.Tensor] = None) -> Tuple[torch.Tensor, torch.Tensor]:
        """tvl13d.py:122-162 for one pair: returns (u [Z,Y,X,3], p [Z,Y,X,3,3])."""
        I0 = self._frame(I0, "I0")
        I1 = self._frame(I1, "I1")
        if I0.shape != I1.shape:
            raise RuntimeError("I0 and I1 must have the same shape")
        nz, ny, nx = I0.shape
        u_out = torch.empty((nz, ny, nx, 3), dtype=torch.float32, device=I0.device)
        p_out = torch.empty((nz, ny, nx, 3, 3), dtype=torch.float32, device=I0.device)
        plan = self.plan_for([(nz, ny, nx)])
        warm = self.num_scales == 1
        plan.solve([I0], [I1], [u_out], [p_out],
                   [u.float().contiguous()] if (warm and u is not None) else None,
                   [p.float().contiguous()] if (warm and p is not None) else None)
        return u_out, p_out

    def compute_batch(self, I0s: Sequence[torch.Tensor], I1s: Sequence[torch.Tensor],
                      want_p: bool = False):
        """Solve many independent pairs (sizes may differ) in one captured graph.
        Returns a list of u (and of p when want_p)."""
        I0s = [self._frame(t, "I0") for t in I0s]
        I1s = [self._frame(t, "I1") for t in I1s]
        dims = [tuple(t.shape) for t in I0s]
        us = [torch.empty(d + (3,), dtype=torch.float32, device=t.device) for d, t in zip(dims, I0s)]
        ps = [torch.empty(d + (3, 3), dtype=torch.float32, device=t.device) for d, t in zip(dims, I0s)] if want_p else None
        self.plan_for(dims).solve(I0s, I1s, us, ps)
        return (us, ps) if want_p else us

    # ------------------------------------------------- reference-structured (plain) form
    def generate_pyramid(self, I0, I1, u, p):
        """tvl13d.py:69-120 on this package's operators."""
        if self.use_gaussian_blur:
            I0 = apply_gaussian_blur3d(I0, self.gaussian_blur_sigma)
            I1 = apply_gaussian_blur3d(I1, self.gaussian_blur_sigma)
        NZ, NY, NX = I0.shape
        LZ, LY, LX = get_mesh_length(self.length_type, NZ, NY, NX, self.length_z, self.length_y, self.length_x)
        mesh_infos = [opticalFlow.MeshInfo3D(NZ, NY, NX, LZ, LY, LX)]
        nz, ny, nx = NZ, NY, NX
        for _ in range(1, self.num_scales):
            nz, ny, nx = math.ceil(0.5 * nz), math.ceil(0.5 * ny), math.ceil(0.5 * nx)
            lz, ly, lx = get_mesh_length(self.length_type, nz, ny, nx, self.length_z, self.length_y, self.length_x)
            mesh_infos.append(opticalFlow.MeshInfo3D(nz, ny, nx, lz, ly, lx))
        I0s, I1s, us, ps = [I0], [I1], [u], [p]
        for s in range(1, self.num_scales):
            op = opticalFlow.Prolongation3D(mesh_infos[s - 1], mesh_infos[s], self.interpolation_type, self.boundary_type)
            I0s.append(op.forward(I0s[s - 1]))
            I1s.append(op.forward(I1s[s - 1]))
            m = mesh_infos[s]
            us.append(torch.zeros([m.getNZ(), m.getNY(), m.getNX(), 3], dtype=I0.dtype, device=self.device))
            ps.append(torch.zeros([m.getNZ(), m.getNY(), m.getNX(), 3, 3], dtype=I0.dtype, device=self.device))
        return I0s, I1s, us, ps, mesh_infos

    def compute_unfused(self, I0, I1, u, p):
        """tvl13d.py:122-162 exactly as the reference structures it (per-operator launches), in
        the inputs' type: float32 (the plain GPU form) or float64 (an FP64 GPU run of the same
        algorithm, the fast oracle for large volumes)."""
        I0s, I1s, us, ps, mesh_infos = self.generate_pyramid(I0, I1, u, p)
        for s in range(self.num_scales - 1, -1, -1):
            us[s], ps[s] = self.step(s, I0s[s], I1s[s], us[s], ps[s], mesh_infos[s])
            if s == 0:
                break
            op = opticalFlow.Prolongation3D(mesh_infos[s], mesh_infos[s - 1], self.interpolation_type, self.boundary_type)
            us[s - 1] = op.forwardVectorField(us[s])
            us[s - 1][..., 0] *= mesh_infos[s - 1].getLX() / mesh_infos[s].getLX()
            us[s - 1][..., 1] *= mesh_infos[s - 1].getLY() / mesh_infos[s].getLY()
            us[s - 1][..., 2] *= mesh_infos[s - 1].getLZ() / mesh_infos[s].getLZ()
            ps[s - 1] = op.forwardMatrixField(ps[s])
        return us[0], ps[0]

    def step(self, s, I0, I1, u, p, meshInfo, record_residuals: bool = False):
        """tvl13d.py:164-255 on this package's operators. The reference's three residual norms
        per iteration (host syncs whose results it never reads) are computed only when
        record_residuals is set."""
        nabla_op = opticalFlow.Nabla3D_CD(meshInfo, self.boundary_type)
        warping_op = opticalFlow.Warping3D(meshInfo, self.interpolation_type, self.boundary_type)
        I1_grad = nabla_op.forward(I1)
        shape = (meshInfo.getNZ(), meshInfo.getNY(), meshInfo.getNX())
        scalars = torch.zeros(shape, dtype=I1.dtype, device=self.device)
        normals = torch.zeros(shape + (3,), dtype=I1.dtype, device=self.device)
        tangents1 = torch.zeros_like(normals)
        tangents2 = torch.zeros_like(normals)
        if self.use_anisotropic_diff:
            aniso = opticalFlow.AnisotropicNabla3D(meshInfo, self.anisotropic_diff_alpha, self.anistropic_diff_beta)
            scalars, normals, tangents1, tangents2 = aniso.computeTangentVecs(I1_grad)
        z = u
        self.residuals = []
        for _ in range(self.max_warps):
            I1_warped = warping_op.forward(I1, u)
            I1_warped_grad = warping_op.forwardVectorField(I1_grad, u)
            rho_c = I1_warped - torch.sum(u * I1_warped_grad, dim=3) - I0
            sigma, tau, gamma = self.sigma, self.tau, self.gamma
            for _n in range(self.max_outer_iterations):
                pold = p
                z_grad = nabla_op.forwardVectorField(z)
                Dz_grad = z_grad
                if self.use_anisotropic_diff:
                    Dz_grad = aniso.forwardVectorField(z_grad, scalars, normals, tangents1, tangents2)
                p = opticalFlow.TVL1OF3D_proxDual(p + sigma * Dz_grad, sigma, self.weight_tv, meshInfo)
                if self.weight_tv == 0.0:
                    p = torch.zeros_like(p)
                uold = u
                rho = rho_c + torch.sum(u * I1_warped_grad, dim=3)
                Dp = p
                if self.use_anisotropic_diff:
                    Dp = aniso.backwardVectorField(p, scalars, normals, tangents1, tangents2)
                u = opticalFlow.TVL1OF3D_proxPrimal(u - tau * nabla_op.backwardVectorField(Dp), tau,
                                                    self.weight_matching, rho, I1_warped_grad, meshInfo)
                if self.primaldual_algorithm_type == 2:
                    theta = 1.0 / math.sqrt(1.0 + 2.0 * gamma * tau)
                    tau *= theta
                    sigma /= theta
                zold = z
                z = u
                if record_residuals:
                    self.residuals.append((torch.norm(p - pold).item(), torch.norm(u - uold).item(),
                                           torch.norm(z - zold).item()))
        return u, p
