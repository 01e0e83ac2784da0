"""Oracle-side driver: the reference's solver loop (svs/modules/flow/tvl13d.py:69-255) and mask
propagation (svs/modules/flow/warping.py:49-65, :205-243) restated so that they can run on ANY
module exposing the `opticalFlow` API. TEST INFRASTRUCTURE ONLY.

With the reference's own compiled extension (oracle/_ref/opticalFlow_cuda_ext/opticalFlow.so,
built by oracle/build_ref.sh) it reproduces the reference's outputs on the GPU box, which is how
the golden fixtures under tests/golden/ are made. The blur is restated from
svs/utils/flow_utils.py:74-112 with torch (cuDNN conv3d, as the reference).
"""
from __future__ import annotations

import importlib.util
import math
import os

import torch
import torch.nn.functional as F

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(_HERE, "_ref", "opticalFlow_cuda_ext", "opticalFlow.so")


def load_reference_module():
    """Import the reference's compiled `opticalFlow` extension (raises if it was not built)."""
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(f"reference extension not built: {REF_SO} (run oracle/build_ref.sh)")
    spec = importlib.util.spec_from_file_location("opticalFlow", REF_SO)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def gaussian_blur3d(vol: torch.Tensor, sigma: float) -> torch.Tensor:
    """flow_utils.py:74-112."""
    ks = int(sigma * 5)
    if ks % 2 == 0:
        ks += 1
    ts = torch.linspace(-ks // 2, ks // 2 + 1, ks)
    gauss = torch.exp((-(ts / sigma) ** 2 / 2))
    k = gauss / gauss.sum()
    k3d = torch.einsum("i,j,k->ijk", k, k, k).to(vol.device)
    k3d = k3d / k3d.sum()
    out = F.conv3d(vol.reshape(1, 1, *vol.shape), k3d.reshape(1, 1, *k3d.shape), stride=1, padding=len(k) // 2)
    return out.reshape(*vol.shape)


def tvl1_compute(of, I0, I1, params, u=None, p=None):
    """tvl13d.py:122-162 with the operators of module `of`. `params` is an
    oracle.SolverParams. Returns (u, p)."""
    dev = I0.device
    interp = getattr(of.InterpolationType, "INTERPOLATE_" + params.interpolation_type)
    bdry = getattr(of.BoundaryType, "BOUNDARY_" + params.boundary_type)
    lx, ly, lz = params.length

    def mesh_len(nz, ny, nx):
        return (nz - 1, ny - 1, nx - 1) if params.length_type == "numDofs" else (lz, ly, lx)

    if params.use_gaussian_blur:
        I0 = gaussian_blur3d(I0, params.gaussian_blur_sigma)
        I1 = gaussian_blur3d(I1, params.gaussian_blur_sigma)
    NZ, NY, NX = I0.shape
    meshes = [of.MeshInfo3D(NZ, NY, NX, *mesh_len(NZ, NY, NX))]
    nz, ny, nx = NZ, NY, NX
    for _ in range(1, params.num_scales):
        nz, ny, nx = math.ceil(0.5 * nz), math.ceil(0.5 * ny), math.ceil(0.5 * nx)
        meshes.append(of.MeshInfo3D(nz, ny, nx, *mesh_len(nz, ny, nx)))
    if u is None:
        u = torch.zeros((NZ, NY, NX, 3), dtype=torch.float32, device=dev)
    if p is None:
        p = torch.zeros((NZ, NY, NX, 3, 3), dtype=torch.float32, device=dev)
    I0s, I1s, us, ps = [I0], [I1], [u], [p]
    for s in range(1, params.num_scales):
        op = of.Prolongation3D(meshes[s - 1], meshes[s], interp, bdry)
        I0s.append(op.forward(I0s[s - 1]))
        I1s.append(op.forward(I1s[s - 1]))
        m = meshes[s]
        us.append(torch.zeros([m.getNZ(), m.getNY(), m.getNX(), 3], dtype=torch.float32, device=dev))
        ps.append(torch.zeros([m.getNZ(), m.getNY(), m.getNX(), 3, 3], dtype=torch.float32, device=dev))
    for s in range(params.num_scales - 1, -1, -1):
        us[s], ps[s] = _step(of, params, interp, bdry, I0s[s], I1s[s], us[s], ps[s], meshes[s])
        if s == 0:
            break
        op = of.Prolongation3D(meshes[s], meshes[s - 1], interp, bdry)
        us[s - 1] = op.forwardVectorField(us[s])
        us[s - 1][..., 0] *= meshes[s - 1].getLX() / meshes[s].getLX()
        us[s - 1][..., 1] *= meshes[s - 1].getLY() / meshes[s].getLY()
        us[s - 1][..., 2] *= meshes[s - 1].getLZ() / meshes[s].getLZ()
        ps[s - 1] = op.forwardMatrixField(ps[s])
    return us[0], ps[0]


def _step(of, P, interp, bdry, I0, I1, u, p, mesh):
    """tvl13d.py:164-255 (the never-read residual norms are left out)."""
    nabla = of.Nabla3D_CD(mesh, bdry)
    warping = of.Warping3D(mesh, interp, bdry)
    g = nabla.forward(I1)
    if P.use_anisotropic_diff:
        aniso = of.AnisotropicNabla3D(mesh, *P.anisotropic_diff_params)
        s, n, t1, t2 = aniso.computeTangentVecs(g)
    sigma0, tau0, _theta, gamma = P.primaldual_algorithm_params
    for _w in range(P.max_warps):
        I1w = warping.forward(I1, u)
        gw = warping.forwardVectorField(g, u)
        rho_c = I1w - torch.sum(u * gw, dim=3) - I0
        sigma, tau = sigma0, tau0
        for _n in range(P.max_outer_iterations):
            zg = nabla.forwardVectorField(u)
            Dz = aniso.forwardVectorField(zg, s, n, t1, t2) if P.use_anisotropic_diff else zg
            p = of.TVL1OF3D_proxDual(p + sigma * Dz, sigma, P.weight_tv, mesh)
            if P.weight_tv == 0.0:
                p = torch.zeros_like(p)
            rho = rho_c + torch.sum(u * gw, dim=3)
            Dp = aniso.backwardVectorField(p, s, n, t1, t2) if P.use_anisotropic_diff else p
            u = of.TVL1OF3D_proxPrimal(u - tau * nabla.backwardVectorField(Dp), tau, P.weight_matching, rho, gw, mesh)
            if P.primaldual_algorithm_type == 2:
                theta = 1.0 / math.sqrt(1.0 + 2.0 * gamma * tau)
                tau *= theta
                sigma /= theta
    return u, p


def propagate_masks(of, initial_mask, final_mask, forward_flow, backward_flow,
                    interpolation="CUBIC_HERMITESPLINE", boundary="MIRROR"):
    """warping.py:49-65 + :205-243 with module `of`. Masks [1,1,Z,Y,X]; flows [T-1,Z,Y,X,3]."""
    interp = getattr(of.InterpolationType, "INTERPOLATE_" + interpolation)
    bdry = getattr(of.BoundaryType, "BOUNDARY_" + boundary)

    def warp(x, u):
        NZ, NY, NX = x.shape[2:]
        mesh = of.MeshInfo3D(NZ, NY, NX, NZ - 1, NY - 1, NX - 1)
        return of.WarpingCNN3D(mesh, interp, bdry).forward(x.contiguous(), u.contiguous())

    fwd, bwd = [initial_mask], [final_mask]
    for t in range(forward_flow.shape[0]):
        fwd.append(warp(fwd[-1], forward_flow[t].unsqueeze(0)))
        bwd.append(warp(bwd[-1], backward_flow[t].unsqueeze(0)))
    bwd.reverse()
    return (torch.where(torch.cat(fwd, 0) > 0.5, 1.0, 0.0), torch.where(torch.cat(bwd, 0) > 0.5, 1.0, 0.0))
