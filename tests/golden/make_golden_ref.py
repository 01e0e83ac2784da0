"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own compiled
extension (oracle/_ref/opticalFlow_cuda_ext/opticalFlow.so, built from the reference sources by
oracle/build_ref.sh) on seeded inputs. Needs a CUDA GPU.

    python tests/golden/make_golden_ref.py OUT_DIR [--full80]

Writes OUT_DIR/ref_ops.npz (per-operator cases), OUT_DIR/ref_solve32.npz (a full default-config
solve of a 32^3 pair, with TF32 convolutions allowed as in the reference's default run and with
TF32 off), OUT_DIR/ref_masks.npz (mask propagation) and, with --full80, OUT_DIR/ref_solve80.npz
(the 80^3 single-pair workload: the flow on every 4th voxel, summary statistics and the
reference's wall time per pair).

The extension must be built with the register cap of oracle/build_ref.sh; built stock for
sm_100a, five of its kernel families fail to launch and every flow comes back zero.

All displacements are kept well inside one volume length, because the reference folds sample
indices only once (svs/src/boundary.cuh:33-46) and reads out of bounds beyond that.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_driver  # noqa: E402
from oracle.oracle import SolverParams  # noqa: E402
from singleventriclesegmentation_b200 import synthetic  # noqa: E402

SHAPE = (7, 9, 11)
BDRY = ["NEAREST", "MIRROR", "REFLECT"]
INTERP = ["NEAREST", "LINEAR", "CUBIC_HERMITESPLINE"]


def t(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def n(x):
    return x.detach().cpu().numpy()


def ops_cases(of):
    rng = np.random.default_rng(1234)
    out = {}
    b = rng.standard_normal(SHAPE).astype(np.float32)
    v = rng.standard_normal(SHAPE + (3,)).astype(np.float32)
    m = rng.standard_normal(SHAPE + (3, 3)).astype(np.float32)
    out["in_b"], out["in_v"], out["in_m"] = b, v, m
    mesh = of.MeshInfo3D(*SHAPE, *(s - 1 for s in SHAPE))
    meshf = of.MeshInfo3D(*SHAPE, 1.0, 2.0, 3.0)  # fixed lengths: h != 1
    for name, mm in (("dofs", mesh), ("fixed", meshf)):
        for bd in BDRY:
            op = of.Nabla3D_CD(mm, getattr(of.BoundaryType, "BOUNDARY_" + bd))
            out[f"nabla_fwd_{name}_{bd}"] = n(op.forward(t(b)))
            out[f"nabla_fwd_vf_{name}_{bd}"] = n(op.forwardVectorField(t(v)))
            out[f"nabla_bwd_{name}_{bd}"] = n(op.backward(t(v)))
            out[f"nabla_bwd_vf_{name}_{bd}"] = n(op.backwardVectorField(t(m)))
    g = (rng.standard_normal(SHAPE + (3,)) * (rng.uniform(size=SHAPE + (1,)) > 0.2)).astype(np.float32)
    out["in_g"] = g
    an = of.AnisotropicNabla3D(mesh, 5.0, 0.5)
    s_, n_, t1, t2 = an.computeTangentVecs(t(g))
    out["aniso_s"], out["aniso_n"], out["aniso_t1"], out["aniso_t2"] = n(s_), n(n_), n(t1), n(t2)
    out["aniso_apply"] = n(an.forwardVectorField(t(m), s_, n_, t1, t2))
    dv = (rng.standard_normal(SHAPE + (3, 3)) * 0.05).astype(np.float32)
    out["in_dv"] = dv
    out["prox_dual"] = n(of.TVL1OF3D_proxDual(t(dv), 0.5, 0.025, mesh))
    rho = (rng.standard_normal(SHAPE) * 0.1).astype(np.float32)
    gw = (rng.standard_normal(SHAPE + (3,)) * 0.3).astype(np.float32)
    gw[0, 0, :3] = 0.0  # exercise the g2 <= 1e-10 branch
    out["in_rho"], out["in_gw"] = rho, gw
    out["prox_primal"] = n(of.TVL1OF3D_proxPrimal(t(v), 0.37, 1.0, t(rho), t(gw), mesh))
    phi = rng.uniform(-3.0, 3.0, size=SHAPE + (3,)).astype(np.float32)
    out["in_phi"] = phi
    go = rng.standard_normal(SHAPE).astype(np.float32)
    out["in_gout"] = go
    for it in INTERP:
        for bd in BDRY:
            w = of.Warping3D(mesh, getattr(of.InterpolationType, "INTERPOLATE_" + it),
                             getattr(of.BoundaryType, "BOUNDARY_" + bd))
            out[f"warp_{it}_{bd}"] = n(w.forward(t(b), t(phi)))
            out[f"warp_vf_{it}_{bd}"] = n(w.forwardVectorField(t(v), t(phi)))
            gu, gp = w.backward(t(b), t(phi), t(go))
            out[f"warp_bwd_u_{it}_{bd}"], out[f"warp_bwd_phi_{it}_{bd}"] = n(gu), n(gp)
    cnn_m = rng.uniform(size=(2, 2) + SHAPE).astype(np.float32)
    cnn_phi = rng.uniform(-2.0, 2.0, size=(2,) + SHAPE + (3,)).astype(np.float32)
    out["in_cnn_m"], out["in_cnn_phi"] = cnn_m, cnn_phi
    for it in INTERP:
        w = of.WarpingCNN3D(mesh, getattr(of.InterpolationType, "INTERPOLATE_" + it), of.BoundaryType.BOUNDARY_MIRROR)
        out[f"warp_cnn_{it}"] = n(w.forward(t(cnn_m), t(cnn_phi)))
    small = (4, 5, 6)
    mesh_s = of.MeshInfo3D(*small, *(s - 1 for s in small))
    for it in INTERP:
        ie = getattr(of.InterpolationType, "INTERPOLATE_" + it)
        down = of.Prolongation3D(mesh, mesh_s, ie, of.BoundaryType.BOUNDARY_MIRROR)
        up = of.Prolongation3D(mesh_s, mesh, ie, of.BoundaryType.BOUNDARY_MIRROR)
        out[f"restrict_{it}"] = n(down.forward(t(b)))
        cv = t(v[:4, :5, :6])
        cm = t(m[:4, :5, :6])
        out[f"prolong_vf_{it}"] = n(up.forwardVectorField(cv))
        out[f"prolong_mf_{it}"] = n(up.forwardMatrixField(cm))
    return out


def solve_case(of, shape, seed, tf32, amplitude=2.0):
    torch.backends.cudnn.allow_tf32 = tf32
    I0, I1, u_true = synthetic.frame_pair(shape, seed=seed, amplitude=amplitude)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    u, p = ref_driver.tvl1_compute(of, t(I0), t(I1), SolverParams())
    torch.cuda.synchronize()
    return I0, I1, u_true, n(u), n(p), time.perf_counter() - t0


def main():
    out_dir = sys.argv[1]
    os.makedirs(out_dir, exist_ok=True)
    of = ref_driver.load_reference_module()
    np.savez_compressed(os.path.join(out_dir, "ref_ops.npz"), **ops_cases(of))
    I0, I1, ut, u, p, dt = solve_case(of, (32, 32, 32), 7, True)
    _, _, _, u_notf, _, _ = solve_case(of, (32, 32, 32), 7, False)
    np.savez_compressed(os.path.join(out_dir, "ref_solve32.npz"), I0=I0, I1=I1, u=u, u_notf32=u_notf,
                        p_absmax=np.abs(p).max(), seconds=dt)
    # mask propagation over a short sequence, flows from the reference solver itself
    torch.backends.cudnn.allow_tf32 = True
    seq = synthetic.cine_sequence(T=5, shape=(24, 24, 24), seed=3)
    P = SolverParams(max_outer_iterations=50, max_warps=5)
    ff = [n(ref_driver.tvl1_compute(of, t(seq[a]), t(seq[b]), P)[0]) for a, b in synthetic.sequence_pairs(5, "forward")]
    bf = [n(ref_driver.tvl1_compute(of, t(seq[a]), t(seq[b]), P)[0]) for a, b in synthetic.sequence_pairs(5, "backward")]
    ff, bf = np.stack(ff), np.stack(bf)
    m0 = synthetic.ellipsoid_mask((24, 24, 24), (7, 6, 5))
    mT = synthetic.ellipsoid_mask((24, 24, 24), (6, 6, 5))
    fm, bm = ref_driver.propagate_masks(of, t(m0)[None, None], t(mT)[None, None], t(ff), t(bf))
    np.savez_compressed(os.path.join(out_dir, "ref_masks.npz"), seq=seq, ff=ff, bf=bf, m0=m0, mT=mT,
                        fwd=n(fm), bwd=n(bm))
    if "--full80" in sys.argv:
        I0, I1, ut, u, p, dt = solve_case(of, (80, 80, 80), 0, True)
        _, _, _, u2, _, dt2 = solve_case(of, (80, 80, 80), 0, True)
        np.savez_compressed(os.path.join(out_dir, "ref_solve80.npz"), u_sub=u[::4, ::4, ::4],
                            u_mean=u.mean(axis=(0, 1, 2)), u_absmax=np.abs(u).max(),
                            epe_vs_truth=np.sqrt(((u - ut) ** 2).sum(-1)).mean(),
                            rerun_max_diff=np.abs(u - u2).max(), seconds=[dt, dt2])
        np.save(os.path.join(out_dir, "ref_u80_full.npy"), u)
        print(f"reference 80^3 solve: {dt:.2f} s, {dt2:.2f} s; rerun max diff {np.abs(u - u2).max():.3e}")
    print("golden fixtures written to", out_dir)


if __name__ == "__main__":
    main()
