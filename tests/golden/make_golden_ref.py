"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own compiled
extension (oracle/_ref/opticalFlow_cuda_ext/opticalFlow.so, built from the reference sources by
oracle/build_ref.sh) on seeded inputs. Needs a CUDA GPU.

    python tests/golden/make_golden_ref.py OUT_DIR [--full80 | --only80]

Writes OUT_DIR/ref_ops.npz (per-operator cases), OUT_DIR/ref_solve32.npz (a full default-config
solve of a 32^3 pair, with TF32 convolutions allowed as in the reference's default run and with
TF32 off), OUT_DIR/ref_masks.npz (mask propagation) and, with --full80 (or --only80, which skips
the small fixtures), the 80^3 fixtures:
  ref_solve80.npz  the single-pair workload (80^3 blob pair, seed 0, default configuration): the
                   flow on every 2nd voxel per axis, whole-field statistics, SHA-256 of the input
                   frames, the ellipsoid mask (semi-axes 15/12/10) warped with the flow (bits),
                   the reference's seconds per pair;
  ref_chain80.npz  the 35-frame 80^3 cine sequence (seed 0): the reference's flows of the forward
                   pairs t -> t+1 (t = 0..11) and backward pairs t -> t-1 (t = 12..1), the masks
                   at t = 0 (15/12/10) and t = 12 (13/12/10) propagated both ways through them
                   (warping.py:205-243, bits per frame), Dice / Hausdorff of the propagated end
                   masks against the given ones (warping.py:245-270), the first and last flow
                   of each direction on every 4th voxel, and the frames' SHA-256.

The extension must be built with the register cap of oracle/build_ref.sh; built stock for
sm_100a, five of its kernel families fail to launch and every flow comes back zero.

All displacements are kept well inside one volume length, because the reference folds sample
indices only once (svs/src/boundary.cuh:33-46) and reads out of bounds beyond that.
"""
from __future__ import annotations

import hashlib
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


def sha256(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float32).tobytes())
    return h.hexdigest()


def bits(masks) -> np.ndarray:
    """Binary masks [..., Z, Y, X] as packed bits over the last three axes."""
    m = np.asarray(masks) > 0.5
    return np.packbits(m.reshape(m.shape[:-3] + (-1,)), axis=-1)


# 80^3 workloads (the cine sequence and its mask times are those of bench.py)
SHAPE80 = (80, 80, 80)
T80, MASK_T1 = 35, 12


def full80(of, out_dir):
    from oracle import oracle as o
    torch.backends.cudnn.allow_tf32 = True  # the reference's default run
    # single pair: flow + warped ellipsoid
    I0, I1, ut = synthetic.frame_pair(SHAPE80, seed=0, device="cuda")
    secs, us = [], []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u, _ = ref_driver.tvl1_compute(of, t(I0), t(I1), SolverParams())
        torch.cuda.synchronize()
        secs.append(time.perf_counter() - t0)
        us.append(n(u))
    u = us[0]
    m = synthetic.ellipsoid_mask(SHAPE80, (15, 12, 10))
    mesh = of.MeshInfo3D(*SHAPE80, *(s - 1 for s in SHAPE80))
    warp = of.WarpingCNN3D(mesh, of.InterpolationType.INTERPOLATE_CUBIC_HERMITESPLINE, of.BoundaryType.BOUNDARY_MIRROR)
    mw = n(warp.forward(t(m)[None, None], t(u)[None]))[0, 0]
    e = np.sqrt(((u.astype(np.float64) - ut) ** 2).sum(-1))
    np.savez_compressed(os.path.join(out_dir, "ref_solve80.npz"), u_sub2=u[::2, ::2, ::2],
                        u_mean=u.mean(axis=(0, 1, 2)), u_absmax=np.abs(u).max(), epe_vs_truth=e.mean(),
                        rerun_max_diff=np.abs(us[0] - us[1]).max(), seconds=np.array(secs),
                        inputs_sha256=sha256(I0, I1), mask_warped_bits=bits(mw))
    print(f"reference 80^3 pair: {secs[0]:.2f} s, {secs[1]:.2f} s; rerun max diff {np.abs(us[0] - us[1]).max():.3e}; "
          f"EPE vs truth {e.mean():.4f}")
    # bidirectional mask chain over the first MASK_T1 steps of the cine sequence
    seq = synthetic.cine_sequence(T=T80, shape=SHAPE80, seed=0, device="cuda")
    fwd_pairs = [(k + 1, k) for k in range(MASK_T1)]           # warp mask t -> t+1
    bwd_pairs = [(k - 1, k) for k in range(MASK_T1, 0, -1)]    # warp mask t -> t-1
    t0 = time.perf_counter()
    ff = np.stack([n(ref_driver.tvl1_compute(of, t(seq[a]), t(seq[b]), SolverParams())[0]) for a, b in fwd_pairs])
    bf = np.stack([n(ref_driver.tvl1_compute(of, t(seq[a]), t(seq[b]), SolverParams())[0]) for a, b in bwd_pairs])
    torch.cuda.synchronize()
    chain_s = time.perf_counter() - t0
    m0 = synthetic.ellipsoid_mask(SHAPE80, (15, 12, 10))
    mT = synthetic.ellipsoid_mask(SHAPE80, (13, 12, 10))
    fm, bm = ref_driver.propagate_masks(of, t(m0)[None, None], t(mT)[None, None], t(ff), t(bf))
    fm, bm = n(fm)[:, 0], n(bm)[:, 0]
    metrics = np.array([o.dice(bm[0], fm[0]), o.dice(fm[-1], bm[-1]),
                        o.hausdorff(bm[0], fm[0]), o.hausdorff(fm[-1], bm[-1])])
    np.savez_compressed(os.path.join(out_dir, "ref_chain80.npz"), fwd_bits=bits(fm), bwd_bits=bits(bm),
                        ff_first_sub4=ff[0, ::4, ::4, ::4], ff_last_sub4=ff[-1, ::4, ::4, ::4],
                        bf_first_sub4=bf[0, ::4, ::4, ::4], bf_last_sub4=bf[-1, ::4, ::4, ::4],
                        fwd_pairs=np.array(fwd_pairs), bwd_pairs=np.array(bwd_pairs),
                        compute_metrics=metrics, frames_sha256=sha256(seq), seconds=chain_s)
    print(f"reference 80^3 chain: {len(fwd_pairs) + len(bwd_pairs)} solves in {chain_s:.1f} s; "
          f"end metrics (dice_bwd, dice_fwd, hd_bwd, hd_fwd) = {metrics}")


def main():
    out_dir = sys.argv[1]
    os.makedirs(out_dir, exist_ok=True)
    of = ref_driver.load_reference_module()
    if "--only80" in sys.argv:
        full80(of, out_dir)
        return
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
        full80(of, out_dir)
    print("golden fixtures written to", out_dir)


if __name__ == "__main__":
    main()
