"""Parity at the 80^3 workloads against the reference itself.

The fixtures ref_solve80.npz and ref_chain80.npz were written by the reference's own compiled
extension on a B200 (tests/golden/make_golden_ref.py --only80): the single-pair workload (an 80^3
blob pair, default configuration, svs/modules/flow/tvl13d.py:122-162) and the bidirectional mask
chain over the first 12 steps of the 35-frame 80^3 cine sequence (svs/modules/flow/warping.py:
205-243) with its end metrics (:245-270). The inputs are regenerated here from their seeds and
checked against the SHA-256 the generator recorded.

Tolerances (about 3x the spread measured on a B200, stated per test):
  flow      mean end-point error and its 99th percentile against the reference's flow; measured
            on the single pair: FP32 storage 0.00031 / 0.0021 voxel, f16-flow32 0.00063 / 0.0037
            (the chain's flows are closer still);
  masks     per frame Dice >= 0.999 and Hausdorff <= 1 voxel between our chain and the
            reference's chain (measured: FP32 identical, f16-flow32 worst Dice 0.99992, HD 1);
            the warped single-pair mask identical up to the same bounds; end metrics within 0.01
            (Dice) and 1 voxel (Hausdorff) of the reference's (measured: equal).
"""
import hashlib
import math
import os

import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import synthetic

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHAPE = (80, 80, 80)
MASK_T1 = 12

# bounds on the flow against the reference (voxels): mean and 99th percentile of the end-point
# error, per storage of the iteration state (arithmetic is FP32 in both)
FLOW_TOL = {"f32": (0.001, 0.0065), "f16-flow32": (0.002, 0.011)}


def load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"golden fixture missing: {path}")
    return np.load(path)


def sha256(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float32).tobytes())
    return h.hexdigest()


def unbits(b, shape=SHAPE) -> np.ndarray:
    n = int(np.prod(shape))
    return np.unpackbits(b, axis=-1)[..., :n].reshape(b.shape[:-1] + tuple(shape)).astype(np.float32)


def epe(a, b):
    return np.sqrt(((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2).sum(-1))


def solver(storage):
    from oracle.oracle import SolverParams
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    P = SolverParams()
    return TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                             P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                             P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma,
                             P.interpolation_type, P.boundary_type, P.length_type, P.length,
                             torch.device("cuda"), storage=storage)


@pytest.fixture(scope="module")
def pair80():
    I0, I1, _ = synthetic.frame_pair(SHAPE, seed=0, device="cuda")
    assert sha256(I0, I1) == str(load("ref_solve80.npz")["inputs_sha256"]), "regenerated inputs differ from the fixture's"
    return I0, I1


@pytest.fixture(scope="module")
def seq80():
    seq = synthetic.cine_sequence(T=35, shape=SHAPE, seed=0, device="cuda")
    assert sha256(seq) == str(load("ref_chain80.npz")["frames_sha256"]), "regenerated frames differ from the fixture's"
    return seq


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16-flow32"])
def test_pair80_flow_and_warped_mask_match_reference(cuda, pair80, storage):
    """Config 1: one 80^3 pair. The plain FP32 form (storage f32) and the headline storage form
    against the reference's flow (every 2nd voxel per axis), and the ellipsoid warped with each
    flow against the reference's warped ellipsoid."""
    from singleventriclesegmentation_b200.warping import Warp, dice, hausdorff
    d = load("ref_solve80.npz")
    I0, I1 = pair80
    u, _ = solver(storage).compute(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())
    e = epe(u[::2, ::2, ::2].cpu().numpy(), d["u_sub2"])
    mean_tol, p99_tol = FLOW_TOL[storage]
    print(f"{storage}: EPE vs reference mean {e.mean():.3g} p99 {np.percentile(e, 99):.3g} max {e.max():.3g}")
    assert e.mean() <= mean_tol and np.percentile(e, 99) <= p99_tol, (e.mean(), np.percentile(e, 99))
    m = torch.from_numpy(synthetic.ellipsoid_mask(SHAPE, (15, 12, 10))).cuda()[None, None]
    mw = (Warp("CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1))(m, u[None]) > 0.5).float()[0, 0]
    ref = torch.from_numpy(unbits(d["mask_warped_bits"])).cuda()
    dc, hd = dice(mw, ref), hausdorff(mw, ref)
    print(f"{storage}: warped mask vs reference Dice {dc:.5f} HD {hd}")
    assert dc >= 0.999 and hd <= 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16-flow32"])
def test_chain80_masks_match_reference(cuda, seq80, storage):
    """Config 2 masks: the 24 pairs of the chain solved in ONE batch (the headline path), the two
    masks propagated both ways with the device warp, compared frame by frame with the reference's
    chain (device Dice and Hausdorff), and the reference's end metrics (warping.py:245-270)
    reproduced within 0.01 Dice and 1 voxel."""
    from singleventriclesegmentation_b200.warping import Warp, compute_metrics, dice, hausdorff, propagate
    d = load("ref_chain80.npz")
    fwd_pairs = [tuple(p) for p in d["fwd_pairs"]]
    bwd_pairs = [tuple(p) for p in d["bwd_pairs"]]
    assert fwd_pairs == [(k + 1, k) for k in range(MASK_T1)]
    pairs = fwd_pairs + bwd_pairs
    seq = torch.from_numpy(seq80).cuda()
    us = solver(storage).compute_batch([seq[a] for a, b in pairs], [seq[b] for a, b in pairs])
    ff = torch.stack(us[:MASK_T1])
    bf = torch.stack(us[MASK_T1:])
    for key, got in (("ff_first_sub4", ff[0]), ("ff_last_sub4", ff[-1]), ("bf_first_sub4", bf[0]),
                     ("bf_last_sub4", bf[-1])):
        e = epe(got[::4, ::4, ::4].cpu().numpy(), d[key])
        print(f"{storage} {key}: EPE mean {e.mean():.3g} p99 {np.percentile(e, 99):.3g}")
        assert e.mean() <= FLOW_TOL[storage][0] and np.percentile(e, 99) <= FLOW_TOL[storage][1]
    m0 = torch.from_numpy(synthetic.ellipsoid_mask(SHAPE, (15, 12, 10))).cuda()[None, None]
    mT = torch.from_numpy(synthetic.ellipsoid_mask(SHAPE, (13, 12, 10))).cuda()[None, None]
    fm, bm = propagate(Warp("CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1)), m0, mT, ff, bf)
    ref_f = torch.from_numpy(unbits(d["fwd_bits"])).cuda()
    ref_b = torch.from_numpy(unbits(d["bwd_bits"])).cuda()
    worst_d, worst_h = 1.0, 0.0
    for t in range(MASK_T1 + 1):
        for got, ref in ((fm[t, 0], ref_f[t]), (bm[t, 0], ref_b[t])):
            dc, hd = dice(got, ref), hausdorff(got, ref)
            worst_d, worst_h = min(worst_d, dc), max(worst_h, hd)
    print(f"{storage}: chain vs reference worst Dice {worst_d:.5f} worst HD {worst_h}")
    assert worst_d >= 0.999 and worst_h <= 1.0
    got = compute_metrics(fm, bm)
    ref = d["compute_metrics"]
    print(f"{storage}: end metrics {got} reference {ref}")
    assert abs(got[0] - ref[0]) <= 0.01 and abs(got[1] - ref[1]) <= 0.01
    assert abs(got[2] - ref[2]) <= 1.0 and abs(got[3] - ref[3]) <= 1.0


def _edge_cases():
    s = (12, 13, 14)
    z = np.zeros(s, np.float32)
    one = z.copy()
    one[5, 6, 7] = 1
    corner = z.copy()
    corner[0, 0, 0] = 1
    border = z.copy()
    border[:, :3, :] = 1  # touches four faces
    full = np.ones(s, np.float32)
    rng = np.random.default_rng(5)
    blob_a = synthetic.ellipsoid_mask(s, (4, 5, 3))
    blob_b = synthetic.ellipsoid_mask(s, (5, 4, 3), center=(6.0, 5.0, 7.5))
    noise = (rng.uniform(size=s) > 0.7).astype(np.float32)
    return [("empty-empty", z, z), ("empty-one", z, one), ("one-one", one, one), ("one-corner", one, corner),
            ("border-blob", border, blob_a), ("full-blob", full, blob_b), ("blob-blob", blob_a, blob_b),
            ("noise-blob", noise, blob_a)]


@pytest.mark.gpu
def test_device_dice_hausdorff_match_oracle(cuda, oracle):
    """The device metrics (warping.dice / warping.hausdorff, monai's definitions as the reference
    calls them) against the oracle's C restatement: empty masks (NaN / inf), single voxels, masks
    touching the volume border, a full volume, overlapping ellipsoids and scattered voxels."""
    from singleventriclesegmentation_b200.warping import dice, hausdorff
    for name, a, b in _edge_cases():
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        hd, hd_ref = hausdorff(ta, tb), oracle.hausdorff(a, b)
        dc, dc_ref = dice(ta, tb), oracle.dice(a, b)
        for got, ref in ((hd, hd_ref), (dc, dc_ref)):
            if math.isnan(ref):
                assert math.isnan(got), name
            elif math.isinf(ref):
                assert math.isinf(got), name
            else:
                assert abs(got - ref) <= 1e-12, (name, got, ref)
