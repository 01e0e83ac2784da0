"""Fused batched solver parity: the CUDA path (C ABI svs_tvl1_solve_batch through
TVL13DOpticalFlow) against the oracle's restatement of tvl13d.py, the plain per-operator form,
and itself (batch invariance, tile invariance, graph reuse).

Tolerance (float32 arithmetic): mean end-point error <= 0.05 voxel against the oracle, the bar
the fused path must meet; the measured errors are far below it and are also bounded tightly."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import synthetic
from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

EPE_TOL = 0.05


def epe(a, b):
    return np.sqrt(((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2).sum(-1))


def make_solver(oracle_params=None, storage="f32", **over):
    from oracle.oracle import SolverParams
    P = oracle_params or SolverParams(**over)
    return TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                             P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                             P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma,
                             P.interpolation_type, P.boundary_type, P.length_type, P.length,
                             torch.device("cuda"), storage=storage), P


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


@pytest.fixture(scope="module")
def pair24():
    return synthetic.frame_pair((24, 24, 24), seed=7)


@pytest.fixture(scope="module")
def pair32():
    return synthetic.frame_pair((32, 32, 32), seed=7, amplitude=2.0)


@pytest.fixture(scope="module")
def oracle32(oracle, pair32):
    I0, I1, _ = pair32
    P = oracle.SolverParams()
    return oracle.tvl1_compute(I0, I1, P, dtype=np.float32)[0], oracle.tvl1_compute(I0, I1, P, dtype=np.float64)[0]


def test_fused_matches_oracle_default_config(cuda, oracle, pair32, oracle32):
    """Full default configuration (3 x 15 x 300). The solve is chaotic at a few voxels where the
    anisotropic operator vanishes, so the bound is on the mean and the 99th percentile; the
    FP32 oracle's own distance to the FP64 oracle calibrates what rounding alone produces."""
    I0, I1, _ = pair32
    solver, P = make_solver()
    u, p = solver.compute(T(I0), T(I1), None, None)
    u32, u64 = oracle32
    e = epe(u.cpu().numpy(), u32)
    spread = epe(u32, u64)
    print(f"fused vs oracle32: mean {e.mean():.3g} p99 {np.percentile(e, 99):.3g} max {e.max():.3g}; "
          f"oracle32 vs oracle64 mean {spread.mean():.3g}")
    assert e.mean() <= 0.01 and np.percentile(e, 99) <= 0.1


def test_fused_matches_fp64_oracle(cuda, oracle, pair32, oracle32):
    I0, I1, _ = pair32
    solver, P = make_solver()
    u, _ = solver.compute(T(I0), T(I1))
    u32, u64 = oracle32
    e = epe(u.cpu().numpy(), u64)
    spread = epe(u32, u64).mean()
    assert e.mean() <= EPE_TOL and e.mean() <= max(3 * spread, 0.005), (e.mean(), spread)


def test_fused_matches_plain_form(cuda, pair24):
    I0, I1, _ = pair24
    solver, P = make_solver(max_warps=4, max_outer_iterations=60)
    u, p = solver.compute(T(I0), T(I1))
    z = torch.zeros((24, 24, 24, 3), device="cuda")
    zp = torch.zeros((24, 24, 24, 3, 3), device="cuda")
    u2, p2 = solver.compute_unfused(T(I0), T(I1), z, zp)
    e = epe(u.cpu().numpy(), u2.cpu().numpy())
    assert e.mean() < 1e-3 and np.percentile(e, 99) < 2e-2, (e.mean(), e.max())


@pytest.mark.parametrize("params", [dict(use_anisotropic_diff=False), dict(primaldual_algorithm_type=1),
                                    dict(boundary_type="NEAREST"), dict(interpolation_type="LINEAR"),
                                    dict(use_gaussian_blur=False, weight_tv=0.0), dict(num_scales=2),
                                    dict(length_type="fixed", length=(20.0, 18.0, 16.0))])
def test_fused_matches_oracle_other_options(cuda, oracle, params):
    I0, I1, _ = synthetic.frame_pair((16, 18, 20), seed=11)
    solver, P = make_solver(max_warps=3, max_outer_iterations=40, **params)
    u, _ = solver.compute(T(I0), T(I1))
    uo, _ = oracle.tvl1_compute(I0, I1, P, dtype=np.float32)
    e = epe(u.cpu().numpy(), uo)
    assert e.mean() < 5e-3 and np.percentile(e, 99) < 0.05, (params, e.mean(), e.max())


def test_warm_start_single_scale(cuda, oracle):
    I0, I1, ut = synthetic.frame_pair((12, 13, 14), seed=5)
    solver, P = make_solver(num_scales=1, max_warps=2, max_outer_iterations=30)
    u0 = (ut * 0.5).astype(np.float32)
    p0 = np.full((12, 13, 14, 3, 3), 0.01, np.float32)
    u, p = solver.compute(T(I0), T(I1), T(u0), T(p0))
    uo, _ = oracle.tvl1_compute(I0, I1, P, u=u0, p=p0, dtype=np.float32)
    assert epe(u.cpu().numpy(), uo).mean() < 5e-3


def test_batch_invariance_and_uneven_sizes(cuda):
    """Each pair's result is bitwise the same alone and inside a batch of mixed sizes."""
    shapes = [(24, 24, 24), (16, 24, 32), (40, 24, 16)]
    pairs = [synthetic.frame_pair(s, seed=20 + i) for i, s in enumerate(shapes)]
    solver, _ = make_solver(max_warps=3, max_outer_iterations=50)
    together = solver.compute_batch([T(p[0]) for p in pairs], [T(p[1]) for p in pairs])
    for (I0, I1, _), ub in zip(pairs, together):
        ua = solver.compute_batch([T(I0)], [T(I1)])[0]
        assert torch.equal(ua, ub)


@pytest.mark.parametrize("storage,shape,over", [
    ("f32", (24, 24, 24), {}),
    ("bf16", (24, 24, 24), {}),
    ("bf16-flow32", (24, 24, 24), {}),
    # odd widths (a last pair of voxels with one outside the volume), two tiles in x and y
    ("f16-flow32", (21, 37, 45), {}),
    ("f32", (21, 37, 45), {"boundary_type": "NEAREST"}),
])
def test_tile_variants_agree(cuda, storage, shape, over):
    """Every iterate-kernel variant (TMA pipelines, split-role TMA pipelines and plain-load forms,
    all tile shapes) gives the same result: bitwise among the TMA and split-role forms (the same
    expression sequence per voxel), bitwise among the plain-load forms, and to rounding across
    the two."""
    from singleventriclesegmentation_b200 import _lib
    I0, I1, _ = synthetic.frame_pair(shape, seed=11)
    solver, _ = make_solver(storage=storage, max_warps=2, max_outer_iterations=30, **over)
    res = {}
    for tid in range(1, _lib.lib().svs_tvl1_num_tiles() + 1):
        solver.tile_id = tid
        solver._plans.clear()
        try:
            res[tid] = solver.compute_batch([T(I0)], [T(I1)])[0]
        except _lib.SVSError as e:   # a variant whose shared memory does not fit this storage
            assert e.status == 5, e
            continue
        for plan in solver._plans.values():
            plan.check()
    forms = {t: _lib.tile_info(t)["form"] for t in res}
    tma = [t for t in res if forms[t] in ("tma", "split")]
    plain = [t for t in res if forms[t] == "plain"]
    assert tma and plain and any(forms[t] == "split" for t in tma)
    for fam in (tma, plain):
        for t in fam[1:]:
            assert torch.equal(res[t], res[fam[0]]), (t, fam[0])
    e = epe(res[tma[0]].cpu().numpy(), res[plain[0]].cpu().numpy())
    assert e.mean() < 1e-4 and e.max() < 1e-2, (e.mean(), e.max())


def test_pair_variant_groups_run_concurrently_with_the_same_result(cuda):
    """Pairs given their own variants (svs_tvl1_plan_set_pair_tile) form groups that run as
    parallel graph branches; TMA and split-role variants are bitwise equal, so the result of every
    pair is unchanged."""
    shapes = [(24, 24, 24), (21, 37, 45), (20, 40, 40)]
    pairs = [synthetic.frame_pair(sh, seed=20 + i) for i, sh in enumerate(shapes)]
    solver, _ = make_solver(storage="f16-flow32", max_warps=2, max_outer_iterations=20)
    ref = solver.compute_batch([T(p[0]) for p in pairs], [T(p[1]) for p in pairs])
    solver._plans.clear()
    plan = solver.plan_for(shapes)
    # level 0: pairs 1 and 2 on two other variants; level 1: pair 0 on another one
    plan.set_pair_tile(0, 1, 17)
    plan.set_pair_tile(0, 2, 12)
    plan.set_pair_tile(1, 0, 9)
    outs = [torch.empty(sh + (3,), device="cuda") for sh in shapes]
    plan.solve([T(p[0]) for p in pairs], [T(p[1]) for p in pairs], outs)
    torch.cuda.synchronize()
    plan.check()
    for a, b in zip(ref, outs):
        assert torch.equal(a, b)
    plan.bench_iterations(0, 4)   # the grouped level also runs outside the graph
    torch.cuda.synchronize()
    plan.check()


def test_automatic_shapes_keep_two_ctas_per_sm(cuda):
    """The variants of the automatic choice for 2-byte fields (40x8 and 32x8 voxel pairs, 32x8 and
    16x16 single voxels) fit two CTAs per SM for every 2-byte storage mode: their register and
    shared-memory budgets are sized for it, and a kernel change that took one over the register
    budget would halve its occupancy without changing any result (a branch in the shrinkage step
    once took the 32x8 pair kernel to 202 registers, one CTA per SM)."""
    from singleventriclesegmentation_b200 import _lib

    def tid(tx, ty, v):
        for t in range(1, _lib.lib().svs_tvl1_num_tiles() + 1):
            i = _lib.tile_info(t)
            if i["form"] == "split" and (i["tx"], i["ty"], i["lane_voxels"]) == (tx, ty, v):
                return t

    pairs40 = _lib.auto_tiles(4, [(80, 80, 80)] * 68, 148)[0]
    pairs32, single32, single16 = tid(32, 8, 2), tid(32, 8, 1), tid(16, 16, 1)
    for storage in (1, 2, 3, 4):   # bf16, f16, bf16-flow32, f16-flow32
        occ = {t: _lib.tile_occupancy(storage, t) for t in (pairs40, pairs32, single32, single16)}
        print("storage", storage, "CTAs per SM", occ)
        assert min(occ.values()) >= 2, occ
    assert _lib.tile_occupancy(0, tid(32, 16, 2)) >= 1   # FP32 fields: 32x16 pairs


def test_automatic_pair_variants_keep_the_result(cuda):
    """At a level whose column tiles fill the GPU twice over, the automatic choice gives the pairs
    of each width the variant with the least modelled work (svs_tvl1_auto_tiles) and the plan runs
    them as groups; the result is bitwise that of one variant for every pair."""
    from singleventriclesegmentation_b200 import _lib
    shapes = [(12, 64, 64)] * 20 + [(12, 80, 80)] * 16 + [(12, 72, 96)] * 4
    pairs = [synthetic.frame_pair(sh, seed=40 + i) for i, sh in enumerate(shapes)]
    I0, I1 = [T(p[0]) for p in pairs], [T(p[1]) for p in pairs]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    main, own = _lib.auto_tiles(4, shapes, sms)   # f16-flow32
    assert len(set(o or main for o in own)) >= 2
    solver, _ = make_solver(storage="f16-flow32", max_warps=1, max_outer_iterations=10)
    plan = solver.plan_for(shapes)
    outs = [torch.empty(sh + (3,), device="cuda") for sh in shapes]
    plan.solve(I0, I1, outs)
    torch.cuda.synchronize()
    plan.check()
    assert plan.level_tiles()[0] == main
    assert plan.pair_tiles(0) == [o or main for o in own]
    solver1, _ = make_solver(storage="f16-flow32", max_warps=1, max_outer_iterations=10)
    solver1.tile_id = 28
    ref = solver1.compute_batch(I0, I1)
    for a, b in zip(ref, outs):
        assert torch.equal(a, b)


@pytest.mark.parametrize("storage", ["f32", "f16-flow32"])
def test_z_chunk_overrides_keep_the_result(cuda, storage):
    """Splitting the columns of a level into more z chunks (svs_tvl1_plan_set_level_chunks, down to
    one plane per chunk) changes only which CTA computes a plane, not its arithmetic: the result
    is bitwise that of the automatic split, for the split-role and the plain-load forms."""
    from singleventriclesegmentation_b200 import _lib
    shapes = [(21, 37, 45), (24, 24, 24)]
    pairs = [synthetic.frame_pair(sh, seed=30 + i) for i, sh in enumerate(shapes)]
    for tid in (0, 6):   # automatic (split-role) and plain-load 32x8
        solver, _ = make_solver(storage=storage, max_warps=2, max_outer_iterations=20)
        solver.tile_id = tid
        ref = solver.compute_batch([T(p[0]) for p in pairs], [T(p[1]) for p in pairs])
        for chunks in ((1, 1), (3, 7), (24, 12)):
            solver._plans.clear()
            plan = solver.plan_for(shapes)
            for level, c in enumerate(chunks):
                plan.set_level_chunks(level, c)
            outs = [torch.empty(sh + (3,), device="cuda") for sh in shapes]
            plan.solve([T(p[0]) for p in pairs], [T(p[1]) for p in pairs], outs)
            torch.cuda.synchronize()
            plan.check()
            for a, b in zip(ref, outs):
                assert torch.equal(a, b), (tid, chunks)
    with pytest.raises(_lib.SVSError):
        plan.set_level_chunks(5, 2)


def test_tail_columns_split_into_chunks_keep_the_result(cuda):
    """A batch whose column tiles overfill the resident CTA slots: the columns beyond the last
    full wave are cut into z chunks placed at the end of the launch, the other columns march whole.
    Every pair's result is bitwise that of one chunk per column."""
    # 34 pairs of 48^3 in 16x16 column tiles: 306 columns, which for 1 to 6 resident CTAs per SM
    # leave both whole-wave columns and a split tail
    shape = (48, 48, 48)
    n = 34
    pairs = [synthetic.frame_pair(shape, seed=40 + i % 4) for i in range(n)]
    solver, _ = make_solver(storage="f16-flow32", num_scales=1, max_warps=1, max_outer_iterations=10)
    plan = solver.plan_for([shape] * n)
    outs = [torch.empty(shape + (3,), device="cuda") for _ in range(n)]
    plan.solve([T(p[0]) for p in pairs], [T(p[1]) for p in pairs], outs)
    torch.cuda.synchronize()
    plan.check()
    tid = plan.level_tiles()[0]
    info = _lib_tile_info(tid)
    cols = n * -(-shape[1] // info["ty"]) * -(-shape[2] // info["tx"])
    auto_ctas = plan.level_ctas(0)
    assert auto_ctas > cols   # the tail columns were split
    plan.set_level_chunks(0, 1)
    ref = [torch.empty_like(o) for o in outs]
    plan.solve([T(p[0]) for p in pairs], [T(p[1]) for p in pairs], ref)
    torch.cuda.synchronize()
    plan.check()
    assert plan.level_ctas(0) == cols
    for a, b in zip(ref, outs):
        assert torch.equal(a, b)


def _lib_tile_info(tid):
    from singleventriclesegmentation_b200 import _lib
    return _lib.tile_info(tid)


def test_graph_reuse_and_new_inputs(cuda):
    solver, _ = make_solver(max_warps=2, max_outer_iterations=20)
    a = synthetic.frame_pair((16, 16, 16), seed=1)
    b = synthetic.frame_pair((16, 16, 16), seed=2)
    ua1 = solver.compute_batch([T(a[0])], [T(a[1])])[0]
    ub = solver.compute_batch([T(b[0])], [T(b[1])])[0]
    ua2 = solver.compute_batch([T(a[0])], [T(a[1])])[0]
    assert torch.equal(ua1, ua2) and not torch.equal(ua1, ub)


@pytest.mark.parametrize("storage,tol", [("f16-flow32", EPE_TOL), ("bf16-flow32", 0.1),
                                         ("bf16", 0.5), ("f16", 0.5)])
def test_reduced_storage_against_fp64_oracle(cuda, oracle, pair32, oracle32, storage, tol):
    """Reduced-precision storage of the iteration state, full default configuration, against
    the FP64 oracle. FP16 fields with an FP32 flow meet the EPE <= 0.05 target (measured 0.020);
    BF16 fields with an FP32 flow land just above it (0.052), and storing the flow itself in 16
    bits loses the small per-iteration updates (0.19 f16, 0.41 bf16): for those the bound is the
    measured behaviour, not the target."""
    I0, I1, _ = pair32
    solver, P = make_solver(storage=storage)
    u, _ = solver.compute(T(I0), T(I1))
    e = epe(u.cpu().numpy(), oracle32[1])
    print(f"{storage}: mean EPE vs fp64 {e.mean():.4g}, p99 {np.percentile(e, 99):.4g}, max {e.max():.4g}")
    assert e.mean() <= tol


def test_in_solve_median_equals_post_filter(cuda, pair24):
    from singleventriclesegmentation_b200.flow_utils import apply_median_filter
    I0, I1, _ = pair24
    s1, _ = make_solver(max_warps=2, max_outer_iterations=20)
    s2, _ = make_solver(max_warps=2, max_outer_iterations=20)
    s2.median_kernel = 3
    u = s1.compute_batch([T(I0)], [T(I1)])[0]
    um = s2.compute_batch([T(I0)], [T(I1)])[0]
    assert torch.equal(apply_median_filter(u, 3), um)


def test_retargeted_plan_equals_fresh_plans(cuda):
    """svs_tvl1_plan_retarget / svs_tvl1_plan_create_reserve: a plan re-used for batches of other
    sizes (fewer pairs, state within its arena) gives bitwise the results of plans made for those
    batches, and refuses a batch it cannot hold."""
    from singleventriclesegmentation_b200 import _lib
    from singleventriclesegmentation_b200.tvl13d import SolverPlan
    solver, _ = make_solver(storage="f16-flow32", max_warps=2, max_outer_iterations=20)
    batches = [[(24, 24, 24), (20, 28, 32)], [(32, 32, 32)], [(16, 16, 24)] * 3]
    reserved = SolverPlan.reserve(solver.params(), 4, 600 << 20, torch.device("cuda"))
    for b, dims in enumerate(batches):
        pairs = [synthetic.frame_pair(d, seed=40 + 3 * b + i) for i, d in enumerate(dims)]
        I0s, I1s = [T(p[0]) for p in pairs], [T(p[1]) for p in pairs]
        ref = solver.compute_batch(I0s, I1s)
        reserved.retarget(dims)
        outs = [torch.empty(d + (3,), device="cuda") for d in dims]
        reserved.solve(I0s, I1s, outs)
        reserved.check()
        for a, o in zip(ref, outs):
            assert torch.equal(a, o)
    with pytest.raises(_lib.SVSError) as e:
        reserved.retarget([(24, 24, 24)] * 5)   # more pairs than at creation
    assert e.value.status == 1
    with pytest.raises(_lib.SVSError) as e:
        reserved.retarget([(256, 256, 256)])    # more state than the arena
    assert e.value.status == 2
    reserved.close()
