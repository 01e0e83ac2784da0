"""The persistent iteration loop (svs_tvl1_plan_set_persistent): every iteration of a warp at a
level in one cooperative launch, CTAs meeting at a grid barrier between iterations. Its result
must be bitwise that of the per-iteration launches (same tiles, same arithmetic per voxel), for
every storage mode and boundary family; levels it cannot serve fall back to per-iteration launches;
and the bounded waits still report a stalled pipeline without hanging."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import _lib, synthetic
from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def make_solver(storage, **over):
    from oracle.oracle import SolverParams
    P = SolverParams(**over)
    return TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                             P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                             P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma,
                             P.interpolation_type, P.boundary_type, P.length_type, P.length,
                             torch.device("cuda"), storage=storage)


def solve(solver, shapes, persistent, seed=0, tile=0):
    pairs = [synthetic.frame_pair(sh, seed=seed + i) for i, sh in enumerate(shapes)]
    plan = solver.plan_for(shapes)
    if tile:
        plan.set_tile(tile)
    plan.set_persistent(persistent)
    outs = [torch.empty(tuple(sh) + (3,), device="cuda") for sh in shapes]
    plan.solve([torch.from_numpy(p[0]).cuda() for p in pairs], [torch.from_numpy(p[1]).cuda() for p in pairs], outs)
    plan.check()
    return outs, plan.level_persistent(solver.num_scales)


@pytest.mark.parametrize("storage,shapes,over", [
    ("f32", [(32, 32, 32)] * 3, {}),
    ("f16-flow32", [(40, 40, 40)] * 4, {}),
    ("bf16-flow32", [(24, 24, 24)] * 2, {}),
    ("f16-flow32", [(21, 37, 45)], {"boundary_type": "NEAREST"}),
])
def test_persistent_loop_equals_per_iteration_launches(cuda, storage, shapes, over):
    solver = make_solver(storage, max_warps=2, max_outer_iterations=30, **over)
    ref, lp0 = solve(solver, shapes, False)
    solver._plans.clear()
    got, lp1 = solve(solver, shapes, True)
    assert not any(lp0) and any(lp1), (lp0, lp1)
    for a, b in zip(ref, got):
        assert torch.equal(a, b)


def test_persistent_full_schedule_single_pair(cuda):
    """The default configuration (3 x 15 x 300) on one 32^3 pair: every warp of every level in
    one launch each."""
    solver = make_solver("f16-flow32")
    ref, _ = solve(solver, [(32, 32, 32)], False, seed=5)
    solver._plans.clear()
    got, lp = solve(solver, [(32, 32, 32)], True, seed=5)
    assert all(lp)
    assert torch.equal(ref[0], got[0])


def test_levels_without_the_form_fall_back(cuda):
    """A variant with no persistent form (a TMA-pipeline variant) keeps per-iteration launches
    with the persistent option on, with the same result."""
    tma = next(t for t in range(1, _lib.lib().svs_tvl1_num_tiles() + 1) if _lib.tile_info(t)["form"] == "tma")
    solver = make_solver("f32", max_warps=1, max_outer_iterations=20)
    ref, _ = solve(solver, [(24, 24, 24)], False, tile=tma)
    solver._plans.clear()
    got, lp = solve(solver, [(24, 24, 24)], True, tile=tma)
    assert not any(lp)
    assert torch.equal(ref[0], got[0])


def test_persistent_stall_times_out_and_recovers(cuda):
    solver = make_solver("f16-flow32", num_scales=1, max_warps=1, max_outer_iterations=4)
    I0, I1, _ = synthetic.frame_pair((24, 24, 24), seed=11)
    I0, I1 = torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda()
    plan = solver.plan_for([(24, 24, 24)])
    plan.set_persistent(True)
    ref = torch.empty((24, 24, 24, 3), device="cuda")
    plan.solve([I0], [I1], [ref])
    plan.check()
    assert plan.level_persistent(1) == [True]
    plan.set_stall_test(level=0, cta=0, plane=1, wait_us=2000)
    bad = torch.empty_like(ref)
    plan.solve([I0], [I1], [bad])
    with pytest.raises(_lib.SVSError) as e:
        plan.check()
    assert e.value.status == _lib.SVS_ERR_TIMEOUT
    plan.set_stall_test()
    again = torch.empty_like(ref)
    plan.solve([I0], [I1], [again])
    plan.check()
    assert torch.equal(again, ref)
