"""The bounded-wait failure path of the TMA iterate kernels, exercised without faulting or hanging
the GPU: a test hook (svs_tvl1_plan_set_stall_test) makes one CTA leave one plane's copies
unissued and shortens every pipeline wait to a few milliseconds. The waiting threads give up,
record SVS_DEV_TIMEOUT, wait (bounded) for the copies their CTA did issue and return; the host
reads SVS_ERR_TIMEOUT from svs_tvl1_plan_check, and the next solve on the same plan and context
is bitwise the result of an undisturbed solve."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import _lib, synthetic

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]


def variants():
    """One variant per pipeline form: the automatic choice (split-role, block barrier per plane),
    the first TMA-pipeline variant and the first decoupled (mbarrier) split-role variant (id 21,
    include/svsflow.h)."""
    n = int(_lib.lib().svs_tvl1_num_tiles())
    info = [(t, _lib.tile_info(t)) for t in range(1, n + 1)]
    tma = next(t for t, i in info if i["form"] == "tma")
    return [0, tma, 21]


@pytest.mark.parametrize("tile", variants())
def test_stalled_plane_times_out_and_context_recovers(cuda, tile):
    from oracle.oracle import SolverParams
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    P = SolverParams(num_scales=1, max_warps=1, max_outer_iterations=4)
    solver = TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                               P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                               P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma,
                               P.interpolation_type, P.boundary_type, P.length_type, P.length,
                               torch.device("cuda"), storage="f16-flow32")
    I0, I1, _ = synthetic.frame_pair((24, 24, 24), seed=11)
    I0, I1 = torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda()
    plan = solver.plan_for([(24, 24, 24)])
    if tile:
        plan.set_tile(tile)
    out = lambda: torch.empty((24, 24, 24, 3), device="cuda")
    ref = out()
    plan.solve([I0], [I1], [ref])
    plan.check()
    plan.set_stall_test(level=0, cta=0, plane=1, wait_us=2000)
    bad = out()
    plan.solve([I0], [I1], [bad])
    with pytest.raises(_lib.SVSError) as e:
        plan.check()
    assert e.value.status == _lib.SVS_ERR_TIMEOUT
    plan.check()  # reported once
    plan.set_stall_test()
    again = out()
    plan.solve([I0], [I1], [again])
    plan.check()
    assert torch.equal(again, ref)
