"""Per-warp FP64 residuals and residual-driven stopping (svs_tvl1_plan_set_residuals): recording
changes no result, the logged value is the RMS flow change over the warp, and a pair that stops
gives the result of the shorter schedule, alone or inside a batch."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import synthetic
from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def solver(num_scales=3, max_warps=3, iters=20):
    return TVL13DOpticalFlow(num_scales, max_warps, iters, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5),
                             True, 1.0, "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), torch.device("cuda"))


def frames(shape, seed):
    I0, I1, _ = synthetic.frame_pair(shape, seed=seed)
    return torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda()


def run(s, pairs, record=False, tol=0.0):
    dims = [tuple(p[0].shape) for p in pairs]
    plan = s.plan_for(dims)
    plan.set_residuals(record, tol)
    outs = [torch.empty(d + (3,), device="cuda") for d in dims]
    plan.solve([p[0] for p in pairs], [p[1] for p in pairs], outs)
    torch.cuda.synchronize()
    plan.check()
    log = plan.residuals() if (record or tol > 0) else None
    s._plans.clear()
    return outs, log


def test_recording_changes_nothing(cuda):
    pair = frames((24, 24, 24), 5)
    s = solver()
    (u0,), _ = run(s, [pair])
    (u1,), log = run(s, [pair], record=True)
    assert torch.equal(u0, u1)
    assert log.shape == (1, 3, 3)
    assert np.all(np.isfinite(log)) and np.all(log > 0)


def test_residual_is_the_rms_flow_change_over_the_warp(cuda):
    pair = frames((20, 24, 28), 6)
    (u1,), _ = run(solver(1, 1), [pair])
    (u2,), log = run(solver(1, 2), [pair], record=True)
    a, b = u1.double().cpu().numpy(), u2.double().cpu().numpy()
    np.testing.assert_allclose(log[0, 0, 0], np.sqrt(np.mean(a ** 2)), rtol=1e-5)        # from u = 0
    np.testing.assert_allclose(log[0, 0, 1], np.sqrt(np.mean((b - a) ** 2)), rtol=1e-5)


def test_stopping_gives_the_shorter_schedule(cuda):
    pair = frames((24, 24, 24), 7)
    (u_short,), _ = run(solver(3, 1), [pair])
    (u_stop,), log = run(solver(3, 3), [pair], tol=1e9)   # every pair stops after its first warp
    assert torch.equal(u_short, u_stop)
    assert np.all(log[:, :, 0] > 0) and np.all(log[:, :, 1:] == -1)


def test_stopping_is_per_pair_inside_a_batch(cuda):
    pairs = [frames((24, 24, 24), 8), frames((16, 24, 32), 9), frames((24, 16, 24), 10)]
    s = solver(3, 4)
    _, free = run(s, pairs, record=True)
    tol = float(np.median(free[:, 0, 1:]))        # some pairs stop early at the finest level
    batch, blog = run(s, pairs, tol=tol)
    assert np.any(blog == -1)                     # at least one warp was skipped
    for i, p in enumerate(pairs):
        (alone,), alog = run(s, [p], tol=tol)
        assert torch.equal(alone, batch[i])
        np.testing.assert_array_equal(alog[0], blog[i])
