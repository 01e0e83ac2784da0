"""The continuous-batching server: admission under a memory budget, frame pairs of several
requests packed into shared batches, and results that are the same alone and in the mix."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import synthetic
from singleventriclesegmentation_b200.serving import FlowServer

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

SMALL = dict(max_warps=2, max_outer_iterations=20)
BATCH = 3 * 24 ** 3   # a batch of about three 24^3 pairs: requests' pairs share batches


def seq(T, shape, seed):
    return torch.from_numpy(synthetic.cine_sequence(T=T, shape=shape, seed=seed))


def server(**kw):
    args = dict(budget_bytes=8 << 30, solver_args=SMALL, batch_voxels=BATCH, max_batch_pairs=8)
    args.update(kw)
    return FlowServer(**args)


def test_results_are_identical_alone_and_in_the_mix(cuda):
    reqs = [(seq(4, (24, 24, 24), 1), None), (seq(3, (16, 24, 32), 2), None), (seq(5, (32, 16, 24), 3), None)]
    m = torch.from_numpy(np.stack([synthetic.ellipsoid_mask((24, 24, 24), (6, 5, 4))] * 2))
    reqs[0] = (reqs[0][0], m)
    alone = []
    for frames, masks in reqs:
        srv = server()
        alone.append(srv.submit(frames, masks, (0, 2)).result(timeout=300))
        srv.close()
    srv = server()
    futs = [srv.submit(frames, masks, (0, 2)) for frames, masks in reqs]
    mixed = [f.result(timeout=300) for f in futs]
    srv.close()
    st = srv.stats()
    assert st["max_concurrent"] >= 2      # the requests were on the device together
    assert st["mixed_batches"] >= 1       # and pairs of different requests shared a batch
    for a, b in zip(alone, mixed):
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
        assert (a[2] is None) == (b[2] is None)
        if a[2] is not None:
            assert torch.equal(a[2], b[2])


def test_flows_equal_the_batched_solver(cuda):
    """A request's flows are those of TVL13DOpticalFlow.compute_batch over its pairs."""
    frames = seq(4, (20, 24, 28), 7)
    srv = server()
    fwd, bwd, _ = srv.submit(frames).result(timeout=300)
    srv.close()
    T = frames.shape[0]
    pairs = [(t + 1, t) for t in range(T - 1)] + [(T - 2 - j, T - 1 - j) for j in range(T - 1)]
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    solver = TVL13DOpticalFlow(device=torch.device("cuda"), storage=srv.storage, **srv.solver_args)
    us = solver.compute_batch([frames[a].cuda() for a, b in pairs], [frames[b].cuda() for a, b in pairs])
    ref = torch.stack(us).cpu()
    assert torch.equal(torch.cat([fwd, bwd]), ref)


def test_budget_admits_as_memory_frees(cuda):
    frames = [seq(3, (24, 24, 24), s) for s in range(4)]
    probe = server(budget_bytes=1 << 40)
    one = probe._estimate(frames[0].shape)
    plans = probe.plan_bytes()
    probe.close()
    srv = server(budget_bytes=plans + int(one * 1.5))   # room for one request at a time
    futs = [srv.submit(f) for f in frames]
    for f in futs:
        f.result(timeout=300)
    srv.close()
    st = srv.stats()
    assert st["completed"] == 4 and st["max_concurrent"] == 1
    big = server(budget_bytes=plans + one // 2)
    with pytest.raises(MemoryError):
        big.submit(frames[0]).result(timeout=10)
    big.close()


def test_active_request_cap(cuda):
    frames = [seq(3, (16, 16, 24), s) for s in range(3)]
    srv = server(max_active=1)
    futs = [srv.submit(f) for f in frames]
    capped = [f.result(timeout=300) for f in futs]
    srv.close()
    assert srv.stats()["completed"] == 3 and srv.stats()["max_concurrent"] == 1
    srv = server()
    free = [srv.submit(f).result(timeout=300) for f in frames]
    srv.close()
    for a, b in zip(capped, free):
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
