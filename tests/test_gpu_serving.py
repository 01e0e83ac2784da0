"""The continuous-batching server: admission under a memory budget, overlapping requests, and
results that are the same alone and in the mix."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import synthetic
from singleventriclesegmentation_b200.serving import FlowServer

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

SMALL = dict(max_warps=2, max_outer_iterations=20)


def seq(T, shape, seed):
    return torch.from_numpy(synthetic.cine_sequence(T=T, shape=shape, seed=seed))


def test_results_are_identical_alone_and_in_the_mix(cuda):
    reqs = [(seq(4, (24, 24, 24), 1), None), (seq(3, (16, 24, 32), 2), None), (seq(5, (32, 16, 24), 3), None)]
    m = torch.from_numpy(np.stack([synthetic.ellipsoid_mask((24, 24, 24), (6, 5, 4))] * 2))
    reqs[0] = (reqs[0][0], m)
    alone = []
    for frames, masks in reqs:
        srv = FlowServer(budget_bytes=8 << 30, solver_args=SMALL)
        alone.append(srv.submit(frames, masks, (0, 2)).result(timeout=300))
        srv.close()
    srv = FlowServer(budget_bytes=8 << 30, solver_args=SMALL)
    futs = [srv.submit(frames, masks, (0, 2)) for frames, masks in reqs]
    mixed = [f.result(timeout=300) for f in futs]
    srv.close()
    assert srv.stats()["max_concurrent"] >= 2   # the requests overlapped on the device
    for a, b in zip(alone, mixed):
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
        assert (a[2] is None) == (b[2] is None)
        if a[2] is not None:
            assert torch.equal(a[2], b[2])


def test_budget_admits_as_memory_frees(cuda):
    frames = [seq(3, (24, 24, 24), s) for s in range(4)]
    probe = FlowServer(budget_bytes=1 << 40, solver_args=SMALL)
    one = probe._estimate(frames[0].shape)
    probe.close()
    srv = FlowServer(budget_bytes=int(one * 1.5), solver_args=SMALL)   # room for one at a time
    futs = [srv.submit(f) for f in frames]
    for f in futs:
        f.result(timeout=300)
    srv.close()
    st = srv.stats()
    assert st["completed"] == 4 and st["max_concurrent"] == 1
    big = FlowServer(budget_bytes=one // 2, solver_args=SMALL)
    with pytest.raises(MemoryError):
        big.submit(frames[0]).result(timeout=10)
    big.close()



def test_active_request_cap(cuda):
    frames = [seq(3, (16, 16, 24), s) for s in range(3)]
    srv = FlowServer(budget_bytes=8 << 30, solver_args=SMALL, max_active=1)
    futs = [srv.submit(f) for f in frames]
    capped = [f.result(timeout=300) for f in futs]
    srv.close()
    assert srv.stats()["completed"] == 3 and srv.stats()["max_concurrent"] == 1
    srv = FlowServer(budget_bytes=8 << 30, solver_args=SMALL, max_active=3)
    free = [srv.submit(f).result(timeout=300) for f in frames]
    srv.close()
    for a, b in zip(capped, free):
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
