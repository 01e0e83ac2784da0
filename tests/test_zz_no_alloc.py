"""The allocation-free entry point, svs_tvl1_solve_noalloc.

Some callers cannot call cudaMalloc: code whose device memory belongs to another allocator (a
framework's caching pool that has already reserved the GPU) and latency-critical loops in which
an allocation or a free would synchronize the device. For them the library offers one solve
whose scratch (pyramid, linearisation, dual state, descriptors, tile lists) lives in a static
32 MiB device array. This file calls it through the C ABI, twice in a row on different pairs, and
checks each flow against the planned batch solve (svs_tvl1_solve_batch with the same plain-load
iterate kernel) within the tolerance the solver tests use for identical kernels: for FP32 and
16-bit storage of the iteration state, with and without the median post-filter (which this
entry point runs on a buffer carved from the same array), and with a single scale. It is named
so that pytest collects it last.
"""
import ctypes

import pytest
import torch

from singleventriclesegmentation_b200 import _lib, synthetic
from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same kernels, same order of operations: equal up to float rounding


def solver(dev, storage="f32", median=0, scales=3):
    s = TVL13DOpticalFlow(scales, 2, 30, 1.0, 0.025, 2, (0.5, 0.5, 0.25, 1.0), True, (5.0, 0.5), True, 1.0,
                          "CUBIC_HERMITESPLINE", "MIRROR", "numDofs", (1, 1, 1), dev, storage=storage,
                          median_kernel=median)
    s.tile_id = 6  # the plain-load iterate kernel, which the allocation-free path uses
    return s


def noalloc(params, I0, I1, u):
    nz, ny, nx = I0.shape
    return _lib.lib().svs_tvl1_solve_noalloc(ctypes.byref(params), I0.data_ptr(), I1.data_ptr(), nz, ny, nx,
                                             u.data_ptr(), torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("storage,median,scales", [("f32", 0, 3), ("f32", 3, 3), ("f16-flow32", 0, 3),
                                                   ("f16-flow32", 3, 3), ("f32", 0, 1)])
def test_noalloc_solve_matches_planned_solve_on_two_calls(cuda, storage, median, scales):
    s = solver(cuda, storage, median, scales)
    params = s.params()
    for seed, shape in ((3, (24, 28, 32)), (4, (24, 28, 32))):
        I0, I1, _ = synthetic.frame_pair(shape, seed=seed)
        I0 = torch.from_numpy(I0).to(cuda)
        I1 = torch.from_numpy(I1).to(cuda)
        ref = s.compute_batch([I0], [I1])[0]
        u = torch.full_like(ref, float("nan"))
        _lib.check(noalloc(params, I0, I1, u))
        torch.cuda.synchronize()
        assert torch.isfinite(u).all()
        assert (u - ref).abs().max().item() <= TOL


def test_noalloc_rejects_volumes_beyond_its_scratch(cuda):
    s = solver(cuda)
    I0 = torch.zeros((80, 80, 80), device=cuda)
    u = torch.empty((80, 80, 80, 3), device=cuda)
    st = noalloc(s.params(), I0, I0, u)
    assert st == 1
    assert b"scratch" in _lib.lib().svs_last_error()
