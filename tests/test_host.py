"""Host logic that needs no GPU: the drop-in module's argument checks, enums and meshes, the
synthetic inputs, the processor's pair list and file layout, and the multi-process replica
plumbing (world_size 2 over gloo)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from singleventriclesegmentation_b200 import opticalFlow, processor, replicas, synthetic
from singleventriclesegmentation_b200.flow_utils import (compute_timepoints, gaussian_kernel3d,
                                                         get_interpolation_type, get_mesh_length)


def test_enums_and_mesh_match_the_reference_binding():
    assert int(opticalFlow.BoundaryType.BOUNDARY_MIRROR) == 1
    assert int(opticalFlow.INTERPOLATE_CUBIC_HERMITESPLINE) == 2
    m = opticalFlow.MeshInfo3D(80, 40, 20, 79, 39, 19)
    assert (m.getNZ(), m.getNY(), m.getNX()) == (80, 40, 20)
    assert m.gethX() == 1.0 and m.getLY() == 39.0
    f = opticalFlow.MeshInfo3D(11, 11, 11, 1, 1, 1)
    assert f.gethZ() == pytest.approx(0.1, rel=1e-7)
    assert get_mesh_length("numDofs", 80, 40, 20, 1, 1, 1) == (79, 39, 19)
    assert get_interpolation_type("LINEAR", "REFLECT") == (opticalFlow.INTERPOLATE_LINEAR, opticalFlow.BOUNDARY_REFLECT)
    with pytest.raises(Exception):
        get_interpolation_type("CUBIC", "MIRROR")


def test_operators_reject_cpu_and_strided_tensors():
    m = opticalFlow.MeshInfo3D(4, 4, 4, 3, 3, 3)
    op = opticalFlow.Nabla3D_CD(m, opticalFlow.BOUNDARY_MIRROR)
    with pytest.raises(RuntimeError, match="CUDA"):
        op.forward(torch.zeros(4, 4, 4))
    with pytest.raises(RuntimeError, match="CUDA"):
        opticalFlow.TVL1OF3D_proxDual(torch.zeros(4, 4, 4, 3, 3), 0.5, 0.025, m)


def test_blur_kernel_is_the_reference_kernel():
    k = gaussian_kernel3d(1.0)
    assert tuple(k.shape) == (5, 5, 5)
    assert float(k.sum()) == pytest.approx(1.0, abs=1e-6)
    ts = torch.linspace(-5 // 2, 5 // 2 + 1, 5)
    assert ts.tolist() == [-3.0, -1.5, 0.0, 1.5, 3.0]


def test_timepoints_and_pairs_follow_the_processor():
    tp, segs, times = compute_timepoints(12, 3, "dia", "sys", "forward")
    assert tp == (3, 12) and segs == ("sys", "dia") and times == list(range(3, 13))
    *_, back = compute_timepoints(0, 4, None, None, "backward")
    assert back == [4, 3, 2, 1, 0]
    assert processor.pair_indices(0, 4, "forward") == [(1, 0), (2, 1), (3, 2), (4, 3)]
    assert processor.pair_indices(0, 4, "backward") == [(3, 4), (2, 3), (1, 2), (0, 1)]
    assert synthetic.sequence_pairs(5, "forward") == processor.pair_indices(0, 4, "forward")


def test_flow_file_layout_round_trip(tmp_path):
    us = torch.arange(2 * 3 * 4 * 5 * 6, dtype=torch.float32).reshape(2, 3, 4, 5, 6)  # (t, 3, x, y, z)
    path = processor.save_flow(str(tmp_path), "P001", "forward", us)
    assert os.path.basename(path) == "P001_forward_flow.npy"
    back = processor.load_flow(str(tmp_path), "P001", "forward")
    assert back.shape == (2, 3, 4, 5, 6) and back.dtype == np.float32
    w = processor.flows_for_warping(back)
    assert tuple(w.shape) == (2, 6, 5, 4, 3)        # (t, z, y, x, 3)
    assert float(w[1, 2, 3, 1, 0]) == float(us[1, 0, 1, 3, 2])


def test_synthetic_inputs_are_seeded_and_bounded():
    a = synthetic.frame_pair((12, 13, 14), seed=5)
    b = synthetic.frame_pair((12, 13, 14), seed=5)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    I0 = a[0]
    assert I0.min() >= 0.0 and I0.max() <= 1.0
    seq = synthetic.cine_sequence(T=4, shape=(10, 10, 10), seed=1)
    assert seq.shape == (4, 10, 10, 10)
    m = synthetic.ellipsoid_mask((80, 80, 80), (15, 12, 10))
    assert abs(m.sum() - 4 / 3 * np.pi * 15 * 12 * 10) / m.sum() < 0.02


def test_shard_covers_every_unit_once():
    for n in range(0, 20):
        for w in (1, 2, 3, 8):
            parts = [replicas.shard(list(range(n)), r, w) for r in range(w)]
            assert sum(parts, []) == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        units = [(i, i + 1) for i in range(68)]
        mine = replicas.shard(units, rank, world)
        slow = replicas.max_over_ranks(1.0 + rank)
        total = replicas.sum_over_ranks(len(mine))
        q.put((rank, len(mine), slow, total))
    finally:
        dist.destroy_process_group()


def test_replicas_over_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [34, 34]
    assert all(r[2] == 2.0 for r in res)      # the slowest rank's time
    assert all(r[3] == 68 for r in res)       # every pair solved once


def test_poisson_stream_shape():
    from singleventriclesegmentation_b200.serving import poisson_requests
    reqs = poisson_requests(rate=5.0, duration_s=4.0, seed=1)
    assert 5 <= len(reqs) <= 40
    for t, T, dims in reqs:
        assert 12 <= T <= 35 and all(64 <= d <= 128 and d % 8 == 0 for d in dims)


def test_time_pading_zero_pads_the_time_axis():
    import torch
    from singleventriclesegmentation_b200.preprocessing import time_pading
    x = torch.arange(2 * 3 * 4 * 5, dtype=torch.float32).reshape(2, 3, 4, 5)
    y = time_pading(8, x)
    assert y.shape == (2, 3, 4, 8)
    assert torch.equal(y[..., :5], x) and torch.count_nonzero(y[..., 5:]) == 0
