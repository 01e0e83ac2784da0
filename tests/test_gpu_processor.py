"""The per-patient flow driver (svs/modules/flow/processor.py:95-121) on the device.

process_sequence must give, in the reference's output layout (T'-1, 3, X, Y, Z), what the
reference's loop gives: for each consecutive pair of the patient's time list, the solve of
(I0 = img[t_{j+1}], I1 = img[t_j]) followed by the median post-filter. The reference loop is
restated here with TVL13DOpticalFlow.compute and flow_utils.apply_median_filter per pair (every
pair is independent: the warm start is overwritten when num_scales > 1). process_patients writes
the same arrays through the asynchronous FlowWriter; the files must equal save_flow's."""
import numpy as np
import pytest
import torch

from singleventriclesegmentation_b200 import processor, synthetic
from singleventriclesegmentation_b200.flow_utils import apply_median_filter, compute_timepoints

pytestmark = pytest.mark.gpu


def make_solver():
    from oracle.oracle import SolverParams
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    P = SolverParams(max_warps=3, max_outer_iterations=40)
    return TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                             P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                             P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma,
                             P.interpolation_type, P.boundary_type, P.length_type, P.length,
                             torch.device("cuda"))


def reference_loop(img, tdia, tsys, mode, solver, ks):
    """processor.py:103-118 pair by pair."""
    *_, times = compute_timepoints(tdia, tsys, None, None, mode)
    nt, nz, ny, nx = img.shape
    us = torch.zeros((len(times) - 1, 3, nx, ny, nz), dtype=torch.float32, device=img.device)
    for j in range(len(times) - 1):
        u, _ = solver.compute(img[times[j + 1]], img[times[j]])
        u = apply_median_filter(u, ks)
        us[j] = u.permute(3, 2, 1, 0)
    return us


@pytest.mark.parametrize("mode", ["forward", "backward"])
def test_process_sequence_matches_reference_loop(cuda, mode):
    img = torch.from_numpy(synthetic.cine_sequence(T=6, shape=(20, 24, 28), seed=2)).cuda()
    solver = make_solver()
    got = processor.process_sequence(img, 1, 4, mode, solver, median_kernel=3)
    ref = reference_loop(img, 1, 4, mode, solver, 3)
    assert got.shape == (3, 3, 28, 24, 20)
    assert torch.equal(got, ref)


def test_process_patients_writes_flow_files_asynchronously(cuda, tmp_path):
    solver = make_solver()
    patients = [(f"p{i}", torch.from_numpy(synthetic.cine_sequence(T=5, shape=(20, 20, 24), seed=10 + i)).cuda(),
                 3 - i, i) for i in range(2)]  # the first patient has tsys < tdia
    paths = processor.process_patients(patients, solver, str(tmp_path / "async"))
    assert len(paths) == 4
    for name, img, tdia, tsys in patients:
        for mode in ("forward", "backward"):
            sync = processor.save_flow(str(tmp_path / "sync"), name, mode,
                                       processor.process_sequence(img, tdia, tsys, mode, solver, 3))
            a = processor.load_flow(str(tmp_path / "async"), name, mode)
            b = np.load(sync)
            assert a.dtype == np.float32 and a.shape == b.shape
            assert np.array_equal(a, b)
