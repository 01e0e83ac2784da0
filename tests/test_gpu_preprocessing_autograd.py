"""Preprocessing resample (svs/preprocessing/prolongation.py:67-85) against the oracle's
prolongation, and the differentiable warp (svs/src/warpingOps.py:13-29): autograd gradients equal
Warping3D.backward and pass a finite-difference check in FP64."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_resample_patient_matches_the_oracle(cuda, oracle):
    from singleventriclesegmentation_b200.preprocessing import resample_patient
    rng = np.random.default_rng(0)
    img = rng.uniform(size=(9, 11, 13, 6)).astype(np.float32)
    seg = (rng.uniform(size=(9, 11, 13)) > 0.5).astype(np.float32)
    out, sd, ss, fac = resample_patient(torch.from_numpy(img).cuda(), torch.from_numpy(seg).cuda(), None,
                                        shape=(16, 18, 20), pad_time=8)
    assert out.shape == (16, 18, 20, 8) and ss is None
    ref = oracle.prolongate(img, (8, 10, 12), (16, 18, 20), (15, 17, 19), interp="LINEAR", bdry="MIRROR")
    np.testing.assert_allclose(out[..., :6].cpu().numpy(), ref, rtol=1e-5, atol=1e-6)
    assert torch.count_nonzero(out[..., 6:]) == 0                   # zero-padded frames
    refm = np.round(oracle.prolongate(seg, (8, 10, 12), (16, 18, 20), (15, 17, 19), interp="LINEAR", bdry="MIRROR"))
    np.testing.assert_array_equal(sd.cpu().numpy(), refm)
    assert fac == (20 / 13, 18 / 11, 16 / 9, 8 / 6)


@pytest.mark.parametrize("interp", ["LINEAR", "CUBIC_HERMITESPLINE"])
def test_autograd_warp(cuda, interp):
    from singleventriclesegmentation_b200 import opticalFlow as of
    from singleventriclesegmentation_b200.warpingOps import warp
    sh = (5, 6, 7)
    rng = np.random.default_rng(1)
    mesh = of.MeshInfo3D(*sh, *(s - 1 for s in sh))
    op = of.Warping3D(mesh, getattr(of.InterpolationType, "INTERPOLATE_" + interp), of.BoundaryType.BOUNDARY_MIRROR)
    img = torch.tensor(rng.standard_normal(sh), dtype=torch.float64, device="cuda", requires_grad=True)
    flow = torch.tensor(rng.uniform(-1.3, 1.3, sh + (3,)), dtype=torch.float64, device="cuda", requires_grad=True)
    g = torch.tensor(rng.standard_normal(sh), dtype=torch.float64, device="cuda")
    (warp(img, flow, op) * g).sum().backward()
    gi, gf = op.backward(img.detach(), flow.detach(), g)
    # the image gradient is scattered with atomic adds, whose order differs from run to run
    torch.testing.assert_close(img.grad, gi, rtol=1e-12, atol=1e-14)
    assert torch.equal(flow.grad, gf)
    assert torch.autograd.gradcheck(lambda a, b: warp(a, b, op), (img, flow), eps=1e-6, atol=1e-5, rtol=1e-4)
