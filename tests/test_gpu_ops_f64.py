"""FP64 forms of the per-operator entry points (svs_*_f64) through the drop-in module with
float64 tensors, against the oracle's double instantiation; and the plain solver run in FP64 on
the GPU (the fast FP64 oracle for large volumes) against the oracle's FP64 solve.

Tolerance: relative 1e-9 per operator (both sides compute in double; only the order of a few
roundings differs). Scalars are exactly representable in float32 because the oracle's C interface
takes float scalars."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SH = (7, 9, 11)
BD = ["NEAREST", "MIRROR", "REFLECT"]
IT = ["NEAREST", "LINEAR", "CUBIC_HERMITESPLINE"]
RT, AT = 1e-9, 1e-11


def D(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def N(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def of():
    from singleventriclesegmentation_b200 import opticalFlow
    return opticalFlow


def mesh(of, sh=SH):
    return of.MeshInfo3D(*sh, *(s - 1 for s in sh))


@pytest.mark.parametrize("bdry", BD)
def test_nabla_f64(cuda, oracle, of, bdry):
    rng = np.random.default_rng(10)
    b, v, m = rng.standard_normal(SH), rng.standard_normal(SH + (3,)), rng.standard_normal(SH + (3, 3))
    op = of.Nabla3D_CD(mesh(of), getattr(of.BoundaryType, "BOUNDARY_" + bdry))
    out = op.forward(D(b))
    assert out.dtype == torch.float64
    np.testing.assert_allclose(N(out), oracle.nabla_forward(b, bdry=bdry), rtol=RT, atol=AT)
    np.testing.assert_allclose(N(op.forwardVectorField(D(v))), oracle.nabla_forward_vf(v, bdry=bdry), rtol=RT, atol=AT)
    np.testing.assert_allclose(N(op.backward(D(v))), oracle.nabla_backward(v, bdry=bdry), rtol=RT, atol=AT)
    np.testing.assert_allclose(N(op.backwardVectorField(D(m))), oracle.nabla_backward_vf(m, bdry=bdry), rtol=RT, atol=AT)


def test_aniso_and_proxes_f64(cuda, oracle, of):
    rng = np.random.default_rng(11)
    g = rng.standard_normal(SH + (3,)) * (rng.uniform(size=SH + (1,)) > 0.2)
    m = rng.standard_normal(SH + (3, 3))
    an = of.AnisotropicNabla3D(mesh(of), 5.0, 0.5)
    got = an.computeTangentVecs(D(g))
    ref = oracle.aniso_tangents(g, 5.0, 0.5)
    for a, b in zip(got, ref):
        np.testing.assert_allclose(N(a), b, rtol=RT, atol=AT)
    np.testing.assert_allclose(N(an.forwardVectorField(D(m), *got)), oracle.aniso_apply(m, *ref[:3]), rtol=RT, atol=AT)
    dv = rng.standard_normal(SH + (3, 3)) * 0.05
    np.testing.assert_allclose(N(of.TVL1OF3D_proxDual(D(dv), 0.5, 0.03125, mesh(of))), oracle.prox_dual(dv, 0.03125),
                               rtol=RT, atol=AT)
    pv, rho, gw = rng.standard_normal(SH + (3,)), rng.standard_normal(SH) * 0.1, rng.standard_normal(SH + (3,)) * 0.3
    np.testing.assert_allclose(N(of.TVL1OF3D_proxPrimal(D(pv), 0.375, 1.0, D(rho), D(gw), mesh(of))),
                               oracle.prox_primal(pv, 0.375, 1.0, rho, gw), rtol=RT, atol=AT)


@pytest.mark.parametrize("interp", IT)
@pytest.mark.parametrize("bdry", BD)
def test_warp_f64(cuda, oracle, of, interp, bdry):
    rng = np.random.default_rng(12)
    b, v = rng.standard_normal(SH), rng.standard_normal(SH + (3,))
    phi = rng.uniform(-3.0, 3.0, size=SH + (3,))
    w = of.Warping3D(mesh(of), getattr(of.InterpolationType, "INTERPOLATE_" + interp),
                     getattr(of.BoundaryType, "BOUNDARY_" + bdry))
    np.testing.assert_allclose(N(w.forward(D(b), D(phi))), oracle.warp(b, phi, interp=interp, bdry=bdry), rtol=RT, atol=AT)
    np.testing.assert_allclose(N(w.forwardVectorField(D(v), D(phi))), oracle.warp(v, phi, interp=interp, bdry=bdry),
                               rtol=RT, atol=AT)
    g = rng.standard_normal(SH)
    gu, gp = w.backward(D(b), D(phi), D(g))
    ru, rp = oracle.warp_backward(b, phi, g, interp=interp, bdry=bdry)
    np.testing.assert_allclose(N(gu), ru, rtol=1e-8, atol=1e-10)   # atomic sums in another order
    np.testing.assert_allclose(N(gp), rp, rtol=RT, atol=AT)
    m = rng.uniform(size=(2, 1) + SH)
    ph2 = rng.uniform(-2, 2, size=(2,) + SH + (3,))
    wc = of.WarpingCNN3D(mesh(of), getattr(of.InterpolationType, "INTERPOLATE_" + interp),
                         getattr(of.BoundaryType, "BOUNDARY_" + bdry))
    np.testing.assert_allclose(N(wc.forward(D(m), D(ph2))), oracle.warp_cnn(m, ph2, interp=interp, bdry=bdry),
                               rtol=RT, atol=AT)


def test_prolongation_blur_median_f64(cuda, oracle, of):
    from singleventriclesegmentation_b200 import flow_utils
    rng = np.random.default_rng(13)
    fine, coarse = SH, (4, 5, 6)
    up = of.Prolongation3D(mesh(of, coarse), mesh(of, fine), of.InterpolationType.INTERPOLATE_CUBIC_HERMITESPLINE,
                           of.BoundaryType.BOUNDARY_MIRROR)
    m = rng.standard_normal(coarse + (3, 3))
    np.testing.assert_allclose(N(up.forwardMatrixField(D(m))), oracle.prolongate(m, (3, 4, 5), fine, (6, 8, 10)),
                               rtol=RT, atol=AT)
    v = rng.uniform(size=(13, 14, 15))
    np.testing.assert_allclose(N(flow_utils.apply_gaussian_blur3d(D(v), 1.0)), oracle.blur(v, 1.0), rtol=RT, atol=AT)
    u = rng.standard_normal((13, 14, 15, 3))
    assert np.array_equal(N(flow_utils.apply_median_filter(D(u), 3)), oracle.median_filter(u, 3))


def test_mixed_dtypes_raise(cuda, of):
    w = of.Warping3D(mesh(of), of.InterpolationType.INTERPOLATE_LINEAR, of.BoundaryType.BOUNDARY_MIRROR)
    with pytest.raises(RuntimeError, match="dtype"):
        w.forward(D(np.zeros(SH)), torch.zeros(SH + (3,), device="cuda"))


def test_plain_solver_in_fp64_matches_the_fp64_oracle(cuda, oracle):
    """The reference's per-operator solver run in double on the GPU: the fast FP64 oracle."""
    from singleventriclesegmentation_b200 import synthetic
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
    I0, I1, _ = synthetic.frame_pair((16, 18, 20), seed=3)
    # weight_tv exactly representable in float32 (the oracle's parameter block holds floats)
    P = oracle.SolverParams(max_warps=2, max_outer_iterations=10, weight_tv=0.03125)
    s = TVL13DOpticalFlow(P.num_scales, P.max_warps, P.max_outer_iterations, P.weight_matching, P.weight_tv,
                          P.primaldual_algorithm_type, P.primaldual_algorithm_params, P.use_anisotropic_diff,
                          P.anisotropic_diff_params, P.use_gaussian_blur, P.gaussian_blur_sigma, P.interpolation_type,
                          P.boundary_type, P.length_type, P.length, torch.device("cuda"))
    u0 = torch.zeros((16, 18, 20, 3), dtype=torch.float64, device="cuda")
    p0 = torch.zeros((16, 18, 20, 3, 3), dtype=torch.float64, device="cuda")
    u, _ = s.compute_unfused(D(I0), D(I1), u0, p0)
    assert u.dtype == torch.float64
    ref = oracle.tvl1_compute(I0.astype(np.float64), I1.astype(np.float64), P, dtype=np.float64)[0]
    e = np.sqrt(((N(u) - ref) ** 2).sum(-1))
    # measured: mean 4e-8, max 6e-7 (five orders of magnitude below the FP32 spread); the voxels
    # where the anisotropic tensor vanishes amplify rounding differences
    assert e.mean() < 1e-6 and e.max() < 1e-5, (e.mean(), e.max())
