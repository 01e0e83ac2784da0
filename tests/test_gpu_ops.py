"""Per-operator parity: the libsvsflow kernels (through the C ABI, via the drop-in
`opticalFlow` module) against the oracle on the same seeded inputs."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SH = (7, 9, 11)
BD = ["NEAREST", "MIRROR", "REFLECT"]
IT = ["NEAREST", "LINEAR", "CUBIC_HERMITESPLINE"]


def T(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


def N(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def of():
    from singleventriclesegmentation_b200 import opticalFlow
    return opticalFlow


def mesh(of, sh=SH, fixed=False):
    L = (1.0, 2.0, 3.0) if fixed else tuple(s - 1 for s in sh)
    return of.MeshInfo3D(*sh, *L)


@pytest.mark.parametrize("bdry", BD)
@pytest.mark.parametrize("fixed", [False, True])
def test_nabla(cuda, oracle, of, bdry, fixed):
    rng = np.random.default_rng(0)
    b = rng.standard_normal(SH).astype(np.float32)
    v = rng.standard_normal(SH + (3,)).astype(np.float32)
    m = rng.standard_normal(SH + (3, 3)).astype(np.float32)
    ms = mesh(of, fixed=fixed)
    h = (ms.gethZ(), ms.gethY(), ms.gethX())
    op = of.Nabla3D_CD(ms, getattr(of.BoundaryType, "BOUNDARY_" + bdry))
    np.testing.assert_allclose(N(op.forward(T(b))), oracle.nabla_forward(b, h, bdry), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(N(op.forwardVectorField(T(v))), oracle.nabla_forward_vf(v, h, bdry), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(N(op.backward(T(v))), oracle.nabla_backward(v, h, bdry), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(N(op.backwardVectorField(T(m))), oracle.nabla_backward_vf(m, h, bdry), rtol=1e-6, atol=1e-6)


def test_aniso(cuda, oracle, of):
    rng = np.random.default_rng(1)
    g = (rng.standard_normal(SH + (3,)) * (rng.uniform(size=SH + (1,)) > 0.2)).astype(np.float32)
    m = rng.standard_normal(SH + (3, 3)).astype(np.float32)
    an = of.AnisotropicNabla3D(mesh(of), 5.0, 0.5)
    got = an.computeTangentVecs(T(g))
    ref = oracle.aniso_tangents(g, 5.0, 0.5)
    for a, b in zip(got, ref):
        np.testing.assert_allclose(N(a), b, rtol=2e-6, atol=2e-7)
    np.testing.assert_allclose(N(an.forwardVectorField(T(m), *got)), oracle.aniso_apply(m, *ref[:3]), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(N(an.backwardVectorField(T(m), *got)), oracle.aniso_apply(m, *ref[:3]), rtol=1e-5, atol=1e-6)


def test_proxes(cuda, oracle, of):
    rng = np.random.default_rng(2)
    dv = (rng.standard_normal(SH + (3, 3)) * 0.05).astype(np.float32)
    np.testing.assert_allclose(N(of.TVL1OF3D_proxDual(T(dv), 0.5, 0.025, mesh(of))), oracle.prox_dual(dv, 0.025),
                               rtol=1e-6, atol=1e-8)
    pv = rng.standard_normal(SH + (3,)).astype(np.float32)
    rho = (rng.standard_normal(SH) * 0.1).astype(np.float32)
    gw = (rng.standard_normal(SH + (3,)) * 0.3).astype(np.float32)
    gw[0, 0, :3] = 0
    np.testing.assert_allclose(N(of.TVL1OF3D_proxPrimal(T(pv), 0.37, 1.0, T(rho), T(gw), mesh(of))),
                               oracle.prox_primal(pv, 0.37, 1.0, rho, gw), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("interp", IT)
@pytest.mark.parametrize("bdry", BD)
def test_warp(cuda, oracle, of, interp, bdry):
    rng = np.random.default_rng(3)
    b = rng.standard_normal(SH).astype(np.float32)
    v = rng.standard_normal(SH + (3,)).astype(np.float32)
    # displacements that cross the boundary by up to 3 voxels, and one far outside (the
    # reference would read out of bounds there; here the fold is clamped)
    phi = rng.uniform(-3.0, 3.0, size=SH + (3,)).astype(np.float32)
    phi[0, 0, 0] = (-40.0, 55.0, -33.0)
    w = of.Warping3D(mesh(of), getattr(of.InterpolationType, "INTERPOLATE_" + interp),
                     getattr(of.BoundaryType, "BOUNDARY_" + bdry))
    np.testing.assert_allclose(N(w.forward(T(b), T(phi))), oracle.warp(b, phi, interp=interp, bdry=bdry), rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose(N(w.forwardVectorField(T(v), T(phi))), oracle.warp(v, phi, interp=interp, bdry=bdry),
                               rtol=1e-5, atol=2e-6)
    g = rng.standard_normal(SH).astype(np.float32)
    gu, gp = w.backward(T(b), T(phi), T(g))
    ru, rp = oracle.warp_backward(b.astype(np.float64), phi.astype(np.float64), g.astype(np.float64), interp=interp, bdry=bdry)
    np.testing.assert_allclose(N(gu), ru, rtol=1e-4, atol=2e-5)
    np.testing.assert_allclose(N(gp), rp, rtol=1e-4, atol=2e-5)


@pytest.mark.parametrize("interp", IT)
def test_warp_cnn(cuda, oracle, of, interp):
    rng = np.random.default_rng(4)
    m = rng.uniform(size=(2, 3) + SH).astype(np.float32)
    phi = rng.uniform(-2, 2, size=(2,) + SH + (3,)).astype(np.float32)
    w = of.WarpingCNN3D(mesh(of), getattr(of.InterpolationType, "INTERPOLATE_" + interp), of.BoundaryType.BOUNDARY_MIRROR)
    np.testing.assert_allclose(N(w.forward(T(m), T(phi))), oracle.warp_cnn(m, phi, interp=interp), rtol=1e-5, atol=2e-6)


@pytest.mark.parametrize("interp", IT)
def test_prolongation(cuda, oracle, of, interp):
    rng = np.random.default_rng(5)
    fine, coarse = SH, (4, 5, 6)
    mf, mc = mesh(of, fine), mesh(of, coarse)
    ie = getattr(of.InterpolationType, "INTERPOLATE_" + interp)
    b = rng.standard_normal(fine).astype(np.float32)
    down = of.Prolongation3D(mf, mc, ie, of.BoundaryType.BOUNDARY_MIRROR)
    np.testing.assert_allclose(N(down.forward(T(b))),
                               oracle.prolongate(b, (6, 8, 10), coarse, (3, 4, 5), interp=interp), rtol=1e-5, atol=2e-6)
    up = of.Prolongation3D(mc, mf, ie, of.BoundaryType.BOUNDARY_MIRROR)
    v = rng.standard_normal(coarse + (3,)).astype(np.float32)
    m = rng.standard_normal(coarse + (3, 3)).astype(np.float32)
    np.testing.assert_allclose(N(up.forwardVectorField(T(v))),
                               oracle.prolongate(v, (3, 4, 5), fine, (6, 8, 10), interp=interp), rtol=1e-5, atol=2e-6)
    np.testing.assert_allclose(N(up.forwardMatrixField(T(m))),
                               oracle.prolongate(m, (3, 4, 5), fine, (6, 8, 10), interp=interp), rtol=1e-5, atol=2e-6)


def test_blur_and_median(cuda, oracle):
    from singleventriclesegmentation_b200 import flow_utils
    rng = np.random.default_rng(6)
    v = rng.uniform(size=(13, 14, 15)).astype(np.float32)
    np.testing.assert_allclose(N(flow_utils.apply_gaussian_blur3d(T(v), 1.0)), oracle.blur(v, 1.0), rtol=1e-6, atol=1e-6)
    u = rng.standard_normal((13, 14, 15, 3)).astype(np.float32)
    u[3, 3, 3] = u[3, 3, 4]
    for ks in (3, 5):
        assert np.array_equal(N(flow_utils.apply_median_filter(T(u), ks)), oracle.median_filter(u, ks))


def test_empty_and_bad_inputs(cuda, of):
    ms = mesh(of)
    op = of.Nabla3D_CD(ms, of.BoundaryType.BOUNDARY_MIRROR)
    with pytest.raises(RuntimeError, match="contiguous"):
        op.forward(torch.zeros((11, 9, 7), device="cuda").transpose(0, 2))
    with pytest.raises(RuntimeError, match="CUDA"):
        op.forward(torch.zeros(SH))
    with pytest.raises(RuntimeError, match="Expected 3d"):
        op.forward(torch.zeros(SH + (1,), device="cuda"))
    # zero-voxel prox calls are a no-op
    e = of.MeshInfo3D(0, 0, 0, 1, 1, 1)
    assert of.TVL1OF3D_proxDual(torch.zeros((0, 0, 0, 3, 3), device="cuda"), 0.5, 0.025, e).numel() == 0
