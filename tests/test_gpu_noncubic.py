"""Non-cubic grids (each axis with its own transform length): spectral
operators, transport and a registration against the oracle, which handles
any N1 x N2 x N3 grid."""
import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("shape", [(32, 48, 16), (64, 32, 128), (16, 96, 32), (32, 150, 16), (150, 32, 64)])
def test_spectral_ops_non_cubic(cb, shape):
    # 150 points (x1 or x2 only): radix 10 x 15 plans, both radix orders
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape).astype(np.float32)
    v = rng.standard_normal((3,) + shape).astype(np.float32)
    variants = cb.fft_variant_candidates(150) if 150 in shape else [None]
    try:
        for var in variants:
            if var is not None:
                cb.set_fft_variant(150, var)
            assert rel(cb.fft_grad(to_dev(f)).cpu().numpy(), R.grad(f.astype(np.float64))) < TOL, var
            assert rel(cb.fft_div(to_dev(v)).cpu().numpy(), R.div(v.astype(np.float64))) < TOL, var
            for norm in ("h1s", "h2"):
                reg = R.Regularization(norm, 1e-2, 1e-4)
                op = cb.Regularization(norm, 1e-2, 1e-4)
                assert rel(op.EvaluateGradient(to_dev(v)).cpu().numpy(), reg.gradient(v.astype(np.float64))) < TOL
                assert rel(op.ApplyInverse(to_dev(v)).cpu().numpy(), reg.apply_inverse(v.astype(np.float64))) < TOL
            b = to_dev(v)
            cb.leray(b, "stokes", (1e-2, 1e-4, 1e-4))
            ref = R.leray_projection(v.astype(np.float64), "stokes", 1e-2, 1e-4)
            assert rel(b.cpu().numpy(), ref) < TOL, var
    finally:
        cb.set_fft_variant(150, 0)


@pytest.mark.parametrize("shape", [(32, 48, 16), (48, 32, 64)])
def test_transport_non_cubic(cb, shape):
    rng = np.random.default_rng(7)
    nt = 4
    v = (0.5 * R.velocity_trig(shape, 1.0, reference_case=False)).astype(np.float32)
    ref = R.trajectory_rk2(v.astype(np.float64), nt, "state")
    disp = cb.SemiLagrangian(nt).ComputeTrajectory(to_dev(v), "state")
    assert rel(disp.cpu().numpy(), ref) < TOL
    f = rng.standard_normal(shape).astype(np.float32)
    out = cb.SemiLagrangian.Interpolate(to_dev(f), disp).cpu().numpy()
    q = R.index_grid(shape) + disp.cpu().numpy().astype(np.float64)
    assert rel(out, R.interp3(f.astype(np.float64), q)) < TOL


@pytest.mark.parametrize("shape", [(32, 48, 32), (32, 150, 32)])
def test_registration_non_cubic(cb, shape):
    nt = 4
    mT = R.rescale(R.template_sin2(shape))
    v = R.velocity_trig(shape, 0.5, reference_case=False)
    mR = R.rescale(R.forward_transport(mT, v, nt))
    mR = mR.astype(np.float32)
    mT = mT.astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
    res = R.gauss_newton(prob, R.GNOptions(maxit=10, gttol=1e-2))
    opt = cb.RegOpt(["-nx", "%dx%dx%d" % shape, "-nt", str(nt), "-regnorm", "h1s", "-beta", "1e-2", "-maxit", "10",
                     "-opttol", "1e-2"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        vg = ci.GetSolution()
    assert vg.shape == (3,) + shape
    assert abs(st["gn_iterations"] - res["iters"]) <= 1
    assert rel(vg, res["v"]) < 1e-4
