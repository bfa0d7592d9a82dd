"""Distance-measure masks (SetMask) for SL2 and NCC against the oracle:
objective, gradient and GN Hessian matvec with weights, a registration with a
mask, and removal of the mask."""
import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def setup(n, nt):
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    x1, x2, x3 = R.grid_coords((n, n, n))
    w = (0.2 + 0.8 * np.cos(0.5 * x1) ** 2 * np.sin(0.5 * x3 + 0.3) ** 2).astype(np.float32)
    return mR.astype(np.float32), mT.astype(np.float32), vs.astype(np.float32), w


@pytest.mark.parametrize("distance,tol", [("sl2", 1e-5), ("ncc", 1e-4)])
def test_masked_objective_gradient_hessian(cb, distance, tol):
    n, nt, norm, beta = 32, 4, "h1s", 1e-2
    mR, mT, vs, w = setup(n, nt)
    rng = np.random.default_rng(4)
    v = (0.3 * vs + 0.02 * rng.standard_normal(vs.shape)).astype(np.float32)
    vt = (0.1 * rng.standard_normal(vs.shape)).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), distance=distance, mask=w)
    J = prob.objective(v.astype(np.float64))
    g = prob.gradient(v.astype(np.float64))
    H = prob.hessian_matvec(vt.astype(np.float64))
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-distance", distance])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.SetMask(w)
        Jg, _, _ = ci.EvaluateObjective(v)
        gg = ci.EvaluateGradient(v)
        Hg = ci.HessianMatVec(v, vt)
        ci.SetMask(None)   # back to the unweighted distance
        J1, _, _ = ci.EvaluateObjective(v)
    assert abs(Jg - J) <= tol * abs(J)
    assert rel(gg, g) < tol
    assert rel(Hg, H) < tol
    J_plain = R.Problem(mR, mT, nt, R.Regularization(norm, beta), distance=distance).objective(v.astype(np.float64))
    assert abs(J1 - J_plain) <= tol * abs(J_plain)


def test_masked_registration_matches_oracle(cb):
    n, nt, norm, beta = 32, 4, "h1s", 1e-2
    mR, mT, _, w = setup(n, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), mask=w)
    res = R.gauss_newton(prob, R.GNOptions(maxit=10, gttol=1e-2))
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-maxit", "10",
                     "-opttol", "1e-2"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.SetMask(w)
        ci.Run()
        st = ci.stats()
        v = ci.GetSolution()
    assert abs(st["gn_iterations"] - res["iters"]) <= 1
    assert rel(v, res["v"]) < 1e-4
