"""NCC distance (-distance ncc, DistanceMeasureNCC) against the oracle.

The NCC distance s (1/2 - 1/2 I^2/(A R)) is a small difference of numbers
near 1/2, and its adjoint final condition c1 mR - c2 m1 a difference of nearly
equal fields, so FP32 device results agree with the FP64 oracle to 1e-4
relative (instead of the 1e-5 of the L2 distance).
"""
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


def opt_ncc(cb, n, nt, norm, beta, extra=()):
    return cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-distance", "ncc"]
                     + list(extra))


def c1_problem(n, nt=4):
    mR, mT, vstar = R.synthetic_c1(n, np.float64, nt)
    return mR.astype(np.float32), mT.astype(np.float32), vstar.astype(np.float32)


@pytest.mark.parametrize("norm,beta,nt", [("h1s", 1e-2, 4), ("h2s", 1e-3, 8)])
def test_ncc_objective_gradient_hessian(cb, norm, beta, nt):
    n = 32
    mR, mT, vstar = c1_problem(n, nt)
    rng = np.random.default_rng(21)
    v = (0.3 * vstar + 0.02 * rng.standard_normal(vstar.shape)).astype(np.float32)
    vt = (0.1 * rng.standard_normal(vstar.shape)).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), distance="ncc")
    J = prob.objective(v.astype(np.float64))
    g = prob.gradient(v.astype(np.float64))
    H = prob.hessian_matvec(vt.astype(np.float64))
    with cb.CLAIREInterface(opt_ncc(cb, n, nt, norm, beta)) as ci:
        ci.set_images(mR, mT)
        J0g, _, _ = ci.EvaluateObjective(np.zeros_like(v))
        Jg, Dg, _ = ci.EvaluateObjective(v)
        gg = ci.EvaluateGradient(v)
        Hg = ci.HessianMatVec(v, vt)
    # the scale makes the NCC distance of m1 = mT equal to the L2 one
    d_l2 = R.Problem(mR, mT, nt, R.Regularization(norm, beta)).objective(np.zeros(v.shape))
    assert abs(J0g - d_l2) <= 1e-5 * d_l2
    assert abs(Dg - prob.last_D) <= 1e-4 * abs(prob.last_D)
    assert abs(Jg - J) <= 1e-4 * abs(J)
    assert rel(gg, g) < 1e-4
    assert rel(Hg, H) < 1e-4


def test_ncc_registration_matches_oracle(cb):
    n, nt, norm, beta, maxit = 32, 4, "h1s", 1e-2, 10
    mR, mT, _ = c1_problem(n, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), distance="ncc")
    res = R.gauss_newton(prob, R.GNOptions(maxit=maxit, gttol=1e-2))
    opt = opt_ncc(cb, n, nt, norm, beta, ["-maxit", str(maxit), "-opttol", "1e-2"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        vg = ci.GetSolution()
    facts = dict(gn=st["gn_iterations"], gn_oracle=res["iters"], v=rel(vg, res["v"]),
                 mis=st["rel_mismatch"], mis_oracle=R.relative_mismatch(prob.mR, res["m1"], prob.mT))
    assert abs(st["gn_iterations"] - res["iters"]) <= 1, facts
    assert facts["v"] < 1e-3, facts
    assert abs(facts["mis"] - facts["mis_oracle"]) <= 1e-3 * facts["mis_oracle"], facts


def test_ncc_batch_and_server_equal_single(cb):
    # each problem keeps its own scale: a batch of different image pairs and a
    # served request give the single-problem results
    n, nt = 32, 4
    probs = [c1_problem(n, nt)]
    rng = np.random.Generator(np.random.PCG64(R.problem_seed(3, 7)))
    mT2 = R.template_ellipsoids((n, n, n), rng)
    v2 = R.velocity_random((n, n, n), rng)
    probs.append((R.forward_transport(mT2, v2, nt).astype(np.float32), mT2.astype(np.float32), None))
    opt = opt_ncc(cb, n, nt, "h1s", 1e-2, ["-maxit", "3", "-opttol", "1e-2"])
    single = []
    for mR, mT, _ in probs:
        with cb.CLAIREInterface(opt) as ci:
            ci.set_images(mR, mT)
            ci.Run()
            single.append(np.asarray(ci.GetSolution()))
    with cb.CLAIREInterface(opt, nbatch=2) as ci:
        for b, (mR, mT, _) in enumerate(probs):
            ci.set_images(mR, mT, b)
        ci.Run()
        for b in range(2):
            assert np.array_equal(ci.GetSolution(b), single[b])
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        ids = [srv.submit(opt, mR, mT) for mR, mT, _ in probs]
        for rid, ref in zip(ids, single):
            assert srv.wait(rid, 120000) == cb.REQ_DONE
            v, _, _ = srv.result(rid, (n, n, n))
            assert np.array_equal(v, ref)


def test_ncc_with_bf16_images_is_rejected(cb):
    with pytest.raises(cb.ClaireError):
        cb.CLAIREInterface(opt_ncc(cb, 32, 4, "h1s", 1e-2, ["-bf16images"]))
