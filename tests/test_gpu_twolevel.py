"""Two-level preconditioner (-precond 2level) against the oracle.

The reference pairs it with the symmetrically preconditioned Hessian
(PRECONDMATVECSYM, src/RegOpt.cpp:602-606): the Krylov operator becomes
hd x + P^1/2 b~[P^1/2 x] (CLAIRE::PrecondHessMatVecSym), the right-hand side
P^1/2 g, and the preconditioner solves the same operator on a grid
ceil(n / gridscale) per axis from restricted velocity and state levels
(src/Preconditioner.cpp:323-1176).  Checked here: the operator, one
preconditioner application with its coarse Krylov solve, whole
registrations, and the combinations the library refuses.
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


def opt2(cb, n, nt, norm, beta, *extra):
    return cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-precond", "2level",
                      *extra])


def problem(n, nt):
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    x1, x2, x3 = R.grid_coords((n, n, n))
    w = (0.2 + 0.8 * np.cos(0.5 * x1) ** 2 * np.sin(0.5 * x3 + 0.3) ** 2).astype(np.float32)
    return mR.astype(np.float32), mT.astype(np.float32), vs.astype(np.float32), w


@pytest.mark.parametrize("flag,beta,projection,masked", [
    ("h1s", 1e-2, None, False),
    ("h2", 1e-3, None, False),
    ("h1s-stokes", 1e-2, "stokes", False),
    ("h1s", 1e-2, None, True),
])
def test_symmetric_hessian_matches_oracle(cb, flag, beta, projection, masked):
    n, nt = 32, 4
    mR, mT, vs, w = problem(n, nt)
    rng = np.random.default_rng(11)
    v = (0.3 * vs + 0.02 * rng.standard_normal(vs.shape)).astype(np.float32)
    vt = (0.1 * rng.standard_normal(vs.shape)).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization(flag.split("-")[0], beta), projection=projection,
                     mask=w if masked else None)
    prob.gradient(v.astype(np.float64))
    H = prob.hessian_sym(vt.astype(np.float64))
    with cb.CLAIREInterface(opt2(cb, n, nt, flag, beta)) as ci:
        ci.set_images(mR, mT)
        if masked:
            ci.SetMask(w)
        Hg = ci.HessianMatVec(v, vt)
    assert rel(Hg, H) < 1e-4


@pytest.mark.parametrize("masked", [False, True])
def test_two_level_application_matches_oracle(cb, masked):
    # coarse tolerance pctolscale * krylovtol outside a solve: 0.1 * 1e-2
    n, nt, beta = 32, 4, 1e-2
    mR, mT, vs, w = problem(n, nt)
    rng = np.random.default_rng(12)
    v = (0.4 * vs).astype(np.float32)
    r = rng.standard_normal(vs.shape).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", beta), mask=w if masked else None)
    prob.gradient(v.astype(np.float64))
    coarse = R.two_level_setup(prob, 2.0)
    z = R.two_level_apply(coarse, r.astype(np.float64), 1e-3)
    with cb.CLAIREInterface(opt2(cb, n, nt, "h1s", beta, "-krylovtol", "1e-2")) as ci:
        ci.set_images(mR, mT)
        if masked:
            ci.SetMask(w)
        ci.EvaluateGradient(v)
        pc0 = ci.stats()["pc_matvecs"]
        zg = ci.ApplyInvRegularizationOperator(r)
        its = ci.stats()["pc_matvecs"] - pc0
    facts = dict(rel=rel(zg, z), its=its, oracle_its=coarse.inner_iters)
    assert abs(its - coarse.inner_iters) <= 1, facts
    assert facts["rel"] < 2e-3, facts
    # outside the coarse band the preconditioner is the identity
    hi = np.stack([R.rect_freq_filter(r[k].astype(np.float64), 0.5, lowpass=False) for k in range(3)])
    assert rel(np.stack([R.rect_freq_filter(zg[k].astype(np.float64), 0.5, lowpass=False) for k in range(3)]),
               hi) < 1e-5


# H2 is left out: its Hessian symbol carries no hd (src/RegularizationH2.cpp:239)
# while the symmetric operator's identity term does, so the pairing is badly
# scaled there and the oracle's own solve stalls in the line search.
@pytest.mark.parametrize("flag,beta,projection", [("h1s", 1e-2, None), ("h1s", 1e-3, None),
                                                  ("h1s-stokes", 1e-2, "stokes")])
def test_two_level_registration_matches_oracle(cb, flag, beta, projection):
    n, nt, maxit, tol = 32, 4, 10, 1e-2
    mR, mT, vs, _ = problem(n, nt)
    reg = R.Regularization(flag.split("-")[0], beta)
    prob = R.Problem(mR, mT, nt, reg, projection=projection)
    res = R.gauss_newton(prob, R.GNOptions(maxit=maxit, gttol=tol, precond="2level"))
    mis = R.relative_mismatch(prob.mR, res["m1"], prob.mT)
    extra = ["-maxit", str(maxit), "-opttol", str(tol)]
    with cb.CLAIREInterface(opt2(cb, n, nt, flag, beta, *extra)) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        vg = ci.GetSolution()
    with cb.CLAIREInterface(cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", flag, "-beta", str(beta),
                                       *extra])) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st_inv = ci.stats()
    facts = dict(gn=st["gn_iterations"], gn_oracle=res["iters"], pcg=st["pcg_iterations"],
                 pcg_oracle=sum(res["pcg_iters"]), pc=st["pc_matvecs"], v=rel(vg, res["v"]),
                 mis=st["rel_mismatch"], mis_oracle=mis, mis_invreg=st_inv["rel_mismatch"],
                 gn_invreg=st_inv["gn_iterations"], pcg_invreg=st_inv["pcg_iterations"])
    assert abs(facts["gn"] - facts["gn_oracle"]) <= 1, facts
    assert abs(facts["pcg"] - facts["pcg_oracle"]) <= 2, facts
    assert facts["pc"] > 0, facts
    assert facts["v"] < 1e-2, facts
    assert abs(facts["mis"] - mis) <= 5e-3 * mis, facts
    assert st["converged_reason"] == 1, facts
    # near the INVREG solve's result (both stop at ||g|| < 1e-2 ||g0||, at
    # different iterates)
    assert abs(facts["mis"] - facts["mis_invreg"]) <= 0.2 * facts["mis_invreg"], facts


def test_two_level_refusals(cb):
    n, nt = 32, 4
    for extra in (["-bf16images"], ["-distance", "ncc"], ["-nx", "32x32x64"], ["-gridscale", "3"]):
        with pytest.raises(cb.ClaireError) as e:
            cb.CLAIREInterface(opt2(cb, n, nt, "h1s", 1e-2, *extra))
        assert e.value.code == -6, extra
    mR, mT, _, _ = problem(n, nt)
    with cb.CLAIREInterface(opt2(cb, n, nt, "h1s", 1e-2, "-gridcont")) as ci:
        ci.set_images(mR, mT)
        with pytest.raises(cb.ClaireError) as e:
            ci.Run()
        assert e.value.code == -6
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        with pytest.raises(cb.ClaireError) as e:
            srv.submit(opt2(cb, n, nt, "h1s", 1e-2), mR, mT)
        assert e.value.code == -6


def test_two_level_batch_equals_single(cb):
    # each problem of a batch runs its own coarse solve (per-problem masks and
    # tolerances): a problem gives the same result alone and in a batch
    n, nt = 32, 4
    mR, mT, _, _ = problem(n, nt)
    rng = np.random.default_rng(21)
    probs = [(mR, mT)]
    for _ in range(2):
        shift = tuple(int(s) for s in rng.integers(1, n, size=3))
        probs.append((np.roll(mR, shift, axis=(0, 1, 2)).copy(), mT))
    opt = opt2(cb, n, nt, "h1s", 1e-2, "-maxit", "5", "-opttol", "1e-2")
    single = []
    for a, b in probs:
        with cb.CLAIREInterface(opt) as ci:
            ci.set_images(a, b)
            ci.Run()
            single.append((np.asarray(ci.GetSolution()), ci.stats()))
    with cb.CLAIREInterface(opt, nbatch=len(probs)) as ci:
        for k, (a, b) in enumerate(probs):
            ci.set_images(a, b, k)
        ci.Run()
        for k in range(len(probs)):
            st = ci.stats(k)
            facts = dict(k=k, gn=(st["gn_iterations"], single[k][1]["gn_iterations"]),
                         pc=(st["pc_matvecs"], single[k][1]["pc_matvecs"]))
            assert st["gn_iterations"] == single[k][1]["gn_iterations"], facts
            assert st["pcg_iterations"] == single[k][1]["pcg_iterations"], facts
            assert rel(ci.GetSolution(k), single[k][0]) < 1e-6, facts
