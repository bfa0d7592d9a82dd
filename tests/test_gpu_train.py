"""Regularisation-parameter search (-train reduce|binary, -jbound) against the
oracle's restatement of RunSolverRegParaContReductSearch / BinarySearch.

The reduce search's decisions have wide margins on this problem, so they must
match exactly.  The bisection steps close to the bound (min det(grad y) within
a fraction of a percent of jbound), where FP32 and FP64 may take different
branches, so its estimate must agree to the search's resolution and keep the
bound."""
import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def problem():
    n, nt = 32, 4
    shape = (n, n, n)
    mT = R.rescale(R.template_sin2(shape))
    v = R.velocity_trig(shape, 1.5, reference_case=False)
    mR = R.rescale(R.forward_transport(mT, v, nt))
    return mR.astype(np.float32), mT.astype(np.float32), n, nt


@pytest.mark.parametrize("strategy", ["reduce", "binary"])
def test_train_search_matches_oracle(cb, strategy):
    mR, mT, n, nt = problem()
    jb = 0.5
    res = R.train_search(mR, mT, nt, R.Regularization("h1s", 1e-2), R.GNOptions(maxit=5, gttol=5e-2),
                         strategy=strategy, jbound=jb)
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", "h1s", "-maxit", "5", "-opttol", "5e-2",
                     "-train", strategy, "-jbound", str(jb)])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        v = np.asarray(ci.GetSolution())
        _, (mn, _, mx) = ci.ComputeDetDefGrad()
    facts = dict(beta=st["beta"], beta_oracle=res["beta"], log=res["log"], det=(mn, mx))
    assert mn > jb and 1.0 / mx > jb, facts
    if strategy == "reduce":
        assert st["beta"] == pytest.approx(res["beta"], rel=1e-12), facts
        nv = np.linalg.norm(res["v"].ravel())
        assert np.linalg.norm((v - res["v"]).ravel()) <= 1e-3 * nv, facts
    else:
        assert abs(st["beta"] - res["beta"]) <= 0.1 * res["beta"], facts


def test_monitordefgrad_raises_beta_like_oracle(cb):
    # -monitordefgrad: beta = 1e-2 breaches min det > 0.5 on this problem; beta
    # is raised halfway toward 10 beta and the solve repeated from zero
    mR, mT, n, nt = problem()
    jb = 0.5
    res = R.monitored_run(mR, mT, nt, R.Regularization("h1s", 1e-2), R.GNOptions(maxit=5, gttol=5e-2), jbound=jb)
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", "h1s", "-beta", "1e-2", "-maxit", "5",
                     "-opttol", "5e-2", "-monitordefgrad", "-jbound", str(jb)])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        v = np.asarray(ci.GetSolution())
    facts = dict(st={k: st[k] for k in ("beta", "solution_status", "det_min", "det_max")},
                 oracle=(res["beta"], res["status"], res["det"]))
    assert st["solution_status"] == res["status"] == 1, facts
    assert st["beta"] == pytest.approx(res["beta"], rel=1e-12), facts
    assert abs(st["det_min"] - res["det"][0]) <= 1e-3 * res["det"][0], facts
    nv = np.linalg.norm(res["v"].ravel())
    assert np.linalg.norm((v - res["v"]).ravel()) <= 1e-3 * nv, facts
