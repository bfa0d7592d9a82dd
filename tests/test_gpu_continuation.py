"""Grid and scale continuation (-gridcont, -scalecont), the spectral grid
change they use, and the initialisation of a warm-started solve, against the
oracle's restatements of RunSolverGridCont / RunSolverScaleCont /
Preprocessing::Restrict / Prolong / InitializeOptimization.
"""
import numpy as np
import pytest

from oracle import claire_ref as R

pytestmark = pytest.mark.gpu

FFT_SIZES = (16, 32, 48, 64, 96, 128, 192, 256)


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


@pytest.mark.parametrize("ns,nt,nf", [(32, 16, 1), (16, 32, 3), (64, 32, 3), (48, 24, 1), (24, 48, 1), (32, 64, 2)])
def test_grid_change_matches_oracle(cb, ns, nt, nf):
    rng = np.random.default_rng(ns * 7 + nt)
    f = rng.standard_normal((nf, ns, ns, ns)).astype(np.float32)
    out = cb.grid_change(to_dev(f), nt).cpu().numpy()
    ref = np.stack([R.grid_transfer(f[k].astype(np.float64), nt) for k in range(nf)])
    assert out.shape == (nf, nt, nt, nt)
    assert rel(out, ref) < 1e-5


def c1(n, nt):
    mR, mT, _ = R.synthetic_c1(n, np.float64, nt)
    return mR.astype(np.float32), mT.astype(np.float32)


def test_warm_start_initialises_at_zero_velocity(cb):
    n, nt = 32, 4
    mR, mT = c1(n, nt)
    _, _, vs = R.synthetic_c1(n, np.float64, nt)
    v0 = (0.2 * vs).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
    res = R.gauss_newton(prob, R.GNOptions(maxit=2, gttol=1e-2), v0=v0)
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", "h1s", "-beta", "1e-2", "-maxit", "2",
                     "-opttol", "1e-2"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.SetInitialGuess(v0)
        ci.Run()
        st = ci.stats()
        v = ci.GetSolution()
    assert abs(st["gnorm0"] - res["g0"]) <= 1e-5 * res["g0"]
    assert rel(v, res["v"]) < 1e-4


def test_grid_continuation_matches_oracle(cb):
    n, nt, norm, beta = 32, 4, "h1s", 1e-2
    mR, mT = c1(n, nt)
    res = R.grid_continuation(mR, mT, nt, R.Regularization(norm, beta), R.GNOptions(maxit=10, gttol=1e-2),
                              supported=lambda k: k in FFT_SIZES)
    assert [lv[0] for lv in res["levels"]] == [16, 32]
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-maxit", "10",
                     "-opttol", "1e-2", "-gridcont"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        v = ci.GetSolution()
    facts = dict(gn=st["gn_iterations"], oracle=res["levels"], v=rel(v, res["v"]))
    assert abs(st["gn_iterations"] - res["iters"]) <= 1, facts
    assert facts["v"] < 1e-3, facts
    mis = R.relative_mismatch(res["prob"].mR, res["m1"], res["prob"].mT)
    assert abs(st["rel_mismatch"] - mis) <= 1e-3 * mis, facts


def test_scale_continuation_matches_oracle(cb):
    n, nt, norm, beta = 32, 4, "h1s", 1e-2
    mR, mT = c1(n, nt)
    res = R.scale_continuation(mR, mT, nt, R.Regularization(norm, beta), R.GNOptions(maxit=10, gttol=1e-2))
    assert [lv[0] for lv in res["levels"]] == [8.0, 4.0, 2.0, 1.0]
    opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta), "-maxit", "10",
                     "-opttol", "1e-2", "-scalecont"])
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st = ci.stats()
        v = ci.GetSolution()
    facts = dict(gn=st["gn_iterations"], oracle=res["levels"], v=rel(v, res["v"]))
    assert abs(st["gn_iterations"] - res["iters"]) <= 1, facts
    assert facts["v"] < 1e-3, facts


def test_server_rejects_continuation_requests(cb):
    mR, mT = c1(32, 4)
    with cb.Server(slots_per_pool=1, idle_ms=50) as srv:
        for flag in ("-gridcont", "-scalecont"):
            opt = cb.RegOpt(["-nx", "32", "-nt", "4", flag])
            with pytest.raises(cb.ClaireError):
                srv.submit(opt, mR, mT)
