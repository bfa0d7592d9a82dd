"""bf16 image storage (-bf16images): mR, mT and the state levels stored as
bfloat16, every gather, FFT and reduction computed in FP32 / FP64.

The oracle emulates the storage exactly (R.bf16_round applied to the images
and to every state level it computes), so the device run is compared with the
FP64 oracle under the same storage at FP32-level tolerances: the stored values
agree bit for bit except where the FP32 and FP64 sums fall on different sides
of a bf16 rounding boundary (a few values in 10^5).  The cost of the format
itself is reported against the FP32-image run of the same problem.
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


def opt16(cb, n, nt, norm, beta, bf16=True, **kw):
    args = ["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", str(beta)]
    if bf16:
        args.append("-bf16images")
    opt = cb.RegOpt(args)
    for k, v in kw.items():
        opt.set(k, v)
    return opt


def c1_problem(n, nt=4):
    mR, mT, vstar = R.synthetic_c1(n, np.float64, nt)
    return mR.astype(np.float32), mT.astype(np.float32), vstar.astype(np.float32)


@pytest.mark.parametrize("n", [16, 30, 32, 48, 64])
def test_interp3_bf16_is_the_fp32_gather_rounded(cb, n):
    # n = 30: N3 % 4 != 0, every tile takes the global-memory path
    import torch
    rng = np.random.default_rng(100 + n)
    shape = (n, n, n)
    f = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda().to(torch.bfloat16)
    disp = torch.from_numpy(rng.uniform(-7.5, 7.5, size=(3,) + shape).astype(np.float32)).cuda()
    out16 = cb.SemiLagrangian.InterpolateBF16(f, disp)
    out32 = cb.SemiLagrangian.Interpolate(f.float().contiguous(), disp)
    torch.cuda.synchronize()
    assert torch.equal(out16, out32.to(torch.bfloat16))
    q = R.index_grid(shape) + disp.cpu().numpy().astype(np.float64)
    ref = R.interp3(f.float().cpu().numpy().astype(np.float64), q)
    assert rel(out16.float().cpu().numpy(), ref) < 4e-3  # one bf16 rounding of the result


@pytest.mark.parametrize("norm,beta,nt", [("h1s", 1e-2, 4), ("h2", 1e-3, 8)])
def test_bf16_objective_gradient_hessian_match_oracle_with_bf16_storage(cb, norm, beta, nt):
    n = 32
    mR, mT, vstar = c1_problem(n, nt)
    rng = np.random.default_rng(5)
    v = (0.3 * vstar + 0.02 * rng.standard_normal(vstar.shape)).astype(np.float32)
    vt = (0.1 * rng.standard_normal(vstar.shape)).astype(np.float32)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), image_store=R.bf16_round)
    J = prob.objective(v.astype(np.float64))
    g = prob.gradient(v.astype(np.float64))
    H = prob.hessian_matvec(vt.astype(np.float64))
    with cb.CLAIREInterface(opt16(cb, n, nt, norm, beta)) as ci:
        ci.set_images(mR, mT)
        Jg, Dg, _ = ci.EvaluateObjective(v)
        gg = ci.EvaluateGradient(v)
        Hg = ci.HessianMatVec(v, vt)
        m1 = ci.GetFinalState()
    assert abs(Jg - J) <= 1e-4 * abs(J)
    assert rel(gg, g) < 1e-3
    assert rel(Hg, H) < 1e-3
    # the final state is bf16-valued and equals the oracle's stored level
    assert np.array_equal(R.bf16_round(m1), np.asarray(m1, np.float64))
    assert rel(m1, prob.solve_state()[nt]) < 1e-4


def test_bf16_registration_matches_oracle_and_fp32(cb):
    n, nt, norm, beta, maxit = 32, 4, "h1s", 1e-2, 10
    mR, mT, _ = c1_problem(n, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, beta), image_store=R.bf16_round)
    res = R.gauss_newton(prob, R.GNOptions(maxit=maxit, gttol=1e-2))
    with cb.CLAIREInterface(opt16(cb, n, nt, norm, beta, maxit=maxit, opttol=1e-2)) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st16 = ci.stats()
        v16 = ci.GetSolution()
    with cb.CLAIREInterface(opt16(cb, n, nt, norm, beta, bf16=False, maxit=maxit, opttol=1e-2)) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        st32 = ci.stats()
        v32 = ci.GetSolution()
    mis = R.relative_mismatch(prob.mR, res["m1"], prob.mT)
    facts = dict(gn16=st16["gn_iterations"], gn_oracle=res["iters"], gn32=st32["gn_iterations"],
                 v_vs_oracle=rel(v16, res["v"]), v_vs_fp32=rel(v16, v32), mis16=st16["rel_mismatch"],
                 mis_oracle=mis, mis32=st32["rel_mismatch"])
    assert abs(st16["gn_iterations"] - res["iters"]) <= 1, facts
    # rounding flips (FP32 and FP64 sums on either side of a bf16 boundary)
    # move a stored value by one bf16 step; ten GN iterations carry them into
    # the velocity at the 1e-3 level
    assert facts["v_vs_oracle"] < 5e-3, facts
    assert abs(facts["mis16"] - mis) <= 2e-3 * mis, facts
    # cost of the storage format on this problem
    assert abs(st16["gn_iterations"] - st32["gn_iterations"]) <= 1, facts
    assert facts["v_vs_fp32"] < 2e-2, facts
    assert abs(facts["mis16"] - facts["mis32"]) <= 2e-2 * facts["mis32"], facts


def test_bf16_context_halves_image_bytes_and_serves(cb):
    n, nt = 32, 4
    o32 = opt16(cb, n, nt, "h1s", 1e-2, bf16=False, maxit=3, opttol=1e-2)
    o16 = opt16(cb, n, nt, "h1s", 1e-2, maxit=3, opttol=1e-2)
    assert o32.estimate_bytes(1) - o16.estimate_bytes(1) == (nt + 3) * n ** 3 * 2
    mR, mT, _ = c1_problem(n, nt)
    with cb.CLAIREInterface(o16) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        v_plain = np.asarray(ci.GetSolution())
    with cb.Server(slots_per_pool=2, idle_ms=100) as srv:
        rid = srv.submit(o16, mR, mT)
        assert srv.wait(rid, 120000) == cb.REQ_DONE
        v_srv, _, _ = srv.result(rid, (n, n, n))
    assert np.array_equal(v_srv, v_plain)
