"""FFT variants and the autotuner (claire_b200_autotune).

Every candidate variant of every grid size (two-stage radix plan x lines per
CTA) must give the oracle's spectral operators within the FFT tolerance
(1e-5 relative L2, FP32 against FP64); the tuner must keep one of the
candidates, and a registration on a tuned size still matches the oracle.
Variants are process-wide, so each test puts the default back.
"""
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


@pytest.mark.parametrize("n", [16, 32, 48, 64, 96, 128, 192, 256])
def test_every_fft_variant_matches_oracle(cb, n):
    rng = np.random.default_rng(500 + n)
    shape = (n, n, n)
    f = rng.standard_normal(shape).astype(np.float32)
    gref = R.grad(f.astype(np.float64))
    small = n <= 96
    if small:
        v = rng.standard_normal((3,) + shape).astype(np.float32)
        dref = R.div(v.astype(np.float64))
        reg = R.Regularization("h2", 1e-3, 1e-4)
        iref = reg.apply_inverse(v.astype(np.float64))
        gr_ref = reg.gradient(v.astype(np.float64))
        op = cb.Regularization("h2", 1e-3, 1e-4)
    try:
        for var in cb.fft_variant_candidates(n):
            cb.set_fft_variant(n, var)
            assert cb.fft_variant(n) == var
            assert rel(cb.fft_grad(to_dev(f)).cpu().numpy(), gref) < TOL, var
            if small:
                dv = to_dev(v)
                assert rel(cb.fft_div(dv).cpu().numpy(), dref) < TOL, var
                assert rel(op.ApplyInverse(dv).cpu().numpy(), iref) < TOL, var
                assert rel(op.EvaluateGradient(dv).cpu().numpy(), gr_ref) < TOL, var
    finally:
        cb.set_fft_variant(n, 0)


def test_unsupported_variants_are_rejected(cb):
    with pytest.raises(cb.ClaireError):
        cb.set_fft_variant(16, 1)      # one radix plan at 16 points
    with pytest.raises(cb.ClaireError):
        cb.set_fft_variant(40, 0)      # no plan for 40 points
    assert cb.fft_variant(40) == -1


def test_autotune_keeps_a_candidate_and_registration_still_matches(cb):
    n, nt = 32, 4
    try:
        v, times = cb.autotune(64, 2)
        assert v in cb.fft_variant_candidates(64) and cb.fft_variant(64) == v
        assert set(times) == set(cb.fft_variant_candidates(64)) and min(times.values()) > 0
        assert times[v] == min(times.values())
        mR, mT, _ = R.synthetic_c1(n, np.float64, nt)
        mR = mR.astype(np.float32)
        mT = mT.astype(np.float32)
        prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
        res = R.gauss_newton(prob, R.GNOptions(maxit=10, gttol=1e-2))
        opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", "h1s", "-beta", "1e-2", "-maxit", "10",
                         "-opttol", "1e-2", "-autotune"])
        with cb.CLAIREInterface(opt) as ci:   # tunes 32-point transforms on creation
            ci.set_images(mR, mT)
            ci.Run()
            st = ci.stats()
            vg = ci.GetSolution()
        assert cb.fft_variant(n) in cb.fft_variant_candidates(n)
        assert abs(st["gn_iterations"] - res["iters"]) <= 1
        assert rel(vg, res["v"]) < 1e-4
    finally:
        cb.set_fft_variant(64, 0)
        cb.set_fft_variant(n, 0)
