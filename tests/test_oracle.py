"""Pin the oracle to the reference's own known-answer checks (CPU only).

The reference ships no golden vectors; what it does check:
tricubic Lagrange reproduction of cubics / node values, spectral operators
exact on trig polynomials, the forward/backward transport round trip of
apps/benchmark.cpp:297-380, the Taylor gradient test and the Hessian
symmetry test of src/OptimizationProblem.cpp:157-496.
"""
import math

import numpy as np
import pytest

from oracle import claire_ref as R


def test_lagrange_weights_partition_of_unity_and_nodes():
    t = np.linspace(1.0, 2.0, 101)[:-1]
    w = R.lagrange_weights(t)
    assert np.allclose(sum(w), 1.0, atol=1e-14)
    w1 = R.lagrange_weights(np.array([1.0]))
    assert [float(x[0]) for x in w1] == [0.0, 1.0, 0.0, 0.0]


def test_tricubic_reproduces_cubics():
    n = 16
    shape = (n, n, n)
    rng = np.random.default_rng(0)
    q = rng.uniform(2, n - 3, size=(3, 2000))
    f = lambda a, b, c: 1 + 0.3 * a - 0.2 * b ** 2 + 0.01 * a * b * c + 0.001 * c ** 3 - 0.002 * a ** 2 * b
    idx = R.index_grid(shape)
    val = R.interp3(f(idx[0], idx[1], idx[2]), q)
    assert np.max(np.abs(val - f(q[0], q[1], q[2]))) < 1e-11


def test_tricubic_periodic_wrap_and_nodes():
    n = 12
    rng = np.random.default_rng(1)
    F = rng.standard_normal((n, n, n))
    idx = R.index_grid((n, n, n))
    shift = rng.integers(-30, 30, size=(3, 1, 1, 1))
    out = R.interp3(F, idx + shift)
    ii = [(idx[d] + shift[d]).astype(int) % n for d in range(3)]
    assert np.array_equal(out, F[ii[0], ii[1], ii[2]])


def test_spectral_gradient_divergence_on_trig_polynomials():
    n = 32
    shape = (n, n, n)
    x1, x2, x3 = R.grid_coords(shape)
    m = np.sin(2 * x1) * np.cos(3 * x2) + np.sin(5 * x3)
    g = R.grad(m)
    assert np.max(np.abs(g[0] - 2 * np.cos(2 * x1) * np.cos(3 * x2))) < 1e-12
    assert np.max(np.abs(g[1] + 3 * np.sin(2 * x1) * np.sin(3 * x2))) < 1e-12
    assert np.max(np.abs(g[2] - 5 * np.cos(5 * x3))) < 1e-12
    v = np.stack([np.sin(x1), np.cos(2 * x2), np.sin(3 * x3)])
    d = R.div(v)
    assert np.max(np.abs(d - (np.cos(x1) - 2 * np.sin(2 * x2) + 3 * np.cos(3 * x3)))) < 1e-12


def test_nyquist_mode_has_zero_derivative():
    n = 16
    x1, _, _ = R.grid_coords((n, n, n))
    m = np.cos(n / 2 * x1)   # pure Nyquist mode along x1
    assert np.max(np.abs(R.grad(m))) < 1e-12


@pytest.mark.parametrize("norm", ["h1s", "h1", "h2", "h2s", "h3", "h3s"])
def test_regularization_symbols_on_a_single_mode(norm):
    n = 16
    shape = (n, n, n)
    x1, x2, x3 = R.grid_coords(shape)
    k = (1, 2, 3)
    kap = float(sum(kk * kk for kk in k))
    mode = np.cos(k[0] * x1 + k[1] * x2 + k[2] * x3)
    v = np.stack([mode, 0.5 * mode, -mode])
    reg = R.Regularization(norm, 1e-2, 1e-4)
    hd = R.lebesgue_measure(shape)
    b0, b1 = 1e-2, 1e-4
    expect = {"h1s": hd * b0 * kap, "h1": hd * b0 * (kap + b1), "h2": b0 * (kap ** 2 + b1),
              "h2s": hd * b0 * kap ** 2, "h3": b0 * (kap ** 3 + b1), "h3s": b0 * kap ** 3}[norm]
    assert np.allclose(reg.gradient(v), expect * v, rtol=1e-12, atol=1e-12 * expect)
    inv = {"h1s": b0 * kap, "h1": b0 * (kap + b1), "h2": b0 * (kap ** 2 + b1), "h2s": b0 * kap ** 2,
           "h3": b0 * (kap ** 3 + b1), "h3s": b0 * kap ** 3}[norm]
    # h1 / h2 amplify the roundoff mean of the mode by 1/(beta0*beta1) at k = 0
    assert np.allclose(reg.apply_inverse(v), v / inv, rtol=1e-12, atol=1e-9)


def test_h2_functional_matches_its_symbol():
    # src/RegularizationH2.cpp:118-164: R = 1/2 hd ||sqrt(b0)(-kappa + sqrt(b1)) v||^2
    n = 16
    shape = (n, n, n)
    x1, x2, x3 = R.grid_coords(shape)
    mode = np.cos(x1 + 2 * x2)
    v = np.stack([mode, mode, mode])
    reg = R.Regularization("h2", 1e-3, 1e-4)
    kap = 5.0
    sym = math.sqrt(1e-3) * (-kap + math.sqrt(1e-4))
    expect = 0.5 * R.lebesgue_measure(shape) * sym ** 2 * 3 * np.sum(mode ** 2)
    assert abs(reg.functional(v) - expect) < 1e-12 * abs(expect)


def test_leray_projection_is_divergence_free():
    n = 16
    rng = np.random.default_rng(2)
    b = rng.standard_normal((3, n, n, n))
    p = R.leray_projection(b, "stokes")
    # away from the Nyquist planes (where the two wavenumber conventions differ)
    k = R.spectral_k((n, n, n))
    dh = sum(1j * k[d] * np.fft.rfftn(p[d]) for d in range(3))
    keep = np.ones(dh.shape, bool)
    keep[n // 2, :, :] = False
    keep[:, n // 2, :] = False
    keep[:, :, n // 2] = False
    assert np.max(np.abs(dh[keep])) < 1e-9 * np.max(np.abs(np.fft.rfftn(b[0])))


def test_forward_backward_round_trip_converges():
    # apps/benchmark.cpp:297-380: transport m0 with v, then with -v
    errs = []
    for n in (16, 32):
        mT = R.template_sin2((n, n, n))
        v = R.velocity_trig((n, n, n), 0.5, reference_case=True)
        m1 = R.forward_transport(mT, v, 4)
        m0 = R.forward_transport(m1, -v, 4)
        errs.append(np.linalg.norm(m0 - mT) / np.linalg.norm(mT))
    assert errs[0] < 2e-2 and errs[1] < 2e-3 and errs[1] < errs[0] / 4


@pytest.mark.parametrize("norm", ["h1s", "h2s"])
def test_taylor_gradient(norm):
    # src/OptimizationProblem.cpp:157-243; the SL gradient is the discretised
    # continuous adjoint, so FD and g.w agree to discretisation accuracy.
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization(norm, 1e-2))
    v = 0.3 * vs
    J0 = prob.objective(v)
    gw = R.dot(prob.gradient(v), vs)
    for h in (1e-3, 1e-4):
        fd = (prob.objective(v + h * vs) - J0) / h
        assert abs(fd - gw) < 1e-2 * abs(gw)


def test_hessian_symmetry():
    # src/OptimizationProblem.cpp:439-496
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
    v = 0.3 * vs
    prob.objective(v)
    prob.gradient(v)
    w1 = vs
    w2 = np.roll(vs, 3, axis=1)
    a = prob.hessian_matvec(w1)
    b = prob.hessian_matvec(w2)
    assert abs(R.dot(a, w2) - R.dot(w1, b)) <= 1e-10 * np.linalg.norm(a) * np.linalg.norm(w2)


def test_pcg_on_spd_diagonal_system():
    rng = np.random.default_rng(3)
    d = rng.uniform(1.0, 100.0, size=(3, 4, 4, 4))
    b = rng.standard_normal((3, 4, 4, 4))
    x, it, reason = R.pcg(lambda p: d * p, lambda r: r / d, b, rtol=1e-10, maxit=50)
    assert reason == "converged" and it == 1
    x, it, reason = R.pcg(lambda p: d * p, lambda r: r, b, rtol=1e-10, maxit=200)
    assert reason == "converged" and np.allclose(d * x, b, atol=1e-8)


def test_forcing_sequence():
    # src/KrylovInterface.cpp:134-165
    assert R.forcing_tolerance(1.0, 1.0) == 0.5
    assert R.forcing_tolerance(0.01, 1.0) == pytest.approx(0.1)
    assert R.forcing_tolerance(0.01, 1.0, "qdfs") == pytest.approx(0.01)


def test_rescale_only_shifts_negative_minimum():
    # src/CLAIREUtils.cpp:691-725
    x = np.array([0.1, 0.5, 0.9])
    assert np.allclose(R.rescale(x), x / 0.8)        # no shift for min >= -1e-6
    y = np.array([-1.0, 0.0, 1.0])
    assert np.allclose(R.rescale(y), [0.0, 0.5, 1.0])


def test_gauss_newton_reduces_gradient_on_reference_problem():
    # CLAIRE's own -synthetic 0 problem, h1s beta 1e-2, nt 4 (small grid)
    n, nt = 16, 4
    mR, mT, _ = R.synthetic_reference(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
    res = R.gauss_newton(prob, R.GNOptions(maxit=10, gttol=1e-2))
    assert res["reason"] == "gttol"
    assert R.relative_mismatch(mR, res["m1"], mT) < 0.5


def test_det_def_grad_known_answers():
    # divergence-free and constant velocities preserve volume: det(grad y) = 1
    n = 16
    v = R.velocity_trig((n, n, n), 0.5)
    jac, (mn, me, mx) = R.det_def_grad(v, 4)
    assert abs(mn - 1) < 1e-12 and abs(mx - 1) < 1e-12 and abs(me - 1) < 1e-12
    vc = np.zeros((3, n, n, n))
    vc[1] += 0.4
    assert np.allclose(R.det_def_grad(vc, 4)[0], 1.0, atol=1e-14)
    # a compressible field changes volume; the inverse map's determinant
    # (a = -1) is its reciprocal to first order
    rng = np.random.Generator(np.random.PCG64(5))
    vr = R.velocity_random((n, n, n), rng, rms=0.1)
    jf, _ = R.det_def_grad(vr, 8)
    ji, _ = R.det_def_grad(vr, 8, inverse=True)
    assert np.abs(jf - 1).max() > 1e-3
    assert np.abs(jf * ji - 1).max() < 0.1 * np.abs(jf - 1).max()


def test_bf16_round_known_answers():
    # round to nearest, ties to even, on the float32 bit pattern
    x = np.array([1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -7, 1 - 2 ** -10, -2.5, 0.0, 3.0e38], np.float32)
    want = np.array([1.0, 1 + 2 ** -6, 1 + 2 ** -7, 1.0, -2.5, 0.0, 2.9996e38], np.float64)
    got = R.bf16_round(x)
    assert np.array_equal(got[:6], want[:6])
    assert abs(got[6] / 3.0e38 - 1) < 2 ** -8
    y = np.random.default_rng(0).standard_normal(1000)
    assert np.max(np.abs(R.bf16_round(y) / y - 1)) <= 2 ** -8


def test_ncc_scale_matches_sl2_at_zero_velocity():
    # src/DistanceMeasureNCC.cpp:78-166: the scale makes D_ncc(m1 = mT) = D_sl2(m1 = mT)
    n, nt = 16, 4
    mR, mT, _ = R.synthetic_c1(n, np.float64, nt)
    reg = R.Regularization("h1s", 1e-2)
    z = np.zeros((3, n, n, n))
    d_ncc = R.Problem(mR, mT, nt, reg, distance="ncc").objective(z)
    d_sl2 = R.Problem(mR, mT, nt, reg).objective(z)
    assert abs(d_ncc - d_sl2) <= 1e-12 * d_sl2


def test_ncc_final_conditions_are_derivatives_of_the_distance():
    # lambda(1) = -(1/hd) dD/dm1 and lambda~(1) = d lambda(1)/dm1 [m~]
    # (src/DistanceMeasureNCC.cpp:251-510), checked by central differences in m1
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2), distance="ncc")
    prob.set_velocity(0.3 * vs)
    m = prob.solve_state()
    m1 = m[nt].copy()
    rng = np.random.default_rng(9)
    w = rng.standard_normal(m1.shape)
    lam = prob.final_condition()
    lt = prob.inc_final_condition(w)

    def with_m1(x):
        prob.m = m.copy()
        prob.m[nt] = x
        return prob.distance(), prob.final_condition()

    h = 1e-5
    (dp, lp), (dm, lm) = with_m1(m1 + h * w), with_m1(m1 - h * w)
    fd = (dp - dm) / (2 * h)
    assert abs(fd + prob.hd * R.dot(lam, w)) <= 1e-6 * abs(fd)
    assert np.linalg.norm(((lp - lm) / (2 * h) - lt).ravel()) <= 1e-6 * np.linalg.norm(lt.ravel())


def test_ncc_taylor_gradient_and_hessian_symmetry():
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2), distance="ncc")
    v = 0.3 * vs
    J0 = prob.objective(v)
    gw = R.dot(prob.gradient(v), vs)
    for h in (1e-3, 1e-4):
        fd = (prob.objective(v + h * vs) - J0) / h
        assert abs(fd - gw) < 1e-2 * abs(gw)
    prob.objective(v)
    prob.gradient(v)
    w2 = np.roll(vs, 3, axis=1)
    a = prob.hessian_matvec(vs)
    b = prob.hessian_matvec(w2)
    assert abs(R.dot(a, w2) - R.dot(vs, b)) <= 1e-10 * np.linalg.norm(a) * np.linalg.norm(w2)


def test_grid_transfer_known_answers():
    # band-limited fields are carried exactly; restriction after prolongation
    # is the identity; modes at or above the coarse Nyquist index are dropped
    n = 16
    x1, x2, x3 = R.grid_coords((n, n, n))
    f = np.sin(2 * x1) * np.cos(3 * x2) + 0.5 * np.cos(x3) + 0.25
    fine = R.grid_transfer(f, 32)
    y1, y2, y3 = R.grid_coords((32, 32, 32))
    assert np.max(np.abs(fine - (np.sin(2 * y1) * np.cos(3 * y2) + 0.5 * np.cos(y3) + 0.25))) < 1e-12
    assert np.max(np.abs(R.grid_transfer(fine, 16) - f)) < 1e-12
    g = np.cos(8 * y1) + np.cos(7 * y2)   # 8 = the Nyquist wavenumber of 16 points
    assert np.max(np.abs(R.grid_transfer(g, 16) - np.cos(7 * x2))) < 1e-12
    assert R.grid_levels(128) == [16, 32, 64, 128] and R.grid_levels(96) == [12, 24, 48, 96]
    assert R.grid_levels(32) == [16, 32]


def test_rect_freq_filter_is_the_restriction_band():
    # ApplyRectFreqFilter at pct = nc / n keeps |k| <= nc/2 - 1 on every axis
    # for an even coarse size: the band that restriction then prolongation
    # carries; low + high pass is the identity; both are projections
    rng = np.random.default_rng(3)
    for n, nc in ((16, 8), (32, 16), (24, 12), (32, 8)):
        f = rng.standard_normal((n, n, n))
        lo = R.rect_freq_filter(f, nc / n)
        hi = R.rect_freq_filter(f, nc / n, lowpass=False)
        assert np.max(np.abs(lo + hi - f)) < 1e-12
        assert np.max(np.abs(R.rect_freq_filter(lo, nc / n) - lo)) < 1e-12
        assert np.max(np.abs(lo - R.grid_transfer(R.grid_transfer(f, nc), n))) < 1e-12
    f = rng.standard_normal((8, 8, 8))
    assert np.array_equal(R.rect_freq_filter(f, 1.0), f)
    assert not np.any(R.rect_freq_filter(f, 1.0, lowpass=False))


def test_symmetric_hessian_is_the_preconditioned_hessian():
    # PrecondHessMatVecSym: hd x + P^1/2 b~[P^1/2 x] equals P^1/2 H P^1/2 x
    # when the regularisation's Hessian symbol is hd times the inverse's
    # reciprocal (H1: hd beta0 (|k|^2 + beta1) against 1 / (beta0 (|k|^2 + beta1)))
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1", 1e-2))
    prob.gradient(0.4 * vs)
    x = np.random.default_rng(4).standard_normal(vs.shape)
    half = lambda y: prob.reg.apply_inverse(y, applysqrt=True)
    ref = half(prob.hessian_matvec(half(x)))
    out = prob.hessian_sym(x)
    assert np.linalg.norm(out - ref) <= 1e-12 * np.linalg.norm(ref)
    assert np.linalg.norm(prob.hessian_sym(x, scale=False) - out / prob.hd) <= 1e-12 * np.linalg.norm(out / prob.hd)


def test_two_level_gauss_newton():
    # -precond 2level: coarse problems restricted from the current iterate,
    # PCG on the symmetric form, the solution mapped back by P^1/2; it
    # converges like the INVREG solve and the preconditioner inverts the
    # low band (coarse solve to 1e-12: M A r is r on a coarse-band input)
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    reg = R.Regularization("h1s", 1e-2)
    res = {}
    for pc in ("invreg", "2level"):
        prob = R.Problem(mR, mT, nt, reg)
        res[pc] = R.gauss_newton(prob, R.GNOptions(maxit=6, gttol=1e-2, precond=pc))
        assert res[pc]["reason"] == "gttol"
    mis = [R.relative_mismatch(R.Problem(mR, mT, nt, reg).mR, res[pc]["m1"], mT) for pc in res]
    assert abs(mis[0] - mis[1]) < 2e-2
    prob = R.Problem(mR, mT, nt, reg)
    prob.gradient(0.5 * vs)
    coarse = R.two_level_setup(prob)
    assert coarse.shape == (8, 8, 8) and np.array_equal(coarse.v[0], R.grid_transfer(0.5 * vs[0], 8))
    rng = np.random.default_rng(5)
    # outside the coarse band M is the identity (zero coarse right-hand side)
    f = rng.standard_normal((3, 16, 16, 16))
    hi = np.stack([R.rect_freq_filter(f[k], 0.5, lowpass=False) for k in range(3)])
    assert np.max(np.abs(R.two_level_apply(coarse, hi, 1e-13) - hi)) < 1e-12
    # inside it, M z is the prolonged coarse solve: it stays in the band
    lo = np.stack([R.rect_freq_filter(f[k], 0.5) for k in range(3)])
    mz = R.two_level_apply(coarse, lo, 1e-13)
    assert np.max(np.abs(np.stack([R.rect_freq_filter(mz[k], 0.5) for k in range(3)]) - mz)) < 1e-12
    assert np.linalg.norm(mz) > 0.1 * np.linalg.norm(lo)


def test_initialization_uses_zero_velocity_for_g0():
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    prob = R.Problem(mR, mT, nt, R.Regularization("h1s", 1e-2))
    g = prob.gradient(np.zeros_like(vs))
    res = R.gauss_newton(prob, R.GNOptions(maxit=1, gttol=1e-2), v0=0.2 * vs)
    assert abs(res["g0"] - np.sqrt(R.dot(g, g))) <= 1e-12 * res["g0"]


@pytest.mark.parametrize("distance", ["sl2", "ncc"])
def test_masked_distance_taylor_gradient_and_unit_mask(distance):
    # src/DistanceMeasureSL2.cpp / DistanceMeasureNCC.cpp with m_Mask: weighted
    # sums and final conditions; the gradient stays consistent with J
    n, nt = 16, 4
    mR, mT, vs = R.synthetic_c1(n, np.float64, nt)
    x1, x2, x3 = R.grid_coords((n, n, n))
    w = 0.5 + 0.5 * np.cos(x1) ** 2
    reg = R.Regularization("h1s", 1e-2)
    prob = R.Problem(mR, mT, nt, reg, distance=distance, mask=w)
    v = 0.3 * vs
    J0 = prob.objective(v)
    gw = R.dot(prob.gradient(v), vs)
    h = 1e-4
    fd = (prob.objective(v + h * vs) - J0) / h
    assert abs(fd - gw) < 1e-2 * abs(gw)
    ones = R.Problem(mR, mT, nt, reg, distance=distance, mask=np.ones((n, n, n)))
    plain = R.Problem(mR, mT, nt, reg, distance=distance)
    assert abs(ones.objective(v) - plain.objective(v)) <= 1e-12 * abs(plain.objective(v))


def test_golden_c1_64_is_the_current_oracle():
    # the committed 64^3 fixture was made by this oracle: its problem
    # description and its initial gradient norm agree with a fresh evaluation
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c1_64.json")))
    p = g["problem"]
    assert (p["n"], p["nt"], p["regnorm"], p["beta"]) == (64, 4, "h1s", 1e-2)
    mR, mT, _ = R.synthetic_c1(p["n"], np.float64, p["nt"])
    prob = R.Problem(mR.astype(np.float32), mT.astype(np.float32), p["nt"], R.Regularization("h1s", p["beta"]))
    z = np.zeros((3,) + prob.shape)
    prob.objective(z)
    gz = prob.gradient(z)
    assert abs(np.sqrt(R.dot(gz, gz)) - g["g0"]) <= 1e-12 * g["g0"]
    assert g["reason"] in ("gttol", "maxit", "steptol") and len(g["pcg_iterations"]) == g["gn_iterations"]
