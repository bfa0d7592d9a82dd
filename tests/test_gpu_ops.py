"""Parity of the CUDA operator seams against the oracle (FP64 NumPy restatement).

Inputs are seeded FP32 fields; the oracle runs in FP64 on the same FP32
values.  Tolerance: relative L2 error <= 1e-5 for transported images and
spectral operators (FP32 arithmetic on the device).
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


def smooth_field(shape, rng, kmax=4):
    x1, x2, x3 = R.grid_coords(shape)
    f = np.zeros(shape)
    for _ in range(6):
        k = rng.integers(-kmax, kmax + 1, size=3)
        ph = rng.uniform(0, 2 * np.pi)
        f += rng.normal() * np.cos(k[0] * x1 + k[1] * x2 + k[2] * x3 + ph)
    return f.astype(np.float32)


def velocity(shape, rng, amp=0.5):
    return np.stack([smooth_field(shape, rng) for _ in range(3)]) * np.float32(amp)


@pytest.fixture(scope="module")
def cb(cuda):
    import claire_b200
    return claire_b200


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("n", [16, 32, 48, 64])
def test_interp3_scalar_and_vector(cb, n):
    rng = np.random.default_rng(n)
    shape = (n, n, n)
    f = rng.standard_normal(shape).astype(np.float32)
    disp = rng.uniform(-7.5, 7.5, size=(3,) + shape).astype(np.float32)
    q = R.index_grid(shape) + disp.astype(np.float64)
    ref = R.interp3(f.astype(np.float64), q)
    out = cb.SemiLagrangian.Interpolate(to_dev(f), to_dev(disp)).cpu().numpy()
    assert rel(out, ref) < TOL
    fv = rng.standard_normal((3,) + shape).astype(np.float32)
    refv = np.stack([R.interp3(fv[d].astype(np.float64), q) for d in range(3)])
    outv = cb.SemiLagrangian.Interpolate(to_dev(fv), to_dev(disp)).cpu().numpy()
    assert rel(outv, refv) < TOL


def test_interp3_reproduces_cubics_and_nodes(cb):
    n = 32
    shape = (n, n, n)
    rng = np.random.default_rng(1)
    idx = R.index_grid(shape)
    # integer displacements: the gather returns node values exactly
    disp = rng.integers(-5, 6, size=(3,) + shape).astype(np.float32)
    f = rng.standard_normal(shape).astype(np.float32)
    out = cb.SemiLagrangian.Interpolate(to_dev(f), to_dev(disp)).cpu().numpy()
    ii = [(idx[d] + disp[d]).astype(np.int64) % n for d in range(3)]
    assert np.array_equal(out, f[ii[0], ii[1], ii[2]])
    # cubic polynomial away from the periodic seam is reproduced to roundoff
    poly = lambda a, b, c: 0.5 + 0.01 * a - 0.002 * b * b + 1e-4 * a * b * c - 2e-5 * c ** 3
    F = poly(idx[0], idx[1], idx[2]).astype(np.float32)
    d = rng.uniform(-0.9, 0.9, size=(3,) + shape).astype(np.float32)
    out = cb.SemiLagrangian.Interpolate(to_dev(F), to_dev(d)).cpu().numpy()
    q = idx + d.astype(np.float64)
    inner = (slice(3, n - 3),) * 3
    exact = poly(q[0], q[1], q[2])
    assert np.max(np.abs(out[inner] - exact[inner])) < 2e-5


@pytest.mark.parametrize("n", [32, 48, 64])
def test_interp3_staged_boxes_across_the_seams(cb, n):
    """Displacements of under a cell keep every tile's footprint box small
    enough to be staged in shared memory, so these gathers take the staged
    path (bulk row copies), not the global fallback of the rougher
    displacements above.  Boxes of border tiles start before the domain and
    rows cross the periodic x3 seam (two copies per row); a uniform
    displacement makes every tile's box the same shape."""
    rng = np.random.default_rng(300 + n)
    shape = (n, n, n)
    f = smooth_field(shape, rng, 6) + 0.1 * rng.standard_normal(shape).astype(np.float32)
    f = f.astype(np.float32)
    idx = R.index_grid(shape)
    for disp in (np.stack([np.full(shape, c, np.float32) for c in (0.37, -0.81, 0.55)]),
                 np.stack([(0.45 * smooth_field(shape, rng, 3) / 6).astype(np.float32) for _ in range(3)])):
        assert np.abs(disp).max() < 1.0
        ref = R.interp3(f.astype(np.float64), idx + disp.astype(np.float64))
        out = cb.SemiLagrangian.Interpolate(to_dev(f), to_dev(disp)).cpu().numpy()
        assert rel(out, ref) < TOL


@pytest.mark.parametrize("n,nt,flag", [(32, 4, "state"), (32, 8, "adjoint"), (48, 4, "state"), (64, 4, "adjoint")])
def test_trajectory(cb, n, nt, flag):
    rng = np.random.default_rng(n + nt)
    shape = (n, n, n)
    v = velocity(shape, rng)
    ref = R.trajectory_rk2(v.astype(np.float64), nt, flag)
    out = cb.SemiLagrangian(nt).ComputeTrajectory(to_dev(v), flag).cpu().numpy()
    assert rel(out, ref) < TOL


@pytest.mark.parametrize("n", [16, 32, 48, 64, 96, 128])
def test_fft_grad_div(cb, n):
    rng = np.random.default_rng(n)
    shape = (n, n, n)
    f = rng.standard_normal(shape).astype(np.float32)
    g = cb.fft_grad(to_dev(f)).cpu().numpy()
    assert rel(g, R.grad(f.astype(np.float64))) < TOL
    v = rng.standard_normal((3,) + shape).astype(np.float32)
    d = cb.fft_div(to_dev(v)).cpu().numpy()
    assert rel(d, R.div(v.astype(np.float64))) < TOL


def test_fft_grad_trig_exact(cb):
    n = 64
    shape = (n, n, n)
    x1, x2, x3 = R.grid_coords(shape)
    m = (np.sin(2 * x1) * np.cos(3 * x2) + np.sin(5 * x3)).astype(np.float32)
    g = cb.fft_grad(to_dev(m)).cpu().numpy()
    ex = np.stack([2 * np.cos(2 * x1) * np.cos(3 * x2), -3 * np.sin(2 * x1) * np.sin(3 * x2), 5 * np.cos(5 * x3)])
    assert np.max(np.abs(g - ex)) < 1e-4


@pytest.mark.parametrize("norm", ["l2", "h1", "h1s", "h2", "h2s", "h3", "h3s"])
@pytest.mark.parametrize("n", [32, 48])
def test_regularization_ops(cb, norm, n):
    rng = np.random.default_rng(7)
    shape = (n, n, n)
    v = velocity(shape, rng) + 0.01 * rng.standard_normal((3,) + shape).astype(np.float32)
    v = v.astype(np.float32)
    reg = R.Regularization(norm, 1e-2, 1e-4)
    op = cb.Regularization(norm, 1e-2, 1e-4)
    dv = to_dev(v)
    assert rel(op.EvaluateGradient(dv).cpu().numpy(), reg.gradient(v.astype(np.float64))) < TOL
    assert rel(op.ApplyInverse(dv).cpu().numpy(), reg.apply_inverse(v.astype(np.float64))) < TOL
    if norm != "l2":
        assert rel(op.ApplyInverse(dv, True).cpu().numpy(), reg.apply_inverse(v.astype(np.float64), True)) < TOL
    Rg = op.EvaluateFunctional(dv)
    Rr = reg.functional(v.astype(np.float64))
    assert abs(Rg - Rr) <= TOL * abs(Rr) + 1e-12


@pytest.mark.parametrize("model", ["stokes", "relaxedstokes"])
def test_leray(cb, model):
    n = 32
    rng = np.random.default_rng(3)
    shape = (n, n, n)
    b = rng.standard_normal((3,) + shape).astype(np.float32)
    ref = R.leray_projection(b.astype(np.float64), model, 1e-2, 1e-4)
    db = to_dev(b)
    cb.leray(db, model, (1e-2, 1e-4, 1e-4))
    assert rel(db.cpu().numpy(), ref) < TOL


def test_leray_divergence_free(cb):
    n = 32
    rng = np.random.default_rng(4)
    b = velocity((n, n, n), rng)
    db = to_dev(b)
    cb.leray(db, "stokes")
    d = cb.fft_div(db).cpu().numpy()
    assert np.max(np.abs(d)) < 1e-4 * np.max(np.abs(b))


def test_smooth_and_distance(cb):
    n = 32
    rng = np.random.default_rng(5)
    shape = (n, n, n)
    f = rng.standard_normal(shape).astype(np.float32)
    s = cb.smooth(to_dev(f)).cpu().numpy()
    assert rel(s, R.gaussian_smooth(f.astype(np.float64), 1.0)) < TOL
    g = rng.standard_normal(shape).astype(np.float32)
    D = cb.DistanceMeasureSL2.EvaluateFunctional(to_dev(f), to_dev(g))
    Dr = 0.5 * R.lebesgue_measure(shape) * np.sum((f.astype(np.float64) - g) ** 2)
    assert abs(D - Dr) <= 1e-12 * abs(Dr)


def test_kernel_launch_counter_moves(cb):
    n = 16
    before = cb.kernel_launches()
    cb.fft_grad(to_dev(np.zeros((n, n, n), np.float32)))
    assert cb.kernel_launches() >= before + 3


def test_file_path_preprocess_matches_oracle(cb, tmp_path):
    # read (NIfTI, int16 with a negative outlier) -> Normalize -> Gaussian smoothing
    # (src/CLAIREUtils.cpp:492-525, src/CLAIREInterface.cpp:594-626)
    n = 32
    rng = np.random.default_rng(77)
    vol = (1000 * smooth_field((n, n, n), rng) + 2500).astype(np.int16)
    vol[3, 4, 5] = -40
    p = str(tmp_path / "img.nii.gz")
    cb.write_nifti(p, vol.astype(np.float32))
    img = cb.read_nifti(p)
    assert np.array_equal(img, vol.astype(np.float32))
    dev = to_dev(img)
    cb.preprocess(dev, rescale=True, sigma=(1.0, 1.0, 1.0))
    ref = R.gaussian_smooth(R.normalize(img.astype(np.float64)), 1.0)
    assert rel(dev.cpu().numpy(), ref) < TOL
    dev2 = to_dev(img)
    cb.preprocess(dev2, rescale=True, sigma=None)
    assert rel(dev2.cpu().numpy(), R.normalize(img.astype(np.float64))) < 1e-6
