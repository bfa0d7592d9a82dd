"""Synthetic registration problems (setup, not the hot path).

* ``template_sin2`` / ``velocity_trig``: CLAIREBase::SetupSyntheticProb's
  -synthetic 0 fields (src/CLAIREBase.cpp:1026-1250): mT = (sin^2 x1 +
  sin^2 x2 + sin^2 x3)/3 and v0*(sin x3 cos x2 sin x2, sin x1 cos x3 sin x3,
  sin x2 cos x1 sin x1); ``reference_case=False`` drops the trailing sine
  factor (the benchmark's 64^3 problem).
* ``ellipsoid_problem``: the benchmark recipe for the 128^3 / batched /
  serving problems: 40 seeded Gaussian ellipsoids (centres U[0,2pi)^3,
  semi-axes U[0.1,0.5] rad, uniform random rotation, intensity U[0.2,1]),
  smoothed with a 1-cell Gaussian (the library's spectral smoother) and
  clipped to [0,1]; velocity with Fourier modes 1 <= |k| <= 6 and complex
  amplitude N(0,0.3)/|k|^2, scaled to RMS 0.3; mR = SL transport of mT by
  that velocity with the library's own forward solver.

Random draws use NumPy's PCG64 with seed 20261203 + 1000*config + problem; the
fields are evaluated with torch on the GPU.
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


# RMS of the random velocity over grid and components (band-limited field:
# independent of the grid size)
VELOCITY_RMS = 0.3


def seed(config_index: int, problem_index: int) -> int:
    return 20261203 + 1000 * config_index + problem_index


def _coords(n, device, dtype):
    import torch
    x = (TWO_PI / n) * torch.arange(n, device=device, dtype=dtype)
    return torch.meshgrid(x, x, x, indexing="ij")


def rescale(x):
    """Rescale (src/CLAIREUtils.cpp:691-725): shift by -min only when min < -1e-6,
    then scale by 1/(max - min)."""
    xmin = float(x.min())
    xmax = float(x.max())
    if -xmin > 1e-6:
        x = x + (-xmin)
    s = 1.0 / (xmax - xmin) if abs(xmax - xmin) > 1e-6 else 1.0
    return x * s


def template_sin2(n, device="cuda"):
    import torch
    x1, x2, x3 = _coords(n, device, torch.float64)
    return ((torch.sin(x1) ** 2 + torch.sin(x2) ** 2 + torch.sin(x3) ** 2) / 3.0).float()


def velocity_trig(n, v0=0.5, reference_case=False, device="cuda"):
    import torch
    x1, x2, x3 = _coords(n, device, torch.float64)
    if reference_case:
        v = torch.stack([torch.sin(x3) * torch.cos(x2) * torch.sin(x2),
                         torch.sin(x1) * torch.cos(x3) * torch.sin(x3),
                         torch.sin(x2) * torch.cos(x1) * torch.sin(x1)])
    else:
        v = torch.stack([torch.sin(x3) * torch.cos(x2), torch.sin(x1) * torch.cos(x3), torch.sin(x2) * torch.cos(x1)])
    return (v0 * v).float().contiguous()


def _wavenumbers(n):
    w = np.arange(n, dtype=np.int64)
    w[w > n // 2] -= n
    w[w == n // 2] = 0
    return w


def draw_ellipsoid_params(rng, count=40):
    """Per-ellipsoid draws in a fixed order: centre(3), sigma(3), amplitude, quaternion(4)."""
    out = []
    for _ in range(count):
        c = rng.uniform(0.0, TWO_PI, size=3)
        sig = rng.uniform(0.1, 0.5, size=3)
        amp = rng.uniform(0.2, 1.0)
        qv = rng.normal(size=4)
        qv /= np.linalg.norm(qv)
        a, b, cq, d = qv
        rot = np.array([
            [a * a + b * b - cq * cq - d * d, 2 * (b * cq - a * d), 2 * (b * d + a * cq)],
            [2 * (b * cq + a * d), a * a - b * b + cq * cq - d * d, 2 * (cq * d - a * b)],
            [2 * (b * d - a * cq), 2 * (cq * d + a * b), a * a - b * b - cq * cq + d * d],
        ])
        out.append((c, sig, amp, rot))
    return out


def draw_velocity_coeffs(rng, n, kmax=6, amp=0.3):
    # Nyquist indices keep their magnitude n/2 > kmax: no Nyquist mode (a +-1
    # checkerboard on the grid) enters the field
    k = np.arange(n, dtype=np.float64)
    k[k > n // 2] -= n
    k3 = k[: n // 2 + 1].copy()
    k3[n // 2] = n // 2
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + k3[None, None, :] ** 2)
    mask = (kk >= 1.0) & (kk <= kmax)
    coeffs = []
    for _ in range(3):
        c = rng.normal(0.0, amp, size=(n, n, n // 2 + 1)) + 1j * rng.normal(0.0, amp, size=(n, n, n // 2 + 1))
        c = np.where(mask, c / np.where(kk > 0, kk * kk, 1.0), 0.0)
        coeffs.append(c)
    return coeffs


def ellipsoid_template(n, params, device="cuda"):
    import torch
    import claire_b200 as cb
    x = _coords(n, device, torch.float64)
    out = torch.zeros((n, n, n), device=device, dtype=torch.float64)
    for c, sig, amp, rot in params:
        dx = [torch.remainder(x[i] - c[i] + math.pi, TWO_PI) - math.pi for i in range(3)]
        acc = 0.0
        for r in range(3):
            u = rot[0, r] * dx[0] + rot[1, r] * dx[1] + rot[2, r] * dx[2]
            acc = acc + (u / sig[r]) ** 2
        out += amp * torch.exp(-0.5 * acc)
    smoothed = cb.smooth(out.float().contiguous(), (1.0, 1.0, 1.0))
    return torch.clamp(smoothed, 0.0, 1.0).contiguous()


def random_velocity(n, coeffs, device="cuda", rms=VELOCITY_RMS):
    """Real field from half-spectrum coefficients: each coefficient contributes
    c e^{ik.x} + c.c. (Hermitian completion of the real inverse transform),
    scaled to the given RMS over grid and components (``rms=None`` keeps the
    raw sum of the ~520 modes per component, RMS ~1.4: a folding map)."""
    import torch
    comps = []
    for c in coeffs:
        ct = torch.from_numpy(c * (n ** 3)).to(device)
        comps.append(torch.fft.irfftn(ct, s=(n, n, n), dim=(0, 1, 2)))
    v = torch.stack(comps)
    if rms is not None:
        v = v * (rms / torch.sqrt(torch.mean(v * v)))
    return v.float().contiguous()


def ellipsoid_problem(n, nt, config_index=1, problem_index=0, device="cuda"):
    """(mR, mT, v) on the GPU for one problem of the benchmark recipe."""
    import claire_b200 as cb
    rng = np.random.Generator(np.random.PCG64(seed(config_index, problem_index)))
    params = draw_ellipsoid_params(rng)
    coeffs = draw_velocity_coeffs(rng, n)
    mT = ellipsoid_template(n, params, device)
    v = random_velocity(n, coeffs, device)
    mR = transport(mT, v, nt)
    return mR, mT, v


def transport(m0, v, nt):
    """m1 = SL transport of m0 along v with the library (SolveForwardProblem)."""
    import torch
    import claire_b200 as cb
    sl = cb.SemiLagrangian(nt)
    disp = sl.ComputeTrajectory(v, "state")
    m = m0.contiguous()
    for _ in range(nt):
        m = sl.Interpolate(m, disp)
    torch.cuda.synchronize()
    return m


def sin2_problem(n, nt, reference_case=False, device="cuda"):
    """Config-1 style problem: rescaled sin^2 template transported by the trig velocity."""
    mT = rescale(template_sin2(n, device))
    v = velocity_trig(n, 0.5, reference_case, device)
    mR = rescale(transport(mT, v, nt))
    return mR.contiguous(), mT.contiguous(), v
