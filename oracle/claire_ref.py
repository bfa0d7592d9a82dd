"""CPU restatement of CLAIRE's Gauss-Newton-Krylov hot path (test oracle).

THIS IS TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import it, and only as the checker or the
timed CPU baseline.  The product path (``claire_b200``) never calls it.

It restates, in NumPy (FP64 by default, FP32 on request), the arithmetic of the
reference CPU code for one periodic registration problem on [0, 2*pi)^3:

* semi-Lagrangian RK2 characteristics and tricubic Lagrange interpolation
  (src/SemiLagrangian.cpp:192-289, src/interp3.cpp:2492-2719,
  src/Interp3_Plan.cpp:344-361);
* state / adjoint / incremental state / incremental adjoint SL solvers
  (src/CLAIRE.cpp:2116-2175, 2550-2722, 3147-3290, 3849-4012);
* SL2 distance and final conditions (src/DistanceMeasureSL2.cpp:93-283);
* spectral regularisation L2/H1/H1SN/H2/H2SN/H3/H3SN
  (src/Regularization*.cpp), Leray projections (src/CLAIREStokes.cpp:407-540,
  src/CLAIREDivReg.cpp:313-460);
* objective, gradient, GN Hessian matvec (src/CLAIRE.cpp:793-1042, 1218-1379);
* inverse-regularisation preconditioner (src/Preconditioner.cpp:507-580);
* PCG with the SLFS/QDFS forcing sequence (src/KrylovInterface.cpp:79-196,
  src/Optimizer.cpp:296-356) and a GN + Armijo outer loop with CLAIRE's own
  stopping test (src/TaoInterface.cpp:391-527).

Parity status.  The reference cannot be built in this environment (it needs
MPI, PETSc 3.9.1, AccFFT and FFTW), and it ships no golden vectors or tests.
The restatement is pinned by the reference's own known-answer checks instead:
tricubic reproduction of cubics and of node values, spectral operators on trig
polynomials, the forward/backward transport round trip of
apps/benchmark.cpp:297-380, the Taylor gradient test and the Hessian symmetry
test of src/OptimizationProblem.cpp:157-496.  The GN/PCG/line-search loop
restates PETSc TAO ``nls`` + Armijo, which lives outside the tree (PETSc
3.9.1): its iteration counts are "parity unpinned".  AccFFT's spectral
derivative convention (also outside the tree) is restated with the Nyquist
wavenumber set to zero, as CLAIRE's own ComputeWaveNumber does
(include/CLAIREUtils.hpp:248-255).

Array conventions (include/CLAIREUtils.hpp:198-212): scalar fields have shape
(N1, N2, N3), row-major with x3 fastest; vector fields have shape (3, N1, N2,
N3) (the flat [x1 | x2 | x3] layout of src/VecField.cpp:396-478).  Grid
x_i = i*h, h = 2*pi/N (src/RegOpt.cpp:935); hd = h1*h2*h3; ht = 1/nt.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

TWO_PI = 2.0 * math.pi

# --------------------------------------------------------------------------
# grid helpers
# --------------------------------------------------------------------------


def wavenumbers(n: int, nyquist_zero: bool = True) -> np.ndarray:
    """Integer wavenumbers of an n-point axis.

    include/CLAIREUtils.hpp:248-255 (ComputeWaveNumber): w > n/2 -> w - n and
    w == n/2 -> 0.  With ``nyquist_zero=False`` the Nyquist index keeps +n/2
    (the inverse-Laplacian convention of src/CLAIREStokes.cpp:455-466).
    """
    w = np.arange(n, dtype=np.int64)
    w[w > n // 2] -= n
    if nyquist_zero:
        w[w == n // 2] = 0
    return w


def spectral_k(shape, nyquist_zero: bool = True):
    """Broadcastable wavenumber arrays (k1, k2, k3) on the r2c half spectrum."""
    n1, n2, n3 = shape
    k1 = wavenumbers(n1, nyquist_zero)[:, None, None].astype(np.float64)
    k2 = wavenumbers(n2, nyquist_zero)[None, :, None].astype(np.float64)
    k3full = wavenumbers(n3, nyquist_zero)
    k3 = k3full[: n3 // 2 + 1].copy()
    if nyquist_zero:
        k3[n3 // 2] = 0
    else:
        k3[n3 // 2] = n3 // 2
    k3 = k3[None, None, :].astype(np.float64)
    return k1, k2, k3


def lebesgue_measure(shape) -> float:
    """hd = hx1*hx2*hx3 (include/RegOpt.hpp:485-489)."""
    return float(np.prod([TWO_PI / n for n in shape]))


def grid_coords(shape, dtype=np.float64):
    """Nodal coordinates x_i = i*h (src/SemiLagrangian.cpp:236-238)."""
    n1, n2, n3 = shape
    x1 = (TWO_PI / n1) * np.arange(n1, dtype=dtype)
    x2 = (TWO_PI / n2) * np.arange(n2, dtype=dtype)
    x3 = (TWO_PI / n3) * np.arange(n3, dtype=dtype)
    return np.meshgrid(x1, x2, x3, indexing="ij")


# --------------------------------------------------------------------------
# tricubic Lagrange interpolation (src/interp3.cpp:2492-2719)
# --------------------------------------------------------------------------

LAGRANGE_DENOM = (-1.0 / 6.0, 0.5, -0.5, 1.0 / 6.0)  # src/interp3.cpp:2508-2512


def lagrange_weights(t: np.ndarray):
    """w_k(t) = c_k * prod_{l != k} (t - l), k = 0..3 (src/interp3.cpp:2524-2535)."""
    return [
        LAGRANGE_DENOM[0] * (t - 1.0) * (t - 2.0) * (t - 3.0),
        LAGRANGE_DENOM[1] * t * (t - 2.0) * (t - 3.0),
        LAGRANGE_DENOM[2] * t * (t - 1.0) * (t - 3.0),
        LAGRANGE_DENOM[3] * t * (t - 1.0) * (t - 2.0),
    ]


class Stencil:
    """Base indices and weights of the 4x4x4 tricubic stencil at query points.

    ``q`` holds query coordinates in grid units (shape (3, ...)); the periodic
    wrap of src/Interp3_Plan.cpp:344-361 and the ghost shift of
    src/interp3.cpp:24-60 reduce to indexing modulo N.  base = floor(q) - 1 and
    t = q - base lies in [1, 2) (src/interp3.cpp:2518-2522).
    """

    def __init__(self, q: np.ndarray, shape):
        self.shape = tuple(shape)
        n1, n2, n3 = self.shape
        dtype = q.dtype
        base = np.floor(q).astype(np.int64) - 1
        t = (q - base).astype(dtype)
        self.w = [lagrange_weights(t[d]) for d in range(3)]
        self.i1 = [((base[0] + a) % n1) * (n2 * n3) for a in range(4)]
        self.i2 = [((base[1] + b) % n2) * n3 for b in range(4)]
        self.i3 = [(base[2] + c) % n3 for c in range(4)]

    def apply(self, f: np.ndarray) -> np.ndarray:
        flat = f.reshape(-1)
        out = None
        for a in range(4):
            acc_a = None
            for b in range(4):
                acc_b = None
                ib = self.i1[a] + self.i2[b]
                for c in range(4):
                    term = self.w[2][c] * flat[ib + self.i3[c]]
                    acc_b = term if acc_b is None else acc_b + term
                term = self.w[1][b] * acc_b
                acc_a = term if acc_a is None else acc_a + term
            term = self.w[0][a] * acc_a
            out = term if out is None else out + term
        return out.astype(f.dtype, copy=False)


def interp3(f: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Tricubic interpolation of a periodic scalar field at grid-unit points q."""
    return Stencil(q, f.shape).apply(f)


# --------------------------------------------------------------------------
# characteristics (src/SemiLagrangian.cpp:192-289)
# --------------------------------------------------------------------------


def index_grid(shape, dtype=np.float64):
    n1, n2, n3 = shape
    return np.stack(
        np.meshgrid(
            np.arange(n1, dtype=dtype),
            np.arange(n2, dtype=dtype),
            np.arange(n3, dtype=dtype),
            indexing="ij",
        )
    )


def trajectory_rk2(v: np.ndarray, nt: int, flag: str = "state"):
    """RK2 characteristic foot points X in grid units.

    src/SemiLagrangian.cpp:217-280: scale = +1 (state) / -1 (adjoint);
    Xt = x - scale*ht*v; vX = v(Xt); X = x - scale*(ht/2)*(v + vX).  Grid
    units are X*N/(2*pi) (the rescale of src/interp3.cpp:24-60 without ghost
    shift).  Returns the displacement q - i, shape (3, N1, N2, N3).
    """
    scale = {"state": 1.0, "adjoint": -1.0}[flag]
    shape = v.shape[1:]
    dtype = v.dtype
    ht = 1.0 / nt
    inv_h = np.array([n / TWO_PI for n in shape], dtype=dtype)
    idx = index_grid(shape, dtype)
    disp1 = np.stack([-scale * ht * v[d] * inv_h[d] for d in range(3)]).astype(dtype)
    st = Stencil(idx + disp1, shape)
    vx = np.stack([st.apply(v[d]) for d in range(3)])
    disp = np.stack(
        [-scale * (0.5 * ht) * (v[d] + vx[d]) * inv_h[d] for d in range(3)]
    ).astype(dtype)
    return disp


class Trajectory:
    """Foot points of one characteristic with a cached stencil."""

    def __init__(self, v: np.ndarray, nt: int, flag: str):
        self.disp = trajectory_rk2(v, nt, flag)
        shape = v.shape[1:]
        self.stencil = Stencil(index_grid(shape, v.dtype) + self.disp, shape)

    def interp(self, f: np.ndarray) -> np.ndarray:
        return self.stencil.apply(f)

    def interp_vec(self, f: np.ndarray) -> np.ndarray:
        return np.stack([self.stencil.apply(f[d]) for d in range(3)])


# --------------------------------------------------------------------------
# spectral operators (AccFFT call sites, e.g. src/CLAIRE.cpp:2622, 2662)
# --------------------------------------------------------------------------


def _rfft(f):
    return np.fft.rfftn(f, axes=(0, 1, 2))


def _irfft(fh, shape, dtype):
    return np.fft.irfftn(fh, s=shape, axes=(0, 1, 2)).astype(dtype)


def grad(f: np.ndarray) -> np.ndarray:
    """Spectral gradient grad f = F^-1(i k F f), Nyquist zeroed (accfft_grad_t)."""
    shape = f.shape
    fh = _rfft(f)
    k = spectral_k(shape)
    return np.stack([_irfft(1j * k[d] * fh, shape, f.dtype) for d in range(3)])


def div(v: np.ndarray) -> np.ndarray:
    """Spectral divergence F^-1(i k . F v), Nyquist zeroed (accfft_divergence_t)."""
    shape = v.shape[1:]
    k = spectral_k(shape)
    acc = sum(1j * k[d] * _rfft(v[d]) for d in range(3))
    return _irfft(acc, shape, v.dtype)


# --------------------------------------------------------------------------
# regularisation (src/Regularization{L2,H1,H1SN,H2,H2SN,H3,H3SN}.cpp)
# --------------------------------------------------------------------------

NORMS = ("l2", "h1", "h1s", "h2", "h2s", "h3", "h3s")


@dataclasses.dataclass
class Regularization:
    """Spectral regularisation model; ``norm`` uses CLAIRE's -regnorm names.

    beta0 = -beta, beta1 defaults to 1e-4 (src/RegOpt.cpp:1073).
    """

    norm: str = "h1s"
    beta0: float = 1e-2
    beta1: float = 1e-4

    def _kappa(self, shape):
        k1, k2, k3 = spectral_k(shape)
        return k1 * k1 + k2 * k2 + k3 * k3

    def grad_symbol(self, shape):
        """Symbol of EvaluateGradient / HessianMatVec (without the 1/N^3 scale)."""
        hd = lebesgue_measure(shape)
        kap = self._kappa(shape)
        b0, b1 = self.beta0, self.beta1
        if self.norm == "h1s":  # src/RegularizationH1SN.cpp:217
            return hd * b0 * kap
        if self.norm == "h1":  # src/RegularizationH1.cpp:229
            return hd * b0 * (kap + b1)
        if self.norm == "h2":  # src/RegularizationH2.cpp:239 (no hd)
            return b0 * (kap * kap + b1)
        if self.norm == "h2s":  # src/RegularizationH2SN.cpp:244
            return hd * b0 * kap * kap
        if self.norm == "h3":  # src/RegularizationH3.cpp:250-254 (no hd)
            return b0 * (kap ** 3 + b1)
        if self.norm == "h3s":  # src/RegularizationH3SN.cpp:246-250 (no hd)
            return b0 * kap ** 3
        raise ValueError(self.norm)

    def inv_symbol(self, shape, applysqrt: bool = False):
        """Symbol of ApplyInverse (without the 1/N^3 scale)."""
        kap = self._kappa(shape)
        b0, b1 = self.beta0, self.beta1
        if self.norm == "h1s":  # src/RegularizationH1SN.cpp:356-359
            op = np.where(kap == 0.0, b0, b0 * kap)
        elif self.norm == "h1":  # src/RegularizationH1.cpp:379-382
            op = b0 * (kap + b1)
        elif self.norm == "h2":  # src/RegularizationH2.cpp:378-381
            op = b0 * (kap * kap + b1)
        elif self.norm == "h2s":  # src/RegularizationH2SN.cpp:388-390
            op = np.where(kap == 0.0, b0, b0 * kap * kap)
        elif self.norm == "h3":  # src/RegularizationH3.cpp:396-399
            op = b0 * (kap ** 3 + b1)
        elif self.norm == "h3s":  # src/RegularizationH3SN.cpp:388-391
            op = np.where(kap == 0.0, b0, b0 * kap ** 3)
        else:
            raise ValueError(self.norm)
        if applysqrt:
            op = np.sqrt(op)
        return 1.0 / op

    def gradient(self, v: np.ndarray) -> np.ndarray:
        if self.beta0 == 0.0:
            return np.zeros_like(v)
        if self.norm == "l2":  # src/RegularizationL2.cpp:100-125
            return self.beta0 * v
        shape = v.shape[1:]
        sym = self.grad_symbol(shape)
        return np.stack([_irfft(sym * _rfft(v[d]), shape, v.dtype) for d in range(3)])

    hessian_matvec = gradient

    def apply_inverse(self, x: np.ndarray, applysqrt: bool = False) -> np.ndarray:
        if self.beta0 == 0.0:
            return x.copy()
        if self.norm == "l2":  # src/RegularizationL2.cpp:190-215
            return x / self.beta0
        shape = x.shape[1:]
        sym = self.inv_symbol(shape, applysqrt)
        return np.stack([_irfft(sym * _rfft(x[d]), shape, x.dtype) for d in range(3)])

    def functional(self, v: np.ndarray) -> float:
        if self.beta0 == 0.0:
            return 0.0
        shape = v.shape[1:]
        hd = lebesgue_measure(shape)
        b0, b1 = self.beta0, self.beta1
        if self.norm == "l2":  # src/RegularizationL2.cpp:64-88
            return 0.5 * hd * b0 * float(np.sum(v.astype(np.float64) ** 2))
        if self.norm in ("h1s", "h1"):
            # src/RegularizationH1SN.cpp:84-141 / src/RegularizationH1.cpp:84-147:
            # spectral gradients of each component, sum of squares.
            h1v = 0.0
            for d in range(3):
                g = grad(v[d])
                h1v += float(np.sum(g.astype(np.float64) ** 2))
            if self.norm == "h1s":
                return 0.5 * hd * b0 * h1v
            l2v = float(np.sum(v.astype(np.float64) ** 2))
            return 0.5 * hd * b0 * (h1v + b1 * l2v)
        kap = self._kappa(shape)
        if self.norm == "h2":  # src/RegularizationH2.cpp:118-164
            sym = math.sqrt(b0) * (-kap + math.sqrt(b1))
            r = sum(
                float(np.sum(_irfft(sym * _rfft(v[d]), shape, np.float64) ** 2))
                for d in range(3)
            )
            return 0.5 * hd * r
        if self.norm == "h2s":  # src/RegularizationH2SN.cpp:120-163
            r = sum(
                float(np.sum(_irfft(-kap * _rfft(v[d]), shape, np.float64) ** 2))
                for d in range(3)
            )
            return 0.5 * b0 * hd * r
        if self.norm in ("h3", "h3s"):
            # src/RegularizationH3.cpp:118-177, src/RegularizationH3SN.cpp:116-175:
            # the real and imaginary parts carry different real multipliers.
            k = spectral_k(shape)
            r = 0.0
            for d in range(3):
                a = k[d] * (-kap)
                vh = _rfft(v[d])
                if self.norm == "h3":
                    mre = math.sqrt(b0) * (a + math.sqrt(b1))
                    mim = math.sqrt(b0) * (-a + math.sqrt(b1))
                else:
                    mre, mim = a, -a
                wh = mre * vh.real + 1j * (mim * vh.imag)
                r += float(np.sum(_irfft(wh, shape, np.float64) ** 2))
            return 0.5 * hd * r * (b0 if self.norm == "h3s" else 1.0)
        raise ValueError(self.norm)


def leray_projection(b: np.ndarray, model: str = "stokes", beta_v: float = 1e-2,
                     beta_w: float = 1e-4) -> np.ndarray:
    """b + F^-1(-c(k) k (k . b^) / kappa) (src/CLAIREStokes.cpp:407-540,
    src/CLAIREDivReg.cpp:313-460).

    Stokes keeps the Nyquist index as +N/2 in kappa and zeroes it in k; the
    relaxed model zeroes it in both and multiplies by
    c = (beta_v (beta_w (kappa + 1))^-1 + 1)^-1.  kappa = 0 maps to -1 in the
    inverse Laplacian.
    """
    shape = b.shape[1:]
    kg = spectral_k(shape, nyquist_zero=True)
    if model == "stokes":
        kl = spectral_k(shape, nyquist_zero=False)
        c = 1.0
    else:
        kl = kg
    kap = kl[0] ** 2 + kl[1] ** 2 + kl[2] ** 2
    lapinv = np.where(kap == 0.0, -1.0, -1.0 / np.where(kap == 0.0, 1.0, kap))
    if model != "stokes":
        kz = kg[0] ** 2 + kg[1] ** 2 + kg[2] ** 2
        opik = 1.0 / (beta_w * (kz + 1.0))
        c = 1.0 / (beta_v * opik + 1.0)
    bh = [_rfft(b[d]) for d in range(3)]
    kdotb = kg[0] * bh[0] + kg[1] * bh[1] + kg[2] * bh[2]
    out = np.stack(
        [b[d] + _irfft(c * lapinv * kg[d] * kdotb, shape, b.dtype) for d in range(3)]
    )
    return out


# --------------------------------------------------------------------------
# registration problem (src/CLAIRE.cpp)
# --------------------------------------------------------------------------


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Values of x stored as bfloat16 (the upper 16 bits of the float32
    pattern), rounded to nearest with ties to even, returned as float64.
    x is first rounded to float32 (the device computes the stored values in
    FP32).  This emulates the library's bf16 image storage; the reference has
    no such format."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class Problem:
    """One SL2 registration problem with the GN (single time level) storage layout.

    The state is kept at nt+1 levels, the adjoint / incremental variables at one
    level (src/CLAIRE.cpp:149-172).
    """

    def __init__(self, mR, mT, nt: int, reg: Regularization, dtype=np.float64,
                 projection: Optional[str] = None, image_store=None, distance: str = "sl2", mask=None):
        # image_store: rounding applied to every stored image value (mR, mT
        # and each state level), e.g. bf16_round; None keeps dtype values
        self.dtype = dtype
        self.image_store = image_store
        if image_store is not None:
            mR = image_store(mR)
            mT = image_store(mT)
        self.mR = np.asarray(mR, dtype=dtype)
        self.mT = np.asarray(mT, dtype=dtype)
        self.shape = self.mR.shape
        self.distance_type = distance
        # SetMask weights of the distance measure (None: weight 1)
        self.mask = None if mask is None else np.asarray(mask, np.float64)
        if distance not in ("sl2", "ncc"):
            raise ValueError(distance)
        self.nt = nt
        self.ht = 1.0 / nt
        self.hd = lebesgue_measure(self.shape)
        self.ncc_scale = self._ncc_setup_scale() if distance == "ncc" else None
        self.reg = reg
        self.projection = projection
        self.beta_w = 1e-4  # -beta-div (src/RegOpt.cpp:729-731, default 1e-4)
        self.v = None
        self.m = None
        self.counters = dict(obj=0, grad=0, hessmatvec=0, pcmatvec=0, pdesolve=0)

    # --- forward (src/CLAIRE.cpp:1861-1984, 2116-2175) ---------------------
    def set_velocity(self, v):
        v = np.asarray(v, dtype=self.dtype)
        if self.v is not None and self.v.shape == v.shape and np.array_equal(self.v, v):
            return
        self.v = v.copy()
        self.m = None
        self._traj_state = None
        self._traj_adj = None
        self._gradm = None
        self._divv = None

    def traj_state(self):
        if self._traj_state is None:
            self._traj_state = Trajectory(self.v, self.nt, "state")
        return self._traj_state

    def traj_adj(self):
        if self._traj_adj is None:
            self._traj_adj = Trajectory(self.v, self.nt, "adjoint")
        return self._traj_adj

    def solve_state(self):
        """m^0 = mT, m^{j+1} = m^j(X) (src/CLAIRE.cpp:2152-2163)."""
        if self.m is not None:
            return self.m
        m = np.empty((self.nt + 1,) + self.shape, dtype=self.dtype)
        m[0] = self.mT
        tr = self.traj_state()
        for j in range(self.nt):
            m[j + 1] = tr.interp(m[j])
            if self.image_store is not None:
                m[j + 1] = self.image_store(m[j + 1])
        self.m = m
        self.counters["pdesolve"] += 1
        return m

    def gradm(self):
        if self._gradm is None:
            m = self.solve_state()
            self._gradm = [grad(m[j]) for j in range(self.nt + 1)]
        return self._gradm

    def divv(self):
        if self._divv is None:
            dv = div(self.v)
            dvx = self.traj_adj().interp(dv)
            self._divv = (dv, dvx)
        return self._divv

    # --- NCC distance (src/DistanceMeasureNCC.cpp, no mask, one component) -
    def _ncc_setup_scale(self) -> float:
        """DistanceMeasureNCC::SetupScale (src/DistanceMeasureNCC.cpp:78-166):
        scale = (1/2 hd sum (mT - mR)^2) / (1/2 - 1/2 <mT,mR>^2 / (|mT|^2 |mR|^2))."""
        mT = self.mT.astype(np.float64).ravel()
        mR = self.mR.astype(np.float64).ravel()
        w = np.ones_like(mT) if self.mask is None else self.mask.ravel()
        l2 = 0.5 * self.hd * float(np.sum(w * (mT - mR) ** 2))
        ncc = 0.5 - 0.5 * float(np.sum(w * mT * mR)) ** 2 / (float(np.sum(w * mT * mT)) * float(np.sum(w * mR * mR)))
        return l2 / ncc

    def _ncc_sums(self):
        m1 = self.solve_state()[self.nt].astype(np.float64).ravel()
        mR = self.mR.astype(np.float64).ravel()
        w = np.ones_like(m1) if self.mask is None else self.mask.ravel()
        return m1, mR, float(np.sum(w * m1 * m1)), float(np.sum(w * mR * mR)), float(np.sum(w * m1 * mR))

    def final_condition(self) -> np.ndarray:
        """Adjoint final condition lambda(1): mR - m1 for SL2
        (src/DistanceMeasureSL2.cpp:156-222); for NCC
        c1 mR - c2 m1, c1 = s I / (hd A R), c2 = s I^2 / (hd A^2 R), with
        A = <m1,m1>, R = <mR,mR>, I = <m1,mR> (src/DistanceMeasureNCC.cpp:251-366)."""
        m = self.solve_state()
        w = 1.0 if self.mask is None else self.mask
        if self.distance_type == "sl2":
            return (w * (self.mR - m[self.nt])).astype(self.dtype)
        m1, mR, A, Rr, I = self._ncc_sums()
        s, hd = self.ncc_scale, self.hd
        c1 = s * I / (hd * A * Rr)
        c2 = s * I * I / (hd * A * A * Rr)
        return (w * (c1 * mR - c2 * m1).reshape(self.shape)).astype(self.dtype)

    def inc_final_condition(self, mt1) -> np.ndarray:
        """Incremental adjoint final condition: -m~(1) for SL2
        (src/DistanceMeasureSL2.cpp:223-283); for NCC the linearisation of the
        adjoint final condition (src/DistanceMeasureNCC.cpp:368-510):
        (c1 - c2) mR + (c3 - c4) m1 - c5 m~ with c1 = s<mR,m~>/(hd A R),
        c2 = 2 s I <m1,m~>/(hd A^2 R), c3 = 4 s I^2 <m1,m~>/(hd A^3 R),
        c4 = 2 s I <mR,m~>/(hd A^2 R), c5 = s I^2/(hd A^2 R)."""
        w = 1.0 if self.mask is None else self.mask
        if self.distance_type == "sl2":
            return (-w * mt1).astype(self.dtype)
        m1, mR, A, Rr, I = self._ncc_sums()
        mt = np.asarray(mt1, np.float64).ravel()
        wf = np.ones_like(mt) if self.mask is None else self.mask.ravel()
        IM, RM = float(np.sum(wf * m1 * mt)), float(np.sum(wf * mR * mt))
        s, hd = self.ncc_scale, self.hd
        c1 = s * RM / (hd * A * Rr)
        c2 = 2.0 * s * I * IM / (hd * A * A * Rr)
        c3 = 4.0 * s * I * I * IM / (hd * A ** 3 * Rr)
        c4 = 2.0 * s * I * RM / (hd * A * A * Rr)
        c5 = s * I * I / (hd * A * A * Rr)
        out = (c1 - c2) * mR + (c3 - c4) * m1 - c5 * mt
        return (w * out.reshape(self.shape)).astype(self.dtype)

    # --- objective (src/CLAIRE.cpp:793-863) --------------------------------
    def distance(self) -> float:
        """D = 1/2 hd sum (mR - m1)^2 (src/DistanceMeasureSL2.cpp:93-155), or
        D = s (1/2 - 1/2 <m1,mR>^2 / (|m1|^2 |mR|^2)) for NCC
        (src/DistanceMeasureNCC.cpp:171-245)."""
        m = self.solve_state()
        if self.distance_type == "ncc":
            _, _, A, Rr, I = self._ncc_sums()
            return self.ncc_scale * (0.5 - 0.5 * I * I / (A * Rr))
        dr = self.mR.astype(np.float64) - m[self.nt].astype(np.float64)
        w = 1.0 if self.mask is None else self.mask
        return 0.5 * self.hd * float(np.sum(w * dr * dr))

    def div_penalty(self, v) -> float:
        """CLAIREDivReg::EvaluteRegularizationDIV (src/CLAIREDivReg.cpp:165-245):
        R_w = 1/2 hd beta_w (||grad div v||^2 + ||div v||^2), beta_w = -beta-div."""
        dv = div(v)
        gd = grad(dv)
        s = float(np.sum(gd.astype(np.float64) ** 2)) + float(np.sum(dv.astype(np.float64) ** 2))
        return 0.5 * self.hd * self.beta_w * s

    def objective(self, v) -> float:
        self.set_velocity(v)
        D = self.distance()
        R = 0.0 if not np.any(self.v) else self.reg.functional(self.v)
        if self.projection == "relaxedstokes" and np.any(self.v):
            # CLAIREDivReg::EvaluateObjective: J = D + R1(v) + R2(div v) (src/CLAIREDivReg.cpp:109-160)
            R += self.div_penalty(self.v)
        self.counters["obj"] += 1
        self.last_D, self.last_R = D, R
        return D + R

    # --- adjoint + gradient (src/CLAIRE.cpp:871-1042, 2181-2356, 2550-2722) -
    def _backward_sl(self, lam):
        """Shared RK2-in-time backward SL loop with trapezoid body force.

        Used by the adjoint (src/CLAIRE.cpp:2646-2709) and the GN incremental
        adjoint (src/CLAIRE.cpp:3940-3999).  Returns the body force (before
        the hd scaling) and the final lambda.
        """
        nt, ht = self.nt, self.ht
        tr = self.traj_adj()
        dv, dvx = self.divv()
        gm = self.gradm()
        b = np.zeros((3,) + self.shape, dtype=self.dtype)
        lam = lam.copy()
        for j in range(nt):
            w = 0.5 * ht if j == 0 else ht
            lx = tr.interp(lam)
            rhs0 = lx * dvx
            rhs1 = (lx + ht * rhs0) * dv
            g = gm[nt - j]
            for d in range(3):
                b[d] += (w * g[d] * lam).astype(self.dtype)
            lam = (lx + 0.5 * ht * (rhs0 + rhs1)).astype(self.dtype)
        g = gm[0]
        for d in range(3):
            b[d] += (0.5 * ht * g[d] * lam).astype(self.dtype)
        return b, lam

    def _project(self, b):
        if self.projection is None:
            return b
        return leray_projection(b, self.projection, self.reg.beta0)

    def body_force(self):
        lam1 = self.final_condition()
        b, lam0 = self._backward_sl(lam1)
        b = self._project(b)
        self.lambda0 = lam0
        return (self.hd * b).astype(self.dtype)

    def gradient(self, v) -> np.ndarray:
        self.set_velocity(v)
        b = self.body_force()
        self.counters["grad"] += 1
        if not np.any(self.v):
            return b
        return (self.reg.gradient(self.v) + b).astype(self.dtype)

    # --- GN Hessian matvec (src/CLAIRE.cpp:1218-1379, 3147-3290, 3849-4012) -
    def inc_state(self, vt) -> np.ndarray:
        nt, ht = self.nt, self.ht
        tr = self.traj_state()
        gm = self.gradm()
        vtx = tr.interp_vec(vt)
        mt = np.zeros(self.shape, dtype=self.dtype)
        for j in range(nt):
            mt = tr.interp(mt)
            gx = tr.interp_vec(gm[j])
            mt = (mt - 0.5 * ht * (gx[0] * vtx[0] + gx[1] * vtx[1] + gx[2] * vtx[2])).astype(self.dtype)
            g = gm[j + 1]
            mt = (mt - 0.5 * ht * (g[0] * vt[0] + g[1] * vt[1] + g[2] * vt[2])).astype(self.dtype)
        return mt

    def inc_body_force(self, mt1) -> np.ndarray:
        bt, _ = self._backward_sl(self.inc_final_condition(mt1))
        bt = self._project(bt)
        return (self.hd * bt).astype(self.dtype)

    def hessian_matvec(self, vt) -> np.ndarray:
        vt = np.asarray(vt, dtype=self.dtype)
        mt1 = self.inc_state(vt)
        bt = self.inc_body_force(mt1)
        self.counters["hessmatvec"] += 1
        return (self.reg.hessian_matvec(vt) + bt).astype(self.dtype)

    def precond(self, x) -> np.ndarray:
        """P x = (beta A)^-1 x (src/Preconditioner.cpp:549-580)."""
        self.counters["pcmatvec"] += 1
        return self.reg.apply_inverse(np.asarray(x, dtype=self.dtype)).astype(self.dtype)

    def hessian_sym(self, vt, scale: bool = True) -> np.ndarray:
        """Symmetrically preconditioned GN Hessian, CLAIRE::PrecondHessMatVecSym
        (src/CLAIRE.cpp:1455-1532): hd vt + P^1/2 b~[P^1/2 vt] with
        P^1/2 = (beta A)^-1/2 (ApplyInverse with applysqrt) and b~ the
        incremental body force (hd and the model's projection included).
        scale=False divides the result by hd (CLAIRE::HessianMatVec with
        scale = false, src/CLAIRE.cpp:1279-1285), as the two-level
        preconditioner's coarse operator does (src/Preconditioner.cpp:963-978)."""
        vt = np.asarray(vt, dtype=self.dtype)
        t = self.reg.apply_inverse(vt, applysqrt=True).astype(self.dtype)
        bt = self.inc_body_force(self.inc_state(t))
        out = (self.hd * vt + self.reg.apply_inverse(bt, applysqrt=True)).astype(self.dtype)
        self.counters["hessmatvec"] += 1
        return out if scale else (out / self.hd).astype(self.dtype)


# --------------------------------------------------------------------------
# Krylov + Gauss-Newton loop
# --------------------------------------------------------------------------


def dot(a, b) -> float:
    return float(np.dot(a.reshape(-1).astype(np.float64), b.reshape(-1).astype(np.float64)))


def pcg(matvec, precond, b, rtol, atol=1e-16, maxit=49, dtol=1e6):
    """Preconditioned CG with the unpreconditioned residual norm.

    Restates PETSc KSPCG as configured at src/Optimizer.cpp:296-356: zero
    initial guess, KSP_NORM_UNPRECONDITIONED, converged when
    ||r|| <= max(rtol*||b||, atol), at most maxit iterations, stop on
    non-positive curvature.  Returns (x, iterations, reason).
    """
    x = np.zeros_like(b)
    r = b.copy()
    rnorm0 = math.sqrt(dot(r, r))
    tol = max(rtol * rnorm0, atol)
    if rnorm0 <= tol:
        return x, 0, "converged"
    z = precond(r)
    p = z.copy()
    rz = dot(r, z)
    it = 0
    reason = "maxit"
    while it < maxit:
        q = matvec(p)
        pq = dot(p, q)
        if pq <= 0.0 or not math.isfinite(pq):
            reason = "indefinite"
            break
        alpha = rz / pq
        x = (x + alpha * p).astype(b.dtype)
        r = (r - alpha * q).astype(b.dtype)
        it += 1
        rnorm = math.sqrt(dot(r, r))
        if rnorm <= tol:
            reason = "converged"
            break
        if rnorm > dtol * rnorm0:
            reason = "diverged"
            break
        z = precond(r)
        rz_new = dot(r, z)
        beta = rz_new / rz
        rz = rz_new
        p = (z + beta * p).astype(b.dtype)
    return x, it, reason


def forcing_tolerance(gnorm, g0norm, fseq="slfs"):
    """src/KrylovInterface.cpp:134-165: SLFS min(1/2, sqrt(g/g0)), QDFS min(1/2, g/g0)."""
    r = gnorm / g0norm
    if fseq == "qdfs":
        return max(1e-16, min(0.5, r))
    return max(1e-16, min(0.5, math.sqrt(r)))


@dataclasses.dataclass
class GNOptions:
    maxit: int = 50          # -maxit (src/RegOpt.cpp:1155-1160)
    gttol: float = 5e-2      # -opttol
    gatol: float = 1e-6
    krylov_maxit: int = 50   # -krylovmaxit; PCG runs maxit-1 (src/Optimizer.cpp:304-305)
    fseq: str = "slfs"
    ls_sigma: float = 1e-4
    ls_max_trials: int = 30
    min_step: float = 2.0 ** -10
    precond: str = "invreg"   # -precond invreg | 2level
    pcgridscale: float = 2.0  # -gridscale (src/RegOpt.cpp:1124)
    pctolscale: float = 1e-1  # -pctolscale (src/RegOpt.cpp:1121)


def gauss_newton(prob: Problem, opts: GNOptions = GNOptions(), v0=None, log=None, g0=None, krylov_g0=None,
                 miniter=0):
    """GN-Krylov with Armijo backtracking and CLAIRE's gradient stopping test.

    ``g0`` / ``krylov_g0`` fix the reference gradient norms (continuation
    levels keep those of the first initialisation); the step and gradient
    tests apply from iteration ``miniter`` on (src/TaoInterface.cpp:438-470).
    Returns a dict with the velocity, iteration counts and monitor values.
    """
    v = np.zeros((3,) + prob.shape, dtype=prob.dtype) if v0 is None else np.asarray(v0, prob.dtype).copy()
    if g0 is None and np.any(v):
        # InitializeOptimization (src/CLAIRE.cpp:227-357): D0, J0 and ||g0|| at
        # the zero velocity, then the loop starts from the initial guess
        z = np.zeros_like(v)
        prob.objective(z)
        D0 = prob.last_D
        gz = prob.gradient(z)
        g0 = math.sqrt(dot(gz, gz))
        g0 = g0 if g0 > 0 else 1.0
        J = prob.objective(v)
    else:
        J = prob.objective(v)
        D0 = prob.last_D
    g = prob.gradient(v)
    gnorm = math.sqrt(dot(g, g))
    if g0 is None:
        g0 = gnorm if gnorm > 0 else 1.0
    it = 0
    step = 1.0
    pcg_iters = []
    reason = None
    while True:
        if not (math.isfinite(J) and math.isfinite(gnorm)):
            reason = "nan"
            break
        if it >= miniter and step < opts.min_step:
            reason = "steptol"
            break
        if it >= miniter and gnorm < opts.gttol * g0:
            reason = "gttol"
            break
        if it >= miniter and gnorm < opts.gatol:
            reason = "gatol"
            break
        if it > opts.maxit - 1:
            reason = "maxit"
            break
        if krylov_g0 is None:
            krylov_g0 = gnorm
        rtol = forcing_tolerance(gnorm, krylov_g0, opts.fseq)
        gls = g  # the gradient the descent test and the line search see
        if opts.precond == "2level":
            # PreKrylovSolve applies P^1/2 to the right-hand side in place
            # (src/CLAIREBase.cpp:936-952); that vector is the optimiser's
            # gradient, so the line search below sees P^1/2 g.  The operator
            # is PrecondHessMatVecSym, the preconditioner the two-level one
            # (set up once per iteration, src/TaoInterface.cpp:546), and
            # PostKrylovSolve maps the solution back (:958-972).
            gls = prob.reg.apply_inverse(g, applysqrt=True).astype(prob.dtype)
            coarse = two_level_setup(prob, opts.pcgridscale)
            inner = max(1e-16, min(0.5, opts.pctolscale * rtol))
            xh, kit, _ = pcg(prob.hessian_sym, lambda r: two_level_apply(coarse, r, inner),
                             (-gls).astype(prob.dtype), rtol, maxit=max(0, opts.krylov_maxit - 1))
            d = prob.reg.apply_inverse(xh, applysqrt=True).astype(prob.dtype)
        else:
            d, kit, _ = pcg(prob.hessian_matvec, prob.precond, (-g).astype(prob.dtype), rtol,
                            maxit=max(0, opts.krylov_maxit - 1))
        pcg_iters.append(kit)
        gd = dot(gls, d)
        if not (gd < 0.0):
            d = (-gls).astype(prob.dtype)
            gd = -dot(gls, gls)
        alpha = 1.0
        accepted = False
        for _ in range(opts.ls_max_trials):
            vt = (v + alpha * d).astype(prob.dtype)
            Jt = prob.objective(vt)
            if Jt <= J + opts.ls_sigma * alpha * gd:
                accepted = True
                break
            alpha *= 0.5
        if not accepted:
            reason = "lsfail"
            break
        v = vt
        J = Jt
        step = alpha
        g = prob.gradient(v)
        gnorm = math.sqrt(dot(g, g))
        it += 1
        if log is not None:
            log(it, J, gnorm / g0, kit, alpha)
    m = prob.solve_state() if prob.v is not None and np.array_equal(prob.v, v) else None
    if m is None:
        prob.set_velocity(v)
        m = prob.solve_state()
    return dict(v=v, J=J, D=prob.last_D if hasattr(prob, "last_D") else None, D0=D0,
                gnorm=gnorm, g0=g0, iters=it, pcg_iters=pcg_iters, reason=reason,
                m1=m[prob.nt].copy(), krylov_g0=krylov_g0)


def beta_continuation(prob: Problem, beta_star: float, opts: GNOptions = GNOptions(), presolve_gttol=1e-1,
                      log=None):
    """Regularisation-parameter continuation (CLAIREInterface::
    RunSolverRegParaContReduction, src/CLAIREInterface.cpp:1300-1376): ||g0||
    at beta = 1 and v = 0; levels beta = 1, 1/10, ... while beta > beta*, each
    warm-started and solved to presolve_gttol with at least one iteration;
    then beta* to opts.gttol.  Returns the last level's result with the list of
    per-level GN iteration counts."""
    import dataclasses
    beta = 1.0
    prob.reg = dataclasses.replace(prob.reg, beta0=beta)
    prob.set_velocity(np.zeros((3,) + prob.shape, dtype=prob.dtype))
    g = prob.gradient(np.zeros((3,) + prob.shape, dtype=prob.dtype))
    g0 = math.sqrt(dot(g, g))
    g0 = g0 if g0 > 0 else 1.0
    v = None
    kg0 = None
    levels = []
    pre = dataclasses.replace(opts, gttol=presolve_gttol)
    while beta > beta_star:
        prob.reg = dataclasses.replace(prob.reg, beta0=beta)
        res = gauss_newton(prob, pre, v0=v, log=log, g0=g0, krylov_g0=kg0, miniter=1)
        v, kg0 = res["v"], res["krylov_g0"]
        levels.append(res["iters"])
        beta /= 10.0
    prob.reg = dataclasses.replace(prob.reg, beta0=beta_star)
    res = gauss_newton(prob, opts, v0=v, log=log, g0=g0, krylov_g0=kg0, miniter=1)
    levels.append(res["iters"])
    res["levels"] = levels
    return res


def grid_transfer(f: np.ndarray, nt: int) -> np.ndarray:
    """Restriction / prolongation of a cubic field to nt^3 points
    (Preprocessing::Restrict / Prolong, src/Preprocessing.cpp:765-917,
    1636-1786, index map of ComputeGridChangeIndices :918-1057): the
    coefficients of the wavenumbers |w| < min(ns, nt)/2 on every axis, scaled
    by 1/ns^3, transformed back unnormalised on the target grid."""
    f = np.asarray(f, np.float64)
    ns = f.shape[0]
    if ns == nt:
        return f.copy()
    nc = min(ns, nt)
    w = np.arange(-((nc + 1) // 2 - 1), (nc + 1) // 2)
    src, dst = w % ns, w % nt
    fh = np.fft.fftn(f)
    out = np.zeros((nt, nt, nt), dtype=complex)
    out[np.ix_(dst, dst, dst)] = fh[np.ix_(src, src, src)] / float(ns) ** 3
    return np.real(np.fft.ifftn(out)) * float(nt) ** 3


def rect_freq_filter(f: np.ndarray, pct: float, lowpass: bool = True) -> np.ndarray:
    """Preprocessing::ApplyRectFreqFilter (src/Preprocessing.cpp:1812-1913):
    keep (lowpass) or drop (highpass) the coefficients whose index w on every
    axis of the r2c spectrum satisfies w < pct (N/2 - 1) or w > N - pct N/2."""
    f = np.asarray(f, np.float64)
    if pct == 1.0:
        return f.copy() if lowpass else np.zeros_like(f)
    shape = f.shape
    fh = np.fft.rfftn(f)
    inside = np.ones(fh.shape, dtype=bool)
    for ax, n in enumerate(shape):
        w = np.arange(fh.shape[ax])
        keep = (w < pct * (n / 2.0 - 1.0)) | (w > n - pct * (n / 2.0))
        sh = [1, 1, 1]
        sh[ax] = -1
        inside &= keep.reshape(sh)
    fh = np.where(inside if lowpass else ~inside, fh, 0.0)
    return np.fft.irfftn(fh, s=shape, axes=(0, 1, 2))


def two_level_setup(prob: Problem, gridscale: float = 2.0) -> Problem:
    """Preconditioner::SetupCoarseGrid + ApplyRestriction
    (src/Preconditioner.cpp:353-499, 676-831): a problem on ceil(N/gridscale)
    points per axis whose velocity, state levels (all nt+1, not re-solved),
    images and mask are the restrictions of the fine problem's at its current
    velocity; its trajectories follow from the restricted velocity
    (CLAIRE::SetStateVariable / SetAdjointVariable)."""
    m = prob.solve_state()
    nf = prob.shape[0]
    nc = int(math.ceil(nf / gridscale))
    cp = Problem(grid_transfer(prob.mR, nc), grid_transfer(prob.mT, nc), prob.nt, prob.reg,
                 projection=prob.projection, mask=None if prob.mask is None else grid_transfer(prob.mask, nc))
    cp.beta_w = prob.beta_w
    cp.set_velocity(np.stack([grid_transfer(prob.v[k], nc) for k in range(3)]))
    cp.m = np.stack([grid_transfer(m[j], nc) for j in range(prob.nt + 1)])
    cp.fine_n = nf
    return cp


def two_level_apply(coarse: Problem, r: np.ndarray, rtol: float, maxit: int = 1000):
    """Preconditioner::Apply2LevelPrecond (src/Preconditioner.cpp:584-673):
    low-pass filter, restrict, solve with the coarse operator (KSPCG, no
    preconditioner, zero guess, rtol = pctolscale * the outer forcing value,
    atol 1e-16, at most 1000 iterations: src/KrylovInterface.cpp:430-521,
    src/Preconditioner.cpp:842-945), prolong, low-pass filter, and add the
    high-pass part of the input."""
    nf = coarse.fine_n
    nc = coarse.shape[0]
    pct = nc / nf
    low = np.stack([rect_freq_filter(r[k], pct) for k in range(3)])
    rc = np.stack([grid_transfer(low[k], nc) for k in range(3)])
    y, its, _ = pcg(lambda x: coarse.hessian_sym(x, scale=False), lambda x: x, rc, rtol, atol=1e-16,
                    maxit=maxit)
    coarse.inner_iters = getattr(coarse, "inner_iters", 0) + its
    yp = np.stack([grid_transfer(y[k], nf) for k in range(3)])
    out = np.stack([rect_freq_filter(yp[k], pct) + rect_freq_filter(r[k], pct, lowpass=False) for k in range(3)])
    return out.astype(r.dtype)


def grid_levels(n: int):
    """Grid sizes of the continuation levels (RegOpt::SetupGridCont,
    src/RegOpt.cpp:1844-1930): ceil(log2 n) - 3 levels, each half the next
    (rounded up), the finest n."""
    nlev = max(1, int(math.ceil(math.log2(n))) - 3)
    sizes = [n]
    for _ in range(nlev - 1):
        sizes.insert(0, int(math.ceil(sizes[0] / 2.0)))
    return sizes


def grid_continuation(mR, mT, nt: int, reg: Regularization, opts: GNOptions = GNOptions(),
                      supported=lambda n: True, **problem_kw):
    """CLAIREInterface::RunSolverGridCont (src/CLAIREInterface.cpp:1510-1705):
    images restricted from the finest grid to every level; v = 0 on the
    coarsest level, prolonged to the next; the gradient tolerance is 10x
    looser below the finest level when it is under 0.01; each level's
    InitializeOptimization sets ||g0|| at v = 0, while the Krylov reference
    norm is the first level's (set once per run, src/KrylovInterface.cpp:125-134).
    Levels whose size `supported` rejects are skipped and the velocity goes
    on from the last solved level."""
    import dataclasses
    sizes = grid_levels(mR.shape[0])
    v, vsize, kg0, res, levels = None, None, None, None, []
    for l, nl in enumerate(sizes):
        if not supported(nl):
            continue
        last = l == len(sizes) - 1
        prob = Problem(grid_transfer(mR, nl), grid_transfer(mT, nl), nt, reg, **problem_kw)
        v0 = None if v is None else np.stack([grid_transfer(v[k], nl) for k in range(3)])
        tol = opts.gttol * 10.0 if (opts.gttol < 0.01 and not last) else opts.gttol
        res = gauss_newton(prob, dataclasses.replace(opts, gttol=tol), v0=v0, krylov_g0=kg0)
        v, vsize, kg0 = res["v"], nl, res["krylov_g0"]
        levels.append((nl, res["iters"]))
    res["levels"] = levels
    res["prob"] = prob
    return res


SCALE_SIGMAS = (32.0, 16.0, 8.0, 4.0, 2.0, 1.0)  # src/RegOpt.cpp:1241-1246


def scale_continuation(mR, mT, nt: int, reg: Regularization, opts: GNOptions = GNOptions(), **problem_kw):
    """CLAIREInterface::RunSolverScaleCont (src/CLAIREInterface.cpp:1387-1505):
    for sigma = 32, 16, ..., 1 grid cells (skipped when n/2 <= sigma) the
    original images are smoothed with sigma, ||g0|| is set at v = 0 and the GN
    solve warm-starts from the previous level's velocity (Krylov reference
    norm from the first level)."""
    n = mR.shape[0]
    v, kg0, res, levels = None, None, None, []
    for sig in SCALE_SIGMAS:
        if n / 2.0 <= sig:
            continue
        prob = Problem(gaussian_smooth(np.asarray(mR, np.float64), sig),
                       gaussian_smooth(np.asarray(mT, np.float64), sig), nt, reg, **problem_kw)
        res = gauss_newton(prob, opts, v0=v, krylov_g0=kg0)
        v, kg0 = res["v"], res["krylov_g0"]
        levels.append((sig, res["iters"]))
    res["levels"] = levels
    res["prob"] = prob
    return res


def train_search(mR, mT, nt: int, reg: Regularization, opts: GNOptions = GNOptions(), strategy="binary",
                 jbound=0.25, betainit=1.0, **problem_kw):
    """Regularisation-parameter search (CLAIREInterface::
    RunSolverRegParaContBinarySearch, src/CLAIREInterface.cpp:955-1186, and
    RunSolverRegParaContReductSearch, :1192-1285): ||g0|| at beta = betainit
    and v = 0; every solve warm-starts from the last solution whose
    det(grad y) stays inside the bound (CheckBounds, src/CLAIREBase.cpp:
    1386-1445), with tests from iteration 1; beta scaled by 1/10 per step (at
    most 10 steps, not below 1e-4 for H1 types, 1e-7 for H2 types); the
    binary search then bisects [beta*/10, beta*] until |dbeta| < 1e-2 beta*.
    A solve that ended on a line-search failure or NaN counts as not
    converged (Optimizer::GetSolutionStatus, src/Optimizer.cpp:557-580).
    Returns beta*, its solution, and the list of (beta, converged, breach)."""
    import dataclasses
    scale, dscale, maxsteps, maxsolves = 1e-1, 1e-2, 10, 64
    betamin = 1e-4 if reg.norm in ("h1", "h1s") else (1e-7 if reg.norm in ("h2", "h2s") else 1e-9)
    prob = Problem(mR, mT, nt, dataclasses.replace(reg, beta0=betainit), **problem_kw)
    z = np.zeros((3,) + prob.shape, dtype=prob.dtype)
    prob.objective(z)
    gz = prob.gradient(z)
    g0 = math.sqrt(dot(gz, gz))
    g0 = g0 if g0 > 0 else 1.0
    state = {"best": z, "kg0": None}
    log = []

    def solve(beta):
        prob.reg = dataclasses.replace(reg, beta0=beta)
        res = gauss_newton(prob, opts, v0=state["best"], g0=g0, krylov_g0=state["kg0"], miniter=1)
        state["kg0"] = res["krylov_g0"]
        converged = res["reason"] not in ("lsfail", "nan")
        _, (mn, _, mx) = det_def_grad(res["v"], nt)
        breach = mn <= jbound or 1.0 / mx <= jbound
        log.append((beta, converged, breach))
        return res, converged, breach

    beta = betastar = betainit
    level = 0
    while level < maxsteps and len(log) < maxsolves:
        res, converged, breach = solve(beta)
        if strategy == "binary" and not converged and level > 0:
            break
        if breach:
            if strategy == "reduce" or level > 0:
                break
            beta /= scale
            level = -1
        else:
            betastar = beta
            state["best"] = res["v"]
            beta *= scale
        if beta < betamin:
            break
        level += 1
    if strategy == "binary":
        betahat = scale * betastar
        dbeta = (betastar - betahat) / 2.0
        beta = betastar - dbeta
        dbetamin = dscale * betastar
        while len(log) < maxsolves:
            res, converged, breach = solve(beta)
            if converged and not breach:
                betastar = beta
                state["best"] = res["v"]
            else:
                betahat = beta
            dbeta = (betastar - betahat) / 2.0
            beta = betastar - dbeta
            if abs(dbeta) < dbetamin:
                break
    prob.reg = dataclasses.replace(reg, beta0=betastar)
    prob.set_velocity(state["best"])
    m1 = prob.solve_state()[nt]
    return dict(beta=betastar, v=state["best"], log=log, m1=m1, prob=prob)


def monitored_run(mR, mT, nt: int, reg: Regularization, opts: GNOptions = GNOptions(), jbound=0.25,
                  **problem_kw):
    """CLAIREInterface::RunSolver with -monitordefgrad (src/CLAIREInterface.cpp:
    790-862): ||g0|| once at the first beta; solve from the initial guess
    (zero); while det(grad y) breaches the bound (at most 10 times) beta moves
    halfway toward beta* = 10 beta and the solve restarts from the guess.
    Status 0: first solution kept the bound, 1: a raised beta did, 2: none
    did (beta reported as beta*)."""
    import dataclasses
    beta = reg.beta0
    betastar = beta / 1e-1
    prob = Problem(mR, mT, nt, reg, **problem_kw)
    z = np.zeros((3,) + prob.shape, dtype=prob.dtype)
    prob.objective(z)
    gz = prob.gradient(z)
    g0 = math.sqrt(dot(gz, gz))
    g0 = g0 if g0 > 0 else 1.0
    level, breach, kg0 = 0, True, None
    while breach and level < 10:
        res = gauss_newton(prob, opts, v0=z, g0=g0, krylov_g0=kg0, miniter=1)
        kg0 = res["krylov_g0"]
        _, (mn, mean, mx) = det_def_grad(res["v"], nt)
        breach = mn <= jbound or 1.0 / mx <= jbound
        if breach:
            beta += (betastar - beta) / 2.0
            prob.reg = dataclasses.replace(prob.reg, beta0=beta)
            level += 1
    status = 0 if level == 0 else (2 if breach else 1)
    res["beta"] = betastar if status == 2 else beta
    res["status"] = status
    res["det"] = (mn, mean, mx)
    return res


def relative_mismatch(mR, m1, mT) -> float:
    """||mR - m1|| / ||mR - mT|| (src/CLAIRE.cpp:4232-4262)."""
    a = np.linalg.norm((mR - m1).astype(np.float64).ravel())
    b = np.linalg.norm((mR - mT).astype(np.float64).ravel())
    return float(a / b) if b > 0 else float(a)


# --------------------------------------------------------------------------
# synthetic problems
# --------------------------------------------------------------------------


def normalize(x: np.ndarray) -> np.ndarray:
    """Normalize for one component (src/CLAIREUtils.cpp:492-525): negative
    values are set to zero (the shift is then zero), then x <- (x - xmin) / xmax
    with xmin / xmax taken before the change (the division is by xmax, not by
    the range, as written)."""
    x = np.asarray(x, np.float64)
    xmin, xmax = float(x.min()), float(x.max())
    if xmin < 0.0:
        x = np.where(x < 0.0, 0.0, x)
        xmin = 0.0
    return (x - xmin) / xmax


def rescale(x: np.ndarray, xminout=0.0, xmaxout=1.0) -> np.ndarray:
    """Single-component Rescale (src/CLAIREUtils.cpp:691-725): shift only when
    min < -1e-6, then scale by xmaxout/(max-min)."""
    x = x.copy()
    xmin = float(x.min())
    xmax = float(x.max())
    xshift = -xmin
    if xshift > 1e-6:
        x += x.dtype.type(xshift)
    xscale = xmaxout / (xmax - xmin) if abs(xmax - xmin) > 1e-6 else 1.0
    return (x * x.dtype.type(xscale)).astype(x.dtype)


def template_sin2(shape, dtype=np.float64):
    """mT = (sin^2 x1 + sin^2 x2 + sin^2 x3)/3 (src/CLAIREBase.cpp:1113-1116)."""
    x1, x2, x3 = grid_coords(shape, np.float64)
    return ((np.sin(x1) ** 2 + np.sin(x2) ** 2 + np.sin(x3) ** 2) / 3.0).astype(dtype)


def velocity_trig(shape, v0=0.5, reference_case=False, dtype=np.float64):
    """Trig velocity.  ``reference_case`` gives CLAIRE's -synthetic 0 field
    v0*(sin x3 cos x2 sin x2, sin x1 cos x3 sin x3, sin x2 cos x1 sin x1)
    (src/CLAIREBase.cpp:1136-1139); otherwise v0*(sin x3 cos x2, sin x1 cos x3,
    sin x2 cos x1)."""
    x1, x2, x3 = grid_coords(shape, np.float64)
    if reference_case:
        v = np.stack([np.sin(x3) * np.cos(x2) * np.sin(x2),
                      np.sin(x1) * np.cos(x3) * np.sin(x3),
                      np.sin(x2) * np.cos(x1) * np.sin(x1)])
    else:
        v = np.stack([np.sin(x3) * np.cos(x2), np.sin(x1) * np.cos(x3), np.sin(x2) * np.cos(x1)])
    return (v0 * v).astype(dtype)


def forward_transport(mT, v, nt):
    """SolveForwardProblem: m1 = SL transport of m0 along v (src/CLAIRE.cpp:2116-2175)."""
    tr = Trajectory(np.asarray(v), nt, "state")
    m = np.asarray(mT).copy()
    for _ in range(nt):
        m = tr.interp(m)
    return m


def det_def_grad(v, nt, inverse=False):
    """det(grad y) by the SL scheme of DeformationFields::ComputeDetDefGradSL
    (src/DeformationFields.cpp:636-739, initial condition 1 at :336): along the
    state characteristic, jX = J(X); rhs0 = a jX divv(X); rhs1 = a (jX + ht
    rhs0) divv; J = jX + ht/2 (rhs0 + rhs1), a = -1 for det(grad(inv(y))).
    Returns (J, (min, mean, max)) as the reference's monitor values (:367-375)."""
    v = np.asarray(v)
    shape = v.shape[1:]
    ht = 1.0 / nt
    a = -1.0 if inverse else 1.0
    tr = Trajectory(v, nt, "state")
    dv = div(v)
    dvx = tr.interp(dv)
    jac = np.ones(shape, dtype=v.dtype)
    for _ in range(nt):
        jx = tr.interp(jac)
        rhs0 = a * jx * dvx
        rhs1 = a * (jx + ht * rhs0) * dv
        jac = jx + 0.5 * ht * (rhs0 + rhs1)
    return jac, (float(jac.min()), float(jac.mean()), float(jac.max()))


def deformation_map(v, nt, inverse=False):
    """DeformationFields::ComputeDeformationMapSLRK2 (src/DeformationFields.cpp:
    1472-1585): y = x on the grid (ComputeRegularGrid), then per time step
    yt = y - ht v(y), y <- y - ht/2 (v(y) + v(yt)), v evaluated at the points by
    tricubic interpolation; ht < 0 for the inverse map.  Returns y (3, ...) in
    physical coordinates."""
    v = np.asarray(v, np.float64)
    shape = v.shape[1:]
    ht = (-1.0 if inverse else 1.0) / nt
    c = np.array([n / (2.0 * math.pi) for n in shape]).reshape(3, 1, 1, 1)  # grid units per length
    grid = index_grid(shape)
    u = np.zeros((3,) + shape)
    for _ in range(nt):
        q = grid + u
        vy = np.stack([interp3(v[k], q) for k in range(3)])
        ut = u - ht * c * vy
        u = u - 0.5 * ht * c * vy
        q = grid + ut
        vyt = np.stack([interp3(v[k], q) for k in range(3)])
        u = u - 0.5 * ht * c * vyt
    return (grid + u) / c


def def_grad(v, nt):
    """DeformationFields::ComputeDefGrad / ComputeDefGradSL
    (src/DeformationFields.cpp:821-1117), tensors component-major (F_ab at
    index 3a + b): F^0 = I, gv_ka = d_a v_k, and per step with FX = F(X),
    gvX = gv(X), rhs_ab = sum_k gvX_ka FX_kb,
    F_ab = FX_ab + ht/2 (rhs_ab + gvX_ab + ht sum_k gv_ka rhs_kb), as written
    there.  Returns (F, det F)."""
    v = np.asarray(v, np.float64)
    ht = 1.0 / nt
    tr = Trajectory(v, nt, "state")
    gv = np.concatenate([grad(v[k]) for k in range(3)])
    gvx = np.stack([tr.interp(gv[c]) for c in range(9)])
    F = np.zeros((9,) + v.shape[1:])
    F[0] = F[4] = F[8] = 1.0
    for _ in range(nt):
        FX = np.stack([tr.interp(F[c]) for c in range(9)])
        rhs = np.stack([sum(gvx[3 * k + a] * FX[3 * k + b] for k in range(3)) for a in range(3) for b in range(3)])
        F = np.stack([FX[3 * a + b] + 0.5 * ht * (rhs[3 * a + b] + gvx[3 * a + b]
                                                   + ht * sum(gv[3 * k + a] * rhs[3 * k + b] for k in range(3)))
                      for a in range(3) for b in range(3)])
    det = (F[0] * F[4] * F[8] + F[1] * F[5] * F[6] + F[2] * F[3] * F[7]
           - F[2] * F[4] * F[6] - F[1] * F[3] * F[8] - F[0] * F[5] * F[7])
    return F, det


def det_def_grad_via_disp(v, nt):
    """DeformationFields::ComputeDetDefGradViaDispField (src/DeformationFields.cpp:
    745-815): gradient of the SL displacement field and det(I - grad u) with
    the reference's signs (the products of three off-diagonal entries enter
    with +)."""
    u = displacement_field(v, nt)
    g = np.concatenate([grad(u[k]) for k in range(3)])
    return ((1 - g[0]) * (1 - g[4]) * (1 - g[8]) + g[1] * g[5] * g[6] + g[2] * g[3] * g[7]
            - g[2] * (1 - g[4]) * g[6] - g[1] * g[3] * (1 - g[8]) - (1 - g[0]) * g[5] * g[7])


def displacement_field(v, nt):
    """DeformationFields::ComputeDisplacementFieldSL (src/DeformationFields.cpp:
    1816-1909): with the state characteristic X, u^0 = 0 and
    u^{j+1} = u^j(X) + ht/2 (v(X) + v)."""
    v = np.asarray(v, np.float64)
    ht = 1.0 / nt
    tr = Trajectory(v, nt, "state")
    vx = tr.interp_vec(v)
    u = np.zeros_like(v)
    for _ in range(nt):
        u = tr.interp_vec(u) + 0.5 * ht * (vx + v)
    return u


def gaussian_smooth(f: np.ndarray, sigma_cells=1.0) -> np.ndarray:
    """Spectral Gaussian smoothing (src/Preprocessing.cpp:1956-2056): multiply by
    exp(-1/2 sum_i k_i^2 (sigma_i h_i)^2), Nyquist index kept as +N/2."""
    shape = f.shape
    k = spectral_k(shape, nyquist_zero=False)
    c = [(sigma_cells * TWO_PI / n) ** 2 for n in shape]
    sik = np.exp(-0.5 * (k[0] ** 2 * c[0] + k[1] ** 2 * c[1] + k[2] ** 2 * c[2]))
    return _irfft(sik * _rfft(f), shape, f.dtype)


def problem_seed(config_index: int, problem_index: int) -> int:
    return 20261203 + 1000 * config_index + problem_index


def template_ellipsoids(shape, rng, count=40, dtype=np.float64):
    """Sum of ``count`` random Gaussian ellipsoids, smoothed (sigma = 1 cell) and
    clipped to [0, 1].  Centres U[0,2pi)^3, semi-axes U[0.1,0.5] rad, uniform
    random rotation, intensity U[0.2,1], periodic minimum-image distance."""
    x = grid_coords(shape, np.float64)
    out = np.zeros(shape, dtype=np.float64)
    for _ in range(count):
        c = rng.uniform(0.0, TWO_PI, size=3)
        sig = rng.uniform(0.1, 0.5, size=3)
        amp = rng.uniform(0.2, 1.0)
        # uniform random rotation from a normalised Gaussian quaternion
        qv = rng.normal(size=4)
        qv /= np.linalg.norm(qv)
        a, b, cq, d = qv
        rot = np.array([
            [a * a + b * b - cq * cq - d * d, 2 * (b * cq - a * d), 2 * (b * d + a * cq)],
            [2 * (b * cq + a * d), a * a - b * b + cq * cq - d * d, 2 * (cq * d - a * b)],
            [2 * (b * d - a * cq), 2 * (cq * d + a * b), a * a - b * b - cq * cq + d * d],
        ])
        dx = [np.mod(x[i] - c[i] + math.pi, TWO_PI) - math.pi for i in range(3)]
        acc = 0.0
        for r in range(3):
            u = rot[0, r] * dx[0] + rot[1, r] * dx[1] + rot[2, r] * dx[2]
            acc = acc + (u / sig[r]) ** 2
        out += amp * np.exp(-0.5 * acc)
    out = gaussian_smooth(out, 1.0)
    return np.clip(out, 0.0, 1.0).astype(dtype)


def velocity_random(shape, rng, kmax=6, amp=0.3, dtype=np.float64, rms=0.3):
    """Random smooth periodic velocity: per component, complex Fourier
    coefficients N(0, amp)/|k|^2 on 1 <= |k| <= kmax, Hermitian through the
    real inverse FFT, Nyquist zero; coefficient c gives c*e^{ik.x} + c.c.

    The ~520 modes per component sum to an RMS of ~1.4 (displacements of up
    to a fifth of the domain per unit time, a folding map); the field is
    scaled to the given RMS over grid and components (``rms=None`` keeps the
    raw sum).  The field is band-limited, so the RMS and the scale factor do
    not depend on the grid size."""
    n1, n2, n3 = shape
    # Nyquist indices keep their magnitude n/2 > kmax, so no Nyquist mode
    # (a +-1 checkerboard on the grid) enters the field
    k1, k2, k3 = spectral_k(shape, nyquist_zero=False)
    kk = np.sqrt(k1 * k1 + k2 * k2 + k3 * k3)
    mask = (kk >= 1.0) & (kk <= kmax)
    out = []
    for _ in range(3):
        c = rng.normal(0.0, amp, size=(n1, n2, n3 // 2 + 1)) + 1j * rng.normal(0.0, amp, size=(n1, n2, n3 // 2 + 1))
        c = np.where(mask, c / np.where(kk > 0, kk * kk, 1.0), 0.0)
        # the real inverse transform completes the half spectrum Hermitian-wise
        out.append(np.fft.irfftn(c * (n1 * n2 * n3), s=shape, axes=(0, 1, 2)))
    v = np.stack(out)
    if rms is not None:
        v *= rms / np.sqrt(np.mean(v * v))
    return v.astype(dtype)


def synthetic_c1(n=64, dtype=np.float64, nt=4):
    """Config 1: sin^2 template, trig velocity v* (no extra sin factor), mR =
    transport(mT, v*), both rescaled to [0,1] (src/CLAIREBase.cpp:1209-1225)."""
    shape = (n, n, n)
    mT = rescale(template_sin2(shape, dtype))
    vstar = velocity_trig(shape, 0.5, reference_case=False, dtype=dtype)
    mR = rescale(forward_transport(mT, vstar, nt).astype(dtype))
    return mR, mT, vstar


def synthetic_reference(n=32, dtype=np.float64, nt=4):
    """CLAIRE's own -synthetic 0 problem (src/CLAIREBase.cpp:1026-1250)."""
    shape = (n, n, n)
    mT = rescale(template_sin2(shape, dtype))
    v = velocity_trig(shape, 0.5, reference_case=True, dtype=dtype)
    mR = rescale(forward_transport(mT, v, nt).astype(dtype))
    return mR, mT, v


def synthetic_ellipsoids(n=128, config_index=1, problem_index=0, nt=8, dtype=np.float64):
    """Configs 2-5 recipe: ellipsoid template, random smooth velocity, mR =
    transport(mT, v) with the same solver."""
    shape = (n, n, n)
    rng = np.random.Generator(np.random.PCG64(problem_seed(config_index, problem_index)))
    mT = template_ellipsoids(shape, rng, dtype=dtype)
    v = velocity_random(shape, rng, dtype=dtype)
    mR = forward_transport(mT, v, nt).astype(dtype)
    return mR, mT, v
