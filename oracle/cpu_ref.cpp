// CPU restatement (C++17 / OpenMP) of CLAIRE's Gauss-Newton-Krylov registration.
//
// THIS IS TEST INFRASTRUCTURE AND THE TIMED CPU BASELINE.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU legs load it (through the C ABI
// at the end of this file); the product library never does.
//
// It restates the reference CPU code (jaekimuh/claire, CPU master branch) with
// the reference's own loop structure, so that its cost is the reference's:
//
// * characteristics: SemiLagrangian::ComputeTrajectoryRK2
//   (src/SemiLagrangian.cpp:192-289): X in coordinates normalised by 2 pi,
//   the periodic wrap of Interp3_Plan (src/Interp3_Plan.cpp:344-361) and the
//   ghost rescale q = X N + g (src/interp3.cpp:24-60, g = 3);
// * interpolation: the ghost layer of accfft_get_ghost_xyz
//   (src/ghost.cpp:555-613) rebuilt on every call and the 64-tap tricubic
//   Lagrange kernel optimized_interp3_ghost_xyz_p (src/interp3.cpp:2492-2719)
//   with its summation order;
// * state / adjoint / incremental state / GN incremental adjoint solvers
//   (src/CLAIRE.cpp:2116-2175, 2550-2722, 3147-3290, 3849-4012): the state
//   trajectory is computed by every state solve, the adjoint trajectory by
//   every adjoint solve, the divergence of v and div v(X) by every adjoint and
//   incremental adjoint solve, and the spectral gradient of a state level
//   every time a step needs it (12 nt + 14 transforms per Hessian matvec);
// * spectral operators with the Nyquist wavenumber zeroed
//   (include/CLAIREUtils.hpp:248-255) and the 1/N^3 scale applied by the
//   callers, as AccFFT's unnormalised r2c / c2r: gradient (1 r2c + 3 c2r),
//   divergence (3 r2c + 1 c2r), regularisation symbols of
//   src/Regularization{L2,H1,H1SN,H2,H2SN,H3,H3SN}.cpp;
// * SL2 distance (src/DistanceMeasureSL2.cpp:93-283), objective, gradient
//   and GN Hessian matvec (src/CLAIRE.cpp:793-1042, 1218-1379), INVREG
//   preconditioner (src/Preconditioner.cpp:507-580);
// * PCG with the SLFS / QDFS forcing sequence (src/KrylovInterface.cpp:79-196,
//   src/Optimizer.cpp:296-356) and the GN + Armijo loop with CLAIRE's
//   stopping test (src/TaoInterface.cpp:391-527), as the NumPy oracle
//   (oracle/claire_ref.py, gauss_newton / pcg) restates PETSc TAO / KSPCG.
//
// The FFT is this file's own: mixed radix 2/3/4 Stockham transforms applied
// along an outer array axis with the inner, contiguous axis as the vector
// dimension (x2 and x1 passes on the half spectrum, the x3 pass on pairs of
// real rows packed into one complex row).
//
// Arithmetic is instantiated for float (the reference's single-precision
// build, the timed baseline) and double (the reference's default build, the
// full-size parity oracle).  Sums of the distance and of dot products are
// accumulated in double, as PETSc's VecTDot / VecNorm do in a double build.

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace cref {

static const double kPi = 3.14159265358979323846;

template <typename R>
struct Cx {
  R re, im;
};

// ---------------------------------------------------------------------------
// 1D FFT plan and the vector-radix Stockham pass
// ---------------------------------------------------------------------------
template <typename R>
struct Plan1 {
  int N = 0;
  std::vector<int> rad;                 // radix of each stage
  std::vector<std::vector<R>> wr, wi;   // forward twiddles per stage: exp(-2 pi i j p / n)

  Plan1() = default;
  explicit Plan1(int n) : N(n) {
    int m = n;
    while (m % 4 == 0 && m > 4) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0 && m > 1) { rad.push_back(2); m /= 2; }
    while (m % 3 == 0 && m > 1) { rad.push_back(3); m /= 3; }
    if (m == 4) { rad.push_back(4); m = 1; }
    if (m != 1) { N = -1; return; }  // unsupported length
    int cur = n;
    for (int p : rad) {
      const int mm = cur / p;
      std::vector<R> a((size_t)mm * (p - 1)), b((size_t)mm * (p - 1));
      for (int q = 0; q < mm; ++q)
        for (int j = 1; j < p; ++j) {
          const double th = 2.0 * kPi * (double)j * (double)q / (double)cur;
          a[(size_t)q * (p - 1) + j - 1] = (R)std::cos(th);
          b[(size_t)q * (p - 1) + j - 1] = (R)(-std::sin(th));
        }
      wr.push_back(std::move(a));
      wi.push_back(std::move(b));
      cur = mm;
    }
  }
};

// Length-N transform along the outer axis of x[N][L] for all L columns;
// sg = +1 forward (exp(-i...)), -1 inverse (exp(+i...)), unnormalised.
// y is scratch of the same size; the result is left in x.
template <typename R>
static void fft_outer(const Plan1<R>& P, Cx<R>* x, Cx<R>* y, int L, int sg) {
  int n = P.N, s = 1;
  Cx<R>* a = x;
  Cx<R>* b = y;
  const R sq3 = (R)(0.86602540378443864676);
  for (size_t st = 0; st < P.rad.size(); ++st) {
    const int p = P.rad[st], m = n / p;
    const R* wr = P.wr[st].data();
    const R* wi = P.wi[st].data();
    for (int pp = 0; pp < m; ++pp) {
      R tr[3], ti[3];
      for (int j = 1; j < p; ++j) {
        tr[j - 1] = wr[(size_t)pp * (p - 1) + j - 1];
        ti[j - 1] = (R)sg * wi[(size_t)pp * (p - 1) + j - 1];
      }
      for (int q = 0; q < s; ++q) {
        if (p == 4) {
          const Cx<R>* x0 = a + (size_t)(q + s * (pp + 0 * m)) * L;
          const Cx<R>* x1 = a + (size_t)(q + s * (pp + 1 * m)) * L;
          const Cx<R>* x2 = a + (size_t)(q + s * (pp + 2 * m)) * L;
          const Cx<R>* x3 = a + (size_t)(q + s * (pp + 3 * m)) * L;
          Cx<R>* y0 = b + (size_t)(q + s * (4 * pp + 0)) * L;
          Cx<R>* y1 = b + (size_t)(q + s * (4 * pp + 1)) * L;
          Cx<R>* y2 = b + (size_t)(q + s * (4 * pp + 2)) * L;
          Cx<R>* y3 = b + (size_t)(q + s * (4 * pp + 3)) * L;
          const R w1r = tr[0], w1i = ti[0], w2r = tr[1], w2i = ti[1], w3r = tr[2], w3i = ti[2];
          const R sgr = (R)sg;
#pragma omp simd
          for (int l = 0; l < L; ++l) {
            const R t0r = x0[l].re + x2[l].re, t0i = x0[l].im + x2[l].im;
            const R t1r = x0[l].re - x2[l].re, t1i = x0[l].im - x2[l].im;
            const R t2r = x1[l].re + x3[l].re, t2i = x1[l].im + x3[l].im;
            const R t3r = x1[l].re - x3[l].re, t3i = x1[l].im - x3[l].im;
            // y1 = t1 - i sg t3, y3 = t1 + i sg t3
            const R u1r = t1r + sgr * t3i, u1i = t1i - sgr * t3r;
            const R u3r = t1r - sgr * t3i, u3i = t1i + sgr * t3r;
            const R u2r = t0r - t2r, u2i = t0i - t2i;
            y0[l].re = t0r + t2r;
            y0[l].im = t0i + t2i;
            y1[l].re = u1r * w1r - u1i * w1i;
            y1[l].im = u1r * w1i + u1i * w1r;
            y2[l].re = u2r * w2r - u2i * w2i;
            y2[l].im = u2r * w2i + u2i * w2r;
            y3[l].re = u3r * w3r - u3i * w3i;
            y3[l].im = u3r * w3i + u3i * w3r;
          }
        } else if (p == 2) {
          const Cx<R>* x0 = a + (size_t)(q + s * (pp + 0 * m)) * L;
          const Cx<R>* x1 = a + (size_t)(q + s * (pp + 1 * m)) * L;
          Cx<R>* y0 = b + (size_t)(q + s * (2 * pp + 0)) * L;
          Cx<R>* y1 = b + (size_t)(q + s * (2 * pp + 1)) * L;
          const R w1r = tr[0], w1i = ti[0];
#pragma omp simd
          for (int l = 0; l < L; ++l) {
            const R dr = x0[l].re - x1[l].re, di = x0[l].im - x1[l].im;
            y0[l].re = x0[l].re + x1[l].re;
            y0[l].im = x0[l].im + x1[l].im;
            y1[l].re = dr * w1r - di * w1i;
            y1[l].im = dr * w1i + di * w1r;
          }
        } else {  // p == 3
          const Cx<R>* x0 = a + (size_t)(q + s * (pp + 0 * m)) * L;
          const Cx<R>* x1 = a + (size_t)(q + s * (pp + 1 * m)) * L;
          const Cx<R>* x2 = a + (size_t)(q + s * (pp + 2 * m)) * L;
          Cx<R>* y0 = b + (size_t)(q + s * (3 * pp + 0)) * L;
          Cx<R>* y1 = b + (size_t)(q + s * (3 * pp + 1)) * L;
          Cx<R>* y2 = b + (size_t)(q + s * (3 * pp + 2)) * L;
          const R w1r = tr[0], w1i = ti[0], w2r = tr[1], w2i = ti[1];
          const R sv = -(R)sg * sq3;  // imaginary part of exp(-sg 2 pi i / 3)
#pragma omp simd
          for (int l = 0; l < L; ++l) {
            const R sr = x1[l].re + x2[l].re, si = x1[l].im + x2[l].im;
            const R dr = x1[l].re - x2[l].re, di = x1[l].im - x2[l].im;
            const R cr = x0[l].re - (R)0.5 * sr, ci = x0[l].im - (R)0.5 * si;
            // y1 = c + i sv d, y2 = c - i sv d
            const R u1r = cr - sv * di, u1i = ci + sv * dr;
            const R u2r = cr + sv * di, u2i = ci - sv * dr;
            y0[l].re = x0[l].re + sr;
            y0[l].im = x0[l].im + si;
            y1[l].re = u1r * w1r - u1i * w1i;
            y1[l].im = u1r * w1i + u1i * w1r;
            y2[l].re = u2r * w2r - u2i * w2i;
            y2[l].im = u2r * w2i + u2i * w2r;
          }
        }
      }
    }
    std::swap(a, b);
    n = m;
    s *= p;
  }
  if (a != x) std::memcpy(x, a, sizeof(Cx<R>) * (size_t)P.N * L);
}

// ---------------------------------------------------------------------------
// 3D real transforms (AccFFT's accfft_execute_r2c_t / c2r_t, unnormalised)
// ---------------------------------------------------------------------------
template <typename R>
struct Fft3 {
  int n1 = 0, n2 = 0, n3 = 0, nh = 0;
  Plan1<R> p1, p2, p3;
  int nthreads = 1;
  std::vector<std::vector<Cx<R>>> scr;  // per-thread scratch

  bool init(int a, int b, int c, int threads) {
    n1 = a; n2 = b; n3 = c; nh = c / 2 + 1;
    p1 = Plan1<R>(a); p2 = Plan1<R>(b); p3 = Plan1<R>(c);
    if (p1.N < 0 || p2.N < 0 || p3.N < 0 || (b % 2) || (c % 2)) return false;
    nthreads = threads;
    const size_t need = 2 * std::max({(size_t)n3 * (n2 / 2), (size_t)n2 * nh, (size_t)n1 * nh});
    scr.assign(threads, std::vector<Cx<R>>(need));
    return true;
  }
  size_t nspec() const { return (size_t)n1 * n2 * nh; }

  void r2c(const R* f, Cx<R>* F) {
    const int h = n2 / 2;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n1; ++i1) {
      Cx<R>* T = scr[omp_get_thread_num()].data();
      Cx<R>* Y = T + scr[0].size() / 2;
      const R* P = f + (size_t)i1 * n2 * n3;
      for (int j = 0; j < h; ++j) {
        const R* ra = P + (size_t)(2 * j) * n3;
        const R* rb = ra + n3;
        for (int x3 = 0; x3 < n3; ++x3) {
          T[(size_t)x3 * h + j].re = ra[x3];
          T[(size_t)x3 * h + j].im = rb[x3];
        }
      }
      fft_outer(p3, T, Y, h, +1);
      Cx<R>* S = F + (size_t)i1 * n2 * nh;
      for (int k3 = 0; k3 < nh; ++k3) {
        const int kr = (n3 - k3) % n3;
        for (int j = 0; j < h; ++j) {
          const Cx<R> z = T[(size_t)k3 * h + j], w = T[(size_t)kr * h + j];
          // A = (z + conj w)/2, B = (z - conj w)/(2i)
          S[(size_t)(2 * j) * nh + k3] = {(R)0.5 * (z.re + w.re), (R)0.5 * (z.im - w.im)};
          S[(size_t)(2 * j + 1) * nh + k3] = {(R)0.5 * (z.im + w.im), (R)0.5 * (w.re - z.re)};
        }
      }
      fft_outer(p2, S, Y, nh, +1);
    }
    pass_x1(F, +1);
  }

  // F is overwritten (used as the transform's workspace)
  void c2r(Cx<R>* F, R* f) {
    pass_x1(F, -1);
    const int h = n2 / 2;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n1; ++i1) {
      Cx<R>* T = scr[omp_get_thread_num()].data();
      Cx<R>* Y = T + scr[0].size() / 2;
      Cx<R>* S = F + (size_t)i1 * n2 * nh;
      fft_outer(p2, S, Y, nh, -1);
      for (int j = 0; j < h; ++j) {
        const Cx<R>* A = S + (size_t)(2 * j) * nh;
        const Cx<R>* B = A + nh;
        for (int k3 = 0; k3 < nh; ++k3) {
          Cx<R> a = A[k3], b = B[k3];
          if (k3 == 0 || 2 * k3 == n3) { a.im = 0; b.im = 0; }  // c2r reads the real part there
          T[(size_t)k3 * h + j] = {a.re - b.im, a.im + b.re};          // A + i B
          if (k3 > 0 && 2 * k3 < n3)
            T[(size_t)(n3 - k3) * h + j] = {a.re + b.im, b.re - a.im};  // conj A + i conj B
        }
      }
      fft_outer(p3, T, Y, h, -1);
      R* P = f + (size_t)i1 * n2 * n3;
      for (int j = 0; j < h; ++j) {
        R* ra = P + (size_t)(2 * j) * n3;
        R* rb = ra + n3;
        for (int x3 = 0; x3 < n3; ++x3) {
          ra[x3] = T[(size_t)x3 * h + j].re;
          rb[x3] = T[(size_t)x3 * h + j].im;
        }
      }
    }
  }

 private:
  void pass_x1(Cx<R>* F, int sg) {
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < n2; ++i2) {
      Cx<R>* G = scr[omp_get_thread_num()].data();
      Cx<R>* Y = G + scr[0].size() / 2;
      for (int i1 = 0; i1 < n1; ++i1)
        std::memcpy(G + (size_t)i1 * nh, F + ((size_t)i1 * n2 + i2) * nh, sizeof(Cx<R>) * nh);
      fft_outer(p1, G, Y, nh, sg);
      for (int i1 = 0; i1 < n1; ++i1)
        std::memcpy(F + ((size_t)i1 * n2 + i2) * nh, G + (size_t)i1 * nh, sizeof(Cx<R>) * nh);
    }
  }
};

// ---------------------------------------------------------------------------
// registration problem
// ---------------------------------------------------------------------------
enum Norm { L2 = 0, H1 = 1, H1SN = 2, H2 = 3, H2SN = 4, H3 = 5, H3SN = 6 };

struct Counters {
  long long obj = 0, grad = 0, hessmatvec = 0, pcmatvec = 0, pdesolve = 0, gathers = 0, ffts = 0;
};

template <typename R>
class Problem {
 public:
  int n[3] = {0, 0, 0};
  long long nl = 0;
  int nt = 4;
  int norm = H1SN;
  double beta0 = 1e-2, beta1 = 1e-4;
  double hd = 0, ht = 0;
  int threads = 1;
  Counters cnt;

  // GN options (oracle/claire_ref.py GNOptions)
  int maxit = 50;
  double gttol = 5e-2, gatol = 1e-6;
  int krylov_maxit = 50;
  int fseq = 0;  // 0 slfs, 1 qdfs, 2 none (rtol = krylov_rtol)
  double krylov_rtol = 1e-2;
  double ls_sigma = 1e-4, min_step = 1.0 / 1024.0;
  int ls_max_trials = 30;

  // GN state
  std::vector<R> v, g;
  double J = 0, D = 0, Rv = 0, D0 = 0, J0 = 0, gnorm = 0, g0 = 0, krylov_g0 = -1, step = 1.0;
  int iter = 0, pcg_total = 0, reason = 0;  // reason: 0 running, 1 gttol, 2 gatol, 3 maxit, 4 steptol, 5 lsfail, -1 nan
  bool done = false;
  double rel_mismatch = -1.0;

  bool init(int a, int b, int c, int nt_, int norm_, double b0, double b1, int th) {
    n[0] = a; n[1] = b; n[2] = c; nt = nt_; norm = norm_; beta0 = b0; beta1 = b1;
    threads = th;
    nl = (long long)a * b * c;
    hd = (2 * kPi / a) * (2 * kPi / b) * (2 * kPi / c);
    ht = 1.0 / nt;
    if (!fft.init(a, b, c, th)) return false;
    gsz[0] = a + 6; gsz[1] = b + 6; gsz[2] = c + 6;
    ghost.resize((size_t)gsz[0] * gsz[1] * gsz[2]);
    spec.resize(3 * fft.nspec());
    spec2.resize(fft.nspec());
    mR.resize(nl); mT.resize(nl);
    m.resize((size_t)(nt + 1) * nl);
    Xs.resize(3 * nl); Xa.resize(3 * nl);
    v.assign(3 * nl, 0); g.assign(3 * nl, 0);
    w1.resize(3 * nl); w2.resize(3 * nl); s1.resize(nl); s2.resize(nl); s3.resize(nl);
    lam.resize(nl); lamx.resize(nl); bfield.resize(3 * nl);
    mt.resize(nl); vtx.resize(3 * nl);
    kx[0] = wavenumbers(a, a); kx[1] = wavenumbers(b, b); kx[2] = wavenumbers(c, c / 2 + 1);
    return true;
  }

  void set_images(const double* r, const double* t) {
    for (long long i = 0; i < nl; ++i) { mR[i] = (R)r[i]; mT[i] = (R)t[i]; }
    state_valid = false;
  }

  // ---------------- interpolation -------------------------------------------
  // accfft_get_ghost_xyz: periodic ghost layer of width 3 (src/ghost.cpp:555-613)
  void pad(const R* f) {
    const int g0 = gsz[0], g1 = gsz[1], g2 = gsz[2];
    cnt.gathers += 1;
#pragma omp parallel for schedule(static)
    for (int a = 0; a < g0; ++a) {
      const int i1 = (a - 3 + n[0]) % n[0];
      for (int b = 0; b < g1; ++b) {
        const int i2 = (b - 3 + n[1]) % n[1];
        const R* row = f + ((size_t)i1 * n[1] + i2) * n[2];
        R* out = ghost.data() + ((size_t)a * g1 + b) * g2;
        for (int c = 0; c < 3; ++c) out[c] = row[n[2] - 3 + c];
        std::memcpy(out + 3, row, sizeof(R) * n[2]);
        for (int c = 0; c < 3; ++c) out[3 + n[2] + c] = row[c];
      }
    }
  }

  // optimized_interp3_ghost_xyz_p (src/interp3.cpp:2492-2719) at the ghost
  // coordinates q (3 per point), with that kernel's summation order
  void interp(const std::vector<R>& q, R* out) {
    const int g1 = gsz[1], g2 = gsz[2];
    const R* gv = ghost.data();
    const R den[4] = {(R)(-1.0 / 6.0), (R)0.5, (R)(-0.5), (R)(1.0 / 6.0)};
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nl; ++i) {
      R M[3][4];
      int gi[3];
      for (int j = 0; j < 3; ++j) {
        R p = q[3 * i + j];
        gi[j] = (int)std::floor(p) - 1;
        p -= (R)gi[j];
        for (int k = 0; k < 4; ++k) {
          R mk = den[k];
          for (int l = 0; l < 4; ++l)
            if (k != l) mk *= (p - (R)l);
          M[j][k] = mk;
        }
      }
      const size_t base = (size_t)g2 * g1 * gi[0] + gi[2] + (size_t)g2 * gi[1];
      R v1[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int j0 = 0; j0 < 4; ++j0) {
        const R* pl = gv + base + (size_t)j0 * g1 * g2;
        for (int j1 = 0; j1 < 4; j1 += 2) {
          const R* pa = pl + (size_t)j1 * g2;
          const R* pb = pa + g2;
          R v2[8];
          for (int c = 0; c < 4; ++c) v2[c] = M[1][j1] * pa[c];
          for (int c = 0; c < 4; ++c) v2[4 + c] = M[1][j1 + 1] * pb[c];
          for (int c = 0; c < 8; ++c) v1[c] += M[0][j0] * v2[c];
        }
      }
      R val = 0;
      for (int c = 0; c < 4; ++c) val += v1[c] * M[2][c];
      for (int c = 0; c < 4; ++c) val += v1[c + 4] * M[2][c];
      out[i] = val;
    }
  }

  void interp_scalar(const R* f, const std::vector<R>& q, R* out) {
    pad(f);
    interp(q, out);
  }

  // wrap (src/Interp3_Plan.cpp:344-361) and ghost rescale (src/interp3.cpp:24-60)
  void to_ghost(std::vector<R>& X) {
    const R h[3] = {(R)(1.0 / n[0]), (R)(1.0 / n[1]), (R)(1.0 / n[2])};
    const R N[3] = {(R)n[0], (R)n[1], (R)n[2]};
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nl; ++i)
      for (int d = 0; d < 3; ++d) {
        R Q = X[3 * i + d];
        while (Q <= -h[d]) Q += (R)1;
        while (Q >= (R)1) Q -= (R)1;
        X[3 * i + d] = Q * N[d] + (R)3;
      }
  }

  // ComputeTrajectoryRK2 (src/SemiLagrangian.cpp:192-289); X keeps the ghost
  // coordinates of the foot points.  scale = +1 state, -1 adjoint.
  void trajectory(const R* vel, R scale, std::vector<R>& X, std::vector<R>* unwrapped = nullptr) {
    const R hx[3] = {(R)(2 * kPi / n[0]), (R)(2 * kPi / n[1]), (R)(2 * kPi / n[2])};
    const R tpi = (R)(2.0 * kPi);
    const R htR = (R)ht, hth = (R)(0.5 * ht);
    const R* v1 = vel;
    const R* v2 = vel + nl;
    const R* v3 = vel + 2 * nl;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n[0]; ++i1)
      for (int i2 = 0; i2 < n[1]; ++i2)
        for (int i3 = 0; i3 < n[2]; ++i3) {
          const long long l = ((long long)i1 * n[1] + i2) * n[2] + i3;
          const R x1 = hx[0] * (R)i1, x2 = hx[1] * (R)i2, x3 = hx[2] * (R)i3;
          X[3 * l + 0] = (x1 - scale * htR * v1[l]) / tpi;
          X[3 * l + 1] = (x2 - scale * htR * v2[l]) / tpi;
          X[3 * l + 2] = (x3 - scale * htR * v3[l]) / tpi;
        }
    to_ghost(X);
    // v(X~), one vector interpolation
    for (int d = 0; d < 3; ++d) interp_scalar(vel + d * nl, X, w2.data() + d * nl);
    const R* vx1 = w2.data();
    const R* vx2 = w2.data() + nl;
    const R* vx3 = w2.data() + 2 * nl;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n[0]; ++i1)
      for (int i2 = 0; i2 < n[1]; ++i2)
        for (int i3 = 0; i3 < n[2]; ++i3) {
          const long long l = ((long long)i1 * n[1] + i2) * n[2] + i3;
          const R x1 = hx[0] * (R)i1, x2 = hx[1] * (R)i2, x3 = hx[2] * (R)i3;
          X[3 * l + 0] = (x1 - scale * hth * (vx1[l] + v1[l])) / tpi;
          X[3 * l + 1] = (x2 - scale * hth * (vx2[l] + v2[l])) / tpi;
          X[3 * l + 2] = (x3 - scale * hth * (vx3[l] + v3[l])) / tpi;
        }
    if (unwrapped) *unwrapped = X;
    to_ghost(X);
  }

  // ---------------- spectral operators ------------------------------------
  // accfft_grad_t: out[d] = F^-1(i k_d F f) / N^3
  void grad(const R* f, R* out) {
    fft.r2c(f, spec.data());
    cnt.ffts += 4;
    const size_t ns = fft.nspec();
    for (int d = 0; d < 3; ++d) {
      mul_ik(spec.data(), spec2.data(), d);
      fft.c2r(spec2.data(), out + d * nl);
    }
    (void)ns;
  }

  // accfft_divergence_t: F^-1(sum_d i k_d F v_d) / N^3
  void div(const R* vel, R* out) {
    const size_t ns = fft.nspec();
    std::fill(spec2.begin(), spec2.end(), Cx<R>{0, 0});
    for (int d = 0; d < 3; ++d) {
      fft.r2c(vel + d * nl, spec.data());
      add_ik(spec.data(), spec2.data(), d);
    }
    fft.c2r(spec2.data(), out);
    cnt.ffts += 4;
    (void)ns;
  }

  // spectral symbol of the regularisation (kind 0: EvaluateGradient /
  // HessianMatVec, 1: ApplyInverse, 2: ApplyInverse with applysqrt); the
  // 1/N^3 scale is folded in.  src/Regularization*.cpp (symbols: oracle
  // Regularization.grad_symbol / inv_symbol).
  double symbol(int kind, double kap) const {
    const double b0 = beta0, b1 = beta1;
    if (kind == 0) {
      switch (norm) {
        case H1SN: return hd * b0 * kap;
        case H1: return hd * b0 * (kap + b1);
        case H2: return b0 * (kap * kap + b1);
        case H2SN: return hd * b0 * kap * kap;
        case H3: return b0 * (kap * kap * kap + b1);
        case H3SN: return b0 * kap * kap * kap;
      }
      return 0.0;
    }
    double op = 1.0;
    switch (norm) {
      case H1SN: op = kap == 0.0 ? b0 : b0 * kap; break;
      case H1: op = b0 * (kap + b1); break;
      case H2: op = b0 * (kap * kap + b1); break;
      case H2SN: op = kap == 0.0 ? b0 : b0 * kap * kap; break;
      case H3: op = b0 * (kap * kap * kap + b1); break;
      case H3SN: op = kap == 0.0 ? b0 : b0 * kap * kap * kap; break;
    }
    if (kind == 2) op = std::sqrt(op);
    return 1.0 / op;
  }

  // out = Reg op (kind) applied to the 3 components of x (3 r2c + 3 c2r)
  void reg_apply(int kind, const R* x, R* out) {
    if (norm == L2) {
      const double f = kind == 0 ? beta0 : 1.0 / beta0;  // oracle: applysqrt is not applied for L2
      if (beta0 == 0.0) { std::memcpy(out, x, sizeof(R) * 3 * nl); return; }
      for (long long i = 0; i < 3 * nl; ++i) out[i] = (R)(f * x[i]);
      return;
    }
    if (beta0 == 0.0) {
      if (kind == 0) std::fill(out, out + 3 * nl, (R)0);
      else std::memcpy(out, x, sizeof(R) * 3 * nl);
      return;
    }
    const double scale = 1.0 / (double)nl;
    for (int d = 0; d < 3; ++d) {
      fft.r2c(x + d * nl, spec.data());
      mul_symbol(spec.data(), kind, scale);
      fft.c2r(spec.data(), out + d * nl);
    }
    cnt.ffts += 6;
  }

  // Regularization::EvaluateFunctional (oracle Regularization.functional)
  double reg_functional(const R* vel) {
    if (beta0 == 0.0) return 0.0;
    const double b0 = beta0, b1 = beta1;
    if (norm == L2) return 0.5 * hd * b0 * sumsq(vel, 3 * nl);
    if (norm == H1SN || norm == H1) {
      double h1 = 0.0;
      for (int d = 0; d < 3; ++d) {
        grad(vel + d * nl, w1.data());
        h1 += sumsq(w1.data(), 3 * nl);
      }
      if (norm == H1SN) return 0.5 * hd * b0 * h1;
      return 0.5 * hd * b0 * (h1 + b1 * sumsq(vel, 3 * nl));
    }
    const double scale = 1.0 / (double)nl;
    double r = 0.0;
    for (int d = 0; d < 3; ++d) {
      fft.r2c(vel + d * nl, spec.data());
      Cx<R>* S = spec.data();
      const int nh = fft.nh;
      for (int i1 = 0; i1 < n[0]; ++i1)
        for (int i2 = 0; i2 < n[1]; ++i2)
          for (int k3 = 0; k3 < nh; ++k3) {
            const size_t idx = ((size_t)i1 * n[1] + i2) * nh + k3;
            const double k1 = kx[0][i1], k2 = kx[1][i2], kk3 = kx[2][k3];
            const double kap = k1 * k1 + k2 * k2 + kk3 * kk3;
            double mre, mim;
            if (norm == H2) { mre = mim = std::sqrt(b0) * (-kap + std::sqrt(b1)); }
            else if (norm == H2SN) { mre = mim = -kap; }
            else {
              const double kd = d == 0 ? k1 : (d == 1 ? k2 : kk3);
              const double a = kd * (-kap);
              if (norm == H3) { mre = std::sqrt(b0) * (a + std::sqrt(b1)); mim = std::sqrt(b0) * (-a + std::sqrt(b1)); }
              else { mre = a; mim = -a; }
            }
            S[idx].re = (R)(mre * scale * S[idx].re);
            S[idx].im = (R)(mim * scale * S[idx].im);
          }
      fft.c2r(spec.data(), s1.data());
      r += sumsq(s1.data(), nl);
    }
    cnt.ffts += 6;
    if (norm == H2) return 0.5 * hd * r;
    if (norm == H2SN) return 0.5 * b0 * hd * r;
    return 0.5 * hd * r * (norm == H3SN ? b0 : 1.0);
  }

  // ---------------- PDE solvers ----------------------------------------------
  // SolveStateEquationSL (src/CLAIRE.cpp:2116-2175)
  void state_solve(const R* vel) {
    trajectory(vel, (R)1, Xs);
    std::memcpy(m.data(), mT.data(), sizeof(R) * nl);
    for (int j = 0; j < nt; ++j) interp_scalar(m.data() + (size_t)j * nl, Xs, m.data() + (size_t)(j + 1) * nl);
    cnt.pdesolve += 1;
    state_valid = true;
  }

  // SL2 distance 1/2 hd sum (mR - m1)^2 (src/DistanceMeasureSL2.cpp:93-155)
  double distance() const {
    const R* m1 = m.data() + (size_t)nt * nl;
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long long i = 0; i < nl; ++i) {
      const double d = (double)mR[i] - (double)m1[i];
      s += d * d;
    }
    return 0.5 * hd * s;
  }

  // EvaluateObjective (src/CLAIRE.cpp:793-863)
  double objective(const R* vel) {
    state_solve(vel);
    D = distance();
    bool nz = false;
    for (long long i = 0; i < 3 * nl && !nz; ++i) nz = vel[i] != (R)0;
    Rv = nz ? reg_functional(vel) : 0.0;
    cnt.obj += 1;
    return D + Rv;
  }

  // backward SL loop shared by the adjoint (src/CLAIRE.cpp:2646-2709) and the
  // GN incremental adjoint (:3940-3999); lam holds lambda(t=1) on entry.
  // b accumulates the body force (before the hd scaling).
  void backward_sl(std::vector<R>& b) {
    const R htR = (R)ht;
    const R inv_nc = (R)1;  // one image component
    // divergence of v and div v(X) (every solve)
    div(v.data(), s1.data());
    interp_scalar(s1.data(), Xa, s2.data());
    std::fill(b.begin(), b.end(), (R)0);
    R scale = htR;
    for (int j = 0; j < nt; ++j) {
      if (j == 0) scale *= (R)0.5;
      interp_scalar(lam.data(), Xa, lamx.data());
      grad(m.data() + (size_t)(nt - j) * nl, w1.data());
      const R* dv = s1.data();
      const R* dvx = s2.data();
      R* L = lam.data();
      const R* LX = lamx.data();
      R* b1 = b.data();
      R* b2 = b.data() + nl;
      R* b3 = b.data() + 2 * nl;
      const R* g1 = w1.data();
      const R* g2 = w1.data() + nl;
      const R* g3 = w1.data() + 2 * nl;
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < nl; ++i) {
        const R lambda = L[i], lx = LX[i];
        const R rhs0 = lx * dvx[i];
        const R rhs1 = (lx + htR * rhs0) * dv[i];
        L[i] = lx + (R)0.5 * htR * (rhs0 + rhs1);
        b1[i] += scale * g1[i] * lambda / inv_nc;
        b2[i] += scale * g2[i] * lambda / inv_nc;
        b3[i] += scale * g3[i] * lambda / inv_nc;
      }
      if (j == 0) scale *= (R)2;
    }
    grad(m.data(), w1.data());
    {
      R* b1 = b.data();
      R* b2 = b.data() + nl;
      R* b3 = b.data() + 2 * nl;
      const R* L = lam.data();
      const R* g1 = w1.data();
      const R* g2 = w1.data() + nl;
      const R* g3 = w1.data() + 2 * nl;
#pragma omp parallel for schedule(static)
      for (long long i = 0; i < nl; ++i) {
        const R lambda = L[i];
        b1[i] += (R)0.5 * scale * g1[i] * lambda / inv_nc;
        b2[i] += (R)0.5 * scale * g2[i] * lambda / inv_nc;
        b3[i] += (R)0.5 * scale * g3[i] * lambda / inv_nc;
      }
    }
  }

  // EvaluateGradient (src/CLAIRE.cpp:871-1042): state solved for vel first
  void gradient(const R* vel, R* out) {
    if (vel != v.data()) std::memcpy(v.data(), vel, sizeof(R) * 3 * nl);
    if (!state_valid || state_of != vel_stamp()) { state_solve(v.data()); state_of = vel_stamp(); }
    trajectory(v.data(), (R)-1, Xa);
    const R* m1 = m.data() + (size_t)nt * nl;
    for (long long i = 0; i < nl; ++i) lam[i] = mR[i] - m1[i];  // SetFinalConditionAE
    backward_sl(bfield);
    bool nz = false;
    for (long long i = 0; i < 3 * nl && !nz; ++i) nz = v[i] != (R)0;
    const R hdR = (R)hd;
    if (!nz) {
      for (long long i = 0; i < 3 * nl; ++i) out[i] = hdR * bfield[i];
    } else {
      reg_apply(0, v.data(), out);
      for (long long i = 0; i < 3 * nl; ++i) out[i] = out[i] + hdR * bfield[i];
    }
    cnt.grad += 1;
  }

  // SolveIncStateEquationSL (src/CLAIRE.cpp:3147-3290), state trajectory reused
  void inc_state(const R* vt) {
    const R hth = (R)(0.5 * ht);
    for (int d = 0; d < 3; ++d) interp_scalar(vt + d * nl, Xs, vtx.data() + d * nl);
    std::fill(mt.begin(), mt.end(), (R)0);
    for (int j = 0; j < nt; ++j) {
      interp_scalar(mt.data(), Xs, s3.data());
      std::memcpy(mt.data(), s3.data(), sizeof(R) * nl);
      grad(m.data() + (size_t)j * nl, w1.data());
      for (int d = 0; d < 3; ++d) interp_scalar(w1.data() + d * nl, Xs, w2.data() + d * nl);
      {
        const R* a1 = w2.data();
        const R* a2 = w2.data() + nl;
        const R* a3 = w2.data() + 2 * nl;
        const R* x1 = vtx.data();
        const R* x2 = vtx.data() + nl;
        const R* x3 = vtx.data() + 2 * nl;
        R* M = mt.data();
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < nl; ++i) M[i] -= hth * (a1[i] * x1[i] + a2[i] * x2[i] + a3[i] * x3[i]);
      }
      grad(m.data() + (size_t)(j + 1) * nl, w1.data());
      {
        const R* a1 = w1.data();
        const R* a2 = w1.data() + nl;
        const R* a3 = w1.data() + 2 * nl;
        const R* x1 = vt;
        const R* x2 = vt + nl;
        const R* x3 = vt + 2 * nl;
        R* M = mt.data();
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < nl; ++i) M[i] -= hth * (a1[i] * x1[i] + a2[i] * x2[i] + a3[i] * x3[i]);
      }
    }
  }

  // HessianMatVec (src/CLAIRE.cpp:1218-1379): GN, adjoint trajectory of the
  // last gradient reused (the SL object keeps it)
  void hessian_matvec(const R* vt, R* out) {
    inc_state(vt);
    for (long long i = 0; i < nl; ++i) lam[i] = -mt[i];  // SetFinalConditionIAE
    backward_sl(bfield);
    reg_apply(0, vt, out);
    const R hdR = (R)hd;
    for (long long i = 0; i < 3 * nl; ++i) out[i] = out[i] + hdR * bfield[i];
    cnt.hessmatvec += 1;
  }

  void precond(const R* x, R* out) {
    reg_apply(1, x, out);
    cnt.pcmatvec += 1;
  }

  // ---------------- Gauss-Newton-Krylov --------------------------------------
  // oracle/claire_ref.py pcg: KSPCG as configured at src/Optimizer.cpp:296-356
  int pcg(const std::vector<R>& b, double rtol, std::vector<R>& x, int kmaxit) {
    const size_t N3 = 3 * nl;
    x.assign(N3, (R)0);
    std::vector<R> r(b), z(N3), p(N3), q(N3);
    const double rn0 = std::sqrt(dot(r.data(), r.data(), N3));
    const double tol = std::max(rtol * rn0, 1e-16);
    if (rn0 <= tol) return 0;
    precond(r.data(), z.data());
    p = z;
    double rz = dot(r.data(), z.data(), N3);
    int it = 0;
    while (it < kmaxit) {
      hessian_matvec(p.data(), q.data());
      const double pq = dot(p.data(), q.data(), N3);
      if (!(pq > 0.0) || !std::isfinite(pq)) break;
      const double alpha = rz / pq;
      const R aR = (R)alpha;
      for (size_t i = 0; i < N3; ++i) { x[i] = x[i] + aR * p[i]; r[i] = r[i] - aR * q[i]; }
      ++it;
      const double rn = std::sqrt(dot(r.data(), r.data(), N3));
      if (rn <= tol) break;
      if (rn > 1e6 * rn0) break;
      precond(r.data(), z.data());
      const double rzn = dot(r.data(), z.data(), N3);
      const double beta = rzn / rz;
      rz = rzn;
      const R bR = (R)beta;
      for (size_t i = 0; i < N3; ++i) p[i] = z[i] + bR * p[i];
    }
    return it;
  }

  double forcing(double gn, double gref) const {
    const double r = gn / gref;
    if (fseq == 2) return krylov_rtol;
    if (fseq == 1) return std::max(1e-16, std::min(0.5, r));
    return std::max(1e-16, std::min(0.5, std::sqrt(r)));
  }

  // InitializeOptimization + first objective / gradient (oracle gauss_newton
  // up to the loop): v = 0
  void begin() {
    std::fill(v.begin(), v.end(), (R)0);
    vel_version++;
    J = objective(v.data());
    D0 = D;
    J0 = J;
    state_of = vel_stamp();
    gradient(v.data(), g.data());
    gnorm = std::sqrt(dot(g.data(), g.data(), 3 * nl));
    g0 = gnorm > 0 ? gnorm : 1.0;
    krylov_g0 = -1;
    iter = 0; step = 1.0; pcg_total = 0; reason = 0; done = false;
    t0 = std::chrono::steady_clock::now();
  }

  // stopping tests at the top of the loop; 1 when stopped
  bool check_stop() {
    if (!(std::isfinite(J) && std::isfinite(gnorm))) { reason = -1; return true; }
    if (step < min_step) { reason = 4; return true; }
    if (gnorm < gttol * g0) { reason = 1; return true; }
    if (gnorm < gatol) { reason = 2; return true; }
    if (iter > maxit - 1) { reason = 3; return true; }
    return false;
  }

  // one GN iteration (forcing, PCG, Armijo, gradient); returns 1 when the
  // solve has stopped (before or after this iteration's work)
  int gn_step() {
    if (done) return 1;
    if (check_stop()) { done = true; return 1; }
    if (krylov_g0 < 0) krylov_g0 = gnorm;
    const double rtol = forcing(gnorm, krylov_g0);
    const size_t N3 = 3 * nl;
    std::vector<R> mg(N3), d;
    for (size_t i = 0; i < N3; ++i) mg[i] = -g[i];
    const int kit = pcg(mg, rtol, d, std::max(0, krylov_maxit - 1));
    pcg_total += kit;
    double gd = dot(g.data(), d.data(), N3);
    if (!(gd < 0.0)) {
      for (size_t i = 0; i < N3; ++i) d[i] = -g[i];
      gd = -dot(g.data(), g.data(), N3);
    }
    double alpha = 1.0;
    bool accepted = false;
    std::vector<R> vt(N3);
    double Jt = 0;
    for (int t = 0; t < ls_max_trials; ++t) {
      const R aR = (R)alpha;
      for (size_t i = 0; i < N3; ++i) vt[i] = v[i] + aR * d[i];
      Jt = objective(vt.data());
      if (Jt <= J + ls_sigma * alpha * gd) { accepted = true; break; }
      alpha *= 0.5;
    }
    if (!accepted) { reason = 5; done = true; return 1; }
    v = vt;
    vel_version++;
    state_of = vel_stamp();  // the accepted trial's state is current
    J = Jt;
    step = alpha;
    gradient(v.data(), g.data());
    gnorm = std::sqrt(dot(g.data(), g.data(), N3));
    iter += 1;
    if (check_stop()) { done = true; return 1; }
    return 0;
  }

  // final relative mismatch |mR - m1| / |mR - mT| (src/CLAIRE.cpp:4232-4262)
  void finish() {
    if (state_of != vel_stamp()) { state_solve(v.data()); state_of = vel_stamp(); }
    const R* m1 = m.data() + (size_t)nt * nl;
    double a = 0, b = 0;
    for (long long i = 0; i < nl; ++i) {
      const double x = (double)mR[i] - (double)m1[i], y = (double)mR[i] - (double)mT[i];
      a += x * x;
      b += y * y;
    }
    rel_mismatch = b > 0 ? std::sqrt(a / b) : 0.0;
    seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  void run() {
    begin();
    while (!gn_step()) {
    }
    finish();
  }

  void last_adjoint(double* lam0, double* bf) const {
    for (long long i = 0; i < nl; ++i) lam0[i] = (double)lam[i];
    for (long long i = 0; i < 3 * nl; ++i) bf[i] = hd * (double)bfield[i];
  }

  double seconds = 0;
  std::vector<R> m, mR, mT;
  std::vector<R> Xs, Xa;  // ghost coordinates of the state / adjoint foot points

  double dot(const R* a, const R* b, size_t len) const {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long long i = 0; i < (long long)len; ++i) s += (double)a[i] * (double)b[i];
    return s;
  }
  double sumsq(const R* a, size_t len) const { return dot(a, a, len); }

  // ---- velocity bookkeeping: the state arrays belong to one velocity ------
  long long vel_version = 0;
  long long vel_stamp() const { return vel_version; }
  long long state_of = -1;
  bool state_valid = false;

 private:
  Fft3<R> fft;
  int gsz[3] = {0, 0, 0};
  std::vector<R> ghost;
  std::vector<Cx<R>> spec, spec2;
  std::vector<R> w1, w2, s1, s2, s3, lam, lamx, bfield, mt, vtx;
  std::vector<double> kx[3];
  std::chrono::steady_clock::time_point t0{};

  static std::vector<double> wavenumbers(int N, int count) {
    std::vector<double> k(count);
    for (int i = 0; i < count; ++i) {
      int w = i;
      if (w > N / 2) w -= N;
      if (2 * w == N) w = 0;  // Nyquist -> 0 (include/CLAIREUtils.hpp:248-255)
      k[i] = (double)w;
    }
    return k;
  }

  void mul_ik(const Cx<R>* S, Cx<R>* O, int d) {
    const int nh = fft.nh;
    const double scale = 1.0 / (double)nl;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n[0]; ++i1)
      for (int i2 = 0; i2 < n[1]; ++i2) {
        const size_t row = ((size_t)i1 * n[1] + i2) * nh;
        for (int k3 = 0; k3 < nh; ++k3) {
          const double kd = d == 0 ? kx[0][i1] : (d == 1 ? kx[1][i2] : kx[2][k3]);
          const R f = (R)(kd * scale);
          const Cx<R> s = S[row + k3];
          O[row + k3] = {-f * s.im, f * s.re};
        }
      }
  }
  void add_ik(const Cx<R>* S, Cx<R>* O, int d) {
    const int nh = fft.nh;
    const double scale = 1.0 / (double)nl;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n[0]; ++i1)
      for (int i2 = 0; i2 < n[1]; ++i2) {
        const size_t row = ((size_t)i1 * n[1] + i2) * nh;
        for (int k3 = 0; k3 < nh; ++k3) {
          const double kd = d == 0 ? kx[0][i1] : (d == 1 ? kx[1][i2] : kx[2][k3]);
          const R f = (R)(kd * scale);
          const Cx<R> s = S[row + k3];
          O[row + k3].re += -f * s.im;
          O[row + k3].im += f * s.re;
        }
      }
  }
  void mul_symbol(Cx<R>* S, int kind, double scale) {
    const int nh = fft.nh;
#pragma omp parallel for schedule(static)
    for (int i1 = 0; i1 < n[0]; ++i1)
      for (int i2 = 0; i2 < n[1]; ++i2) {
        const size_t row = ((size_t)i1 * n[1] + i2) * nh;
        for (int k3 = 0; k3 < nh; ++k3) {
          const double kap = kx[0][i1] * kx[0][i1] + kx[1][i2] * kx[1][i2] + kx[2][k3] * kx[2][k3];
          const R f = (R)(symbol(kind, kap) * scale);
          S[row + k3].re *= f;
          S[row + k3].im *= f;
        }
      }
  }
};

}  // namespace cref

// ---------------------------------------------------------------------------
// C ABI (ctypes): arrays in and out are float64, converted at the boundary
// ---------------------------------------------------------------------------
namespace {

struct Handle {
  int fp64 = 1;
  std::unique_ptr<cref::Problem<float>> f;
  std::unique_ptr<cref::Problem<double>> d;
  std::vector<float> a, b;  // conversion buffers
};

template <typename R>
static std::vector<R> conv(const double* in, size_t len) {
  std::vector<R> out(len);
  for (size_t i = 0; i < len; ++i) out[i] = (R)in[i];
  return out;
}

template <typename R>
static void back(const R* in, double* out, size_t len) {
  for (size_t i = 0; i < len; ++i) out[i] = (double)in[i];
}

template <typename F>
static int dispatch(void* h, F&& fn) {
  if (!h) return -1;
  Handle* H = (Handle*)h;
  if (H->fp64) return fn(*H->d);
  return fn(*H->f);
}

}  // namespace

extern "C" {

// norm: 0 l2, 1 h1, 2 h1s, 3 h2, 4 h2s, 5 h3, 6 h3s; fp64: 1 double, 0 float
void* cref_create(int n1, int n2, int n3, int nt, int norm, double beta0, double beta1, int fp64, int threads) {
  if (threads <= 0) threads = omp_get_max_threads();
  omp_set_num_threads(threads);
  Handle* H = new Handle();
  H->fp64 = fp64 ? 1 : 0;
  bool ok;
  if (H->fp64) {
    H->d.reset(new cref::Problem<double>());
    ok = H->d->init(n1, n2, n3, nt, norm, beta0, beta1, threads);
  } else {
    H->f.reset(new cref::Problem<float>());
    ok = H->f->init(n1, n2, n3, nt, norm, beta0, beta1, threads);
  }
  if (!ok) {
    delete H;
    return nullptr;
  }
  return H;
}

void cref_destroy(void* h) { delete (Handle*)h; }

int cref_max_threads(void) { return omp_get_max_threads(); }

int cref_set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  return omp_get_max_threads();
}

// fseq: 0 slfs, 1 qdfs, 2 none (fixed relative tolerance krylov_rtol)
int cref_set_gn(void* h, int maxit, double gttol, double gatol, int krylov_maxit, int fseq, double krylov_rtol) {
  return dispatch(h, [&](auto& P) {
    P.maxit = maxit; P.gttol = gttol; P.gatol = gatol; P.krylov_maxit = krylov_maxit; P.fseq = fseq;
    P.krylov_rtol = krylov_rtol;
    return 0;
  });
}

int cref_set_images(void* h, const double* mR, const double* mT) {
  return dispatch(h, [&](auto& P) { P.set_images(mR, mT); return 0; });
}

// J, D, R at v (3 n)
int cref_objective(void* h, const double* v, double* out3) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    const double J = P.objective(vv.data());
    out3[0] = J; out3[1] = P.D; out3[2] = P.Rv;
    return 0;
  });
}

int cref_gradient(void* h, const double* v, double* g) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    P.vel_version++;
    P.state_of = -1;
    std::vector<R> out(3 * P.nl);
    P.gradient(vv.data(), out.data());
    back(out.data(), g, 3 * P.nl);
    return 0;
  });
}

// GN Hessian matvec at v (objective and gradient evaluated at v first, as the
// solver has them when it runs the Krylov solve)
int cref_hessian_matvec(void* h, const double* v, const double* vt, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    auto tt = conv<R>(vt, 3 * P.nl);
    P.vel_version++;
    P.state_of = -1;
    std::vector<R> gg(3 * P.nl), o(3 * P.nl);
    P.gradient(vv.data(), gg.data());
    P.hessian_matvec(tt.data(), o.data());
    back(o.data(), out, 3 * P.nl);
    return 0;
  });
}

// GN Hessian matvec at the velocity of the last cref_gradient call (its state,
// adjoint and characteristics are reused, as HessianMatVec reuses them after
// EvaluateGradient in the reference, src/CLAIRE.cpp:1218-1303).
int cref_hessian_matvec_current(void* h, const double* vt, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto tt = conv<R>(vt, 3 * P.nl);
    std::vector<R> o(3 * P.nl);
    P.hessian_matvec(tt.data(), o.data());
    back(o.data(), out, 3 * P.nl);
    return 0;
  });
}

int cref_precond(void* h, const double* x, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto xx = conv<R>(x, 3 * P.nl);
    std::vector<R> o(3 * P.nl);
    P.precond(xx.data(), o.data());
    back(o.data(), out, 3 * P.nl);
    return 0;
  });
}

// kind 0: EvaluateGradient, 1: ApplyInverse, 2: ApplyInverse (applysqrt)
int cref_reg_apply(void* h, int kind, const double* x, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto xx = conv<R>(x, 3 * P.nl);
    std::vector<R> o(3 * P.nl);
    P.reg_apply(kind, xx.data(), o.data());
    back(o.data(), out, 3 * P.nl);
    return 0;
  });
}

int cref_reg_functional(void* h, const double* v, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    *out = P.reg_functional(vv.data());
    return 0;
  });
}

// spectral gradient (f: n -> out: 3n) and divergence (v: 3n -> out: n)
int cref_grad(void* h, const double* f, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto ff = conv<R>(f, P.nl);
    std::vector<R> o(3 * P.nl);
    P.grad(ff.data(), o.data());
    back(o.data(), out, 3 * P.nl);
    return 0;
  });
}

int cref_div(void* h, const double* v, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    std::vector<R> o(P.nl);
    P.div(vv.data(), o.data());
    back(o.data(), out, P.nl);
    return 0;
  });
}

// RK2 foot points of v (flag +1 state, -1 adjoint) as displacements in grid
// units, X N - i before the wrap (the oracle's trajectory_rk2 form)
int cref_trajectory(void* h, const double* v, int flag, double* disp) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    std::vector<R> X(3 * P.nl), U;
    P.trajectory(vv.data(), (R)flag, X, &U);
    const int n1 = P.n[0], n2 = P.n[1], n3 = P.n[2];
    for (int i1 = 0; i1 < n1; ++i1)
      for (int i2 = 0; i2 < n2; ++i2)
        for (int i3 = 0; i3 < n3; ++i3) {
          const long long l = ((long long)i1 * n2 + i2) * n3 + i3;
          disp[0 * P.nl + l] = (double)U[3 * l + 0] * n1 - i1;
          disp[1 * P.nl + l] = (double)U[3 * l + 1] * n2 - i2;
          disp[2 * P.nl + l] = (double)U[3 * l + 2] * n3 - i3;
        }
    return 0;
  });
}

// tricubic interpolation of f at x + disp (disp in grid units, 3 n)
int cref_interp(void* h, const double* f, const double* disp, double* out) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto ff = conv<R>(f, P.nl);
    const int n1 = P.n[0], n2 = P.n[1], n3 = P.n[2];
    std::vector<R> X(3 * P.nl), o(P.nl);
    for (int i1 = 0; i1 < n1; ++i1)
      for (int i2 = 0; i2 < n2; ++i2)
        for (int i3 = 0; i3 < n3; ++i3) {
          const long long l = ((long long)i1 * n2 + i2) * n3 + i3;
          X[3 * l + 0] = (R)((i1 + disp[0 * P.nl + l]) / n1);
          X[3 * l + 1] = (R)((i2 + disp[1 * P.nl + l]) / n2);
          X[3 * l + 2] = (R)((i3 + disp[2 * P.nl + l]) / n3);
        }
    P.to_ghost(X);
    P.interp_scalar(ff.data(), X, o.data());
    back(o.data(), out, P.nl);
    return 0;
  });
}

// state at t = 1 of m0 transported by v (SolveForwardProblem)
int cref_forward(void* h, const double* v, const double* m0, double* m1) {
  return dispatch(h, [&](auto& P) {
    using R = typename std::remove_reference<decltype(P.v[0])>::type;
    auto vv = conv<R>(v, 3 * P.nl);
    auto mm = conv<R>(m0, P.nl);
    std::vector<R> keep(P.mT);
    P.mT = mm;
    P.state_solve(vv.data());
    P.mT = keep;
    P.vel_version++;
    P.state_of = -1;
    back(P.m.data() + (size_t)P.nt * P.nl, m1, P.nl);
    return 0;
  });
}

int cref_begin(void* h) { return dispatch(h, [&](auto& P) { P.begin(); return 0; }); }

// one GN iteration; 1 when the solve has stopped
int cref_step(void* h) { return dispatch(h, [&](auto& P) { return P.gn_step(); }); }

int cref_finish(void* h) { return dispatch(h, [&](auto& P) { P.finish(); return 0; }); }

int cref_run(void* h) { return dispatch(h, [&](auto& P) { P.run(); return 0; }); }

int cref_get_velocity(void* h, double* v) {
  return dispatch(h, [&](auto& P) { back(P.v.data(), v, 3 * P.nl); return 0; });
}

int cref_get_final_state(void* h, double* m1) {
  return dispatch(h, [&](auto& P) { back(P.m.data() + (size_t)P.nt * P.nl, m1, P.nl); return 0; });
}

// stats (20 doubles): J, D, R, J0, D0, gnorm, g0, iter, pcg_total, reason,
// rel_mismatch, seconds, obj, grad, hessmatvec, pcmatvec, pdesolve,
// scalar gathers, 3D real transforms, krylov_g0
int cref_stats(void* h, double* out) {
  return dispatch(h, [&](auto& P) {
    const double s[20] = {P.J, P.D, P.Rv, P.J0, P.D0, P.gnorm, P.g0, (double)P.iter, (double)P.pcg_total,
                          (double)P.reason, P.rel_mismatch, P.seconds, (double)P.cnt.obj, (double)P.cnt.grad,
                          (double)P.cnt.hessmatvec, (double)P.cnt.pcmatvec, (double)P.cnt.pdesolve,
                          (double)P.cnt.gathers, (double)P.cnt.ffts, P.krylov_g0};
    std::memcpy(out, s, sizeof(s));
    return 0;
  });
}

// lambda at t = 0 and the body force hd b of the last gradient or Hessian
// matvec (the incremental adjoint and body force after a matvec)
int cref_last_adjoint(void* h, double* lam0, double* body_force) {
  return dispatch(h, [&](auto& P) {
    P.last_adjoint(lam0, body_force);
    return 0;
  });
}

int cref_reset_counters(void* h) {
  return dispatch(h, [&](auto& P) { P.cnt = cref::Counters(); return 0; });
}

}  // extern "C"
