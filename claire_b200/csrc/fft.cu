// Batched 3D real FFTs with fused spectral operators, and 1D spectral
// derivatives, for periodic N^3 grids (N in {16,32,48,64,96,128,192,256}).
//
// These replace AccFFT's accfft_execute_r2c_t / accfft_execute_c2r_t /
// accfft_grad_t / accfft_divergence_t at the reference's call sites
// (src/CLAIRE.cpp:2622, 2662, 2695, 3243, 3261, 3911, 3949, 3984;
// src/Regularization*.cpp) and the diagonal "Hadamard" loops that follow
// them (e.g. src/RegularizationH2.cpp:212-244).
//
// 3D transform = three passes over HBM:
//   rows (x3, r2c via pair packing) -> columns x2 -> x1 pencil.
// The x1 pencil pass of the forward transform, the spectral multiply and the
// x1 pass of the inverse transform are one kernel; then columns x2 (inverse)
// and rows (c2r) with a fused epilogue (store / accumulate / sum of squares).
// Spectral derivatives are separable: d/dx_k of a periodic field only needs
// the 1D transform along axis k, so gradient and divergence are one pass per
// axis over real data.
//
// Every global->shared load is two-phase: a thread issues all of its loads
// into registers (compile-time count) before it stores any of them, so each
// thread keeps 8-32 independent loads in flight.
#include <atomic>
#include <cstdio>
#include <mutex>
#include <vector>

#include "fft_engine.cuh"
#include "spectral.cuh"
#include "reduce.cuh"

namespace cb {

// ---------------------------------------------------------------------------
// twiddle tables W_N^m = exp(-2 pi i m / N), computed in double on the host
// ---------------------------------------------------------------------------
static std::mutex g_tw_mutex;
static std::vector<std::pair<long long, float2*>> g_tw;  // key: device*1024 + N

static const float2* twiddles(int n) {
  int dev = 0;
  cudaGetDevice(&dev);
  long long key = (long long)dev * 1024 + n;
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  for (auto& e : g_tw)
    if (e.first == key) return e.second;
  std::vector<float2> h(n);
  for (int m = 0; m < n; ++m) {
    double a = kTwoPi * (double)m / (double)n;
    h[m] = make_float2((float)cos(a), (float)(-sin(a)));
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(float2)) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
  g_tw.push_back({key, d});
  return d;
}

// Lengths with a plan on every axis, and the extra lengths the column and
// pencil passes (axes x1, x2) also take: 150 = 10 x 15 (the x2 length of the
// reference's example brains, 128 x 150 x 128).  Row passes need N % 16 == 0
// (16-byte row loads, whole float4 per thread).
bool fft_size_supported(int n) {
  switch (n) {
    case 16: case 32: case 48: case 64: case 96: case 128: case 192: case 256: return true;
    default: return false;
  }
}

bool fft_col_size_supported(int n) { return fft_size_supported(n) || n == 150; }

// Packed lines per CTA for row kernels, and columns per CTA for column kernels.
// With 256 threads and at least 32 lines a warp's lanes are 32 consecutive
// lines at one element index in every radix stage, so the split re / im
// arrays (odd line pitch) are read and written without bank conflicts; grids
// of 192 and 256 points use 16 lines to keep two CTAs per SM.  Variant bit 1
// selects the alternative line counts the autotuner tries (row chunks must
// split into whole float4 per thread: P * N % 512 == 0; the 4-field pencil of
// 256 points keeps 16 columns to fit shared memory).
template <int N> struct RowLines {
  static constexpr int base = N <= 32 ? 64 : (N <= 128 ? 32 : 16);
  static constexpr int alt = N == 16 ? 32 : (N == 32 ? 32 : (N == 48 ? 64 : (N <= 128 ? 16 : 32)));
};
template <int N> struct ColLines {
  static constexpr int base = N <= 128 ? 32 : 16;
  static constexpr int alt = N <= 128 ? 16 : (N == 192 ? 32 : 16);
};
template <int N, int V = 0> struct RowCfg {
  static constexpr int P = (V & 2) ? RowLines<N>::alt : RowLines<N>::base;
  static constexpr int PITCH = P + 1;
};
template <int N, int V = 0> struct ColCfg {
  static constexpr int C = (V & 2) ? ColLines<N>::alt : ColLines<N>::base;
  // 16 lines: pitch 16 with rotated first-stage writes (RotateFirst); 32
  // lines: odd pitch (a warp's lanes are the 32 lines at one element)
  static constexpr int PITCH = C == 16 ? 16 : C + 1;
};

constexpr int kThreads = kFftThreads;

// Epilogue of the row kernels: value of row r, element e sits at
// ((r & 1) ? im : re)[e * PITCH + r / 2]; store it, add it to dst, or
// accumulate its square.  For EPI_ADD the old values of a group of 8 elements
// are loaded before any of them is stored, so the loads overlap.
template <int N, int P, int PITCH>
CB_DEVICE double rows_epilogue(const float* re, const float* im, float* __restrict__ dst,
                               const float* __restrict__ other, int row0, int nr, int epi, float al) {
  constexpr int TOTAL = 2 * P * N;
  constexpr int G = 8;
  const bool add = (epi == EPI_ADD || epi == EPI_ADD_DOT);
  const bool dot = (epi == EPI_STORE_DOT || epi == EPI_ADD_DOT);
  double acc = 0.0;
  for (int i0 = threadIdx.x; i0 < TOTAL; i0 += G * kThreads) {
    float old[G], oth[G];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int idx = i0 + u * kThreads;
      const int r = idx / N, e = idx - r * N;
      const bool in = idx < TOTAL && r < nr;
      const long long gi = (long long)(row0 + r) * N + e;
      old[u] = (add && in) ? dst[gi] : 0.f;
      oth[u] = (dot && in) ? other[gi] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int idx = i0 + u * kThreads;
      const int r = idx / N, e = idx - r * N;
      if (idx >= TOTAL || r >= nr) continue;
      const float val = al * ((r & 1) ? im : re)[e * PITCH + (r >> 1)];
      const long long gi = (long long)(row0 + r) * N + e;
      if (epi == EPI_SUMSQ) {
        acc += (double)val * (double)val;
        continue;
      }
      const float nv = add ? old[u] + val : val;
      dst[gi] = nv;
      if (dot) acc += (double)nv * (double)oth[u];
    }
  }
  return acc;
}

CB_DEVICE bool epi_reduces(int epi) { return epi == EPI_SUMSQ || epi == EPI_STORE_DOT || epi == EPI_ADD_DOT; }

// ---------------------------------------------------------------------------
// load helpers
// ---------------------------------------------------------------------------
// Column tile: N elements (es apart) of the thread's column into split
// re/im shared arrays.  The thread owns column c = tid % C and rows
// e = tid / C + k * (kThreads / C).  colp == nullptr loads zeros.
// Lengths that RSTEP does not divide (150) take K = ceil(N / RSTEP) steps and
// skip the elements e >= N; for the others the test is compile-time true.
template <int N, int RSTEP>
CB_DEVICE bool in_line(int e) {
  return (N % RSTEP == 0) || e < N;
}

template <int N, int C, int PITCH>
CB_DEVICE void load_col_tile(float* re, float* im, const float2* __restrict__ colp, long long es) {
  constexpr int RSTEP = kThreads / C;
  constexpr int K = (N + RSTEP - 1) / RSTEP;
  const int c = threadIdx.x % C, e0 = threadIdx.x / C;
  float2 v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = e0 + k * RSTEP;
    v[k] = (colp && in_line<N, RSTEP>(e)) ? __ldg(colp + (long long)e * es) : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = e0 + k * RSTEP;
    if (!in_line<N, RSTEP>(e)) continue;
    re[e * PITCH + c] = v[k].x;
    im[e * PITCH + c] = v[k].y;
  }
}

template <int N, int C, int PITCH>
CB_DEVICE void store_col_tile(const float* re, const float* im, float2* __restrict__ colp, long long es) {
  constexpr int RSTEP = kThreads / C;
  constexpr int K = (N + RSTEP - 1) / RSTEP;
  const int c = threadIdx.x % C, e0 = threadIdx.x / C;
  if (!colp) return;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = e0 + k * RSTEP;
    if (!in_line<N, RSTEP>(e)) continue;
    colp[(long long)e * es] = make_float2(re[e * PITCH + c], im[e * PITCH + c]);
  }
}

// Row chunk: 2P contiguous real rows of N floats -> pair-packed complex lines
// (row 2p -> real part, row 2p+1 -> imaginary part of line p).  float4 loads.
template <int N, int P, int PITCH>
CB_DEVICE void load_row_chunk(float* re, float* im, const float* __restrict__ src, int nr) {
  constexpr int Q = 2 * P * N / 4;          // float4s in the chunk
  constexpr int K = Q / kThreads;           // per thread (exact for all plans)
  static_assert(Q % kThreads == 0, "row chunk must split evenly");
  float4 v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int q = threadIdx.x + k * kThreads;
    const int r = (4 * q) / N;
    v[k] = (r < nr) ? __ldg(reinterpret_cast<const float4*>(src) + q) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  // lane l writes its four elements in the order rotated by l / 8, so the 32
  // lanes of each store hit 32 distinct banks (e * PITCH strides otherwise
  // fold four lanes onto one bank)
  const int rot = (threadIdx.x >> 3) & 3;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int q = threadIdx.x + k * kThreads;
    const int r = (4 * q) / N, e = 4 * q - r * N;
    float* dst = ((r & 1) ? im : re) + (r >> 1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = (i + rot) & 3;
      const float val = c == 0 ? v[k].x : (c == 1 ? v[k].y : (c == 2 ? v[k].z : v[k].w));
      dst[(e + c) * PITCH] = val;
    }
  }
}

// ---------------------------------------------------------------------------
// rows: r2c along x3.  Two real rows a, b are packed as z = a + i b; after
// the complex FFT Z, A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / 2i.
// ---------------------------------------------------------------------------
template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_r2c_rows(const float* __restrict__ in, long long ip,
                                                        long long ifs, float2* __restrict__ out,
                                                        long long op, long long ofs, int nrows,
                                                        const float2* __restrict__ twg,
                                                        const int* __restrict__ active) {
  constexpr int P = RowCfg<N, V>::P, PITCH = RowCfg<N, V>::PITCH, NH = N / 2 + 1;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* re = smem + 2 * N;
  float* im = re + N * PITCH;
  float* sre = im + N * PITCH;
  float* sim = sre + N * PITCH;
  const float* src = in + blockIdx.z * ip + blockIdx.y * ifs;
  float2* dst = out + blockIdx.z * op + blockIdx.y * ofs;
  const int row0 = blockIdx.x * 2 * P;
  const int nr = min(2 * P, nrows - row0);
  load_twiddles<N>(tw, twg);
  load_row_chunk<N, P, PITCH>(re, im, src + (long long)row0 * N, nr);
  __syncthreads();
  fft_lines<N, false, P, PITCH, V>(re, im, sre, sim, tw);
  for (int idx = threadIdx.x; idx < 2 * P * NH; idx += kThreads) {
    const int r = idx / NH, k = idx - r * NH;
    if (r >= nr) continue;
    const int line = r >> 1;
    const int km = (k == 0) ? 0 : N - k;
    const float zr = re[k * PITCH + line], zi = im[k * PITCH + line];
    const float mr = re[km * PITCH + line], mi = im[km * PITCH + line];
    float2 x;
    if (r & 1) x = make_float2(0.5f * (zi + mi), -0.5f * (zr - mr));
    else x = make_float2(0.5f * (zr + mr), 0.5f * (zi - mi));
    dst[(long long)(row0 + r) * NH + k] = x;
  }
}

// ---------------------------------------------------------------------------
// rows: c2r along x3 with epilogue.  Z[k] = A[k] + i B[k], Z[N-k] =
// conj(A[k]) + i conj(B[k]); the imaginary parts of the DC and Nyquist bins
// are ignored (the c2r convention of FFTW / pocketfft).
// ---------------------------------------------------------------------------
template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_c2r_rows(const float2* __restrict__ in, long long ip,
                                                        long long ifs, float* __restrict__ out,
                                                        long long op, long long ofs, int nrows,
                                                        const float2* __restrict__ twg, int epi,
                                                        const float* __restrict__ alpha,
                                                        double* __restrict__ partials, int nparts,
                                                        const float* __restrict__ other,
                                                        const int* __restrict__ active) {
  constexpr int P = RowCfg<N, V>::P, PITCH = RowCfg<N, V>::PITCH, NH = N / 2 + 1;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* re = smem + 2 * N;
  float* im = re + N * PITCH;
  float* sre = im + N * PITCH;
  float* sim = sre + N * PITCH;
  // staging of the 2P half-spectrum rows: it is dead before the transform
  // starts, so it shares the transform's scratch (sre / sim) when that is large
  // enough (row_smem sizes the block for the larger of the two)
  float* str = sre;
  float* sti = str + 2 * P * NH;
  const float2* src = in + blockIdx.z * ip + blockIdx.y * ifs;
  float* dst = out ? out + blockIdx.z * op + blockIdx.y * ofs : nullptr;
  const float* oth = other ? other + blockIdx.z * op + blockIdx.y * ofs : nullptr;
  const int row0 = blockIdx.x * 2 * P;
  const int nr = min(2 * P, nrows - row0);
  load_twiddles<N>(tw, twg);
  {
    // two-phase load of the 2P x NH complex chunk (contiguous)
    constexpr int TOT = 2 * P * NH;
    constexpr int K = (TOT + kThreads - 1) / kThreads;
    const float2* s0 = src + (long long)row0 * NH;
    float2 v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int idx = threadIdx.x + k * kThreads;
      v[k] = (idx < TOT && idx / NH < nr) ? __ldg(s0 + idx) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int idx = threadIdx.x + k * kThreads;
      if (idx >= TOT) continue;
      const int kk = idx % NH;
      float2 w = v[k];
      if (kk == 0 || kk == N / 2) w.y = 0.f;
      str[idx] = w.x;
      sti[idx] = w.y;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < P * N; idx += kThreads) {
    const int line = idx / N, e = idx - line * N;
    const int a = 2 * line, b = 2 * line + 1;
    float zr, zi;
    if (e <= N / 2) {
      const float ar = str[a * NH + e], ai = sti[a * NH + e];
      const float br = str[b * NH + e], bi = sti[b * NH + e];
      zr = ar - bi;
      zi = ai + br;
    } else {
      const int k = N - e;
      const float ar = str[a * NH + k], ai = -sti[a * NH + k];
      const float br = str[b * NH + k], bi = -sti[b * NH + k];
      zr = ar - bi;
      zi = ai + br;
    }
    re[e * PITCH + line] = zr;
    im[e * PITCH + line] = zi;
  }
  __syncthreads();
  fft_lines<N, true, P, PITCH, V>(re, im, sre, sim, tw);
  const float al = alpha ? alpha[blockIdx.z] : 1.f;
  const double acc = rows_epilogue<N, P, PITCH>(re, im, dst, oth, row0, nr, epi, al);
  if (epi_reduces(epi)) {
    block_reduce_store(acc, partials + (long long)blockIdx.z * nparts, blockIdx.x + gridDim.x * blockIdx.y);
  }
}

// ---------------------------------------------------------------------------
// complex column FFT along a strided axis, in place
// column g starts at (g / cpg) * gs + (g % cpg); elements are es apart
// ---------------------------------------------------------------------------
template <int N, bool INV, int V>
__global__ void __launch_bounds__(kThreads) k_cols(float2* __restrict__ data, long long pstr,
                                                    long long fstr, int ncols, int cpg, long long gs,
                                                    long long es, const float2* __restrict__ twg,
                                                    const int* __restrict__ active) {
  constexpr int C = ColCfg<N, V>::C, PITCH = ColCfg<N, V>::PITCH;
  using PL = Plan<N, V>;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* sre = smem + 2 * N;
  float* sim = sre + N * PITCH;
  float2* base = data + blockIdx.z * pstr + blockIdx.y * fstr;
  const int g = blockIdx.x * C + threadIdx.x % C;
  float2* colp = (g < ncols) ? base + (long long)(g / cpg) * gs + (g % cpg) : nullptr;
  load_twiddles<N>(tw, twg);
  // first stage straight from the columns, last stage straight back: every
  // column element passes through shared memory once (in place: all reads of
  // the CTA's columns finish before the barrier, all writes follow it)
  fft_stage_load<N, PL::R0, INV, C, PITCH>(colp, es, sre, sim);
  __syncthreads();
  fft_stage_store<N, PL::R1, PL::R0, INV, C, PITCH>(sre, sim, tw, colp, es);
}

// ---------------------------------------------------------------------------
// spectral symbols (src/Regularization*.cpp, src/CLAIREStokes.cpp:407-540,
// src/CLAIREDivReg.cpp:313-460, src/Preprocessing.cpp:1956-2056)
// ---------------------------------------------------------------------------
CB_DEVICE float reg_grad_symbol(const SpecParams& q, float kap) {
  switch (q.norm) {
    case NORM_L2: return q.beta0;
    case NORM_H1SN: return q.hd * q.beta0 * kap;
    case NORM_H1: return q.hd * q.beta0 * (kap + q.beta1);
    case NORM_H2: return q.beta0 * (kap * kap + q.beta1);
    case NORM_H2SN: return q.hd * q.beta0 * kap * kap;
    case NORM_H3: return q.beta0 * (kap * kap * kap + q.beta1);
    case NORM_H3SN: return q.beta0 * kap * kap * kap;
    default: return 0.f;
  }
}

CB_DEVICE float reg_inv_operator(const SpecParams& q, float kap) {
  switch (q.norm) {
    case NORM_L2: return q.beta0;
    case NORM_H1SN: return kap == 0.f ? q.beta0 : q.beta0 * kap;
    case NORM_H1: return q.beta0 * (kap + q.beta1);
    case NORM_H2: return q.beta0 * (kap * kap + q.beta1);
    case NORM_H2SN: return kap == 0.f ? q.beta0 : q.beta0 * kap * kap;
    case NORM_H3: return q.beta0 * (kap * kap * kap + q.beta1);
    case NORM_H3SN: return kap == 0.f ? q.beta0 : q.beta0 * kap * kap * kap;
    default: return 1.f;
  }
}

// Wavenumber data of one spectral column (x2 index i2, x3 index i3) and a
// spectral element of it along x1 (index i1).
struct ColumnK {
  float k2, k3, l2, l3;   // Nyquist-zeroed and Nyquist-kept wavenumbers
};

CB_DEVICE ColumnK column_k(int i2, int i3, const Dims& d) {
  ColumnK c;
  c.k2 = (float)wavenumber(i2, d.n2);
  c.k3 = (float)wavenumber(i3, d.n3);
  c.l2 = (float)wavenumber_keep_nyquist(i2, d.n2);
  c.l3 = (float)wavenumber_keep_nyquist(i3, d.n3);
  return c;
}

// Per-field diagonal operators (one field, component index comp for H3/H3SN).
CB_DEVICE float2 apply_op1(int op, const SpecParams& q, const Dims& d, int i1, const ColumnK& ck, int comp,
                           float2 x, float s) {
  const float k1 = (float)wavenumber(i1, d.n1);
  const float kap = k1 * k1 + ck.k2 * ck.k2 + ck.k3 * ck.k3;
  switch (op) {
    case OP_REG_GRAD: {
      const float sig = s * reg_grad_symbol(q, kap);
      return make_float2(x.x * sig, x.y * sig);
    }
    case OP_REG_INV:
    case OP_REG_SQRTINV: {
      float o = reg_inv_operator(q, kap);
      if (op == OP_REG_SQRTINV) o = sqrtf(o);
      const float sig = s / o;
      return make_float2(x.x * sig, x.y * sig);
    }
    case OP_REG_FUNC: {
      if (q.norm == NORM_L2) {
        const float sig = s * sqrtf(q.beta0);
        return make_float2(x.x * sig, x.y * sig);
      }
      if (q.norm == NORM_H2) {
        const float sig = s * sqrtf(q.beta0) * (-kap + sqrtf(q.beta1));
        return make_float2(x.x * sig, x.y * sig);
      }
      if (q.norm == NORM_H2SN) {
        const float sig = -s * kap;
        return make_float2(x.x * sig, x.y * sig);
      }
      // H3 / H3SN: separate multipliers on real and imaginary parts
      const float kc = comp == 0 ? k1 : (comp == 1 ? ck.k2 : ck.k3);
      const float a = kc * (-kap);
      float mre, mim;
      if (q.norm == NORM_H3) {
        const float sb0 = sqrtf(q.beta0), sb1 = sqrtf(q.beta1);
        mre = s * sb0 * (a + sb1);
        mim = s * sb0 * (-a + sb1);
      } else {
        mre = s * a;
        mim = -s * a;
      }
      return make_float2(x.x * mre, x.y * mim);
    }
    case OP_GAUSS: {
      const float l1 = (float)wavenumber_keep_nyquist(i1, d.n1);
      const float c1 = q.sigma[0] * (float)(kTwoPi / d.n1), c2 = q.sigma[1] * (float)(kTwoPi / d.n2),
                  c3 = q.sigma[2] * (float)(kTwoPi / d.n3);
      const float sik = expf(-0.5f * (l1 * l1 * c1 * c1 + ck.l2 * ck.l2 * c2 * c2 + ck.l3 * ck.l3 * c3 * c3));
      return make_float2(x.x * s * sik, x.y * s * sik);
    }
    default:
      return make_float2(x.x * s, x.y * s);
  }
}

// Coupled 3-field projections b -> F^-1(-c k (k . b^)/kappa): Stokes keeps the
// Nyquist index in kappa, the relaxed model zeroes it and scales by
// c = (beta_v (beta_w (kappa + 1))^-1 + 1)^-1.
CB_DEVICE void apply_op3(int op, const SpecParams& q, const Dims& d, int i1, const ColumnK& ck, float2 (&x)[3],
                         float s) {
  const float k1 = (float)wavenumber(i1, d.n1);
  const float kap = k1 * k1 + ck.k2 * ck.k2 + ck.k3 * ck.k3;
  float kl, c = 1.f;
  if (op == OP_LERAY) {
    const float l1 = (float)wavenumber_keep_nyquist(i1, d.n1);
    kl = l1 * l1 + ck.l2 * ck.l2 + ck.l3 * ck.l3;
  } else {
    kl = kap;
    const float opik = 1.f / (q.beta2 * (kap + 1.f));
    c = 1.f / (q.beta0 * opik + 1.f);
  }
  const float L = (kl == 0.f) ? -1.f : -1.f / kl;
  const float2 kd = make_float2(k1 * x[0].x + ck.k2 * x[1].x + ck.k3 * x[2].x,
                                k1 * x[0].y + ck.k2 * x[1].y + ck.k3 * x[2].y);
  const float g = s * c * L;
  x[0] = make_float2(g * k1 * kd.x, g * k1 * kd.y);
  x[1] = make_float2(g * ck.k2 * kd.x, g * ck.k2 * kd.y);
  x[2] = make_float2(g * ck.k3 * kd.x, g * ck.k3 * kd.y);
}

// x1 pencil, one field per CTA (grid.y = field): forward FFT along x1, the
// diagonal symbol, inverse FFT.
template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_pencil1(float2* __restrict__ spec, long long pstr, long long fstr,
                                                       Dims d, int op, const SpecParams* __restrict__ params,
                                                       const float2* __restrict__ twg,
                                                       const int* __restrict__ active) {
  constexpr int C = ColCfg<N, V>::C, PITCH = ColCfg<N, V>::PITCH;
  constexpr int RSTEP = kThreads / C, K = (N + RSTEP - 1) / RSTEP;
  using PL = Plan<N, V>;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* re = smem + 2 * N;
  float* im = re + N * PITCH;
  float* sre = im + N * PITCH;
  float* sim = sre + N * PITCH;
  const int n3h = d.n3 / 2 + 1;
  const int ncols = d.n2 * n3h;
  const int c = threadIdx.x % C, e0 = threadIdx.x / C;
  const int g = blockIdx.x * C + c;
  float2* colp = (g < ncols) ? spec + blockIdx.z * pstr + blockIdx.y * fstr + g : nullptr;
  const SpecParams q = params[blockIdx.z];
  const ColumnK ck = column_k(g / n3h, g % n3h, d);
  const float s = 1.f / (float)((double)d.n1 * d.n2 * d.n3);
  load_twiddles<N>(tw, twg);
  // forward transform: first stage straight from the column, second into (re, im)
  fft_stage_load<N, PL::R0, false, C, PITCH>(colp, ncols, sre, sim);
  __syncthreads();
  fft_stage<N, PL::R1, PL::R0, false, C, PITCH>(sre, sim, re, im, tw);
  __syncthreads();
  // one copy of the symbol code (a rolled loop keeps the kernel small enough
  // for the instruction cache)
#pragma unroll 1
  for (int k = 0; k < K; ++k) {
    const int e = e0 + k * RSTEP;
    if (!in_line<N, RSTEP>(e)) continue;
    const int a = e * PITCH + c;
    const float2 y = apply_op1(op, q, d, e, ck, blockIdx.y, make_float2(re[a], im[a]), s);
    re[a] = y.x;
    im[a] = y.y;
  }
  __syncthreads();
  // inverse transform: first stage in shared memory, last straight to the column
  fft_stage<N, PL::R0, 1, true, C, PITCH>(re, im, sre, sim, tw);
  __syncthreads();
  fft_stage_store<N, PL::R1, PL::R0, true, C, PITCH>(sre, sim, tw, colp, ncols);
}

// x1 pencil with the three fields in one CTA (coupled projections).
template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_pencil3(float2* __restrict__ spec, long long pstr, long long fstr,
                                                       Dims d, int op, const SpecParams* __restrict__ params,
                                                       const float2* __restrict__ twg,
                                                       const int* __restrict__ active) {
  constexpr int C = ColCfg<N, V>::C, PITCH = ColCfg<N, V>::PITCH;
  constexpr int RSTEP = kThreads / C, K = (N + RSTEP - 1) / RSTEP;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* sre = smem + 2 * N;
  float* sim = sre + N * PITCH;
  float* fre[3];
  float* fim[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    fre[f] = sim + N * PITCH + 2 * f * N * PITCH;
    fim[f] = fre[f] + N * PITCH;
  }
  const int n3h = d.n3 / 2 + 1;
  const int ncols = d.n2 * n3h;
  const int c = threadIdx.x % C, e0 = threadIdx.x / C;
  const int g = blockIdx.x * C + c;
  float2* colp = (g < ncols) ? spec + blockIdx.z * pstr + g : nullptr;
  const SpecParams q = params[blockIdx.z];
  const ColumnK ck = column_k(g / n3h, g % n3h, d);
  const float s = 1.f / (float)((double)d.n1 * d.n2 * d.n3);
  using PL = Plan<N, V>;
  load_twiddles<N>(tw, twg);
  // forward transforms: first stage straight from each field's column into
  // the scratch, second stage into the field's lines
#pragma unroll 1
  for (int f = 0; f < 3; ++f) {
    fft_stage_load<N, PL::R0, false, C, PITCH>(colp ? colp + f * fstr : nullptr, ncols, sre, sim);
    __syncthreads();
    fft_stage<N, PL::R1, PL::R0, false, C, PITCH>(sre, sim, fre[f], fim[f], tw);
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int e = e0 + k * RSTEP;
    if (!in_line<N, RSTEP>(e)) continue;
    const int a = e * PITCH + c;
    float2 x[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) x[f] = make_float2(fre[f][a], fim[f][a]);
    apply_op3(op, q, d, e, ck, x, s);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      fre[f][a] = x[f].x;
      fim[f][a] = x[f].y;
    }
  }
  __syncthreads();
  // inverse transforms: first stage into the scratch, last straight to the column
#pragma unroll 1
  for (int f = 0; f < 3; ++f) {
    fft_stage<N, PL::R0, 1, true, C, PITCH>(fre[f], fim[f], sre, sim, tw);
    __syncthreads();
    fft_stage_store<N, PL::R1, PL::R0, true, C, PITCH>(sre, sim, tw, colp ? colp + f * fstr : nullptr, ncols);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// 1D spectral derivative of real fields.  Two real lines a, b are packed as
// a + i b; i*k/N with the Nyquist wavenumber zeroed is Hermitian, so the real
// and imaginary parts of the result are the derivatives of a and b.
// AXIS 2: rows (x3, contiguous).  AXIS 0/1: columns along x1 / x2.
// ---------------------------------------------------------------------------
template <int N, int NL, int PITCH>
CB_DEVICE void mul_ik(float* re, float* im, float hscale) {
  for (int idx = threadIdx.x; idx < NL * N; idx += kThreads) {
    const int e = idx / NL, p = idx - e * NL;
    const float k = (float)wavenumber(e, N) * hscale;
    const int a = e * PITCH + p;
    const float xr = re[a], xi = im[a];
    re[a] = -k * xi;
    im[a] = k * xr;
  }
}

template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_deriv_rows(const float* __restrict__ in, long long ip,
                                                          long long ifs, float* __restrict__ out,
                                                          long long op, long long ofs, int nrows,
                                                          const float2* __restrict__ twg, int epi,
                                                          double* __restrict__ partials, int nparts,
                                                          const int* __restrict__ active) {
  constexpr int P = RowCfg<N, V>::P, PITCH = RowCfg<N, V>::PITCH;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* re = smem + 2 * N;
  float* im = re + N * PITCH;
  float* sre = im + N * PITCH;
  float* sim = sre + N * PITCH;
  const float* src = in + blockIdx.z * ip + blockIdx.y * ifs;
  float* dst = out ? out + blockIdx.z * op + blockIdx.y * ofs : nullptr;
  const int row0 = blockIdx.x * 2 * P;
  const int nr = min(2 * P, nrows - row0);
  load_twiddles<N>(tw, twg);
  load_row_chunk<N, P, PITCH>(re, im, src + (long long)row0 * N, nr);
  __syncthreads();
  fft_lines<N, false, P, PITCH, V>(re, im, sre, sim, tw);
  mul_ik<N, P, PITCH>(re, im, 1.f / (float)N);
  __syncthreads();
  fft_lines<N, true, P, PITCH, V>(re, im, sre, sim, tw);
  const double acc = rows_epilogue<N, P, PITCH>(re, im, dst, nullptr, row0, nr, epi, 1.f);
  if (epi == EPI_SUMSQ)
    block_reduce_store(acc, partials + (long long)blockIdx.z * nparts, blockIdx.x + gridDim.x * blockIdx.y);
}

// Column derivative: the thread's packed line p holds real columns 2p (real
// part) and 2p + 1 (imaginary part); the forward transform's first stage reads
// them from global memory, its last stage multiplies by i k / N on the way to
// shared memory, and the inverse transform's last stage hands both columns to
// the epilogue (store, add, or sum of squares) straight from registers.
template <int N>
struct DerivColLoad {
  const float* src;
  long long ca, cb, es;
  bool oka, okb;
  CB_DEVICE float2 operator()(int, int e) const {
    return make_float2(oka ? __ldg(src + ca + (long long)e * es) : 0.f, okb ? __ldg(src + cb + (long long)e * es) : 0.f);
  }
};

template <int N, int PITCH>
struct MulIkStore {
  float* re;
  float* im;
  CB_DEVICE void operator()(int p, int e, float2 v) const {
    const float k = (float)wavenumber(e, N) * (1.f / (float)N);
    re[e * PITCH + p] = -k * v.y;
    im[e * PITCH + p] = k * v.x;
  }
};

struct DerivColEpi {
  float* dst;
  long long ca, cb, es;
  bool oka, okb;
  int epi;
  double* acc;
  CB_DEVICE void put(long long c, float val) const {
    if (epi == EPI_SUMSQ) *acc += (double)val * (double)val;  // no output array needed
    else if (!dst) return;
    else if (epi == EPI_STORE) dst[c] = val;
    else if (epi == EPI_ADD) dst[c] = dst[c] + val;
  }
  CB_DEVICE void operator()(int, int e, float2 v) const {
    if (oka) put(ca + (long long)e * es, v.x);
    if (okb) put(cb + (long long)e * es, v.y);
  }
};

template <int N, int V>
__global__ void __launch_bounds__(kThreads) k_deriv_cols(const float* __restrict__ in, long long ip,
                                                          long long ifs, float* __restrict__ out,
                                                          long long op, long long ofs, int ncols,
                                                          int cpg, long long gs, long long es,
                                                          const float2* __restrict__ twg, int epi,
                                                          double* __restrict__ partials, int nparts,
                                                          const int* __restrict__ active) {
  constexpr int L = ColCfg<N, V>::C;       // packed complex lines per CTA
  constexpr int PITCH = ColCfg<N, V>::PITCH;
  using PL = Plan<N, V>;
  if (active && !active[blockIdx.z]) return;
  extern __shared__ float smem[];
  float2* tw = reinterpret_cast<float2*>(smem);
  float* re = smem + 2 * N;
  float* im = re + N * PITCH;
  float* sre = im + N * PITCH;
  float* sim = sre + N * PITCH;
  const float* src = in + blockIdx.z * ip + blockIdx.y * ifs;
  float* dst = out ? out + blockIdx.z * op + blockIdx.y * ofs : nullptr;
  const int p = threadIdx.x % L;
  const int ga = blockIdx.x * 2 * L + 2 * p, gb = ga + 1;
  const bool oka = ga < ncols, okb = gb < ncols;
  const long long ca = oka ? (long long)(ga / cpg) * gs + (ga % cpg) : 0;
  const long long cb = okb ? (long long)(gb / cpg) * gs + (gb % cpg) : 0;
  load_twiddles<N>(tw, twg);
  fft_stage_in<N, PL::R0, false, L, PITCH>(DerivColLoad<N>{src, ca, cb, es, oka, okb}, sre, sim);
  __syncthreads();
  fft_stage_out<N, PL::R1, PL::R0, false, L, PITCH>(sre, sim, tw, MulIkStore<N, PITCH>{re, im});
  __syncthreads();
  fft_stage<N, PL::R0, 1, true, L, PITCH>(re, im, sre, sim, tw);
  __syncthreads();
  double acc = 0.0;
  fft_stage_out<N, PL::R1, PL::R0, true, L, PITCH>(
      sre, sim, tw, DerivColEpi{dst, ca, cb, es, oka, okb, epi, &acc});
  if (epi == EPI_SUMSQ)
    block_reduce_store(acc, partials + (long long)blockIdx.z * nparts, blockIdx.x + gridDim.x * blockIdx.y);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <int N, int V> static size_t row_smem(bool c2r) {
  const size_t scratch = 2 * N * RowCfg<N, V>::PITCH;           // sre + sim
  const size_t staging = 2 * 2 * RowCfg<N, V>::P * (N / 2 + 1);  // c2r half-spectrum rows (shares scratch)
  const size_t tail = (c2r && staging > scratch) ? staging : scratch;
  return (2 * N + 2 * N * RowCfg<N, V>::PITCH + tail) * sizeof(float);
}
template <int N, int V> static size_t col_smem(int nbuf) {
  return (2 * N + 2 * nbuf * N * ColCfg<N, V>::PITCH) * sizeof(float);
}

template <typename K> static int set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024 && !g_graph_capture) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
  }
  return 0;
}

static bool aligned16(const void* p) { return (reinterpret_cast<unsigned long long>(p) & 15) == 0; }

#define CB_DISPATCH_N(n, CALL)                         \
  switch (n) {                                         \
    case 16: { constexpr int NN = 16; CALL; } break;   \
    case 32: { constexpr int NN = 32; CALL; } break;   \
    case 48: { constexpr int NN = 48; CALL; } break;   \
    case 64: { constexpr int NN = 64; CALL; } break;   \
    case 96: { constexpr int NN = 96; CALL; } break;   \
    case 128: { constexpr int NN = 128; CALL; } break; \
    case 192: { constexpr int NN = 192; CALL; } break; \
    case 256: { constexpr int NN = 256; CALL; } break; \
    default: return (int)cudaErrorInvalidValue;        \
  }

// ---------------------------------------------------------------------------
// FFT variants (plan factorization x lines per CTA) chosen per grid size.
// The table is process-wide; the autotuner (fft_autotune) or
// set_fft_variant change it, and every launch reads it, so it must only
// change while no transform of that size is in flight (contexts tune when
// they are created, before any of their work).
// ---------------------------------------------------------------------------
static std::atomic<int> g_fft_var[9];

static int size_slot(int n) {
  switch (n) {
    case 16: return 0;
    case 32: return 1;
    case 48: return 2;
    case 64: return 3;
    case 96: return 4;
    case 128: return 5;
    case 192: return 6;
    case 256: return 7;
    case 150: return 8;
    default: return -1;
  }
}

int fft_variant_candidates(int n, int* out) {
  const int k = size_slot(n);
  if (k < 0) return 0;
  if (n == 16 || n == 256) {  // one factorization: line counts only
    out[0] = 0;
    out[1] = 2;
    return 2;
  }
  if (n == 150) {  // column passes only, one line count: radix orders only
    out[0] = 0;
    out[1] = 1;
    return 2;
  }
  for (int v = 0; v < 4; ++v) out[v] = v;
  return 4;
}

int fft_variant(int n) {
  const int k = size_slot(n);
  return k < 0 ? 0 : g_fft_var[k].load(std::memory_order_relaxed);
}

int set_fft_variant(int n, int v) {
  int cand[4];
  const int nc = fft_variant_candidates(n, cand);
  for (int i = 0; i < nc; ++i)
    if (cand[i] == v) {
      g_fft_var[size_slot(n)].store(v, std::memory_order_relaxed);
      return 0;
    }
  return (int)cudaErrorInvalidValue;
}

#define CB_V(VV_, CALL) \
  case VV_: {           \
    constexpr int VV = VV_; \
    CALL;               \
  } break;
#define CB_VSW4(N_, CALL)                                                                  \
  {                                                                                        \
    constexpr int NN = N_;                                                                 \
    switch (fft_variant(N_)) { CB_V(0, CALL) CB_V(1, CALL) CB_V(2, CALL) CB_V(3, CALL)     \
      default: return (int)cudaErrorInvalidValue; }                                        \
  } break;
#define CB_VSW2(N_, CALL)                                                                  \
  {                                                                                        \
    constexpr int NN = N_;                                                                 \
    switch (fft_variant(N_)) { CB_V(0, CALL) CB_V(2, CALL)                                 \
      default: return (int)cudaErrorInvalidValue; }                                        \
  } break;
#define CB_VSW01(N_, CALL)                                                                 \
  {                                                                                        \
    constexpr int NN = N_;                                                                 \
    switch (fft_variant(N_)) { CB_V(0, CALL) CB_V(1, CALL)                                 \
      default: return (int)cudaErrorInvalidValue; }                                        \
  } break;
// CB_DISPATCH_N with the size's current variant as the constexpr VV
#define CB_DISPATCH_NV(n, CALL)      \
  switch (n) {                       \
    case 16: CB_VSW2(16, CALL)       \
    case 32: CB_VSW4(32, CALL)       \
    case 48: CB_VSW4(48, CALL)       \
    case 64: CB_VSW4(64, CALL)       \
    case 96: CB_VSW4(96, CALL)       \
    case 128: CB_VSW4(128, CALL)     \
    case 192: CB_VSW4(192, CALL)     \
    case 256: CB_VSW2(256, CALL)     \
    default: return (int)cudaErrorInvalidValue; \
  }
// the same for column / pencil passes, which also take 150 points
#define CB_DISPATCH_NV_COL(n, CALL)  \
  switch (n) {                       \
    case 16: CB_VSW2(16, CALL)       \
    case 32: CB_VSW4(32, CALL)       \
    case 48: CB_VSW4(48, CALL)       \
    case 64: CB_VSW4(64, CALL)       \
    case 96: CB_VSW4(96, CALL)       \
    case 128: CB_VSW4(128, CALL)     \
    case 150: CB_VSW01(150, CALL)    \
    case 192: CB_VSW4(192, CALL)     \
    case 256: CB_VSW2(256, CALL)     \
    default: return (int)cudaErrorInvalidValue; \
  }

template <int N, int V>
static int r2c_rows_impl(const float* in, long long ip, long long ifs, float2* out, long long op,
                         long long ofs, int nrows, int nf, int nprob, const int* active,
                         cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  size_t sm = row_smem<N, V>(false);
  int e = set_smem(k_r2c_rows<N, V>, sm);
  if (e) return e;
  dim3 grid((nrows + 2 * RowCfg<N, V>::P - 1) / (2 * RowCfg<N, V>::P), nf, nprob);
  k_r2c_rows<N, V><<<grid, kThreads, sm, s>>>(in, ip, ifs, out, op, ofs, nrows, tw, active);
  return (int)cudaGetLastError();
}

template <int N, int V>
static int c2r_rows_impl(const float2* in, long long ip, long long ifs, float* out, long long op,
                         long long ofs, int nrows, int nf, int nprob, int epi, const float* alpha,
                         double* partials, int nparts, const float* other, const int* active, cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  size_t sm = row_smem<N, V>(true);
  int e = set_smem(k_c2r_rows<N, V>, sm);
  if (e) return e;
  dim3 grid((nrows + 2 * RowCfg<N, V>::P - 1) / (2 * RowCfg<N, V>::P), nf, nprob);
  k_c2r_rows<N, V><<<grid, kThreads, sm, s>>>(in, ip, ifs, out, op, ofs, nrows, tw, epi, alpha, partials,
                                            nparts, other, active);
  return (int)cudaGetLastError();
}

template <int N, bool INV, int V>
static int cols_impl(float2* data, long long pstr, long long fstr, int ncols, int cpg, long long gs,
                     long long es, int nf, int nprob, const int* active, cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  size_t sm = col_smem<N, V>(1);  // one line buffer: the first stage reads global memory
  int e = set_smem(k_cols<N, INV, V>, sm);
  if (e) return e;
  dim3 grid((ncols + ColCfg<N, V>::C - 1) / ColCfg<N, V>::C, nf, nprob);
  k_cols<N, INV, V><<<grid, kThreads, sm, s>>>(data, pstr, fstr, ncols, cpg, gs, es, tw, active);
  return (int)cudaGetLastError();
}

template <int N, int V>
static int pencil_impl(float2* spec, long long sp, long long fstr, int nprob, const Dims& d, int op,
                       const SpecParams* params, int nin, int nout, const int* active, cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  const int ncols = d.n2 * (d.n3 / 2 + 1);
  if (op == OP_LERAY || op == OP_LERAY_RELAXED) {
    if (nin != 3 || nout != 3) return (int)cudaErrorInvalidValue;
    size_t sm = col_smem<N, V>(4);
    int e = set_smem(k_pencil3<N, V>, sm);
    if (e) return e;
    dim3 grid((ncols + ColCfg<N, V>::C - 1) / ColCfg<N, V>::C, 1, nprob);
    k_pencil3<N, V><<<grid, kThreads, sm, s>>>(spec, sp, fstr, d, op, params, tw, active);
  } else {
    if (nin != nout) return (int)cudaErrorInvalidValue;
    size_t sm = col_smem<N, V>(2);
    int e = set_smem(k_pencil1<N, V>, sm);
    if (e) return e;
    dim3 grid((ncols + ColCfg<N, V>::C - 1) / ColCfg<N, V>::C, nin, nprob);
    k_pencil1<N, V><<<grid, kThreads, sm, s>>>(spec, sp, fstr, d, op, params, tw, active);
  }
  return (int)cudaGetLastError();
}

// Every axis has its own transform (rows: x3, columns: x2, pencils: x1), so
// grids need not be cubic; each axis length must have a plan.
static bool axes_supported(const Dims& d) {
  return fft_col_size_supported(d.n1) && fft_col_size_supported(d.n2) && fft_size_supported(d.n3);
}
static bool cubic_supported(const Dims& d) { return d.n1 == d.n2 && d.n2 == d.n3 && axes_supported(d); }

int launch_r2c3d(const float* in, long long ip, long long ifs, float2* spec, long long sp, int nf,
                 int nprob, const Dims& d, const int* active, cudaStream_t s) {
  if (!axes_supported(d) || !aligned16(in) || ((ip | ifs) & 3)) return (int)cudaErrorInvalidValue;
  const long long nc = d.nc();
  const int n3h = d.n3 / 2 + 1;
  int e = 0;
  CB_DISPATCH_NV(d.n3, e = (r2c_rows_impl<NN, VV>(in, ip, ifs, spec, sp, nc, d.n1 * d.n2, nf, nprob, active, s)));
  if (e) return e;
  // x2 columns: column g = (i1, k3) starts at i1*n2*n3h + k3, stride n3h
  CB_DISPATCH_NV_COL(d.n2, e = (cols_impl<NN, false, VV>(spec, sp, nc, d.n1 * n3h, n3h, (long long)d.n2 * n3h, n3h,
                                                nf, nprob, active, s)));
  return e;
}

int launch_pencil(float2* spec, long long sp, int nprob, const Dims& d, int op,
                  const SpecParams* dparams, int nin, int nout, const int* active, cudaStream_t s) {
  if (!axes_supported(d)) return (int)cudaErrorInvalidValue;
  int e = 0;
  CB_DISPATCH_NV_COL(d.n1, e = (pencil_impl<NN, VV>(spec, sp, d.nc(), nprob, d, op, dparams, nin, nout, active, s)));
  return e;
}

// Lines per CTA of the size's current variant (min_over_variants: the
// smallest over its candidates, which sizes reduction buffers for any variant).
static int row_lines(int n, bool min_over_variants = false) {
  int base = 0, alt = 0;
  switch (n) {
    case 16: base = RowLines<16>::base; alt = RowLines<16>::alt; break;
    case 32: base = RowLines<32>::base; alt = RowLines<32>::alt; break;
    case 48: base = RowLines<48>::base; alt = RowLines<48>::alt; break;
    case 64: base = RowLines<64>::base; alt = RowLines<64>::alt; break;
    case 96: base = RowLines<96>::base; alt = RowLines<96>::alt; break;
    case 128: base = RowLines<128>::base; alt = RowLines<128>::alt; break;
    case 192: base = RowLines<192>::base; alt = RowLines<192>::alt; break;
    case 256: base = RowLines<256>::base; alt = RowLines<256>::alt; break;
    default: return 0;
  }
  if (min_over_variants) return base < alt ? base : alt;
  return (fft_variant(n) & 2) ? alt : base;
}

static int col_lines(int n, bool min_over_variants = false) {
  int base = 0, alt = 0;
  switch (n) {
    case 16: base = ColLines<16>::base; alt = ColLines<16>::alt; break;
    case 32: base = ColLines<32>::base; alt = ColLines<32>::alt; break;
    case 48: base = ColLines<48>::base; alt = ColLines<48>::alt; break;
    case 64: base = ColLines<64>::base; alt = ColLines<64>::alt; break;
    case 96: base = ColLines<96>::base; alt = ColLines<96>::alt; break;
    case 128: base = ColLines<128>::base; alt = ColLines<128>::alt; break;
    case 192: base = ColLines<192>::base; alt = ColLines<192>::alt; break;
    case 256: base = ColLines<256>::base; alt = ColLines<256>::alt; break;
    case 150: base = ColLines<150>::base; alt = ColLines<150>::alt; break;
    default: return 0;
  }
  if (min_over_variants) return base < alt ? base : alt;
  return (fft_variant(n) & 2) ? alt : base;
}

int c2r_partials(const Dims& d, int nf, bool any_variant) {
  const int P = row_lines(d.n3, any_variant);
  if (!P) return 0;
  const int nrows = d.n1 * d.n2;
  return ((nrows + 2 * P - 1) / (2 * P)) * nf;
}

int launch_c2r3d(float2* spec, long long sp, float* out, long long op_, long long ofs, int nf,
                 int nprob, const Dims& d, int epi, const float* alpha, double* partials, int nparts,
                 const int* active, cudaStream_t s, const float* other) {
  if ((epi == EPI_STORE_DOT || epi == EPI_ADD_DOT) && !other) return (int)cudaErrorInvalidValue;
  if (!axes_supported(d)) return (int)cudaErrorInvalidValue;
  const long long nc = d.nc();
  const int n3h = d.n3 / 2 + 1;
  int e = 0;
  CB_DISPATCH_NV_COL(d.n2, e = (cols_impl<NN, true, VV>(spec, sp, nc, d.n1 * n3h, n3h, (long long)d.n2 * n3h, n3h,
                                               nf, nprob, active, s)));
  if (e) return e;
  CB_DISPATCH_NV(d.n3, e = (c2r_rows_impl<NN, VV>(spec, sp, nc, out, op_, ofs, d.n1 * d.n2, nf, nprob, epi, alpha,
                                            partials, nparts, other, active, s)));
  return e;
}

template <int N, int V>
static int deriv_rows_impl(const float* in, long long ip, long long ifs, float* out, long long op_, long long ofs,
                           int nf, int nprob, const Dims& d, int epi, double* partials, int nparts,
                           const int* active, cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  size_t sm = row_smem<N, V>(false);
  int e = set_smem(k_deriv_rows<N, V>, sm);
  if (e) return e;
  const int nrows = d.n1 * d.n2;
  dim3 grid((nrows + 2 * RowCfg<N, V>::P - 1) / (2 * RowCfg<N, V>::P), nf, nprob);
  k_deriv_rows<N, V><<<grid, kThreads, sm, s>>>(in, ip, ifs, out, op_, ofs, nrows, tw, epi, partials, nparts, active);
  return (int)cudaGetLastError();
}

template <int N, int V>
static int deriv_cols_impl(const float* in, long long ip, long long ifs, float* out, long long op_, long long ofs,
                           int nf, int nprob, const Dims& d, int axis, int epi, double* partials, int nparts,
                           const int* active, cudaStream_t s) {
  const float2* tw = twiddles(N);
  if (!tw) return (int)cudaErrorMemoryAllocation;
  size_t sm = col_smem<N, V>(2);
  int e = set_smem(k_deriv_cols<N, V>, sm);
  if (e) return e;
  int ncols, cpg;
  long long gs, es;
  if (axis == 1) {  // lines along x2: column (i1, i3)
    ncols = d.n1 * d.n3; cpg = d.n3; gs = (long long)d.n2 * d.n3; es = d.n3;
  } else {          // lines along x1: column (i2, i3)
    ncols = d.n2 * d.n3; cpg = ncols; gs = 0; es = (long long)d.n2 * d.n3;
  }
  constexpr int C = 2 * ColCfg<N, V>::C;
  dim3 grid((ncols + C - 1) / C, nf, nprob);
  k_deriv_cols<N, V><<<grid, kThreads, sm, s>>>(in, ip, ifs, out, op_, ofs, ncols, cpg, gs, es, tw, epi, partials,
                                                nparts, active);
  return (int)cudaGetLastError();
}

int deriv_partials(const Dims& d, int axis, int nf, bool any_variant) {
  const int n = (axis == 0) ? d.n1 : (axis == 1 ? d.n2 : d.n3);
  if (axis == 2) {
    const int P = row_lines(n, any_variant);
    if (!P) return 0;
    return ((d.n1 * d.n2 + 2 * P - 1) / (2 * P)) * nf;
  }
  const int C = col_lines(n, any_variant);
  if (!C) return 0;
  const int ncols = (axis == 1) ? d.n1 * d.n3 : d.n2 * d.n3;
  return ((ncols + 2 * C - 1) / (2 * C)) * nf;
}

int launch_deriv(const float* in, long long ip, long long ifs, float* out, long long op_,
                 long long ofs, int nf, int nprob, const Dims& d, int axis, int epi,
                 double* partials, int nparts, const int* active, cudaStream_t s) {
  if (!axes_supported(d)) return (int)cudaErrorInvalidValue;
  if (axis == 2 && (!aligned16(in) || ((ip | ifs) & 3))) return (int)cudaErrorInvalidValue;
  const int n = (axis == 0) ? d.n1 : (axis == 1 ? d.n2 : d.n3);
  int e = 0;
  if (axis == 2) {
    CB_DISPATCH_NV(n, e = (deriv_rows_impl<NN, VV>(in, ip, ifs, out, op_, ofs, nf, nprob, d, epi, partials, nparts,
                                                   active, s)));
  } else {
    CB_DISPATCH_NV_COL(n, e = (deriv_cols_impl<NN, VV>(in, ip, ifs, out, op_, ofs, nf, nprob, d, axis, epi,
                                                       partials, nparts, active, s)));
  }
  return e;
}

// 3-field spectral operator (r2c, x1 op, c2r store) on caller-provided
// spectrum workspace and twiddle table: the launches allocate nothing.
template <int N, int V>
static int spectral3_explicit_impl(const float* in, float* out, float2* spec, const SpecParams* params,
                                   const Dims& d, int op, const float2* tw, cudaStream_t s) {
  const long long n = d.n(), nc = d.nc();
  const int n3h = N / 2 + 1;
  const int nrows = d.n1 * d.n2;
  int e = set_smem(k_r2c_rows<N, V>, row_smem<N, V>(false));
  if (!e) e = set_smem(k_cols<N, false, V>, col_smem<N, V>(1));
  if (!e) e = set_smem(k_cols<N, true, V>, col_smem<N, V>(1));
  if (!e) e = set_smem(k_pencil1<N, V>, col_smem<N, V>(2));
  if (!e) e = set_smem(k_c2r_rows<N, V>, row_smem<N, V>(true));
  if (e) return e;
  const dim3 rows((nrows + 2 * RowCfg<N, V>::P - 1) / (2 * RowCfg<N, V>::P), 3, 1);
  const int ncx2 = d.n1 * n3h;
  const dim3 cols((ncx2 + ColCfg<N, V>::C - 1) / ColCfg<N, V>::C, 3, 1);
  const int ncx1 = d.n2 * n3h;
  const dim3 pen((ncx1 + ColCfg<N, V>::C - 1) / ColCfg<N, V>::C, 3, 1);
  k_r2c_rows<N, V><<<rows, kThreads, row_smem<N, V>(false), s>>>(in, 0, n, spec, 0, nc, nrows, tw, nullptr);
  k_cols<N, false, V><<<cols, kThreads, col_smem<N, V>(1), s>>>(spec, 0, nc, ncx2, n3h, (long long)d.n2 * n3h, n3h, tw,
                                                          nullptr);
  k_pencil1<N, V><<<pen, kThreads, col_smem<N, V>(2), s>>>(spec, 0, nc, d, op, params, tw, nullptr);
  k_cols<N, true, V><<<cols, kThreads, col_smem<N, V>(1), s>>>(spec, 0, nc, ncx2, n3h, (long long)d.n2 * n3h, n3h, tw,
                                                         nullptr);
  k_c2r_rows<N, V><<<rows, kThreads, row_smem<N, V>(true), s>>>(spec, 0, nc, out, 0, n, nrows, tw, EPI_STORE, nullptr,
                                                           nullptr, 0, nullptr, nullptr);
  return (int)cudaGetLastError();
}

int launch_spectral3_explicit(const float* in, float* out, float2* spec, const SpecParams* params, const Dims& d,
                              int op, const float2* tw, cudaStream_t s) {
  if (!cubic_supported(d) || !aligned16(in)) return (int)cudaErrorInvalidValue;
  int e = 0;
  CB_DISPATCH_N(d.n1, e = (spectral3_explicit_impl<NN, 0>(in, out, spec, params, d, op, tw, s)));
  return e;
}

// ---------------------------------------------------------------------------
// autotuner: CLAIRE plans its transforms by measurement (accfft_plan_dft_3d_r2c
// with ACCFFT_MEASURE, src/RegOpt.cpp:993-994); here the candidates are the
// variants above, timed on the work the solver does with them.
// ---------------------------------------------------------------------------
__global__ void k_tune_fill(float* x, long long len) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    x[i] = __sinf(0.001f * (float)(i % 100003));
}

static std::atomic<bool> g_fft_tuned[9];
static std::mutex g_tune_mutex;

bool fft_tuned(int n) {
  const int k = size_slot(n);
  return k >= 0 && g_fft_tuned[k].load();
}

int fft_autotune_once(int n, int nprob, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  if (fft_tuned(n)) return 0;
  int best = 0;
  return fft_autotune(n, nprob, s, &best, nullptr);
}

int fft_autotune(int n, int nprob, cudaStream_t s, int* best, float* ms) {
  int cand[4];
  const int ncand = fft_variant_candidates(n, cand);
  if (!ncand || nprob < 1) return (int)cudaErrorInvalidValue;
  const Dims d{n, n, fft_size_supported(n) ? n : 64};  // 150: column / pencil passes only
  const long long nn = d.n(), nc = d.nc();
  float *in = nullptr, *out = nullptr;
  float2* spec = nullptr;
  SpecParams* par = nullptr;
  int e = 0;
  if (cudaMalloc(&in, sizeof(float) * 3 * nn * nprob) != cudaSuccess ||
      cudaMalloc(&out, sizeof(float) * 3 * nn * nprob) != cudaSuccess ||
      cudaMalloc(&spec, sizeof(float2) * 3 * nc * nprob) != cudaSuccess ||
      cudaMalloc(&par, sizeof(SpecParams) * nprob) != cudaSuccess)
    e = (int)cudaErrorMemoryAllocation;
  std::vector<SpecParams> hp(nprob);
  for (auto& p : hp) {
    p.norm = NORM_H2;
    p.beta0 = 1e-3f;
    p.beta1 = 1e-4f;
    p.beta2 = 1e-4f;
    p.hd = 1.f;
    p.sigma[0] = p.sigma[1] = p.sigma[2] = 1.f;
  }
  if (!e) e = (int)cudaMemcpyAsync(par, hp.data(), sizeof(SpecParams) * nprob, cudaMemcpyHostToDevice, s);
  if (!e) {
    k_tune_fill<<<148 * 4, 256, 0, s>>>(in, 3 * nn * nprob);
    e = (int)cudaGetLastError();
  }
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (!e && (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess)) e = (int)cudaErrorUnknown;
  const int old = fft_variant(n);
  float best_ms = 0.f;
  int best_v = old;
  auto work = [&]() -> int {
    int r = launch_r2c3d(in, 3 * nn, nn, spec, 3 * nc, 3, nprob, d, nullptr, s);
    if (!r) r = launch_pencil(spec, 3 * nc, nprob, d, OP_REG_INV, par, 3, 3, nullptr, s);
    if (!r) r = launch_c2r3d(spec, 3 * nc, out, 3 * nn, nn, 3, nprob, d, EPI_STORE, nullptr, nullptr, 0, nullptr, s);
    for (int a = 0; a < 3 && !r; ++a)
      r = launch_deriv(in, 3 * nn, nn, out + a * nn, 3 * nn, 3 * nn, 1, nprob, d, a, EPI_STORE, nullptr, 0, nullptr,
                       s);
    return r;
  };
  for (int i = 0; i < ncand && !e; ++i) {
    g_fft_var[size_slot(n)].store(cand[i], std::memory_order_relaxed);
    for (int w = 0; w < 2 && !e; ++w) e = work();
    constexpr int kReps = 5;
    if (!e) e = (int)cudaEventRecord(t0, s);
    for (int r = 0; r < kReps && !e; ++r) e = work();
    if (!e) e = (int)cudaEventRecord(t1, s);
    if (!e) e = (int)cudaEventSynchronize(t1);
    float t = 0.f;
    if (!e) e = (int)cudaEventElapsedTime(&t, t0, t1);
    t /= kReps;
    if (ms) ms[i] = t;
    if (!e && (i == 0 || t < best_ms)) {
      best_ms = t;
      best_v = cand[i];
    }
  }
  g_fft_var[size_slot(n)].store(e ? old : best_v, std::memory_order_relaxed);
  if (!e) g_fft_tuned[size_slot(n)].store(true);
  if (best) *best = e ? old : best_v;
  cudaStreamSynchronize(s);
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  cudaFree(in);
  cudaFree(out);
  cudaFree(spec);
  cudaFree(par);
  return e;
}

}  // namespace cb
