// In-shared-memory batched complex FFT engine (mixed radix, Stockham).
//
// A CTA transforms `nlines` complex lines of length N that live in shared
// memory as split real/imaginary arrays: element e of line p sits at
// re[e*PITCH + p], im[e*PITCH + p] (line index fastest; PITCH odd for 32 or
// more lines, so that consecutive lines hit distinct banks, and 16 for 16
// lines, see RotateFirst).  Line count and pitch are
// compile-time so every loop has a known trip count.  Every plan has exactly two radix
// stages (N = R0*R1, R0, R1 in {4, 8, 10, 12, 15, 16}), each an in-register DFT
// followed by one shared-memory exchange, so the result lands back in the
// source buffer after one ping-pong through the scratch buffer.
//
// Stockham stage with radix R and span Ns (product of earlier radices):
//   for j in [0, N/R): k = j mod Ns
//     v[r] = x[j + r*N/R] * W_N^(r*k*N/(Ns*R));  v = DFT_R(v)
//     y[(j - k)*R + k + r*Ns] = v[r]
// Twiddles W_N^m = exp(-2*pi*i*m/N) come from a table computed on the host
// in double precision and staged in shared memory.
#pragma once

#include "common.cuh"

namespace cb {

// exp(-2*pi*i*m/16) and exp(-2*pi*i*m/12), m = 0..R-1.
__device__ __constant__ float2 kTw16[16] = {
    {1.000000000f, -0.000000000f}, {0.923879533f, -0.382683432f}, {0.707106781f, -0.707106781f},
    {0.382683432f, -0.923879533f}, {0.000000000f, -1.000000000f}, {-0.382683432f, -0.923879533f},
    {-0.707106781f, -0.707106781f}, {-0.923879533f, -0.382683432f}, {-1.000000000f, -0.000000000f},
    {-0.923879533f, 0.382683432f}, {-0.707106781f, 0.707106781f}, {-0.382683432f, 0.923879533f},
    {-0.000000000f, 1.000000000f}, {0.382683432f, 0.923879533f}, {0.707106781f, 0.707106781f},
    {0.923879533f, 0.382683432f}};
__device__ __constant__ float2 kTw12[12] = {
    {1.000000000f, -0.000000000f}, {0.866025404f, -0.500000000f}, {0.500000000f, -0.866025404f},
    {0.000000000f, -1.000000000f}, {-0.500000000f, -0.866025404f}, {-0.866025404f, -0.500000000f},
    {-1.000000000f, -0.000000000f}, {-0.866025404f, 0.500000000f}, {-0.500000000f, 0.866025404f},
    {-0.000000000f, 1.000000000f}, {0.500000000f, 0.866025404f}, {0.866025404f, 0.500000000f}};

// exp(-2*pi*i*m/60), m = 0..59: the small twiddles of radices 5, 10, 15
// (grids with a factor 5, such as 150 points).
__device__ __constant__ float2 kTw60[60] = {
    {1.000000000f, -0.000000000f},
    {0.994521895f, -0.104528463f},
    {0.978147601f, -0.207911691f},
    {0.951056516f, -0.309016994f},
    {0.913545458f, -0.406736643f},
    {0.866025404f, -0.500000000f},
    {0.809016994f, -0.587785252f},
    {0.743144825f, -0.669130606f},
    {0.669130606f, -0.743144825f},
    {0.587785252f, -0.809016994f},
    {0.500000000f, -0.866025404f},
    {0.406736643f, -0.913545458f},
    {0.309016994f, -0.951056516f},
    {0.207911691f, -0.978147601f},
    {0.104528463f, -0.994521895f},
    {0.000000000f, -1.000000000f},
    {-0.104528463f, -0.994521895f},
    {-0.207911691f, -0.978147601f},
    {-0.309016994f, -0.951056516f},
    {-0.406736643f, -0.913545458f},
    {-0.500000000f, -0.866025404f},
    {-0.587785252f, -0.809016994f},
    {-0.669130606f, -0.743144825f},
    {-0.743144825f, -0.669130606f},
    {-0.809016994f, -0.587785252f},
    {-0.866025404f, -0.500000000f},
    {-0.913545458f, -0.406736643f},
    {-0.951056516f, -0.309016994f},
    {-0.978147601f, -0.207911691f},
    {-0.994521895f, -0.104528463f},
    {-1.000000000f, -0.000000000f},
    {-0.994521895f, 0.104528463f},
    {-0.978147601f, 0.207911691f},
    {-0.951056516f, 0.309016994f},
    {-0.913545458f, 0.406736643f},
    {-0.866025404f, 0.500000000f},
    {-0.809016994f, 0.587785252f},
    {-0.743144825f, 0.669130606f},
    {-0.669130606f, 0.743144825f},
    {-0.587785252f, 0.809016994f},
    {-0.500000000f, 0.866025404f},
    {-0.406736643f, 0.913545458f},
    {-0.309016994f, 0.951056516f},
    {-0.207911691f, 0.978147601f},
    {-0.104528463f, 0.994521895f},
    {-0.000000000f, 1.000000000f},
    {0.104528463f, 0.994521895f},
    {0.207911691f, 0.978147601f},
    {0.309016994f, 0.951056516f},
    {0.406736643f, 0.913545458f},
    {0.500000000f, 0.866025404f},
    {0.587785252f, 0.809016994f},
    {0.669130606f, 0.743144825f},
    {0.743144825f, 0.669130606f},
    {0.809016994f, 0.587785252f},
    {0.866025404f, 0.500000000f},
    {0.913545458f, 0.406736643f},
    {0.951056516f, 0.309016994f},
    {0.978147601f, 0.207911691f},
    {0.994521895f, 0.104528463f}
};

CB_DEVICE float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
CB_DEVICE float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
CB_DEVICE float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
CB_DEVICE float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// W_R^m (forward) or its conjugate (inverse), R divides 16, 12 or 60.
template <int R, bool INV>
CB_DEVICE float2 wsmall(int m) {
  float2 w;
  if (16 % R == 0) w = kTw16[(m * (16 / R)) % 16];
  else if (12 % R == 0) w = kTw12[(m * (12 / R)) % 12];
  else w = kTw60[(m * (60 / R)) % 60];
  if (INV) w.y = -w.y;
  return w;
}

template <int R> struct Factor;
template <> struct Factor<6> { static constexpr int A = 2, B = 3; };
template <> struct Factor<8> { static constexpr int A = 2, B = 4; };
template <> struct Factor<12> { static constexpr int A = 3, B = 4; };
template <> struct Factor<16> { static constexpr int A = 4, B = 4; };
template <> struct Factor<10> { static constexpr int A = 2, B = 5; };
template <> struct Factor<15> { static constexpr int A = 3, B = 5; };

template <int R, bool INV> struct Dft;

template <bool INV> struct Dft<2, INV> {
  static CB_DEVICE void run(float2 (&v)[2]) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV> struct Dft<3, INV> {
  static CB_DEVICE void run(float2 (&v)[3]) {
    const float s = INV ? -0.866025404f : 0.866025404f;
    float2 t = cadd(v[1], v[2]);
    float2 u = csub(v[1], v[2]);
    float2 a = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    // -i*s*u = (s*u.y, -s*u.x)
    float2 r = make_float2(s * u.y, -s * u.x);
    v[0] = cadd(v[0], t);
    v[1] = cadd(a, r);
    v[2] = csub(a, r);
  }
};

// Radix 5: with t1 = x1 + x4, t2 = x2 + x3, t3 = x1 - x4, t4 = x2 - x3,
//   X1,4 = x0 + c1 t1 + c2 t2 -/+ i (s1 t3 + s2 t4)
//   X2,3 = x0 + c2 t1 + c1 t2 -/+ i (s2 t3 - s1 t4)
// c1 = cos(2 pi/5), c2 = cos(4 pi/5), s1 = sin(2 pi/5), s2 = sin(4 pi/5);
// the inverse flips the sign of i.
template <bool INV> struct Dft<5, INV> {
  static CB_DEVICE void run(float2 (&v)[5]) {
    const float c1 = 0.309016994f, c2 = -0.809016994f;
    const float s1 = INV ? -0.951056516f : 0.951056516f, s2 = INV ? -0.587785252f : 0.587785252f;
    const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    const float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    v[0] = cadd(v[0], cadd(t1, t2));
    // -i b = (b.y, -b.x)
    v[1] = make_float2(a1.x + b1.y, a1.y - b1.x);
    v[4] = make_float2(a1.x - b1.y, a1.y + b1.x);
    v[2] = make_float2(a2.x + b2.y, a2.y - b2.x);
    v[3] = make_float2(a2.x - b2.y, a2.y + b2.x);
  }
};

template <bool INV> struct Dft<4, INV> {
  static CB_DEVICE void run(float2 (&v)[4]) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    // forward: y1 = t1 - i*t3, y3 = t1 + i*t3
    float2 it3 = INV ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, it3);
    v[3] = csub(t1, it3);
  }
};

// Composite R = A*B: X[k1 + A*k2] = sum_n2 W_B^(n2 k2) W_R^(n2 k1) sum_n1 x[B n1 + n2] W_A^(n1 k1)
template <int R, bool INV> struct Dft {
  static CB_DEVICE void run(float2 (&v)[R]) {
    constexpr int A = Factor<R>::A, B = Factor<R>::B;
    float2 y[A][B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      float2 t[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
      Dft<A, INV>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        y[k1][n2] = (n2 * k1 == 0) ? t[k1] : cmul(t[k1], wsmall<R, INV>(n2 * k1));
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      float2 t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) t[n2] = y[k1][n2];
      Dft<B, INV>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
    }
  }
};

// Two-stage plans N = R0 * R1.  Variant bit 0 selects the alternative
// factorization (the other factor order, or 16 x 4 for 64); the autotuner
// picks per grid size whichever runs faster (Plan0 where there is none).
template <int N> struct Plan0;
template <> struct Plan0<16> { static constexpr int R0 = 4, R1 = 4; };
template <> struct Plan0<32> { static constexpr int R0 = 4, R1 = 8; };
template <> struct Plan0<48> { static constexpr int R0 = 12, R1 = 4; };
template <> struct Plan0<64> { static constexpr int R0 = 8, R1 = 8; };
template <> struct Plan0<96> { static constexpr int R0 = 12, R1 = 8; };
template <> struct Plan0<128> { static constexpr int R0 = 16, R1 = 8; };
template <> struct Plan0<192> { static constexpr int R0 = 12, R1 = 16; };
template <> struct Plan0<256> { static constexpr int R0 = 16, R1 = 16; };
template <> struct Plan0<150> { static constexpr int R0 = 10, R1 = 15; };
template <int N> struct Plan1;
template <> struct Plan1<16> { static constexpr int R0 = 4, R1 = 4; };
template <> struct Plan1<32> { static constexpr int R0 = 8, R1 = 4; };
template <> struct Plan1<48> { static constexpr int R0 = 4, R1 = 12; };
template <> struct Plan1<64> { static constexpr int R0 = 16, R1 = 4; };
template <> struct Plan1<96> { static constexpr int R0 = 8, R1 = 12; };
template <> struct Plan1<128> { static constexpr int R0 = 8, R1 = 16; };
template <> struct Plan1<192> { static constexpr int R0 = 16, R1 = 12; };
template <> struct Plan1<256> { static constexpr int R0 = 16, R1 = 16; };
template <> struct Plan1<150> { static constexpr int R0 = 15, R1 = 10; };
template <int N, int V = 0> struct Plan {
  static constexpr int R0 = (V & 1) ? Plan1<N>::R0 : Plan0<N>::R0;
  static constexpr int R1 = (V & 1) ? Plan1<N>::R1 : Plan0<N>::R1;
  static_assert(R0 * R1 == N, "plan must factor N");
};

constexpr int kFftThreads = 256;  // threads per CTA of every FFT kernel

// Bank spread of a 16-line layout.  Lanes 0-15 and 16-31 of a warp hold one
// element index apart (j and j + 1).  A pitch of 16 (mod 32) puts the two
// half-warps in opposite halves of the bank space for every read and every
// write of a later stage (element offsets 1 or odd).  A first-stage (span 1)
// write puts the two half-warps R elements apart: for even R that is the same
// half.  So there the upper half-warp writes its R outputs rotated by one,
// which makes the offset R + 1 (or 1), odd again.  Every output is still
// written once, with the same value.
template <int NL, int PITCH, int R>
struct RotateFirst {
  static constexpr bool value = NL == 16 && PITCH % 32 == 16 && R % 2 == 0;
};

template <int N, int R, int NS, bool INV, int NL, int PITCH>
CB_DEVICE void fft_stage(const float* __restrict__ sre, const float* __restrict__ sim,
                         float* __restrict__ dre, float* __restrict__ dim, const float2* __restrict__ tw) {
  constexpr int J = N / R;
  constexpr int total = NL * J;
#pragma unroll 2
  for (int u = threadIdx.x; u < total; u += kFftThreads) {
    const int p = u % NL;
    const int j = u / NL;
    const int k = j % NS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int idx = (j + r * J) * PITCH + p;
      v[r] = make_float2(sre[idx], sim[idx]);
    }
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * k * (N / (NS * R))];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int o = (j - k) * R + k;
    if constexpr (NS == 1 && RotateFirst<NL, PITCH, R>::value) {
      const int h = j & 1;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int rr = (r + h == R) ? 0 : r + h;
        const float2 x = h ? v[(r + 1) % R] : v[r];
        const int idx = (o + rr) * PITCH + p;
        dre[idx] = x.x;
        dim[idx] = x.y;
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int idx = (o + r * NS) * PITCH + p;
        dre[idx] = v[r].x;
        dim[idx] = v[r].y;
      }
    }
  }
}

// Transform nlines lines held in (re, im); (sre, sim) is scratch of the same
// size.  The result is back in (re, im).  Caller synchronises before; this
// function synchronises after each stage.
template <int N, bool INV, int NL, int PITCH, int V = 0>
CB_DEVICE void fft_lines(float* re, float* im, float* sre, float* sim, const float2* tw) {
  using P = Plan<N, V>;
  fft_stage<N, P::R0, 1, INV, NL, PITCH>(re, im, sre, sim, tw);
  __syncthreads();
  fft_stage<N, P::R1, P::R0, INV, NL, PITCH>(sre, sim, re, im, tw);
  __syncthreads();
}

// Column layout (lines are columns of a strided array; the thread's line p is
// threadIdx.x % NL in every stage because kFftThreads % NL == 0): the first
// stage can read its inputs straight from global memory and the last one
// write its outputs straight back, the warp's lanes covering NL adjacent
// columns at one element (coalesced).  The arithmetic is fft_stage's, so
// results are bit-identical to staging the lines in shared memory first.

// First stage (span 1: no twiddles) reading element e of the thread's line p
// through ld(p, e) (a float2), into (dre, dim).
template <int N, int R, bool INV, int NL, int PITCH, class Load>
CB_DEVICE void fft_stage_in(const Load& ld, float* __restrict__ dre, float* __restrict__ dim) {
  constexpr int J = N / R;
  constexpr int total = NL * J;
  static_assert(kFftThreads % NL == 0, "a thread keeps its line across stages");
#pragma unroll 2
  for (int u = threadIdx.x; u < total; u += kFftThreads) {
    const int p = u % NL;
    const int j = u / NL;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ld(p, j + r * J);
    Dft<R, INV>::run(v);
    if constexpr (RotateFirst<NL, PITCH, R>::value) {
      const int h = j & 1;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int rr = (r + h == R) ? 0 : r + h;
        const float2 x = h ? v[(r + 1) % R] : v[r];
        const int idx = (j * R + rr) * PITCH + p;
        dre[idx] = x.x;
        dim[idx] = x.y;
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int idx = (j * R + r) * PITCH + p;
        dre[idx] = v[r].x;
        dim[idx] = v[r].y;
      }
    }
  }
}

// Last stage (span NS) from (sre, sim), handing element e of line p to
// st(p, e, value).
template <int N, int R, int NS, bool INV, int NL, int PITCH, class Store>
CB_DEVICE void fft_stage_out(const float* __restrict__ sre, const float* __restrict__ sim,
                             const float2* __restrict__ tw, const Store& st) {
  constexpr int J = N / R;
  constexpr int total = NL * J;
  static_assert(kFftThreads % NL == 0, "a thread keeps its line across stages");
#pragma unroll 2
  for (int u = threadIdx.x; u < total; u += kFftThreads) {
    const int p = u % NL;
    const int j = u / NL;
    const int k = j % NS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int idx = (j + r * J) * PITCH + p;
      v[r] = make_float2(sre[idx], sim[idx]);
    }
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * k * (N / (NS * R))];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Dft<R, INV>::run(v);
    const int o = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) st(p, o + r * NS, v[r]);
  }
}

// The two for a column of complex elements colp[e * es] (colp null: zeros in,
// nothing out).
struct ColumnLoad {
  const float2* colp;
  long long es;
  CB_DEVICE float2 operator()(int, int e) const {
    return colp ? __ldg(colp + (long long)e * es) : make_float2(0.f, 0.f);
  }
};
struct ColumnStore {
  float2* colp;
  long long es;
  CB_DEVICE void operator()(int, int e, float2 v) const {
    if (colp) colp[(long long)e * es] = v;
  }
};

// Shared-memory lines (re, im) as a stage's destination.
template <int PITCH>
struct SmemStore {
  float* re;
  float* im;
  CB_DEVICE void operator()(int p, int e, float2 v) const {
    re[e * PITCH + p] = v.x;
    im[e * PITCH + p] = v.y;
  }
};

template <int N, int R, bool INV, int NL, int PITCH>
CB_DEVICE void fft_stage_load(const float2* __restrict__ colp, long long es, float* __restrict__ dre,
                              float* __restrict__ dim) {
  fft_stage_in<N, R, INV, NL, PITCH>(ColumnLoad{colp, es}, dre, dim);
}

template <int N, int R, int NS, bool INV, int NL, int PITCH>
CB_DEVICE void fft_stage_store(const float* __restrict__ sre, const float* __restrict__ sim,
                               const float2* __restrict__ tw, float2* __restrict__ colp, long long es) {
  fft_stage_out<N, R, NS, INV, NL, PITCH>(sre, sim, tw, ColumnStore{colp, es});
}

// Stage the N-entry twiddle table into shared memory.
template <int N>
CB_DEVICE void load_twiddles(float2* dst, const float2* __restrict__ src) {
  for (int i = threadIdx.x; i < N; i += kFftThreads) dst[i] = src[i];
}

}  // namespace cb
