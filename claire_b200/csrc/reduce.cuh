// Deterministic FP64 reductions and fused vector updates.
//
// Reductions are two-level: each CTA reduces its share in FP64 with warp
// shuffles and stores one partial per CTA; a finalize kernel sums a problem's
// partials in a fixed order.  The result does not depend on scheduling, so a
// problem gives the same numbers alone and inside a batch.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace cb {

CB_DEVICE double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; thread 0 stores the result to dst[idx].  All threads of
// the CTA must call it.
CB_DEVICE void block_reduce_store(double v, double* dst, int idx) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double t = (lane < nw) ? ws[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) dst[idx] = t;
  }
}

// Host launchers.  Problem p's partials start at partials + p*stride.
// out[p] = scale * sum(partials[p][0..count)) (+ out[p] when accumulate), for the
// problems whose active entry is nonzero (all when active is null).
int launch_finalize(const double* partials, int stride, int count, double* out, int nprob, double scale,
                    bool accumulate, cudaStream_t s, const int* active = nullptr);

// Partials written by the dot / norm kernels for vectors of length len.
int dot_partials(long long len);

// partials[p*stride + k], k < dot_partials(len) <- partial sums of a[p][i]*b[p][i]
// (FP32 inputs, FP64 sums).  Inactive problems are skipped.
int launch_dot(const float* a, long long ap, const float* b, long long bp, long long len, int nprob,
               double* partials, int stride, const int* active, cudaStream_t s);

// PCG update of problem p: x += alpha[p] p, r -= alpha[p] q; partials of the new
// r.r in the dot layout.  len % 4 == 0 and 16-byte aligned vectors (vp apart).
int launch_cg_update(float* x, float* r, const float* p, const float* q, long long vp, long long len,
                     const double* alpha, int nprob, double* partials, int stride, const int* active,
                     cudaStream_t s);
// y = a + b and partial sums of y.c per problem (vectors vp apart; y may be a)
int launch_add_dot(float* y, const float* a, const float* b, const float* c, long long vp, long long len, int nprob,
                   double* partials, int stride, const int* active, cudaStream_t s);

// y[p][i] = value, i < len
int launch_fill(float* y, long long yp, float value, long long len, int nprob, const int* active, cudaStream_t s);

// same layout, partial sums of (a[p][i] - b[p][i])^2
int launch_diff_sumsq(const float* a, long long ap, const float* b, long long bp, long long len,
                      int nprob, double* partials, int stride, const int* active, cudaStream_t s);

// ---- bf16 image volumes (FP32 arithmetic, bf16 storage) -----------------------
// dst[p][i] = bf16(src[p][i]) (round to nearest even)
int launch_to_bf16(const float* src, long long sp, bf16* dst, long long dp, long long len, int nprob,
                   const int* active, cudaStream_t s);
// dst[p][l*dl + i] = float(src[p][l*sl + i]), l < nlev
int launch_from_bf16(const bf16* src, long long sp, long long sl, float* dst, long long dp, long long dl,
                     long long len, int nlev, int nprob, const int* active, cudaStream_t s);
// dst[p][i] = src[p][i] (len % 8 == 0, 16-byte aligned rows)
int launch_copy_bf16(bf16* dst, long long dp, const bf16* src, long long sp, long long len, int nprob,
                     const int* active, cudaStream_t s);
// dot layout partial sums of (a[p][i] - b[p][i])^2 in FP64
int launch_diff_sumsq16(const bf16* a, long long ap, const bf16* b, long long bp, long long len, int nprob,
                        double* partials, int stride, const int* active, cudaStream_t s);
// y[p][i] = a[p][i] - b[p][i] in FP32
int launch_diff16(float* y, long long yp, const bf16* a, long long ap, const bf16* b, long long bp, long long len,
                  int nprob, const int* active, cudaStream_t s);

// ---- mask weights w (SetMask): sum w (a - b)^2, y = w (a - b), sum w a b, y *= w
int launch_wdiff_sumsq(const float* a, long long ap, const float* b, long long bp, const float* w, long long wp,
                       long long len, int nprob, double* partials, int stride, const int* active, cudaStream_t s);
int launch_wdiff_sumsq(const bf16* a, long long ap, const bf16* b, long long bp, const float* w, long long wp,
                       long long len, int nprob, double* partials, int stride, const int* active, cudaStream_t s);
int launch_wdiff(float* y, long long yp, const float* a, long long ap, const float* b, long long bp, const float* w,
                 long long wp, long long len, int nprob, const int* active, cudaStream_t s);
int launch_wdiff(float* y, long long yp, const bf16* a, long long ap, const bf16* b, long long bp, const float* w,
                 long long wp, long long len, int nprob, const int* active, cudaStream_t s);
int launch_wdot(const float* a, long long ap, const float* b, long long bp, const float* w, long long wp, long long len,
                int nprob, double* partials, int stride, const int* active, cudaStream_t s);
int launch_mulw(float* y, long long yp, const float* w, long long wp, long long len, int nprob, const int* active,
                cudaStream_t s);

}  // namespace cb
