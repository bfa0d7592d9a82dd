// FP64 reductions (dot products, squared distances) and fused elementwise
// vector updates used by the distance, the PCG and the line search.
//
// Replaces PETSc VecTDot / VecNorm / VecAXPY / VecWAXPY on the hot path
// (e.g. src/RegularizationH1.cpp:105-143, src/VecField.cpp:577-694) and the
// serial loop of src/DistanceMeasureSL2.cpp:119-150.
#include "reduce.cuh"
#include "sl.cuh"

namespace cb {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 2;  // per problem; one wave on 148 SMs

int dot_partials(long long len) {
  long long need = (len + kRedThreads * 4 - 1) / (kRedThreads * 4);
  return (int)(need < kRedBlocks ? (need < 1 ? 1 : need) : kRedBlocks);
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

__global__ void __launch_bounds__(kRedThreads) k_dot(const float* __restrict__ a, long long ap,
                                                      const float* __restrict__ b, long long bp,
                                                      long long len, double* __restrict__ partials,
                                                      int nparts, const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const float* pa = a + blockIdx.y * ap;
  const float* pb = b + blockIdx.y * bp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x)
    acc += (double)pa[i] * (double)pb[i];
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

// float4 form (len % 4 == 0, 16-byte aligned rows): four products per load
__global__ void __launch_bounds__(kRedThreads) k_dot4(const float4* __restrict__ a, long long ap,
                                                       const float4* __restrict__ b, long long bp,
                                                       long long len4, double* __restrict__ partials,
                                                       int nparts, const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const float4* pa = a + blockIdx.y * ap;
  const float4* pb = b + blockIdx.y * bp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len4;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 x = __ldg(pa + i), y = __ldg(pb + i);
    acc += (double)x.x * (double)y.x + (double)x.y * (double)y.y + (double)x.z * (double)y.z +
           (double)x.w * (double)y.w;
  }
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

// PCG update x += alpha p, r -= alpha q, partial sums of r.r (the new residual)
__global__ void __launch_bounds__(kRedThreads) k_cg_update(float4* __restrict__ x, float4* __restrict__ r,
                                                            const float4* __restrict__ p,
                                                            const float4* __restrict__ q, long long vp,
                                                            long long len4, const double* __restrict__ alpha,
                                                            double* __restrict__ partials, int nparts,
                                                            const int* __restrict__ active) {
  const int pb = blockIdx.y;
  if (active && !active[pb]) return;
  const float al = (float)alpha[pb];
  float4* px = x + pb * vp;
  float4* pr = r + pb * vp;
  const float4* pp = p + pb * vp;
  const float4* pq = q + pb * vp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len4;
       i += (long long)gridDim.x * blockDim.x) {
    float4 xv = px[i], rv = pr[i];
    const float4 pv = __ldg(pp + i), qv = __ldg(pq + i);
    xv.x += al * pv.x; xv.y += al * pv.y; xv.z += al * pv.z; xv.w += al * pv.w;
    rv.x -= al * qv.x; rv.y -= al * qv.y; rv.z -= al * qv.z; rv.w -= al * qv.w;
    px[i] = xv;
    pr[i] = rv;
    acc += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y + (double)rv.z * (double)rv.z +
           (double)rv.w * (double)rv.w;
  }
  block_reduce_store(acc, partials + (long long)pb * nparts, blockIdx.x);
}

int launch_cg_update(float* x, float* r, const float* p, const float* q, long long vp, long long len,
                     const double* alpha, int nprob, double* partials, int stride, const int* active,
                     cudaStream_t s) {
  if ((len & 3) || (vp & 3) || !aligned16(x) || !aligned16(r) || !aligned16(p) || !aligned16(q))
    return (int)cudaErrorInvalidValue;
  dim3 grid(dot_partials(len), nprob);
  k_cg_update<<<grid, kRedThreads, 0, s>>>(reinterpret_cast<float4*>(x), reinterpret_cast<float4*>(r),
                                            reinterpret_cast<const float4*>(p), reinterpret_cast<const float4*>(q),
                                            vp / 4, len / 4, alpha, partials, stride, active);
  return (int)cudaGetLastError();
}

// y = a + b and partial sums of y.c (y may be a)
__global__ void __launch_bounds__(kRedThreads) k_add_dot4(float4* y, const float4* a, const float4* __restrict__ b,
                                                           const float4* __restrict__ c, long long vp,
                                                           long long len4, double* __restrict__ partials,
                                                           int nparts, const int* __restrict__ active) {
  const int pb = blockIdx.y;
  if (active && !active[pb]) return;
  float4* py = y + pb * vp;
  const float4* pa = a + pb * vp;
  const float4* pbv = b + pb * vp;
  const float4* pc = c + pb * vp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len4;
       i += (long long)gridDim.x * blockDim.x) {
    float4 v = pa[i];
    const float4 w = __ldg(pbv + i), cv = __ldg(pc + i);
    v.x += w.x; v.y += w.y; v.z += w.z; v.w += w.w;
    py[i] = v;
    acc += (double)v.x * (double)cv.x + (double)v.y * (double)cv.y + (double)v.z * (double)cv.z +
           (double)v.w * (double)cv.w;
  }
  block_reduce_store(acc, partials + (long long)pb * nparts, blockIdx.x);
}

int launch_add_dot(float* y, const float* a, const float* b, const float* c, long long vp, long long len, int nprob,
                   double* partials, int stride, const int* active, cudaStream_t s) {
  if ((len & 3) || (vp & 3) || !aligned16(y) || !aligned16(a) || !aligned16(b) || !aligned16(c))
    return (int)cudaErrorInvalidValue;
  dim3 grid(dot_partials(len), nprob);
  k_add_dot4<<<grid, kRedThreads, 0, s>>>(reinterpret_cast<float4*>(y), reinterpret_cast<const float4*>(a),
                                           reinterpret_cast<const float4*>(b), reinterpret_cast<const float4*>(c),
                                           vp / 4, len / 4, partials, stride, active);
  return (int)cudaGetLastError();
}

__global__ void __launch_bounds__(kRedThreads) k_diff_sumsq(const float* __restrict__ a, long long ap,
                                                             const float* __restrict__ b, long long bp,
                                                             long long len, double* __restrict__ partials,
                                                             int nparts, const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const float* pa = a + blockIdx.y * ap;
  const float* pb = b + blockIdx.y * bp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)pa[i] - (double)pb[i];
    acc += d * d;
  }
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

__global__ void k_finalize(const double* __restrict__ partials, int stride, int nparts,
                           double* __restrict__ out, double scale, int accumulate, const int* __restrict__ active) {
  if (active && !active[blockIdx.x]) return;  // other problems' results stay as they are
  const double* p = partials + (long long)blockIdx.x * stride;
  double acc = 0.0;
  // fixed-order: thread t sums entries t, t+32, ...; then a fixed shuffle tree
  for (int i = threadIdx.x; i < nparts; i += 32) acc += p[i];
  acc = warp_sum(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = (accumulate ? out[blockIdx.x] : 0.0) + scale * acc;
}

int launch_finalize(const double* partials, int stride, int count, double* out, int nprob, double scale,
                    bool accumulate, cudaStream_t s, const int* active) {
  k_finalize<<<nprob, 32, 0, s>>>(partials, stride, count, out, scale, accumulate ? 1 : 0, active);
  return (int)cudaGetLastError();
}

int launch_dot(const float* a, long long ap, const float* b, long long bp, long long len, int nprob,
               double* partials, int stride, const int* active, cudaStream_t s) {
  dim3 grid(dot_partials(len), nprob);
  if (!(len & 3) && !(ap & 3) && !(bp & 3) && aligned16(a) && aligned16(b))
    k_dot4<<<grid, kRedThreads, 0, s>>>(reinterpret_cast<const float4*>(a), ap / 4,
                                        reinterpret_cast<const float4*>(b), bp / 4, len / 4, partials, stride,
                                        active);
  else
    k_dot<<<grid, kRedThreads, 0, s>>>(a, ap, b, bp, len, partials, stride, active);
  return (int)cudaGetLastError();
}

int launch_diff_sumsq(const float* a, long long ap, const float* b, long long bp, long long len,
                      int nprob, double* partials, int stride, const int* active, cudaStream_t s) {
  dim3 grid(dot_partials(len), nprob);
  k_diff_sumsq<<<grid, kRedThreads, 0, s>>>(a, ap, b, bp, len, partials, stride, active);
  return (int)cudaGetLastError();
}

// y = (sa*ca[p]) * a + (sb*cb[p]) * b   (ca / cb may be null: coefficient sa / sb)
// Inactive problems (active[p] == 0) are skipped.
__global__ void k_lincomb(float* y, long long yp, const float* a, long long ap,
                          const double* __restrict__ ca, double sa, const float* b,
                          long long bp, const double* __restrict__ cb, double sb, long long len,
                          const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const float fa = (float)(sa * (ca ? ca[p] : 1.0));
  const float fb = b ? (float)(sb * (cb ? cb[p] : 1.0)) : 0.f;
  float* py = y + p * yp;
  const float* pa = a + p * ap;
  const float* pb = b ? b + p * bp : nullptr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    float v = fa * pa[i];
    if (pb) v += fb * pb[i];
    py[i] = v;
  }
}

// float4 form of k_lincomb
__global__ void k_lincomb4(float4* y, long long yp, const float4* a, long long ap, const double* __restrict__ ca,
                           double sa, const float4* b, long long bp, const double* __restrict__ cb, double sb,
                           long long len4, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const float fa = (float)(sa * (ca ? ca[p] : 1.0));
  const float fb = b ? (float)(sb * (cb ? cb[p] : 1.0)) : 0.f;
  float4* py = y + p * yp;
  const float4* pa = a + p * ap;
  const float4* pb = b ? b + p * bp : nullptr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len4;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 u = pa[i];
    float4 v = make_float4(fa * u.x, fa * u.y, fa * u.z, fa * u.w);
    if (pb) {
      const float4 w = pb[i];
      v.x += fb * w.x;
      v.y += fb * w.y;
      v.z += fb * w.z;
      v.w += fb * w.w;
    }
    py[i] = v;
  }
}

__global__ void k_fill(float* y, long long yp, float value, long long len, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  float* py = y + p * yp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x)
    py[i] = value;
}

int launch_fill(float* y, long long yp, float value, long long len, int nprob, const int* active, cudaStream_t s) {
  long long blocks = (len + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_fill<<<dim3((unsigned)blocks, nprob), 256, 0, s>>>(y, yp, value, len, active);
  return (int)cudaGetLastError();
}

int launch_lincomb(float* y, long long yp, const float* a, long long ap, const double* ca, double sa,
                   const float* b, long long bp, const double* cb, double sb, long long len,
                   int nprob, const int* active, cudaStream_t s) {
  if (!(len & 3) && !(yp & 3) && !(ap & 3) && (!b || !(bp & 3)) && aligned16(y) && aligned16(a) &&
      (!b || aligned16(b))) {
    long long blocks = (len / 4 + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    dim3 grid((unsigned)blocks, nprob);
    k_lincomb4<<<grid, 256, 0, s>>>(reinterpret_cast<float4*>(y), yp / 4, reinterpret_cast<const float4*>(a),
                                    ap / 4, ca, sa, reinterpret_cast<const float4*>(b), bp / 4, cb, sb, len / 4,
                                    active);
    return (int)cudaGetLastError();
  }
  long long blocks = (len + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  dim3 grid((unsigned)blocks, nprob);
  k_lincomb<<<grid, 256, 0, s>>>(y, yp, a, ap, ca, sa, b, bp, cb, sb, len, active);
  return (int)cudaGetLastError();
}

// ---- bf16 image volumes -------------------------------------------------------

static dim3 stream_grid(long long work, int nprob, int nz = 1) {
  long long blocks = (work + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  return dim3((unsigned)blocks, nprob, nz);
}

__global__ void k_to_bf16(const float* __restrict__ src, long long sp, bf16* __restrict__ dst, long long dp,
                          long long len, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const float* a = src + p * sp;
  bf16* y = dst + p * dp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(a[i]);
}

__global__ void k_from_bf16(const bf16* __restrict__ src, long long sp, long long sl, float* __restrict__ dst,
                            long long dp, long long dl, long long len, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const bf16* a = src + p * sp + blockIdx.z * sl;
  float* y = dst + p * dp + blockIdx.z * dl;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[i] = __bfloat162float(a[i]);
}

// 8 bf16 per 16-byte unit
__global__ void k_copy16(uint4* __restrict__ dst, long long dp, const uint4* __restrict__ src, long long sp,
                         long long units, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < units;
       i += (long long)gridDim.x * blockDim.x)
    dst[p * dp + i] = src[p * sp + i];
}

__global__ void __launch_bounds__(kRedThreads) k_diff_sumsq16(const bf16* __restrict__ a, long long ap,
                                                               const bf16* __restrict__ b, long long bp,
                                                               long long len, double* __restrict__ partials,
                                                               int nparts, const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const bf16* pa = a + blockIdx.y * ap;
  const bf16* pb = b + blockIdx.y * bp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)__bfloat162float(pa[i]) - (double)__bfloat162float(pb[i]);
    acc += d * d;
  }
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

__global__ void k_diff16(float* __restrict__ y, long long yp, const bf16* __restrict__ a, long long ap,
                         const bf16* __restrict__ b, long long bp, long long len, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[p * yp + i] = __bfloat162float(a[p * ap + i]) - __bfloat162float(b[p * bp + i]);
}

int launch_to_bf16(const float* src, long long sp, bf16* dst, long long dp, long long len, int nprob,
                   const int* active, cudaStream_t s) {
  k_to_bf16<<<stream_grid(len, nprob), 256, 0, s>>>(src, sp, dst, dp, len, active);
  return (int)cudaGetLastError();
}

int launch_from_bf16(const bf16* src, long long sp, long long sl, float* dst, long long dp, long long dl,
                     long long len, int nlev, int nprob, const int* active, cudaStream_t s) {
  k_from_bf16<<<stream_grid(len, nprob, nlev), 256, 0, s>>>(src, sp, sl, dst, dp, dl, len, active);
  return (int)cudaGetLastError();
}

int launch_copy_bf16(bf16* dst, long long dp, const bf16* src, long long sp, long long len, int nprob,
                     const int* active, cudaStream_t s) {
  if ((len & 7) || (dp & 7) || (sp & 7) || !aligned16(dst) || !aligned16(src)) return (int)cudaErrorInvalidValue;
  k_copy16<<<stream_grid(len / 8, nprob), 256, 0, s>>>(reinterpret_cast<uint4*>(dst), dp / 8,
                                                       reinterpret_cast<const uint4*>(src), sp / 8, len / 8, active);
  return (int)cudaGetLastError();
}

int launch_diff_sumsq16(const bf16* a, long long ap, const bf16* b, long long bp, long long len, int nprob,
                        double* partials, int stride, const int* active, cudaStream_t s) {
  dim3 grid(dot_partials(len), nprob);
  k_diff_sumsq16<<<grid, kRedThreads, 0, s>>>(a, ap, b, bp, len, partials, stride, active);
  return (int)cudaGetLastError();
}

int launch_diff16(float* y, long long yp, const bf16* a, long long ap, const bf16* b, long long bp, long long len,
                  int nprob, const int* active, cudaStream_t s) {
  k_diff16<<<stream_grid(len, nprob), 256, 0, s>>>(y, yp, a, ap, b, bp, len, active);
  return (int)cudaGetLastError();
}

// ---- mask-weighted distance terms (DistanceMeasure with SetMask) --------------

CB_DEVICE float ldv(const float* p, long long i) { return p[i]; }
CB_DEVICE float ldv(const bf16* p, long long i) { return __bfloat162float(p[i]); }

template <class T>
__global__ void __launch_bounds__(kRedThreads) k_wdiff_sumsq(const T* __restrict__ a, long long ap,
                                                              const T* __restrict__ b, long long bp,
                                                              const float* __restrict__ w, long long wp,
                                                              long long len, double* __restrict__ partials,
                                                              int nparts, const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const T* pa = a + blockIdx.y * ap;
  const T* pb = b + blockIdx.y * bp;
  const float* pw = w + blockIdx.y * wp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)ldv(pa, i) - (double)ldv(pb, i);
    acc += (double)pw[i] * d * d;
  }
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

template <class T>
__global__ void k_wdiff(float* __restrict__ y, long long yp, const T* __restrict__ a, long long ap,
                        const T* __restrict__ b, long long bp, const float* __restrict__ w, long long wp,
                        long long len, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[p * yp + i] = w[p * wp + i] * (ldv(a + p * ap, i) - ldv(b + p * bp, i));
}

__global__ void __launch_bounds__(kRedThreads) k_wdot(const float* __restrict__ a, long long ap,
                                                       const float* __restrict__ b, long long bp,
                                                       const float* __restrict__ w, long long wp, long long len,
                                                       double* __restrict__ partials, int nparts,
                                                       const int* __restrict__ active) {
  if (active && !active[blockIdx.y]) return;
  const float* pa = a + blockIdx.y * ap;
  const float* pb = b + blockIdx.y * bp;
  const float* pw = w + blockIdx.y * wp;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x)
    acc += (double)pw[i] * (double)pa[i] * (double)pb[i];
  block_reduce_store(acc, partials + (long long)blockIdx.y * nparts, blockIdx.x);
}

__global__ void k_mulw(float* __restrict__ y, long long yp, const float* __restrict__ w, long long wp, long long len,
                       const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    y[p * yp + i] *= w[p * wp + i];
}

int launch_wdiff_sumsq(const float* a, long long ap, const float* b, long long bp, const float* w, long long wp,
                       long long len, int nprob, double* partials, int stride, const int* active, cudaStream_t s) {
  k_wdiff_sumsq<float><<<dim3(dot_partials(len), nprob), kRedThreads, 0, s>>>(a, ap, b, bp, w, wp, len, partials,
                                                                              stride, active);
  return (int)cudaGetLastError();
}

int launch_wdiff_sumsq(const bf16* a, long long ap, const bf16* b, long long bp, const float* w, long long wp,
                       long long len, int nprob, double* partials, int stride, const int* active, cudaStream_t s) {
  k_wdiff_sumsq<bf16><<<dim3(dot_partials(len), nprob), kRedThreads, 0, s>>>(a, ap, b, bp, w, wp, len, partials,
                                                                             stride, active);
  return (int)cudaGetLastError();
}

int launch_wdiff(float* y, long long yp, const float* a, long long ap, const float* b, long long bp, const float* w,
                 long long wp, long long len, int nprob, const int* active, cudaStream_t s) {
  k_wdiff<float><<<stream_grid(len, nprob), 256, 0, s>>>(y, yp, a, ap, b, bp, w, wp, len, active);
  return (int)cudaGetLastError();
}

int launch_wdiff(float* y, long long yp, const bf16* a, long long ap, const bf16* b, long long bp, const float* w,
                 long long wp, long long len, int nprob, const int* active, cudaStream_t s) {
  k_wdiff<bf16><<<stream_grid(len, nprob), 256, 0, s>>>(y, yp, a, ap, b, bp, w, wp, len, active);
  return (int)cudaGetLastError();
}

int launch_wdot(const float* a, long long ap, const float* b, long long bp, const float* w, long long wp, long long len,
                int nprob, double* partials, int stride, const int* active, cudaStream_t s) {
  k_wdot<<<dim3(dot_partials(len), nprob), kRedThreads, 0, s>>>(a, ap, b, bp, w, wp, len, partials, stride, active);
  return (int)cudaGetLastError();
}

int launch_mulw(float* y, long long yp, const float* w, long long wp, long long len, int nprob, const int* active,
                cudaStream_t s) {
  k_mulw<<<stream_grid(len, nprob), 256, 0, s>>>(y, yp, w, wp, len, active);
  return (int)cudaGetLastError();
}

}  // namespace cb
