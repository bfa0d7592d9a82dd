// Semi-Lagrangian kernels: RK2 characteristics, tricubic gathers and the
// state / adjoint / incremental time steps built on them.
//
// Reference loops: SemiLagrangian::ComputeTrajectoryRK2
// (src/SemiLagrangian.cpp:192-289), Interp3_Plan::interpolate +
// optimized_interp3_ghost_xyz_p (src/Interp3_Plan.cpp:699-846,
// src/interp3.cpp:2492-2719), SolveStateEquationSL / SolveAdjointEquationSL /
// SolveIncStateEquationSL / SolveIncAdjointEquationGNSL
// (src/CLAIRE.cpp:2116-2175, 2550-2722, 3147-3290, 3849-4012).  The MPI
// scatter, ghost exchange and owner lookup of the reference are not needed on
// one GPU: the periodic wrap is applied while each CTA stages its footprint
// box in shared memory (sl_tile.cuh).
//
// Every time step is one gather with a pointwise epilogue: the adjoint step's
// right-hand side collapses to a per-point factor (launch_adjoint_coef), the
// incremental state's sources are formed for all steps in one streaming pass
// (launch_incstate_source), and the body force is summed once over the stored
// adjoint levels (launch_body_force) instead of being accumulated step by step.
#include "sl_tile.cuh"

namespace cb {

constexpr int kSlThreads = 256;

static dim3 tile_grid(const Dims& d, int nprob, int nz) { return dim3(tile_count(d), nprob, nz); }

template <typename K>
static int allow_smem(K kernel) {
  if (g_graph_capture) return 0;
  return (int)cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGatherSmemBytes);
}

// ---- point sources and tile epilogues ---------------------------------------

// First RK2 stage of the characteristic: disp = -sign*ht*v*N/(2 pi).
struct VelocitySource {
  const float* v;
  float c0, c1, c2;  // -sign*ht*N_k/(2 pi)
  CB_DEVICE void load(float (&dd)[kTilePts][3], const TileThread& tt, const Dims& d) const {
    const float* v2 = v + d.n();
    const float* v3 = v2 + d.n();
#pragma unroll
    for (int a = 0; a < kTilePts; ++a) {
      const bool ok = tt.valid_idx(a);
      const unsigned i = tt.idx(a);
      dd[a][0] = ok ? c0 * __ldg(v + i) : 0.f;
      dd[a][1] = ok ? c1 * __ldg(v2 + i) : 0.f;
      dd[a][2] = ok ? c2 * __ldg(v3 + i) : 0.f;
    }
  }
};

// Component k of X = x - sign*(ht/2)*(v + v(X~)) as a displacement:
// disp_k = h_k (v_k + v_k(X~)), h_k = -sign*(ht/2)*N_k/(2 pi).
struct TrajectoryEpi {
  const float* vk;
  float* dk;
  float h;
  CB_DEVICE void operator()(const TileThread& tt, int a, float vx) const {
    if (tt.valid_idx(a)) dk[tt.idx(a)] = h * (__ldg(vk + tt.idx(a)) + vx);
  }
};

// Epilogues of the table-driven gathers: operator()(tt, a, value, aux_a) with
// aux_a = aux[point] prefetched by the gather (aux may be null).
struct StoreEpi {
  float* dst;
  const float* aux = nullptr;
  CB_DEVICE void operator()(const TileThread& tt, int a, float val, float) const {
    if (tt.valid_idx(a)) dst[tt.idx(a)] = val;
  }
};

// bf16 image output (round to nearest even)
struct Store16Epi {
  bf16* dst;
  const float* aux = nullptr;
  CB_DEVICE void operator()(const TileThread& tt, int a, float val, float) const {
    if (tt.valid_idx(a)) dst[tt.idx(a)] = __float2bfloat16_rn(val);
  }
};

// out = c * val (aux = c)
struct ScaleEpi {
  float* out;
  const float* aux;
  CB_DEVICE void operator()(const TileThread& tt, int a, float val, float c) const {
    if (tt.valid_idx(a)) out[tt.idx(a)] = c * val;
  }
};

// out = sign * (val + src) (aux = src)
struct AddEpi {
  float* out;
  float sign;
  const float* aux;
  CB_DEVICE void operator()(const TileThread& tt, int a, float val, float src) const {
    if (tt.valid_idx(a)) out[tt.idx(a)] = sign * (val + src);
  }
};

// out = 1 + ht/2 (s dx + s dv + ht dx dv), dx = divv(X) (the gathered value),
// dv = divv (aux), s = +-1
struct AdjCoefEpi {
  float* out;
  float ht, sgn;
  const float* aux;
  CB_DEVICE void operator()(const TileThread& tt, int a, float dx, float dv) const {
    if (tt.valid_idx(a)) out[tt.idx(a)] = 1.f + 0.5f * ht * (sgn * (dx + dv) + ht * dx * dv);
  }
};

// per-problem partials of sum, min and max of a scalar field (FP64 sum)
__global__ void __launch_bounds__(256) k_field_stats(const float* __restrict__ f, long long fp, long long n,
                                                     double* __restrict__ out, int nparts) {
  const float* pf = f + blockIdx.y * fp;
  double s = 0.0;
  float mn = INFINITY, mx = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = pf[i];
    s += (double)x;
    mn = fminf(mn, x);
    mx = fmaxf(mx, x);
  }
  __shared__ double ss[8];
  __shared__ float smn[8], smx[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    ss[w] = s;
    smn[w] = mn;
    smx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s = ss[0];
    mn = smn[0];
    mx = smx[0];
    for (int k = 1; k < 8; ++k) {
      s += ss[k];
      mn = fminf(mn, smn[k]);
      mx = fmaxf(mx, smx[k]);
    }
    double* o = out + (long long)blockIdx.y * 3 * nparts;
    o[blockIdx.x] = s;
    o[nparts + blockIdx.x] = mn;
    o[2 * nparts + blockIdx.x] = mx;
  }
}

// ---- gather kernels (grid: tiles x problems x fields) -------------------------

__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_trajectory(const float* __restrict__ v, long long vp, float* __restrict__ disp, long long dp, Dims d,
                 float ht, float sign, const int* __restrict__ active) {
  const int p = blockIdx.y, k = blockIdx.z;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  const float* v1 = v + p * vp;
  const float c0 = (float)(d.n1 / kTwoPi), c1 = (float)(d.n2 / kTwoPi), c2 = (float)(d.n3 / kTwoPi);
  VelocitySource src{v1, -sign * ht * c0, -sign * ht * c1, -sign * ht * c2};
  const float ck = k == 0 ? c0 : (k == 1 ? c1 : c2);
  const float* vk = v1 + k * d.n();
  TrajectoryEpi epi{vk, disp + p * dp + k * d.n(), -sign * 0.5f * ht * ck};
  tile_gather(sbuf, src, vk, d, epi);
}

// field z of f (ff apart) -> field z of out (of apart)
__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_interp(const float* __restrict__ f, long long fp, long long ff, const float* __restrict__ disp, long long dp,
             const int4* __restrict__ tab, long long tp, float* __restrict__ out, long long op, long long of, Dims d,
             const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  StoreEpi epi{out + p * op + (long long)blockIdx.z * of, nullptr};
  tile_gather_tab(sbuf, disp + p * dp, tab + p * tp, f + p * fp + (long long)blockIdx.z * ff, d, epi);
}

// bf16 image field of problem p -> bf16 out (one state time step)
__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_interp16(const bf16* __restrict__ f, long long fp, const float* __restrict__ disp, long long dp,
               const int4* __restrict__ tab, long long tp, bf16* __restrict__ out, long long op, Dims d,
               const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  Store16Epi epi{out + p * op, nullptr};
  tile_gather_tab(sbuf, disp + p * dp, tab + p * tp, f + p * fp, d, epi);
}

__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_gather_scale(const float* __restrict__ f, long long fp, const float* __restrict__ disp, long long dp,
                   const int4* __restrict__ tab, long long tp, const float* __restrict__ c, long long cp,
                   float* __restrict__ out, long long op, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  ScaleEpi epi{out + p * op, c + p * cp};
  tile_gather_tab(sbuf, disp + p * dp, tab + p * tp, f + p * fp, d, epi);
}

__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_gather_add(const float* __restrict__ f, long long fp, const float* __restrict__ disp, long long dp,
                 const int4* __restrict__ tab, long long tp, const float* __restrict__ s, long long sp,
                 float* __restrict__ out, long long op, float sign, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  AddEpi epi{out + p * op, sign, s + p * sp};
  tile_gather_tab(sbuf, disp + p * dp, tab + p * tp, f + p * fp, d, epi);
}

__global__ void __launch_bounds__(kTileThreads, kGatherMinBlocks)
    k_adjoint_coef(const float* __restrict__ divv, long long vp, const float* __restrict__ disp, long long dp,
                   const int4* __restrict__ tab, long long tp, float* __restrict__ out, long long op, float ht,
                   float sgn, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  AdjCoefEpi epi{out + p * op, ht, sgn, divv + p * vp};
  tile_gather_tab(sbuf, disp + p * dp, tab + p * tp, divv + p * vp, d, epi);
}

// Box table of a displacement field (sl_tile.cuh box_from_table layout).
__global__ void __launch_bounds__(kTileThreads)
    k_tile_table(const float* __restrict__ disp, long long dp, int4* __restrict__ tab, long long tp, Dims d,
                 const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const TileThread tt = tile_thread(d);
  float dd[kTilePts][3];
  DispSource{disp + p * dp}.load(dd, tt, d);
  int lo[3], hi[3];
  tile_bounds(dd, tt, lo, hi);
  if (threadIdx.x == 0) {
    int4* t = tab + p * tp + 2 * blockIdx.x;
    pack_box(box_from_bounds(lo, hi, d), t[0], t[1]);
  }
}

// ---- pointwise kernels (4 consecutive points per thread, float4) ---------------

__global__ void k_body_force(const float* __restrict__ lam, long long lp, const float* __restrict__ gm, long long gp,
                             float* __restrict__ b, long long bp, int nt, float ht, float scale, long long n,
                             const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const long long i = 4 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  if (i >= n) return;
  const float* L = lam + p * lp;
  const float* G = gm + p * gp;
  float4 acc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int l = 0; l <= nt; ++l) {
    const float w = (l == 0 || l == nt) ? 0.5f * ht : ht;
    const float4 lv = __ldg(reinterpret_cast<const float4*>(L + l * n + i));
    const float4 wl = make_float4(w * lv.x, w * lv.y, w * lv.z, w * lv.w);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 g = __ldg(reinterpret_cast<const float4*>(G + (3 * l + k) * n + i));
      acc[k].x += wl.x * g.x;
      acc[k].y += wl.y * g.y;
      acc[k].z += wl.z * g.z;
      acc[k].w += wl.w * g.w;
    }
  }
  float* bb = b + p * bp;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    *reinterpret_cast<float4*>(bb + k * n + i) =
        make_float4(scale * acc[k].x, scale * acc[k].y, scale * acc[k].z, scale * acc[k].w);
}

// Second RK2 stage of the deformation-gradient transport
// (DeformationFields::ComputeDefGradSL, src/DeformationFields.cpp:1060-1085),
// as written there: with tensors stored component-major (T_ab at T + (3a+b)n),
// rhs_ab = sum_k gvX_ka jX_kb and
// j_ab = jX_ab + ht/2 (rhs_ab + gvX_ab + ht sum_k gv_ka rhs_kb).
__global__ void k_defgrad_step(const float* __restrict__ jx, const float* __restrict__ gvx,
                               const float* __restrict__ gv, float* __restrict__ j, long long pstride, float ht,
                               long long n, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const long long off = p * pstride;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float JX[9], GX[9], G[9], rhs[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      JX[c] = jx[off + c * n + i];
      GX[c] = gvx[off + c * n + i];
      G[c] = gv[off + c * n + i];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        rhs[3 * a + b] = GX[a] * JX[b] + GX[3 + a] * JX[3 + b] + GX[6 + a] * JX[6 + b];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float s = G[a] * rhs[b] + G[3 + a] * rhs[3 + b] + G[6 + a] * rhs[6 + b];
        j[off + (3 * a + b) * n + i] = JX[3 * a + b] + 0.5f * ht * (rhs[3 * a + b] + (GX[3 * a + b] + ht * s));
      }
  }
}

int launch_defgrad_step(const float* jx, const float* gvx, const float* gv, float* j, long long pstride, float ht,
                        int nprob, long long n, const int* active, cudaStream_t s) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_defgrad_step<<<dim3((unsigned)blocks, nprob), 256, 0, s>>>(jx, gvx, gv, j, pstride, ht, n, active);
  return (int)cudaGetLastError();
}

__global__ void k_incstate_source(const float* __restrict__ gx, long long gxp, const float* __restrict__ vtx,
                                  long long vtxp, const float* __restrict__ gm, long long gmp,
                                  const float* __restrict__ vt, long long vtp, float* __restrict__ s, long long sp,
                                  int nt, float ht, long long n, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const long long i = 4 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  if (i >= n) return;
  float4 a[3], c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a[k] = __ldg(reinterpret_cast<const float4*>(vtx + p * vtxp + k * n + i));
    c[k] = __ldg(reinterpret_cast<const float4*>(vt + p * vtp + k * n + i));
  }
  const float hh = -0.5f * ht;
  const float* GX = gx + p * gxp;
  const float* GM = gm + p * gmp;
  float* S = s + p * sp;
  for (int j = 0; j < nt; ++j) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f), u = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 x = __ldg(reinterpret_cast<const float4*>(GX + (3 * j + k) * n + i));
      const float4 y = __ldg(reinterpret_cast<const float4*>(GM + (3 * (j + 1) + k) * n + i));
      t.x += x.x * a[k].x; t.y += x.y * a[k].y; t.z += x.z * a[k].z; t.w += x.w * a[k].w;
      u.x += y.x * c[k].x; u.y += y.y * c[k].y; u.z += y.z * c[k].z; u.w += y.w * c[k].w;
    }
    *reinterpret_cast<float4*>(S + j * n + i) =
        make_float4(hh * (t.x + u.x), hh * (t.y + u.y), hh * (t.z + u.z), hh * (t.w + u.w));
  }
}

// ---- launchers ---------------------------------------------------------------

int launch_trajectory(const float* v, long long vp, float* disp, long long dp, int nprob,
                      const Dims& d, float ht, float sign, const int* active, cudaStream_t s) {
  int e = allow_smem(k_trajectory);
  if (e) return e;
  k_trajectory<<<tile_grid(d, nprob, 3), kTileThreads, kGatherSmemBytes, s>>>(v, vp, disp, dp, d, ht, sign, active);
  return (int)cudaGetLastError();
}

long long tile_table_int4s(const Dims& d) { return 2LL * tile_count(d); }

int launch_tile_table(const float* disp, long long dp, int4* tab, long long tp, int nprob, const Dims& d,
                      const int* active, cudaStream_t s) {
  k_tile_table<<<tile_grid(d, nprob, 1), kTileThreads, 0, s>>>(disp, dp, tab, tp, d, active);
  return (int)cudaGetLastError();
}

int launch_interp(const float* f, long long fp, long long ff, const float* disp, long long dp, const int4* tab,
                  long long tp, float* out, long long op, long long of, int nf, int nprob, const Dims& d,
                  const int* active, cudaStream_t s) {
  int e = allow_smem(k_interp);
  if (e) return e;
  k_interp<<<tile_grid(d, nprob, nf), kTileThreads, kGatherSmemBytes, s>>>(f, fp, ff, disp, dp, tab, tp, out, op,
                                                                           of, d, active);
  return (int)cudaGetLastError();
}

int launch_interp16(const bf16* f, long long fp, const float* disp, long long dp, const int4* tab, long long tp,
                    bf16* out, long long op, int nprob, const Dims& d, const int* active, cudaStream_t s) {
  // staged boxes load 4-element chunks as 8-byte words (only when N3 % 4 == 0)
  if (!(d.n3 & 3) && ((reinterpret_cast<uintptr_t>(f) & 7) || (fp & 3))) return (int)cudaErrorInvalidValue;
  int e = allow_smem(k_interp16);
  if (e) return e;
  k_interp16<<<tile_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(f, fp, disp, dp, tab, tp, out, op, d,
                                                                            active);
  return (int)cudaGetLastError();
}

int launch_gather_scale(const float* f, long long fp, const float* disp, long long dp, const int4* tab,
                        long long tp, const float* c, long long cp, float* out, long long op, int nprob,
                        const Dims& d, const int* active, cudaStream_t s) {
  int e = allow_smem(k_gather_scale);
  if (e) return e;
  k_gather_scale<<<tile_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(f, fp, disp, dp, tab, tp, c, cp,
                                                                                out, op, d, active);
  return (int)cudaGetLastError();
}

int launch_gather_add(const float* f, long long fp, const float* disp, long long dp, const int4* tab,
                      long long tp, const float* src, long long sp, float* out, long long op, float sign, int nprob,
                      const Dims& d, const int* active, cudaStream_t s) {
  int e = allow_smem(k_gather_add);
  if (e) return e;
  k_gather_add<<<tile_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(f, fp, disp, dp, tab, tp, src, sp,
                                                                              out, op, sign, d, active);
  return (int)cudaGetLastError();
}

int launch_adjoint_coef(const float* divv, long long vp, const float* disp, long long dp, const int4* tab,
                        long long tp, float* out, long long op, float ht, int nprob, const Dims& d,
                        const int* active, cudaStream_t s, float sgn) {
  int e = allow_smem(k_adjoint_coef);
  if (e) return e;
  k_adjoint_coef<<<tile_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(divv, vp, disp, dp, tab, tp, out,
                                                                                op, ht, sgn, d, active);
  return (int)cudaGetLastError();
}

static dim3 quad_grid(long long n, int nprob) {
  const long long q = n / 4;
  return dim3((unsigned)((q + kSlThreads - 1) / kSlThreads), nprob);
}

int launch_body_force(const float* lam, long long lp, const float* gm, long long gp, float* b, long long bp,
                      int nt, float ht, float scale, int nprob, long long n, const int* active, cudaStream_t s) {
  if (n % 4) return (int)cudaErrorInvalidValue;
  k_body_force<<<quad_grid(n, nprob), kSlThreads, 0, s>>>(lam, lp, gm, gp, b, bp, nt, ht, scale, n, active);
  return (int)cudaGetLastError();
}

int launch_incstate_source(const float* gx, long long gxp, const float* vtx, long long vtxp, const float* gm,
                           long long gmp, const float* vt, long long vtp, float* src, long long sp, int nt,
                           float ht, int nprob, long long n, const int* active, cudaStream_t s) {
  if (n % 4) return (int)cudaErrorInvalidValue;
  k_incstate_source<<<quad_grid(n, nprob), kSlThreads, 0, s>>>(gx, gxp, vtx, vtxp, gm, gmp, vt, vtp, src, sp, nt,
                                                               ht, n, active);
  return (int)cudaGetLastError();
}

}  // namespace cb

namespace cb {

int field_stats_parts(long long n) {
  const long long b = (n + 256 * 8 - 1) / (256 * 8);
  return (int)(b < 296 ? (b < 1 ? 1 : b) : 296);
}

int launch_field_stats(const float* f, long long fp, long long n, int nprob, double* partials, cudaStream_t s) {
  const int np = field_stats_parts(n);
  k_field_stats<<<dim3(np, nprob), 256, 0, s>>>(f, fp, n, partials, np);
  return (int)cudaGetLastError();
}

// Health of the box copies' bounded waits: tile gathers on this device whose
// box copy did not complete within the wait limit (each skipped its tile).
int stage_timeouts(unsigned long long* count, cudaStream_t s) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_stage_timeouts, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return (int)cudaGetLastError();
  *count = v;
  return 0;
}

// Self-test of the bounded wait: one CTA arms its barrier for 16 bytes that no
// copy delivers and waits wait_ns, so the wait runs out, is counted, and the
// kernel returns; the context stays usable.
__global__ void __launch_bounds__(kTileThreads) k_stage_wait_selftest(unsigned long long wait_ns) {
  __shared__ alignas(8) unsigned long long mbar;
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&mbar);
  if (threadIdx.x == 0) {
    mbar_init(bar);
    mbar_arrive_expect(bar, 16u);
  }
  __syncthreads();
  if (threadIdx.x == 0) stage_box_wait(bar, wait_ns);  // nothing delivers the 16 bytes
}

int launch_stage_wait_selftest(unsigned long long wait_ns, cudaStream_t s) {
  k_stage_wait_selftest<<<1, kTileThreads, 0, s>>>(wait_ns);
  return (int)cudaGetLastError();
}

}  // namespace cb
