// Semi-Lagrangian kernels: RK2 characteristics, tricubic gathers and the
// fused state / adjoint / incremental time steps.
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
#include <mutex>

#include "sl_tile.cuh"

namespace cb {

constexpr int kSlThreads = 256;

static dim3 point_grid(long long n, int nprob) {
  return dim3((unsigned)((n + kSlThreads - 1) / kSlThreads), nprob);
}

// Persistent grid: two CTAs per SM (each holds two 48 KB boxes), capped by
// the number of tiles.
static dim3 persist_grid(const Dims& d, int nprob, int nz) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const unsigned nt = tile_count(d);
  const unsigned cap = (unsigned)(kPersistCtasPerSm * sms);
  return dim3(nt < cap ? nt : cap, nprob, nz);
}

template <typename K>
static int allow_gather_smem(K kernel) {
  return (int)cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGatherSmemBytes);
}

// ---- point sources and tile epilogues ---------------------------------------

// First RK2 stage of the characteristic: disp = -sign*ht*v*N/(2 pi).
struct VelocitySource {
  const float* v;
  float c0, c1, c2;  // -sign*ht*N_k/(2 pi)
  CB_DEVICE void points(TilePoint (&pts)[kTX1], const TileRow& row, const Dims& d) const {
    const long long n = d.n();
#pragma unroll
    for (int a = 0; a < kTX1; ++a) {
      if (!row.valid(a, d)) {
        pts[a] = TilePoint{{0, 0, 0}, {0.f, 0.f, 0.f}};
        continue;
      }
      const long long i = row.idx(a);
      set_point(pts[a], row.t1 + a, row.i2, row.i3, c0 * __ldg(v + i), c1 * __ldg(v + n + i),
                c2 * __ldg(v + 2 * n + i));
    }
  }
};

// X = x - sign*(ht/2)*(v + v(Xt)) as a displacement.
struct TrajectoryEpi {
  const float* v;
  float* disp;
  float h0, h1, h2;  // -sign*(ht/2)*N_k/(2 pi)
  Dims d;
  CB_DEVICE void operator()(const TileRow& row, const float (&vx)[3][kTX1]) const {
    const long long n = d.n();
#pragma unroll
    for (int a = 0; a < kTX1; ++a) {
      if (!row.valid(a, d)) continue;
      const long long i = row.idx(a);
      disp[i] = h0 * (__ldg(v + i) + vx[0][a]);
      disp[n + i] = h1 * (__ldg(v + n + i) + vx[1][a]);
      disp[2 * n + i] = h2 * (__ldg(v + 2 * n + i) + vx[2][a]);
    }
  }
};

template <int NF>
struct StoreEpi {
  float* dst;
  long long of;
  Dims d;
  CB_DEVICE void operator()(const TileRow& row, const float (&vals)[NF][kTX1]) const {
#pragma unroll
    for (int k = 0; k < NF; ++k)
#pragma unroll
      for (int a = 0; a < kTX1; ++a)
        if (row.valid(a, d)) dst[k * of + row.idx(a)] = vals[k][a];
  }
};

// lam_out = lx + ht/2 (rhs0 + rhs1), rhs0 = lx*divvx, rhs1 = (lx + ht*rhs0)*divv;
// b += w * g * lam_in  (src/CLAIRE.cpp:2646-2686, 3940-3971)
struct AdjointEpi {
  const float *lam_in, *divv, *divvx, *g;
  float *lam_out, *b;
  float ht, w;
  Dims d;
  CB_DEVICE void operator()(const TileRow& row, const float (&lx)[1][kTX1]) const {
    const long long n = d.n();
#pragma unroll
    for (int a = 0; a < kTX1; ++a) {
      if (!row.valid(a, d)) continue;
      const long long i = row.idx(a);
      const float lam = __ldg(lam_in + i);
      const float rhs0 = lx[0][a] * __ldg(divvx + i);
      const float rhs1 = (lx[0][a] + ht * rhs0) * __ldg(divv + i);
      b[i] += w * __ldg(g + i) * lam;
      b[n + i] += w * __ldg(g + n + i) * lam;
      b[2 * n + i] += w * __ldg(g + 2 * n + i) * lam;
      lam_out[i] = lx[0][a] + 0.5f * ht * (rhs0 + rhs1);
    }
  }
};

// mt_out = mt_in(X) - ht/2 (gx . vtx) - ht/2 (g1 . vt)  (src/CLAIRE.cpp:3220-3276)
struct IncStateEpi {
  const float *gx, *vtx, *g1, *vt;
  float* mt_out;
  float ht;
  Dims d;
  CB_DEVICE void operator()(const TileRow& row, const float (&mx)[1][kTX1]) const {
    const long long n = d.n();
    const float hh = 0.5f * ht;
#pragma unroll
    for (int a = 0; a < kTX1; ++a) {
      if (!row.valid(a, d)) continue;
      const long long i = row.idx(a);
      float m = mx[0][a];
      m -= hh * (__ldg(gx + i) * __ldg(vtx + i) + __ldg(gx + n + i) * __ldg(vtx + n + i) +
                 __ldg(gx + 2 * n + i) * __ldg(vtx + 2 * n + i));
      m -= hh * (__ldg(g1 + i) * __ldg(vt + i) + __ldg(g1 + n + i) * __ldg(vt + n + i) +
                 __ldg(g1 + 2 * n + i) * __ldg(vt + 2 * n + i));
      mt_out[i] = m;
    }
  }
};

// ---- kernels ----------------------------------------------------------------

__global__ void __launch_bounds__(kTileThreads, kPersistCtasPerSm)
    k_trajectory(const float* __restrict__ v, long long vp, float* __restrict__ disp, long long dp, Dims d,
                 float ht, float sign, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  const float* v1 = v + p * vp;
  const float c0 = (float)(d.n1 / kTwoPi), c1 = (float)(d.n2 / kTwoPi), c2 = (float)(d.n3 / kTwoPi);
  VelocitySource src{v1, -sign * ht * c0, -sign * ht * c1, -sign * ht * c2};
  const float hh = 0.5f * ht;
  TrajectoryEpi epi{v1, disp + p * dp, -sign * hh * c0, -sign * hh * c1, -sign * hh * c2, d};
  pipelined_gather<3>(sbuf, src, v1, d.n(), d, epi);
}

// NF fields (1 or 3) gathered at one characteristic; grid.z runs over groups
// of NF fields (group g: fields g*NF .. g*NF+NF-1).
template <int NF>
__global__ void __launch_bounds__(kTileThreads, kPersistCtasPerSm)
    k_interp(const float* __restrict__ f, long long fp, long long ff, const float* __restrict__ disp, long long dp,
             float* __restrict__ out, long long op, long long of, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  DispSource src{disp + p * dp};
  StoreEpi<NF> epi{out + p * op + (long long)blockIdx.z * NF * of, of, d};
  pipelined_gather<NF>(sbuf, src, f + p * fp + (long long)blockIdx.z * NF * ff, ff, d, epi);
}

__global__ void __launch_bounds__(kTileThreads, kPersistCtasPerSm) k_adjoint_step(
    const float* __restrict__ lam_in, float* __restrict__ lam_out, long long lp,
    const float* __restrict__ disp, long long dp, const float* __restrict__ divv,
    const float* __restrict__ divvx, long long vp, const float* __restrict__ g, long long gp,
    float* __restrict__ b, long long bp, float ht, float w, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  DispSource src{disp + p * dp};
  AdjointEpi epi{lam_in + p * lp, divv + p * vp, divvx + p * vp, g + p * gp, lam_out + p * lp, b + p * bp, ht, w, d};
  pipelined_gather<1>(sbuf, src, lam_in + p * lp, 0, d, epi);
}

__global__ void k_body_force_final(float* __restrict__ b, long long bp, const float* __restrict__ g,
                                   long long gp, const float* __restrict__ lam, long long lp, float w,
                                   float hd, long long n, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float l = lam[p * lp + i];
  float* bb = b + p * bp;
  const float* gg = g + p * gp;
  bb[i] = hd * (bb[i] + w * gg[i] * l);
  bb[n + i] = hd * (bb[n + i] + w * gg[n + i] * l);
  bb[2 * n + i] = hd * (bb[2 * n + i] + w * gg[2 * n + i] * l);
}

__global__ void __launch_bounds__(kTileThreads, kPersistCtasPerSm) k_incstate_step(
    const float* __restrict__ mt_in, float* __restrict__ mt_out, long long mp,
    const float* __restrict__ disp, long long dp, const float* __restrict__ gx, long long gxp,
    const float* __restrict__ vtx, const float* __restrict__ g1, long long g1p,
    const float* __restrict__ vt, long long vtp, float ht, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  extern __shared__ __align__(16) float sbuf[];
  DispSource src{disp + p * dp};
  IncStateEpi epi{gx + p * gxp, vtx + p * vtp, g1 + p * g1p, vt + p * vtp, mt_out + p * mp, ht, d};
  pipelined_gather<1>(sbuf, src, mt_in + p * mp, 0, d, epi);
}

// ---- launchers ---------------------------------------------------------------

int launch_trajectory(const float* v, long long vp, float* disp, long long dp, int nprob,
                      const Dims& d, float ht, float sign, const int* active, cudaStream_t s) {
  int e = allow_gather_smem(k_trajectory);
  if (e) return e;
  k_trajectory<<<persist_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(v, vp, disp, dp, d, ht, sign,
                                                                                  active);
  return (int)cudaGetLastError();
}

int launch_interp(const float* f, long long fp, long long ff, const float* disp, long long dp,
                  float* out, long long op, long long of, int nf, int nprob, const Dims& d,
                  const int* active, cudaStream_t s) {
  int e = 0;
  if (nf % 3 == 0) {
    e = allow_gather_smem(k_interp<3>);
    if (e) return e;
    k_interp<3><<<persist_grid(d, nprob, nf / 3), kTileThreads, kGatherSmemBytes, s>>>(f, fp, ff, disp, dp, out,
                                                                                       op, of, d, active);
  } else {
    e = allow_gather_smem(k_interp<1>);
    if (e) return e;
    k_interp<1><<<persist_grid(d, nprob, nf), kTileThreads, kGatherSmemBytes, s>>>(f, fp, ff, disp, dp, out, op,
                                                                                   of, d, active);
  }
  return (int)cudaGetLastError();
}

int launch_adjoint_step(const float* lam_in, float* lam_out, long long lp, const float* disp,
                        long long dp, const float* divv, const float* divvx, long long vp,
                        const float* g, long long gp, float* b, long long bp, float ht, float w,
                        int nprob, const Dims& d, const int* active, cudaStream_t s) {
  int e = allow_gather_smem(k_adjoint_step);
  if (e) return e;
  k_adjoint_step<<<persist_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(
      lam_in, lam_out, lp, disp, dp, divv, divvx, vp, g, gp, b, bp, ht, w, d, active);
  return (int)cudaGetLastError();
}

int launch_body_force_final(float* b, long long bp, const float* g, long long gp, const float* lam,
                            long long lp, float w, float hd_scale, int nprob, long long n,
                            const int* active, cudaStream_t s) {
  k_body_force_final<<<point_grid(n, nprob), kSlThreads, 0, s>>>(b, bp, g, gp, lam, lp, w, hd_scale, n, active);
  return (int)cudaGetLastError();
}

int launch_incstate_step(const float* mt_in, float* mt_out, long long mp, const float* disp,
                         long long dp, const float* gx, long long gxp, const float* vtx,
                         const float* g1, long long g1p, const float* vt, long long vtp, float ht,
                         int nprob, const Dims& d, const int* active, cudaStream_t s) {
  int e = allow_gather_smem(k_incstate_step);
  if (e) return e;
  k_incstate_step<<<persist_grid(d, nprob, 1), kTileThreads, kGatherSmemBytes, s>>>(
      mt_in, mt_out, mp, disp, dp, gx, gxp, vtx, g1, g1p, vt, vtp, ht, d, active);
  return (int)cudaGetLastError();
}

}  // namespace cb
