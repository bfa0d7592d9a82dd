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
// one GPU: the periodic wrap is applied while staging each CTA's footprint
// box in shared memory (sl_tile.cuh).
#include "sl_tile.cuh"

namespace cb {

constexpr int kSlThreads = 256;

static dim3 point_grid(long long n, int nprob) {
  return dim3((unsigned)((n + kSlThreads - 1) / kSlThreads), nprob);
}

#ifndef CB_TILE_MIN_BLOCKS
#define CB_TILE_MIN_BLOCKS 2
#endif
constexpr int kTileMinBlocks = CB_TILE_MIN_BLOCKS;  // resident CTAs per SM the register budget targets

static dim3 tile_grid(const Dims& d, int nprob, int nz = 1) { return dim3(tile_blocks(d), nprob, nz); }

// Xt = x - sign*ht*v; vX = v(Xt); X = x - sign*(ht/2)*(v + vX)  (grid units)
__global__ void __launch_bounds__(kTileThreads, kTileMinBlocks) k_trajectory(const float* __restrict__ v, long long vp,
                                                                float* __restrict__ disp, long long dp, Dims d,
                                                                float ht, float sign, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  __shared__ __align__(16) float sb[kBoxBudget];
  const long long n = d.n();
  const float* v1 = v + p * vp;
  const float c1 = (float)(d.n1 / kTwoPi), c2 = (float)(d.n2 / kTwoPi), c3 = (float)(d.n3 / kTwoPi);
  const TileRow row = tile_row(d);
  TilePoint pts[kTX1];
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (!row.valid(a, d)) {
      pts[a] = TilePoint{{0, 0, 0}, {0.f, 0.f, 0.f}};
      continue;
    }
    const long long i = row.idx(a);
    set_point(pts[a], row.t1 + a, row.i2, row.i3, -sign * ht * v1[i] * c1, -sign * ht * v1[n + i] * c2,
              -sign * ht * v1[2 * n + i] * c3);
  }
  const TileBox box = tile_box(pts, row, d);
  float vx[3][kTX1];
  tile_gather<3>(sb, v1, n, pts, row, box, d, vx);
  float* o = disp + p * dp;
  const float hh = 0.5f * ht;
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (!row.valid(a, d)) continue;
    const long long i = row.idx(a);
    o[i] = -sign * hh * (v1[i] + vx[0][a]) * c1;
    o[n + i] = -sign * hh * (v1[n + i] + vx[1][a]) * c2;
    o[2 * n + i] = -sign * hh * (v1[2 * n + i] + vx[2][a]) * c3;
  }
}

// NF fields (1 or 3) gathered at one characteristic; grid.z runs over groups
// of NF fields (group g: fields g*NF .. g*NF+NF-1).
template <int NF>
__global__ void __launch_bounds__(kTileThreads, kTileMinBlocks)
    k_interp(const float* __restrict__ f, long long fp, long long ff, const float* __restrict__ disp, long long dp,
             float* __restrict__ out, long long op, long long of, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  __shared__ __align__(16) float sb[kBoxBudget];
  const TileRow row = tile_row(d);
  TilePoint pts[kTX1];
  tile_points_from_disp(pts, row, disp + p * dp, d);
  const TileBox box = tile_box(pts, row, d);
  const float* src = f + p * fp + (long long)blockIdx.z * NF * ff;
  float* dst = out + p * op + (long long)blockIdx.z * NF * of;
  float vals[NF][kTX1];
  tile_gather<NF>(sb, src, ff, pts, row, box, d, vals);
#pragma unroll
  for (int k = 0; k < NF; ++k)
#pragma unroll
    for (int a = 0; a < kTX1; ++a)
      if (row.valid(a, d)) dst[k * of + row.idx(a)] = vals[k][a];
}

__global__ void __launch_bounds__(kTileThreads, kTileMinBlocks) k_adjoint_step(
    const float* __restrict__ lam_in, float* __restrict__ lam_out, long long lp,
    const float* __restrict__ disp, long long dp, const float* __restrict__ divv,
    const float* __restrict__ divvx, long long vp, const float* __restrict__ g, long long gp,
    float* __restrict__ b, long long bp, float ht, float w, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  __shared__ __align__(16) float sb[kBoxBudget];
  const long long n = d.n();
  const TileRow row = tile_row(d);
  TilePoint pts[kTX1];
  tile_points_from_disp(pts, row, disp + p * dp, d);
  const TileBox box = tile_box(pts, row, d);
  const float* li = lam_in + p * lp;
  float lx[1][kTX1];
  tile_gather<1>(sb, li, 0, pts, row, box, d, lx);
  const float* gg = g + p * gp;
  float* bb = b + p * bp;
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (!row.valid(a, d)) continue;
    const long long i = row.idx(a);
    const float lam = li[i];
    const float dvx = divvx[p * vp + i], dv = divv[p * vp + i];
    const float rhs0 = lx[0][a] * dvx;
    const float rhs1 = (lx[0][a] + ht * rhs0) * dv;
    bb[i] += w * gg[i] * lam;
    bb[n + i] += w * gg[n + i] * lam;
    bb[2 * n + i] += w * gg[2 * n + i] * lam;
    lam_out[p * lp + i] = lx[0][a] + 0.5f * ht * (rhs0 + rhs1);
  }
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

__global__ void __launch_bounds__(kTileThreads, kTileMinBlocks) k_incstate_step(
    const float* __restrict__ mt_in, float* __restrict__ mt_out, long long mp,
    const float* __restrict__ disp, long long dp, const float* __restrict__ gx, long long gxp,
    const float* __restrict__ vtx, const float* __restrict__ g1, long long g1p,
    const float* __restrict__ vt, long long vtp, float ht, Dims d, const int* __restrict__ active) {
  const int p = blockIdx.y;
  if (active && !active[p]) return;
  __shared__ __align__(16) float sb[kBoxBudget];
  const long long n = d.n();
  const TileRow row = tile_row(d);
  TilePoint pts[kTX1];
  tile_points_from_disp(pts, row, disp + p * dp, d);
  const TileBox box = tile_box(pts, row, d);
  float mx[1][kTX1];
  tile_gather<1>(sb, mt_in + p * mp, 0, pts, row, box, d, mx);
  const float hh = 0.5f * ht;
  const float* a3 = gx + p * gxp;
  const float* ax = vtx + p * vtp;
  const float* c3 = g1 + p * g1p;
  const float* cv = vt + p * vtp;
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (!row.valid(a, d)) continue;
    const long long i = row.idx(a);
    float m = mx[0][a];
    m -= hh * (a3[i] * ax[i] + a3[n + i] * ax[n + i] + a3[2 * n + i] * ax[2 * n + i]);
    m -= hh * (c3[i] * cv[i] + c3[n + i] * cv[n + i] + c3[2 * n + i] * cv[2 * n + i]);
    mt_out[p * mp + i] = m;
  }
}

int launch_trajectory(const float* v, long long vp, float* disp, long long dp, int nprob,
                      const Dims& d, float ht, float sign, const int* active, cudaStream_t s) {
  k_trajectory<<<tile_grid(d, nprob), kTileThreads, 0, s>>>(v, vp, disp, dp, d, ht, sign, active);
  return (int)cudaGetLastError();
}

int launch_interp(const float* f, long long fp, long long ff, const float* disp, long long dp,
                  float* out, long long op, long long of, int nf, int nprob, const Dims& d,
                  const int* active, cudaStream_t s) {
  if (nf % 3 == 0) {
    k_interp<3><<<tile_grid(d, nprob, nf / 3), kTileThreads, 0, s>>>(f, fp, ff, disp, dp, out, op, of, d, active);
  } else {
    k_interp<1><<<tile_grid(d, nprob, nf), kTileThreads, 0, s>>>(f, fp, ff, disp, dp, out, op, of, d, active);
  }
  return (int)cudaGetLastError();
}

int launch_adjoint_step(const float* lam_in, float* lam_out, long long lp, const float* disp,
                        long long dp, const float* divv, const float* divvx, long long vp,
                        const float* g, long long gp, float* b, long long bp, float ht, float w,
                        int nprob, const Dims& d, const int* active, cudaStream_t s) {
  k_adjoint_step<<<tile_grid(d, nprob), kTileThreads, 0, s>>>(lam_in, lam_out, lp, disp, dp, divv, divvx, vp, g,
                                                                gp, b, bp, ht, w, d, active);
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
  k_incstate_step<<<tile_grid(d, nprob), kTileThreads, 0, s>>>(mt_in, mt_out, mp, disp, dp, gx, gxp, vtx, g1, g1p,
                                                                 vt, vtp, ht, d, active);
  return (int)cudaGetLastError();
}

}  // namespace cb
