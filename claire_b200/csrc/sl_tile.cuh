// Shared-memory tiled tricubic gathers.
//
// One CTA of 256 threads owns a tile of 8 (x1) x 8 (x2) x 16 (x3) output
// points.  Warp w covers x2 row w of the tile; lanes 0-15 and 16-31 cover the
// 16 x3 points of two adjacent x1 planes, and each thread holds 4 points
// (x1 = 2a + h, a < 4, h = lane / 16).
//
// The CTA reads its points' displacements, reduces the bounding box of every
// stencil tap over the tile (min / max of i + floor(d), widened by the
// stencil's -1 .. +2) and, when the box fits, copies it into shared memory
// with bulk asynchronous copies (the TMA engine's untiled form), one per x3
// row of the box (two where the row crosses the periodic x3 seam; the x1 / x2
// wrap is applied per row), which complete on an mbarrier that every thread
// waits on (bounded).  The 64 taps
// per point are then served from shared memory; tiles whose box is too large
// (large, rough displacements) gather from global memory instead.
//
// Shared-memory layout of a box: x3 rows of pitch P floats (32 or 64, a
// multiple of 32, so lanes whose taps fall in different x2 rows still hit
// distinct banks), x1 planes of stride Q = ext2 * P + 16 (16 mod 32: the two
// half-warps, one plane apart, use opposite halves of the bank space).  Every
// shared-memory index is inside the box by construction: each point's taps lie
// in [i + floor(d) - 1, i + floor(d) + 2] and the box spans the min / max of
// exactly those values over the tile's points; points outside the grid
// (partial tiles) read the box origin and are never stored.
//
// The kernels are not persistent: several CTAs per SM (one tile each) overlap
// one another's copies with their gathers.
#pragma once

#include <climits>
#include <type_traits>

#include "sl.cuh"

namespace cb {

constexpr int kT1 = 8, kT2 = 8, kT3 = 16;
constexpr int kTileThreads = 256;
constexpr int kTilePts = 4;  // points per thread

// Shared-memory budget of a CTA (one box): 4 CTAs of 256 threads per SM.
constexpr int kGatherBudget = 8192;  // floats
constexpr int kGatherSmemBytes = kGatherBudget * 4;
constexpr int kGatherMinBlocks = 4;

__host__ __device__ inline unsigned tile_count(const Dims& d) {
  return (unsigned)(((d.n1 + kT1 - 1) / kT1) * ((d.n2 + kT2 - 1) / kT2) * ((d.n3 + kT3 - 1) / kT3));
}

// q / m for 0 <= q < 2^22 and 1 <= m < 2^12 without an integer division:
// float estimate, then one correction each way.
CB_DEVICE int small_div(int q, int m) {
  int t = __float2int_rz((float)q * (1.f / (float)m));
  const int r = q - t * m;
  t += (r >= m) ? 1 : 0;
  t -= (r < 0) ? 1 : 0;
  return t;
}

// x mod n for x in [-n, 2n)
CB_DEVICE int wrap_near(int x, int n) {
  x += (x < 0) ? n : 0;
  x -= (x >= n) ? n : 0;
  return x;
}

// This thread's points in the CTA's tile: (t1 + 2a, i2, i3), a < 4.  Point
// indices are 32-bit (grids up to 1024^3 points).
struct TileThread {
  int t1, i2, i3;
  unsigned vmask;  // bit a: point a lies inside the grid
  unsigned idx0, step2;
  CB_DEVICE bool valid_idx(int a) const { return (vmask >> a) & 1u; }
  CB_DEVICE bool valid(int a, const Dims&) const { return valid_idx(a); }
  CB_DEVICE int x1(int a) const { return t1 + 2 * a; }
  CB_DEVICE unsigned idx(int a) const { return idx0 + a * step2; }
};

CB_DEVICE TileThread tile_thread(const Dims& d) {
  const int nb3 = (d.n3 + kT3 - 1) / kT3, nb2 = (d.n2 + kT2 - 1) / kT2;
  const int t = blockIdx.x;
  const int r = small_div(t, nb3), c3 = t - r * nb3;
  const int c1 = small_div(r, nb2), c2 = r - c1 * nb2;
  const int lane = threadIdx.x & 31;
  TileThread tt;
  tt.t1 = c1 * kT1 + (lane >> 4);
  tt.i2 = c2 * kT2 + (threadIdx.x >> 5);
  tt.i3 = c3 * kT3 + (lane & 15);
  const bool row_ok = (tt.i2 < d.n2) && (tt.i3 < d.n3);
  tt.vmask = 0;
#pragma unroll
  for (int a = 0; a < kTilePts; ++a) tt.vmask |= (row_ok && tt.t1 + 2 * a < d.n1) ? (1u << a) : 0u;
  const unsigned plane = (unsigned)d.n2 * (unsigned)d.n3;
  tt.step2 = 2 * plane;
  tt.idx0 = (unsigned)tt.t1 * plane + (unsigned)tt.i2 * (unsigned)d.n3 + (unsigned)tt.i3;
  return tt;
}

struct TileBox {
  int lo[3];
  int e1, e2, e3;  // extents (e3 in whole 16-byte chunks)
  int P, Q;        // x3 row pitch, x1 plane stride (floats)
  int vol;         // e1 * Q, rounded up to a multiple of 32
  bool within;     // copyable (one wrap per axis, whole chunks)
};

// Box of the stencil bases b in [lo, hi] per axis (taps b .. b+3).
CB_DEVICE TileBox box_from_bounds(const int (&lo)[3], const int (&hi)[3], const Dims& d) {
  TileBox bx;
  int ext[3];
  bool within = true;
  const int nk[3] = {d.n1, d.n2, d.n3};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    bx.lo[k] = lo[k];
    const long long e = (long long)hi[k] - (long long)lo[k] + 4;
    ext[k] = (e > 0 && e <= 4096) ? (int)e : 4096;
    // one wrap per coordinate in the copy, origin within one period
    within = within && e > 0 && e <= nk[k] && lo[k] >= -nk[k] && lo[k] < nk[k];
  }
  // x3: start on a multiple of 4 floats and cover whole 4-float chunks so the
  // box is copied in 16-byte pieces (N3 % 4 == 0: no chunk straddles the seam)
  const int lo3a = bx.lo[2] & ~3;
  bx.e3 = ((bx.lo[2] + ext[2] - lo3a) + 3) & ~3;
  bx.lo[2] = lo3a;
  within = within && bx.e3 <= d.n3 && bx.e3 <= 64 && (d.n3 & 3) == 0;
  bx.e1 = ext[0];
  bx.e2 = ext[1];
  bx.P = bx.e3 <= 32 ? 32 : 64;
  bx.Q = bx.e2 * bx.P + 16;
  const long long vol = ((long long)bx.e1 * bx.Q + 31) & ~31LL;
  bx.vol = vol < (1 << 24) ? (int)vol : (1 << 24);
  bx.within = within;
  return bx;
}

// Block-wide min / max of the stencil bases of the tile's valid points.
// Contains __syncthreads: call once, from uniform control flow.
CB_DEVICE void tile_bounds(const float (&dd)[kTilePts][3], const TileThread& tt, int (&lo)[3], int (&hi)[3]) {
  __shared__ int red[6][kTileThreads / 32];
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
  for (int a = 0; a < kTilePts; ++a) {
    if (!tt.valid_idx(a)) continue;
    const int b1 = tt.x1(a) + (int)floorf(dd[a][0]) - 1;
    const int b2 = tt.i2 + (int)floorf(dd[a][1]) - 1;
    const int b3 = tt.i3 + (int)floorf(dd[a][2]) - 1;
    mn[0] = min(mn[0], b1);
    mx[0] = max(mx[0], b1);
    mn[1] = min(mn[1], b2);
    mx[1] = max(mx[1], b2);
    mn[2] = min(mn[2], b3);
    mx[2] = max(mx[2], b3);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    mn[k] = __reduce_min_sync(0xffffffffu, mn[k]);
    mx[k] = __reduce_max_sync(0xffffffffu, mx[k]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      red[k][warp] = mn[k];
      red[3 + k][warp] = mx[k];
    }
  }
  __syncthreads();
  // every warp reduces the 8 warp partials itself (lane l reads partial l % 8)
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = __reduce_min_sync(0xffffffffu, red[k][lane & 7]);
    hi[k] = __reduce_max_sync(0xffffffffu, red[3 + k][lane & 7]);
  }
}

CB_DEVICE TileBox tile_box(const float (&dd)[kTilePts][3], const TileThread& tt, const Dims& d) {
  int lo[3], hi[3];
  tile_bounds(dd, tt, lo, hi);
  return box_from_bounds(lo, hi, d);
}

// Per-tile box table of a displacement field: the tile's TileBox packed in two
// int4, {lo1, lo2, lo3, e1 | e2 << 16}, {e3 | P << 16, Q, vol, within}.  It
// depends on the displacement only, so one table serves every gather at that
// characteristic (all time steps, all matvecs of a GN iterate).
CB_DEVICE void pack_box(const TileBox& bx, int4& a, int4& b) {
  a = make_int4(bx.lo[0], bx.lo[1], bx.lo[2], (bx.e1 & 0xffff) | (bx.e2 << 16));
  b = make_int4((bx.e3 & 0xffff) | (bx.P << 16), bx.Q, bx.vol, bx.within ? 1 : 0);
}

CB_DEVICE TileBox box_from_table(const int4* __restrict__ tab, const Dims&) {
  const int4 a = __ldg(tab + 2 * blockIdx.x), b = __ldg(tab + 2 * blockIdx.x + 1);
  TileBox bx;
  bx.lo[0] = a.x;
  bx.lo[1] = a.y;
  bx.lo[2] = a.z;
  bx.e1 = a.w & 0xffff;
  bx.e2 = a.w >> 16;
  bx.e3 = b.x & 0xffff;
  bx.P = b.x >> 16;
  bx.Q = b.y;
  bx.vol = b.z;
  bx.within = b.w != 0;
  return bx;
}

// ---- bulk box copies completing on an mbarrier ------------------------------
// Count of tile gathers whose box copy did not complete within the wait limit
// (the gather then skips its points); read by stage_timeouts().
__device__ unsigned g_stage_timeouts = 0;

// Wait limit of a box copy (ns of %globaltimer); the copies of one box take
// microseconds.
constexpr unsigned long long kStageWaitNs = 200000000ull;

CB_DEVICE unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
CB_DEVICE void mbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n\tfence.mbarrier_init.release.cluster;" ::"r"(bar)
               : "memory");
}
// the barrier's one arrival, announcing the bytes its copies will deliver
CB_DEVICE void mbar_arrive_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// One try_wait on phase 0; a thread whose phase is not complete is suspended
// by the hardware for up to hint_ns (or until the phase completes).
CB_DEVICE bool mbar_test(unsigned bar, unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
// Wait for phase 0 of the barrier for at most limit_ns; false on timeout.
// Waiting threads sleep in try_wait (1 us at a time) instead of spinning.
CB_DEVICE bool mbar_wait(unsigned bar, unsigned long long limit_ns) {
  if (mbar_test(bar, 1000u)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(bar, 1000u))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
CB_DEVICE void bulk_copy(unsigned dst, const float* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Bytes of a staged box (every copy of it lands on the barrier).
CB_DEVICE unsigned box_bytes(const TileBox& bx) { return 4u * (unsigned)(bx.e1 * bx.e2 * bx.e3); }

// Bulk copies of field f's box into the box at shared address sbase: row r of
// the box (x1 plane r / e2, x2 row r % e2) by thread r (mod the CTA size).
// Every source and destination is 16-byte aligned and every size a multiple
// of 16 bytes: x3 starts on a multiple of 4 floats, N3 % 4 == 0, and P, Q are
// multiples of 4.  (Issuing all rows from one warp instead ran 1.6 times
// slower: the copies of a box must start from many threads at once.)
CB_DEVICE void issue_box_bulk(unsigned sbase, const float* __restrict__ f, const TileBox& bx, const Dims& d,
                              unsigned bar) {
  const int rows = bx.e1 * bx.e2;
  const int g3 = wrap_near(bx.lo[2], d.n3);
  const int first = min(bx.e3, d.n3 - g3);  // floats before the x3 seam
  const unsigned row = (unsigned)d.n3, plane = (unsigned)d.n2 * (unsigned)d.n3;
  for (int r = threadIdx.x; r < rows; r += kTileThreads) {
    const int l1 = small_div(r, bx.e2), l2 = r - l1 * bx.e2;
    const int g1 = wrap_near(bx.lo[0] + l1, d.n1), g2 = wrap_near(bx.lo[1] + l2, d.n2);
    const float* src = f + ((unsigned)g1 * plane + (unsigned)g2 * row);
    const unsigned dst = sbase + 4u * (unsigned)(l1 * bx.Q + l2 * bx.P);
    bulk_copy(dst, src + g3, 4u * (unsigned)first, bar);
    if (first < bx.e3) bulk_copy(dst + 4u * (unsigned)first, src, 4u * (unsigned)(bx.e3 - first), bar);
  }
}

// Start the bulk copy of a staged box: barrier set up and armed with the box's
// bytes by thread 0, published to the CTA, then the row copies.  Contains
// __syncthreads: call from uniform control flow.
CB_DEVICE void stage_box_start(unsigned sbase, const float* __restrict__ f, const TileBox& bx, const Dims& d,
                               unsigned bar) {
  if (threadIdx.x == 0) {
    mbar_init(bar);
    mbar_arrive_expect(bar, box_bytes(bx));
  }
  __syncthreads();
  issue_box_bulk(sbase, f, bx, d, bar);
}

// Wait for the box; on timeout count it, wait once more for the copies still
// in flight (bounded as well) and report false: the caller skips its points.
CB_DEVICE bool stage_box_wait(unsigned bar, unsigned long long limit_ns) {
  if (mbar_wait(bar, limit_ns)) return true;
  if (threadIdx.x == 0) atomicAdd(&g_stage_timeouts, 1u);
  mbar_wait(bar, limit_ns);
  return false;
}

// bf16 image field: the box is widened to FP32 while it is staged, with plain
// loads and stores.  Warp w copies x1 planes w, w + 8, ...; its lanes cover
// whole x3 rows of 4-element chunks, rows advancing without divisions (one
// conditional wrap per row along x2 and per plane along x1).  Each chunk is
// one 8-byte load (x3 offsets are multiples of 4 and N3 % 4 == 0, so every
// chunk is 8-byte aligned) and one 16-byte shared store; the shared-memory
// layout, and so the gather that reads it, is the FP32 one.
CB_DEVICE void issue_box(float* __restrict__ sb, const bf16* __restrict__ f, const TileBox& bx, const Dims& d) {
  const int nck = bx.e3 >> 2;
  const int rpi = small_div(32, nck);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = small_div(lane, nck), lc = lane - lr * nck;
  if (lr >= rpi || lr >= bx.e2) return;
  int g1 = wrap_near(bx.lo[0] + warp, d.n1);
  const int w2 = wrap_near(bx.lo[1] + lr, d.n2);
  int g3 = wrap_near(bx.lo[2], d.n3) + 4 * lc;
  g3 -= (g3 >= d.n3) ? d.n3 : 0;
  const bf16* fb = f + g3;
  const unsigned row = (unsigned)d.n3, plane = (unsigned)d.n2 * (unsigned)d.n3;
  constexpr int kWarps = kTileThreads / 32;
  for (int l1 = warp; l1 < bx.e1; l1 += kWarps) {
    const bf16* fp = fb + (unsigned)g1 * plane;
    float* sp = sb + l1 * bx.Q + lr * bx.P + 4 * lc;
    int g2 = w2;
    for (int l2 = lr; l2 < bx.e2; l2 += rpi) {
      const uint2 raw = __ldg(reinterpret_cast<const uint2*>(fp + (unsigned)g2 * row));
      const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
      const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
      *reinterpret_cast<float4*>(sp) = make_float4(lo.x, lo.y, hi.x, hi.y);
      sp += rpi * bx.P;
      g2 += rpi;
      while (g2 >= d.n2) g2 -= d.n2;
    }
    g1 += kWarps;
    g1 -= (g1 >= d.n1) ? d.n1 : 0;
  }
}

// Four consecutive floats at byte offset OFF from addr, weighted by w.
template <int OFF>
CB_DEVICE float row4(unsigned addr, const float (&w)[4]) {
  float x0, x1, x2, x3;
  asm volatile(
      "ld.shared.f32 %0, [%4+%5];\n\t"
      "ld.shared.f32 %1, [%4+%6];\n\t"
      "ld.shared.f32 %2, [%4+%7];\n\t"
      "ld.shared.f32 %3, [%4+%8];\n"
      : "=f"(x0), "=f"(x1), "=f"(x2), "=f"(x3)
      : "r"(addr), "n"(OFF), "n"(OFF + 4), "n"(OFF + 8), "n"(OFF + 12));
  return w[0] * x0 + w[1] * x1 + w[2] * x2 + w[3] * x3;
}

// 64-tap gather from a staged box with row pitch P (floats) and plane stride
// qb (bytes); base = shared address of the point's tap (0, 0, 0).
template <int P>
CB_DEVICE float gather_box(unsigned base, unsigned qb, const float (&w1)[4], const float (&w2)[4],
                           const float (&w3)[4]) {
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const unsigned pa = base + a * qb;
    const float t = w2[0] * row4<0>(pa, w3) + w2[1] * row4<P * 4>(pa, w3) + w2[2] * row4<P * 8>(pa, w3) +
                    w2[3] * row4<P * 12>(pa, w3);
    acc += w1[a] * t;
  }
  return acc;
}

// Shared-memory stencil of one point: tap (0,0,0) offset and weights.
struct BoxPoint {
  unsigned off;  // floats from the box origin
  float w1[4], w2[4], w3[4];
};

CB_DEVICE BoxPoint box_point(const float (&dp)[3], int x1, const TileThread& tt, bool ok, const TileBox& bx) {
  BoxPoint bp;
  const float f1 = floorf(dp[0]), f2 = floorf(dp[1]), f3 = floorf(dp[2]);
  lagrange4(dp[0] - f1, bp.w1);
  lagrange4(dp[1] - f2, bp.w2);
  lagrange4(dp[2] - f3, bp.w3);
  const int o1 = ok ? x1 + (int)f1 - 1 - bx.lo[0] : 0;
  const int o2 = ok ? tt.i2 + (int)f2 - 1 - bx.lo[1] : 0;
  const int o3 = ok ? tt.i3 + (int)f3 - 1 - bx.lo[2] : 0;
  bp.off = (unsigned)(o1 * bx.Q + o2 * bx.P + o3);
  return bp;
}

CB_DEVICE float gather_staged(unsigned sb, const BoxPoint& bp, const TileBox& bx) {
  const unsigned base = sb + bp.off * 4u;
  const unsigned qb = (unsigned)bx.Q * 4u;
  return bx.P == 32 ? gather_box<32>(base, qb, bp.w1, bp.w2, bp.w3) : gather_box<64>(base, qb, bp.w1, bp.w2, bp.w3);
}

// ---- two points per instruction: packed FP32 pairs (fma.rn.f32x2) ------------
// The thread's points a and a+1 are gathered together: their weights and
// partial sums live in 64-bit register pairs and every multiply-add of the
// tensor product is one f32x2 instruction for both points (each lane an
// ordinary round-to-nearest FP32 FMA, in the scalar code's order).
typedef unsigned long long f32x2;

CB_DEVICE f32x2 pk2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
CB_DEVICE float2 upk2(f32x2 r) {
  float2 o;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
  return o;
}
CB_DEVICE f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
CB_DEVICE f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
CB_DEVICE f32x2 dup2(float c) { return pk2(c, c); }

// lagrange4 of two fractions at once (same Horner steps)
CB_DEVICE void lagrange4x2(f32x2 s, f32x2 (&w)[4]) {
  w[0] = mul2(s, fma2(s, fma2(s, dup2(-1.f / 6.f), dup2(0.5f)), dup2(-1.f / 3.f)));
  w[1] = fma2(s, fma2(s, fma2(s, dup2(0.5f), dup2(-1.f)), dup2(-0.5f)), dup2(1.f));
  w[2] = mul2(s, fma2(s, fma2(s, dup2(-0.5f), dup2(0.5f)), dup2(1.f)));
  w[3] = mul2(s, fma2(mul2(s, s), dup2(1.f / 6.f), dup2(-1.f / 6.f)));
}

// Four consecutive floats at OFF from each of two addresses, weighted.
template <int OFF>
CB_DEVICE f32x2 row4x2(unsigned pa, unsigned pb, const f32x2 (&w)[4]) {
  float a0, a1, a2, a3, b0, b1, b2, b3;
  asm volatile(
      "ld.shared.f32 %0, [%8+%10];\n\t"
      "ld.shared.f32 %1, [%8+%11];\n\t"
      "ld.shared.f32 %2, [%8+%12];\n\t"
      "ld.shared.f32 %3, [%8+%13];\n\t"
      "ld.shared.f32 %4, [%9+%10];\n\t"
      "ld.shared.f32 %5, [%9+%11];\n\t"
      "ld.shared.f32 %6, [%9+%12];\n\t"
      "ld.shared.f32 %7, [%9+%13];\n"
      : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(b0), "=f"(b1), "=f"(b2), "=f"(b3)
      : "r"(pa), "r"(pb), "n"(OFF), "n"(OFF + 4), "n"(OFF + 8), "n"(OFF + 12));
  f32x2 r = mul2(w[0], pk2(a0, b0));
  r = fma2(w[1], pk2(a1, b1), r);
  r = fma2(w[2], pk2(a2, b2), r);
  return fma2(w[3], pk2(a3, b3), r);
}

template <int P>
CB_DEVICE f32x2 gather_box_x2(unsigned ba, unsigned bb, unsigned qb, const f32x2 (&w1)[4], const f32x2 (&w2)[4],
                              const f32x2 (&w3)[4]) {
  f32x2 acc = 0ull;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const unsigned pa = ba + a * qb, pb = bb + a * qb;
    f32x2 t = mul2(w2[0], row4x2<0>(pa, pb, w3));
    t = fma2(w2[1], row4x2<P * 4>(pa, pb, w3), t);
    t = fma2(w2[2], row4x2<P * 8>(pa, pb, w3), t);
    t = fma2(w2[3], row4x2<P * 12>(pa, pb, w3), t);
    acc = (a == 0) ? mul2(w1[0], t) : fma2(w1[a], t, acc);
  }
  return acc;
}

// Staged gather of the thread's points a and a+1: values (x, y).
CB_DEVICE float2 gather_staged_pair(unsigned sb, const float (&da)[3], const float (&db)[3], int a,
                                    const TileThread& tt, const TileBox& bx) {
  float fa[3], fb[3];
  int oa[3], ob[3];
  const int xa[3] = {tt.x1(a), tt.i2, tt.i3}, xb[3] = {tt.x1(a + 1), tt.i2, tt.i3};
  const bool okA = tt.valid_idx(a), okB = tt.valid_idx(a + 1);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float la = floorf(da[k]), lb = floorf(db[k]);
    fa[k] = da[k] - la;
    fb[k] = db[k] - lb;
    oa[k] = okA ? xa[k] + (int)la - 1 - bx.lo[k] : 0;
    ob[k] = okB ? xb[k] + (int)lb - 1 - bx.lo[k] : 0;
  }
  f32x2 w1[4], w2[4], w3[4];
  lagrange4x2(pk2(fa[0], fb[0]), w1);
  lagrange4x2(pk2(fa[1], fb[1]), w2);
  lagrange4x2(pk2(fa[2], fb[2]), w3);
  const unsigned ba = sb + 4u * (unsigned)(oa[0] * bx.Q + oa[1] * bx.P + oa[2]);
  const unsigned bb = sb + 4u * (unsigned)(ob[0] * bx.Q + ob[1] * bx.P + ob[2]);
  const unsigned qb = (unsigned)bx.Q * 4u;
  const f32x2 r = bx.P == 32 ? gather_box_x2<32>(ba, bb, qb, w1, w2, w3) : gather_box_x2<64>(ba, bb, qb, w1, w2, w3);
  return upk2(r);
}

// Tile gather of one field at the displacements Src loads; epi(tt, a, value)
// consumes the value at the thread's point a.  sb holds kGatherBudget floats
// (16-byte aligned).  Tiles whose box does not fit gather from global memory.
// Several fields at one characteristic run as several CTAs (grid.z), each
// reducing the same box: the extra displacement reads are L2 hits.
template <class Src, class Epi>
CB_DEVICE void tile_gather(float* sb, const Src& src, const float* __restrict__ f, const Dims& d, const Epi& epi) {
  const TileThread tt = tile_thread(d);
  // the box barrier is set up first: tile_box's own barriers publish it
  __shared__ alignas(8) unsigned long long mbar;
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&mbar);
  if (threadIdx.x == 0) mbar_init(bar);
  float dd[kTilePts][3];
  src.load(dd, tt, d);
  const TileBox bx = tile_box(dd, tt, d);
  if (bx.within && bx.vol <= kGatherBudget) {
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(sb);
    // thread 0 arms the barrier while the copies start: bytes that land
    // before the arrival take its transaction count below zero, and the
    // phase cannot complete before the arrival
    if (threadIdx.x == 0) mbar_arrive_expect(bar, box_bytes(bx));
    issue_box_bulk(sbase, f, bx, d, bar);
    if (!stage_box_wait(bar, kStageWaitNs)) return;
    // two points per instruction (packed f32x2 pairs), as the table-driven gathers
#pragma unroll
    for (int a = 0; a < kTilePts; a += 2) {
      const float2 r = gather_staged_pair(sbase, dd[a], dd[a + 1], a, tt, bx);
      epi(tt, a, r.x);
      epi(tt, a + 1, r.y);
    }
  } else {
#pragma unroll
    for (int a = 0; a < kTilePts; ++a) {
      if (!tt.valid_idx(a)) continue;
      Stencil st;
      make_stencil(tt.x1(a), tt.i2, tt.i3, dd[a][0], dd[a][1], dd[a][2], d, st);
      epi(tt, a, gather(f, st));
    }
  }
}

// Tile gather of one field at a displacement field with a precomputed box
// table: the box copy is issued first and the points' displacements (and the
// epilogue's per-point operand epi.aux, when it has one) load while it is in
// flight; epi(tt, a, value, aux_a) finishes point a.  T = bf16 stages an
// image field synchronously (widened to FP32 on the way to shared memory).
template <class Epi, class T = float>
CB_DEVICE void tile_gather_tab(float* sb, const float* __restrict__ disp, const int4* __restrict__ tab,
                               const T* __restrict__ f, const Dims& d, const Epi& epi) {
  const TileBox bx = box_from_table(tab, d);
  const bool staged = bx.within && bx.vol <= kGatherBudget;
  __shared__ alignas(8) unsigned long long mbar;
  const unsigned bar = (unsigned)__cvta_generic_to_shared(&mbar);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(sb);
  if (staged) {
    if constexpr (std::is_same<T, float>::value) {
      stage_box_start(sbase, f, bx, d, bar);
    } else {
      issue_box(sb, f, bx, d);  // bf16: widened to FP32 while staged (synchronous)
    }
  }
  const TileThread tt = tile_thread(d);
  float dd[kTilePts][3], aux[kTilePts];
  const float* d2 = disp + d.n();
  const float* d3 = d2 + d.n();
#pragma unroll
  for (int a = 0; a < kTilePts; ++a) {
    const bool ok = tt.valid_idx(a);
    const unsigned i = tt.idx(a);
    dd[a][0] = ok ? __ldg(disp + i) : 0.f;
    dd[a][1] = ok ? __ldg(d2 + i) : 0.f;
    dd[a][2] = ok ? __ldg(d3 + i) : 0.f;
    aux[a] = (ok && epi.aux) ? __ldg(epi.aux + i) : 0.f;
  }
  if (staged) {
    if constexpr (std::is_same<T, float>::value) {
      if (!stage_box_wait(bar, kStageWaitNs)) return;
    } else {
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < kTilePts; a += 2) {
      const float2 r = gather_staged_pair(sbase, dd[a], dd[a + 1], a, tt, bx);
      epi(tt, a, r.x, aux[a]);
      epi(tt, a + 1, r.y, aux[a + 1]);
    }
  } else {
#pragma unroll
    for (int a = 0; a < kTilePts; ++a) {
      if (!tt.valid_idx(a)) continue;
      Stencil st;
      make_stencil(tt.x1(a), tt.i2, tt.i3, dd[a][0], dd[a][1], dd[a][2], d, st);
      epi(tt, a, gather(f, st), aux[a]);
    }
  }
}

// Displacements of the tile's points from a displacement field (3 arrays n apart).
struct DispSource {
  const float* ds;
  CB_DEVICE void load(float (&dd)[kTilePts][3], const TileThread& tt, const Dims& d) const {
    const float* d2 = ds + d.n();
    const float* d3 = d2 + d.n();
#pragma unroll
    for (int a = 0; a < kTilePts; ++a) {
      const bool ok = tt.valid(a, d);
      const unsigned i = tt.idx(a);
      dd[a][0] = ok ? __ldg(ds + i) : 0.f;
      dd[a][1] = ok ? __ldg(d2 + i) : 0.f;
      dd[a][2] = ok ? __ldg(d3 + i) : 0.f;
    }
  }
};

}  // namespace cb
