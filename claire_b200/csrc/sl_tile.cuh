// Shared-memory tiled tricubic gathers with a double-buffered pipeline.
//
// A tile is TX1 x TX2 x TX3 output points (x3 fastest; each warp covers 32
// consecutive x3 points of one (x1, x2) row and each thread TX1 points along
// x1).  For a tile the CTA reads the points' displacements, reduces the
// bounding box of every stencil tap (min/max over the tile of i + floor(d),
// widened by the stencil's -1 .. +2) and, when the box fits the budget, copies
// it into shared memory with 16-byte cp.async (periodic wrap applied while
// copying).  The 64 taps per point are then served from shared memory; tiles
// whose box is too large (large, rough displacements) gather from global
// memory instead.
//
// CTAs are persistent: CTA b walks tiles b, b + gridDim.x, ...  While it
// gathers (tile, field) item i from one buffer, the copy of item i+1 is in
// flight into the other, so copy latency overlaps the gathers.
//
// The box's x3 row pitch is a multiple of 32 floats, so warps whose points
// straddle box rows still hit 32 distinct banks.  Every shared-memory index is
// inside the box by construction: each point's taps lie in [i + floor(d) - 1,
// i + floor(d) + 2] and the box spans the min / max of exactly those values
// over the tile's points; points outside the grid (partial tiles) are moved to
// the box origin and never stored.
#pragma once

#include <climits>

#include "sl.cuh"

namespace cb {

constexpr int kTX1 = 4, kTX2 = 8, kTX3 = 32;
constexpr int kTileThreads = kTX2 * kTX3;  // 256
constexpr int kBoxBudget = 12224;           // floats per buffer
constexpr int kPersistCtasPerSm = 2;        // two 48 KB double buffers per SM pair
constexpr int kGatherSmemBytes = 2 * kBoxBudget * 4;

// Per point: unwrapped tap base floor(i + disp) - 1 and the fraction of disp.
struct TilePoint {
  int b[3];
  float s[3];
};

// The thread's points in a tile are (t1 + a, i2, i3) for a < kTX1.
struct TileRow {
  int t1, i2, i3;
  bool row_ok;
  long long idx0, step;
  CB_DEVICE bool valid(int a, const Dims& d) const { return row_ok && (t1 + a < d.n1); }
  CB_DEVICE long long idx(int a) const { return idx0 + a * step; }
};

struct TileBox {
  int lo[3];
  int ext[3];   // extents of the tap box (x3 rounded to whole 16-byte chunks)
  int pitch;    // x3 row pitch in shared memory (multiple of 32)
  bool fits;
};

CB_DEVICE TileRow tile_row(const Dims& d, int tile) {
  const int nb3 = (d.n3 + kTX3 - 1) / kTX3;
  const int nb2 = (d.n2 + kTX2 - 1) / kTX2;
  const int c3 = tile % nb3;
  const int r = tile / nb3;
  const int c2 = r % nb2;
  const int c1 = r / nb2;
  TileRow row;
  row.t1 = c1 * kTX1;
  row.i2 = c2 * kTX2 + (threadIdx.x >> 5);
  row.i3 = c3 * kTX3 + (threadIdx.x & 31);
  row.row_ok = (row.i2 < d.n2) && (row.i3 < d.n3);
  row.step = (long long)d.n2 * d.n3;
  row.idx0 = (long long)row.t1 * row.step + (long long)row.i2 * d.n3 + row.i3;
  return row;
}

__host__ __device__ inline unsigned tile_count(const Dims& d) {
  return (unsigned)(((d.n1 + kTX1 - 1) / kTX1) * ((d.n2 + kTX2 - 1) / kTX2) * ((d.n3 + kTX3 - 1) / kTX3));
}

CB_DEVICE void set_point(TilePoint& pt, int i1, int i2, int i3, float d1, float d2, float d3) {
  const float f1 = floorf(d1), f2 = floorf(d2), f3 = floorf(d3);
  pt.s[0] = d1 - f1;
  pt.s[1] = d2 - f2;
  pt.s[2] = d3 - f3;
  pt.b[0] = i1 + (int)f1 - 1;
  pt.b[1] = i2 + (int)f2 - 1;
  pt.b[2] = i3 + (int)f3 - 1;
}

// Block-wide bounding box of the taps of the tile's valid points; invalid
// points are moved to the box origin so every later read stays in the box.
// Contains __syncthreads: call from uniform control flow.
CB_DEVICE TileBox tile_box(TilePoint (&pts)[kTX1], const TileRow& row, const Dims& d) {
  __shared__ int red[6][kTileThreads / 32];
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (!row.valid(a, d)) continue;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      mn[k] = min(mn[k], pts[a].b[k]);
      mx[k] = max(mx[k], pts[a].b[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    mn[k] = __reduce_min_sync(0xffffffffu, mn[k]);
    mx[k] = __reduce_max_sync(0xffffffffu, mx[k]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // the previous tile's readers of red[] are done
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      red[k][warp] = mn[k];
      red[3 + k][warp] = mx[k];
    }
  }
  __syncthreads();
  TileBox box;
  bool within = true, sane = true;
  const int nk[3] = {d.n1, d.n2, d.n3};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
    for (int w = 0; w < kTileThreads / 32; ++w) {
      lo = min(lo, red[k][w]);
      hi = max(hi, red[3 + k][w]);
    }
    box.lo[k] = lo;
    const long long ext = (long long)hi - (long long)lo + 4;  // taps b .. b+3
    sane = sane && ext > 0 && ext <= 4096;
    box.ext[k] = (ext > 0 && ext <= 4096) ? (int)ext : 4096;
    within = within && ext <= nk[k];  // one wrap per coordinate in the copy
  }
  // x3: start on a multiple of 4 floats and cover whole 4-float chunks so the
  // box is copied in 16-byte pieces (N3 % 4 == 0: no chunk straddles the seam)
  const int lo3a = box.lo[2] & ~3;
  box.ext[2] = ((box.lo[2] + box.ext[2] - lo3a) + 3) & ~3;
  box.lo[2] = lo3a;
  within = within && box.ext[2] <= d.n3 && box.ext[2] <= 128 && (d.n3 & 3) == 0;
  box.pitch = (box.ext[2] + 31) & ~31;
  const long long vol = (long long)box.ext[0] * box.ext[1] * box.pitch;
  box.fits = sane && within && vol <= kBoxBudget;
#pragma unroll
  for (int a = 0; a < kTX1; ++a) {
    if (row.valid(a, d)) continue;
    pts[a].b[0] = box.lo[0];
    pts[a].b[1] = box.lo[1];
    pts[a].b[2] = box.lo[2];
    pts[a].s[0] = pts[a].s[1] = pts[a].s[2] = 0.f;
  }
  return box;
}

CB_DEVICE void cp_async16(float* smem_dst, const float* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
CB_DEVICE void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPENDING>
CB_DEVICE void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPENDING) : "memory"); }

// Issue the 16-byte asynchronous copies of field f's box (periodic wrap on
// load) into sb.  Lanes cover the chunks of one or more x3 rows (coalesced).
// The box never exceeds the grid along an axis (tile_box), so one
// conditional subtraction wraps each coordinate.  Caller commits the group.
CB_DEVICE void issue_box(float* __restrict__ sb, const float* __restrict__ f, const TileBox& box, const Dims& d) {
  const int e1 = box.ext[0], e2 = box.ext[1], pitch = box.pitch;
  const int nck = box.ext[2] >> 2;  // 16-byte chunks per row (<= 32)
  const int rpi = 32 / nck;         // rows a warp copies per step
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int lr = lane / nck, lc = lane - lr * nck;
  if (lr >= rpi) return;
  const int w1 = wrap(box.lo[0], d.n1), w2 = wrap(box.lo[1], d.n2), w3 = wrap(box.lo[2], d.n3);
  int g3 = w3 + 4 * lc;
  g3 -= (g3 >= d.n3) ? d.n3 : 0;
  const int step = rpi * nw;  // rows between this lane's copies
  const int r0 = warp * rpi + lr;
  int l1 = r0 / e2, l2 = r0 - l1 * e2;
  while (l1 < e1) {
    int g1 = w1 + l1, g2 = w2 + l2;
    g1 -= (g1 >= d.n1) ? d.n1 : 0;
    g2 -= (g2 >= d.n2) ? d.n2 : 0;
    cp_async16(sb + (l1 * e2 + l2) * pitch + 4 * lc, f + ((long long)g1 * d.n2 + g2) * d.n3 + g3);
    l2 += step;
    while (l2 >= e2) {
      l2 -= e2;
      ++l1;
    }
  }
}

CB_DEVICE void lagrange4(float s, float (&w)[4]) {
  const float sm1 = s - 1.f, sm2 = s - 2.f, sp1 = s + 1.f;
  w[0] = (-1.f / 6.f) * s * sm1 * sm2;
  w[1] = 0.5f * sp1 * sm1 * sm2;
  w[2] = -0.5f * sp1 * s * sm2;
  w[3] = (1.f / 6.f) * sp1 * s * sm1;
}

// Four consecutive floats from shared memory (immediate offsets, any alignment).
CB_DEVICE float dot4_shared(unsigned addr, const float (&w)[4]) {
  float x0, x1, x2, x3;
  asm volatile(
      "ld.shared.f32 %0, [%4];\n\t"
      "ld.shared.f32 %1, [%4+4];\n\t"
      "ld.shared.f32 %2, [%4+8];\n\t"
      "ld.shared.f32 %3, [%4+12];\n"
      : "=f"(x0), "=f"(x1), "=f"(x2), "=f"(x3)
      : "r"(addr));
  return w[0] * x0 + w[1] * x1 + w[2] * x2 + w[3] * x3;
}

// 64-tap gather from a staged box (32-bit shared addresses).
CB_DEVICE float gather_box(unsigned sbase, const TileBox& box, const TilePoint& pt) {
  float w1[4], w2[4], w3[4];
  lagrange4(pt.s[0], w1);
  lagrange4(pt.s[1], w2);
  lagrange4(pt.s[2], w3);
  const unsigned rowb = (unsigned)box.pitch * 4u;
  const unsigned planeb = rowb * (unsigned)box.ext[1];
  const unsigned base = sbase + (unsigned)((pt.b[0] - box.lo[0]) * box.ext[1] * box.pitch +
                                           (pt.b[1] - box.lo[1]) * box.pitch + (pt.b[2] - box.lo[2])) * 4u;
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    float acc_a = 0.f;
#pragma unroll
    for (int b = 0; b < 4; ++b) acc_a += w2[b] * dot4_shared(base + a * planeb + b * rowb, w3);
    acc += w1[a] * acc_a;
  }
  return acc;
}

// 64-tap gather straight from global memory (tiles whose box is too large).
CB_DEVICE float gather_point_global(const float* __restrict__ f, const TilePoint& pt, const Dims& d) {
  Stencil st;
  int c1 = wrap(pt.b[0], d.n1), c2 = wrap(pt.b[1], d.n2), c3 = wrap(pt.b[2], d.n3);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    st.o1[k] = c1 * d.n2 * d.n3;
    st.o2[k] = c2 * d.n3;
    st.o3[k] = c3;
    c1 = (c1 + 1 == d.n1) ? 0 : c1 + 1;
    c2 = (c2 + 1 == d.n2) ? 0 : c2 + 1;
    c3 = (c3 + 1 == d.n3) ? 0 : c3 + 1;
  }
  lagrange4(pt.s[0], st.w1);
  lagrange4(pt.s[1], st.w2);
  lagrange4(pt.s[2], st.w3);
  return gather(f, st);
}

// Points of a tile from a displacement field (3 arrays n apart).
struct DispSource {
  const float* ds;
  CB_DEVICE void points(TilePoint (&pts)[kTX1], const TileRow& row, const Dims& d) const {
    const long long n = d.n();
#pragma unroll
    for (int a = 0; a < kTX1; ++a) {
      if (!row.valid(a, d)) {
        pts[a] = TilePoint{{0, 0, 0}, {0.f, 0.f, 0.f}};
        continue;
      }
      const long long i = row.idx(a);
      set_point(pts[a], row.t1 + a, row.i2, row.i3, __ldg(ds + i), __ldg(ds + n + i), __ldg(ds + 2 * n + i));
    }
  }
};

// Persistent double-buffered gather of NF fields (ff apart) over all tiles of
// one grid; epi(row, vals) finishes a tile once its NF fields are gathered.
// sbuf holds 2 * kBoxBudget floats (16-byte aligned).
template <int NF, class Src, class Epi>
CB_DEVICE void pipelined_gather(float* sbuf, const Src& src, const float* __restrict__ f, long long ff,
                                const Dims& d, Epi& epi) {
  const int ntiles = (int)tile_count(d);
  int t = blockIdx.x;
  if (t >= ntiles) return;
  const unsigned sb0 = (unsigned)__cvta_generic_to_shared(sbuf);
  TileRow row = tile_row(d, t);
  TilePoint pts[kTX1];
  src.points(pts, row, d);
  TileBox box = tile_box(pts, row, d);
  int k = 0, buf = 0;
  if (box.fits) {
    issue_box(sbuf, f, box, d);
    cp_async_commit();
  }
  float vals[NF][kTX1];
  while (true) {
    // the next item: next field of this tile, or field 0 of the next tile
    int tn = t, kn = k + 1;
    if (kn == NF) {
      tn = t + gridDim.x;
      kn = 0;
    }
    const bool has_next = tn < ntiles;
    TileRow rown = row;
    TileBox boxn = box;
    if (has_next && tn != t) {
      rown = tile_row(d, tn);
      TilePoint ptsn[kTX1];
      src.points(ptsn, rown, d);
      boxn = tile_box(ptsn, rown, d);
    }
    const bool issued = has_next && boxn.fits;
    if (issued) {
      issue_box(sbuf + (buf ^ 1) * kBoxBudget, f + kn * ff, boxn, d);
      cp_async_commit();
    }
    float cur[kTX1];
    if (box.fits) {
      if (issued) cp_async_wait<1>();
      else cp_async_wait<0>();
      __syncthreads();
      const unsigned sb = sb0 + (unsigned)(buf * kBoxBudget * 4);
#pragma unroll
      for (int a = 0; a < kTX1; ++a) cur[a] = gather_box(sb, box, pts[a]);
    } else {
#pragma unroll
      for (int a = 0; a < kTX1; ++a) cur[a] = row.valid(a, d) ? gather_point_global(f + k * ff, pts[a], d) : 0.f;
    }
    // compile-time indices only (no local-memory array)
#pragma unroll
    for (int kk = 0; kk < NF; ++kk)
      if (kk == k) {
#pragma unroll
        for (int a = 0; a < kTX1; ++a) vals[kk][a] = cur[a];
      }
    if (k == NF - 1) epi(row, vals);
    __syncthreads();  // every thread is done with this buffer before it is refilled
    if (!has_next) break;
    if (tn != t) {
      t = tn;
      row = rown;
      src.points(pts, row, d);
      // re-derive the moved-to-origin invalid points for this box
#pragma unroll
      for (int a = 0; a < kTX1; ++a)
        if (!row.valid(a, d)) {
          pts[a].b[0] = boxn.lo[0];
          pts[a].b[1] = boxn.lo[1];
          pts[a].b[2] = boxn.lo[2];
        }
      box = boxn;
    }
    k = kn;
    buf ^= 1;
  }
}

}  // namespace cb
