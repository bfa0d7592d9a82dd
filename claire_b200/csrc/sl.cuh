// Semi-Lagrangian transport: tricubic gathers and fused time-step kernels.
#pragma once

#include "common.cuh"

namespace cb {

// Field loads of the gathers: FP32 fields, or bf16 image volumes widened to
// FP32 (the tricubic sums are always FP32).
CB_DEVICE float ld_field(const float* p) { return __ldg(p); }
CB_DEVICE float ld_field(const bf16* p) { return __bfloat162float(__ldg(p)); }

// Tricubic Lagrange stencil at point i + disp (grid units), periodic.
// Reference: src/interp3.cpp:2492-2719 (base = floor(q) - 1, t = q - base in
// [1,2), w_k(t) = c_k prod_{l != k}(t - l)).  With s = t - 1 = frac(disp):
//   w0 = -s(s-1)(s-2)/6, w1 = (s+1)(s-1)(s-2)/2, w2 = -(s+1)s(s-2)/2,
//   w3 = (s+1)s(s-1)/6.
// Splitting q = i + disp into floor/frac on the displacement keeps the
// fraction exact to float precision for every grid size.
struct Stencil {
  int o1[4], o2[4], o3[4];
  float w1[4], w2[4], w3[4];
};

// The four weights at fraction s, each cubic in Horner form.
CB_DEVICE void lagrange4(float s, float (&w)[4]) {
  w[0] = s * fmaf(s, fmaf(s, -1.f / 6.f, 0.5f), -1.f / 3.f);
  w[1] = fmaf(s, fmaf(s, fmaf(s, 0.5f, -1.f), -0.5f), 1.f);
  w[2] = s * fmaf(s, fmaf(s, -0.5f, 0.5f), 1.f);
  w[3] = s * fmaf(s * s, 1.f / 6.f, -1.f / 6.f);
}

CB_DEVICE void axis_stencil(int i, float disp, int n, int stride, int (&o)[4], float (&w)[4]) {
  const float fl = floorf(disp);
  int b = wrap(i + (int)fl - 1, n);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    o[k] = b * stride;
    b = (b + 1 == n) ? 0 : b + 1;
  }
  lagrange4(disp - fl, w);
}

CB_DEVICE void make_stencil(int i1, int i2, int i3, float d1, float d2, float d3, const Dims& d,
                            Stencil& st) {
  axis_stencil(i1, d1, d.n1, d.n2 * d.n3, st.o1, st.w1);
  axis_stencil(i2, d2, d.n2, d.n3, st.o2, st.w2);
  axis_stencil(i3, d3, d.n3, 1, st.o3, st.w3);
}

// Sum over one x1 plane of the stencil (16 taps).
template <class T>
CB_DEVICE float gather_plane(const T* __restrict__ plane, const Stencil& st) {
  float acc = 0.f;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const T* row = plane + st.o2[b];
    const float r = st.w3[0] * ld_field(row + st.o3[0]) + st.w3[1] * ld_field(row + st.o3[1]) +
                    st.w3[2] * ld_field(row + st.o3[2]) + st.w3[3] * ld_field(row + st.o3[3]);
    acc += st.w2[b] * r;
  }
  return acc;
}

// 64-tap gather.  The x1 planes are visited one after another (16 loads in
// flight per thread) so the kernel stays at a register count that keeps 32+
// warps resident per SM; the plane loop selects offsets and weights with
// compile-time indices only.
template <class T>
CB_DEVICE float gather(const T* __restrict__ f, const Stencil& st) {
  float acc = st.w1[0] * gather_plane(f + st.o1[0], st);
  acc += st.w1[1] * gather_plane(f + st.o1[1], st);
  acc += st.w1[2] * gather_plane(f + st.o1[2], st);
  acc += st.w1[3] * gather_plane(f + st.o1[3], st);
  return acc;
}

CB_DEVICE void point_index(long long i, const Dims& d, int& i1, int& i2, int& i3) {
  i3 = (int)(i % d.n3);
  const long long t = i / d.n3;
  i2 = (int)(t % d.n2);
  i1 = (int)(t / d.n2);
}

// ---- host launchers ---------------------------------------------------------
// disp[p] (3 fields, each n) <- RK2 characteristic of v[p]; sign +1 state, -1 adjoint.
int launch_trajectory(const float* v, long long vp, float* disp, long long dp, int nprob,
                      const Dims& d, float ht, float sign, const int* active, cudaStream_t s);

// Box table of displacement field disp[p] for the tile gathers below:
// 2 int4 per 8x8x16 tile (tile_table_int4s(d) int4 per problem, tp apart).
// Box copies of the tile gathers that ran out of their bounded wait (count on
// the current device; read on stream s after its work), and a self-test that
// makes one wait run out.
int stage_timeouts(unsigned long long* count, cudaStream_t s = nullptr);
int launch_stage_wait_selftest(unsigned long long wait_ns, cudaStream_t s);
int launch_tile_table(const float* disp, long long dp, int4* tab, long long tp, int nprob, const Dims& d,
                      const int* active, cudaStream_t s);
long long tile_table_int4s(const Dims& d);

// out[p][f] <- f[p][f](i + disp[p](i)), f = 0..nf-1; fields ff apart; tab =
// disp's box table.
int launch_interp(const float* f, long long fp, long long ff, const float* disp, long long dp, const int4* tab,
                  long long tp, float* out, long long op, long long of, int nf, int nprob, const Dims& d,
                  const int* active, cudaStream_t s);

// Same for one bf16 image field per problem (state levels stored in bf16):
// taps widened to FP32, sums in FP32, the result rounded to bf16.
int launch_interp16(const bf16* f, long long fp, const float* disp, long long dp, const int4* tab, long long tp,
                    bf16* out, long long op, int nprob, const Dims& d, const int* active, cudaStream_t s);

// out[p] = c[p] * f[p](i + disp[p](i)): one backward RK2 step of the
// (incremental) adjoint, lambda^{l-1} = c * lambda^l(X) with the per-point
// factor c of launch_adjoint_coef (src/CLAIRE.cpp:2646-2686, 3940-3971).
int launch_gather_scale(const float* f, long long fp, const float* disp, long long dp, const int4* tab,
                        long long tp, const float* c, long long cp, float* out, long long op, int nprob,
                        const Dims& d, const int* active, cudaStream_t s);

// out[p] = sign * (f[p](i + disp[p](i)) + src[p](i)): one incremental state
// step m~^{j+1} = m~^j(X) + s_j (src/CLAIRE.cpp:3220-3276); sign -1 writes the
// incremental adjoint's final condition -m~(t=1) (src/DistanceMeasureSL2.cpp:223-283).
int launch_gather_add(const float* f, long long fp, const float* disp, long long dp, const int4* tab,
                      long long tp, const float* src, long long sp, float* out, long long op, float sign, int nprob,
                      const Dims& d, const int* active, cudaStream_t s);

// RK2 adjoint step factor: with dx = divv(X) and dv = divv,
//   lx + ht/2 (rhs0 + rhs1), rhs0 = lx dx, rhs1 = (lx + ht rhs0) dv
// equals lx * (1 + ht/2 (dx + dv + ht dx dv)); out = that factor.
// sgn -1: the factor of det(grad(inv(y))) (src/DeformationFields.cpp:686-712)
int launch_adjoint_coef(const float* divv, long long vp, const float* disp, long long dp, const int4* tab,
                        long long tp, float* out, long long op, float ht, int nprob, const Dims& d,
                        const int* active, cudaStream_t s, float sgn = 1.f);

// partials[p][0..3*np): np sums, np minima, np maxima of f[p] (n values);
// np = field_stats_parts(n)
int field_stats_parts(long long n);
int launch_field_stats(const float* f, long long fp, long long n, int nprob, double* partials, cudaStream_t s);

// Trapezoid body force over the stored adjoint levels (src/CLAIRE.cpp:2646-2709):
//   b[k] = scale * sum_l w_l lam^l (d/dx_k m^l),  w_0 = w_nt = ht/2, else ht.
// lam holds nt+1 levels (n apart), gm nt+1 levels of 3 fields (3n apart).
int launch_body_force(const float* lam, long long lp, const float* gm, long long gp, float* b, long long bp,
                      int nt, float ht, float scale, int nprob, long long n, const int* active, cudaStream_t s);

// Incremental state sources (src/CLAIRE.cpp:3220-3276), j < nt:
//   s_j = -ht/2 ((grad m^j)(X) . v~(X) + grad m^{j+1} . v~)
// gx: nt levels of 3 fields, gm: nt+1 levels of 3 fields, s: nt levels.
int launch_incstate_source(const float* gx, long long gxp, const float* vtx, long long vtxp, const float* gm,
                           long long gmp, const float* vt, long long vtp, float* src, long long sp, int nt,
                           float ht, int nprob, long long n, const int* active, cudaStream_t s);

// Second RK2 stage of the deformation-gradient transport (9-component
// tensors jX, gv(X), gv, output j; problem p at base + p * pstride).
int launch_defgrad_step(const float* jx, const float* gvx, const float* gv, float* j, long long pstride, float ht,
                        int nprob, long long n, const int* active, cudaStream_t s);

int launch_lincomb(float* y, long long yp, const float* a, long long ap, const double* ca, double sa,
                   const float* b, long long bp, const double* cb, double sb, long long len,
                   int nprob, const int* active, cudaStream_t s);

}  // namespace cb
