// Spectral operator parameters and the host-side launch interface of the FFT
// kernels.
#pragma once

#include "common.cuh"

namespace cb {

// Regularisation norms, numbered like CLAIRE's -regnorm choices.
enum RegNorm : int { NORM_L2 = 0, NORM_H1 = 1, NORM_H1SN = 2, NORM_H2 = 3, NORM_H2SN = 4,
                     NORM_H3 = 5, NORM_H3SN = 6 };

// Operators applied in the x1 pencil pass between the forward and the
// inverse transform.
enum SpecOp : int {
  OP_REG_GRAD = 0,   // EvaluateGradient / HessianMatVec symbol, 3 -> 3
  OP_REG_INV = 1,    // ApplyInverse symbol, 3 -> 3
  OP_REG_SQRTINV = 2,// ApplyInverse with applysqrt, 3 -> 3
  OP_REG_FUNC = 3,   // symbol whose squared output norm is the functional, 3 -> 3
  OP_LERAY = 4,      // Stokes projection addend, 3 -> 3
  OP_LERAY_RELAXED = 5, // relaxed-Stokes projection addend, 3 -> 3
  OP_GAUSS = 6,      // Gaussian smoothing, 1 -> 1
  OP_IDENTITY = 7,   // scale by 1/N^3 only (round-trip test), 1 -> 1
};

// Per-problem parameters read by the pencil kernel.
struct SpecParams {
  int norm;
  float beta0, beta1, beta2;  // regularisation weights (beta2: relaxed Stokes)
  float hd;                   // Lebesgue measure
  float sigma[3];             // Gaussian width in grid cells
};

// Epilogue of the inverse row pass.
// Epilogues of the inverse transforms: store, accumulate, sum of squares, or
// store / accumulate and sum out * other (FP64 partials, c2r only).
enum Epi : int { EPI_STORE = 0, EPI_ADD = 1, EPI_SUMSQ = 2, EPI_STORE_DOT = 3, EPI_ADD_DOT = 4 };

struct Batch {
  int nprob;              // problems in the launch
  long long pstride;      // elements between problems' fields
};

// ---- host launchers (return cudaError_t as int) ---------------------------
// All take an optional per-problem `active` mask (null: all problems).
// Forward r2c of nf real fields: in[p*ip + f*ifs] -> spec[p*sp + f*nc].
int launch_r2c3d(const float* in, long long ip, long long ifs, float2* spec, long long sp, int nf,
                 int nprob, const Dims& d, const int* active, cudaStream_t s);
// Apply op in the x1 pass (in place on spec, nin fields in, nout out).
int launch_pencil(float2* spec, long long sp, int nprob, const Dims& d, int op,
                  const SpecParams* dparams, int nin, int nout, const int* active, cudaStream_t s);
// Inverse c2r of nf fields with epilogue: out[p*op + f*ofs] = alpha[p]*x (+ out) or sumsq.
int launch_c2r3d(float2* spec, long long sp, float* out, long long op_, long long ofs, int nf,
                 int nprob, const Dims& d, int epi, const float* alpha, double* partials, int nparts,
                 const int* active, cudaStream_t s, const float* other = nullptr);

// Spectral first derivative along one axis (0:x1, 1:x2, 2:x3) of nf real
// fields with Nyquist set to zero; out = d/dx_axis in (+ out) or sumsq.
int launch_deriv(const float* in, long long ip, long long ifs, float* out, long long op_,
                 long long ofs, int nf, int nprob, const Dims& d, int axis, int epi,
                 double* partials, int nparts, const int* active, cudaStream_t s);

// Number of reduction partials a launch with these arguments writes per problem
// (any_variant: the largest count over the size's FFT variants, for sizing).
int deriv_partials(const Dims& d, int axis, int nf, bool any_variant = false);
int c2r_partials(const Dims& d, int nf, bool any_variant = false);

// FFT variant of an N-point axis: bit 0 the alternative two-stage radix plan,
// bit 1 the alternative lines per CTA.  Process-wide, default 0; change it
// only while no transform of that size is in flight.
int fft_variant(int n);
int set_fft_variant(int n, int v);
// candidate variants of size n into out[0..3]; returns their count (0: unsupported)
int fft_variant_candidates(int n, int* out);
// Time every candidate on a batch of nprob problems (a 3-field regularisation
// operator and a 3-field gradient per problem) and keep the fastest.  ms[i]
// receives the time of candidate i (ms may be null).  Allocates its own
// buffers; synchronises the stream.
int fft_autotune(int n, int nprob, cudaStream_t s, int* best, float* ms);
// whether size n was tuned in this process; tune it once (serialised)
bool fft_tuned(int n);
int fft_autotune_once(int n, int nprob, cudaStream_t s);

bool fft_size_supported(int n);      // every axis (rows need N % 16 == 0)
bool fft_col_size_supported(int n);  // axes x1 and x2 (column / pencil passes): also 150

// Spectral grid change (restriction / prolongation) of nf cubic fields, ns^3
// (ip apart) -> nt^3 (op apart); work: grid_change_work(ns, nt, nf) floats.
long long grid_change_work(int ns, int nt, int nf);
int launch_grid_change(const float* in, long long ip, int ns, float* out, long long op, int nt, int nf, float* work,
                       cudaStream_t s);

// 3-field op (forward r2c, op in the x1 pass, inverse c2r stored to out) using
// a caller-provided spectrum workspace (3 * nc float2) and twiddle table
// (W_N^m, m < N); allocates nothing.
int launch_spectral3_explicit(const float* in, float* out, float2* spec, const SpecParams* params, const Dims& d,
                              int op, const float2* tw, cudaStream_t s);

}  // namespace cb
