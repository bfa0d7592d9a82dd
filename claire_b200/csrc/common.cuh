// Shared device/host definitions for the claire_b200 kernels.
//
// Data layout in HBM (one registration problem): scalar fields are N1*N2*N3
// float32 arrays, row-major with x3 fastest (CLAIRE's GetLinearIndex,
// include/CLAIREUtils.hpp:198-212).  Vector fields are three consecutive
// scalar fields ([x1 | x2 | x3], src/VecField.cpp:396-478).  A batch of B
// problems of one grid size stores problem p's field at base + p*pstride.
// Spectral data is the r2c half spectrum N1 x N2 x (N3/2+1) float2, row-major.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define CB_DEVICE __device__ __forceinline__

namespace cb {

// Storage type of image volumes in the bf16-image mode (mR, mT and the state
// levels); arithmetic on them is FP32.
using bf16 = __nv_bfloat16;

// Set by a host thread while it records a CUDA graph: launchers skip
// non-stream calls (function attributes are set by an earlier uncaptured run).
inline thread_local bool g_graph_capture = false;

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 6.28318530717958647692;

struct Dims {
  int n1, n2, n3;
  __host__ __device__ long long n() const { return (long long)n1 * n2 * n3; }
  __host__ __device__ int n3h() const { return n3 / 2 + 1; }
  __host__ __device__ long long nc() const { return (long long)n1 * n2 * (n3 / 2 + 1); }
};

// Wavenumber of index i on an n-point axis with CLAIRE's convention:
// w > n/2 -> w - n, w == n/2 -> 0 (include/CLAIREUtils.hpp:248-255).
CB_DEVICE int wavenumber(int i, int n) {
  int w = i;
  if (w > n / 2) w -= n;
  else if (w == n / 2) w = 0;
  return w;
}

// Same, but the Nyquist index keeps +n/2 (inverse-Laplacian convention of
// src/CLAIREStokes.cpp:455-466 and src/Preprocessing.cpp:2013-2016).
CB_DEVICE int wavenumber_keep_nyquist(int i, int n) {
  return (i > n / 2) ? i - n : i;
}

CB_DEVICE int wrap(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

}  // namespace cb
