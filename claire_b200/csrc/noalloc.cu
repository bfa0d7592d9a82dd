// claire_b200_reg_apply_noalloc: the regularisation operator seam without any
// device allocation.
//
// Some callers cannot allocate device memory while they run this operator: a
// host that has already handed the whole GPU memory budget to its own pool,
// or code driving the preconditioner from a context where an allocation
// would synchronise the device or could fail midway (a real-time loop, an
// allocator-free embedding).  For them the FFT workspace of the operator (a
// three-field half spectrum), its parameter block and the twiddle tables
// live in fixed device arrays inside this library instead of coming from
// cudaMalloc / cudaMallocAsync.
//
// Limits and behaviour:
// * grids up to 64^3 (cubic N in {16, 32, 48, 64}); larger grids are rejected
//   with CB_ERR_TOO_LARGE before anything is launched.  The arrays take
//   3.3 MB of device memory on every GPU that loads the library, until the
//   process exits.
// * every call shares the arrays: calls that may overlap on the GPU (different
//   streams, other host threads) race and must be serialised by the caller.
//   The spectrum is fully rewritten by each call, so nothing has to start at
//   zero; the parameter block is rewritten by each call (a one-thread kernel
//   stores the block it receives as a launch argument, in stream order).
// * v and out must be 16-byte aligned (CB_ERR_ARG otherwise, before anything
//   is launched).
// * the first call on a device sets that device up (looks up the arrays'
//   device addresses with that device current and uploads the twiddle
//   tables); make that first call before any stream capture.
#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/claire_b200.h"
#include "reduce.cuh"
#include "sl.cuh"
#include "spectral.cuh"

namespace cb {
void note_launches(int k);
}

namespace {

constexpr int kMaxN = 64;
constexpr long long kSpecEntries = 3LL * kMaxN * kMaxN * (kMaxN / 2 + 1);
constexpr int kTwOffset16 = 0, kTwOffset32 = 16, kTwOffset48 = 48, kTwOffset64 = 96, kTwEntries = 160;

static __device__ __align__(256) float2 g_spec[kSpecEntries];
static __device__ __align__(256) cb::SpecParams g_params;
static __device__ __align__(256) float2 g_twiddles[kTwEntries];

// Writes the call's parameter block: the block travels as a kernel argument,
// so no host buffer has to outlive the call.
__global__ void k_set_params(cb::SpecParams p) { g_params = p; }

struct DeviceArrays {
  bool ready = false;
  float2* spec = nullptr;
  cb::SpecParams* params = nullptr;
  float2* tw = nullptr;
};

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
DeviceArrays g_dev[kMaxDevices];

// Called with `dev` current: resolve the arrays' device addresses and upload
// the twiddle tables W_N^m = exp(-2 pi i m / N) (computed in double).
int setup(int dev, DeviceArrays& out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceArrays& a = g_dev[dev];
  if (!a.ready) {
    if (cudaGetSymbolAddress((void**)&a.spec, g_spec) != cudaSuccess) return CB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&a.params, g_params) != cudaSuccess) return CB_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&a.tw, g_twiddles) != cudaSuccess) return CB_ERR_CUDA;
    float2 h[kTwEntries];
    const int sizes[4] = {16, 32, 48, 64};
    const int offs[4] = {kTwOffset16, kTwOffset32, kTwOffset48, kTwOffset64};
    for (int k = 0; k < 4; ++k)
      for (int m = 0; m < sizes[k]; ++m) {
        const double ang = cb::kTwoPi * (double)m / (double)sizes[k];
        h[offs[k] + m] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
      }
    if (cudaMemcpy(a.tw, h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) return CB_ERR_CUDA;
    a.ready = true;
  }
  out = a;
  return CB_OK;
}

int twiddle_offset(int n) {
  switch (n) {
    case 16: return kTwOffset16;
    case 32: return kTwOffset32;
    case 48: return kTwOffset48;
    case 64: return kTwOffset64;
    default: return -1;
  }
}

}  // namespace

extern "C" int claire_b200_reg_apply_noalloc(const float* v, float* out, const int nx[3], int regnorm,
                                             const double beta[2], int kind, void* stream) {
  if (!v || !out || !nx || !beta || regnorm < CB_NORM_L2 || regnorm > CB_NORM_H3SN ||
      kind < CB_REG_GRADIENT || kind > CB_REG_SQRTINVERSE)
    return CB_ERR_ARG;
  if (nx[0] <= 0 || nx[1] <= 0 || nx[2] <= 0) return CB_ERR_ARG;
  // the transform kernels read and write 16-byte vectors
  if ((reinterpret_cast<uintptr_t>(v) & 15) || (reinterpret_cast<uintptr_t>(out) & 15)) return CB_ERR_ARG;
  if (!(nx[0] == nx[1] && nx[1] == nx[2])) return CB_ERR_UNSUPPORTED;
  if (nx[0] > kMaxN) return CB_ERR_TOO_LARGE;
  const int toff = twiddle_offset(nx[0]);
  if (toff < 0) return CB_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CB_ERR_CUDA;
  DeviceArrays a;
  int e = setup(dev, a);
  if (e) return e;
  cb::Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t st = (cudaStream_t)stream;
  if (regnorm == CB_NORM_L2 || beta[0] == 0.0) {
    // src/RegularizationL2.cpp: beta*v and v/beta in real space (no workspace)
    double c = 1.0;
    if (beta[0] != 0.0)
      c = (kind == CB_REG_GRADIENT) ? beta[0] : (kind == CB_REG_INVERSE ? 1.0 / beta[0] : 1.0 / std::sqrt(beta[0]));
    else if (kind == CB_REG_GRADIENT)
      c = 0.0;
    cb::note_launches(1);
    e = cb::launch_lincomb(out, 0, v, 0, nullptr, c, nullptr, 0, nullptr, 0.0, 3 * d.n(), 1, nullptr, st);
    return e ? CB_ERR_CUDA : CB_OK;
  }
  cb::SpecParams p{};
  p.norm = regnorm;
  p.beta0 = (float)beta[0];
  p.beta1 = (float)beta[1];
  p.beta2 = 0.f;
  p.hd = (float)((cb::kTwoPi / d.n1) * (cb::kTwoPi / d.n2) * (cb::kTwoPi / d.n3));
  p.sigma[0] = p.sigma[1] = p.sigma[2] = 1.f;
  k_set_params<<<1, 1, 0, st>>>(p);
  if (cudaGetLastError() != cudaSuccess) return CB_ERR_CUDA;
  const int op = kind == CB_REG_GRADIENT ? cb::OP_REG_GRAD
                                         : (kind == CB_REG_INVERSE ? cb::OP_REG_INV : cb::OP_REG_SQRTINV);
  cb::note_launches(6);
  e = cb::launch_spectral3_explicit(v, out, a.spec, a.params, d, op, a.tw + toff, st);
  return e ? CB_ERR_CUDA : CB_OK;
}
