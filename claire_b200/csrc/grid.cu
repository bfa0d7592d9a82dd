// Spectral grid change between cubic grids: restriction (fine -> coarse) and
// prolongation (coarse -> fine) of scalar and vector fields.
//
// Reference: Preprocessing::Restrict / Prolong (src/Preprocessing.cpp:733-917,
// 1605-1786) with the index map of ComputeGridChangeIndices (:918-1057): the
// coefficients of wavenumbers |w| < Nc/2 on every axis (the coarse grid's
// Nyquist index excluded) are carried over, scaled by the source grid's FFT
// scale 1/Ns^3, and transformed back unnormalised on the target grid; all
// other target coefficients are zero.
//
// That map is a tensor product of one 1D map per axis, so it is applied here
// as three axis passes, each a small dense real matrix (target length x source
// length) built on the host in FP64:
//   T[j][i] = (1/Ns) (1 + 2 sum_{w=1}^{Nc/2-1} cos(2 pi w (j/Nt - i/Ns))),
// Nc = min(Ns, Nt).  A grid change happens once per continuation level, so
// the passes favour simplicity: one thread per output value, the line read
// through the cache.
#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"

namespace cb {

namespace {

std::mutex g_mat_mutex;
std::map<std::pair<long long, long long>, float*> g_mats;  // (device, ns*1024+nt) -> T

const float* transfer_matrix(int ns, int nt) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair((long long)dev, (long long)ns * 1024 + nt);
  std::lock_guard<std::mutex> lock(g_mat_mutex);
  auto it = g_mats.find(key);
  if (it != g_mats.end()) return it->second;
  const int nc = ns < nt ? ns : nt;
  std::vector<float> h((size_t)nt * ns);
  for (int j = 0; j < nt; ++j)
    for (int i = 0; i < ns; ++i) {
      const double u = (double)j / nt - (double)i / ns;
      double acc = 1.0;
      for (int w = 1; w < (nc + 1) / 2; ++w) acc += 2.0 * std::cos(kTwoPi * w * u);
      h[(size_t)j * ns + i] = (float)(acc / ns);
    }
  float* d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(float)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  g_mats[key] = d;
  return d;
}

// out (dims o) = T applied along `axis` of in (dims i; i and o differ only
// along axis).  Fields: blockIdx.y; in / out fields ip / op apart.
__global__ void k_transfer_axis(const float* __restrict__ in, long long ip, Dims di, float* __restrict__ out,
                                long long op, Dims dout, int axis, const float* __restrict__ T) {
  const long long no = dout.n();
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= no) return;
  const float* src = in + blockIdx.y * ip;
  const int o3 = (int)(idx % dout.n3);
  const long long r = idx / dout.n3;
  const int o2 = (int)(r % dout.n2), o1 = (int)(r / dout.n2);
  int j, ns;
  long long base, stride;
  if (axis == 2) {
    j = o3;
    ns = di.n3;
    base = ((long long)o1 * di.n2 + o2) * di.n3;
    stride = 1;
  } else if (axis == 1) {
    j = o2;
    ns = di.n2;
    base = (long long)o1 * di.n2 * di.n3 + o3;
    stride = di.n3;
  } else {
    j = o1;
    ns = di.n1;
    base = (long long)o2 * di.n3 + o3;
    stride = (long long)di.n2 * di.n3;
  }
  const float* t = T + (long long)j * ns;
  float acc = 0.f;
  for (int i = 0; i < ns; ++i) acc = fmaf(__ldg(t + i), __ldg(src + base + i * stride), acc);
  out[blockIdx.y * op + idx] = acc;
}

int transfer_pass(const float* in, long long ip, const Dims& di, float* out, long long op, const Dims& dout, int axis,
                  int nf, cudaStream_t s) {
  const int ns = axis == 0 ? di.n1 : (axis == 1 ? di.n2 : di.n3);
  const int nt = axis == 0 ? dout.n1 : (axis == 1 ? dout.n2 : dout.n3);
  const float* T = transfer_matrix(ns, nt);
  if (!T) return (int)cudaErrorMemoryAllocation;
  const long long no = dout.n();
  k_transfer_axis<<<dim3((unsigned)((no + 255) / 256), nf), 256, 0, s>>>(in, ip, di, out, op, dout, axis, T);
  return (int)cudaGetLastError();
}

}  // namespace

// Grid change of nf fields (in: ns^3 each, ip apart; out: nt^3 each, op apart).
// work holds 2 * nf * max(ns, nt)^2 * min(ns, nt)... floats: see grid_change_work.
long long grid_change_work(int ns, int nt, int nf) {
  const long long a = (long long)ns * ns * nt, b = (long long)ns * nt * nt;
  return (long long)nf * (a + b);
}

int launch_grid_change(const float* in, long long ip, int ns, float* out, long long op, int nt, int nf, float* work,
                       cudaStream_t s) {
  if (ns == nt) {
    for (int f = 0; f < nf; ++f)
      if (cudaMemcpyAsync(out + f * op, in + f * ip, sizeof(float) * (size_t)ns * ns * ns, cudaMemcpyDeviceToDevice,
                          s) != cudaSuccess)
        return (int)cudaErrorUnknown;
    return 0;
  }
  const Dims d0{ns, ns, ns}, d1{ns, ns, nt}, d2{ns, nt, nt}, d3{nt, nt, nt};
  float* w1 = work;                       // nf fields of d1
  float* w2 = work + (long long)nf * d1.n();  // nf fields of d2
  int e = transfer_pass(in, ip, d0, w1, d1.n(), d1, 2, nf, s);
  if (!e) e = transfer_pass(w1, d1.n(), d1, w2, d2.n(), d2, 1, nf, s);
  if (!e) e = transfer_pass(w2, d2.n(), d2, out, op, d3, 0, nf, s);
  return e;
}

}  // namespace cb
