// Gauss-Newton-Krylov driver (host C++) for a batch of registration problems.
//
// Restates, for one GPU, the control flow of the reference's
// CLAIREInterface::RunSolver -> Optimizer::Run -> TAO nls (PETSc 3.9.1) with
// KSPCG + PCSHELL (INVREG) + Armijo (src/CLAIREInterface.cpp:771-885,
// src/Optimizer.cpp:235-530, src/TaoInterface.cpp:40-606,
// src/KrylovInterface.cpp:79-196), and the problem class CLAIRE's objective /
// gradient / GN Hessian matvec (src/CLAIRE.cpp:227-357, 793-1042,
// 1218-1379).  Scalars that steer the PCG (alpha, beta, residual checks) are
// computed on the device; the host reads one flag vector per PCG iteration.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "reduce.cuh"
#include "sl.cuh"
#include "solver.cuh"

namespace cb {

#define CB_TRY(x)                      \
  do {                                 \
    int _e = (x);                      \
    if (_e) return _e;                 \
  } while (0)

// ---------------------------------------------------------------------------
// small scalar kernels (one thread per problem)
// ---------------------------------------------------------------------------
// rn0 = sqrt(rr); tol = max(rtol*rn0, atol); stop when rn0 <= tol
__global__ void k_pcg_init(double* __restrict__ sc, int* __restrict__ isc, int* __restrict__ act, int B,
                           double atol) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B || !act[p]) return;
  double* RR = sc + Solver::S_RR * B;
  double* RN0 = sc + Solver::S_RN0 * B;
  double* TOL = sc + Solver::S_TOL * B;
  double* RTOL = sc + Solver::S_RTOL * B;
  const double rn0 = sqrt(RR[p]);
  RN0[p] = rn0;
  TOL[p] = fmax(RTOL[p] * rn0, atol);
  isc[Solver::I_IT * B + p] = 0;
  isc[Solver::I_REASON * B + p] = 0;
  if (rn0 <= TOL[p]) {
    act[p] = 0;
    isc[Solver::I_REASON * B + p] = 1;  // converged
  }
}

// NCC distance scalars (src/DistanceMeasureNCC.cpp), FP64, one thread per problem.
// which 0: scale = (1/2 hd |mT - mR|^2) / (1/2 - 1/2 I^2/(A R))     (:78-166)
// which 1: D = scale (1/2 - 1/2 I^2/(A R))                         (:171-245)
// which 2: lambda(1) = CA mR + CB m1, CA = s I/(hd A R), CB = -s I^2/(hd A^2 R)   (:251-366)
// which 3: lambda~(1) = CA mR + CB m1 + CC m~ with the linearised coefficients    (:368-510)
// A = <x,x> (x = mT for the scale, else m1), R = <mR,mR>, I = <x,mR>.
__global__ void k_ncc(double* __restrict__ sc, const int* __restrict__ act, int B, int which, double hd) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B || (act && !act[p])) return;
  const double A = sc[Solver::S_NA * B + p], R = sc[Solver::S_NRR * B + p], I = sc[Solver::S_NI * B + p];
  const double s = sc[Solver::S_NS * B + p];
  if (which == 0) {
    sc[Solver::S_NS * B + p] = (0.5 * hd * sc[Solver::S_NL2 * B + p]) / (0.5 - 0.5 * I * I / (A * R));
  } else if (which == 1) {
    sc[Solver::S_D * B + p] = s * (0.5 - 0.5 * I * I / (A * R));
  } else if (which == 2) {
    sc[Solver::S_CA * B + p] = s * I / (hd * A * R);
    sc[Solver::S_CB * B + p] = -s * I * I / (hd * A * A * R);
  } else {
    const double IM = sc[Solver::S_NIM * B + p], RM = sc[Solver::S_NRM * B + p];
    const double c1 = s * RM / (hd * A * R);
    const double c2 = 2.0 * s * I * IM / (hd * A * A * R);
    const double c3 = 4.0 * s * I * I * IM / (hd * A * A * A * R);
    const double c4 = 2.0 * s * I * RM / (hd * A * A * R);
    const double c5 = s * I * I / (hd * A * A * R);
    sc[Solver::S_CA * B + p] = c1 - c2;
    sc[Solver::S_CB * B + p] = c3 - c4;
    sc[Solver::S_CC * B + p] = -c5;
  }
}

// alpha = rz / pq, stop on non-positive curvature
__global__ void k_pcg_alpha(double* __restrict__ sc, int* __restrict__ isc, int* __restrict__ act, int B) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B || !act[p]) return;
  const double pq = sc[Solver::S_PQ * B + p];
  if (!(pq > 0.0) || !isfinite(pq)) {
    act[p] = 0;
    sc[Solver::S_ALPHA * B + p] = 0.0;
    isc[Solver::I_REASON * B + p] = 3;  // indefinite
    return;
  }
  sc[Solver::S_ALPHA * B + p] = sc[Solver::S_RZ * B + p] / pq;
}

// residual test after x += alpha p, r -= alpha q (KSPConvergedDefault)
__global__ void k_pcg_check(double* __restrict__ sc, int* __restrict__ isc, int* __restrict__ act, int B,
                            int maxit, double dtol) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B || !act[p]) return;
  const int it = ++isc[Solver::I_IT * B + p];
  const double rn = sqrt(sc[Solver::S_RR * B + p]);
  if (rn <= sc[Solver::S_TOL * B + p]) {
    act[p] = 0;
    isc[Solver::I_REASON * B + p] = 1;
  } else if (rn > dtol * sc[Solver::S_RN0 * B + p] || !isfinite(rn)) {
    act[p] = 0;
    isc[Solver::I_REASON * B + p] = 4;  // diverged
  } else if (it >= maxit) {
    act[p] = 0;
    isc[Solver::I_REASON * B + p] = 2;  // maxit
  }
}

// beta = rz_new / rz; rz = rz_new
__global__ void k_pcg_beta(double* __restrict__ sc, int* __restrict__ act, int B) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B || !act[p]) return;
  const double rzn = sc[Solver::S_RZNEW * B + p];
  sc[Solver::S_BETA * B + p] = rzn / sc[Solver::S_RZ * B + p];
  sc[Solver::S_RZ * B + p] = rzn;
}

// a1 = act and flag, a0 = act and not flag
__global__ void k_split_mask(const int* __restrict__ act, const int* __restrict__ flag, int* __restrict__ a1,
                             int* __restrict__ a0, int B) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B) return;
  const int a = act[p] != 0, f = flag[p] != 0;
  a1[p] = a && f;
  a0[p] = a && !f;
}

static dim3 pgrid(int B) { return dim3((B + 127) / 128); }

// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------
Solver::~Solver() {
  coarse.reset();  // it issues work on this solver's stream
  prof_clear();
  if (pcg_exec) cudaGraphExecDestroy(pcg_exec);
  void* ptrs[] = {mR, mT, m, mR16, mT16, m16, wmask, v, vtrial, disp_st, disp_adj, tab_st, tab_adj, gm, gx, divv, cadj, lamh, bf, g, x,
                  r, z, pv, q, vtx, mt, mt2, sj, work3, sreg, spec, partials, dsc, dact, dint, dparams, gwork};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (hsc) cudaFreeHost(hsc);
  if (hint) cudaFreeHost(hint);
  if (own_stream) cudaStreamDestroy(own_stream);
}

int Solver::alloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    err = std::string("cudaMalloc failed: ") + cudaGetErrorString(e);
    return CB_ERR_ALLOC;
  }
  bytes_ += (long long)bytes;
  return 0;
}

static int max_parts(const Dims& d) {
  int mp = dot_partials(3 * d.n());
  for (int a = 0; a < 3; ++a) mp = std::max(mp, deriv_partials(d, a, 3, true));
  mp = std::max(mp, c2r_partials(d, 3, true));
  mp = std::max(mp, 3 * field_stats_parts(d.n()));
  return mp;
}

// Options of the two-level preconditioner's coarse problems
// (Preconditioner::SetupCoarseGrid, src/Preconditioner.cpp:370-387): every
// option of the fine grid but nx = ceil(nx / gridscale); the coarse Krylov
// solve has no preconditioner (src/Preconditioner.cpp:947-951).
static claire_b200_opts coarse_opts(const claire_b200_opts& o) {
  claire_b200_opts oc = o;
  for (int k = 0; k < 3; ++k) oc.nx[k] = (int)std::ceil((double)o.nx[k] / o.pcgridscale);
  oc.precond = CB_PC_NONE;
  oc.betacont = 0.0;
  oc.scalecont = oc.gridcont = oc.train = oc.monitordefgrad = 0;
  return oc;
}

long long Solver::estimate_bytes(const claire_b200_opts& o, int B) {
  Dims d{o.nx[0], o.nx[1], o.nx[2]};
  const long long n = d.n(), nc = d.nc();
  const int nt = o.nt;
  long long floats = 0;
  const long long image_bytes = (nt + 3) * n * (o.bf16_images ? 2 : 4);  // mR, mT, state levels
  floats += 2 * 3 * n;                // v, vtrial
  floats += 2 * 3 * n;                // trajectories
  floats += (nt + 1) * 3 * n;         // grad m cache
  floats += nt * 3 * n;               // grad m (X) cache
  floats += 2 * n + 2 * n;            // divv, adjoint step factor, incremental state x2
  floats += (nt + 1) * n;             // adjoint levels
  floats += nt * n;                   // incremental state sources
  floats += 3 * n * 10;               // bf, g, x, r, z, p, q, vtx, work3, Reg p
  long long bytes = floats * 4 + image_bytes + 3 * nc * 8;
  bytes += 2 * tile_table_int4s(d) * 16;  // box tables of the two characteristics
  bytes += (long long)max_parts(d) * 8;
  bytes *= B;
  if (o.precond == CB_PC_TWOLEVEL) {
    // the coarse problems and the grid-change workspace
    const claire_b200_opts oc = coarse_opts(o);
    bytes += estimate_bytes(oc, B);
    bytes += 4 * grid_change_work(d.n1, oc.nx[0], std::max(3, nt + 1));
  }
  return bytes;
}

// A tile gather whose box copy ran out of its bounded wait skipped its tile
// (sl_tile.cuh); report it once, at the next GN-iteration boundary.
int Solver::check_stage() {
  unsigned long long t = 0;
  if (stage_timeouts(&t, stream)) return CB_ERR_CUDA;
  if (t <= stage_seen) return 0;
  stage_seen = t;
  err = "a tile gather's shared-memory box copy did not complete within its wait limit";
  return CB_ERR_CUDA;
}

int Solver::init(const claire_b200_opts& o, int Bn) {
  opts = o;
  B = Bn;
  stage_timeouts(&stage_seen);
  d = Dims{o.nx[0], o.nx[1], o.nx[2]};
  nt = o.nt;
  if (B < 1 || B > 1024 || nt < 1) {
    err = "invalid batch size or nt";
    return CB_ERR_ARG;
  }
  if (!(fft_col_size_supported(d.n1) && fft_col_size_supported(d.n2) && fft_size_supported(d.n3))) {
    err = "grid size has no FFT plan (each axis one of 16,32,48,64,96,128,192,256; x1 and x2 also 150)";
    return CB_ERR_UNSUPPORTED;
  }
  n = d.n();
  nc = d.nc();
  {
    // CLAIRE_B200_GRAPHS=0 runs PCG iterations as direct launches
    const char* ge = std::getenv("CLAIRE_B200_GRAPHS");
    graphs = !(ge && ge[0] == '0');
    const char* fd = std::getenv("CLAIRE_B200_FUSED_DOTS");
    fused_dots = fd && fd[0] == '1';
    const char* rr = std::getenv("CLAIRE_B200_REG_RECURRENCE");
    reg_rec_enabled = !(rr && rr[0] == '0');
  }
  ht = (float)(1.0 / nt);
  hd = (float)((kTwoPi / d.n1) * (kTwoPi / d.n2) * (kTwoPi / d.n3));
  {
    // refuse before allocating anything when the footprint cannot fit
    size_t freeb = 0, total = 0;
    if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
      err = "cudaMemGetInfo failed";
      return CB_ERR_CUDA;
    }
    const long long need = estimate_bytes(o, B);
    if (need > (long long)freeb) {
      err = "footprint " + std::to_string(need) + " bytes exceeds the free device memory (" +
            std::to_string((long long)freeb) + " bytes)";
      return CB_ERR_TOO_LARGE;
    }
  }
  if (cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    err = "stream creation failed";
    return CB_ERR_CUDA;
  }
  stream = own_stream;
  if (o.autotune)
    for (int axis_n : {d.n1, d.n2, d.n3})
      if (!fft_tuned(axis_n) && fft_autotune_once(axis_n, B, stream)) {
        err = "FFT autotuning failed";
        return CB_ERR_CUDA;
      }
  const size_t S = sizeof(float) * n * B, V = 3 * S;
  img16 = o.bf16_images != 0;
  ncc = o.distance == CB_DIST_NCC;
  if (ncc && img16) {
    err = "the NCC distance needs FP32 images";
    return CB_ERR_UNSUPPORTED;
  }
  mv_kind = o.precond == CB_PC_TWOLEVEL ? 1 : 0;
  if (mv_kind) {
    // the coarse grid must have an FFT plan, and an even size makes the
    // rectangular filters of Apply2LevelPrecond the restriction's band
    nc1 = coarse_opts(o).nx[0];
    if (img16 || ncc || d.n1 != d.n2 || d.n2 != d.n3) {
      err = "the two-level preconditioner needs a cubic grid, FP32 images and the SL2 distance";
      return CB_ERR_UNSUPPORTED;
    }
    if (nc1 < 2 || nc1 > d.n1 || (nc1 % 2) || !fft_size_supported(nc1)) {
      err = "the two-level preconditioner's coarse grid (ceil(nx / gridscale) points) is odd or has no FFT plan";
      return CB_ERR_UNSUPPORTED;
    }
  }
  if (img16) {
    const size_t S16 = sizeof(bf16) * n * B;
    CB_TRY(alloc((void**)&mR16, S16));
    CB_TRY(alloc((void**)&mT16, S16));
    CB_TRY(alloc((void**)&m16, S16 * (nt + 1)));
  } else {
    CB_TRY(alloc((void**)&mR, S));
    CB_TRY(alloc((void**)&mT, S));
    CB_TRY(alloc((void**)&m, S * (nt + 1)));
  }
  CB_TRY(alloc((void**)&v, V));
  CB_TRY(alloc((void**)&vtrial, V));
  CB_TRY(alloc((void**)&disp_st, V));
  CB_TRY(alloc((void**)&disp_adj, V));
  TP = tile_table_int4s(d);
  CB_TRY(alloc((void**)&tab_st, sizeof(int4) * TP * B));
  CB_TRY(alloc((void**)&tab_adj, sizeof(int4) * TP * B));
  CB_TRY(alloc((void**)&gm, V * (nt + 1)));
  CB_TRY(alloc((void**)&gx, V * nt));
  CB_TRY(alloc((void**)&divv, S));
  CB_TRY(alloc((void**)&cadj, S));
  CB_TRY(alloc((void**)&lamh, S * (nt + 1)));
  CB_TRY(alloc((void**)&mt, S));
  CB_TRY(alloc((void**)&mt2, S));
  CB_TRY(alloc((void**)&sj, S * nt));
  CB_TRY(alloc((void**)&bf, V));
  CB_TRY(alloc((void**)&g, V));
  CB_TRY(alloc((void**)&x, V));
  CB_TRY(alloc((void**)&r, V));
  CB_TRY(alloc((void**)&z, V));
  CB_TRY(alloc((void**)&pv, V));
  CB_TRY(alloc((void**)&q, V));
  CB_TRY(alloc((void**)&vtx, V));
  CB_TRY(alloc((void**)&work3, V));
  CB_TRY(alloc((void**)&sreg, V));
  CB_TRY(alloc((void**)&spec, sizeof(float2) * 3 * nc * B));
  maxparts = max_parts(d);
  CB_TRY(alloc((void**)&partials, sizeof(double) * maxparts * B));
  CB_TRY(alloc((void**)&dsc, sizeof(double) * NSLOT * B));
  CB_TRY(alloc((void**)&dact, sizeof(int) * 11 * B));  // masks; 8..10: PCG recurrence flags and splits
  dact2 = dact + B;
  CB_TRY(alloc((void**)&dint, sizeof(int) * NISLOT * B));
  CB_TRY(alloc((void**)&dparams, sizeof(SpecParams) * B));
  if (cudaMallocHost((void**)&hsc, sizeof(double) * NSLOT * B) != cudaSuccess ||
      cudaMallocHost((void**)&hint, sizeof(int) * NISLOT * B) != cudaSuccess) {
    err = "pinned host allocation failed";
    return CB_ERR_ALLOC;
  }
  cudaMemsetAsync(v, 0, V, stream);
  if (img16) {
    cudaMemsetAsync(mR16, 0, sizeof(bf16) * n * B, stream);
    cudaMemsetAsync(mT16, 0, sizeof(bf16) * n * B, stream);
  } else {
    cudaMemsetAsync(mR, 0, S, stream);
    cudaMemsetAsync(mT, 0, S, stream);
  }
  cudaMemsetAsync(dsc, 0, sizeof(double) * NSLOT * B, stream);
  cudaMemsetAsync(dint, 0, sizeof(int) * NISLOT * B, stream);
  ps.assign(B, ProbState());
  for (int b = 0; b < B; ++b) {
    ps[b].norm = o.regnorm;
    ps[b].model = o.model;
    ps[b].beta0 = o.beta[0];
    ps[b].beta1 = o.beta[1];
    ps[b].beta2 = o.beta[2];
  }
  state_of.assign(B, 0);
  ncc_scale_ok.assign(B, 0);
  CB_TRY(upload_params());
  if (cudaStreamSynchronize(stream) != cudaSuccess) {
    err = "initialisation failed";
    return CB_ERR_CUDA;
  }
  return 0;
}

int Solver::set_problem(int b, const claire_b200_opts& o, bool upload) {
  if (b < 0 || b >= B) return CB_ERR_ARG;
  if (o.nx[0] != d.n1 || o.nx[1] != d.n2 || o.nx[2] != d.n3 || o.nt != nt) {
    err = "per-problem options must keep nx and nt";
    return CB_ERR_ARG;
  }
  ps[b].norm = o.regnorm;
  ps[b].beta0 = o.beta[0];
  ps[b].beta1 = o.beta[1];
  ps[b].beta2 = o.beta[2];
  return upload ? upload_params() : 0;
}

int Solver::upload_params() {
  std::vector<SpecParams> h(B);
  for (int b = 0; b < B; ++b) {
    h[b].norm = ps[b].norm;
    h[b].beta0 = (float)ps[b].beta0;
    h[b].beta1 = (float)ps[b].beta1;
    h[b].beta2 = (float)ps[b].beta2;
    h[b].hd = hd;
    h[b].sigma[0] = h[b].sigma[1] = h[b].sigma[2] = 1.f;
  }
  if (cudaMemcpyAsync(dparams, h.data(), sizeof(SpecParams) * B, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return CB_ERR_CUDA;
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

int Solver::upload_mask(const std::vector<int>& sel, int* dmask) {
  if (cudaMemcpyAsync(dmask, sel.data(), sizeof(int) * B, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return CB_ERR_CUDA;
  return 0;
}

int Solver::fetch_scalars() {
  cudaError_t e = cudaMemcpyAsync(hsc, dsc, sizeof(double) * NSLOT * B, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hint, dint, sizeof(int) * NISLOT * B, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    err = std::string("device error: ") + cudaGetErrorString(e);
    return CB_ERR_CUDA;
  }
  return 0;
}

int Solver::dot(const float* a, long long ap, const float* b, long long bp, long long len, int s,
                const int* act, double scale) {
  const int np = dot_partials(len);
  CB_TRY(launch_dot(a, ap, b, bp, len, B, partials, maxparts, act, stream));
  CB_TRY(launch_finalize(partials, maxparts, np, slot(s), B, scale, false, stream, act));
  note_launches(2);
  return 0;
}

// ---------------------------------------------------------------------------
// forward problem (src/CLAIRE.cpp:1861-1984, 2116-2175)
// ---------------------------------------------------------------------------
// RK2 characteristic (sign +1 state into disp_st, -1 adjoint into disp_adj)
// and the box table its gathers use.
int Solver::characteristic(const float* vel, float sign, const int* act) {
  float* disp = sign > 0 ? disp_st : disp_adj;
  int4* tab = sign > 0 ? tab_st : tab_adj;
  CB_TRY(launch_trajectory(vel, 3 * n, disp, 3 * n, B, d, ht, sign, act, stream));
  CB_TRY(launch_tile_table(disp, 3 * n, tab, TP, B, d, act, stream));
  note_launches(1);
  return 0;
}

int Solver::state_solve(const float* vel, const int* act) {
  CB_TRY(characteristic(vel, 1.f, act));
  CB_TRY(state_init(nullptr, act));
  return state_steps(act);
}

// ---- image state in its storage type ------------------------------------------
// FP32 images: m, mR, mT.  bf16 images: m16, mR16, mT16, with every gather and
// every reduction computed in FP32 / FP64 and only the stored values rounded.

int Solver::state_init(const float* m0, const int* act) {
  const long long PM = (nt + 1) * n;
  if (img16) {
    if (m0) CB_TRY(launch_to_bf16(m0, n, m16, PM, n, B, act, stream));
    else CB_TRY(launch_copy_bf16(m16, PM, mT16, n, n, B, act, stream));
  } else {
    CB_TRY(launch_lincomb(m, PM, m0 ? m0 : mT, n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, n, B, act, stream));
  }
  note_launches(1);
  return 0;
}

int Solver::state_steps(const int* act) {
  const long long PM = (nt + 1) * n;
  for (int j = 0; j < nt; ++j) {
    CB_TRY(prof_mark(CB_PROF_STATE_STEP));
    if (img16)
      CB_TRY(launch_interp16(m16 + j * n, PM, disp_st, 3 * n, tab_st, TP, m16 + (j + 1) * n, PM, B, d, act, stream));
    else
      CB_TRY(launch_interp(m + j * n, PM, n, disp_st, 3 * n, tab_st, TP, m + (j + 1) * n, PM, n, 1, B, d, act,
                           stream));
    CB_TRY(prof_mark(CB_PROF_STATE_STEP));
  }
  note_launches(nt);
  return 0;
}

int Solver::state_out(float* m1, long long m1p, const int* act) {
  const long long PM = (nt + 1) * n;
  if (img16) CB_TRY(launch_from_bf16(m16 + nt * n, PM, 0, m1, m1p, 0, n, 1, B, act, stream));
  else CB_TRY(launch_lincomb(m1, m1p, m + nt * n, PM, nullptr, 1.0, nullptr, 0, nullptr, 0.0, n, B, act, stream));
  note_launches(1);
  return 0;
}

int Solver::image_diff_sumsq(bool template_image, const int* act, bool weighted) {
  const long long PM = (nt + 1) * n;
  const bool w = weighted && wmask;
  if (img16) {
    const bf16* b = template_image ? mT16 : m16 + nt * n;
    if (w) CB_TRY(launch_wdiff_sumsq(mR16, n, b, template_image ? n : PM, wmask, n, n, B, partials, maxparts, act, stream));
    else CB_TRY(launch_diff_sumsq16(mR16, n, b, template_image ? n : PM, n, B, partials, maxparts, act, stream));
  } else {
    const float* b = template_image ? mT : m + nt * n;
    if (w) CB_TRY(launch_wdiff_sumsq(mR, n, b, template_image ? n : PM, wmask, n, n, B, partials, maxparts, act, stream));
    else CB_TRY(launch_diff_sumsq(mR, n, b, template_image ? n : PM, n, B, partials, maxparts, act, stream));
  }
  note_launches(1);
  return 0;
}

int Solver::wdot(const float* a, long long ap, const float* b, long long bp, int s, const int* act) {
  if (!wmask) return dot(a, ap, b, bp, n, s, act);
  CB_TRY(launch_wdot(a, ap, b, bp, wmask, n, n, B, partials, maxparts, act, stream));
  CB_TRY(launch_finalize(partials, maxparts, dot_partials(n), slot(s), B, 1.0, false, stream, act));
  note_launches(2);
  return 0;
}

int Solver::set_mask(int b, const float* w) {
  if (b < 0 || b >= B) return CB_ERR_ARG;
  if (!wmask) {
    if (!w) return 0;  // no mask anywhere: nothing to do
    CB_TRY(alloc((void**)&wmask, sizeof(float) * n * B));
    CB_TRY(launch_fill(wmask, n, 1.f, n, B, nullptr, stream));
  }
  if (w) {
    if (cudaMemcpyAsync(wmask + b * n, w, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
  } else {
    CB_TRY(launch_fill(wmask + b * n, 0, 1.f, n, 1, nullptr, stream));
  }
  images_changed(b);
  coarse.reset();  // rebuilt with a mask by the next two-level setup
  // the recorded PCG iteration may lack the weighting: record it again
  if (pcg_exec) {
    cudaGraphExecDestroy(pcg_exec);
    pcg_exec = nullptr;
  }
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

int Solver::image_residual(float* y, long long yp, const int* act) {
  const long long PM = (nt + 1) * n;
  if (wmask) {
    // DistanceMeasureSL2::SetFinalConditionAE with a mask: w (mR - m1)
    if (img16) CB_TRY(launch_wdiff(y, yp, mR16, n, m16 + nt * n, PM, wmask, n, n, B, act, stream));
    else CB_TRY(launch_wdiff(y, yp, mR, n, m + nt * n, PM, wmask, n, n, B, act, stream));
  } else if (img16) CB_TRY(launch_diff16(y, yp, mR16, n, m16 + nt * n, PM, n, B, act, stream));
  else CB_TRY(launch_lincomb(y, yp, mR, n, nullptr, 1.0, m + nt * n, PM, nullptr, -1.0, n, B, act, stream));
  note_launches(1);
  return 0;
}

// grad m^j for j = 0..nt into gm.  bf16 levels are widened into gx first: gx
// is free here (it caches (grad m^j)(X), rebuilt by hessian_prep after every
// gradient) and holds 3nt >= nt+1 fields per problem.
int Solver::image_grad(const int* act) {
  const long long PM = (nt + 1) * n, PGM = (nt + 1) * 3 * n, PGX = nt * 3 * n;
  if (img16) {
    CB_TRY(launch_from_bf16(m16, PM, n, gx, PGX, n, n, nt + 1, B, act, stream));
    note_launches(1);
    return grad_fields(gx, PGX, n, gm, PGM, 3 * n, nt + 1, act);
  }
  return grad_fields(m, PM, n, gm, PGM, 3 * n, nt + 1, act);
}

int Solver::load_images(int b, const float* mRd, const float* mTd) {
  if (b < 0 || b >= B) return CB_ERR_ARG;
  if (img16) {
    CB_TRY(launch_to_bf16(mRd, 0, mR16 + b * n, 0, n, 1, nullptr, stream));
    CB_TRY(launch_to_bf16(mTd, 0, mT16 + b * n, 0, n, 1, nullptr, stream));
  } else if (cudaMemcpyAsync(mR + b * n, mRd, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
             cudaMemcpyAsync(mT + b * n, mTd, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) {
    return CB_ERR_CUDA;
  }
  state_of[b] = 0;
  return 0;
}

// ---------------------------------------------------------------------------
// device timers
// ---------------------------------------------------------------------------
// Events come from a recycled pool: creating one per mark costs host time
// between the launches being timed, which would stretch the measured gaps.
int Solver::prof_reserve(int count) {
  while ((int)prof_pool.size() < count) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return CB_ERR_CUDA;
    prof_pool.push_back(e);
  }
  return 0;
}

int Solver::prof_mark(int cat) {
  if (!prof_on) return 0;
  cudaEvent_t e;
  if (!prof_pool.empty()) {
    e = prof_pool.back();
    prof_pool.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    return CB_ERR_CUDA;
  }
  prof_ev[cat].push_back(e);
  return cudaEventRecord(e, stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

int Solver::prof_read(int cat, double* ms, long long* count) {
  if (cudaStreamSynchronize(stream) != cudaSuccess) return CB_ERR_CUDA;
  double total = 0.0;
  std::vector<cudaEvent_t>& ev = prof_ev[cat];
  for (size_t i = 0; i + 1 < ev.size(); i += 2) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) == cudaSuccess) total += t;
  }
  if (ms) *ms = total;
  if (count) *count = (long long)(ev.size() / 2);
  prof_pool.insert(prof_pool.end(), ev.begin(), ev.end());
  ev.clear();
  return 0;
}

void Solver::prof_clear() {
  for (int c = 0; c < CB_PROF_NCAT; ++c) {
    for (cudaEvent_t e : prof_ev[c]) cudaEventDestroy(e);
    prof_ev[c].clear();
  }
  for (cudaEvent_t e : prof_pool) cudaEventDestroy(e);
  prof_pool.clear();
}

// D = 1/2 hd sum (mR - m1)^2 (src/DistanceMeasureSL2.cpp:93-155), or the NCC
// distance (src/DistanceMeasureNCC.cpp:171-245)
int Solver::distance(const std::vector<int>& sel, const int* act) {
  const int np = dot_partials(n);
  if (ncc) {
    const long long PM = (nt + 1) * n;
    CB_TRY(ncc_setup_scale(sel));
    const float* m1 = m + nt * n;
    CB_TRY(wdot(m1, PM, m1, PM, S_NA, act));
    CB_TRY(wdot(mR, n, mR, n, S_NRR, act));
    CB_TRY(wdot(m1, PM, mR, n, S_NI, act));
    k_ncc<<<pgrid(B), 128, 0, stream>>>(dsc, act, B, 1, (double)hd);
    note_launches(1);
    return (int)cudaGetLastError();
  }
  CB_TRY(image_diff_sumsq(false, act, true));
  CB_TRY(launch_finalize(partials, maxparts, np, slot(S_D), B, 0.5 * (double)hd, false, stream, act));
  note_launches(1);
  return 0;
}

// DistanceMeasureNCC::SetupScale for the selected problems whose images
// changed since their scale was set (src/CLAIREBase.cpp:686-689 calls it once
// the images are known).
int Solver::ncc_setup_scale(const std::vector<int>& sel) {
  std::vector<int> need(B, 0);
  bool any = false;
  for (int b = 0; b < B; ++b)
    if (sel[b] && !ncc_scale_ok[b]) { need[b] = 1; any = true; }
  if (!any) return 0;
  int* m3 = dact + 2 * B;
  CB_TRY(upload_mask(need, m3));
  CB_TRY(wdot(mT, n, mT, n, S_NA, m3));
  CB_TRY(wdot(mR, n, mR, n, S_NRR, m3));
  CB_TRY(wdot(mT, n, mR, n, S_NI, m3));
  if (wmask) CB_TRY(launch_wdiff_sumsq(mT, n, mR, n, wmask, n, n, B, partials, maxparts, m3, stream));
  else CB_TRY(launch_diff_sumsq(mT, n, mR, n, n, B, partials, maxparts, m3, stream));
  CB_TRY(launch_finalize(partials, maxparts, dot_partials(n), slot(S_NL2), B, 1.0, false, stream, m3));
  k_ncc<<<pgrid(B), 128, 0, stream>>>(dsc, m3, B, 0, (double)hd);
  note_launches(3);
  CB_TRY((int)cudaGetLastError());
  for (int b = 0; b < B; ++b)
    if (need[b]) ncc_scale_ok[b] = 1;
  return 0;
}

int Solver::ncc_final_condition(float* lam, long long lp, const int* act) {
  const long long PM = (nt + 1) * n;
  const float* m1 = m + nt * n;
  CB_TRY(wdot(m1, PM, m1, PM, S_NA, act));
  CB_TRY(wdot(mR, n, mR, n, S_NRR, act));
  CB_TRY(wdot(m1, PM, mR, n, S_NI, act));
  k_ncc<<<pgrid(B), 128, 0, stream>>>(dsc, act, B, 2, (double)hd);
  CB_TRY((int)cudaGetLastError());
  CB_TRY(launch_lincomb(lam, lp, mR, n, slot(S_CA), 1.0, m1, PM, slot(S_CB), 1.0, n, B, act, stream));
  if (wmask) CB_TRY(launch_mulw(lam, lp, wmask, n, n, B, act, stream));
  note_launches(3);
  return 0;
}

// lam holds m~(1) on entry and lambda~(1) on exit; the sums of m1 and mR are
// those of the last gradient (the GN iterate).
int Solver::ncc_inc_final_condition(float* lam, long long lp, const int* act) {
  const long long PM = (nt + 1) * n;
  const float* m1 = m + nt * n;
  CB_TRY(wdot(m1, PM, lam, lp, S_NIM, act));
  CB_TRY(wdot(mR, n, lam, lp, S_NRM, act));
  k_ncc<<<pgrid(B), 128, 0, stream>>>(dsc, act, B, 3, (double)hd);
  CB_TRY((int)cudaGetLastError());
  CB_TRY(launch_lincomb(lam, lp, lam, lp, slot(S_CC), 1.0, mR, n, slot(S_CA), 1.0, n, B, act, stream));
  CB_TRY(launch_lincomb(lam, lp, lam, lp, nullptr, 1.0, m1, PM, slot(S_CB), 1.0, n, B, act, stream));
  if (wmask) CB_TRY(launch_mulw(lam, lp, wmask, n, n, B, act, stream));
  note_launches(4);
  return 0;
}

// Regularization::EvaluateFunctional.  Raw sums land in S_R (and S_RV for
// H1's L2 part); the per-norm factors are applied on the host.
int Solver::reg_functional(const float* vel, const std::vector<int>& sel, const int* act) {
  std::vector<int> ma(B, 0), mb(B, 0);
  bool any_a = false, any_b = false;
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    if (ps[b].norm == NORM_H1 || ps[b].norm == NORM_H1SN) { ma[b] = 1; any_a = true; }
    else { mb[b] = 1; any_b = true; }
  }
  int* dma = dact + 4 * B;
  int* dmb = dact + 5 * B;
  if (any_a) {
    // sum_i sum_k ||d/dx_k v_i||^2 with spectral derivatives (src/RegularizationH1SN.cpp:84-141)
    CB_TRY(upload_mask(ma, dma));
    for (int a = 0; a < 3; ++a) {
      const int np = deriv_partials(d, a, 3);
      CB_TRY(launch_deriv(vel, 3 * n, n, nullptr, 0, 0, 3, B, d, a, EPI_SUMSQ, partials, maxparts, dma, stream));
      CB_TRY(launch_finalize(partials, maxparts, np, slot(S_R), B, 1.0, a > 0, stream, dma));
    }
    note_launches(6);
    CB_TRY(dot(vel, 3 * n, vel, 3 * n, 3 * n, S_RV, dma));
  }
  if (any_b) {
    CB_TRY(upload_mask(mb, dmb));
    CB_TRY(launch_r2c3d(vel, 3 * n, n, spec, 3 * nc, 3, B, d, dmb, stream));
    CB_TRY(launch_pencil(spec, 3 * nc, B, d, OP_REG_FUNC, dparams, 3, 3, dmb, stream));
    const int np = c2r_partials(d, 3);
    CB_TRY(launch_c2r3d(spec, 3 * nc, nullptr, 0, 0, 3, B, d, EPI_SUMSQ, nullptr, partials, maxparts, dmb, stream));
    // finalize only the selected problems' slots: unselected keep stale values
    CB_TRY(launch_finalize(partials, maxparts, np, slot(S_R), B, 1.0, false, stream, dmb));
    note_launches(6);
    (void)any_a;
  }
  (void)act;
  return 0;
}

// CLAIREDivReg::EvaluteRegularizationDIV (src/CLAIREDivReg.cpp:165-245):
// S_RW = ||grad div v||^2 + ||div v||^2 (spectral derivatives, FP64 sums);
// the caller scales by hd beta_w / 2.
int Solver::div_penalty(const float* vel, const int* act) {
  float* dv = work3;  // div v of problem p at dv + p*n (scratch)
  CB_TRY(divergence(vel, dv, act));
  CB_TRY(dot(dv, n, dv, n, n, S_RW, act));
  for (int a = 0; a < 3; ++a) {
    const int np = deriv_partials(d, a, 1);
    CB_TRY(launch_deriv(dv, n, n, nullptr, 0, 0, 1, B, d, a, EPI_SUMSQ, partials, maxparts, act, stream));
    CB_TRY(launch_finalize(partials, maxparts, np, slot(S_RW), B, 1.0, true, stream, act));
  }
  note_launches(6);
  return 0;
}

static double reg_factor(const ProbState& s, double hd, double sumsq, double vv) {
  switch (s.norm) {
    case NORM_H1SN: return 0.5 * hd * s.beta0 * sumsq;
    case NORM_H1: return 0.5 * hd * s.beta0 * (sumsq + s.beta1 * vv);
    case NORM_L2: return 0.5 * hd * sumsq;               // symbol sqrt(beta)
    case NORM_H2: return 0.5 * hd * sumsq;
    case NORM_H2SN: return 0.5 * hd * s.beta0 * sumsq;
    case NORM_H3: return 0.5 * hd * sumsq;
    case NORM_H3SN: return 0.5 * hd * s.beta0 * sumsq;
    default: return 0.0;
  }
}

int Solver::objective_at(const float* vel, const std::vector<int>& sel) {
  CB_TRY(prof_mark(CB_PROF_OBJECTIVE));
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(state_solve(vel, dact));
  CB_TRY(distance(sel, dact));
  // mixed-class batches run reg_functional's two passes with their own masks;
  // the finalize of the second pass must not clobber the first, so run classes
  // one after another and read back in between.
  std::vector<int> sa(B, 0), sb(B, 0);
  bool any_a = false, any_b = false;
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    if (ps[b].norm == NORM_H1 || ps[b].norm == NORM_H1SN) { sa[b] = 1; any_a = true; }
    else { sb[b] = 1; any_b = true; }
  }
  std::vector<double> R(B, 0.0);
  if (any_a) {
    CB_TRY(reg_functional(vel, sa, dact));
    CB_TRY(fetch_scalars());
    for (int b = 0; b < B; ++b)
      if (sa[b]) R[b] = reg_factor(ps[b], hd, hsc[S_R * B + b], hsc[S_RV * B + b]);
  }
  if (any_b) {
    CB_TRY(reg_functional(vel, sb, dact));
  }
  if (opts.model == CB_MODEL_RELAXEDSTOKES) CB_TRY(div_penalty(vel, dact));
  CB_TRY(fetch_scalars());
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    if (sb[b]) R[b] = reg_factor(ps[b], hd, hsc[S_R * B + b], 0.0);
    // CLAIREDivReg::EvaluateObjective: J = D + R1(v) + R2(div v) (src/CLAIREDivReg.cpp:109-160)
    if (opts.model == CB_MODEL_RELAXEDSTOKES) R[b] += 0.5 * hd * ps[b].beta2 * hsc[S_RW * B + b];
    ps[b].D = hsc[S_D * B + b];
    ps[b].R = R[b];
    ps[b].J = ps[b].D + ps[b].R;
    ps[b].obj_evals++;
    ps[b].pde_solves++;
    state_of[b] = (vel == v) ? 1 : 2;
  }
  return prof_mark(CB_PROF_OBJECTIVE);
}

// ---------------------------------------------------------------------------
// spectral building blocks
// ---------------------------------------------------------------------------
// out = F^-1(symbol F(vin)) with epilogue epi; with dot_with, out . dot_with
// (FP64) lands in slot dot_slot (the inverse transform's epilogue sums it).
int Solver::reg_op(const float* vin, float* out, int op, int epi, const int* act, const float* dot_with,
                   int dot_slot) {
  CB_TRY(launch_r2c3d(vin, 3 * n, n, spec, 3 * nc, 3, B, d, act, stream));
  CB_TRY(launch_pencil(spec, 3 * nc, B, d, op, dparams, 3, 3, act, stream));
  if (dot_with && fused_dots) {
    const int e2 = (epi == EPI_ADD) ? EPI_ADD_DOT : EPI_STORE_DOT;
    CB_TRY(launch_c2r3d(spec, 3 * nc, out, 3 * n, n, 3, B, d, e2, nullptr, partials, maxparts, act, stream,
                        dot_with));
    CB_TRY(launch_finalize(partials, maxparts, c2r_partials(d, 3), slot(dot_slot), B, 1.0, false, stream, act));
    note_launches(6);
    return 0;
  }
  if (dot_with) {
    CB_TRY(launch_c2r3d(spec, 3 * nc, out, 3 * n, n, 3, B, d, epi, nullptr, nullptr, 0, act, stream));
    note_launches(5);
    return dot(out, 3 * n, dot_with, 3 * n, 3 * n, dot_slot, act);
  }
  CB_TRY(launch_c2r3d(spec, 3 * nc, out, 3 * n, n, 3, B, d, epi, nullptr, nullptr, 0, act, stream));
  note_launches(5);
  return 0;
}

// out[level j][axis a] = d/dx_a f[level j]
int Solver::grad_fields(const float* f, long long fp, long long ifs, float* out, long long op,
                        long long ofs, int nf, const int* act) {
  for (int a = 0; a < 3; ++a)
    CB_TRY(launch_deriv(f, fp, ifs, out + a * n, op, ofs, nf, B, d, a, EPI_STORE, nullptr, 0, act, stream));
  note_launches(3);
  return 0;
}

int Solver::divergence(const float* vel, float* out, const int* act) {
  for (int a = 0; a < 3; ++a)
    CB_TRY(launch_deriv(vel + a * n, 3 * n, n, out, n, n, 1, B, d, a, a == 0 ? EPI_STORE : EPI_ADD, nullptr, 0,
                        act, stream));
  note_launches(3);
  return 0;
}

// Backward RK2 sweep (src/CLAIRE.cpp:2646-2686, 3940-3971) over the stored
// adjoint levels, then the trapezoid body force (:2689-2709), the projection
// (src/CLAIRE.cpp:2338) and the hd scaling (:2341).  On entry level nt of
// `lamh` holds lambda(t=1); on exit every level 0..nt is filled.  With
// add_reg (no projection), bout receives the body force and is then expected
// to be completed by an accumulating regularisation pass.
int Solver::adjoint_sweep(float* bout, const int* act, double hscale) {
  const double hfac = hscale >= 0.0 ? hscale : (double)hd;
  const long long PGM = (nt + 1) * 3 * n, PL = (nt + 1) * n;
  for (int j = 0; j < nt; ++j) {
    const int l = nt - j;  // lambda^{l-1} = c * lambda^l(X_adj)
    CB_TRY(prof_mark(CB_PROF_ADJOINT_STEP));
    CB_TRY(launch_gather_scale(lamh + l * n, PL, disp_adj, 3 * n, tab_adj, TP, cadj, n, lamh + (l - 1) * n, PL, B,
                               d, act, stream));
    CB_TRY(prof_mark(CB_PROF_ADJOINT_STEP));
  }
  const bool proj = opts.model != CB_MODEL_COMPRESSIBLE;
  CB_TRY(launch_body_force(lamh, PL, gm, PGM, bout, 3 * n, nt, ht, proj ? 1.f : (float)hfac, B, n, act, stream));
  note_launches(nt + 1);
  if (proj) {
    CB_TRY(launch_r2c3d(bout, 3 * n, n, spec, 3 * nc, 3, B, d, act, stream));
    CB_TRY(launch_pencil(spec, 3 * nc, B, d, opts.model == CB_MODEL_STOKES ? OP_LERAY : OP_LERAY_RELAXED, dparams,
                         3, 3, act, stream));
    CB_TRY(launch_c2r3d(spec, 3 * nc, bout, 3 * n, n, 3, B, d, EPI_ADD, nullptr, nullptr, 0, act, stream));
    CB_TRY(launch_lincomb(bout, 3 * n, bout, 3 * n, nullptr, hfac, nullptr, 0, nullptr, 0.0, 3 * n, B, act,
                          stream));
    note_launches(6);
  }
  return 0;
}

// out = Reg.EvaluateGradient(vin) + body force (src/CLAIRE.cpp:1356-1361,
// 1015-1042).  Without a projection the body force is written into out first
// and the regularisation's inverse transform accumulates into it.
int Solver::finish_with_reg(const float* vin, float* out, const int* act, const float* dot_with, int dot_slot) {
  const bool proj = opts.model != CB_MODEL_COMPRESSIBLE;
  if (reg_in) {
    // Reg(vin) supplied by the PCG's recurrence for the problems of rec_act:
    // out = body force + Reg(vin); the others transform as below
    float* bfo = proj ? bf : out;
    CB_TRY(adjoint_sweep(bfo, act));
    if (norec_act) {
      if (proj) {
        CB_TRY(reg_op(vin, out, OP_REG_GRAD, EPI_STORE, norec_act));
        CB_TRY(launch_lincomb(out, 3 * n, out, 3 * n, nullptr, 1.0, bf, 3 * n, nullptr, 1.0, 3 * n, B, norec_act,
                              stream));
        note_launches(1);
        if (dot_with) CB_TRY(dot(out, 3 * n, dot_with, 3 * n, 3 * n, dot_slot, norec_act));
      } else {
        CB_TRY(reg_op(vin, out, OP_REG_GRAD, EPI_ADD, norec_act, dot_with, dot_slot));
      }
    }
    if (dot_with) {
      CB_TRY(launch_add_dot(out, bfo, reg_in, dot_with, 3 * n, 3 * n, B, partials, maxparts, rec_act, stream));
      CB_TRY(launch_finalize(partials, maxparts, dot_partials(3 * n), slot(dot_slot), B, 1.0, false, stream,
                             rec_act));
      note_launches(2);
    } else {
      CB_TRY(launch_lincomb(out, 3 * n, bfo, 3 * n, nullptr, 1.0, reg_in, 3 * n, nullptr, 1.0, 3 * n, B, rec_act,
                            stream));
      note_launches(1);
    }
    return 0;
  }
  if (!proj) {
    CB_TRY(adjoint_sweep(out, act));
    CB_TRY(reg_op(vin, out, OP_REG_GRAD, EPI_ADD, act, dot_with, dot_slot));
    return 0;
  }
  CB_TRY(adjoint_sweep(bf, act));
  CB_TRY(reg_op(vin, out, OP_REG_GRAD, EPI_STORE, act));
  CB_TRY(launch_lincomb(out, 3 * n, out, 3 * n, nullptr, 1.0, bf, 3 * n, nullptr, 1.0, 3 * n, B, act, stream));
  note_launches(1);
  if (dot_with) CB_TRY(dot(out, 3 * n, dot_with, 3 * n, 3 * n, dot_slot, act));
  return 0;
}

// EvaluateGradient at v (src/CLAIRE.cpp:871-1042); the state must be valid for v.
int Solver::gradient(const int* act) {
  const long long PM = (nt + 1) * n, PGM = (nt + 1) * 3 * n, PL = (nt + 1) * n;
  CB_TRY(prof_mark(CB_PROF_GRADIENT));
  CB_TRY(characteristic(v, -1.f, act));
  CB_TRY(image_grad(act));
  CB_TRY(divergence(v, divv, act));
  CB_TRY(launch_adjoint_coef(divv, n, disp_adj, 3 * n, tab_adj, TP, cadj, n, ht, B, d, act, stream));
  // lambda(t=1) = mR - m1 (src/DistanceMeasureSL2.cpp:156-222), or NCC's
  if (ncc) CB_TRY(ncc_final_condition(lamh + nt * n, PL, act));
  else CB_TRY(image_residual(lamh + nt * n, PL, act));
  note_launches(2);
  CB_TRY(finish_with_reg(v, g, act));
  CB_TRY(dot(g, 3 * n, g, 3 * n, 3 * n, S_GG, act));
  return prof_mark(CB_PROF_GRADIENT);
}

// caches for the Hessian: (grad m^j)(X_state), j < nt
int Solver::hessian_prep(const int* act) {
  const long long PGM = (nt + 1) * 3 * n, PGX = nt * 3 * n;
  CB_TRY(launch_interp(gm, PGM, n, disp_st, 3 * n, tab_st, TP, gx, PGX, n, 3 * nt, B, d, act, stream));
  note_launches(1);
  return 0;
}

// GN Hessian matvec (src/CLAIRE.cpp:1311-1379, 3147-3290, 3307-3490, 3849-4012).
// m~^0 = 0, so m~^1 = s_0; steps j = 1 .. nt-1 gather; the last one writes
// lambda~(t=1) = -m~(t=1) straight into the adjoint's level nt.
int Solver::inc_state(const float* vin, const int* act) {
  const long long PGM = (nt + 1) * 3 * n, PGX = nt * 3 * n, PL = (nt + 1) * n, PS = nt * n;
  CB_TRY(launch_interp(vin, 3 * n, n, disp_st, 3 * n, tab_st, TP, vtx, 3 * n, n, 3, B, d, act, stream));
  CB_TRY(launch_incstate_source(gx, PGX, vtx, 3 * n, gm, PGM, vin, 3 * n, sj, PS, nt, ht, B, n, act, stream));
  note_launches(2);
  float* lam_end = lamh + nt * n;
  // SL2: lambda~(1) = -m~(1), written by the last step; NCC: m~(1) there first
  const float fin = ncc ? 1.f : -1.f;
  if (nt == 1) {
    CB_TRY(launch_lincomb(lam_end, PL, sj, PS, nullptr, fin, nullptr, 0, nullptr, 0.0, n, B, act, stream));
    note_launches(1);
  }
  const float* cur = sj;  // m~^1 = s_0
  long long cp = PS;
  float* bufs[2] = {mt, mt2};
  for (int j = 1; j < nt; ++j) {
    const bool last = (j == nt - 1);
    float* out = last ? lam_end : bufs[j & 1];
    CB_TRY(prof_mark(CB_PROF_INCSTATE_STEP));
    CB_TRY(launch_gather_add(cur, cp, disp_st, 3 * n, tab_st, TP, sj + j * n, PS, out, last ? PL : n,
                             last ? fin : 1.f, B, d, act, stream));
    CB_TRY(prof_mark(CB_PROF_INCSTATE_STEP));
    cur = out;
    cp = n;
  }
  note_launches(nt - 1);
  if (ncc) CB_TRY(ncc_inc_final_condition(lam_end, PL, act));
  // DistanceMeasureSL2::SetFinalConditionIAE with a mask: -w m~(1)
  else if (wmask) CB_TRY(launch_mulw(lam_end, PL, wmask, n, n, B, act, stream));
  return 0;
}

int Solver::hessian(const float* vin, float* hout, const int* act, int pq_slot) {
  CB_TRY(inc_state(vin, act));
  CB_TRY(finish_with_reg(vin, hout, act, pq_slot >= 0 ? vin : nullptr, pq_slot));
  return 0;
}

// Symmetrically preconditioned GN Hessian, CLAIRE::PrecondHessMatVecSym
// (src/CLAIRE.cpp:1455-1532): hout = hd vin + P^1/2 b~[P^1/2 vin], with
// P^1/2 = (beta A)^-1/2 (ApplyInverse, applysqrt) and b~ the incremental body
// force (hd and the projection included).  mv_kind 2 divides by hd
// (HessianMatVec with scale = false, src/CLAIRE.cpp:1279-1285): hd drops out
// of the first term and the body force is formed with factor 1.
int Solver::hessian_sym(const float* vin, float* hout, const int* act, int pq_slot) {
  float* t = work3;  // P^1/2 vin
  CB_TRY(reg_op(vin, t, OP_REG_SQRTINV, EPI_STORE, act));
  CB_TRY(inc_state(t, act));
  const bool unscaled = mv_kind == 2;
  CB_TRY(adjoint_sweep(bf, act, unscaled ? 1.0 : (double)hd));
  CB_TRY(launch_lincomb(hout, 3 * n, vin, 3 * n, nullptr, unscaled ? 1.0 : (double)hd, nullptr, 0, nullptr, 0.0,
                        3 * n, B, act, stream));
  note_launches(1);
  return reg_op(bf, hout, OP_REG_SQRTINV, EPI_ADD, act, pq_slot >= 0 ? vin : nullptr, pq_slot);
}

// det(grad y) (inverse: det(grad(inv(y)))) of the selected problems at their
// velocity v by the SL scheme of DeformationFields::ComputeDetDefGradSL
// (src/DeformationFields.cpp:636-739): J^0 = 1, J^{j+1} = c J^j(X_state) with
// the RK2 factor c of the signed divergence terms.  J lands in the first n
// floats of each problem's work3 block; stats[b] = (min, mean, max).
int Solver::det_def_grad(const std::vector<int>& sel, bool inverse, std::vector<double>& stats) {
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(characteristic(v, 1.f, dact));
  CB_TRY(divergence(v, divv, dact));
  float* c = work3 + n;      // step factor
  float* j0 = work3;         // J (final result)
  float* j1 = work3 + 2 * n; // ping-pong buffer
  CB_TRY(launch_adjoint_coef(divv, n, disp_st, 3 * n, tab_st, TP, c, 3 * n, ht, B, d, dact, stream,
                             inverse ? -1.f : 1.f));
  CB_TRY(launch_fill(j0, 3 * n, 1.f, n, B, dact, stream));  // J^0 = 1 (:336)
  float* cur = j0;
  float* nxt = j1;
  for (int j = 0; j < nt; ++j) {
    CB_TRY(launch_gather_scale(cur, 3 * n, disp_st, 3 * n, tab_st, TP, c, 3 * n, nxt, 3 * n, B, d, dact, stream));
    std::swap(cur, nxt);
  }
  if (cur != j0) CB_TRY(launch_lincomb(j0, 3 * n, cur, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, n, B, dact,
                                       stream));
  note_launches(nt + 5);
  // the state characteristic now belongs to v: cached state levels are stale
  for (int b = 0; b < B; ++b)
    if (sel[b]) state_of[b] = 0;
  const int np = field_stats_parts(n);
  CB_TRY(launch_field_stats(j0, 3 * n, n, B, partials, stream));
  note_launches(1);
  std::vector<double> h((size_t)3 * np * B);
  if (cudaMemcpyAsync(h.data(), partials, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return CB_ERR_CUDA;
  stats.assign((size_t)3 * B, 0.0);
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    const double* pp = h.data() + (size_t)3 * np * b;
    double sum = 0.0, mn = pp[np], mx = pp[2 * np];
    for (int k = 0; k < np; ++k) {
      sum += pp[k];
      mn = std::min(mn, pp[np + k]);
      mx = std::max(mx, pp[2 * np + k]);
    }
    stats[3 * b] = mn;
    stats[3 * b + 1] = sum / (double)n;
    stats[3 * b + 2] = mx;
  }
  return 0;
}

// Deformation map of the selected problems at their velocity v,
// DeformationFields::ComputeDeformationMapSLRK2 (src/DeformationFields.cpp:
// 1472-1585; ComputeDeformationMap, :1189-1268): particles start on the grid
// (y = x) and move backward along v with RK2, v evaluated at the current
// positions by the tricubic gather: yt = y - ht v(y), y <- y - ht/2 (v(y) +
// v(yt)) per time step (ht < 0 for the inverse map).  The positions are kept
// as displacements u = y - x in grid units (x: u, r: yt - x, z: v at the
// query points); the gathers take any displacement (periodic wrap).
int Solver::deformation_map(const std::vector<int>& sel, bool inverse) {
  CB_TRY(upload_mask(sel, dact));
  const double h = inverse ? -(double)ht : (double)ht;
  const double c[3] = {d.n1 / kTwoPi, d.n2 / kTwoPi, d.n3 / kTwoPi};  // grid units per unit length
  float *u = x, *ut = r, *vy = z;
  CB_TRY(launch_fill(u, 3 * n, 0.f, 3 * n, B, dact, stream));
  note_launches(1);
  for (int j = 0; j < nt; ++j) {
    CB_TRY(launch_tile_table(u, 3 * n, tab_st, TP, B, d, dact, stream));
    CB_TRY(launch_interp(v, 3 * n, n, u, 3 * n, tab_st, TP, vy, 3 * n, n, 3, B, d, dact, stream));
    for (int k = 0; k < 3; ++k) {
      CB_TRY(launch_lincomb(ut + k * n, 3 * n, u + k * n, 3 * n, nullptr, 1.0, vy + k * n, 3 * n, nullptr,
                            -h * c[k], n, B, dact, stream));
      CB_TRY(launch_lincomb(u + k * n, 3 * n, u + k * n, 3 * n, nullptr, 1.0, vy + k * n, 3 * n, nullptr,
                            -0.5 * h * c[k], n, B, dact, stream));
    }
    CB_TRY(launch_tile_table(ut, 3 * n, tab_st, TP, B, d, dact, stream));
    CB_TRY(launch_interp(v, 3 * n, n, ut, 3 * n, tab_st, TP, vy, 3 * n, n, 3, B, d, dact, stream));
    for (int k = 0; k < 3; ++k)
      CB_TRY(launch_lincomb(u + k * n, 3 * n, u + k * n, 3 * n, nullptr, 1.0, vy + k * n, 3 * n, nullptr,
                            -0.5 * h * c[k], n, B, dact, stream));
    note_launches(13);
  }
  // the state characteristic's box table now belongs to u: cached levels are stale
  for (int b = 0; b < B; ++b)
    if (sel[b]) state_of[b] = 0;
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

// Displacement field by the SL scheme, DeformationFields::
// ComputeDisplacementFieldSL (src/DeformationFields.cpp:1816-1909): with the
// state characteristic X of v, u^0 = 0 and u^{j+1} = u^j(X) + ht/2 (v(X) + v).
int Solver::displacement_field(const std::vector<int>& sel) {
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(characteristic(v, 1.f, dact));
  float *u = x, *ux = r, *vx = z;
  CB_TRY(launch_interp(v, 3 * n, n, disp_st, 3 * n, tab_st, TP, vx, 3 * n, n, 3, B, d, dact, stream));
  CB_TRY(launch_fill(u, 3 * n, 0.f, 3 * n, B, dact, stream));
  note_launches(2);
  for (int j = 0; j < nt; ++j) {
    CB_TRY(launch_interp(u, 3 * n, n, disp_st, 3 * n, tab_st, TP, ux, 3 * n, n, 3, B, d, dact, stream));
    CB_TRY(launch_lincomb(u, 3 * n, ux, 3 * n, nullptr, 1.0, vx, 3 * n, nullptr, 0.5 * ht, 3 * n, B, dact, stream));
    CB_TRY(launch_lincomb(u, 3 * n, u, 3 * n, nullptr, 1.0, v, 3 * n, nullptr, 0.5 * ht, 3 * n, B, dact, stream));
    note_launches(3);
  }
  for (int b = 0; b < B; ++b)
    if (sel[b]) state_of[b] = 0;  // the state characteristic is v's, but the levels are not solved
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

// Deformation gradient by the SL scheme, DeformationFields::ComputeDefGrad /
// ComputeDefGradSL (src/DeformationFields.cpp:821-955, 956-1117): F^0 = I,
// gv = grad v (spectral), gv(X) on the state characteristic, and per time step
// F <- the second RK2 stage of k_defgrad_step applied to F(X).  Work arrays of
// 36 n floats are allocated for the call.
int Solver::def_grad(int b, float* F9) {
  std::vector<int> sel(B, 0);
  sel[b] = 1;
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(characteristic(v, 1.f, dact));
  // scratch for problem b alone: the scratch arrays take problem stride 0
  // (only b is active in the mask)
  float* w = nullptr;
  if (cudaMalloc(&w, sizeof(float) * 36 * n) != cudaSuccess) {
    cudaGetLastError();
    err = "deformation gradient: allocation failed";
    return CB_ERR_ALLOC;
  }
  float *F = w, *FX = w + 9 * n, *gv = w + 18 * n, *gvx = w + 27 * n;
  const long long P9 = 9 * n;
  int e = grad_fields(v, 3 * n, n, gv, 0, 3 * n, 3, dact);  // gv[3k + a] = d_a v_k
  if (!e) e = launch_interp(gv, 0, n, disp_st, 3 * n, tab_st, TP, gvx, 0, n, 9, B, d, dact, stream);
  for (int c = 0; c < 9 && !e; ++c)
    e = launch_fill(F + c * n, 0, (c % 4 == 0) ? 1.f : 0.f, n, B, dact, stream);
  for (int j = 0; j < nt && !e; ++j) {
    e = launch_interp(F, 0, n, disp_st, 3 * n, tab_st, TP, FX, 0, n, 9, B, d, dact, stream);
    if (!e) e = launch_defgrad_step(FX, gvx, gv, F, 0, ht, B, n, dact, stream);
  }
  note_launches(2 + 9 + 2 * nt);
  if (!e && (cudaMemcpyAsync(F9, F, sizeof(float) * P9, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
             cudaStreamSynchronize(stream) != cudaSuccess))
    e = CB_ERR_CUDA;
  cudaFree(w);
  state_of[b] = 0;  // the state characteristic's tables were rebuilt for v
  return e ? (e < 0 ? e : CB_ERR_CUDA) : 0;
}

// Gradient of the SL displacement field, the first half of
// DeformationFields::ComputeDetDefGradViaDispField (src/DeformationFields.cpp:
// 745-815): u by displacement_field, then the spectral gradient of each
// component.
int Solver::disp_grad(int b, float* G9) {
  std::vector<int> sel(B, 0);
  sel[b] = 1;
  CB_TRY(displacement_field(sel));
  float* w = nullptr;
  if (cudaMalloc(&w, sizeof(float) * 9 * n) != cudaSuccess) {  // problem b alone (stride 0)
    cudaGetLastError();
    err = "displacement gradient: allocation failed";
    return CB_ERR_ALLOC;
  }
  int e = grad_fields(x, 3 * n, n, w, 0, 3 * n, 3, dact);
  if (!e && (cudaMemcpyAsync(G9, w, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost, stream) !=
                 cudaSuccess ||
             cudaStreamSynchronize(stream) != cudaSuccess))
    e = CB_ERR_CUDA;
  cudaFree(w);
  return e ? (e < 0 ? e : CB_ERR_CUDA) : 0;
}

// ---------------------------------------------------------------------------
// public single-shot operations
// ---------------------------------------------------------------------------
int Solver::gradient_at_current(const std::vector<int>& sel) {
  if (ncc) CB_TRY(ncc_setup_scale(sel));
  std::vector<int> need(B, 0);
  bool any = false;
  for (int b = 0; b < B; ++b)
    if (sel[b] && state_of[b] != 1) { need[b] = 1; any = true; }
  if (any) CB_TRY(objective_at(v, need));
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(gradient(dact));
  CB_TRY(fetch_scalars());
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ps[b].gnorm = std::sqrt(hsc[S_GG * B + b]);
      ps[b].grad_evals++;
      ps[b].pde_solves++;
    }
  return 0;
}

int Solver::hessian_matvec(const float* vin, float* hout, const std::vector<int>& sel) {
  CB_TRY(gradient_at_current(sel));  // state, adjoint trajectory and caches for v
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(hessian_prep(dact));
  CB_TRY(apply_op(vin, hout, dact));
  if (cudaStreamSynchronize(stream) != cudaSuccess) return CB_ERR_CUDA;
  for (int b = 0; b < B; ++b)
    if (sel[b]) ps[b].hess_matvecs++;
  return 0;
}

int Solver::precond(const float* rin, float* zout, const std::vector<int>& sel) {
  if (opts.precond == CB_PC_TWOLEVEL) {
    // set up at the current velocity; coarse tolerance pctolscale * the
    // Krylov relative tolerance (-krylovtol), as outside a GN solve
    CB_TRY(gradient_at_current(sel));
    CB_TRY(twolevel_setup(sel));
    outer_rtol.assign(B, opts.krylovtol[0]);
    if (rin != r &&
        cudaMemcpyAsync(r, rin, sizeof(float) * 3 * n * B, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
    CB_TRY(upload_mask(sel, dact));
    CB_TRY(twolevel_apply(sel, dact, S_RZ));
    if (zout != z &&
        cudaMemcpyAsync(zout, z, sizeof(float) * 3 * n * B, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
  }
  CB_TRY(upload_mask(sel, dact));
  if (opts.precond) CB_TRY(reg_op(rin, zout, OP_REG_INV, EPI_STORE, dact));
  else CB_TRY(launch_lincomb(zout, 3 * n, rin, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, dact, stream));
  for (int b = 0; b < B; ++b)
    if (sel[b]) ps[b].pc_matvecs++;
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

int Solver::forward(const float* m0, float* m1, const std::vector<int>& sel) {
  // m0 / m1 are device arrays laid out like mT (problem stride n)
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(characteristic(v, 1.f, dact));
  CB_TRY(state_init(m0, dact));
  CB_TRY(state_steps(dact));
  CB_TRY(state_out(m1, n, dact));
  for (int b = 0; b < B; ++b)
    if (sel[b]) state_of[b] = 0;  // state now belongs to m0, not mT
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

int Solver::final_state(float* m1, int b) {
  if (state_of[b] != 1) {
    std::vector<int> sel(B, 0);
    sel[b] = 1;
    CB_TRY(objective_at(v, sel));
  }
  const long long PM = (nt + 1) * n;
  if (img16) {
    CB_TRY(launch_from_bf16(m16 + b * PM + nt * n, 0, 0, m1, 0, 0, n, 1, 1, nullptr, stream));
  } else if (cudaMemcpyAsync(m1, m + b * PM + nt * n, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream) !=
             cudaSuccess) {
    return CB_ERR_CUDA;
  }
  return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
}

// The INVREG preconditioner is the inverse of the regularisation operator, so
// for the full norms with beta1 > 0 Reg P = c I holds symbol by symbol
// (H1: hd beta0 (k^2 + beta1) / (beta0 (k^2 + beta1)) = hd; H2, H3, L2: 1;
// src/RegularizationH1.cpp:229 and :379-382, and likewise for the others).
// The seminorms drop the k = 0 modes from Reg and keep them in P, so there
// Reg P is not a multiple of the identity.
// Decided per problem, so a problem computes the same alone and in a batch.
void Solver::reg_recurrence(const std::vector<int>& sel, std::vector<double>& c) const {
  c.assign(B, 0.0);
  if (!reg_rec_enabled || opts.precond != CB_PC_INVREG || mv_kind != 0) return;
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    const ProbState& s = ps[b];
    if (!(s.beta0 > 0.0)) continue;
    if (s.norm == NORM_H1 && s.beta1 > 0.0) c[b] = (double)hd;
    else if ((s.norm == NORM_H2 || s.norm == NORM_H3) && s.beta1 > 0.0) c[b] = 1.0;
    else if (s.norm == NORM_L2) c[b] = 1.0;
  }
}

// ---------------------------------------------------------------------------
// PCG (KSPCG, unpreconditioned residual norm, zero initial guess;
// src/Optimizer.cpp:296-356)
//
// Where Reg P = c I (reg_recurrence) the regularisation part of q = H p is
// not transformed each iteration: with z = P r and p = z + beta p,
// Reg p = c r + beta Reg p, started from Reg p0 = Reg P r0 = c r0.  In exact
// arithmetic this is the same Reg p the spectral pass computes; it saves one
// 3-field forward and inverse transform per iteration.
// ---------------------------------------------------------------------------
int Solver::pcg(const std::vector<int>& sel, double maxit_d) {
  const int maxit = (int)maxit_d;
  int* act = dact2;
  CB_TRY(upload_mask(sel, act));
  std::vector<double> rc;
  reg_recurrence(sel, rc);
  std::vector<int> flag(B, 0);
  bool any_rec = false, any_norec = false;
  for (int b = 0; b < B; ++b) {
    flag[b] = rc[b] > 0.0;
    if (sel[b]) (flag[b] ? any_rec : any_norec) = true;
  }
  const bool rec = any_rec;
  const int mode = (any_rec ? 1 : 0) | (any_norec ? 2 : 0);
  int* dflag = dact + 8 * B;
  int* act_rec = dact + 9 * B;
  int* act_norec = dact + 10 * B;
  if (rec) {
    if (cudaMemcpyAsync(slot(S_RC), rc.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
    CB_TRY(upload_mask(flag, dflag));
  }
  if (pcg_exec && pcg_exec_mode != mode) {  // recorded for another mix of forms
    cudaGraphExecDestroy(pcg_exec);
    pcg_exec = nullptr;
  }
  auto split = [&]() {
    k_split_mask<<<pgrid(B), 128, 0, stream>>>(act, dflag, act_rec, act_norec, B);
    note_launches(1);
  };
  // r = -g, x = 0
  CB_TRY(launch_lincomb(r, 3 * n, g, 3 * n, nullptr, -1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
  CB_TRY(launch_lincomb(x, 3 * n, g, 3 * n, nullptr, 0.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
  note_launches(2);
  CB_TRY(dot(r, 3 * n, r, 3 * n, 3 * n, S_RR, act));
  k_pcg_init<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B, opts.krylovtol[1]);
  note_launches(1);
  // z = P r and r.z into slot s (the inverse transform's epilogue sums it)
  auto apply_pc = [&](int s) -> int {
    if (opts.precond) {
      CB_TRY(prof_mark(CB_PROF_PRECOND));
      CB_TRY(reg_op(r, z, OP_REG_INV, EPI_STORE, act, r, s));
      return prof_mark(CB_PROF_PRECOND);
    }
    note_launches(1);
    CB_TRY(launch_lincomb(z, 3 * n, r, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
    return dot(r, 3 * n, z, 3 * n, 3 * n, s, act);
  };
  CB_TRY(apply_pc(S_RZ));
  CB_TRY(launch_lincomb(pv, 3 * n, z, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
  note_launches(1);
  if (rec) {  // Reg p0 = c r0
    split();
    CB_TRY(launch_lincomb(sreg, 3 * n, r, 3 * n, slot(S_RC), 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act_rec,
                          stream));
    note_launches(1);
  }
  std::vector<int> hact(B);
  // One PCG iteration.  It reads and writes device data only (vectors, the
  // per-problem scalars and the active mask, which k_pcg_alpha / k_pcg_check
  // clear when a problem stops), so it is recorded once as a CUDA graph and
  // replayed, and several iterations can run between host checks.
  auto body = [&]() -> int {
    if (rec) {
      split();
      reg_in = sreg;
      rec_act = act_rec;
      norec_act = any_norec ? act_norec : nullptr;
    }
    CB_TRY(prof_mark(CB_PROF_HESSIAN));
    const int he = apply_op(pv, q, act, S_PQ);  // q = H p and p.q
    if (!he) CB_TRY(prof_mark(CB_PROF_HESSIAN));
    reg_in = nullptr;
    rec_act = norec_act = nullptr;
    CB_TRY(he);
    k_pcg_alpha<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B);
    // x += alpha p, r -= alpha q and the new r.r in one pass
    CB_TRY(launch_cg_update(x, r, pv, q, 3 * n, 3 * n, slot(S_ALPHA), B, partials, maxparts, act, stream));
    CB_TRY(launch_finalize(partials, maxparts, dot_partials(3 * n), slot(S_RR), B, 1.0, false, stream, act));
    k_pcg_check<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B, maxit, opts.krylovtol[2]);
    note_launches(4);
    CB_TRY(apply_pc(S_RZNEW));
    k_pcg_beta<<<pgrid(B), 128, 0, stream>>>(dsc, act, B);
    CB_TRY(launch_lincomb(pv, 3 * n, z, 3 * n, nullptr, 1.0, pv, 3 * n, slot(S_BETA), 1.0, 3 * n, B, act, stream));
    note_launches(2);
    if (rec) {  // Reg p = c r + beta Reg p
      split();
      CB_TRY(launch_lincomb(sreg, 3 * n, r, 3 * n, slot(S_RC), 1.0, sreg, 3 * n, slot(S_BETA), 1.0, 3 * n, B,
                            act_rec, stream));
      note_launches(1);
    }
    return 0;
  };
  auto run_body = [&]() -> int {
    if (!graphs || prof_on) return body();
    if (!pcg_exec) {
      if (!pcg_warm) {  // first run uncaptured: sets function attributes, builds FFT tables
        pcg_warm = true;
        return body();
      }
      const long long l0 = launches();
      g_graph_capture = true;
      cudaError_t ce = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
      int e = ce == cudaSuccess ? body() : CB_ERR_CUDA;
      cudaGraph_t gr = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(stream, &gr);
      g_graph_capture = false;
      pcg_exec_launches = launches() - l0;
      pcg_exec_mode = mode;
      if (!e && ee == cudaSuccess && gr && cudaGraphInstantiate(&pcg_exec, gr, 0) != cudaSuccess) pcg_exec = nullptr;
      if (gr) cudaGraphDestroy(gr);
      if (e || ee != cudaSuccess || !pcg_exec) {
        cudaGetLastError();
        graphs = false;  // fall back to direct launches for this solver
        return body();
      }
      // the recorded launches were not executed: replay them now
    }
    note_launches(pcg_exec_launches);
    return cudaGraphLaunch(pcg_exec, stream) == cudaSuccess ? 0 : CB_ERR_CUDA;
  };
  constexpr int kItersPerCheck = 2;
  int launched = 0;
  while (true) {
    if (cudaMemcpyAsync(hact.data(), act, sizeof(int) * B, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
      err = "device error in PCG";
      return CB_ERR_CUDA;
    }
    bool any = false;
    for (int b = 0; b < B; ++b) any |= hact[b] != 0;
    if (!any || launched >= maxit) break;
    for (int k = 0; k < kItersPerCheck && launched < maxit; ++k, ++launched) CB_TRY(run_body());
  }
  CB_TRY(fetch_scalars());
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    // Hessian applications: every iteration a problem entered active; an
    // iteration that stopped on indefinite curvature applied it without
    // counting; the preconditioner ran once up front and after every
    // iteration that did not stop
    const int its = hint[I_IT * B + b], reason = hint[I_REASON * B + b];
    const bool stopped_at_check = reason == 1 || reason == 2 || reason == 4;
    ps[b].hess_matvecs += its + (reason == 3 ? 1 : 0);
    ps[b].pc_matvecs += 1 + its - (stopped_at_check ? 1 : 0);
    ps[b].pcg_total += its;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Two-level preconditioner (-precond 2level: TWOLEVEL with PRECONDMATVECSYM,
// src/RegOpt.cpp:602-606; src/Preconditioner.cpp:323-1176,
// src/KrylovInterface.cpp:405-521).
//
// M r = L P y + (I - L) r with y the coarse solve of R L r, L the rectangular
// low-pass filter of ApplyRectFreqFilter at pct = nc / n, R / P the spectral
// restriction / prolongation.  For an even coarse size L keeps exactly the
// band R carries (|k| <= nc/2 - 1 on every axis), so R L = R and L P = P, and
// M r = r + P (y - R r): one restriction and one prolongation per application.
// ---------------------------------------------------------------------------
int Solver::ensure_wmask() {
  if (wmask) return 0;
  CB_TRY(alloc((void**)&wmask, sizeof(float) * n * B));
  CB_TRY(launch_fill(wmask, n, 1.f, n, B, nullptr, stream));
  return 0;
}

// CLAIRE::SetStateVariable / SetAdjointVariable (src/CLAIRE.cpp:599-725): both
// characteristics from the (restricted) velocity; then the caches the GN
// Hessian reads: grad m^j, div v, the adjoint step factor, (grad m^j)(X).
int Solver::prepare_from_state(const int* act) {
  CB_TRY(characteristic(v, 1.f, act));
  CB_TRY(characteristic(v, -1.f, act));
  CB_TRY(image_grad(act));
  CB_TRY(divergence(v, divv, act));
  CB_TRY(launch_adjoint_coef(divv, n, disp_adj, 3 * n, tab_adj, TP, cadj, n, ht, B, d, act, stream));
  note_launches(1);
  return hessian_prep(act);
}

int Solver::inner_solve(const std::vector<int>& sel, const std::vector<double>& rtol, int maxit) {
  if (cudaMemcpyAsync(slot(S_RTOL), rtol.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream) !=
      cudaSuccess)
    return CB_ERR_CUDA;
  return pcg(sel, maxit);
}

// Preconditioner::SetupCoarseGrid + ApplyRestriction (src/Preconditioner.cpp:
// 353-499, 676-831): coarse problems with every option of the fine ones but
// the grid; velocity, the nt+1 state levels (restricted, not re-solved) and
// the mask restricted from the selected problems' current ones; the current
// regularisation weights handed down.
int Solver::twolevel_setup(const std::vector<int>& sel) {
  if (!coarse) {
    coarse.reset(new (std::nothrow) Solver());
    if (!coarse) return CB_ERR_ALLOC;
    if (int e = coarse->init(coarse_opts(opts), B)) {
      err = "two-level preconditioner, coarse grid: " + coarse->err;
      coarse.reset();
      return e;
    }
    coarse->mv_kind = 2;
    coarse->graphs = graphs;
    if (wmask) CB_TRY(coarse->ensure_wmask());
  }
  Solver& c = *coarse;
  c.stream = stream;
  const long long need = grid_change_work(d.n1, nc1, std::max(3, nt + 1));
  if (gwork_floats < need) {
    if (gwork) {
      cudaFree(gwork);
      bytes_ -= (long long)sizeof(float) * gwork_floats;
      gwork = nullptr;
      gwork_floats = 0;
    }
    CB_TRY(alloc((void**)&gwork, sizeof(float) * need));
    gwork_floats = need;
  }
  const long long cn = c.n, PM = (nt + 1) * n, PMc = (nt + 1) * cn;
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    c.ps[b].norm = ps[b].norm;
    c.ps[b].beta0 = ps[b].beta0;
    c.ps[b].beta1 = ps[b].beta1;
    c.ps[b].beta2 = ps[b].beta2;
    if (launch_grid_change(v + b * 3 * n, n, d.n1, c.v + b * 3 * cn, cn, nc1, 3, gwork, stream) ||
        launch_grid_change(m + b * PM, n, d.n1, c.m + b * PMc, cn, nc1, nt + 1, gwork, stream) ||
        (wmask && launch_grid_change(wmask + b * n, n, d.n1, c.wmask + b * cn, cn, nc1, 1, gwork, stream)))
      return CB_ERR_CUDA;
    c.state_of[b] = 0;
  }
  note_launches(9);
  CB_TRY(c.upload_params());
  CB_TRY(c.upload_mask(sel, c.dact));
  return c.prepare_from_state(c.dact);
}

// Preconditioner::Apply2LevelPrecond (src/Preconditioner.cpp:584-673) on r,
// result in z.  The coarse solve is KSPCG without a preconditioner, zero
// initial guess, on the symmetric coarse operator divided by hd, with
// rtol = pctolscale * the outer forcing value in [1e-16, 1/2], atol 1e-16,
// dtol 1e6 and at most 1000 iterations (InvertPrecondPreKrylovSolve,
// src/KrylovInterface.cpp:430-521; SetupKrylovMethod, src/Preconditioner.cpp:
// 842-945).  Each coarse Hessian application counts as a preconditioner
// matvec (src/Preconditioner.cpp:980).
int Solver::twolevel_apply(const std::vector<int>& sel, const int* act, int rz_slot) {
  Solver& c = *coarse;
  const long long cn = c.n;
  for (int b = 0; b < B; ++b)
    if (sel[b] && launch_grid_change(r + b * 3 * n, n, d.n1, c.g + b * 3 * cn, cn, nc1, 3, gwork, stream))
      return CB_ERR_CUDA;
  // the coarse PCG starts from r = -g: g = -R r
  CB_TRY(c.upload_mask(sel, c.dact));
  CB_TRY(launch_lincomb(c.g, 3 * cn, c.g, 3 * cn, nullptr, -1.0, nullptr, 0, nullptr, 0.0, 3 * cn, B, c.dact,
                        stream));
  std::vector<double> rt(B, 0.5);
  std::vector<int> before(B, 0);
  for (int b = 0; b < B; ++b) {
    const double outer = b < (int)outer_rtol.size() ? outer_rtol[b] : opts.krylovtol[0];
    rt[b] = std::max(1e-16, std::min(0.5, opts.pctolscale * outer));
    before[b] = c.ps[b].hess_matvecs;
  }
  CB_TRY(c.inner_solve(sel, rt, 1000));
  // y - R r = x + g, prolonged; z = r + P (y - R r)
  CB_TRY(c.upload_mask(sel, c.dact));
  CB_TRY(launch_lincomb(c.x, 3 * cn, c.x, 3 * cn, nullptr, 1.0, c.g, 3 * cn, nullptr, 1.0, 3 * cn, B, c.dact,
                        stream));
  for (int b = 0; b < B; ++b)
    if (sel[b] && launch_grid_change(c.x + b * 3 * cn, cn, nc1, z + b * 3 * n, n, d.n1, 3, gwork, stream))
      return CB_ERR_CUDA;
  CB_TRY(launch_lincomb(z, 3 * n, z, 3 * n, nullptr, 1.0, r, 3 * n, nullptr, 1.0, 3 * n, B, act, stream));
  note_launches(9);
  CB_TRY(dot(r, 3 * n, z, 3 * n, 3 * n, rz_slot, act));
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ps[b].pc_matvecs += c.ps[b].hess_matvecs - before[b];
      if (opts.verbosity > 0)
        std::fprintf(stderr, "[claire_b200] p%d two-level coarse solve: %d iterations (rtol %.3e)\n", b,
                     c.ps[b].hess_matvecs - before[b], rt[b]);
    }
  return 0;
}

// KSPCG on the symmetrically preconditioned Hessian with the two-level
// preconditioner.  The iteration is pcg()'s; the preconditioner runs a nested
// Krylov solve driven from the host, so these iterations are direct launches
// with the active set read back before every preconditioner application.
int Solver::pcg_twolevel(const std::vector<int>& sel, double maxit_d) {
  const int maxit = (int)maxit_d;
  int* act = dact2;
  CB_TRY(upload_mask(sel, act));
  // PreKrylovSolve (src/KrylovInterface.cpp:79-196, src/CLAIREBase.cpp:936-952):
  // the right-hand side is the optimiser's gradient vector itself and becomes
  // P^1/2 g in place (the forcing value was taken from ||g|| before)
  CB_TRY(reg_op(g, g, OP_REG_SQRTINV, EPI_STORE, act));
  CB_TRY(launch_lincomb(r, 3 * n, g, 3 * n, nullptr, -1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
  CB_TRY(launch_lincomb(x, 3 * n, g, 3 * n, nullptr, 0.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
  note_launches(2);
  CB_TRY(dot(r, 3 * n, r, 3 * n, 3 * n, S_RR, act));
  k_pcg_init<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B, opts.krylovtol[1]);
  note_launches(1);
  // DoSetup at the first preconditioner application of every GN iteration
  // (src/KrylovInterface.cpp:444-447, reset by src/TaoInterface.cpp:546)
  CB_TRY(twolevel_setup(sel));
  std::vector<int> hact(B, 0);
  bool any = false;
  auto read_active = [&]() -> int {
    if (cudaMemcpyAsync(hact.data(), act, sizeof(int) * B, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
      err = "device error in PCG";
      return CB_ERR_CUDA;
    }
    any = false;
    for (int b = 0; b < B; ++b) any |= hact[b] != 0;
    return 0;
  };
  CB_TRY(read_active());
  if (any) {
    CB_TRY(twolevel_apply(hact, act, S_RZ));
    CB_TRY(launch_lincomb(pv, 3 * n, z, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, act, stream));
    note_launches(1);
  }
  for (int it = 0; it < maxit && any; ++it) {
    CB_TRY(apply_op(pv, q, act, S_PQ));  // q = A p and p.q
    k_pcg_alpha<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B);
    CB_TRY(launch_cg_update(x, r, pv, q, 3 * n, 3 * n, slot(S_ALPHA), B, partials, maxparts, act, stream));
    CB_TRY(launch_finalize(partials, maxparts, dot_partials(3 * n), slot(S_RR), B, 1.0, false, stream, act));
    k_pcg_check<<<pgrid(B), 128, 0, stream>>>(dsc, dint, act, B, maxit, opts.krylovtol[2]);
    note_launches(4);
    CB_TRY(read_active());
    if (!any) break;
    CB_TRY(twolevel_apply(hact, act, S_RZNEW));
    k_pcg_beta<<<pgrid(B), 128, 0, stream>>>(dsc, act, B);
    CB_TRY(launch_lincomb(pv, 3 * n, z, 3 * n, nullptr, 1.0, pv, 3 * n, slot(S_BETA), 1.0, 3 * n, B, act, stream));
    note_launches(2);
  }
  // PostKrylovSolve (src/CLAIREBase.cpp:958-972): x <- P^1/2 x
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(reg_op(x, x, OP_REG_SQRTINV, EPI_STORE, dact));
  CB_TRY(fetch_scalars());
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    const int its = hint[I_IT * B + b], reason = hint[I_REASON * B + b];
    ps[b].hess_matvecs += its + (reason == 3 ? 1 : 0);
    ps[b].pcg_total += its;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Armijo backtracking (PETSc TaoLineSearch "armijo": alpha0 = 1, beta = 1/2,
// sigma = 1e-4) on the step x; accepted problems get v <- v + alpha x.
// ---------------------------------------------------------------------------
int Solver::line_search(std::vector<int>& sel) {
  // descent test g.x < 0, else fall back to the steepest-descent direction
  CB_TRY(upload_mask(sel, dact));
  CB_TRY(dot(g, 3 * n, x, 3 * n, 3 * n, S_GD, dact));
  CB_TRY(fetch_scalars());
  std::vector<double> gd(B, 0.0), alpha(B, 1.0);
  std::vector<int> fallback(B, 0);
  bool anyfb = false;
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    gd[b] = hsc[S_GD * B + b];
    if (!(gd[b] < 0.0)) {
      fallback[b] = 1;
      anyfb = true;
    }
  }
  if (anyfb) {
    // direction -g, slope -|g|^2 of the gradient vector the solve left in g
    // (P^1/2 g with the two-level preconditioner's PreKrylovSolve)
    CB_TRY(upload_mask(fallback, dact + 3 * B));
    CB_TRY(dot(g, 3 * n, g, 3 * n, 3 * n, S_GG, dact + 3 * B));
    CB_TRY(fetch_scalars());
    for (int b = 0; b < B; ++b)
      if (fallback[b]) gd[b] = -hsc[S_GG * B + b];
    CB_TRY(launch_lincomb(x, 3 * n, g, 3 * n, nullptr, -1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, dact + 3 * B, stream));
    note_launches(1);
  }
  std::vector<int> trial = sel, accepted(B, 0);
  const int max_trials = 30;
  const double sigma = 1e-4;
  for (int t = 0; t < max_trials; ++t) {
    bool any = false;
    for (int b = 0; b < B; ++b) any |= (trial[b] != 0);
    if (!any) break;
    // vtrial = v + alpha x  (alpha per problem through S_ALPHA)
    std::vector<double> al(B, 0.0);
    for (int b = 0; b < B; ++b) al[b] = alpha[b];
    // pageable source: the copy is staged before the call returns
    if (cudaMemcpyAsync(slot(S_ALPHA), al.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
    CB_TRY(upload_mask(trial, dact + 6 * B));
    CB_TRY(launch_lincomb(vtrial, 3 * n, v, 3 * n, nullptr, 1.0, x, 3 * n, slot(S_ALPHA), 1.0, 3 * n, B,
                          dact + 6 * B, stream));
    note_launches(1);
    std::vector<double> J0(B);
    for (int b = 0; b < B; ++b) J0[b] = ps[b].J;
    std::vector<double> D0(B), R0(B);
    for (int b = 0; b < B; ++b) { D0[b] = ps[b].D; R0[b] = ps[b].R; }
    CB_TRY(objective_at(vtrial, trial));
    for (int b = 0; b < B; ++b) {
      if (!trial[b]) continue;
      const double Jt = ps[b].J;
      if (std::isfinite(Jt) && Jt <= J0[b] + sigma * alpha[b] * gd[b]) {
        accepted[b] = 1;
        trial[b] = 0;
        ps[b].step = alpha[b];
      } else {
        // restore the monitor values of the current iterate
        ps[b].J = J0[b];
        ps[b].D = D0[b];
        ps[b].R = R0[b];
        alpha[b] *= 0.5;
      }
    }
  }
  for (int b = 0; b < B; ++b)
    if (trial[b]) {  // line search failed
      sel[b] = 0;
      ps[b].done = true;
      ps[b].reason = 5;
    }
  bool anyacc = false;
  for (int b = 0; b < B; ++b) anyacc |= (accepted[b] != 0);
  if (anyacc) {
    CB_TRY(upload_mask(accepted, dact + 7 * B));
    CB_TRY(launch_lincomb(v, 3 * n, vtrial, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, dact + 7 * B,
                          stream));
    note_launches(1);
    for (int b = 0; b < B; ++b)
      if (accepted[b]) state_of[b] = 1;  // the state was computed at vtrial == new v
  }
  for (int b = 0; b < B; ++b) sel[b] = accepted[b];
  return 0;
}

// ---------------------------------------------------------------------------
// GN loop with CLAIRE's stopping test (src/TaoInterface.cpp:391-527)
// ---------------------------------------------------------------------------
// InitializeOptimization (src/CLAIRE.cpp:227-357) for the selected problems:
// J0, D0, ||g0|| at the current velocity; the problems join the GN loop.
int Solver::begin(const std::vector<int>& sel) {
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ProbState keep = ps[b];
      ps[b] = ProbState();
      ps[b].norm = keep.norm;
      ps[b].model = keep.model;
      ps[b].beta0 = keep.beta0;
      ps[b].beta1 = keep.beta1;
      ps[b].beta2 = keep.beta2;
      ps[b].running = true;
      ps[b].t0 = std::chrono::steady_clock::now();
      if ((int)carry_krylov_g0.size() == B) ps[b].krylov_g0 = carry_krylov_g0[b];
      state_of[b] = 0;
    }
  // InitializeOptimization (src/CLAIRE.cpp:227-357): D0, J0 and ||g0|| at the
  // zero velocity; a nonzero initial guess is set aside meanwhile and the GN
  // loop then starts from it.
  CB_TRY(upload_mask(sel, dact2));
  CB_TRY(dot(v, 3 * n, v, 3 * n, 3 * n, S_GD, dact2));
  CB_TRY(fetch_scalars());
  std::vector<int> guess(B, 0);
  bool any_guess = false;
  for (int b = 0; b < B; ++b)
    if (sel[b] && hsc[S_GD * B + b] > 0.0) { guess[b] = 1; any_guess = true; }
  if (any_guess) {
    CB_TRY(upload_mask(guess, dact2));
    CB_TRY(launch_lincomb(x, 3 * n, v, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, dact2, stream));
    CB_TRY(launch_fill(v, 3 * n, 0.f, 3 * n, B, dact2, stream));
    note_launches(2);
  }
  CB_TRY(objective_at(v, sel));
  CB_TRY(gradient_at_current(sel));
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ps[b].J0 = ps[b].J;
      ps[b].D0 = ps[b].D;
      ps[b].gnorm0 = ps[b].gnorm > 0.0 ? ps[b].gnorm : 1.0;
    }
  if (any_guess) {
    CB_TRY(upload_mask(guess, dact2));
    CB_TRY(launch_lincomb(v, 3 * n, x, 3 * n, nullptr, 1.0, nullptr, 0, nullptr, 0.0, 3 * n, B, dact2, stream));
    note_launches(1);
    for (int b = 0; b < B; ++b)
      if (guess[b]) state_of[b] = 0;
    CB_TRY(objective_at(v, guess));
    CB_TRY(gradient_at_current(guess));
  }
  return 0;
}

// One GN iteration (src/Optimizer.cpp:257-445) of every running problem that
// has not met a stopping test (src/TaoInterface.cpp:391-527).  Problems that
// stop are listed in `finished` (running, done, final values pending).
int Solver::step(std::vector<int>& finished, double gttol, int miniter) {
  finished.assign(B, 0);
  if (gttol < 0) gttol = opts.opttol;
  const double gatol = opts.gatol, minstep = 1.0 / 1024.0;
  std::vector<int> act(B, 0);
  bool any = false;
  for (int b = 0; b < B; ++b) {
    if (!ps[b].running || ps[b].done) continue;
    ProbState& s = ps[b];
    // step / gradient tests only from iteration miniter on (src/TaoInterface.cpp:438-470)
    const bool tests = s.iter >= miniter;
    if (!std::isfinite(s.J) || !std::isfinite(s.gnorm)) { s.done = true; s.reason = -1; }
    else if (tests && s.step < minstep) { s.done = true; s.reason = 4; }
    else if (tests && s.gnorm < gttol * s.gnorm0) { s.done = true; s.reason = 1; }
    else if (tests && s.gnorm < gatol) { s.done = true; s.reason = 2; }
    else if (s.iter > opts.maxit - 1) { s.done = true; s.reason = 3; }
    if (s.done) { finished[b] = 1; continue; }
    act[b] = 1;
    any = true;
  }
  if (!any) return 0;
  // forcing sequence (src/KrylovInterface.cpp:134-165)
  std::vector<double> rtol(B, opts.krylovtol[0]);
  for (int b = 0; b < B; ++b) {
    if (!act[b]) continue;
    ProbState& s = ps[b];
    if (opts.krylovfseq != CB_FSEQ_NONE) {
      if (s.krylov_g0 < 0) s.krylov_g0 = s.gnorm;
      const double gr = s.gnorm / s.krylov_g0;
      double rt = (opts.krylovfseq == CB_FSEQ_QUADRATIC) ? gr : std::sqrt(gr);
      rt = std::max(1e-16, std::min(0.5, rt));
      rtol[b] = rt;
    }
  }
  if (cudaMemcpyAsync(slot(S_RTOL), rtol.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return CB_ERR_CUDA;
  outer_rtol = rtol;
  CB_TRY(upload_mask(act, dact));
  CB_TRY(hessian_prep(dact));
  if (opts.precond == CB_PC_TWOLEVEL) CB_TRY(pcg_twolevel(act, std::max(0, opts.krylovmaxit - 1)));
  else CB_TRY(pcg(act, std::max(0, opts.krylovmaxit - 1)));
  std::vector<int> acc = act;
  CB_TRY(line_search(acc));
  bool anyacc = false;
  for (int b = 0; b < B; ++b) anyacc |= (acc[b] != 0);
  if (anyacc) CB_TRY(gradient_at_current(acc));
  for (int b = 0; b < B; ++b)
    if (acc[b]) ps[b].iter++;
  CB_TRY(check_stage());
  if (opts.verbosity > 0) {
    // OptimizationMonitor line (src/TaoInterface.cpp:529-606)
    for (int b = 0; b < B; ++b)
      if (act[b])
        std::fprintf(stderr, "[claire_b200] p%d it %d J/J0 %.6e D/D0 %.6e |g|/|g0| %.6e pcg %d reason %d step %.3e\n",
                     b, ps[b].iter, ps[b].J / ps[b].J0, ps[b].D / ps[b].D0, ps[b].gnorm / ps[b].gnorm0,
                     hint[I_IT * B + b], hint[I_REASON * B + b], ps[b].step);
  }
  return 0;
}

// Final relative mismatch ||mR - m1|| / ||mR - mT|| (src/CLAIRE.cpp:4232-4262)
// of the selected problems; they leave the GN loop.
int Solver::finish(const std::vector<int>& sel) {
  std::vector<int> need(B, 0);
  bool anyneed = false, anysel = false;
  for (int b = 0; b < B; ++b) {
    anysel |= sel[b] != 0;
    if (sel[b] && state_of[b] != 1) { need[b] = 1; anyneed = true; }
  }
  if (!anysel) return 0;
  if (anyneed) CB_TRY(objective_at(v, need));
  CB_TRY(upload_mask(sel, dact));
  const int np = dot_partials(n);
  CB_TRY(image_diff_sumsq(false, dact));
  CB_TRY(launch_finalize(partials, maxparts, np, slot(S_PQ), B, 1.0, false, stream, dact));
  CB_TRY(image_diff_sumsq(true, dact));
  CB_TRY(launch_finalize(partials, maxparts, np, slot(S_RR), B, 1.0, false, stream, dact));
  note_launches(2);
  CB_TRY(fetch_scalars());
  CB_TRY(check_stage());
  const auto t1 = std::chrono::steady_clock::now();
  for (int b = 0; b < B; ++b) {
    if (!sel[b]) continue;
    const double num = std::sqrt(hsc[S_PQ * B + b]), den = std::sqrt(hsc[S_RR * B + b]);
    ps[b].rel_mismatch = den > 0 ? num / den : num;
    ps[b].seconds = std::chrono::duration<double>(t1 - ps[b].t0).count();
    ps[b].running = false;
    ps[b].done = true;
  }
  return 0;
}

// Regularisation-parameter continuation (CLAIREInterface::RunSolverRegParaContReduction,
// src/CLAIREInterface.cpp:1300-1376): J0 and ||g0|| at beta = 1 (:1324-1331);
// levels beta = 1, 1/10, ... while beta > beta*, each a GN solve to the
// presolve tolerance warm-started from the previous level (Optimizer::Run with
// presolve, src/Optimizer.cpp:451-494; at least one iteration per level,
// src/RegOpt.cpp:757-760); then the solve at beta* to opttol.  The Krylov
// forcing reference ||g|| is set once (src/KrylovInterface.cpp:125-139).
int Solver::run_betacont(const std::vector<int>& sel, double beta_star, double presolve_gttol) {
  if (!(beta_star > 0.0 && beta_star < 1.0)) {
    err = "target beta not in (0,1)";
    return CB_ERR_ARG;
  }
  auto set_beta = [&](double beta) -> int {
    for (int b = 0; b < B; ++b)
      if (sel[b]) ps[b].beta0 = beta;
    return upload_params();
  };
  auto level = [&](double gttol) -> int { return solve_level(sel, gttol); };
  double beta = 1.0;
  CB_TRY(set_beta(beta));
  CB_TRY(begin(sel));
  while (beta > beta_star) {
    CB_TRY(level(presolve_gttol));
    beta /= 10.0;
    CB_TRY(set_beta(beta));
  }
  CB_TRY(set_beta(beta_star));
  CB_TRY(level(opts.opttol));
  return finish(sel);
}

int Solver::solve_level(const std::vector<int>& sel, double gttol) {
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ps[b].iter = 0;
      ps[b].done = false;
      ps[b].running = true;
      ps[b].reason = 0;
      ps[b].step = 1.0;
      state_of[b] = 0;  // the objective changed with beta
    }
  CB_TRY(objective_at(v, sel));
  CB_TRY(gradient_at_current(sel));
  std::vector<int> fin;
  while (true) {
    bool running = false;
    for (int b = 0; b < B; ++b) running |= sel[b] && ps[b].running && !ps[b].done;
    if (!running) break;
    CB_TRY(step(fin, gttol, 1));
  }
  return 0;
}

// Regularisation-parameter searches of CLAIREInterface (src/CLAIREInterface.cpp):
// RunSolverRegParaContBinarySearch (:955-1186) and ReductSearch (:1192-1285).
// ||g0|| comes from one initialisation at beta = -betainit and v = 0; every
// solve starts from the last solution whose det(grad y) stayed inside the
// bound (CheckBounds, src/CLAIREBase.cpp:1386-1445: min J <= jbound or
// 1 / max J <= jbound is a breach); a solve counts as converged unless it
// ended on a line-search failure or NaN (Optimizer::GetSolutionStatus,
// src/Optimizer.cpp:557-580).  Constants of src/RegOpt.hpp:337-343: beta is
// scaled by 1/10 per step, at most 10 steps, down to 1e-4 (H1 types) or
// 1e-7 (H2 types); the bisection stops when |dbeta| < 1e-2 beta*.  The
// reported solution is the last valid one, with beta* in the stats.
int Solver::run_train(const std::vector<int>& sel, int strategy) {
  constexpr double kScale = 1e-1, kDScale = 1e-2;
  constexpr int kMaxSteps = 10, kMaxSolves = 64;  // kMaxSolves: guard against endless re-lifting
  std::vector<double> det_keep((size_t)3 * B, 0.0);
  float* best = nullptr;
  if (cudaMalloc((void**)&best, sizeof(float) * 3 * n) != cudaSuccess) return CB_ERR_ALLOC;
  struct Free {
    float* p;
    ~Free() { cudaFree(p); }
  } free_best{best};
  for (int pb = 0; pb < B; ++pb) {
    if (!sel[pb]) continue;
    std::vector<int> one(B, 0);
    one[pb] = 1;
    const int norm = ps[pb].norm;
    const double betamin =
        (norm == NORM_H1 || norm == NORM_H1SN) ? 1e-4 : ((norm == NORM_H2 || norm == NORM_H2SN) ? 1e-7 : 1e-9);
    float* vb = v + pb * 3 * n;
    auto set_beta = [&](double beta) -> int {
      ps[pb].beta0 = beta;
      return upload_params();
    };
    auto save_best = [&]() -> int {
      return cudaMemcpyAsync(best, vb, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess
                 ? 0 : CB_ERR_CUDA;
    };
    auto load_best = [&]() -> int {
      state_of[pb] = 0;
      return cudaMemcpyAsync(vb, best, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess
                 ? 0 : CB_ERR_CUDA;
    };
    // one solve at beta from the best solution: converged, bound reached
    int solves = 0;
    double best_det[3] = {0.0, 0.0, 0.0};  // det(grad y) of the last valid solution
    auto solve = [&](double beta, bool& converged, bool& breach) -> int {
      ++solves;
      CB_TRY(set_beta(beta));
      CB_TRY(load_best());
      CB_TRY(solve_level(one, opts.opttol));
      converged = ps[pb].reason != 5 && ps[pb].reason != -1;
      std::vector<double> st;
      CB_TRY(det_def_grad(one, false, st));
      breach = st[3 * pb] <= opts.jbound || 1.0 / st[3 * pb + 2] <= opts.jbound;
      if (!breach)
        for (int k = 0; k < 3; ++k) best_det[k] = st[3 * pb + k];
      return 0;
    };
    double beta = opts.betainit, betastar = beta;
    CB_TRY(set_beta(beta));
    CB_TRY(begin(one));  // InitializeOptimization at beta0, v = initial guess
    CB_TRY(save_best());
    bool converged = true, breach = false;
    for (int level = 0; level < kMaxSteps && solves < kMaxSolves; ++level) {
      CB_TRY(solve(beta, converged, breach));
      if (strategy == CB_TRAIN_BINARY && !converged && level > 0) break;
      if (breach) {
        if (strategy == CB_TRAIN_REDUCE || level > 0) break;
        beta /= kScale;  // bound reached with the first beta: lift it
        level = -1;
      } else {
        betastar = beta;
        CB_TRY(save_best());
        beta *= kScale;
      }
      if (beta < betamin) break;
    }
    if (strategy == CB_TRAIN_BINARY) {
      double betahat = kScale * betastar;
      double dbeta = (betastar - betahat) / 2.0;
      beta = betastar - dbeta;
      const double dbetamin = kDScale * betastar;
      bool stop = false;
      while (!stop && solves < kMaxSolves) {
        CB_TRY(solve(beta, converged, breach));
        if (converged && !breach) {
          betastar = beta;
          CB_TRY(save_best());
        } else {
          betahat = beta;
        }
        dbeta = (betastar - betahat) / 2.0;
        beta = betastar - dbeta;
        if (std::fabs(dbeta) < dbetamin) stop = true;
      }
    }
    // Finalize(m_Solution): the last valid solution at beta*
    CB_TRY(set_beta(betastar));
    CB_TRY(load_best());
    for (int k = 0; k < 3; ++k) det_keep[(size_t)3 * pb + k] = best_det[k];
  }
  CB_TRY(finish(sel));
  for (int b = 0; b < B; ++b)
    if (sel[b])
      for (int k = 0; k < 3; ++k) ps[b].det[k] = det_keep[(size_t)3 * b + k];
  return 0;
}

// RunSolver with -monitordefgrad (src/CLAIREInterface.cpp:790-862): after a
// solve from the initial guess, CheckBounds; while breached (at most 10
// times) beta moves halfway toward beta* = 10 beta (RegNorm.beta[3] is never
// set, :806-810) and the problem is solved again from the initial guess.
// solution_status 0: the first solution kept the bound, 1: a raised beta
// did, 2: none did (beta is then reported as beta*).
int Solver::run_monitored(const std::vector<int>& sel) {
  float* guess = nullptr;
  if (cudaMalloc((void**)&guess, sizeof(float) * 3 * n) != cudaSuccess) return CB_ERR_ALLOC;
  struct Free {
    float* p;
    ~Free() { cudaFree(p); }
  } free_guess{guess};
  std::vector<double> det_keep((size_t)3 * B, 0.0);
  std::vector<int> status(B, 0);
  for (int pb = 0; pb < B; ++pb) {
    if (!sel[pb]) continue;
    std::vector<int> one(B, 0);
    one[pb] = 1;
    float* vb = v + pb * 3 * n;
    if (cudaMemcpyAsync(guess, vb, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return CB_ERR_CUDA;
    double beta = ps[pb].beta0;
    const double betastar = beta / 1e-1;
    CB_TRY(begin(one));  // InitializeOptimization once, at the first beta
    bool breach = true;
    int level = 0;
    std::vector<double> st;
    while (breach && level < 10) {
      if (cudaMemcpyAsync(vb, guess, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        return CB_ERR_CUDA;
      state_of[pb] = 0;
      CB_TRY(solve_level(one, opts.opttol));
      CB_TRY(det_def_grad(one, false, st));
      breach = st[3 * pb] <= opts.jbound || 1.0 / st[3 * pb + 2] <= opts.jbound;
      if (breach) {
        beta += (betastar - beta) / 2.0;
        ps[pb].beta0 = beta;
        CB_TRY(upload_params());
        ++level;
      }
    }
    status[pb] = level == 0 ? 0 : (breach ? 2 : 1);
    if (status[pb] == 2) {
      ps[pb].beta0 = betastar;
      CB_TRY(upload_params());
    }
    for (int k = 0; k < 3; ++k) det_keep[(size_t)3 * pb + k] = st[3 * pb + k];
  }
  CB_TRY(finish(sel));
  for (int b = 0; b < B; ++b)
    if (sel[b]) {
      ps[b].solution_status = status[b];
      for (int k = 0; k < 3; ++k) ps[b].det[k] = det_keep[(size_t)3 * b + k];
    }
  return 0;
}

int Solver::run(const std::vector<int>& sel) {
  if (opts.betacont > 0.0) return run_betacont(sel, opts.betacont, opts.presolvetol);
  CB_TRY(begin(sel));
  std::vector<int> fin;
  while (true) {
    bool running = false;
    for (int b = 0; b < B; ++b) running |= sel[b] && ps[b].running && !ps[b].done;
    if (!running) break;
    CB_TRY(step(fin));
  }
  return finish(sel);
}

}  // namespace cb
