// extern "C" boundary of libclaire_b200.so (declared in include/claire_b200.h).
//
// The context functions mirror reg::CLAIREInterface / reg::RegOpt
// (include/CLAIREInterface.hpp:42-90, include/RegOpt.hpp:475-635); the
// operator functions mirror the inner seams SemiLagrangian, Regularization,
// DistanceMeasureSL2 and the AccFFT spectral calls so each piece can be
// swapped and tested on its own.  No exception crosses the ABI.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/claire_b200.h"
#include "reduce.cuh"
#include "sl.cuh"
#include "solver.cuh"
#include "spectral.cuh"

namespace cb {
static std::atomic<long long> g_launches{0};
void note_launches(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace cb

using namespace cb;

struct claire_b200_ctx {
  Solver solver;
  std::string last_error;
};

static int cuda_status(int e) { return e == 0 ? CB_OK : (e < 0 ? e : CB_ERR_CUDA); }

extern "C" {

int claire_b200_default_opts(claire_b200_opts* o) {
  if (!o) return CB_ERR_ARG;
  std::memset(o, 0, sizeof(*o));
  o->nx[0] = o->nx[1] = o->nx[2] = 32;
  o->nt = 4;
  o->regnorm = CB_NORM_H1SN;
  // RegOpt::Initialize defaults to RELAXEDSTOKES when -regnorm is absent
  // (src/RegOpt.cpp:1066); every -regnorm choice selects COMPRESSIBLE.
  o->model = CB_MODEL_RELAXEDSTOKES;
  o->beta[0] = 1e-2;
  o->beta[1] = 1e-4;
  o->beta[2] = 1e-4;
  o->maxit = 50;
  o->opttol = 5e-2;
  o->gatol = 1e-6;
  o->krylovmaxit = 50;
  o->krylovtol[0] = 1e-12;
  o->krylovtol[1] = 1e-16;
  o->krylovtol[2] = 1e6;
  o->krylovfseq = CB_FSEQ_SUPERLINEAR;
  o->betacont = 0.0;
  o->presolvetol = 1e-1;  // src/RegOpt.cpp:1172
  o->precond = 1;
  o->iporder = 3;
  o->verbosity = 0;
  o->bf16_images = 0;
  o->autotune = 0;
  o->distance = CB_DIST_SL2;  // src/RegOpt.cpp:1079
  o->scalecont = 0;
  o->gridcont = 0;
  o->train = CB_TRAIN_OFF;
  o->jbound = 2.5e-1;  // src/RegOpt.cpp:1254
  o->betainit = 1.0;   // src/RegOpt.cpp:1228
  o->monitordefgrad = 0;
  o->pcgridscale = 2.0;   // src/RegOpt.cpp:1124
  o->pctolscale = 1e-1;   // src/RegOpt.cpp:1121
  o->pcsolvermaxit = 10;  // src/RegOpt.cpp:1123
  return CB_OK;
}

int claire_b200_parse_args(claire_b200_opts* o, int argc, const char* const* argv) {
  if (!o || (argc > 0 && !argv)) return CB_ERR_ARG;
  for (int i = 0; i < argc; ++i) {
    const char* a = argv[i];
    auto next = [&](const char** val) -> int {
      if (i + 1 >= argc) return CB_ERR_ARG;
      *val = argv[++i];
      return CB_OK;
    };
    const char* val = nullptr;
    if (!std::strcmp(a, "-nx")) {
      if (next(&val)) return CB_ERR_ARG;
      int v[3] = {0, 0, 0};
      int cnt = std::sscanf(val, "%dx%dx%d", &v[0], &v[1], &v[2]);
      if (cnt == 1) v[1] = v[2] = v[0];
      else if (cnt != 3) return CB_ERR_ARG;
      for (int k = 0; k < 3; ++k) o->nx[k] = v[k];
    } else if (!std::strcmp(a, "-nt")) {
      if (next(&val)) return CB_ERR_ARG;
      o->nt = std::atoi(val);
    } else if (!std::strcmp(a, "-regnorm")) {
      if (next(&val)) return CB_ERR_ARG;
      o->model = CB_MODEL_COMPRESSIBLE;
      if (!std::strcmp(val, "h1s")) o->regnorm = CB_NORM_H1SN;
      else if (!std::strcmp(val, "h2s")) o->regnorm = CB_NORM_H2SN;
      else if (!std::strcmp(val, "h3s")) o->regnorm = CB_NORM_H3SN;
      else if (!std::strcmp(val, "h1")) o->regnorm = CB_NORM_H1;
      else if (!std::strcmp(val, "h2")) o->regnorm = CB_NORM_H2;
      else if (!std::strcmp(val, "h3")) o->regnorm = CB_NORM_H3;
      else if (!std::strcmp(val, "l2")) o->regnorm = CB_NORM_L2;
      else if (!std::strcmp(val, "h1s-div")) { o->regnorm = CB_NORM_H1SN; o->model = CB_MODEL_RELAXEDSTOKES; }
      else if (!std::strcmp(val, "h1s-stokes")) { o->regnorm = CB_NORM_H1SN; o->model = CB_MODEL_STOKES; }
      else return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-beta")) {
      if (next(&val)) return CB_ERR_ARG;
      o->beta[0] = std::atof(val);
    } else if (!std::strcmp(a, "-beta-div")) {
      if (next(&val)) return CB_ERR_ARG;
      o->beta[2] = std::atof(val);
    } else if (!std::strcmp(a, "-maxit")) {
      if (next(&val)) return CB_ERR_ARG;
      o->maxit = std::atoi(val);
    } else if (!std::strcmp(a, "-opttol")) {
      if (next(&val)) return CB_ERR_ARG;
      o->opttol = std::atof(val);
    } else if (!std::strcmp(a, "-gabs")) {
      if (next(&val)) return CB_ERR_ARG;
      o->gatol = std::atof(val);
    } else if (!std::strcmp(a, "-krylovmaxit")) {
      if (next(&val)) return CB_ERR_ARG;
      o->krylovmaxit = std::atoi(val);
    } else if (!std::strcmp(a, "-krylovtol")) {
      if (next(&val)) return CB_ERR_ARG;
      o->krylovtol[0] = std::atof(val);
    } else if (!std::strcmp(a, "-betacont")) {
      // src/RegOpt.cpp:755-765
      if (next(&val)) return CB_ERR_ARG;
      o->betacont = std::atof(val);
    } else if (!std::strcmp(a, "-krylovfseq")) {
      if (next(&val)) return CB_ERR_ARG;
      if (!std::strcmp(val, "none")) o->krylovfseq = CB_FSEQ_NONE;
      else if (!std::strcmp(val, "quadratic")) o->krylovfseq = CB_FSEQ_QUADRATIC;
      else if (!std::strcmp(val, "suplinear")) o->krylovfseq = CB_FSEQ_SUPERLINEAR;
      else return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-precond")) {
      if (next(&val)) return CB_ERR_ARG;
      // src/RegOpt.cpp:592-611
      if (!std::strcmp(val, "none")) o->precond = CB_PC_NONE;
      else if (!std::strcmp(val, "invreg")) o->precond = CB_PC_INVREG;
      else if (!std::strcmp(val, "2level")) o->precond = CB_PC_TWOLEVEL;
      else return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-gridscale")) {
      if (next(&val)) return CB_ERR_ARG;
      o->pcgridscale = std::atof(val);  // src/RegOpt.cpp:612-614
      if (!(o->pcgridscale >= 1.0)) return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-pcsolver")) {
      // src/RegOpt.cpp:615-631: the coarse solve runs KSPCG; the flexible and
      // Chebyshev solvers are not on this path
      if (next(&val)) return CB_ERR_ARG;
      if (std::strcmp(val, "pcg")) {
        if (!std::strcmp(val, "fpcg") || !std::strcmp(val, "gmres") || !std::strcmp(val, "fgmres") ||
            !std::strcmp(val, "cheb"))
          return CB_ERR_UNSUPPORTED;
        return CB_ERR_ARG;
      }
    } else if (!std::strcmp(a, "-pctolscale")) {
      if (next(&val)) return CB_ERR_ARG;
      o->pctolscale = std::atof(val);  // src/RegOpt.cpp:645-647, checked at :1696-1700
      if (!(o->pctolscale >= 0.0 && o->pctolscale < 1.0)) return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-pcsolvermaxit")) {
      if (next(&val)) return CB_ERR_ARG;
      o->pcsolvermaxit = std::atoi(val);  // src/RegOpt.cpp:648-650
    } else if (!std::strcmp(a, "-monitorpcsolver")) {
      // src/RegOpt.cpp:643-644: prints the coarse solver's residuals (here:
      // its iteration count per application at -verbosity > 0)
    } else if (!std::strcmp(a, "-iporder")) {
      if (next(&val)) return CB_ERR_ARG;
      o->iporder = std::atoi(val);
      if (o->iporder != 3) return CB_ERR_UNSUPPORTED;
    } else if (!std::strcmp(a, "-distance")) {
      // src/RegOpt.cpp:680-690
      if (next(&val)) return CB_ERR_ARG;
      if (!std::strcmp(val, "sl2")) o->distance = CB_DIST_SL2;
      else if (!std::strcmp(val, "ncc")) o->distance = CB_DIST_NCC;
      else return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-train")) {
      // src/RegOpt.cpp:730-755; a search runs at least one GN iteration per solve
      if (next(&val)) return CB_ERR_ARG;
      if (o->betacont > 0.0) return CB_ERR_ARG;  // no training and continuation together
      if (!std::strcmp(val, "binary")) o->train = CB_TRAIN_BINARY;
      else if (!std::strcmp(val, "reduce")) o->train = CB_TRAIN_REDUCE;
      else return CB_ERR_ARG;
    } else if (!std::strcmp(a, "-monitordefgrad")) {
      o->monitordefgrad = 1;  // src/RegOpt.cpp:779-780
    } else if (!std::strcmp(a, "-jbound")) {
      if (next(&val)) return CB_ERR_ARG;
      o->jbound = std::atof(val);  // src/RegOpt.cpp:551-553
    } else if (!std::strcmp(a, "-betainit")) {
      if (next(&val)) return CB_ERR_ARG;
      o->betainit = std::atof(val);  // src/RegOpt.cpp:767-769
    } else if (!std::strcmp(a, "-scalecont")) {
      o->scalecont = 1;  // src/RegOpt.cpp:769-770
    } else if (!std::strcmp(a, "-gridcont")) {
      o->gridcont = 1;  // src/RegOpt.cpp:771-772
    } else if (!std::strcmp(a, "-autotune")) {
      o->autotune = 1;
    } else if (!std::strcmp(a, "-bf16images")) {
      o->bf16_images = 1;  // no reference counterpart: bf16 storage of the image volumes
    } else if (!std::strcmp(a, "-verbosity")) {
      if (next(&val)) return CB_ERR_ARG;
      o->verbosity = std::atoi(val);
    } else if (!std::strcmp(a, "-disablesmoothing") || !std::strcmp(a, "-synthetic")) {
      if (!std::strcmp(a, "-synthetic") && i + 1 < argc && argv[i + 1][0] != '-') ++i;
    } else {
      return CB_ERR_ARG;
    }
  }
  return CB_OK;
}

long long claire_b200_estimate_bytes(const claire_b200_opts* o, int nbatch) {
  if (!o) return -1;
  return Solver::estimate_bytes(*o, nbatch);
}

int claire_b200_create(const claire_b200_opts* o, int nbatch, claire_b200_ctx** out) {
  if (!o || !out) return CB_ERR_ARG;
  *out = nullptr;
  claire_b200_ctx* c = new (std::nothrow) claire_b200_ctx();
  if (!c) return CB_ERR_ALLOC;
  int e = c->solver.init(*o, nbatch);
  if (e) {
    delete c;
    return e < 0 ? e : CB_ERR_CUDA;
  }
  *out = c;
  return CB_OK;
}

int claire_b200_destroy(claire_b200_ctx* c) {
  delete c;
  return CB_OK;
}

const char* claire_b200_last_error(const claire_b200_ctx* c) {
  if (!c) return "null context";
  return c->solver.err.c_str();
}

long long claire_b200_footprint_bytes(const claire_b200_ctx* c) { return c ? c->solver.footprint() : -1; }

int claire_b200_set_problem_opts(claire_b200_ctx* c, int b, const claire_b200_opts* o) {
  if (!c || !o) return CB_ERR_ARG;
  return c->solver.set_problem(b, *o);
}

static int copy_in(Solver& s, float* dst, const float* src, long long count, int on_device) {
  cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(float) * count,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s.stream);
  if (e != cudaSuccess) return CB_ERR_CUDA;
  return cudaStreamSynchronize(s.stream) == cudaSuccess ? CB_OK : CB_ERR_CUDA;
}

static int copy_out(Solver& s, float* dst, const float* src, long long count, int on_device) {
  cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(float) * count,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s.stream);
  if (e != cudaSuccess) return CB_ERR_CUDA;
  return cudaStreamSynchronize(s.stream) == cudaSuccess ? CB_OK : CB_ERR_CUDA;
}

int claire_b200_set_images(claire_b200_ctx* c, int b, const float* mR, const float* mT, int on_device) {
  if (!c || !mR || !mT || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  if (s.img16) {
    // host images stage through problem b's PCG work vector (2n of its 3n
    // floats; idle between solver calls), then round to bf16
    const float *dR = mR, *dT = mT;
    if (!on_device) {
      float* st = s.x + b * 3 * s.n;
      int e = copy_in(s, st, mR, s.n, 0);
      if (!e) e = copy_in(s, st + s.n, mT, s.n, 0);
      if (e) return e;
      dR = st;
      dT = st + s.n;
    }
    int e = s.load_images(b, dR, dT);
    if (!e && cudaStreamSynchronize(s.stream) != cudaSuccess) e = CB_ERR_CUDA;
    return cuda_status(e);
  }
  int e = copy_in(s, s.mR + b * s.n, mR, s.n, on_device);
  if (!e) e = copy_in(s, s.mT + b * s.n, mT, s.n, on_device);
  s.images_changed(b);
  return e;
}

int claire_b200_set_mask(claire_b200_ctx* c, int b, const float* w, int on_device) {
  if (!c || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  const float* src = w;
  if (w && !on_device) {
    float* st = s.x + b * 3 * s.n;  // problem b's PCG work vector, idle between solver calls
    if (int e = copy_in(s, st, w, s.n, 0)) return e;
    src = st;
  }
  return cuda_status(s.set_mask(b, src));
}

int claire_b200_set_velocity(claire_b200_ctx* c, int b, const float* v, int on_device) {
  if (!c || !v || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  s.state_of[b] = 0;
  return copy_in(s, s.v + b * 3 * s.n, v, 3 * s.n, on_device);
}

int claire_b200_get_velocity(const claire_b200_ctx* c, int b, float* v, int on_device) {
  if (!c || !v || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = const_cast<Solver&>(c->solver);
  return copy_out(s, v, s.v + b * 3 * s.n, 3 * s.n, on_device);
}

}  // extern "C"

namespace {

// Device buffer freed on scope exit.
struct DevBuf {
  float* p = nullptr;
  int alloc(long long floats) { return cudaMalloc((void**)&p, sizeof(float) * (size_t)floats) == cudaSuccess ? 0 : CB_ERR_ALLOC; }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

// Carry the per-problem options (norm, weights) of `from` to a level solver.
int copy_problem_opts(const Solver& from, Solver& to) {
  for (int b = 0; b < from.B; ++b) {
    claire_b200_opts o = to.opts;
    o.regnorm = from.ps[b].norm;
    o.beta[0] = from.ps[b].beta0;
    o.beta[1] = from.ps[b].beta1;
    o.beta[2] = from.ps[b].beta2;
    if (int e = to.set_problem(b, o)) return e;
  }
  return 0;
}

// CLAIREInterface::RunSolverScaleCont (src/CLAIREInterface.cpp:1387-1505): the
// original images are smoothed with sigma = 32, 16, ..., 1 grid cells (levels
// with n/2 <= sigma skipped, sigmas of src/RegOpt.cpp:1241-1246); every level
// re-initialises ||g0|| at v = 0 and warm-starts from the current velocity.
int run_scalecont(Solver& s, const std::vector<int>& sel) {
  if (s.img16) {
    s.err = "scale continuation needs FP32 images";
    return CB_ERR_UNSUPPORTED;
  }
  const long long n = s.n;
  DevBuf orig;
  if (int e = orig.alloc(2 * n * s.B)) return e;
  if (cudaMemcpyAsync(orig.p, s.mR, sizeof(float) * n * s.B, cudaMemcpyDeviceToDevice, s.stream) != cudaSuccess ||
      cudaMemcpyAsync(orig.p + n * s.B, s.mT, sizeof(float) * n * s.B, cudaMemcpyDeviceToDevice, s.stream) !=
          cudaSuccess)
    return CB_ERR_CUDA;
  SpecParams* par = nullptr;
  if (cudaMalloc((void**)&par, sizeof(SpecParams) * s.B) != cudaSuccess) return CB_ERR_ALLOC;
  static const double kSigmas[6] = {32.0, 16.0, 8.0, 4.0, 2.0, 1.0};
  int e = 0;
  bool first = true;
  for (int l = 0; l < 6 && !e; ++l) {
    const double sig = kSigmas[l];
    if (0.5 * s.d.n1 <= sig) continue;
    std::vector<SpecParams> hp(s.B);
    for (auto& p : hp) {
      p = SpecParams{};
      p.hd = s.hd;
      p.sigma[0] = p.sigma[1] = p.sigma[2] = (float)sig;
    }
    e = cudaMemcpyAsync(par, hp.data(), sizeof(SpecParams) * s.B, cudaMemcpyHostToDevice, s.stream) ? CB_ERR_CUDA : 0;
    // Preprocessing::Smooth of both originals (2B fields through the 3-field spectrum workspace)
    for (int img = 0; img < 2 && !e; ++img) {
      const float* src = orig.p + img * n * s.B;
      float* dst = img == 0 ? s.mR : s.mT;
      e = launch_r2c3d(src, n, n, s.spec, 3 * s.nc, 1, s.B, s.d, nullptr, s.stream);
      if (!e) e = launch_pencil(s.spec, 3 * s.nc, s.B, s.d, OP_GAUSS, par, 1, 1, nullptr, s.stream);
      if (!e) e = launch_c2r3d(s.spec, 3 * s.nc, dst, n, n, 1, s.B, s.d, EPI_STORE, nullptr, nullptr, 0, nullptr,
                               s.stream);
    }
    if (e) break;
    for (int b = 0; b < s.B; ++b) s.images_changed(b);
    if (!first) {
      s.carry_krylov_g0.assign(s.B, -1.0);
      for (int b = 0; b < s.B; ++b) s.carry_krylov_g0[b] = s.ps[b].krylov_g0;
    }
    e = s.run(sel);
    first = false;
  }
  s.carry_krylov_g0.clear();
  cudaFree(par);
  return e;
}

// CLAIREInterface::RunSolverGridCont (src/CLAIREInterface.cpp:1510-1705):
// levels of RegOpt::SetupGridCont (src/RegOpt.cpp:1844-1930), images
// restricted from the finest grid to each level, v = 0 on the coarsest level
// and prolonged to the next, the gradient tolerance 10x looser below the
// finest level when it is under 0.01, the Krylov reference norm of the first
// solve kept.  The finest level is the context's own solver.
int run_gridcont(Solver& s, const std::vector<int>& sel) {
  if (s.d.n1 != s.d.n2 || s.d.n2 != s.d.n3) {
    s.err = "grid continuation needs a cubic grid";
    return CB_ERR_UNSUPPORTED;
  }
  if (s.img16) {
    s.err = "grid continuation needs FP32 images";
    return CB_ERR_UNSUPPORTED;
  }
  const int nf = s.d.n1;
  int nlev = (int)std::ceil(std::log2((double)nf)) - 3;
  if (nlev < 1) nlev = 1;
  std::vector<int> sizes(nlev);
  sizes[nlev - 1] = nf;
  for (int l = nlev - 2; l >= 0; --l) sizes[l] = (sizes[l + 1] + 1) / 2;
  const double greltol = s.opts.opttol;
  DevBuf vprev, work;
  long long wmax = 0;
  for (int l = 0; l < nlev; ++l) {
    wmax = std::max(wmax, grid_change_work(nf, sizes[l], s.B));
    if (l + 1 < nlev) wmax = std::max(wmax, grid_change_work(sizes[l], sizes[l + 1], 3 * s.B));
  }
  if (int e = work.alloc(std::max(wmax, 1LL))) return e;
  int prev = 0;  // size of the last solved level (0: none yet)
  std::vector<double> kg0;
  for (int l = 0; l < nlev; ++l) {
    const int nl = sizes[l];
    const bool last = l == nlev - 1;
    if (!last && !fft_size_supported(nl)) continue;  // no FFT plan for this size here
    std::unique_ptr<Solver> own;
    Solver* lv = &s;
    if (!last) {
      claire_b200_opts o = s.opts;
      o.nx[0] = o.nx[1] = o.nx[2] = nl;
      o.gridcont = 0;
      if (greltol < 0.01) o.opttol = 10.0 * greltol;
      own.reset(new (std::nothrow) Solver());
      if (!own) return CB_ERR_ALLOC;
      if (int e = own->init(o, s.B)) {
        s.err = own->err;
        return e;
      }
      own->stream = s.stream;
      if (int e = copy_problem_opts(s, *own)) return e;
      lv = own.get();
      const long long nn = (long long)nl * nl * nl;
      if (int e = launch_grid_change(s.mR, s.n, nf, lv->mR, nn, nl, s.B, work.p, s.stream)) return CB_ERR_CUDA;
      if (int e = launch_grid_change(s.mT, s.n, nf, lv->mT, nn, nl, s.B, work.p, s.stream)) return CB_ERR_CUDA;
      for (int b = 0; b < s.B; ++b) lv->images_changed(b);
    }
    const long long nn = (long long)nl * nl * nl;
    if (prev) {
      const long long np = (long long)prev * prev * prev;
      if (launch_grid_change(vprev.p, np, prev, lv->v, nn, nl, 3 * s.B, work.p, s.stream)) return CB_ERR_CUDA;
    } else if (cudaMemsetAsync(lv->v, 0, sizeof(float) * 3 * nn * s.B, s.stream) != cudaSuccess) {
      return CB_ERR_CUDA;
    }
    for (int b = 0; b < s.B; ++b) lv->state_of[b] = 0;
    lv->carry_krylov_g0 = kg0;
    if (int e = lv->run(sel)) {
      if (lv != &s) s.err = lv->err;
      return e;
    }
    lv->carry_krylov_g0.clear();
    kg0.assign(s.B, -1.0);
    for (int b = 0; b < s.B; ++b) kg0[b] = lv->ps[b].krylov_g0;
    if (!last) {
      DevBuf nv;
      if (int e = nv.alloc(3 * nn * s.B)) return e;
      if (cudaMemcpyAsync(nv.p, lv->v, sizeof(float) * 3 * nn * s.B, cudaMemcpyDeviceToDevice, s.stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(s.stream) != cudaSuccess)
        return CB_ERR_CUDA;
      std::swap(vprev.p, nv.p);
      prev = nl;
    }
  }
  return 0;
}

int run_dispatch(Solver& s, const std::vector<int>& sel) {
  // RunSolverRegParaCont first (src/CLAIREInterface.cpp:729-753)
  if (s.opts.train != CB_TRAIN_OFF) return s.run_train(sel, s.opts.train);
  if (s.opts.betacont > 0.0) return s.run(sel);
  if (s.opts.scalecont) return run_scalecont(s, sel);
  if (s.opts.gridcont) {
    if (s.opts.precond == CB_PC_TWOLEVEL) {
      // the coarsest continuation levels would need coarse grids below the
      // smallest transform size
      s.err = "grid continuation with the two-level preconditioner is not supported";
      return CB_ERR_UNSUPPORTED;
    }
    return run_gridcont(s, sel);
  }
  if (s.opts.monitordefgrad) return s.run_monitored(sel);
  return s.run(sel);
}

}  // namespace

extern "C" {

int claire_b200_run(claire_b200_ctx* c) {
  if (!c) return CB_ERR_ARG;
  std::vector<int> sel(c->solver.B, 1);
  return cuda_status(run_dispatch(c->solver, sel));
}

int claire_b200_run_masked(claire_b200_ctx* c, const int* mask) {
  if (!c || !mask) return CB_ERR_ARG;
  std::vector<int> sel(mask, mask + c->solver.B);
  return cuda_status(run_dispatch(c->solver, sel));
}

int claire_b200_get_final_state(claire_b200_ctx* c, int b, float* m1, int on_device) {
  if (!c || !m1 || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  float* tmp = nullptr;
  if (!on_device) {
    if (cudaMalloc(&tmp, sizeof(float) * s.n) != cudaSuccess) return CB_ERR_ALLOC;
  }
  int e = s.final_state(on_device ? m1 : tmp, b);
  if (!e && !on_device) e = copy_out(s, m1, tmp, s.n, 0);
  if (tmp) cudaFree(tmp);
  return cuda_status(e);
}

int claire_b200_forward(claire_b200_ctx* c, int b, const float* m0, float* m1, int on_device) {
  if (!c || !m0 || !m1 || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  // stage through the work field r (problem stride 3n, first n entries)
  float* in = s.r + b * 3 * s.n;
  float* out = s.z + b * 3 * s.n;
  int e = copy_in(s, in, m0, s.n, on_device);
  if (e) return e;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  // forward() uses a problem stride of n for m0/m1: pass shifted bases
  e = s.forward(s.r + b * 3 * s.n - b * s.n, s.z + b * 3 * s.n - b * s.n, sel);
  if (e) return cuda_status(e);
  return copy_out(s, m1, out, s.n, on_device);
}

int claire_b200_get_stats(const claire_b200_ctx* c, int b, claire_b200_stats* st) {
  if (!c || !st || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  const ProbState& p = c->solver.ps[b];
  st->gn_iterations = p.iter;
  st->pcg_iterations = p.pcg_total;
  st->obj_evals = p.obj_evals;
  st->grad_evals = p.grad_evals;
  st->hess_matvecs = p.hess_matvecs;
  st->pc_matvecs = p.pc_matvecs;
  st->pde_solves = p.pde_solves;
  st->converged_reason = p.reason;
  st->J = p.J;
  st->J0 = p.J0;
  st->D = p.D;
  st->D0 = p.D0;
  st->R = p.R;
  st->gnorm = p.gnorm;
  st->gnorm0 = p.gnorm0;
  st->rel_mismatch = p.rel_mismatch;
  st->seconds = p.seconds;
  st->beta = p.beta0;
  st->solution_status = p.solution_status;
  st->det_min = p.det[0];
  st->det_mean = p.det[1];
  st->det_max = p.det[2];
  return CB_OK;
}

int claire_b200_objective(claire_b200_ctx* c, int b, const float* v, double* J, double* D, double* R) {
  if (!c || !v || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  int e = claire_b200_set_velocity(c, b, v, 0);
  if (e) return e;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  e = s.objective_at(s.v, sel);
  if (e) return cuda_status(e);
  if (J) *J = s.ps[b].J;
  if (D) *D = s.ps[b].D;
  if (R) *R = s.ps[b].R;
  return CB_OK;
}

int claire_b200_gradient(claire_b200_ctx* c, int b, const float* v, float* gout) {
  if (!c || !v || !gout || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  int e = claire_b200_set_velocity(c, b, v, 0);
  if (e) return e;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  e = s.gradient_at_current(sel);
  if (e) return cuda_status(e);
  return copy_out(s, gout, s.g + b * 3 * s.n, 3 * s.n, 0);
}

int claire_b200_hessian_matvec(claire_b200_ctx* c, int b, const float* v, const float* vt, float* hvt) {
  if (!c || !v || !vt || !hvt || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  int e = claire_b200_set_velocity(c, b, v, 0);
  if (e) return e;
  e = copy_in(s, s.pv + b * 3 * s.n, vt, 3 * s.n, 0);
  if (e) return e;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  e = s.hessian_matvec(s.pv, s.q, sel);
  if (e) return cuda_status(e);
  return copy_out(s, hvt, s.q + b * 3 * s.n, 3 * s.n, 0);
}

int claire_b200_precond(claire_b200_ctx* c, int b, const float* xin, float* px) {
  if (!c || !xin || !px || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  int e = copy_in(s, s.r + b * 3 * s.n, xin, 3 * s.n, 0);
  if (e) return e;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  e = s.precond(s.r, s.z, sel);
  if (e) return cuda_status(e);
  return copy_out(s, px, s.z + b * 3 * s.n, 3 * s.n, 0);
}

int claire_b200_det_def_grad(claire_b200_ctx* c, int b, int inverse, float* jac, double stats[3]) {
  if (!c || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  std::vector<double> st;
  int e = s.det_def_grad(sel, inverse != 0, st);
  if (e) return cuda_status(e);
  if (stats) {
    stats[0] = st[3 * b];
    stats[1] = st[3 * b + 1];
    stats[2] = st[3 * b + 2];
  }
  if (jac) return copy_out(s, jac, s.work3 + b * 3 * s.n, s.n, 0);
  return CB_OK;
}

int claire_b200_deformation_map(claire_b200_ctx* c, int b, int inverse, float* y) {
  if (!c || !y || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  int e = s.deformation_map(sel, inverse != 0);
  if (e) return cuda_status(e);
  e = copy_out(s, y, s.x + b * 3 * s.n, 3 * s.n, 0);
  if (e) return e;
  // positions y = x + u h (ComputeRegularGrid: x_i = i h, h = 2 pi / N per axis)
  const int n1 = s.d.n1, n2 = s.d.n2, n3 = s.d.n3;
  const double h[3] = {cb::kTwoPi / n1, cb::kTwoPi / n2, cb::kTwoPi / n3};
  for (int i1 = 0; i1 < n1; ++i1)
    for (int i2 = 0; i2 < n2; ++i2)
      for (int i3 = 0; i3 < n3; ++i3) {
        const long long i = ((long long)i1 * n2 + i2) * n3 + i3;
        y[i] = (float)((i1 + (double)y[i]) * h[0]);
        y[s.n + i] = (float)((i2 + (double)y[s.n + i]) * h[1]);
        y[2 * s.n + i] = (float)((i3 + (double)y[2 * s.n + i]) * h[2]);
      }
  return CB_OK;
}

int claire_b200_def_grad(claire_b200_ctx* c, int b, float* F, float* det, double stats[3]) {
  if (!c || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  const long long n = s.n;
  std::vector<float> own;
  float* F9 = F;
  if (!F9) {
    own.resize((size_t)(9 * n));
    F9 = own.data();
  }
  int e = s.def_grad(b, F9);
  if (e) return cuda_status(e);
  // det F and its min / mean / max (ComputeDefGrad, src/DeformationFields.cpp:902-935)
  double mn = 1e300, mx = -1e300, sum = 0.0;
  for (long long i = 0; i < n; ++i) {
    const float* f = F9;
    const float j11 = f[i], j12 = f[n + i], j13 = f[2 * n + i], j21 = f[3 * n + i], j22 = f[4 * n + i],
                j23 = f[5 * n + i], j31 = f[6 * n + i], j32 = f[7 * n + i], j33 = f[8 * n + i];
    const float phi = j11 * j22 * j33 + j12 * j23 * j31 + j13 * j21 * j32 - j13 * j22 * j31 - j12 * j21 * j33 -
                      j11 * j23 * j32;
    if (det) det[i] = phi;
    mn = std::min(mn, (double)phi);
    mx = std::max(mx, (double)phi);
    sum += phi;
  }
  if (stats) {
    stats[0] = mn;
    stats[1] = sum / (double)n;
    stats[2] = mx;
  }
  return CB_OK;
}

int claire_b200_det_def_grad_disp(claire_b200_ctx* c, int b, float* jac, double stats[3]) {
  if (!c || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  const long long n = s.n;
  std::vector<float> g((size_t)(9 * n));
  int e = s.disp_grad(b, g.data());
  if (e) return cuda_status(e);
  // ComputeDetDefGradViaDispField (src/DeformationFields.cpp:788-800), with
  // its signs as written (the terms with three off-diagonal entries enter with +)
  double mn = 1e300, mx = -1e300, sum = 0.0;
  const float* u = g.data();
  for (long long i = 0; i < n; ++i) {
    const float g11 = u[i], g12 = u[n + i], g13 = u[2 * n + i], g21 = u[3 * n + i], g22 = u[4 * n + i],
                g23 = u[5 * n + i], g31 = u[6 * n + i], g32 = u[7 * n + i], g33 = u[8 * n + i];
    const float phi = (1.f - g11) * (1.f - g22) * (1.f - g33) + g12 * g23 * g31 + g13 * g21 * g32 -
                      g13 * (1.f - g22) * g31 - g12 * g21 * (1.f - g33) - (1.f - g11) * g23 * g32;
    if (jac) jac[i] = phi;
    mn = std::min(mn, (double)phi);
    mx = std::max(mx, (double)phi);
    sum += phi;
  }
  if (stats) {
    stats[0] = mn;
    stats[1] = sum / (double)n;
    stats[2] = mx;
  }
  return CB_OK;
}

int claire_b200_displacement_field(claire_b200_ctx* c, int b, float* u) {
  if (!c || !u || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  std::vector<int> sel(s.B, 0);
  sel[b] = 1;
  int e = s.displacement_field(sel);
  if (e) return cuda_status(e);
  return copy_out(s, u, s.x + b * 3 * s.n, 3 * s.n, 0);
}

int claire_b200_get_adjoint(claire_b200_ctx* c, int b, float* lambda0, float* body_force) {
  if (!c || b < 0 || b >= c->solver.B) return CB_ERR_ARG;
  Solver& s = c->solver;
  int e = CB_OK;
  if (lambda0) e = copy_out(s, lambda0, s.lamh + b * (s.nt + 1) * s.n, s.n, 0);
  if (!e && body_force) {
    if (s.opts.model == CB_MODEL_COMPRESSIBLE) {
      // without a projection the sweep writes its body force straight into the
      // gradient / matvec output; re-form it from the stored adjoint levels
      e = cuda_status(launch_body_force(s.lamh + b * (s.nt + 1) * s.n, 0, s.gm + b * (s.nt + 1) * 3 * s.n, 0,
                                        s.bf + b * 3 * s.n, 0, s.nt, s.ht, s.hd, 1, s.n, nullptr, s.stream));
      note_launches(1);
    }
    if (!e) e = copy_out(s, body_force, s.bf + b * 3 * s.n, 3 * s.n, 0);
  }
  return e;
}

int claire_b200_synchronize(claire_b200_ctx* c) {
  if (!c) return CB_ERR_ARG;
  return cudaStreamSynchronize(c->solver.stream) == cudaSuccess ? CB_OK : CB_ERR_CUDA;
}

int claire_b200_set_stream(claire_b200_ctx* c, void* stream) {
  if (!c) return CB_ERR_ARG;
  Solver& s = c->solver;
  if (cudaStreamSynchronize(s.stream) != cudaSuccess) return CB_ERR_CUDA;
  s.stream = stream ? (cudaStream_t)stream : s.own_stream;
  return CB_OK;
}

// ---------------------------------------------------------------------------
// operator seams; scratch comes from the stream-ordered allocator
// ---------------------------------------------------------------------------
static bool dims_ok(const int nx[3]) {
  return nx && nx[0] > 0 && nx[1] > 0 && nx[2] > 0;
}
static bool fft_ok(const int nx[3]) {
  return fft_col_size_supported(nx[0]) && fft_col_size_supported(nx[1]) && fft_size_supported(nx[2]);
}

int claire_b200_trajectory(const float* v, float* disp, const int nx[3], int nt, int flag, void* stream) {
  if (!v || !disp || !dims_ok(nx) || nt < 1 || (flag != 0 && flag != 1)) return CB_ERR_ARG;
  Dims d{nx[0], nx[1], nx[2]};
  const float sign = flag == 0 ? 1.f : -1.f;
  note_launches(1);
  return cuda_status(launch_trajectory(v, 0, disp, 0, 1, d, (float)(1.0 / nt), sign, nullptr, (cudaStream_t)stream));
}

int claire_b200_interp3(const float* f, const float* disp, float* out, const int nx[3], int dof, void* stream) {
  if (!f || !disp || !out || !dims_ok(nx) || (dof != 1 && dof != 3)) return CB_ERR_ARG;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t s = (cudaStream_t)stream;
  // box table of this displacement (stream-ordered scratch, freed in order)
  int4* tab = nullptr;
  if (cudaMallocAsync((void**)&tab, sizeof(int4) * tile_table_int4s(d), s) != cudaSuccess) return CB_ERR_ALLOC;
  int e = launch_tile_table(disp, 0, tab, 0, 1, d, nullptr, s);
  if (!e) e = launch_interp(f, 0, d.n(), disp, 0, tab, 0, out, 0, d.n(), dof, 1, d, nullptr, s);
  cudaFreeAsync(tab, s);
  note_launches(2);
  return cuda_status(e);
}

int claire_b200_stage_timeouts(long long* count) {
  if (!count) return CB_ERR_ARG;
  unsigned long long t = 0;
  if (stage_timeouts(&t)) return CB_ERR_CUDA;
  *count = (long long)t;
  return CB_OK;
}

int claire_b200_stage_wait_selftest(long long wait_ns, void* stream) {
  if (wait_ns < 0 || wait_ns > 10000000000LL) return CB_ERR_ARG;
  note_launches(1);
  return cuda_status(launch_stage_wait_selftest((unsigned long long)wait_ns, (cudaStream_t)stream));
}

int claire_b200_interp3_bf16(const unsigned short* f, const float* disp, unsigned short* out, const int nx[3],
                             void* stream) {
  if (!f || !disp || !out || !dims_ok(nx)) return CB_ERR_ARG;
  if (!(nx[2] & 3) && (reinterpret_cast<uintptr_t>(f) & 7)) return CB_ERR_ARG;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t s = (cudaStream_t)stream;
  int4* tab = nullptr;
  if (cudaMallocAsync((void**)&tab, sizeof(int4) * tile_table_int4s(d), s) != cudaSuccess) return CB_ERR_ALLOC;
  int e = launch_tile_table(disp, 0, tab, 0, 1, d, nullptr, s);
  if (!e)
    e = launch_interp16(reinterpret_cast<const bf16*>(f), 0, disp, 0, tab, 0, reinterpret_cast<bf16*>(out), 0, 1, d,
                        nullptr, s);
  cudaFreeAsync(tab, s);
  note_launches(2);
  return cuda_status(e);
}

int claire_b200_autotune(int n, int nbatch, void* stream, int* variant, float* ms) {
  if (!fft_col_size_supported(n) || nbatch < 1) return CB_ERR_ARG;
  float t[4] = {-1.f, -1.f, -1.f, -1.f};
  int best = 0;
  const int e = fft_autotune(n, nbatch, (cudaStream_t)stream, &best, t);
  if (e) return e == (int)cudaErrorMemoryAllocation ? CB_ERR_ALLOC : CB_ERR_CUDA;
  if (variant) *variant = best;
  if (ms)
    for (int i = 0; i < 4; ++i) ms[i] = t[i];
  return CB_OK;
}

int claire_b200_fft_variant(int n) { return fft_col_size_supported(n) ? fft_variant(n) : -1; }

int claire_b200_set_fft_variant(int n, int variant) {
  if (!fft_col_size_supported(n)) return CB_ERR_ARG;
  return set_fft_variant(n, variant) ? CB_ERR_ARG : CB_OK;
}

int claire_b200_grid_change(const float* in, int ns, float* out, int nt, int nf, void* stream) {
  if (!in || !out || ns < 2 || nt < 2 || nf < 1 || ns > 1024 || nt > 1024) return CB_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  float* work = nullptr;
  const long long w = std::max(grid_change_work(ns, nt, nf), 1LL);
  if (cudaMallocAsync((void**)&work, sizeof(float) * (size_t)w, st) != cudaSuccess) return CB_ERR_ALLOC;
  const long long ni = (long long)ns * ns * ns, no = (long long)nt * nt * nt;
  const int e = launch_grid_change(in, ni, ns, out, no, nt, nf, work, st);
  cudaFreeAsync(work, st);
  note_launches(3);
  return cuda_status(e);
}

int claire_b200_fft_grad(const float* f, float* gout, const int nx[3], void* stream) {
  if (!f || !gout || !dims_ok(nx)) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  const long long n = d.n();
  for (int a = 0; a < 3; ++a) {
    int e = launch_deriv(f, 0, n, gout + a * n, 0, n, 1, 1, d, a, EPI_STORE, nullptr, 0, nullptr, (cudaStream_t)stream);
    if (e) return cuda_status(e);
  }
  note_launches(3);
  return CB_OK;
}

int claire_b200_fft_div(const float* v, float* dout, const int nx[3], void* stream) {
  if (!v || !dout || !dims_ok(nx)) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  const long long n = d.n();
  for (int a = 0; a < 3; ++a) {
    int e = launch_deriv(v + a * n, 0, n, dout, 0, n, 1, 1, d, a, a == 0 ? EPI_STORE : EPI_ADD, nullptr, 0, nullptr,
                         (cudaStream_t)stream);
    if (e) return cuda_status(e);
  }
  note_launches(3);
  return CB_OK;
}

// scratch for a 3-field spectral op: spectrum, params, partials, result slot
struct Scratch {
  float2* spec = nullptr;
  SpecParams* params = nullptr;
  double* partials = nullptr;
  double* result = nullptr;
  cudaStream_t s = nullptr;
  int alloc(const Dims& d, int nparts, cudaStream_t st) {
    s = st;
    if (cudaMallocAsync((void**)&spec, sizeof(float2) * 3 * d.nc(), s) != cudaSuccess) return CB_ERR_ALLOC;
    if (cudaMallocAsync((void**)&params, sizeof(SpecParams), s) != cudaSuccess) return CB_ERR_ALLOC;
    if (cudaMallocAsync((void**)&partials, sizeof(double) * (nparts + 1), s) != cudaSuccess) return CB_ERR_ALLOC;
    result = partials + nparts;
    return CB_OK;
  }
  ~Scratch() {
    if (spec) cudaFreeAsync(spec, s);
    if (params) cudaFreeAsync(params, s);
    if (partials) cudaFreeAsync(partials, s);
  }
};

static SpecParams make_params(const Dims& d, int regnorm, const double* beta, double beta2) {
  SpecParams p{};
  p.norm = regnorm;
  p.beta0 = beta ? (float)beta[0] : 0.f;
  p.beta1 = beta ? (float)beta[1] : 0.f;
  p.beta2 = (float)beta2;
  p.hd = (float)((kTwoPi / d.n1) * (kTwoPi / d.n2) * (kTwoPi / d.n3));
  p.sigma[0] = p.sigma[1] = p.sigma[2] = 1.f;
  return p;
}

static int spectral3(const float* in, float* out, const Dims& d, int op, const SpecParams& hp, int epi,
                     double* sumsq, cudaStream_t st) {
  Scratch sc;
  const int np = std::max(1, c2r_partials(d, 3));
  int e = sc.alloc(d, np, st);
  if (e) return e;
  if (cudaMemcpyAsync(sc.params, &hp, sizeof(SpecParams), cudaMemcpyHostToDevice, st) != cudaSuccess) return CB_ERR_CUDA;
  const long long n = d.n(), nc = d.nc();
  e = launch_r2c3d(in, 0, n, sc.spec, 0, 3, 1, d, nullptr, st);
  if (!e) e = launch_pencil(sc.spec, 0, 1, d, op, sc.params, 3, 3, nullptr, st);
  if (!e) e = launch_c2r3d(sc.spec, 0, out, 0, n, 3, 1, d, epi, nullptr, sc.partials, np, nullptr, st);
  if (!e && epi == EPI_SUMSQ) e = launch_finalize(sc.partials, np, np, sc.result, 1, 1.0, false, st);
  note_launches(6);
  if (e) return cuda_status(e);
  if (epi == EPI_SUMSQ && sumsq) {
    if (cudaMemcpyAsync(sumsq, sc.result, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CB_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CB_ERR_CUDA;
  }
  (void)nc;
  return CB_OK;
}

int claire_b200_reg_apply(const float* v, float* out, const int nx[3], int regnorm, const double beta[2],
                          int kind, void* stream) {
  if (!v || !out || !dims_ok(nx) || !beta || regnorm < 0 || regnorm > CB_NORM_H3SN) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t st = (cudaStream_t)stream;
  if (regnorm == CB_NORM_L2 || beta[0] == 0.0) {
    // src/RegularizationL2.cpp:100-215: beta*v and v/beta in real space
    double c = 1.0;
    if (beta[0] != 0.0) c = (kind == CB_REG_GRADIENT) ? beta[0] : (kind == CB_REG_INVERSE ? 1.0 / beta[0] : 1.0 / std::sqrt(beta[0]));
    else if (kind == CB_REG_GRADIENT) c = 0.0;
    note_launches(1);
    return cuda_status(launch_lincomb(out, 0, v, 0, nullptr, c, nullptr, 0, nullptr, 0.0, 3 * d.n(), 1, nullptr, st));
  }
  int op = kind == CB_REG_GRADIENT ? OP_REG_GRAD : (kind == CB_REG_INVERSE ? OP_REG_INV : OP_REG_SQRTINV);
  return spectral3(v, out, d, op, make_params(d, regnorm, beta, 0.0), EPI_STORE, nullptr, st);
}

int claire_b200_reg_functional(const float* v, double* R, const int nx[3], int regnorm, const double beta[2],
                               void* stream) {
  if (!v || !R || !dims_ok(nx) || !beta || regnorm < 0 || regnorm > CB_NORM_H3SN) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t st = (cudaStream_t)stream;
  const double hd = (kTwoPi / d.n1) * (kTwoPi / d.n2) * (kTwoPi / d.n3);
  if (beta[0] == 0.0) {
    *R = 0.0;
    return CB_OK;
  }
  const long long n = d.n();
  if (regnorm == CB_NORM_H1 || regnorm == CB_NORM_H1SN || regnorm == CB_NORM_L2) {
    int np = dot_partials(3 * n);
    for (int a = 0; a < 3; ++a) np = std::max(np, deriv_partials(d, a, 3));
    double* buf = nullptr;
    if (cudaMallocAsync((void**)&buf, sizeof(double) * (np + 2), st) != cudaSuccess) return CB_ERR_ALLOC;
    double* res = buf + np;
    int e = 0;
    if (regnorm != CB_NORM_L2) {
      for (int a = 0; a < 3 && !e; ++a) {
        const int p = deriv_partials(d, a, 3);
        e = launch_deriv(v, 0, n, nullptr, 0, 0, 3, 1, d, a, EPI_SUMSQ, buf, np, nullptr, st);
        if (!e) e = launch_finalize(buf, np, p, res, 1, 1.0, a > 0, st);
      }
      note_launches(6);
    }
    if (!e) e = launch_dot(v, 0, v, 0, 3 * n, 1, buf, np, nullptr, st);
    if (!e) e = launch_finalize(buf, np, dot_partials(3 * n), res + 1, 1, 1.0, false, st);
    note_launches(2);
    double h[2] = {0.0, 0.0};
    if (!e && cudaMemcpyAsync(h, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) e = CB_ERR_CUDA;
    if (!e && cudaStreamSynchronize(st) != cudaSuccess) e = CB_ERR_CUDA;
    cudaFreeAsync(buf, st);
    if (e) return cuda_status(e);
    if (regnorm == CB_NORM_H1SN) *R = 0.5 * hd * beta[0] * h[0];
    else if (regnorm == CB_NORM_H1) *R = 0.5 * hd * beta[0] * (h[0] + beta[1] * h[1]);
    else *R = 0.5 * hd * beta[0] * h[1];
    return CB_OK;
  }
  double s = 0.0;
  int e = spectral3(v, nullptr, d, OP_REG_FUNC, make_params(d, regnorm, beta, 0.0), EPI_SUMSQ, &s, st);
  if (e) return e;
  if (regnorm == CB_NORM_H2SN || regnorm == CB_NORM_H3SN) *R = 0.5 * hd * beta[0] * s;
  else *R = 0.5 * hd * s;
  return CB_OK;
}

int claire_b200_leray(float* b, const int nx[3], int model, const double beta[3], void* stream) {
  if (!b || !dims_ok(nx) || (model != CB_MODEL_STOKES && model != CB_MODEL_RELAXEDSTOKES)) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  double bb[2] = {beta ? beta[0] : 1e-2, beta ? beta[1] : 1e-4};
  SpecParams p = make_params(d, CB_NORM_H1SN, bb, beta ? beta[2] : 1e-4);
  return spectral3(b, b, d, model == CB_MODEL_STOKES ? OP_LERAY : OP_LERAY_RELAXED, p, EPI_ADD, nullptr,
                   (cudaStream_t)stream);
}

int claire_b200_smooth(const float* f, float* out, const int nx[3], const double sigma[3], void* stream) {
  if (!f || !out || !dims_ok(nx) || !sigma) return CB_ERR_ARG;
  if (!fft_ok(nx)) return CB_ERR_UNSUPPORTED;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t st = (cudaStream_t)stream;
  Scratch sc;
  int e = sc.alloc(d, 1, st);
  if (e) return e;
  SpecParams p = make_params(d, 0, nullptr, 0.0);
  for (int k = 0; k < 3; ++k) p.sigma[k] = (float)sigma[k];
  if (cudaMemcpyAsync(sc.params, &p, sizeof(SpecParams), cudaMemcpyHostToDevice, st) != cudaSuccess) return CB_ERR_CUDA;
  const long long n = d.n();
  e = launch_r2c3d(f, 0, n, sc.spec, 0, 1, 1, d, nullptr, st);
  if (!e) e = launch_pencil(sc.spec, 0, 1, d, OP_GAUSS, sc.params, 1, 1, nullptr, st);
  if (!e) e = launch_c2r3d(sc.spec, 0, out, 0, n, 1, 1, d, EPI_STORE, nullptr, nullptr, 0, nullptr, st);
  note_launches(5);
  return cuda_status(e);
}

int claire_b200_distance(const float* mR, const float* m1, const int nx[3], double* D, void* stream) {
  if (!mR || !m1 || !D || !dims_ok(nx)) return CB_ERR_ARG;
  Dims d{nx[0], nx[1], nx[2]};
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = d.n();
  const int np = dot_partials(n);
  double* buf = nullptr;
  if (cudaMallocAsync((void**)&buf, sizeof(double) * (np + 1), st) != cudaSuccess) return CB_ERR_ALLOC;
  const double hd = (kTwoPi / d.n1) * (kTwoPi / d.n2) * (kTwoPi / d.n3);
  int e = launch_diff_sumsq(mR, 0, m1, 0, n, 1, buf, np, nullptr, st);
  if (!e) e = launch_finalize(buf, np, np, buf + np, 1, 0.5 * hd, false, st);
  note_launches(2);
  if (!e && cudaMemcpyAsync(D, buf + np, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) e = CB_ERR_CUDA;
  if (!e && cudaStreamSynchronize(st) != cudaSuccess) e = CB_ERR_CUDA;
  cudaFreeAsync(buf, st);
  return cuda_status(e);
}

long long claire_b200_kernel_launches(void) { return launches(); }

int claire_b200_profile(claire_b200_ctx* c, int enable) {
  if (!c) return CB_ERR_ARG;
  Solver& s = c->solver;
  if (!enable) {
    if (cudaStreamSynchronize(s.stream) != cudaSuccess) return CB_ERR_CUDA;
    s.prof_clear();
  } else if (s.prof_reserve(4096)) {
    return CB_ERR_CUDA;
  }
  s.prof_on = enable != 0;
  return CB_OK;
}

int claire_b200_profile_read(claire_b200_ctx* c, int category, double* total_ms, long long* launches_out) {
  if (!c || category < 0 || category >= CB_PROF_NCAT) return CB_ERR_ARG;
  return c->solver.prof_read(category, total_ms, launches_out);
}

}  // extern "C"
