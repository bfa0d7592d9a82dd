/*
 * claire_b200.h -- C ABI of the B200-native CLAIRE Gauss-Newton-Krylov path.
 *
 * Plain pointers, sizes and int status codes; no C++ or torch types.  Every
 * entry point returns CB_OK (0) or a negative CB_ERR_* code.  Device pointers
 * are float32 arrays on the current CUDA device; `stream` is a cudaStream_t
 * (NULL = legacy default stream).
 *
 * Grids are periodic on [0, 2*pi)^3, row-major with x3 fastest
 * (include/CLAIREUtils.hpp:198-212 of the reference).  Vector fields are three
 * consecutive scalar fields [x1 | x2 | x3] (src/VecField.cpp:396-478).
 * Displacements ("disp") are characteristic foot points X minus the grid
 * node, in grid units: X = (i + disp) * 2*pi / N.
 */
#ifndef CLAIRE_B200_H_
#define CLAIRE_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define CB_OK 0
#define CB_ERR_ARG (-1)       /* invalid argument */
#define CB_ERR_ALLOC (-2)     /* device or host allocation failed */
#define CB_ERR_CUDA (-3)      /* a CUDA call or kernel launch failed */
#define CB_ERR_NUMERIC (-4)   /* NaN / Inf in objective or gradient */
#define CB_ERR_STATE (-5)     /* call out of order (e.g. run before images) */
#define CB_ERR_UNSUPPORTED (-6) /* grid size without an FFT plan */
#define CB_ERR_TOO_LARGE (-7)   /* grid exceeds a fixed-size workspace, or the footprint exceeds the
                                   free device memory / the server's HBM budget */
#define CB_ERR_CANCELLED (-8)   /* the registration request was cancelled (claire_b200_server_cancel) */

/* Regularisation norms (-regnorm): l2 h1 h1s h2 h2s h3 h3s. */
enum {
  CB_NORM_L2 = 0, CB_NORM_H1 = 1, CB_NORM_H1SN = 2, CB_NORM_H2 = 3,
  CB_NORM_H2SN = 4, CB_NORM_H3 = 5, CB_NORM_H3SN = 6
};
/* Regularisation-parameter searches (-train): binary search and reduction. */
enum { CB_TRAIN_OFF = 0, CB_TRAIN_BINARY = 1, CB_TRAIN_REDUCE = 2 };
/* Registration models: CLAIRE (no projection), Stokes, relaxed Stokes. */
enum { CB_MODEL_COMPRESSIBLE = 0, CB_MODEL_STOKES = 1, CB_MODEL_RELAXEDSTOKES = 2 };
/* Distance measures (-distance): squared L2 (DistanceMeasureSL2) or
 * normalised cross-correlation (DistanceMeasureNCC). */
enum { CB_DIST_SL2 = 0, CB_DIST_NCC = 1 };
/* Krylov forcing sequences (-krylovfseq). */
enum { CB_FSEQ_NONE = 0, CB_FSEQ_QUADRATIC = 1, CB_FSEQ_SUPERLINEAR = 2 };
/* Preconditioners (-precond): none, inverse regularisation, two-level
 * (coarse-grid solve of the symmetrically preconditioned Hessian). */
enum { CB_PC_NONE = 0, CB_PC_INVREG = 1, CB_PC_TWOLEVEL = 2 };
/* Regularisation operator kinds for claire_b200_reg_apply. */
enum { CB_REG_GRADIENT = 0, CB_REG_INVERSE = 1, CB_REG_SQRTINVERSE = 2 };

/*
 * Hot-path subset of reg::RegOpt (include/RegOpt.hpp:475-635); defaults from
 * RegOpt::Initialize (src/RegOpt.cpp:1032-1293).
 */
typedef struct claire_b200_opts {
  int nx[3];            /* -nx */
  int nt;               /* -nt (4) */
  int regnorm;          /* -regnorm (CB_NORM_H1SN) */
  int model;            /* registration model (CB_MODEL_COMPRESSIBLE when -regnorm given) */
  double beta[3];       /* -beta sets beta[0] (1e-2); beta[1] = 1e-4; beta[2] = 1e-4 */
  int maxit;            /* -maxit (50) */
  double opttol;        /* -opttol: ||g|| < opttol*||g0|| (5e-2) */
  double gatol;         /* ||g|| < gatol (1e-6) */
  int krylovmaxit;      /* -krylovmaxit (50); PCG runs krylovmaxit-1 iterations */
  double krylovtol[3];  /* rtol 1e-12, atol 1e-16, dtol 1e6 */
  int krylovfseq;       /* -krylovfseq (CB_FSEQ_SUPERLINEAR) */
  int precond;          /* -precond: CB_PC_INVREG (default), CB_PC_NONE, CB_PC_TWOLEVEL */
  int iporder;          /* -iporder: 3 (tricubic) is the only order on this path */
  int verbosity;        /* -verbosity */
  int bf16_images;      /* store transported images in bf16 (gathers accumulate in fp32) */
  double betacont;      /* -betacont beta*: regularisation-parameter continuation to beta* (0: off) */
  double presolvetol;   /* relative gradient tolerance of the continuation levels (1e-1) */
  int autotune;         /* -autotune: measure the FFT variants of this grid size when the first
                           context of that size is created (claire_b200_autotune) */
  int distance;         /* -distance sl2|ncc (CB_DIST_SL2); NCC needs FP32 images */
  int scalecont;        /* -scalecont: continuation over image smoothing widths */
  int gridcont;         /* -gridcont: continuation over grid sizes */
  int train;            /* -train binary|reduce: search beta against the det(grad y) bound (0: off) */
  double jbound;        /* -jbound: bound on min det(grad y) and 1/max det(grad y) (0.25) */
  double betainit;      /* -betainit: first beta of -train and -betacont searches (1.0) */
  int monitordefgrad;   /* -monitordefgrad: check det(grad y) against -jbound after the solve and
                           raise beta toward 10 beta while it is breached (RunSolver) */
  double pcgridscale;   /* -gridscale: coarse grid of the two-level preconditioner, ceil(nx / 2) */
  double pctolscale;    /* -pctolscale: coarse solve tolerance = pctolscale * forcing value (0.1) */
  int pcsolvermaxit;    /* -pcsolvermaxit (10): iterations of a flexible outer solver's coarse
                           solve; the PCG outer solver used here runs the coarse solve to its
                           tolerance (at most 1000 iterations) */
} claire_b200_opts;

typedef struct claire_b200_stats {
  int gn_iterations;        /* outer iterations */
  int pcg_iterations;       /* total inner iterations */
  int obj_evals, grad_evals, hess_matvecs, pc_matvecs, pde_solves;
  int converged_reason;     /* 1 gttol, 2 gatol, 3 maxit, 4 steptol, 5 lsfail, -1 nan */
  double J, J0, D, D0, R;   /* objective, distance, regularisation (FP64) */
  double gnorm, gnorm0;     /* ||g|| and ||g0|| (FP64) */
  double rel_mismatch;      /* ||mR - m1|| / ||mR - mT|| */
  double seconds;           /* wall time of claire_b200_run */
  double beta;              /* regularisation weight of the solution (the estimate of -train) */
  int solution_status;      /* -monitordefgrad: 0 bound kept, 1 kept after raising beta, 2 still breached */
  double det_min, det_mean, det_max; /* det(grad y) of the solution (-monitordefgrad / -train) */
} claire_b200_stats;

typedef struct claire_b200_ctx claire_b200_ctx;

/* ---- options (reg::RegOpt) ------------------------------------------------ */
/* Fill with RegOpt::Initialize defaults (src/RegOpt.cpp:1032-1293). */
int claire_b200_default_opts(claire_b200_opts* opts);
/* Parse the hot-path flags of RegOpt::ParseArguments (src/RegOpt.cpp:260-834):
 * -nx -nt -regnorm -beta -maxit -opttol -gabs -krylovmaxit -krylovtol
 * -krylovfseq -precond -iporder -verbosity. */
int claire_b200_parse_args(claire_b200_opts* opts, int argc, const char* const* argv);

/* ---- registration context (reg::CLAIREInterface) -------------------------- */
/* Create a context holding `nbatch` independent problems of one grid size;
 * allocates all device state up front (include/CLAIREInterface.hpp:42-90).
 * CB_ERR_TOO_LARGE, with nothing allocated, when claire_b200_estimate_bytes
 * exceeds the device's free memory; CB_ERR_ALLOC when an allocation fails. */
int claire_b200_create(const claire_b200_opts* opts, int nbatch, claire_b200_ctx** ctx);
int claire_b200_destroy(claire_b200_ctx* ctx);
const char* claire_b200_last_error(const claire_b200_ctx* ctx);
/* Bytes of device memory the context holds (admission accounting). */
long long claire_b200_footprint_bytes(const claire_b200_ctx* ctx);
long long claire_b200_estimate_bytes(const claire_b200_opts* opts, int nbatch);
/* Per-problem options inside a batch (norm, beta, ...); nx and nt must match. */
int claire_b200_set_problem_opts(claire_b200_ctx* ctx, int b, const claire_b200_opts* opts);
/* SetReferenceImage / SetTemplateImage (src/CLAIREInterface.cpp:594-660). */
int claire_b200_set_images(claire_b200_ctx* ctx, int b, const float* mR, const float* mT, int on_device);
/* SetMask (src/CLAIREInterface.cpp:277-286): weights w (n floats, host or
 * device) of problem b's distance measure (DistanceMeasureSL2 / NCC with a
 * mask: weighted sums and final conditions); w = NULL removes the mask. */
int claire_b200_set_mask(claire_b200_ctx* ctx, int b, const float* w, int on_device);
/* SetInitialGuess (src/CLAIREInterface.cpp: copy semantics). */
int claire_b200_set_velocity(claire_b200_ctx* ctx, int b, const float* v, int on_device);
int claire_b200_get_velocity(const claire_b200_ctx* ctx, int b, float* v, int on_device);
/* Run: GN-Krylov solve of every problem in the context (CLAIREInterface::Run,
 * src/CLAIREInterface.cpp:709-885): with -betacont the parameter
 * continuation, else with -scalecont the smoothing continuation
 * (RunSolverScaleCont, :1387-1505: sigma = 32, 16, ..., 1 cells while below
 * n/2), else with -gridcont the grid continuation (RunSolverGridCont,
 * :1510-1705: ceil(log2 n) - 3 levels of halved grids, images restricted,
 * velocity prolonged; sizes without an FFT plan here are skipped), else
 * RunSolver.  Continuation runs end with the images of their last level in
 * the context (smoothed with sigma = 1 for -scalecont). */
int claire_b200_run(claire_b200_ctx* ctx);
/* Solve only the problems whose mask entry is nonzero. */
int claire_b200_run_masked(claire_b200_ctx* ctx, const int* mask);
/* GetFinalState: m(t=1) for the current velocity. */
int claire_b200_get_final_state(claire_b200_ctx* ctx, int b, float* m1, int on_device);
/* SolveForwardProblem(m1, m0) with the current velocity (src/CLAIREInterface.cpp:1890). */
int claire_b200_forward(claire_b200_ctx* ctx, int b, const float* m0, float* m1, int on_device);
int claire_b200_get_stats(const claire_b200_ctx* ctx, int b, claire_b200_stats* stats);
/* Objective J(v), gradient g(v) and GN Hessian matvec H*vt at velocity v for
 * problem b (OptimizationProblem::{EvaluateObjective, EvaluateGradient,
 * HessianMatVec}, include/OptimizationProblem.hpp:51-121).  Host pointers.
 * With -precond 2level the matvec is the Krylov operator of that mode,
 * hd vt + P^1/2 b~[P^1/2 vt] (CLAIRE::PrecondHessMatVecSym,
 * src/CLAIRE.cpp:1455-1532). */
int claire_b200_objective(claire_b200_ctx* ctx, int b, const float* v, double* J, double* D, double* R);
int claire_b200_gradient(claire_b200_ctx* ctx, int b, const float* v, float* g);
int claire_b200_hessian_matvec(claire_b200_ctx* ctx, int b, const float* v, const float* vt, float* hvt);
/* Preconditioner::MatVec (src/Preconditioner.cpp:507-580): INVREG
 * P x = (beta A)^-1 x; with -precond 2level Apply2LevelPrecond (:584-673),
 * set up at the problem's current velocity, coarse tolerance
 * pctolscale * krylovtol[0]. */
int claire_b200_precond(claire_b200_ctx* ctx, int b, const float* x, float* px);
/* det(grad y) of problem b at its current velocity (inverse != 0:
 * det(grad(inv(y)))), DeformationFields::ComputeDetDefGrad with the SL solver
 * (src/DeformationFields.cpp:315-388, 636-739; CLAIREInterface::ComputeDetDefGrad,
 * include/CLAIREInterface.hpp:42-90).  jac (host, n floats) may be NULL;
 * stats = {min, mean, max} (the reference's monitor values, :367-375). */
int claire_b200_det_def_grad(claire_b200_ctx* ctx, int b, int inverse, float* jac, double stats[3]);
/* Deformation map y of problem b at its current velocity (inverse != 0: the
 * inverse map), DeformationFields::ComputeDeformationMap with the SL RK2
 * scheme (src/DeformationFields.cpp:1189-1268, 1472-1585): y (host, 3 nl
 * floats [y1 | y2 | y3]) holds physical coordinates in [0, 2 pi), unwrapped. */
int claire_b200_deformation_map(claire_b200_ctx* ctx, int b, int inverse, float* y);
/* Displacement field u of problem b at its current velocity by the SL scheme,
 * DeformationFields::ComputeDisplacementFieldSL (src/DeformationFields.cpp:
 * 1816-1909): u (host, 3 nl floats), physical units. */
int claire_b200_displacement_field(claire_b200_ctx* ctx, int b, float* u);
/* Deformation gradient F of problem b at its current velocity by the SL
 * scheme, DeformationFields::ComputeDefGrad / ComputeDefGradSL
 * (src/DeformationFields.cpp:821-1117): F (host, 9 nl floats, F_ab at
 * (3a + b) nl, may be NULL), det F (host, nl floats, may be NULL) and its
 * {min, mean, max} (may be NULL). */
int claire_b200_def_grad(claire_b200_ctx* ctx, int b, float* F, float* det, double stats[3]);
/* det(grad y) through the displacement field (-detdefgradfromdeffield,
 * DeformationFields::ComputeDetDefGradViaDispField,
 * src/DeformationFields.cpp:745-815): the SL displacement field u, its
 * spectral gradient, and det(I - grad u) with the reference's signs; jac
 * (host, nl floats) and {min, mean, max} may be NULL. */
int claire_b200_det_def_grad_disp(claire_b200_ctx* ctx, int b, float* jac, double stats[3]);
/* Adjoint state lambda(t=0) and body force b of the last adjoint solve (the
 * last gradient evaluation or Hessian matvec of problem b). */
int claire_b200_get_adjoint(claire_b200_ctx* ctx, int b, float* lambda0, float* body_force);
int claire_b200_synchronize(claire_b200_ctx* ctx);
/* Run the context's work on the caller's stream from now on (NULL: the
 * context's own stream).  The caller keeps ownership of the stream. */
int claire_b200_set_stream(claire_b200_ctx* ctx, void* stream);

/* ---- operator seams on device buffers (one problem, explicit stream) ------ */
/* SemiLagrangian::ComputeTrajectory (src/SemiLagrangian.cpp:192-289):
 * flag 0 = "state" (+1), 1 = "adjoint" (-1).  v: 3n, disp: 3n. */
int claire_b200_trajectory(const float* v, float* disp, const int nx[3], int nt, int flag, void* stream);
/* SemiLagrangian::Interpolate (src/SemiLagrangian.cpp:536-727): out[k] =
 * f[k](i + disp) for k < dof (dof 1 or 3), tricubic (src/interp3.cpp:2492-2719). */
int claire_b200_interp3(const float* f, const float* disp, float* out, const int nx[3], int dof, void* stream);
/* The same gather of one bfloat16 volume (the -bf16images storage of the
 * images and state levels): f and out hold bfloat16 bit patterns, the 64-tap
 * sum is FP32 and rounded to nearest even.  No reference counterpart (the
 * reference interpolates single or double precision images); f must be
 * 8-byte aligned when nx[2] % 4 == 0. */
int claire_b200_interp3_bf16(const unsigned short* f, const float* disp, unsigned short* out, const int nx[3],
                             void* stream);
/* FFT planning by measurement, the counterpart of the reference's
 * accfft_plan_dft_3d_r2c(..., ACCFFT_MEASURE) (src/RegOpt.cpp:993-994): times
 * every variant of the n-point transforms (two-stage radix plan x lines per
 * CTA) on nbatch problems of the solver's spectral work (a 3-field
 * regularisation operator and a 3-field gradient) and keeps the fastest for
 * this process.  variant receives the choice; ms[i] the time of candidate i
 * (4 entries, -1 where a size has fewer candidates; may be NULL).  Variants
 * differ only in rounding (each within the FFT tolerance of the others).
 * The choice is process-wide: tune, or set a variant, only while no
 * transform of that size is in flight.  Allocates scratch; synchronises. */
int claire_b200_autotune(int n, int nbatch, void* stream, int* variant, float* ms);
/* Current FFT variant of size n (-1: unsupported), and a stored choice. */
int claire_b200_fft_variant(int n);
int claire_b200_set_fft_variant(int n, int variant);
/* ---- file input / output (the path before and after the registration) ----- */
/* ReadWriteReg::ReadNII (src/ReadWriteReg.cpp:794-1128): one scalar volume of
 * a single-file NIfTI-1 image (.nii or .nii.gz; uint8/int8/int16/uint16/
 * int32/uint32/int64/uint64/float32/float64).  nx receives CLAIRE's grid
 * (nx[0] = NIfTI nz, nx[2] = NIfTI nx, src/ReadWriteReg.cpp:813-815); data
 * (host, at least nx[0]*nx[1]*nx[2] floats = capacity, or NULL to query the
 * size) receives the raw voxel values as float, in file order (x3 fastest).
 * Two-file images (.hdr + .img, magic "ni1") are read when either name is
 * given.  CB_ERR_UNSUPPORTED for several volumes or components, or other
 * data types. */
int claire_b200_read_nifti(const char* path, int nx[3], float* data, long long capacity);
/* ReadWriteReg::WriteNII (src/ReadWriteReg.cpp:1130-1475): float32 NIfTI-1,
 * gzip-compressed when the path ends in .gz; pixdim = 2*pi/nx.  A path ending
 * in .hdr or .img (optionally .gz) writes the two-file pair. */
int claire_b200_write_nifti(const char* path, const int nx[3], const float* data);
/* ReadWriteReg::ReadBIN / WriteBIN (src/ReadWriteReg.cpp:1476-1535): PETSc
 * binary vectors (VecLoad / VecView layout: big-endian int32 class id
 * 1211214, int32 length, big-endian values).  Written as 8-byte doubles (the
 * reference's default build); read as doubles or 4-byte floats by file size.
 * The file holds no grid: nx (CLAIRE order) gives it, and the stored length
 * must equal nx[0]*nx[1]*nx[2]. */
int claire_b200_read_bin(const char* path, const int nx[3], float* data);
int claire_b200_write_bin(const char* path, const int nx[3], const float* data);
/* Image preparation of the file path on a device field (one problem):
 * rescale != 0 applies Normalize (src/CLAIREUtils.cpp:492-525, called by
 * CLAIREInterface::SetReferenceImage / SetTemplateImage,
 * src/CLAIREInterface.cpp:254-320): negatives to zero, x <- (x - min) / max;
 * sigma != NULL then applies the Gaussian smoothing of
 * CLAIREInterface::SetupData (src/CLAIREInterface.cpp:594-626) with sigma
 * grid cells per axis.  Synchronises the stream. */
int claire_b200_preprocess(float* m, const int nx[3], int rescale, const double sigma[3], void* stream);
/* Preprocessing::Restrict / Prolong (src/Preprocessing.cpp:733-917,
 * 1605-1786): nf cubic fields of ns^3 points (consecutive) to nt^3 points
 * (consecutive) by spectral truncation / zero padding, coefficients
 * |w| < min(ns, nt)/2 per axis.  Scratch from the stream-ordered allocator. */
int claire_b200_grid_change(const float* in, int ns, float* out, int nt, int nf, void* stream);
/* accfft_grad_t: g (3n) = spectral gradient of f (n), Nyquist zeroed. */
int claire_b200_fft_grad(const float* f, float* g, const int nx[3], void* stream);
/* accfft_divergence_t: d (n) = spectral divergence of v (3n). */
int claire_b200_fft_div(const float* v, float* d, const int nx[3], void* stream);
/* Regularization::{EvaluateGradient, ApplyInverse} (src/Regularization*.cpp):
 * out (3n) = op(v (3n)); kind = CB_REG_GRADIENT / CB_REG_INVERSE / CB_REG_SQRTINVERSE. */
int claire_b200_reg_apply(const float* v, float* out, const int nx[3], int regnorm, const double beta[2],
                          int kind, void* stream);
/* Same operator as claire_b200_reg_apply, for callers that cannot allocate
 * device memory while it runs (their allocator owns the whole GPU budget, or
 * an allocation would synchronise or may fail mid-run).  No counterpart in the
 * reference.  The FFT workspace, parameter block and twiddle tables are fixed
 * device arrays inside the library (3.3 MB on every GPU that loads it, held
 * until exit); nothing is allocated per call.  Grids up to 64^3 only (N in
 * 16, 32, 48, 64): larger grids return CB_ERR_TOO_LARGE.  All calls share the
 * workspace, so calls that overlap on the GPU race; serialise them.  The first
 * call on a device sets it up (symbol lookup and twiddle upload with that
 * device current): make it before any stream capture. */
int claire_b200_reg_apply_noalloc(const float* v, float* out, const int nx[3], int regnorm, const double beta[2],
                                  int kind, void* stream);
/* Regularization::EvaluateFunctional: R(v) in FP64 (host result). */
int claire_b200_reg_functional(const float* v, double* R, const int nx[3], int regnorm,
                               const double beta[2], void* stream);
/* CLAIREStokes / CLAIREDivReg ::ApplyProjection: b (3n) += Leray addend. */
int claire_b200_leray(float* b, const int nx[3], int model, const double beta[3], void* stream);
/* Preprocessing::GaussianSmoothing (src/Preprocessing.cpp:1956-2056): sigma in cells. */
int claire_b200_smooth(const float* f, float* out, const int nx[3], const double sigma[3], void* stream);
/* DistanceMeasureSL2::EvaluateFunctional: D = 1/2 hd sum (mR - m1)^2 (FP64 host result). */
int claire_b200_distance(const float* mR, const float* m1, const int nx[3], double* D, void* stream);
/* Number of CUDA kernel launches issued by this library since load (all threads). */
long long claire_b200_kernel_launches(void);

/* Health of the tricubic gathers' bounded waits.  Each tile gather stages its
 * box of the field in shared memory with bulk asynchronous copies that
 * complete on a barrier; every wait for them is bounded (200 ms), and a wait
 * that runs out is counted, its tile skipped and the kernel returns.
 * claire_b200_stage_timeouts returns the count on the current device (a
 * context's next GN step reports CB_ERR_CUDA when it grew).
 * claire_b200_stage_wait_selftest launches one block that waits wait_ns for a
 * copy that is never issued, so the count grows by one and the context stays
 * usable.  The reference's interpolation has no device waits
 * (src/interp3.cpp:2492-2719 runs on the host). */
int claire_b200_stage_timeouts(long long* count);
int claire_b200_stage_wait_selftest(long long wait_ns, void* stream);

/* ---- Serving: continuous batching of independent registrations ----------
 * The reference runs one registration per CLAIREInterface::Run call
 * (src/CLAIREInterface.cpp:709-885) and has no serving layer; a server runs
 * many such calls concurrently on one GPU.  It keeps pools of solver slots,
 * one pool per (grid, nt, solver-wide options), each with its own stream and
 * host thread.  A submitted request waits until a slot of its pool is free,
 * is admitted at the next GN-iteration boundary, keeps its state on the device
 * until its stopping test fires and frees the slot.  Pools are created while
 * their footprint (claire_b200_estimate_bytes) fits the HBM budget and release
 * their memory after idling.  Per-request options that may differ inside a
 * pool: regnorm and beta.  Results equal those of claire_b200_run on the same
 * inputs (no data is shared between slots). */
typedef struct claire_b200_server claire_b200_server;
typedef struct claire_b200_server_opts {
  long long hbm_budget_bytes; /* device memory all pools may hold (0: 90% of the free memory) */
  int slots_per_pool;         /* problems per pool (batch width) */
  int idle_ms;                /* a pool without work for this long releases its memory */
  int device;                 /* CUDA device of the server */
  int batch_window_us;        /* an idle pool that receives a request waits up to this long for more
                                 requests of its key before starting (0: start at once, the default) */
} claire_b200_server_opts;
#define CB_REQ_QUEUED 0
#define CB_REQ_RUNNING 1
#define CB_REQ_DONE 2
#define CB_REQ_FAILED 3
#define CB_REQ_CANCELLED 4
void claire_b200_server_default_opts(claire_b200_server_opts* o);
int claire_b200_server_create(const claire_b200_server_opts* o, claire_b200_server** srv);
/* Queue a registration of host images mR, mT (nx[0]*nx[1]*nx[2] floats each,
 * copied); zero initial velocity.  CB_ERR_TOO_LARGE if one pool of its key
 * cannot fit the budget. */
int claire_b200_server_submit(claire_b200_server* srv, const claire_b200_opts* o, const float* mR, const float* mT,
                              long long* request_id);
int claire_b200_server_poll(claire_b200_server* srv, long long request_id, int* status);
/* Cancel a request.  A queued request is removed at once; a running one
 * leaves its slot at its pool's next GN-iteration boundary (no kernel of it is
 * interrupted), after which its status is CB_REQ_CANCELLED and
 * claire_b200_server_result returns CB_ERR_CANCELLED.  CB_ERR_STATE when the
 * request has already finished.  The reference has no serving layer and so no
 * counterpart (a CLAIREInterface::Run call, src/CLAIREInterface.cpp:709-885,
 * runs to its stopping test). */
int claire_b200_server_cancel(claire_b200_server* srv, long long request_id);
/* Block until the request is done, failed or cancelled (timeout_ms < 0: no limit). */
int claire_b200_server_wait(claire_b200_server* srv, long long request_id, int timeout_ms, int* status);
/* Velocity (host, 3n floats, may be NULL), statistics and submit-to-done
 * latency of a finished request; releases it.  A failed request returns its
 * error code. */
int claire_b200_server_result(claire_b200_server* srv, long long request_id, float* v, claire_b200_stats* stats,
                              double* latency_ms);
int claire_b200_server_info(claire_b200_server* srv, int* pools, long long* bytes_used, int* queued);
/* Fails queued requests, waits for running ones' pools to stop, frees everything. */
int claire_b200_server_destroy(claire_b200_server* srv);

/* Device timers of the solver's time steps and operations, the counterpart
 * of the reference's per-phase timers and counters (include/RegOpt.hpp:183-202).
 * While enabled, every launch or call of a category is bracketed by CUDA
 * events on the context's stream (host overhead per launch: use for
 * instrumented runs; PCG iterations then run without graph replay).  An
 * operation category (objective, gradient, Hessian) covers every launch of
 * one call, including the waits for its host-side decisions.
 * claire_b200_profile_read synchronizes the stream, returns the summed device
 * time and the count of a category since the last read, and resets it. */
#define CB_PROF_ADJOINT_STEP 0  /* lambda^{l-1} = c * lambda^l(X): one per adjoint step */
#define CB_PROF_INCSTATE_STEP 1 /* m~^{j+1} = m~^j(X) + s_j: one per incremental step */
#define CB_PROF_STATE_STEP 2    /* m^{j+1} = m^j(X): one per state step */
#define CB_PROF_PRECOND 3       /* z = P r in the PCG: one 3-field forward + inverse transform with the
                                   inverse symbol, per Krylov iteration (Preconditioner::MatVec,
                                   src/Preconditioner.cpp:507-580) */
#define CB_PROF_OBJECTIVE 4     /* one objective evaluation: state solve, distance, regularisation functional
                                   (OptimizationProblem::EvaluateObjective) */
#define CB_PROF_GRADIENT 5      /* one gradient: adjoint solve, body force, regularisation (EvaluateGradient) */
#define CB_PROF_HESSIAN 6       /* one GN Hessian matvec in the PCG (HessianMatVec) */
#define CB_PROF_NCAT 7
int claire_b200_profile(claire_b200_ctx* ctx, int enable);
int claire_b200_profile_read(claire_b200_ctx* ctx, int category, double* total_ms, long long* launches);

#ifdef __cplusplus
}
#endif

#endif /* CLAIRE_B200_H_ */
