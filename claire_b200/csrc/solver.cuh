// Host-side Gauss-Newton-Krylov driver over the B200 kernels.
//
// One Solver owns B independent registration problems of one grid size and
// time-step count (B = 1 is the plain single-problem path).  All problems'
// fields live in one allocation per array (problem p at base + p*stride), so
// every kernel launch covers the whole batch and a per-problem `active` mask
// on the device switches problems off once they converge.
#pragma once

#include <chrono>
#include <memory>
#include <string>
#include <vector>

#include "../../include/claire_b200.h"
#include "common.cuh"
#include "spectral.cuh"

namespace cb {

void note_launches(int k);
long long launches();

struct ProbState {
  int norm = NORM_H1SN;
  int model = CB_MODEL_COMPRESSIBLE;
  double beta0 = 1e-2, beta1 = 1e-4, beta2 = 1e-4;
  // GN monitor values (src/RegOpt.hpp m_Monitor)
  double J = 0, J0 = 0, D = 0, D0 = 0, R = 0, gnorm = 0, gnorm0 = 0, krylov_g0 = -1;
  double step = 1.0;
  int iter = 0, pcg_total = 0, reason = 0;
  bool done = false;
  bool running = false;  // between begin() and finish()
  std::chrono::steady_clock::time_point t0{};
  int obj_evals = 0, grad_evals = 0, hess_matvecs = 0, pc_matvecs = 0, pde_solves = 0;
  double seconds = 0.0, rel_mismatch = -1.0;
  int solution_status = 0;
  double det[3] = {0.0, 0.0, 0.0};  // min, mean, max of det(grad y) when checked
};

class Solver {
 public:
  Solver() = default;
  ~Solver();
  int init(const claire_b200_opts& o, int B);
  static long long estimate_bytes(const claire_b200_opts& o, int B);

  // ---- public operations (problems selected by the host mask `sel`) -------
  int run(const std::vector<int>& sel);                  // begin + steps + finish
  int begin(const std::vector<int>& sel);                // join the GN loop (J0, ||g0||)
  int step(std::vector<int>& finished, double gttol = -1.0, int miniter = 0);  // one GN iteration
  int run_betacont(const std::vector<int>& sel, double beta_star, double presolve_gttol);
  // -train binary|reduce: beta search against the det(grad y) bound, one problem at a time
  int run_train(const std::vector<int>& sel, int strategy);
  // -monitordefgrad: RunSolver's bound check and beta raising
  int run_monitored(const std::vector<int>& sel);
  // one solve at the current weights from the current velocity, stopping tests
  // from iteration 1 on, reference norms of the last begin() (a continuation level)
  int solve_level(const std::vector<int>& sel, double gttol);
  int finish(const std::vector<int>& sel);               // final mismatch; leave the loop
  int objective_at(const float* vel, const std::vector<int>& sel);  // fills ps[p].J/D/R
  int gradient_at_current(const std::vector<int>& sel);              // g, ||g|| for v
  int hessian_matvec(const float* vin, float* hout, const std::vector<int>& sel);
  int precond(const float* rin, float* zout, const std::vector<int>& sel);
  int forward(const float* m0, float* m1, const std::vector<int>& sel);
  int det_def_grad(const std::vector<int>& sel, bool inverse, std::vector<double>& stats);
  // deformation map y - x in grid units (3 fields per problem, in x)
  int deformation_map(const std::vector<int>& sel, bool inverse);
  // displacement field u (3 fields per problem, physical units, in x)
  int displacement_field(const std::vector<int>& sel);
  // deformation gradient F of problem b (9 fields, component-major) into the
  // host array F9 (9 n floats)
  int def_grad(int b, float* F9);
  // spectral gradient of problem b's displacement field (9 fields, gu_ka =
  // d_a u_k at index 3k + a) into the host array G9 (9 n floats)
  int disp_grad(int b, float* G9);
  int final_state(float* m1, int b);
  // images of problem b from device arrays (n floats each), converted to the
  // storage type; not synchronised
  int load_images(int b, const float* mRd, const float* mTd);
  // SetMask (src/CLAIREInterface.cpp:277-286): weights w (device, n floats) of
  // problem b's distance, or none (w = null: weight 1)
  int set_mask(int b, const float* w);
  // per-problem norm and weights; upload = false leaves the upload (and its
  // synchronisation) to a later upload_problems()
  int set_problem(int b, const claire_b200_opts& o, bool upload = true);
  int upload_problems() { return upload_params(); }
  long long footprint() const { return bytes_; }

  // grid and sizes
  Dims d{};
  int nt = 4, B = 0;
  long long n = 0, nc = 0;
  float ht = 0.25f, hd = 0.f;
  claire_b200_opts opts{};
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  std::vector<ProbState> ps;
  std::string err;
  unsigned long long stage_seen = 0;  // box-copy timeouts of the device already reported
  int check_stage();                  // CB_ERR_CUDA when a gather's box copy ran out of its wait

  // device state: one allocation per array, problem p at base + p * stride
  float *mR = nullptr, *mT = nullptr, *v = nullptr, *vtrial = nullptr, *m = nullptr;
  float *disp_st = nullptr, *disp_adj = nullptr, *gm = nullptr, *gx = nullptr;
  int4 *tab_st = nullptr, *tab_adj = nullptr;  // box tables of the two characteristics
  long long TP = 0;                              // int4 per problem in a box table
  float *divv = nullptr, *cadj = nullptr, *lamh = nullptr, *bf = nullptr;
  float *g = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *pv = nullptr, *q = nullptr;
  float *vtx = nullptr, *mt = nullptr, *mt2 = nullptr, *sj = nullptr, *work3 = nullptr;
  // PCG: the regularisation operator applied to the search direction, Reg p,
  // carried by a recurrence instead of a spectral pass per iteration
  float* sreg = nullptr;
  const float* reg_in = nullptr;  // set: finish_with_reg adds this as Reg(vin) for the
  const int* rec_act = nullptr;   // problems of rec_act, and transforms for those of
  const int* norec_act = nullptr; // norec_act (null: none)
  int pcg_exec_mode = 0;          // recorded PCG iteration: bit 0 some, bit 1 not all problems recurrent
  // bf16-image mode (opts.bf16_images): mR, mT and the state levels live in
  // these arrays instead (same layout); mR / mT / m above stay null.
  bool img16 = false;
  // distance weights (n per problem), allocated by the first set_mask
  float* wmask = nullptr;
  bf16 *mR16 = nullptr, *mT16 = nullptr, *m16 = nullptr;
  float2* spec = nullptr;
  double* partials = nullptr;
  int maxparts = 0;
  double* dsc = nullptr;   // device scalars [NSLOT][B]
  int* dact = nullptr;     // device mask [B]
  int* dact2 = nullptr;    // device mask [B] (PCG)
  int* dint = nullptr;     // device ints [NISLOT][B]
  SpecParams* dparams = nullptr;
  double* hsc = nullptr;   // pinned host mirror of dsc
  int* hint = nullptr;     // pinned host mirror of dint

  enum Slot { S_D = 0, S_R, S_RV, S_GG, S_PQ, S_RR, S_RZ, S_RZNEW, S_ALPHA, S_BETA, S_TOL,
              S_RN0, S_GD, S_RTOL, S_RW,
              // NCC: sums <x,x> of m1 (or mT), <mR,mR>, <x,mR>, |mT - mR|^2, the
              // scale, <m1,m~>, <mR,m~>, and final-condition coefficients
              S_NA, S_NRR, S_NI, S_NL2, S_NS, S_NIM, S_NRM, S_CA, S_CB, S_CC,
              // PCG: the constant c of Reg P = c I (regularisation recurrence)
              S_RC, NSLOT };
  enum ISlot { I_IT = 0, I_REASON, NISLOT };

  // Krylov reference norms handed to the next begin() (continuation levels keep
  // the first solve's, src/KrylovInterface.cpp:125-134); empty: fresh
  std::vector<double> carry_krylov_g0;
  // velocity for which m / disp_st are valid, per problem: 0 none, 1 v, 2 vtrial
  std::vector<int> state_of;
  // NCC distance (opts.distance == CB_DIST_NCC): scale set up per image pair
  bool ncc = false;
  std::vector<char> ncc_scale_ok;
  void images_changed(int b) {
    state_of[b] = 0;
    if (b >= 0 && b < (int)ncc_scale_ok.size()) ncc_scale_ok[b] = 0;
  }

  // ---- two-level preconditioner (-precond 2level) --------------------------
  // Hessian operator of the Krylov solve: 0 the GN Hessian (DEFAULTMATVEC),
  // 1 its symmetrically preconditioned form hd x + P^1/2 b~[P^1/2 x]
  // (PRECONDMATVECSYM), 2 that form divided by hd (the coarse operator).
  int mv_kind = 0;
  // coarse-grid problems (same batch layout), created by the first setup
  std::unique_ptr<Solver> coarse;
  int nc1 = 0;                 // coarse points per axis, ceil(n1 / gridscale)
  float* gwork = nullptr;      // grid-change workspace
  long long gwork_floats = 0;
  std::vector<double> outer_rtol;  // forcing value of the current Krylov solve, per problem
  // DoSetup / ApplyRestriction: coarse velocity, state levels and mask from
  // the selected problems' current ones; coarse trajectories and caches
  int twolevel_setup(const std::vector<int>& sel);
  // Apply2LevelPrecond: z = M r and r.z into slot rz_slot for the problems in
  // sel (act: the same set on the device)
  int twolevel_apply(const std::vector<int>& sel, const int* act, int rz_slot);
  // coarse side: trajectories, grad m levels and the Hessian caches from the
  // velocity and state levels already in v and m
  int prepare_from_state(const int* act);
  // coarse side: CG on the operator mv_kind with rhs -g, no preconditioner,
  // per-problem relative tolerances; the solution lands in x
  int inner_solve(const std::vector<int>& sel, const std::vector<double>& rtol, int maxit);
  int ensure_wmask();

  // PCG iteration recorded as a CUDA graph (built on the second iteration the
  // solver runs; graphs = false switches replay off)
  bool graphs = true, pcg_warm = false;
  // Reg p by recurrence in the PCG where Reg P = c I (CLAIRE_B200_REG_RECURRENCE=0: off)
  bool reg_rec_enabled = true;
  // p.q and r.z summed inside the inverse transforms' epilogues instead of a
  // separate dot pass (CLAIRE_B200_FUSED_DOTS=1)
  bool fused_dots = false;
  cudaGraphExec_t pcg_exec = nullptr;
  long long pcg_exec_launches = 0;

  // device timers per category (CB_PROF_*): event pairs recorded around launches
  bool prof_on = false;
  std::vector<cudaEvent_t> prof_ev[CB_PROF_NCAT];
  std::vector<cudaEvent_t> prof_pool;  // recorded-and-read events, reused by prof_mark
  int prof_reserve(int count);         // pre-creates events for the pool
  int prof_mark(int cat);  // records one event (call before and after a launch)
  int prof_read(int cat, double* ms, long long* count);
  void prof_clear();

 private:
  long long bytes_ = 0;
  int alloc(void** p, size_t bytes);
  int upload_mask(const std::vector<int>& sel, int* dmask);
  int upload_params();
  double* slot(int s) { return dsc + (long long)s * B; }
  int* islot(int s) { return dint + (long long)s * B; }
  int fetch_scalars();

  // building blocks (act: device mask)
  int characteristic(const float* vel, float sign, const int* act);
  // image-state steps in the storage type (FP32 or bf16)
  int state_init(const float* m0, const int* act);  // m^0 = m0 (device, stride n), or mT if null
  int state_steps(const int* act);                  // m^{j+1} = m^j(X_state), j < nt
  int state_out(float* m1, long long m1p, const int* act);  // m1 = m^nt (FP32)
  // partials of (mR - m^nt or mT)^2, mask-weighted when `weighted` and a mask is set
  int image_diff_sumsq(bool template_image, const int* act, bool weighted = false);
  int wdot(const float* a, long long ap, const float* b, long long bp, int slot, const int* act);  // mask-weighted dot
  int image_residual(float* y, long long yp, const int* act);  // y = mR - m^nt
  int image_grad(const int* act);                              // gm = grad m^j, j <= nt
  int state_solve(const float* vel, const int* act);
  int distance(const std::vector<int>& sel, const int* act);
  int ncc_setup_scale(const std::vector<int>& sel);   // DistanceMeasureNCC::SetupScale where needed
  int ncc_final_condition(float* lam, long long lp, const int* act);       // lambda(1)
  int ncc_inc_final_condition(float* lam, long long lp, const int* act);   // lambda~(1) from m~(1) in lam
  int reg_functional(const float* vel, const std::vector<int>& sel, const int* act);
  int reg_op(const float* vin, float* out, int op, int epi, const int* act, const float* dot_with = nullptr,
             int dot_slot = -1);
  int grad_fields(const float* f, long long fp, long long ifs, float* out, long long op,
                  long long ofs, int nf, const int* act);
  int divergence(const float* vel, float* out, const int* act);
  int div_penalty(const float* vel, const int* act);
  // hscale >= 0 replaces hd as the body force's final factor
  int adjoint_sweep(float* bout, const int* act, double hscale = -1.0);
  int finish_with_reg(const float* vin, float* out, const int* act, const float* dot_with = nullptr,
                      int dot_slot = -1);
  int gradient(const int* act);
  int hessian_prep(const int* act);
  // incremental state and adjoint final condition for vin (everything of the
  // Hessian matvec before the incremental adjoint sweep)
  int inc_state(const float* vin, const int* act);
  int hessian(const float* vin, float* hout, const int* act, int pq_slot = -1);
  int hessian_sym(const float* vin, float* hout, const int* act, int pq_slot = -1);
  int apply_op(const float* vin, float* hout, const int* act, int pq_slot = -1) {
    return mv_kind ? hessian_sym(vin, hout, act, pq_slot) : hessian(vin, hout, act, pq_slot);
  }
  int pcg(const std::vector<int>& sel, double maxit);
  int pcg_twolevel(const std::vector<int>& sel, double maxit);
  // per problem: whether Reg P = c I holds, and c (0: it does not)
  void reg_recurrence(const std::vector<int>& sel, std::vector<double>& c) const;
  int line_search(std::vector<int>& sel);
  int dot(const float* a, long long ap, const float* b, long long bp, long long len, int slot,
          const int* act, double scale = 1.0);
};

}  // namespace cb
