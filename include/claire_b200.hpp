// claire_b200.hpp -- header-only C++ facade over the C ABI with the class
// names of the reference's public C++ surface (namespace reg):
//   reg::RegOpt            (include/RegOpt.hpp:479-483)
//   reg::CLAIREInterface   (include/CLAIREInterface.hpp:42-90)
//   reg::SemiLagrangian    (include/SemiLagrangian.hpp:43-58)
//   reg::Regularization    (include/Regularization.hpp:46-50)
//   reg::DistanceMeasureSL2 (include/DistanceMeasure.hpp:44-50)
//   reg::Preconditioner    (include/Preconditioner.hpp: MatVec)
//   reg::VecField          (include/VecField.hpp; flat [x1 | x2 | x3])
// Images and fields are plain float arrays in place of PETSc Vec (host arrays
// for CLAIREInterface, device arrays for the operator classes).  Every method
// returns an int status like the reference's PetscErrorCode: 0 on success,
// a negative CB_ERR_* code otherwise; nothing throws.
#ifndef CLAIRE_B200_HPP_
#define CLAIRE_B200_HPP_

#include <string>
#include <vector>

#include "claire_b200.h"

namespace reg {

using ErrorCode = int;  // plays the role of PetscErrorCode

class RegOpt {
 public:
  // RegOpt::Initialize defaults (src/RegOpt.cpp:1032-1293)
  RegOpt() { status_ = claire_b200_default_opts(&opts_); }
  // RegOpt(argc, argv): Initialize + ParseArguments (src/RegOpt.cpp:260-834);
  // argv[0] is the program name, as in the reference
  RegOpt(int argc, char** argv) {
    status_ = claire_b200_default_opts(&opts_);
    if (!status_ && argc > 1) status_ = claire_b200_parse_args(&opts_, argc - 1, argv + 1);
  }
  ErrorCode status() const { return status_; }
  claire_b200_opts& opts() { return opts_; }
  const claire_b200_opts& opts() const { return opts_; }
  long long nl() const { return (long long)opts_.nx[0] * opts_.nx[1] * opts_.nx[2]; }
  int nt() const { return opts_.nt; }
  long long EstimateBytes(int nbatch = 1) const { return claire_b200_estimate_bytes(&opts_, nbatch); }

 private:
  claire_b200_opts opts_{};
  ErrorCode status_ = 0;
};

// Three-component velocity field on the host, components stored one after
// another (VecField::GetComponents / SetComponents layout).
class VecField {
 public:
  explicit VecField(const RegOpt& opt) : n_(opt.nl()), data_(3 * opt.nl(), 0.f) {}
  long long nl() const { return n_; }
  float* x1() { return data_.data(); }
  float* x2() { return data_.data() + n_; }
  float* x3() { return data_.data() + 2 * n_; }
  float* data() { return data_.data(); }
  const float* data() const { return data_.data(); }
  ErrorCode SetValue(float value) {
    for (auto& v : data_) v = value;
    return 0;
  }
  ErrorCode SetComponents(const float* flat) {
    for (long long i = 0; i < 3 * n_; ++i) data_[i] = flat[i];
    return 0;
  }
  ErrorCode GetComponents(float* flat) const {
    for (long long i = 0; i < 3 * n_; ++i) flat[i] = data_[i];
    return 0;
  }

 private:
  long long n_;
  std::vector<float> data_;
};

// One registration context (problem b of a batch; b = 0 for the plain form).
class CLAIREInterface {
 public:
  explicit CLAIREInterface(RegOpt* opt, int nbatch = 1) : opt_(opt) {
    status_ = claire_b200_create(&opt->opts(), nbatch, &ctx_);
  }
  ~CLAIREInterface() {
    if (ctx_) claire_b200_destroy(ctx_);
  }
  CLAIREInterface(const CLAIREInterface&) = delete;
  CLAIREInterface& operator=(const CLAIREInterface&) = delete;

  ErrorCode status() const { return status_; }
  const char* LastError() const { return ctx_ ? claire_b200_last_error(ctx_) : "context not created"; }

  // SetReferenceImage / SetTemplateImage (src/CLAIREInterface.cpp:254-320):
  // host arrays of nl floats; the images are sent once both are known
  ErrorCode SetReferenceImage(const float* mR, int b = 0) {
    mR_ = mR;
    return mT_ ? SetImages(b) : 0;
  }
  ErrorCode SetTemplateImage(const float* mT, int b = 0) {
    mT_ = mT;
    return mR_ ? SetImages(b) : 0;
  }
  ErrorCode SetMask(const float* w, int b = 0) { return check(claire_b200_set_mask(ctx_, b, w, 0)); }
  ErrorCode SetInitialGuess(const VecField* v, int b = 0) {
    return check(claire_b200_set_velocity(ctx_, b, v->data(), 0));
  }
  ErrorCode Run() { return check(claire_b200_run(ctx_)); }
  ErrorCode GetSolution(VecField* v, int b = 0) { return check(claire_b200_get_velocity(ctx_, b, v->data(), 0)); }
  ErrorCode GetFinalState(float* m1, int b = 0) { return check(claire_b200_get_final_state(ctx_, b, m1, 0)); }
  // SolveForwardProblem(m1, m0) (src/CLAIREInterface.cpp:1890)
  ErrorCode SolveForwardProblem(float* m1, const float* m0, int b = 0) {
    return check(claire_b200_forward(ctx_, b, m0, m1, 0));
  }
  // ComputeDetDefGrad: det(grad y) into jac (nl floats, may be null) and
  // {min, mean, max} into stats (may be null)
  ErrorCode ComputeDetDefGrad(float* jac = nullptr, double* stats = nullptr, bool inverse = false, int b = 0) {
    double s[3];
    const ErrorCode e = check(claire_b200_det_def_grad(ctx_, b, inverse ? 1 : 0, jac, s));
    if (!e && stats)
      for (int k = 0; k < 3; ++k) stats[k] = s[k];
    return e;
  }
  // ComputeDefGrad: F (9 nl floats, F_ab at (3a + b) nl), det F (nl floats) and
  // {min, mean, max}; any of them may be null
  ErrorCode ComputeDefGrad(float* F = nullptr, float* det = nullptr, double* stats = nullptr, int b = 0) {
    return check(claire_b200_def_grad(ctx_, b, F, det, stats));
  }
  // ComputeDeformationMap: y (3 nl floats, physical coordinates), or the inverse map
  ErrorCode ComputeDeformationMap(float* y, bool inverse = false, int b = 0) {
    return check(claire_b200_deformation_map(ctx_, b, inverse ? 1 : 0, y));
  }
  ErrorCode GetStats(claire_b200_stats* st, int b = 0) const { return claire_b200_get_stats(ctx_, b, st); }
  claire_b200_ctx* handle() { return ctx_; }

 private:
  ErrorCode SetImages(int b) {
    const ErrorCode e = check(claire_b200_set_images(ctx_, b, mR_, mT_, 0));
    mR_ = mT_ = nullptr;
    return e;
  }
  ErrorCode check(int e) const { return ctx_ ? e : CB_ERR_STATE; }

  RegOpt* opt_;
  claire_b200_ctx* ctx_ = nullptr;
  ErrorCode status_ = 0;
  const float* mR_ = nullptr;
  const float* mT_ = nullptr;
};

// Preconditioner::MatVec (src/Preconditioner.cpp:507-580) of a registration
// context's problem b on host arrays of 3 nl floats: INVREG P x = (beta A)^-1 x,
// or with -precond 2level Apply2LevelPrecond (:584-673), set up at the
// problem's current velocity.
class Preconditioner {
 public:
  explicit Preconditioner(CLAIREInterface* problem) : problem_(problem) {}
  ErrorCode MatVec(float* Px, const float* x, int b = 0) {
    return claire_b200_precond(problem_ ? problem_->handle() : nullptr, b, x, Px);
  }
  ErrorCode MatVec(VecField* Px, const VecField* x, int b = 0) { return MatVec(Px->data(), x->data(), b); }

 private:
  CLAIREInterface* problem_;
};

// Operator seams on device arrays (one problem, explicit stream).
class SemiLagrangian {
 public:
  explicit SemiLagrangian(const RegOpt* opt, void* stream = nullptr) : opt_(opt), stream_(stream) {}
  // ComputeTrajectory(v, "state" | "adjoint"): displacements in grid units
  ErrorCode ComputeTrajectory(const float* v, float* disp, const std::string& flag) const {
    const int f = flag == "adjoint" ? 1 : 0;
    return claire_b200_trajectory(v, disp, opt_->opts().nx, opt_->opts().nt, f, stream_);
  }
  // Interpolate(out, in) of a scalar (dof 1) or vector (dof 3) field
  ErrorCode Interpolate(float* out, const float* in, const float* disp, int dof = 1) const {
    return claire_b200_interp3(in, disp, out, opt_->opts().nx, dof, stream_);
  }

 private:
  const RegOpt* opt_;
  void* stream_;
};

class Regularization {
 public:
  explicit Regularization(const RegOpt* opt, void* stream = nullptr) : opt_(opt), stream_(stream) {}
  ErrorCode EvaluateGradient(float* g, const float* v) const { return apply(v, g, CB_REG_GRADIENT); }
  ErrorCode HessianMatVec(float* hv, const float* vt) const { return apply(vt, hv, CB_REG_GRADIENT); }
  ErrorCode ApplyInverse(float* ainvx, const float* x, bool applysqrt = false) const {
    return apply(x, ainvx, applysqrt ? CB_REG_SQRTINVERSE : CB_REG_INVERSE);
  }
  ErrorCode EvaluateFunctional(double* R, const float* v) const {
    const double beta[2] = {opt_->opts().beta[0], opt_->opts().beta[1]};
    return claire_b200_reg_functional(v, R, opt_->opts().nx, opt_->opts().regnorm, beta, stream_);
  }

 private:
  ErrorCode apply(const float* in, float* out, int kind) const {
    const double beta[2] = {opt_->opts().beta[0], opt_->opts().beta[1]};
    return claire_b200_reg_apply(in, out, opt_->opts().nx, opt_->opts().regnorm, beta, kind, stream_);
  }
  const RegOpt* opt_;
  void* stream_;
};

class DistanceMeasureSL2 {
 public:
  explicit DistanceMeasureSL2(const RegOpt* opt, void* stream = nullptr) : opt_(opt), stream_(stream) {}
  // D = 1/2 hd sum (mR - m1)^2 on device arrays
  ErrorCode EvaluateFunctional(double* D, const float* mR, const float* m1) const {
    return claire_b200_distance(mR, m1, opt_->opts().nx, D, stream_);
  }

 private:
  const RegOpt* opt_;
  void* stream_;
};

}  // namespace reg

#endif  // CLAIRE_B200_HPP_
