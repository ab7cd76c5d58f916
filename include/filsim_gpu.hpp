// filsim_gpu.hpp -- header-only C++ mirror of FilSim's hot-path classes over
// the C-ABI of filsim_gpu.h, so a main.cpp-shaped driver keeps its calls:
//
//   FcmGpu            struct Fcm (FCMfunctions.hpp:7-59): Y, F, T in, V, W out
//   LinkedListGpu     struct LinkedList (CollisionBarrierFilament.hpp:19-57)
//   SuspensionGpu     the filament vector with Filament's per-step calls and
//                     filamentJsolver (FilamentJacobianSolver.hpp:14-87), plus
//                     the whole time step of main.cpp:284-754
//
// Errors throw filsim::Error carrying the fs_status. Pointers are device
// pointers unless a method name ends in _host.
#ifndef FILSIM_GPU_HPP
#define FILSIM_GPU_HPP

#include <stdexcept>
#include <string>
#include <vector>
#include "filsim_gpu.h"

namespace filsim {

struct Error : std::runtime_error {
  fs_status status;
  Error(fs_status s, const char *where)
      : std::runtime_error(std::string(where) + ": " + fs_status_string(s)), status(s) {}
};

inline void check(fs_status s, const char *where) {
  if (s != FS_OK) throw Error(s, where);
}

// Owns the fs_ctx; Fcm::initialise + LinkedList::initialise in one.
class Context {
 public:
  Context(const fs_params &p, int max_beads, int max_filaments, void *stream = nullptr) {
    check(fs_create(&p, max_beads, max_filaments, stream, &ctx_), "fs_create");
  }
  ~Context() { fs_destroy(ctx_); }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  fs_ctx *get() const { return ctx_; }
  void synchronize() { check(fs_synchronize(ctx_), "fs_synchronize"); }
  void set_precision(int prec) { check(fs_set_precision(ctx_, prec), "fs_set_precision"); }
  // 2: the first bead of each filament started from 3X - 3Xt + Xtt (1: the reference's 2X - Xt)
  void set_start_order(int order) { check(fs_set_start_order(ctx_, order), "fs_set_start_order"); }
  // 1: tensions extrapolated linearly after lambda_extrap_step (2: the reference's quadratic)
  void set_tension_extrapolation(int order) {
    check(fs_set_tension_extrapolation(ctx_, order), "fs_set_tension_extrapolation");
  }
  // one predicted Broyden update of this weight before each step's first residual (0: off)
  void set_velocity_predictor(double weight) {
    check(fs_set_velocity_predictor(ctx_, weight), "fs_set_velocity_predictor");
  }
  // Broyden memory across steps (fs_set_broyden_memory; all zero: off)
  void set_broyden_memory(int keep_columns, int carry_columns, int threshold, int restart_after) {
    check(fs_set_broyden_memory(ctx_, keep_columns, carry_columns, threshold, restart_after),
          "fs_set_broyden_memory");
  }
  // FP32 steps not converged after after_iters Broyden iterations finish in FP64 (0: off)
  void set_precision_escalation(int after_iters) {
    check(fs_set_precision_escalation(ctx_, after_iters), "fs_set_precision_escalation");
  }
  // steady steps as CUDA graphs with the Broyden loop on the device
  void set_graph_mode(bool on) { check(fs_set_graph_mode(ctx_, on ? 1 : 0), "fs_set_graph_mode"); }
  // fastest launch variants for the uploaded suspension; returns ms per mobility solve
  float autotune(int reps = 3, int *choice = nullptr) {
    int c[4];
    float ms = 0.f;
    check(fs_autotune(ctx_, reps, choice ? choice : c, &ms), "fs_autotune");
    return ms;
  }

 private:
  fs_ctx *ctx_ = nullptr;
};

// independent boxes advanced together, one graph launch per ensemble step
class Batch {
 public:
  Batch(fs_ctx *const *ctxs, int n) : n_(n) { check(fs_batch_create(ctxs, n, &b_), "fs_batch_create"); }
  ~Batch() { fs_batch_destroy(b_); }
  Batch(const Batch &) = delete;
  Batch &operator=(const Batch &) = delete;
  // iterations [nsteps x n]; box_ms (optional) per-box step times; returns the call's device ms
  float run(int nt_start, int nsteps, std::vector<int> &iters, std::vector<float> *box_ms = nullptr) {
    iters.assign((size_t)nsteps * n_, 0);
    if (box_ms) box_ms->assign((size_t)nsteps * n_, 0.f);
    float total = 0.f;
    fs_status s = fs_batch_run(b_, nt_start, nsteps, iters.data(), box_ms ? box_ms->data() : nullptr, &total);
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) throw Error(s, "fs_batch_run");
    return total;
  }

 private:
  fs_batch *b_ = nullptr;
  int n_;
};

// struct Fcm: the caller owns the Np x 3 device arrays (row-major doubles).
class FcmGpu {
 public:
  FcmGpu(Context &ctx, int np) : ctx_(ctx), np_(np) {}
  double *Y = nullptr, *F = nullptr, *T = nullptr, *V = nullptr, *W = nullptr;
  void mobility_solve() { check(fs_fcm_mobility(ctx_.get(), Y, F, T, V, W, np_), "Fcm::mobility_solve"); }
  void friction_mobility_solve() { check(fs_fcm_friction(ctx_.get(), F, T, V, W, np_), "Fcm::friction_mobility_solve"); }
  // host arrays, copies inside
  void mobility_solve_host(const double *Y_h, const double *F_h, const double *T_h, double *V_h, double *W_h) {
    check(fs_fcm_mobility_host(ctx_.get(), Y_h, F_h, T_h, V_h, W_h, np_), "Fcm::mobility_solve_host");
  }

 private:
  Context &ctx_;
  int np_;
};

// struct LinkedList
class LinkedListGpu {
 public:
  explicit LinkedListGpu(Context &ctx) : ctx_(ctx) { check(fs_cells_dims(ctx.get(), M_), "fs_cells_dims"); }
  void link(const double *Xs, int np) { check(fs_cells_link(ctx_.get(), Xs, np), "LinkedList::link"); }
  // adds the barrier forces into F (fcm.F in the reference); returns the minimum squared distance
  double apply_collision_barrier(const double *Y, double *F, int np, int nt, const int *fil_id = nullptr,
                                 const int *seg_id = nullptr) {
    double md = 0;
    check(fs_collision_barrier(ctx_.get(), Y, F, np, nt, fil_id, seg_id, &md), "LinkedList::apply_collision_barrier");
    return md;
  }
  const int *cells() const { return M_; }

 private:
  Context &ctx_;
  int M_[3] = {0, 0, 0};
};

// The filament suspension, resident on the device, and the implicit step.
class SuspensionGpu {
 public:
  SuspensionGpu(Context &ctx, const fs_host_state &s) : ctx_(ctx) { upload(s); }
  void upload(const fs_host_state &s) { check(fs_state_upload(ctx_.get(), &s), "fs_state_upload"); }
  void download(fs_host_state &s) { check(fs_state_download(ctx_.get(), &s), "fs_state_download"); }
  // Filament::initialGuess for every filament
  void initialGuess() { check(fs_initial_guess(ctx_.get()), "initialGuess"); }
  // unRobotArmify + forces/torques + Fcm::assign_filament_data
  void forces(int nt) { check(fs_filament_forces(ctx_.get(), nt), "forces"); }
  // swimming drive: per filament {Alpha, Beta, Phase, Wavenumber, AngFrequency}; nullptr switches it off
  void setSwimming(const double *swim, double curvature, bool spermCurvatureDecay) {
    check(fs_set_swimming(ctx_.get(), swim, curvature, spermCurvatureDecay ? 1 : 0), "setSwimming");
  }
  // spring_links: 2 global bead indices per link, NetworkSpringConstant, NetworkSpringNaturalLength
  void setSpringLinks(int nlinks, const int *beads, double k, double l0) {
    check(fs_set_spring_links(ctx_.get(), nlinks, beads, k, l0), "setSpringLinks");
  }
  // LinkedList::apply_collision_barrier / _not_swimmer / _not_test_particles, or none (FS_BARRIER_*)
  void setBarrierMode(int mode) { check(fs_set_barrier_mode(ctx_.get(), mode), "setBarrierMode"); }
  // one step of main_gaitreset.cpp: iters[3]; vwf (optional) [3][Nw0][9] V, W, F of filament 0
  void stepGaitReset(int nt, int iters[3], double *vwf = nullptr) {
    fs_status s = fs_step_gait_reset(ctx_.get(), nt, iters, vwf);
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) throw Error(s, "fs_step_gait_reset");
  }
  // filamentJsolver::buildJacobian
  void buildJacobian(int nt) { check(fs_jacobian_build(ctx_.get(), nt), "filamentJsolver::buildJacobian"); }
  // filamentJsolver::solve
  void solve(const double *b, double *x, int iter) { check(fs_broyden_apply(ctx_.get(), b, x, iter), "filamentJsolver::solve"); }
  // ErrorCheckFCM; returns check
  bool errorCheck(const double *V, const double *W, double *err, int nt) {
    int c = 0;
    check(fs_error_check(ctx_.get(), V, W, err, nt, &c), "ErrorCheckFCM");
    return c != 0;
  }
  void update(const double *u) { check(fs_state_update(ctx_.get(), u), "Filament::update"); }
  void step(int nt) { check(fs_step(ctx_.get(), nt), "Filament::step"); }
  // one whole time step (main.cpp:284-754); returns the Broyden iterations
  int stepImplicit(int nt) {
    int it = 0;
    fs_status s = fs_step_implicit(ctx_.get(), nt, &it);
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) throw Error(s, "fs_step_implicit");
    return it;
  }
  std::vector<int> run(int nt_start, int nsteps) {
    std::vector<int> its(nsteps > 0 ? nsteps : 0);
    fs_status s = fs_run_steps(ctx_.get(), nt_start, nsteps, its.data());
    if (s != FS_OK && s != FS_ERR_NOT_CONVERGED) throw Error(s, "fs_run_steps");
    return its;
  }

 private:
  Context &ctx_;
};

}  // namespace filsim

#endif  // FILSIM_GPU_HPP
