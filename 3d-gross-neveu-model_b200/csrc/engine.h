// engine.h -- internal C++ interface of the device engine behind the C-ABI.
// One Engine per lattice (L) and device; it owns every device buffer of that
// lattice and one CUDA stream.  All fields live in the reference's fermion
// order (see geometry.cuh) as real planes of V = L^3 values.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gn_b200.h"
#include "cg_kernel.cuh"
#include "geometry.cuh"

namespace gn {

constexpr int kNumWorkVecs = 4;  // FP64 solver vectors r, p0, p1, t per right-hand side

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

// Result of one solve, per right-hand side.
struct SolveInfo {
  int status;       // CgStatus
  long long iters;  // iterations the reference would count (0 if not counted)
  double r2;        // final |r|^2 of the stopping test
  double b2;
  long long inner;  // mixed precision: low-precision iterations
  long long reliable;  // mixed precision: reliable updates
};

// Parity mode for one operation's operators (the engine's `exact` flag set
// on entry when asked for, restored on every exit).
struct ExactScope {
  bool &flag, saved;
  ExactScope(bool &f, bool on) : flag(f), saved(f) { flag = flag || on; }
  ~ExactScope() { flag = saved; }
};

class Engine {
 public:
  Engine(int L, int device);
  ~Engine();

  int L() const { return L_; }
  int64_t V() const { return V_; }
  const Geom &geom() const { return g_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }

  // ---- device-pointer operations (asynchronous on stream(), FP64)
  void sigma_mass(const double *sigma, const double *P, double eps, double *sigma_out, double *sm);
  void dirac(const double *sm, const double *in, double *out, int ncomp, int op);
  void momenta(double *P, const double *F, double eps);
  void force(const double *X, const double *Y, const double *sigma, double beta_s, double *F, double *P, double pcoef);
  // H terms (sum P^2/2, sum 1/2 phi X, sum sigma^2), compensated; synchronises.
  void energy_terms(const double *P, const double *phi, const double *X, const double *sigma, double out[3]);
  // sum Re(conj v D)/V, sum Re(conj v D), sum Im(conj v D); synchronises.
  void cond_dots(const double *v, const double *D, double out[3]);
  // CondensateSigmaPi of a device sigma (fermion order), of |(sigma, pi)| when
  // pi is given (the U(1) model): the 8 outputs in the reference's argument order
  void sigma_observables(const double *sigma, const double *pi, double out[8]);
  void cond_fill(int mode, const signed char *signs, const double *table, const double *sm, double *v);

  // CG on M M^T for nrhs right-hand sides of ncomp planes each (b[k], x[k] are
  // device pointers of ncomp*V).  precision: GN_PREC_FP64 or GN_PREC_MIXED.
  // Synchronises and fills info[k].
  int solve(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol, int variant,
            int rel, long long max_iter, int precision, SolveInfo *info);

  // ---- resident sigma-HMC state
  double *sigma() { return sigma_[cur_]; }
  double *sigma_alt() { return sigma_[cur_ ^ 1]; }
  void swap_sigma() { cur_ ^= 1; }
  double *sm() { return sm_; }
  double *P() { return P_; }
  double *F() { return F_; }
  double *chi() { return chi_; }
  double *phi() { return phi_; }
  double *X() { return X_; }
  double *Y() { return Y_; }
  double *scratch(int i) { return scratch_[i]; }  // 4 scratch planes pairs of 2V
  signed char *signs() { return signs_; }
  double *table() { return table_; }
  double distance = 0.0;  // lat->distance_sigma of the resident state
  long long launches = 0; // kernels launched by this engine (for launch accounting)
  // Parity mode: M^T in the reference's scatter order and serial sums in the
  // energy and the condensate (set by gn_set_parity_mode and by the
  // operations run with precision GN_PREC_FP64_EXACT).
  bool exact = false;
  // trajectories run the MD alone on the resident P and phi (phi is not
  // formed from chi), as the reference's EvolveSigmaInTime* helpers
  bool keep_phi = false;
  int reliable_every = 100;  // mixed precision: a reliable update at least every this many iterations

  // One trajectory on the resident state; see gn_trajectory in gn_b200.h.
  int trajectory(const gn_hmc_params &hp, double (*gauss)(void), double (*uniform)(void), const double *pre_P,
                 const double *pre_chi, gn_traj_result *res);
  // The reference's EvolveSigmaInTime* helpers on the resident sigma, P, phi
  // and X (evolve_schedule); see gn_evolve_sigma_in_time in gn_b200.h.
  int evolve_in_time(const gn_hmc_params &hp, gn_traj_result *res);

  // Full condensate measurement (condensate.c:114-244) on device pointers.
  int condensate(const double *sm, double tol, double *target, double *D, double (*uniform)(void), double out[11],
                 double *iterations, long long *calls, int precision);

  // ---- the U(1) model (PI_INTERACTION), u1.cu; its state is allocated on
  // first use.  Complex fields are two planes (real, imaginary); a field of
  // both flavours is four planes (flavour f: planes 2f, 2f + 1).
  bool u1() const { return u1_; }
  void set_u1(bool on);  // allocates and zeroes pi on first use
  double *pi() { return pi_[pcur_]; }
  double *pi_alt() { return pi_[pcur_ ^ 1]; }
  void swap_pi() { pcur_ ^= 1; }
  double *pm() { return pm_; }
  double *Ppi() { return Ppi_; }
  double *Fpi() { return Fpi_; }
  double *chi_c() { return chi_c_; }
  double *phi_c() { return phi_c_; }
  double *X_c() { return X_c_; }
  double *Y_c() { return Y_c_; }
  // M, M^dagger or out - M psi with the complex mass on nsys complex systems
  void dirac_cm(const double *sm, const double *pm, const double *in, double *out, int nsys, int op);
  // CG on M M^dagger for nrhs complex systems (b[k], x[k]: 2V each);
  // precision GN_PREC_FP64 or GN_PREC_MIXED
  int solve_cm(const double *sm, const double *pm, const double *const *b, double *const *x, int nrhs, double tol,
               int variant, int rel, long long max_iter, SolveInfo *info, int precision = GN_PREC_FP64);
  // fermion force of sigma (pi = false) or pi (pi = true) from complex X, Y
  // (4V each), minus gcoef * field, with the fused step P += pcoef F if P
  void force_cm(bool pi, const double *X, const double *Y, const double *field, double gcoef, double *F, double *P,
                double pcoef);
  // (sum P^2/2, sum_f 1/2 Re(conj phi_f X_f), sum field^2); synchronises
  void energy_cm(const double *P, const double *phi, const double *X, const double *field, double out[3]);
  // LeapFrog2Pi (moleculardynamics.c:1743-1870) on the resident sigma, pi
  int trajectory_pi(const gn_hmc_params &hp, void (*gauss_pair)(double *, double *), double (*gauss)(void),
                    double (*uniform)(void), gn_traj_result *res);

  // failure-detection self-test: a team barrier whose partner block never
  // arrives runs out of polls; returns GN_ERR_TIMEOUT (selftest.cu)
  int selftest_wait_timeout();

  // host staging (pinned), at least 4*V doubles
  double *host_stage() { return h_stage_; }
  int *abort_flag_host() { return h_abort_; }

  void check(cudaError_t e, const char *what);

 private:
  int finish_solve(int nrhs, SolveInfo *info);
  // pm: the U(1) model's pi mass (complex systems with the mass sm + i eps pm), else null
  int solve_exact(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                  int variant, int rel, long long max_iter, SolveInfo *info, const double *pm = nullptr);
  void mt_exact(const double *sm, const double *in, double *out, int ncomp);
  void mt_exact_cm(const double *sm, const double *pm, const double *in, double *out, int nsys);
  void energy_exact(const double *P, const double *phi, const double *X, const double *sigma, double out[3]);
  void energy_cm_exact(const double *P, const double *phi, const double *X, const double *field, double out[3]);
  void energy_launch(const double *P, const double *phi, const double *X, const double *sigma, double *dst);
  void cond_dots_exact(const double *v, const double *D, double out[4]);
  void mixed_init();
  const void *mixed_kernel_ptr(int ncomp, int nrhs, int w);
  const void *fp64_kernel_ptr(int ncomp, int nrhs, int w);
  // pm != nullptr: the U(1) model's complex mass (ncomp = 2)
  int solve_mixed(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                  int variant, int rel, long long max_iter, SolveInfo *info, const double *pm = nullptr);
  void *alloc(size_t bytes);
  int cg_blocks(int ncomp, int nrhs, bool mixed, int w);
  int trajectory_u1(const gn_hmc_params &hp, double (*gauss)(void), double (*uniform)(void), const double *pre_P,
                    const double *pre_chi, gn_traj_result *res);

  int L_, device_;
  int64_t V_;
  Geom g_;
  cudaStream_t stream_ = nullptr;
  int num_sms_ = 0;
  std::vector<void *> allocs_;
  double *sigma_[2] = {nullptr, nullptr};
  int cur_ = 0;
  double *sm_ = nullptr, *P_ = nullptr, *F_ = nullptr;
  double *chi_ = nullptr, *phi_ = nullptr, *X_ = nullptr, *Y_ = nullptr;
  double *scratch_[4] = {nullptr, nullptr, nullptr, nullptr};
  signed char *signs_ = nullptr;
  double *table_ = nullptr;
  // solver workspace
  double *cg_work_ = nullptr;  // kMaxRhs * 4 vectors * 2 planes * V
  float *mx_work_ = nullptr;   // mixed precision: kMaxRhs * 5 vectors * 2 planes * V
  float *sm32_ = nullptr;
  float *pm32_ = nullptr;  // the U(1) model: FP32 copy of the pi mass
  // the second system of a two-team mixed solve (cg_mixed_duo_kernel): its
  // arrival counter and its FP32 copy of sm (each team writes its own)
  PhaseBar *bar2_ = nullptr;
  float *sm32b_ = nullptr;
  float *pm32b_ = nullptr;  // ... and of the pi mass (the U(1) model)
  bool mixed_duo_ = true;
  double *partials_ = nullptr;
  double *h_partials_ = nullptr;
  PhaseBar *bar_ = nullptr;
  int *err_ = nullptr;
  CgState *state_ = nullptr;  // the solvers' state slots (traj_states_ slots in a deferred trajectory)
  CgState *h_state_ = nullptr;
  CgState *state_base_ = nullptr;
  // a trajectory queued without a host round trip per solve (trajectory()):
  // finish_solve then returns at once, and the states and energies are read
  // back together at the end
  bool defer_ = false;
  static constexpr int kTrajSolves = 256;  // two-flavour solves of one deferred trajectory, at most
  CgState *traj_states_ = nullptr, *h_traj_states_ = nullptr;
  double *traj_partials_ = nullptr, *h_traj_partials_ = nullptr;
  int *h_abort_ = nullptr;
  int *d_abort_ = nullptr;
  double *h_stage_ = nullptr;
  int max_blocks_ = 0;
  int cg_blocks_cache_[2][2][kMaxRhs][3] = {};  // [mixed][ncomp-1][nrhs-1][log2 w]
  // U(1) model
  bool u1_ = false;
  double *pi_[2] = {nullptr, nullptr};
  int pcur_ = 0;
  double *pm_ = nullptr, *Ppi_ = nullptr, *Fpi_ = nullptr;
  double *chi_c_ = nullptr, *phi_c_ = nullptr, *X_c_ = nullptr, *Y_c_ = nullptr;
};

// Host-side compensated sum of (hi, lo) block partials.
double sum_partials(const double *part, int nb, int q);
// Blocks of the elementwise kernels.
int op_blocks(int64_t V, int num_sms);
// kit->iterations / kit->CG_call bookkeeping of a flavour loop that stops at
// the first failure (moleculardynamics.c:593-597).
void count_flavours(const SolveInfo *info, int n, double &iters, long long &calls, long long &inner, long long &rel);

}  // namespace gn
