// u1.cu -- the U(1) Gross-Neveu model (the reference's PI_INTERACTION): the
// complex-mass operators, the FP64 CG on M M^dagger, the sigma and pi forces
// and energies on complex fermion fields, the sigma integrators over them and
// LeapFrog2Pi.  Built with --fmad=false: the FP64 results follow the
// reference's operations (its complex products as C forms them).
//
// Fields: sigma, pi and their masses are real (V); fermion fields are
// complex, two planes each; both flavours of one are four planes (flavour f:
// planes 2f, 2f + 1).  chi stays real as the reference draws it (fermion.c:
// 337-345), so its imaginary planes are zero.
#include <cmath>
#include <cstring>

#include "engine.h"
#include "errors.h"
#include "launch.h"
#include "ops_kernels.cuh"
#include "schedule.h"
#include "trace.h"

namespace gn {

void Engine::set_u1(bool on) {
  if (on && pi_[0] == nullptr) {
    const size_t V = size_t(V_), d = sizeof(double);
    pi_[0] = (double *)alloc(V * d);
    pi_[1] = (double *)alloc(V * d);
    pm_ = (double *)alloc(V * d);
    Ppi_ = (double *)alloc(V * d);
    Fpi_ = (double *)alloc(V * d);
    chi_c_ = (double *)alloc(4 * V * d);
    phi_c_ = (double *)alloc(4 * V * d);
    X_c_ = (double *)alloc(4 * V * d);
    Y_c_ = (double *)alloc(4 * V * d);
    check(cudaStreamSynchronize(stream_), "u1 state");
  }
  u1_ = on;
}

void Engine::dirac_cm(const double *sm, const double *pm, const double *in, double *out, int nsys, int op) {
  if (exact && op == GN_OP_MT) {  // parity mode: the reference's scatter order
    mt_exact_cm(sm, pm, in, out, nsys);
    return;
  }
  const void *ptrs[4] = {sm, pm, in, out};
  const int W = fp64_width(L_, ptrs, 4);
  const dim3 grid(unsigned((V_ / W + kOpThreads - 1) / kOpThreads), unsigned(nsys));
  if (W == 2) {
    if (op == GN_OP_M) dirac_cm_kernel<2, 0><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
    else if (op == GN_OP_MT) dirac_cm_kernel<2, 1><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
    else dirac_cm_kernel<2, 2><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
  } else {
    if (op == GN_OP_M) dirac_cm_kernel<1, 0><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
    else if (op == GN_OP_MT) dirac_cm_kernel<1, 1><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
    else dirac_cm_kernel<1, 2><<<grid, kOpThreads, 0, stream_>>>(g_, sm, pm, in, out);
  }
  check(cudaGetLastError(), "dirac_cm_kernel");
  launches++;
}

template <int W>
static const void *cm_kernel(int nr) {
  return nr == 1 ? (const void *)cg_kernel<double, 2, 1, kSolverThreads, W, true>
                 : (const void *)cg_kernel<double, 2, 2, kSolverThreads, W, true>;
}

int Engine::solve_cm(const double *sm, const double *pm, const double *const *b, double *const *x, int nrhs,
                     double tol, int variant, int rel, long long max_iter, SolveInfo *info, int precision) {
  TraceRange tr(precision == GN_PREC_MIXED ? "gn cg u1 mixed" : "gn cg u1 fp64");
  if (nrhs < 1 || nrhs > 2) throw GnError(GN_ERR_ARG, "the U(1) solve takes 1 or 2 systems");
  if (precision != GN_PREC_FP64 && precision != GN_PREC_MIXED && precision != GN_PREC_FP64_EXACT)
    throw GnError(GN_ERR_ARG, "unknown precision");
  if (max_iter <= 0) max_iter = V_ + 1;  // MAX_CONJUGATE_GRADIENT_ITERATION, macro.h:134
  if (precision == GN_PREC_MIXED) return solve_mixed(sm, b, x, nrhs, 2, tol, variant, rel, max_iter, info, pm);
  if (precision == GN_PREC_FP64_EXACT) return solve_exact(sm, b, x, nrhs, 2, tol, variant, rel, max_iter, info, pm);
  const size_t V = size_t(V_);
  CgArgs<double> a;
  memset(&a, 0, sizeof a);
  a.g = g_;
  a.sm = sm;
  a.pm = pm;
  for (int k = 0; k < nrhs; k++) {
    double *w = cg_work_ + size_t(k) * kNumWorkVecs * 2 * V;
    a.b[k] = b[k];
    a.x[k] = x[k];
    a.r[k] = w;
    a.p0[k] = w + 2 * V;
    a.p1[k] = w + 4 * V;
    a.t[k] = w + 6 * V;
  }
  a.nrhs = nrhs;
  a.variant = variant;
  a.rel = rel;
  a.tol = tol;
  a.max_iter = max_iter;
  a.partials = partials_;
  a.bar = bar_;
  a.err = err_;
  a.abort_flag = d_abort_;
  a.state = state_;
  check(cudaMemsetAsync(bar_, 0, sizeof(PhaseBar), stream_), "memset");
  check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  const void *ptrs[2 * kMaxRhs + 2] = {sm, pm};
  for (int k = 0; k < nrhs; k++) {
    ptrs[2 + 2 * k] = b[k];
    ptrs[3 + 2 * k] = x[k];
  }
  const int w = fp64_width(L_, ptrs, 2 + 2 * nrhs);
  const int nr = rhs_slots(nrhs);
  const void *fn = w == 2 ? cm_kernel<2>(nr) : cm_kernel<1>(nr);
  const int capacity = coop_capacity(fn, kSolverThreads);
  if (capacity < 1) throw GnError(GN_ERR_CUDA, "CG kernel cannot be resident as a cooperative grid");
  const int nb = solver_grid(solver_units(V_, w, nrhs), capacity, max_blocks_, kSolverThreads);
  check(launch_solver(fn, nb, kSolverThreads, a, stream_), "cg_kernel (U(1)) launch");
  launches++;
  return finish_solve(nrhs, info);
}

void Engine::force_cm(bool pi, const double *X, const double *Y, const double *field, double gcoef, double *F,
                      double *P, double pcoef) {
  if (pi)
    force_cm_kernel<true><<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(g_, X, Y, field, gcoef, F, P, pcoef);
  else
    force_cm_kernel<false><<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(g_, X, Y, field, gcoef, F, P, pcoef);
  check(cudaGetLastError(), "force_cm_kernel");
  launches++;
}

void Engine::energy_cm(const double *P, const double *phi, const double *X, const double *field, double out[3]) {
  if (exact) {  // parity mode: the reference's serial sums
    energy_cm_exact(P, phi, X, field, out);
    return;
  }
  const int nb = op_blocks(V_, num_sms_);
  energy_cm_kernel<<<nb, kOpThreads, 0, stream_>>>(uint32_t(V_), P, phi, X, field, partials_);
  check(cudaGetLastError(), "energy_cm_kernel");
  launches++;
  check(cudaMemcpyAsync(h_partials_, partials_, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "energy sync");
  for (int q = 0; q < 3; q++) out[q] = sum_partials(h_partials_, nb, q);
}

namespace {

// chi_f (real draws, V each) -> complex planes; phi_f = M chi_f
void load_chi(Engine &E, const double *host_chi, const double *dev_chi) {
  const size_t V = size_t(E.V());
  double *c = E.chi_c();
  for (int f = 0; f < 2; f++) {
    double *re = c + size_t(2 * f) * V;
    if (host_chi)
      E.check(cudaMemcpyAsync(re, host_chi + size_t(f) * V, V * sizeof(double), cudaMemcpyHostToDevice, E.stream()),
              "upload chi");
    else
      E.check(cudaMemcpyAsync(re, dev_chi + size_t(f) * V, V * sizeof(double), cudaMemcpyDeviceToDevice, E.stream()),
              "copy chi");
    E.check(cudaMemsetAsync(re + V, 0, V * sizeof(double), E.stream()), "chi imaginary part");
  }
}

}  // namespace

// The sigma integrators (the schedules of schedule.h) with the complex M.
int Engine::trajectory_u1(const gn_hmc_params &hp, double (*gauss)(void), double (*uniform)(void), const double *pre_P,
                          const double *pre_chi, gn_traj_result *res) {
  TraceRange tr("gn trajectory u1");
  if (hp.precision != GN_PREC_FP64 && hp.precision != GN_PREC_MIXED && hp.precision != GN_PREC_FP64_EXACT)
    throw GnError(GN_ERR_ARG, "unknown precision");
  ExactScope exact_scope(exact, hp.precision == GN_PREC_FP64_EXACT);
  const size_t V = size_t(V_);
  memset(res, 0, sizeof *res);
  // draws: P, chi_0, chi_1 (moleculardynamics.c:1240-1247)
  if (gauss != nullptr) {
    double *h = h_stage_;
    for (size_t i = 0; i < 3 * V; i++) h[i] = gauss();
    check(cudaMemcpyAsync(P_, h, V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload P");
    load_chi(*this, h + V, nullptr);
  } else {
    if (pre_P) check(cudaMemcpyAsync(P_, pre_P, V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy P");
    if (pre_chi) load_chi(*this, nullptr, pre_chi);
  }
  if (!keep_phi) dirac_cm(sm_, pm_, chi_c_, phi_c_, 2, GN_OP_M);
  double *sigma_copy = scratch_[3];
  check(cudaMemcpyAsync(sigma_copy, sigma(), V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy sigma");
  auto restore = [&]() {
    check(cudaMemcpyAsync(sigma(), sigma_copy, V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "restore");
    sigma_mass(sigma(), nullptr, 0.0, nullptr, sm_);
  };
  const double *phis[2] = {phi_c_, phi_c_ + 2 * V};
  double *Xs[2] = {X_c_, X_c_ + 2 * V};
  SolveInfo info[2];
  double iters = 0.0;
  long long calls = 0, inner = 0, rel = 0;
  auto finish = [&](int ok) {
    res->ok = ok;
    res->cg_iterations = iters;
    res->cg_calls = calls;
    res->inner_iterations = inner;
    res->reliable_updates = rel;
  };
  auto fail = [&]() {
    restore();
    check(cudaStreamSynchronize(stream_), "restore");
    finish(0);
    return GN_NOT_CONVERGED;
  };
  int st = solve_cm(sm_, pm_, phis, Xs, 2, hp.tol_high, 1, hp.relative, 0, info, hp.precision);
  count_flavours(info, 2, iters, calls, inner, rel);
  if (st != GN_OK) return fail();
  const double ccoef = (4 * hp.beta_s / 4.0);  // (NFLAV * beta_scalar / 4.0), moleculardynamics.c:316
  const double gcoef = (4 * hp.beta_s / 2.0);  // (NFLAV * beta_scalar / 2.0), moleculardynamics.c:580
  double e[3];
  energy_cm(P_, phi_c_, X_c_, sigma(), e);
  const double h0 = (e[0] + e[1]) + ccoef * e[2];
  const std::vector<Op> ops = schedule(hp.integrator, hp.eps, hp.steps);
  for (size_t k = 0; k < ops.size(); k++) {
    const Op &o = ops[k];
    if (o.op == OP_F_MED || o.op == OP_F_HIGH) {
      const double tol = o.op == OP_F_MED ? hp.tol_medium : hp.tol_high;
      st = solve_cm(sm_, pm_, phis, Xs, 2, tol, 0, hp.relative, 0, info, hp.precision);
      count_flavours(info, 2, iters, calls, inner, rel);
      if (st != GN_OK) return fail();
      dirac_cm(sm_, pm_, X_c_, Y_c_, 2, GN_OP_MT);
      if (k + 1 < ops.size() && ops[k + 1].op == OP_P) {
        force_cm(false, X_c_, Y_c_, sigma(), gcoef, F_, P_, ops[k + 1].c);
        k++;
      } else {
        force_cm(false, X_c_, Y_c_, sigma(), gcoef, F_, nullptr, 0.0);
      }
    } else if (o.op == OP_P) {
      momenta(P_, F_, o.c);
    } else if (o.op == OP_Q) {
      sigma_mass(sigma(), P_, o.c, sigma_alt(), sm_);
      swap_sigma();
      distance += o.c;
      res->distance += o.c;
    } else {
      st = solve_cm(sm_, pm_, phis, Xs, 2, hp.tol_high, 1, hp.relative, 0, info, hp.precision);
      count_flavours(info, 2, iters, calls, inner, rel);
      if (st != GN_OK) return fail();
    }
  }
  energy_cm(P_, phi_c_, X_c_, sigma(), e);
  const double h1 = (e[0] + e[1]) + ccoef * e[2];
  res->H0 = h0;
  res->H1 = h1;
  res->dH = h1 - h0;
  const int acc = uniform != nullptr ? (uniform() <= std::exp(-(h1 - h0))) : 1;
  res->accepted = acc;
  if (!acc) restore();
  check(cudaStreamSynchronize(stream_), "trajectory");
  finish(1);
  return GN_OK;
}

// LeapFrog2Pi (moleculardynamics.c:1743-1870): draws P_pi (pairs, as
// DrawPiMomentaFromGaussianDistribution draws them), then chi_f and
// phi_f = M chi_f; every inversion is ConjugateGradientFastDiracAdjFast-
// DiracToTheMinusOne (variant 0) at hp.tol_high, as ComputePiForce calls it.
//   F, P += F eps/2; (Q eps, F, P += F eps) x (step - 1); Q eps, F, P += F eps/2
// with H = sum P^2/2 + sum_f 1/2 Re(conj phi_f X_f) + (N_f beta_s / 8) sum pi^2.
int Engine::trajectory_pi(const gn_hmc_params &hp, void (*gauss_pair)(double *, double *), double (*gauss)(void),
                          double (*uniform)(void), gn_traj_result *res) {
  TraceRange tr("gn trajectory pi");
  if (!u1_) throw GnError(GN_ERR_ARG, "the context is not in the U(1) model (load pi first)");
  if (hp.steps < 1) throw GnError(GN_ERR_ARG, "steps must be >= 1");
  if (hp.precision != GN_PREC_FP64 && hp.precision != GN_PREC_MIXED && hp.precision != GN_PREC_FP64_EXACT)
    throw GnError(GN_ERR_ARG, "unknown precision");
  ExactScope exact_scope(exact, hp.precision == GN_PREC_FP64_EXACT);
  const size_t V = size_t(V_);
  memset(res, 0, sizeof *res);
  double *h = h_stage_;
  if (gauss_pair != nullptr) {  // DrawPiMomentaFromGaussianDistribution (moleculardynamics.c:810-815)
    for (size_t x = 0; x < V / 2; x++) gauss_pair(&h[x], &h[x + V / 2]);
    check(cudaMemcpyAsync(Ppi_, h, V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload P pi");
  }
  if (gauss != nullptr) {  // then chi_0, chi_1 (DrawFullFermionFromGaussianDistribution)
    for (size_t i = 0; i < 2 * V; i++) h[V + i] = gauss();
    load_chi(*this, h + V, nullptr);
  }
  dirac_cm(sm_, pm_, chi_c_, phi_c_, 2, GN_OP_M);
  double *pi_copy = scratch_[3];
  check(cudaMemcpyAsync(pi_copy, pi(), V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy pi");
  auto restore = [&]() {
    check(cudaMemcpyAsync(pi(), pi_copy, V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "restore pi");
    sigma_mass(pi(), nullptr, 0.0, nullptr, pm_);  // ComputeFullPiMass: the same 8-corner mean
  };
  const double *phis[2] = {phi_c_, phi_c_ + 2 * V};
  double *Xs[2] = {X_c_, X_c_ + 2 * V};
  SolveInfo info[2];
  double iters = 0.0;
  long long calls = 0, inner = 0, rel = 0;
  auto finish = [&](int ok) {
    res->ok = ok;
    res->cg_iterations = iters;
    res->cg_calls = calls;
    res->inner_iterations = inner;
    res->reliable_updates = rel;
  };
  auto fail = [&]() {
    restore();
    check(cudaStreamSynchronize(stream_), "restore");
    finish(0);
    return GN_NOT_CONVERGED;
  };
  const double ecoef = (4 * hp.beta_s / 8.0);  // (NFLAV * beta_scalar / 8.0), moleculardynamics.c:365
  const double gcoef = (4 * hp.beta_s / 4.0);  // (NFLAV * beta_scalar / 4.0), moleculardynamics.c:685
  auto pi_force = [&](double pcoef) {  // ComputePiForce, then P_pi += pcoef F_pi
    const int s = solve_cm(sm_, pm_, phis, Xs, 2, hp.tol_high, 0, hp.relative, 0, info, hp.precision);
    count_flavours(info, 2, iters, calls, inner, rel);
    if (s != GN_OK) return false;
    dirac_cm(sm_, pm_, X_c_, Y_c_, 2, GN_OP_MT);
    force_cm(true, X_c_, Y_c_, pi(), gcoef, Fpi_, Ppi_, pcoef);
    return true;
  };
  auto pi_step = [&](double eps) {  // EvolveCoordinatesPi: pi += eps P, then pi mass
    sigma_mass(pi(), Ppi_, eps, pi_alt(), pm_);
    swap_pi();
  };
  int st = solve_cm(sm_, pm_, phis, Xs, 2, hp.tol_high, 0, hp.relative, 0, info, hp.precision);
  count_flavours(info, 2, iters, calls, inner, rel);
  if (st != GN_OK) return fail();
  double e[3];
  energy_cm(Ppi_, phi_c_, X_c_, pi(), e);
  const double h0 = (e[0] + e[1]) + ecoef * e[2];
  if (!pi_force(hp.eps / 2.0)) return fail();
  for (int s = 0; s < hp.steps - 1; s++) {
    pi_step(hp.eps);
    if (!pi_force(hp.eps)) return fail();
  }
  pi_step(hp.eps);
  if (!pi_force(hp.eps / 2.0)) return fail();
  energy_cm(Ppi_, phi_c_, X_c_, pi(), e);
  const double h1 = (e[0] + e[1]) + ecoef * e[2];
  res->H0 = h0;
  res->H1 = h1;
  res->dH = h1 - h0;
  const int acc = uniform != nullptr ? (uniform() <= std::exp(-(h1 - h0))) : 1;
  res->accepted = acc;
  if (!acc) restore();
  check(cudaStreamSynchronize(stream_), "trajectory pi");
  finish(1);
  return GN_OK;
}

}  // namespace gn
