// engine.cu -- device engine of the sigma-HMC fermion path (FP64 kernels).
// Built with --fmad=false: the FP64 kernels follow the reference's rounding
// (mul then add) wherever the reference's result is reproducible bit for bit.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "engine.h"
#include "schedule.h"
#include "errors.h"
#include "launch.h"
#include "ops_kernels.cuh"
#include "trace.h"

namespace gn {


void Engine::check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    throw GnError(GN_ERR_CUDA, buf);
  }
}

void *Engine::alloc(size_t bytes) {
  void *p = nullptr;
  check(cudaMalloc(&p, bytes), "cudaMalloc");
  allocs_.push_back(p);
  check(cudaMemsetAsync(p, 0, bytes, stream_), "cudaMemsetAsync");
  return p;
}

Engine::Engine(int L, int device) : L_(L), device_(device) {
  if (L < 4 || L > 256 || (L & 1)) throw GnError(GN_ERR_ARG, "L must be even and in [4, 256]");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    throw GnError(GN_ERR_NO_DEVICE, "no such CUDA device");
  check(cudaSetDevice(device), "cudaSetDevice");
  cudaDeviceProp prop;
  check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major != 10) throw GnError(GN_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only");
  if (!prop.cooperativeLaunch) throw GnError(GN_ERR_NO_DEVICE, "device lacks cooperative launch");
  num_sms_ = prop.multiProcessorCount;
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  g_ = make_geom(L);
  V_ = g_.V;
  const size_t V = size_t(V_);
  const size_t d = sizeof(double);
  sigma_[0] = (double *)alloc(V * d);
  sigma_[1] = (double *)alloc(V * d);
  sm_ = (double *)alloc(V * d);
  P_ = (double *)alloc(V * d);
  F_ = (double *)alloc(V * d);
  chi_ = (double *)alloc(2 * V * d);
  phi_ = (double *)alloc(2 * V * d);
  X_ = (double *)alloc(2 * V * d);
  Y_ = (double *)alloc(2 * V * d);
  for (int i = 0; i < 4; i++) scratch_[i] = (double *)alloc(2 * V * d);
  signs_ = (signed char *)alloc(V);
  table_ = (double *)alloc(2 * 256 * d);
  cg_work_ = (double *)alloc(size_t(kMaxRhs) * kNumWorkVecs * 2 * V * d);
  max_blocks_ = num_sms_ * 8;
  partials_ = (double *)alloc(size_t(32) * max_blocks_ * d);
  bar_ = (PhaseBar *)alloc(sizeof(PhaseBar));
  err_ = (int *)alloc(sizeof(int));
  state_ = (CgState *)alloc(sizeof(CgState) * kMaxRhs);
  state_base_ = state_;
  traj_states_ = (CgState *)alloc(sizeof(CgState) * 2 * kTrajSolves);
  traj_partials_ = (double *)alloc(sizeof(double) * 12 * op_blocks(V_, num_sms_));
  check(cudaHostAlloc((void **)&h_traj_states_, sizeof(CgState) * 2 * kTrajSolves, cudaHostAllocDefault),
        "cudaHostAlloc");
  check(cudaHostAlloc((void **)&h_traj_partials_, sizeof(double) * 12 * op_blocks(V_, num_sms_),
                      cudaHostAllocDefault), "cudaHostAlloc");
  check(cudaHostAlloc((void **)&h_partials_, size_t(32) * max_blocks_ * d, cudaHostAllocDefault), "cudaHostAlloc");
  check(cudaHostAlloc((void **)&h_state_, sizeof(CgState) * kMaxRhs, cudaHostAllocDefault), "cudaHostAlloc");
  check(cudaHostAlloc((void **)&h_abort_, sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
  *h_abort_ = 0;
  check(cudaHostGetDevicePointer((void **)&d_abort_, h_abort_, 0), "cudaHostGetDevicePointer");
  check(cudaHostAlloc((void **)&h_stage_, 4 * V * d, cudaHostAllocDefault), "cudaHostAlloc");
  mixed_init();
  check(cudaStreamSynchronize(stream_), "init");
}

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (void *p : allocs_) cudaFree(p);
  if (h_partials_) cudaFreeHost(h_partials_);
  if (h_state_) cudaFreeHost(h_state_);
  if (h_traj_states_) cudaFreeHost(h_traj_states_);
  if (h_traj_partials_) cudaFreeHost(h_traj_partials_);
  if (h_abort_) cudaFreeHost(h_abort_);
  if (h_stage_) cudaFreeHost(h_stage_);
  if (stream_) cudaStreamDestroy(stream_);
}

int op_blocks(int64_t V, int num_sms) {
  int64_t b = (V + kOpThreads - 1) / kOpThreads;
  int64_t cap = int64_t(num_sms) * (2048 / kOpThreads);
  return int(b < cap ? b : cap);
}

void Engine::sigma_mass(const double *sigma, const double *P, double eps, double *sigma_out, double *sm) {
  sigma_mass_kernel<double><<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(g_, sigma, P, eps, sigma_out, sm);
  check(cudaGetLastError(), "sigma_mass_kernel");
  launches++;
}

void Engine::dirac(const double *sm, const double *in, double *out, int ncomp, int op) {
  if (exact && op == GN_OP_MT) {
    mt_exact(sm, in, out, ncomp);
    return;
  }
  // W sites per thread (rowvec.cuh), 128-bit loads when L/2 is even and the arrays are 16-byte aligned
  const void *ptrs[3] = {sm, in, out};
  const int W = fp64_width(L_, ptrs, 3);
  const dim3 grid(unsigned((V_ / W + kOpThreads - 1) / kOpThreads), unsigned(ncomp));
  if (W == 2) {
    if (op == GN_OP_M) dirac_item_kernel<2, 0><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
    else if (op == GN_OP_MT) dirac_item_kernel<2, 1><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
    else dirac_item_kernel<2, 2><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
  } else {
    if (op == GN_OP_M) dirac_item_kernel<1, 0><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
    else if (op == GN_OP_MT) dirac_item_kernel<1, 1><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
    else dirac_item_kernel<1, 2><<<grid, kOpThreads, 0, stream_>>>(g_, sm, in, out);
  }
  check(cudaGetLastError(), "dirac_item_kernel");
  launches++;
}

void Engine::momenta(double *P, const double *F, double eps) {
  momenta_kernel<double><<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(uint32_t(V_), P, F, eps);
  check(cudaGetLastError(), "momenta_kernel");
  launches++;
}

void Engine::force(const double *X, const double *Y, const double *sigma, double beta_s, double *F, double *P,
                   double pcoef) {
  TraceRange tr("gn sigma force");
  const double gcoef = (4 * beta_s / 2.0);  // (NFLAV * beta_scalar / 2.0), moleculardynamics.c:580
  force_kernel<double><<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(g_, X, Y, sigma, gcoef, F, P, pcoef);
  check(cudaGetLastError(), "force_kernel");
  launches++;
}

double sum_partials(const double *part, int nb, int q) {
  // Neumaier over the block (hi, lo) pairs
  double s = 0.0, c = 0.0;
  for (int b = 0; b < nb; b++) {
    for (int h = 0; h < 2; h++) {
      const double v = part[(size_t(q) * nb + b) * 2 + h];
      const double t = s + v;
      if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v;
      else c += (v - t) + s;
      s = t;
    }
  }
  return s + c;
}

void Engine::energy_terms(const double *P, const double *phi, const double *X, const double *sigma, double out[3]) {
  if (exact) {
    energy_exact(P, phi, X, sigma, out);
    return;
  }
  const int nb = op_blocks(V_, num_sms_);
  energy_kernel<double><<<nb, kOpThreads, 0, stream_>>>(uint32_t(V_), P, phi, X, sigma, partials_);
  check(cudaGetLastError(), "energy_kernel");
  launches++;
  check(cudaMemcpyAsync(h_partials_, partials_, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "energy sync");
  for (int q = 0; q < 3; q++) out[q] = sum_partials(h_partials_, nb, q);
}

// The energy kernel's partial sums (6 per block) into dst, without a host copy.
void Engine::energy_launch(const double *P, const double *phi, const double *X, const double *sigma, double *dst) {
  const int nb = op_blocks(V_, num_sms_);
  energy_kernel<double><<<nb, kOpThreads, 0, stream_>>>(uint32_t(V_), P, phi, X, sigma, dst);
  check(cudaGetLastError(), "energy_kernel");
  launches++;
}

void Engine::cond_dots(const double *v, const double *D, double out[3]) {
  const int nb = op_blocks(V_, num_sms_);
  cond_dot_kernel<<<nb, kOpThreads, 0, stream_>>>(uint32_t(V_), v, D, partials_);
  check(cudaGetLastError(), "cond_dot_kernel");
  launches++;
  check(cudaMemcpyAsync(h_partials_, partials_, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "dots sync");
  for (int q = 0; q < 3; q++) out[q] = sum_partials(h_partials_, nb, q);
}

void Engine::sigma_observables(const double *sigma, const double *pi, double out[8]) {
  const int nb = op_blocks(V_, num_sms_);
  sigma_obs_kernel<<<nb, kOpThreads, 0, stream_>>>(g_, sigma, pi, partials_);
  check(cudaGetLastError(), "sigma_obs_kernel");
  launches++;
  check(cudaMemcpyAsync(h_partials_, partials_, sizeof(double) * 2 * kSigmaObsSums * nb, cudaMemcpyDeviceToHost,
                        stream_),
        "copy");
  check(cudaStreamSynchronize(stream_), "sigma observables sync");
  double sums[kSigmaObsSums], o[kSigmaObs];
  for (int q = 0; q < kSigmaObsSums; q++) sums[q] = sum_partials(h_partials_, nb, q);
  sigma_obs_finish(sums, double(V_), o);
  for (int q = 0; q < kSigmaObs; q++) out[q] = o[q];
}

void Engine::cond_fill(int mode, const signed char *signs, const double *table, const double *sm, double *v) {
  cond_fill_kernel<<<op_blocks(V_, num_sms_), kOpThreads, 0, stream_>>>(g_, mode, signs, table, sm, v);
  check(cudaGetLastError(), "cond_fill_kernel");
  launches++;
}

template <int W>
static const void *fp64_kernel(int ncomp, int nr) {
  if (ncomp == 1) {
    if (nr == 1) return (const void *)cg_kernel<double, 1, 1, kWideThreads, W>;
    if (nr == 2) return (const void *)cg_kernel<double, 1, 2, kWideThreads, W>;
    return (const void *)cg_kernel<double, 1, 4, kSolverThreads, W>;
  }
  if (nr == 1) return (const void *)cg_kernel<double, 2, 1, kSolverThreads, W>;
  if (nr == 2) return (const void *)cg_kernel<double, 2, 2, kSolverThreads, W>;
  throw GnError(GN_ERR_ARG, "complex systems: at most 2 right-hand sides per solve");
}

const void *Engine::fp64_kernel_ptr(int ncomp, int nrhs, int w) {
  const int nr = rhs_slots(nrhs);
  return w == 2 ? fp64_kernel<2>(ncomp, nr) : fp64_kernel<1>(ncomp, nr);
}

// Grid of a solve (cached per kernel and system count): one work unit per
// thread of its hot sweeps (the FP64 ones of the FP64 solver, the FP32 ones of
// the mixed solver, whose rarer FP64 sweeps then take two rounds).
int Engine::cg_blocks(int ncomp, int nrhs, bool mixed, int w) {
  int &cached = cg_blocks_cache_[mixed ? 1 : 0][ncomp - 1][nrhs - 1][w == 4 ? 2 : w - 1];
  if (cached) return cached;
  const void *fn = mixed ? mixed_kernel_ptr(ncomp, nrhs, w) : fp64_kernel_ptr(ncomp, nrhs, w);
  const int bs = threads_for(ncomp, nrhs);
  const int capacity = coop_capacity(fn, bs);
  if (capacity < 1) throw GnError(GN_ERR_CUDA, "CG kernel cannot be resident as a cooperative grid");
  cached = solver_grid(solver_units(V_, w, nrhs), capacity, max_blocks_, bs);
  return cached;
}

int Engine::solve(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                  int variant, int rel, long long max_iter, int precision, SolveInfo *info) {
  TraceRange tr(precision == GN_PREC_MIXED ? "gn cg mixed" : "gn cg fp64");
  if (nrhs < 1 || nrhs > kMaxRhs || ncomp < 1 || ncomp > 2) throw GnError(GN_ERR_ARG, "bad nrhs / ncomp");
  if (max_iter <= 0) max_iter = V_ + 1;  // MAX_CONJUGATE_GRADIENT_ITERATION, macro.h:134
  if (precision == GN_PREC_MIXED) return solve_mixed(sm, b, x, nrhs, ncomp, tol, variant, rel, max_iter, info);
  if (precision == GN_PREC_FP64_EXACT) return solve_exact(sm, b, x, nrhs, ncomp, tol, variant, rel, max_iter, info);
  const size_t V = size_t(V_);
  CgArgs<double> a;
  memset(&a, 0, sizeof a);
  a.g = g_;
  a.sm = sm;
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
  if (!defer_) check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  const void *ptrs[2 * kMaxRhs + 1] = {sm};
  for (int k = 0; k < nrhs; k++) {
    ptrs[1 + 2 * k] = b[k];
    ptrs[2 + 2 * k] = x[k];
  }
  const int w = fp64_width(L_, ptrs, 1 + 2 * nrhs);
  const int nb = cg_blocks(ncomp, nrhs, false, w);
  check(launch_solver(fp64_kernel_ptr(ncomp, nrhs, w), nb, threads_for(ncomp, nrhs), a, stream_),
        "cg_kernel launch");
  launches++;
  return finish_solve(nrhs, info);
}

int Engine::finish_solve(int nrhs, SolveInfo *info) {
  if (defer_) return GN_OK;  // the caller reads the states when its queue is done
  int h_err = 0;
  check(cudaMemcpyAsync(h_state_, state_, sizeof(CgState) * nrhs, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaMemcpyAsync(&h_err, err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "cg sync");
  if (h_err == 1) throw GnError(GN_ERR_TIMEOUT, "CG grid barrier timed out");
  if (h_err == 2) throw GnError(GN_ERR_ABORTED, "CG aborted on request");
  bool all = true;
  for (int k = 0; k < nrhs; k++) {
    info[k].status = h_state_[k].status;
    info[k].iters = h_state_[k].iters;
    info[k].r2 = h_state_[k].r2;
    info[k].b2 = h_state_[k].b2;
    info[k].inner = h_state_[k].iters;
    info[k].reliable = h_state_[k].reliable;
    if (info[k].status != kCgConverged && info[k].status != kCgConvergedStart) all = false;
  }
  return all ? GN_OK : GN_NOT_CONVERGED;
}

// ------------------------------------------------------------------ trajectory
// kit->iterations / kit->CG_call bookkeeping of a flavour loop that stops at
// the first failure (moleculardynamics.c:593-597).
void count_flavours(const SolveInfo *info, int n, double &iters, long long &calls, long long &inner,
                           long long &rel) {
  for (int k = 0; k < n; k++) {
    if (info[k].status == kCgConverged) {
      iters += double(info[k].iters);
      calls++;
    }
    inner += info[k].inner;
    rel += info[k].reliable;
    if (info[k].status != kCgConverged && info[k].status != kCgConvergedStart) break;
  }
}

int Engine::trajectory(const gn_hmc_params &hp, double (*gauss)(void), double (*uniform)(void), const double *pre_P,
                       const double *pre_chi, gn_traj_result *res) {
  TraceRange tr("gn trajectory");
  if (hp.steps < 1) throw GnError(GN_ERR_ARG, "steps must be >= 1");
  if (hp.integrator < 0 || hp.integrator > 2) throw GnError(GN_ERR_ARG, "unknown integrator");
  if (u1_) return trajectory_u1(hp, gauss, uniform, pre_P, pre_chi, res);
  const size_t V = size_t(V_);
  memset(res, 0, sizeof *res);
  ExactScope exact_scope(exact, hp.precision == GN_PREC_FP64_EXACT);
  // draws: P, chi_0, chi_1 (moleculardynamics.c:1240-1247), uploaded in one copy
  if (gauss != nullptr) {
    double *h = h_stage_;
    for (size_t i = 0; i < 3 * V; i++) h[i] = gauss();
    check(cudaMemcpyAsync(P_, h, V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload P");
    check(cudaMemcpyAsync(chi_, h + V, 2 * V * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload chi");
  } else {
    if (pre_P) check(cudaMemcpyAsync(P_, pre_P, V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy P");
    if (pre_chi)
      check(cudaMemcpyAsync(chi_, pre_chi, 2 * V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy chi");
  }
  if (!keep_phi) dirac(sm_, chi_, phi_, 2, GN_OP_M);  // phi_f = M chi_f (both flavours as planes)
  double *sigma_copy = scratch_[3];
  check(cudaMemcpyAsync(sigma_copy, sigma(), V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy sigma");
  auto restore = [&]() {
    check(cudaMemcpyAsync(sigma(), sigma_copy, V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "restore");
    sigma_mass(sigma(), nullptr, 0.0, nullptr, sm_);
  };
  const double *phis[2] = {phi_, phi_ + V};
  double *Xs[2] = {X_, X_ + V};
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
  const std::vector<Op> ops = schedule(hp.integrator, hp.eps, hp.steps);
  // Deferred mode: the whole trajectory is queued on the stream with no host
  // round trip; every solve leaves its two states in traj_states_ and the
  // energies their partial sums in traj_partials_, read back once at the end
  // (a failed solve is then found in order, and sigma restored, as the
  // reference's early return would leave it).  The exact-order mode, whose
  // energies are serial sums on the host path, checks every solve as it goes.
  int nsolve = 1;
  for (const Op &o : ops) nsolve += (o.op == OP_F_MED || o.op == OP_F_HIGH || o.op == OP_S_HIGH) ? 1 : 0;
  const bool defer = !exact && nsolve <= kTrajSolves;
  struct DeferScope {  // finish_solve and the solvers' state slots back to normal on every exit
    Engine &e;
    bool on;
    DeferScope(Engine &en, bool d) : e(en), on(d) {
      if (on) {
        e.check(cudaMemsetAsync(e.err_, 0, sizeof(int), e.stream_), "memset");  // may throw: before the flag
        e.defer_ = true;
      }
    }
    ~DeferScope() {
      e.defer_ = false;
      e.state_ = e.state_base_;
    }
  } defer_scope(*this, defer);
  std::vector<double> dist_before;  // deferred: the sigma distance before each solve
  int isolve = 0;
  // one two-flavour solve; false when it failed (synchronous mode only)
  auto run_solve = [&](double tol, int variant) {
    if (defer) {
      state_ = traj_states_ + 2 * isolve++;
      dist_before.push_back(res->distance);
      solve(sm_, phis, Xs, 2, 1, tol, variant, hp.relative, 0, hp.precision, info);
      return true;
    }
    const int st = solve(sm_, phis, Xs, 2, 1, tol, variant, hp.relative, 0, hp.precision, info);
    count_flavours(info, 2, iters, calls, inner, rel);
    if (st != GN_OK) {
      restore();
      check(cudaStreamSynchronize(stream_), "restore");
      finish(0);
      distance += res->distance;
      return false;
    }
    return true;
  };
  const double ccoef = (4 * hp.beta_s / 4.0);  // (NFLAV * beta_scalar / 4.0), moleculardynamics.c:316
  const int enb = op_blocks(V_, num_sms_);
  double e[3];
  double h0 = 0.0;
  if (!run_solve(hp.tol_high, 1)) return GN_NOT_CONVERGED;
  if (defer) {
    energy_launch(P_, phi_, X_, sigma(), traj_partials_);
  } else {
    energy_terms(P_, phi_, X_, sigma(), e);
    h0 = (e[0] + e[1]) + ccoef * e[2];
  }
  for (size_t k = 0; k < ops.size(); k++) {
    const Op &o = ops[k];
    if (o.op == OP_F_MED || o.op == OP_F_HIGH) {
      if (!run_solve(o.op == OP_F_MED ? hp.tol_medium : hp.tol_high, 0)) return GN_NOT_CONVERGED;
      dirac(sm_, X_, Y_, 2, GN_OP_MT);
      if (k + 1 < ops.size() && ops[k + 1].op == OP_P) {
        force(X_, Y_, sigma(), hp.beta_s, F_, P_, ops[k + 1].c);
        k++;
      } else {
        force(X_, Y_, sigma(), hp.beta_s, F_, nullptr, 0.0);
      }
    } else if (o.op == OP_P) {
      momenta(P_, F_, o.c);
    } else if (o.op == OP_Q) {
      sigma_mass(sigma(), P_, o.c, sigma_alt(), sm_);
      swap_sigma();
      res->distance += o.c;
    } else {
      if (!run_solve(hp.tol_high, 1)) return GN_NOT_CONVERGED;
    }
  }
  double h1 = 0.0;
  if (defer) {
    energy_launch(P_, phi_, X_, sigma(), traj_partials_ + 6 * enb);
    int h_err = 0;
    check(cudaMemcpyAsync(h_traj_states_, traj_states_, sizeof(CgState) * 2 * isolve, cudaMemcpyDeviceToHost,
                          stream_), "copy states");
    check(cudaMemcpyAsync(h_traj_partials_, traj_partials_, sizeof(double) * 12 * enb, cudaMemcpyDeviceToHost,
                          stream_), "copy partials");
    check(cudaMemcpyAsync(&h_err, err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy err");
    check(cudaStreamSynchronize(stream_), "trajectory");
    if (h_err == 1) throw GnError(GN_ERR_TIMEOUT, "CG grid barrier timed out");
    if (h_err == 2) throw GnError(GN_ERR_ABORTED, "CG aborted on request");
    for (int j = 0; j < isolve; j++) {
      bool ok = true;
      for (int f = 0; f < 2; f++) {
        const CgState &c = h_traj_states_[2 * j + f];
        info[f].status = c.status;
        info[f].iters = c.iters;
        info[f].r2 = c.r2;
        info[f].b2 = c.b2;
        info[f].inner = c.iters;
        info[f].reliable = c.reliable;
        if (c.status != kCgConverged && c.status != kCgConvergedStart) ok = false;
      }
      count_flavours(info, 2, iters, calls, inner, rel);
      if (!ok) {  // the reference returns here: sigma restored, its later steps undone
        res->distance = dist_before[j];
        restore();
        check(cudaStreamSynchronize(stream_), "restore");
        finish(0);
        distance += res->distance;
        return GN_NOT_CONVERGED;
      }
    }
    for (int q = 0; q < 3; q++) e[q] = sum_partials(h_traj_partials_, enb, q);
    h0 = (e[0] + e[1]) + ccoef * e[2];
    for (int q = 0; q < 3; q++) e[q] = sum_partials(h_traj_partials_ + 6 * enb, enb, q);
    h1 = (e[0] + e[1]) + ccoef * e[2];
  } else {
    energy_terms(P_, phi_, X_, sigma(), e);
    h1 = (e[0] + e[1]) + ccoef * e[2];
  }
  distance += res->distance;
  res->H0 = h0;
  res->H1 = h1;
  res->dH = h1 - h0;
  // Metropolis on the host with the reference's uniform (moleculardynamics.c:1385)
  const int acc = uniform != nullptr ? (uniform() <= std::exp(-(h1 - h0))) : 1;
  res->accepted = acc;
  if (!acc) restore();
  check(cudaStreamSynchronize(stream_), "trajectory");
  finish(1);
  return GN_OK;
}

// The reference's MD helpers (moleculardynamics.c:1460-1625) as they behave:
// every solve's bool is ignored; a force whose solve fails is left at zero
// (ComputeSigmaForce zeroes it first, :634) and its flavour loop stops at the
// failure; sigma is never restored.  In a context holding pi (the U(1)
// model) the same steps run with the complex M on the complex phi and X, as
// the PI_INTERACTION build's ComputeSigmaForce does (:590-647).
int Engine::evolve_in_time(const gn_hmc_params &hp, gn_traj_result *res) {
  TraceRange tr("gn evolve in time");
  if (hp.steps < 1) throw GnError(GN_ERR_ARG, "steps must be >= 1");
  if (hp.integrator < 0 || hp.integrator > 2) throw GnError(GN_ERR_ARG, "unknown integrator");
  const size_t V = size_t(V_);
  memset(res, 0, sizeof *res);
  ExactScope exact_scope(exact, hp.precision == GN_PREC_FP64_EXACT);
  const bool cm = u1_;
  const size_t fl = cm ? 2 * V : V;  // one flavour's planes
  double *phi = cm ? phi_c_ : phi_, *X = cm ? X_c_ : X_, *Y = cm ? Y_c_ : Y_;
  const double *phis[2] = {phi, phi + fl};
  double *Xs[2] = {X, X + fl};
  SolveInfo info[2];
  double iters = 0.0;
  long long calls = 0, inner = 0, rel = 0;
  int all_ok = 1;
  auto solve2 = [&](double tol, int variant) {
    return cm ? solve_cm(sm_, pm_, phis, Xs, 2, tol, variant, hp.relative, 0, info, hp.precision)
              : solve(sm_, phis, Xs, 2, 1, tol, variant, hp.relative, 0, hp.precision, info);
  };
  // Y = M^dagger X, F from X, Y and sigma, then P += pcoef F when P is given
  auto force_from_x = [&](double *P, double pcoef) {
    if (cm) {
      dirac_cm(sm_, pm_, X, Y, 2, GN_OP_MT);
      force_cm(false, X, Y, sigma(), (4 * hp.beta_s / 2.0), F_, P, pcoef);  // (NFLAV * beta_scalar / 2.0), :580
    } else {
      dirac(sm_, X, Y, 2, GN_OP_MT);
      force(X, Y, sigma(), hp.beta_s, F_, P, pcoef);
    }
  };
  const std::vector<Op> ops = evolve_schedule(hp.integrator, hp.eps, hp.steps);
  for (size_t k = 0; k < ops.size(); k++) {
    const Op &o = ops[k];
    if (o.op == OP_F_MED || o.op == OP_F_HIGH) {
      const double tol = o.op == OP_F_MED ? hp.tol_medium : hp.tol_high;
      const int st = solve2(tol, 0);
      count_flavours(info, 2, iters, calls, inner, rel);
      if (st != GN_OK) {
        all_ok = 0;
        check(cudaMemsetAsync(F_, 0, V * sizeof(double), stream_), "zero force");
        continue;
      }
      if (k + 1 < ops.size() && ops[k + 1].op == OP_P) {
        force_from_x(P_, ops[k + 1].c);
        k++;
      } else {
        force_from_x(nullptr, 0.0);
      }
    } else if (o.op == OP_P) {
      momenta(P_, F_, o.c);
    } else if (o.op == OP_Q) {
      sigma_mass(sigma(), P_, o.c, sigma_alt(), sm_);
      swap_sigma();
      distance += o.c;
      res->distance += o.c;
    } else {  // OP_S_HIGH / OP_C_HIGH: both flavours, results not checked
      const int st = solve2(hp.tol_high, o.op == OP_S_HIGH ? 1 : 0);
      count_flavours(info, 2, iters, calls, inner, rel);
      if (st != GN_OK) all_ok = 0;
    }
  }
  check(cudaStreamSynchronize(stream_), "evolve in time");
  res->ok = all_ok;
  res->accepted = 1;
  res->cg_iterations = iters;
  res->cg_calls = calls;
  res->inner_iterations = inner;
  res->reliable_updates = rel;
  return all_ok ? GN_OK : GN_NOT_CONVERGED;
}

// ------------------------------------------------------------------ condensate
int Engine::condensate(const double *sm, double tol, double *target, double *D, double (*uniform)(void),
                       double out[11], double *iterations, long long *calls, int precision) {
  TraceRange tr("gn condensate");
  const size_t V = size_t(V_);
  ExactScope exact_scope(exact, precision == GN_PREC_FP64_EXACT);
  // dot products: the compensated tree, or the reference's serial loop in parity mode
  auto dots = [&](const double *v, const double *Dv, double q[4]) {
    if (exact) {
      cond_dots_exact(v, Dv, q);
    } else {
      cond_dots(v, Dv, q);
      q[3] = q[0];
    }
  };
  double *vec = scratch_[0];
  double *z = scratch_[1];
  signed char *h_signs = reinterpret_cast<signed char *>(h_stage_);
  SolveInfo info[1];
  int all_ok = 1;
  auto solve1 = [&](const double *b) {
    const double *bs[1] = {b};
    double *xs[1] = {target};
    // U(1) model: the same solves with M = D + sm + i eps pm (the resident pi mass)
    const int st = u1_ ? solve_cm(sm, pm_, bs, xs, 1, tol, 0, 0, 0, info, precision)
                       : solve(sm, bs, xs, 1, 2, tol, 0, 0, 0, precision, info);
    if (info[0].status == kCgConverged) {
      *iterations += double(info[0].iters);
      (*calls)++;
    }
    if (st != GN_OK) all_ok = 0;
  };
  auto z2 = [&]() {  // Z2NoiseFullRandomVec, condensate.c:52-60: one uniform per site
    check(cudaStreamSynchronize(stream_), "z2 sync");
    for (size_t x = 0; x < V; x++) h_signs[x] = (uniform() <= 0.5) ? 1 : -1;
    check(cudaMemcpyAsync(signs_, h_signs, V, cudaMemcpyHostToDevice, stream_), "upload signs");
    cond_fill(0, signs_, nullptr, nullptr, vec);
  };
  auto adj = [&]() {  // D = M^dagger target (AdjDiracFermion)
    if (u1_) dirac_cm(sm, pm_, target, D, 1, GN_OP_MT);
    else dirac(sm, target, D, 2, GN_OP_MT);
  };
  double q[4];
  for (int k = 0; k < 11; k++) out[k] = 0.0;
  double temp[4];
  for (int p = 0; p < 4; p++) {
    z2();
    solve1(vec);
    adj();
    dots(vec, D, q);
    temp[p] = q[0];
  }
  const double tr0 = temp[0], tr1 = temp[1], tr2 = temp[2], tr3 = temp[3];
  out[0] = (tr0 + tr1 + tr2 + tr3) / 4.0;
  out[1] = std::fabs(out[0]);
  out[2] = ((tr0 * tr1) + (tr0 * tr2) + (tr0 * tr3) + (tr1 * tr2) + (tr1 * tr3) + (tr2 * tr3)) / 6.0;
  out[3] = (tr0 * tr1 * tr2 * tr3);
  // mu2, chi: the 1/V vector (condensate.c:167-181)
  cond_fill(1, nullptr, nullptr, nullptr, vec);
  solve1(vec);
  adj();
  dots(vec, D, q);
  out[4] = q[1];
  out[5] = out[4] * out[4];
  out[6] = double(int(V)) * out[4];
  out[7] = std::fabs(out[6]);
  // chi_p: e^{i pi/L x2} / V (condensate.c:84-89, :185-197); the table is
  // formed on the host with the same expression as the reference.
  {
    double *h_tab = h_stage_ + V;  // past the sign bytes
    const double pi = 3.141592653589793238462643383279502884197169399375105820974944;
    for (int t = 0; t < L_; t++) {
      const double th = (pi / L_) * t;
      // cexp(I * (pi/L) * t) / V: real part cos, imaginary part sin
      h_tab[2 * t] = std::cos(th) / double(int(V));
      h_tab[2 * t + 1] = std::sin(th) / double(int(V));
    }
    check(cudaMemcpyAsync(table_, h_tab, sizeof(double) * 2 * L_, cudaMemcpyHostToDevice, stream_), "table");
    cond_fill(2, nullptr, table_, nullptr, vec);
    solve1(vec);
    adj();
    dots(vec, D, q);
    out[8] = q[2] * double(int(V));
  }
  // <chibar1 chi2> without sigma (condensate.c:201-212)
  z2();
  check(cudaMemcpyAsync(z, vec, 2 * V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy z");
  solve1(vec);
  adj();
  solve1(D);
  adj();
  dots(z, D, q);
  out[9] = q[3];
  // with sigma-mass insertions (condensate.c:216-230)
  z2();
  check(cudaMemcpyAsync(z, vec, 2 * V * sizeof(double), cudaMemcpyDeviceToDevice, stream_), "copy z");
  cond_fill(3, nullptr, nullptr, sm, vec);
  solve1(vec);
  adj();
  cond_fill(3, nullptr, nullptr, sm, D);
  solve1(D);
  adj();
  dots(z, D, q);
  out[10] = q[3];
  check(cudaStreamSynchronize(stream_), "condensate");
  return all_ok ? GN_OK : GN_NOT_CONVERGED;
}

}  // namespace gn
