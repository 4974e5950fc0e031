// mixed.cu -- host side of the mixed-precision solver (FP32 inner iterations,
// FP64 reliable updates).  Built with FMA contraction on: nothing in this
// translation unit reproduces a reference result bit for bit.
#include <cstdlib>
#include <cstring>

#include "engine.h"
#include "errors.h"
#include "launch.h"
#include "mixed_kernel.cuh"

namespace gn {

constexpr int kMixedVecs = 5;  // r^, p^, u^, a^, x^ per right-hand side
constexpr double kDelta = 0.01;  // reliable update when |r^| drops by this factor

void Engine::mixed_init() {
  const size_t V = size_t(V_);
  mx_work_ = (float *)alloc(size_t(kMaxRhs) * kMixedVecs * 2 * V * sizeof(float));
  sm32_ = (float *)alloc(V * sizeof(float));
  pm32_ = (float *)alloc(V * sizeof(float));
  sm32b_ = (float *)alloc(V * sizeof(float));
  pm32b_ = (float *)alloc(V * sizeof(float));
  bar2_ = (PhaseBar *)alloc(sizeof(PhaseBar));
  const char *duo = getenv("GN_MIXED_DUO");
  mixed_duo_ = !(duo != nullptr && duo[0] == '0');
}

// Two systems as two teams of half blocks (cg_mixed_duo_kernel): two real
// systems in 1024-thread blocks, or the U(1) model's two complex systems in
// 512-thread blocks (the block shapes of the lock-step kernels).
template <int W>
static const void *mixed_duo_kernel(bool cm) {
  return cm ? (const void *)cg_mixed_duo_kernel<2, kSolverThreads, W, true>
            : (const void *)cg_mixed_duo_kernel<1, kWideThreads, W>;
}
static const void *mixed_duo_kernel_ptr(int w, bool cm) {
  return w == 4 ? mixed_duo_kernel<4>(cm) : w == 2 ? mixed_duo_kernel<2>(cm) : mixed_duo_kernel<1>(cm);
}

template <int W>
static const void *mixed_kernel(int ncomp, int nr) {
  if (ncomp == 1) {
    if (nr == 1) return (const void *)cg_mixed_kernel<1, 1, kWideThreads, W>;
    if (nr == 2) return (const void *)cg_mixed_kernel<1, 2, kWideThreads, W>;
    return (const void *)cg_mixed_kernel<1, 4, kSolverThreads, W>;
  }
  if (nr == 1) return (const void *)cg_mixed_kernel<2, 1, kSolverThreads, W>;
  if (nr == 2) return (const void *)cg_mixed_kernel<2, 2, kSolverThreads, W>;
  throw GnError(GN_ERR_ARG, "complex systems: at most 2 right-hand sides per solve");
}

// the U(1) model: complex mass, one or two complex systems
template <int W>
static const void *mixed_cm_kernel(int nr) {
  if (nr == 1) return (const void *)cg_mixed_kernel<2, 1, kSolverThreads, W, true>;
  if (nr == 2) return (const void *)cg_mixed_kernel<2, 2, kSolverThreads, W, true>;
  throw GnError(GN_ERR_ARG, "complex systems: at most 2 right-hand sides per solve");
}

// w: sites per item of the FP32 sweeps (1, 2 or 4)
const void *Engine::mixed_kernel_ptr(int ncomp, int nrhs, int w) {
  const int nr = rhs_slots(nrhs);
  if (w == 4) return mixed_kernel<4>(ncomp, nr);
  if (w == 2) return mixed_kernel<2>(ncomp, nr);
  return mixed_kernel<1>(ncomp, nr);
}

int Engine::solve_mixed(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                        int variant, int rel, long long max_iter, SolveInfo *info, const double *pm) {
  if (pm != nullptr && ncomp != 2) throw GnError(GN_ERR_ARG, "the complex mass needs complex systems");
  const size_t V = size_t(V_);
  MixedArgs a;
  memset(&a, 0, sizeof a);
  a.g = g_;
  a.sm = sm;
  a.sm32 = sm32_;
  a.pm = pm;
  a.pm32 = pm32_;
  for (int k = 0; k < nrhs; k++) {
    float *w = mx_work_ + size_t(k) * kMixedVecs * 2 * V;
    a.b[k] = b[k];
    a.x[k] = x[k];
    a.t64[k] = cg_work_ + size_t(k) * 4 * 2 * V;
    a.rh[k] = w;
    a.ph[k] = w + 2 * V;
    a.uh[k] = w + 4 * V;
    a.ah[k] = w + 6 * V;
    a.xh[k] = w + 8 * V;
  }
  a.nrhs = nrhs;
  a.variant = variant;
  a.rel = rel;
  a.scheme = mixed_scheme(V_, nrhs, ncomp);
  a.tol = tol;
  a.max_iter = max_iter;
  a.delta = kDelta;
  a.n_ru = reliable_every;
  a.partials = partials_;
  a.bar = bar_;
  a.err = err_;
  a.abort_flag = d_abort_;
  a.state = state_;
  check(cudaMemsetAsync(bar_, 0, sizeof(PhaseBar), stream_), "memset");
  if (!defer_) check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  // FP32 sweeps in items of up to 4 sites (float4) when the caller's FP64
  // arrays allow the 2-site FP64 sweeps, else one site per item throughout
  const void *ptrs[2 * kMaxRhs + 2] = {sm, pm != nullptr ? pm : sm};
  for (int k = 0; k < nrhs; k++) {
    ptrs[2 + 2 * k] = b[k];
    ptrs[3 + 2 * k] = x[k];
  }
  const int w = fp64_width(L_, ptrs, 2 + 2 * nrhs) == 2 ? row_width(L_, 4) : 1;
  const int nb = cg_blocks(ncomp, nrhs, true, w);
  const bool cm = pm != nullptr;
  if (mixed_duo_ && nrhs == 2 && (cm ? ncomp == 2 : ncomp == 1)) {
    // the two systems as two teams of half blocks: the same units per thread,
    // each team with its own counter, partials (after the first team's
    // 2 (kSyncQ + 1) nb slots), sm32 copy and state slot
    const void *fn = mixed_duo_kernel_ptr(w, cm);
    const int bs = cm ? kSolverThreads : kWideThreads;
    const int cap = coop_capacity(fn, bs);
    if (cap < 1) throw GnError(GN_ERR_CUDA, "CG kernel cannot be resident as a cooperative grid");
    const int nbd = nb < cap ? nb : cap;
    MixedArgs a1 = a;
    a.nrhs = a1.nrhs = 1;
    a1.b[0] = a.b[1];
    a1.x[0] = a.x[1];
    a1.t64[0] = a.t64[1];
    a1.rh[0] = a.rh[1];
    a1.ph[0] = a.ph[1];
    a1.uh[0] = a.uh[1];
    a1.ah[0] = a.ah[1];
    a1.xh[0] = a.xh[1];
    for (int k = 1; k < kMaxRhs; k++) {
      a.b[k] = a1.b[k] = nullptr;
      a.x[k] = a1.x[k] = nullptr;
    }
    a1.sm32 = sm32b_;
    a1.pm32 = pm32b_;
    a1.bar = bar2_;
    a1.partials = partials_ + size_t(2) * (kSyncQ + 1) * nbd;
    a1.state = state_ + 1;
    a.lead = nullptr;
    a1.lead = &bar_->arrived;  // team 1 starts after team 0's first phase
    a1.lead_count = (unsigned long long)nbd;
    check(cudaMemsetAsync(bar2_, 0, sizeof(PhaseBar), stream_), "memset");
    void *args[] = {(void *)&a, (void *)&a1};
    check(cudaLaunchCooperativeKernel(fn, dim3(nbd), dim3(bs), args, 0, stream_),
          "cg_mixed_duo_kernel launch");
    launches++;
    return finish_solve(nrhs, info);
  }
  const void *fn;
  if (pm != nullptr) {
    const int nr = rhs_slots(nrhs);
    fn = w == 4 ? mixed_cm_kernel<4>(nr) : w == 2 ? mixed_cm_kernel<2>(nr) : mixed_cm_kernel<1>(nr);
  } else {
    fn = mixed_kernel_ptr(ncomp, nrhs, w);
  }
  check(launch_solver(fn, nb, threads_for(ncomp, nrhs), a, stream_), "cg_mixed_kernel launch");
  launches++;
  return finish_solve(nrhs, info);
}

}  // namespace gn
