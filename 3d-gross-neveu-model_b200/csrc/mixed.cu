// mixed.cu -- host side of the mixed-precision solver (FP32 inner iterations,
// FP64 reliable updates).  Built with FMA contraction on: nothing in this
// translation unit reproduces a reference result bit for bit.
#include <cstring>

#include "engine.h"
#include "errors.h"
#include "launch.h"
#include "mixed_kernel.cuh"

namespace gn {

constexpr int kMixedVecs = 5;  // r^, p^0, p^1, t^, x^ per right-hand side
constexpr double kDelta = 0.01;  // reliable update when |r^| drops by this factor
constexpr int kReliableEvery = 50;

void Engine::mixed_init() {
  const size_t V = size_t(V_);
  mx_work_ = (float *)alloc(size_t(kMaxRhs) * kMixedVecs * 2 * V * sizeof(float));
  sm32_ = (float *)alloc(V * sizeof(float));
}

const void *Engine::mixed_kernel_ptr(int ncomp, int nrhs) {
  const int nr = rhs_slots(nrhs);
  constexpr int B = kSolverThreads;
  const bool wide = solver_threads() == 768;
  if (ncomp == 1) {
    if (nr == 1) return wide ? (const void *)cg_mixed_kernel<1, 1, 768> : (const void *)cg_mixed_kernel<1, 1, 512>;
    if (nr == 2) return wide ? (const void *)cg_mixed_kernel<1, 2, 768> : (const void *)cg_mixed_kernel<1, 2, 512>;
    return (const void *)cg_mixed_kernel<1, 4, B>;
  }
  if (nr == 1) return (const void *)cg_mixed_kernel<2, 1, B>;
  if (nr == 2) return (const void *)cg_mixed_kernel<2, 2, B>;
  throw GnError(GN_ERR_ARG, "complex systems: at most 2 right-hand sides per solve");
}

int Engine::solve_mixed(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                        int variant, int rel, long long max_iter, SolveInfo *info) {
  const size_t V = size_t(V_);
  MixedArgs a;
  memset(&a, 0, sizeof a);
  a.g = g_;
  a.sm = sm;
  a.sm32 = sm32_;
  for (int k = 0; k < nrhs; k++) {
    float *w = mx_work_ + size_t(k) * kMixedVecs * 2 * V;
    a.b[k] = b[k];
    a.x[k] = x[k];
    a.t64[k] = cg_work_ + size_t(k) * 4 * 2 * V;
    a.rh[k] = w;
    a.ph0[k] = w + 2 * V;
    a.ph1[k] = w + 4 * V;
    a.th[k] = w + 6 * V;
    a.xh[k] = w + 8 * V;
  }
  a.nrhs = nrhs;
  a.variant = variant;
  a.rel = rel;
  a.tol = tol;
  a.max_iter = max_iter;
  a.delta = kDelta;
  a.n_ru = kReliableEvery;
  a.partials = partials_;
  a.bar = bar_;
  a.err = err_;
  a.abort_flag = d_abort_;
  a.state = state_;
  check(cudaMemsetAsync(bar_, 0, sizeof(PhaseBar), stream_), "memset");
  check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  const int nb = cg_blocks(ncomp, nrhs, true);
  check(launch_solver(mixed_kernel_ptr(ncomp, nrhs), nb, threads_for(ncomp, nrhs), a, stream_),
        "cg_mixed_kernel launch");
  launches++;
  return finish_solve(nrhs, info);
}

}  // namespace gn
