// exact.cu -- host side of the exact-order FP64 mode (GN_PREC_FP64_EXACT):
// solves one right-hand side after another in one block each, M^T in the
// reference's scatter order, serial energies and condensate sums; for the Z2
// model and for the U(1) model's complex mass.  Built with
// --fmad=false, like every FP64 kernel that reproduces the reference.
#include <cstring>

#include "engine.h"
#include "errors.h"
#include "exact_kernel.cuh"

namespace gn {

int Engine::solve_exact(const double *sm, const double *const *b, double *const *x, int nrhs, int ncomp, double tol,
                        int variant, int rel, long long max_iter, SolveInfo *info, const double *pm) {
  if (pm != nullptr && ncomp != 2) throw GnError(GN_ERR_ARG, "the complex mass needs complex systems");
  const size_t V = size_t(V_);
  for (int k = 0; k < nrhs; k++) {
    ExactArgs a;
    memset(&a, 0, sizeof a);
    double *w = cg_work_;  // r, p, t, Ap: 2V each
    a.g = g_;
    a.sm = sm;
    a.pm = pm;
    a.b = b[k];
    a.x = x[k];
    a.r = w;
    a.p = w + 2 * V;
    a.t = w + 4 * V;
    a.ap = w + 6 * V;
    a.nc = ncomp;
    a.variant = variant;
    a.rel = rel;
    a.tol = tol;
    a.max_iter = max_iter;
    a.state = state_ + k;
    cg_exact_kernel<<<1, kExactThreads, 0, stream_>>>(a);
    check(cudaGetLastError(), "cg_exact_kernel");
    launches++;
  }
  check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  return finish_solve(nrhs, info);
}

void Engine::mt_exact(const double *sm, const double *in, double *out, int ncomp) {
  const dim3 grid(unsigned((V_ + 255) / 256), unsigned(ncomp));
  mt_exact_kernel<<<grid, 256, 0, stream_>>>(g_, sm, in, out);
  check(cudaGetLastError(), "mt_exact_kernel");
  launches++;
}

void Engine::mt_exact_cm(const double *sm, const double *pm, const double *in, double *out, int nsys) {
  const dim3 grid(unsigned((V_ + 255) / 256), unsigned(nsys));
  mt_exact_cm_kernel<<<grid, 256, 0, stream_>>>(g_, sm, pm, in, out);
  check(cudaGetLastError(), "mt_exact_cm_kernel");
  launches++;
}

// out[0] = sum P^2/2 + the fermion terms (one serial accumulator, as the
// reference's energy functions add them), out[1] = 0, out[2] = sum field^2
void Engine::energy_cm_exact(const double *P, const double *phi, const double *X, const double *field,
                             double out[3]) {
  energy_cm_exact_kernel<<<1, 32, 0, stream_>>>(uint32_t(V_), P, phi, X, field, partials_);
  check(cudaGetLastError(), "energy_cm_exact_kernel");
  launches++;
  double h[2];
  check(cudaMemcpyAsync(h, partials_, sizeof h, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "energy sync");
  out[0] = h[0];
  out[1] = 0.0;
  out[2] = h[1];
}

void Engine::energy_exact(const double *P, const double *phi, const double *X, const double *sigma, double out[3]) {
  energy_exact_kernel<<<1, 32, 0, stream_>>>(uint32_t(V_), P, phi, X, sigma, partials_);
  check(cudaGetLastError(), "energy_exact_kernel");
  launches++;
  double h[2];
  check(cudaMemcpyAsync(h, partials_, sizeof h, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "energy sync");
  out[0] = h[0];
  out[1] = 0.0;
  out[2] = h[1];
}

void Engine::cond_dots_exact(const double *v, const double *D, double out[4]) {
  cond_dot_exact_kernel<<<1, 32, 0, stream_>>>(uint32_t(V_), v, D, partials_);
  check(cudaGetLastError(), "cond_dot_exact_kernel");
  launches++;
  check(cudaMemcpyAsync(out, partials_, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "dots sync");
}

}  // namespace gn
