// capi.cu -- the extern "C" functions of include/gn_b200.h.  Each host-buffer
// function copies its inputs into the context's device I/O area, runs the
// engine and copies the outputs back before returning.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/gn_b200.h"
#include "checkpoint.h"
#include "engine.h"
#include "errors.h"

struct gn_context {
  std::unique_ptr<gn::Engine> eng;
  double *io = nullptr;     // 24 V doubles of device staging for the host-buffer API
  void *flush = nullptr;    // 512 MB, allocated on the first gn_flush_l2
};

namespace {

thread_local std::string g_last_error;

int fail(int status, const char *msg) {
  g_last_error = msg;
  return status;
}

template <typename F>
int guarded(gn_context *ctx, F &&f) {
  if (ctx == nullptr || !ctx->eng) return fail(GN_ERR_ARG, "null context");
  try {
    cudaSetDevice(ctx->eng->device());
    return f(*ctx->eng);
  } catch (const gn::GnError &e) {
    return fail(e.status, e.what());
  } catch (const std::exception &e) {
    return fail(GN_ERR_CUDA, e.what());
  }
}

void up(gn::Engine &E, double *dst, const double *src, size_t n) {
  E.check(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, E.stream()), "upload");
}
void down(gn::Engine &E, double *dst, const double *src, size_t n) {
  E.check(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, E.stream()), "download");
}
void sync(gn::Engine &E) { E.check(cudaStreamSynchronize(E.stream()), "synchronize"); }

void fill_info(const gn::SolveInfo &s, gn_cg_info *o) {
  o->status = s.status;
  o->counted = s.status == gn::kCgConverged;
  o->iterations = s.iters;
  o->residual = std::sqrt(s.r2);
  o->b_norm = std::sqrt(s.b2);
  o->inner_iterations = s.inner;
  o->reliable_updates = s.reliable;
}

}  // namespace

int gn::set_last_error(int status, const char *msg) { return fail(status, msg); }

extern "C" {

const char *gn_last_error(void) { return g_last_error.c_str(); }

int gn_create(gn_context **out, int L, int device) {
  if (out == nullptr) return fail(GN_ERR_ARG, "null output pointer");
  *out = nullptr;
  try {
    auto ctx = std::make_unique<gn_context>();
    ctx->eng = std::make_unique<gn::Engine>(L, device);
    const size_t V = size_t(ctx->eng->V());
    ctx->eng->check(cudaMalloc(&ctx->io, 24 * V * sizeof(double)), "cudaMalloc io");
    *out = ctx.release();
    return GN_OK;
  } catch (const gn::GnError &e) {
    return fail(e.status, e.what());
  } catch (const std::exception &e) {
    return fail(GN_ERR_CUDA, e.what());
  }
}

void gn_destroy(gn_context *ctx) {
  if (ctx == nullptr) return;
  if (ctx->eng) {
    cudaSetDevice(ctx->eng->device());
    cudaStreamSynchronize(ctx->eng->stream());
  }
  if (ctx->io) cudaFree(ctx->io);
  if (ctx->flush) cudaFree(ctx->flush);
  delete ctx;
}

int gn_set_parity_mode(gn_context *ctx, int on) {
  return guarded(ctx, [&](gn::Engine &E) {
    E.exact = on != 0;
    return GN_OK;
  });
}

int gn_set_reliable_interval(gn_context *ctx, int n) {
  if (n < 1) return fail(GN_ERR_ARG, "reliable-update interval must be >= 1");
  return guarded(ctx, [&](gn::Engine &E) {
    E.reliable_every = n;
    return GN_OK;
  });
}

long long gn_volume(const gn_context *ctx) { return (ctx && ctx->eng) ? (long long)ctx->eng->V() : 0; }

void gn_request_abort(gn_context *ctx, int on) {
  if (ctx && ctx->eng) *(volatile int *)ctx->eng->abort_flag_host() = on;
}

int gn_selftest_wait_timeout(gn_context *ctx) {
  return guarded(ctx, [&](gn::Engine &E) { return E.selftest_wait_timeout(); });
}

int gn_sigma_mass(gn_context *ctx, const double *sigma, double *sigmamass) {
  if (!sigma || !sigmamass) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_s = ctx->io, *d_sm = ctx->io + V;
    up(E, d_s, sigma, V);
    E.sigma_mass(d_s, nullptr, 0.0, nullptr, d_sm);
    down(E, sigmamass, d_sm, V);
    sync(E);
    return GN_OK;
  });
}

int gn_dirac(gn_context *ctx, const double *sigmamass, const double *in, double *out, int ncomp, int op) {
  if (!sigmamass || !in || !out) return fail(GN_ERR_ARG, "null pointer");
  if (ncomp < 1 || ncomp > 2 || op < 0 || op > 2) return fail(GN_ERR_ARG, "bad ncomp or op");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V()), n = size_t(ncomp) * V;
    double *d_sm = ctx->io, *d_in = ctx->io + V, *d_out = ctx->io + 3 * V;
    up(E, d_sm, sigmamass, V);
    up(E, d_in, in, n);
    if (op == GN_OP_SUB_M) up(E, d_out, out, n);
    E.dirac(d_sm, d_in, d_out, ncomp, op);
    down(E, out, d_out, n);
    sync(E);
    return GN_OK;
  });
}

int gn_cg(gn_context *ctx, const double *sigmamass, const double *b, double *x, int nrhs, int ncomp, double tol,
          int variant, int relative, long long max_iter, int precision, gn_cg_info *info) {
  if (!sigmamass || !b || !x) return fail(GN_ERR_ARG, "null pointer");
  if (nrhs < 1 || nrhs > gn::kMaxRhs || ncomp < 1 || ncomp > 2) return fail(GN_ERR_ARG, "bad nrhs or ncomp");
  if (variant < 0 || variant > 1 || precision < 0 || precision > 2) return fail(GN_ERR_ARG, "bad variant/precision");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V()), n = size_t(nrhs) * ncomp * V;
    double *d_sm = ctx->io, *d_b = ctx->io + V, *d_x = ctx->io + V + n;
    up(E, d_sm, sigmamass, V);
    up(E, d_b, b, n);
    up(E, d_x, x, n);
    const double *bs[gn::kMaxRhs];
    double *xs[gn::kMaxRhs];
    for (int k = 0; k < nrhs; k++) {
      bs[k] = d_b + size_t(k) * ncomp * V;
      xs[k] = d_x + size_t(k) * ncomp * V;
    }
    gn::SolveInfo si[gn::kMaxRhs];
    const int st = E.solve(d_sm, bs, xs, nrhs, ncomp, tol, variant, relative, max_iter, precision, si);
    down(E, x, d_x, n);
    sync(E);
    if (info)
      for (int k = 0; k < nrhs; k++) fill_info(si[k], &info[k]);
    return st;
  });
}

int gn_sigma_force(gn_context *ctx, double beta_s, const double *sigma, const double *sigmamass, const double *phi,
                   double *X, double *Y, double tol, double *force, int precision, gn_cg_info *info) {
  if (!sigma || !sigmamass || !phi || !X || !Y || !force) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_s = ctx->io, *d_sm = d_s + V, *d_phi = d_sm + V, *d_X = d_phi + 2 * V, *d_Y = d_X + 2 * V,
           *d_F = d_Y + 2 * V;
    up(E, d_s, sigma, V);
    up(E, d_sm, sigmamass, V);
    up(E, d_phi, phi, 2 * V);
    up(E, d_X, X, 2 * V);
    const double *bs[2] = {d_phi, d_phi + V};
    double *xs[2] = {d_X, d_X + V};
    gn::SolveInfo si[2];
    const int st = E.solve(d_sm, bs, xs, 2, 1, tol, 0, 0, 0, precision, si);
    if (st == GN_OK) {
      const bool saved = E.exact;
      E.exact = saved || precision == GN_PREC_FP64_EXACT;
      E.dirac(d_sm, d_X, d_Y, 2, GN_OP_MT);
      E.exact = saved;
      E.force(d_X, d_Y, d_s, beta_s, d_F, nullptr, 0.0);
      down(E, Y, d_Y, 2 * V);
      down(E, force, d_F, V);
    }
    down(E, X, d_X, 2 * V);
    sync(E);
    if (st != GN_OK) memset(force, 0, V * sizeof(double));  // SetForceSigmaToZero ran first
    if (info)
      for (int k = 0; k < 2; k++) fill_info(si[k], &info[k]);
    return st;
  });
}

int gn_energy(gn_context *ctx, double beta_s, const double *sigma, const double *P, const double *phi,
              const double *X, double *H) {
  if (!sigma || !P || !phi || !X || !H) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_s = ctx->io, *d_P = d_s + V, *d_phi = d_P + V, *d_X = d_phi + 2 * V;
    up(E, d_s, sigma, V);
    up(E, d_P, P, V);
    up(E, d_phi, phi, 2 * V);
    up(E, d_X, X, 2 * V);
    double e[3];
    E.energy_terms(d_P, d_phi, d_X, d_s, e);
    *H = (e[0] + e[1]) + (4 * beta_s / 4.0) * e[2];
    return GN_OK;
  });
}

int gn_evolve_sigma(gn_context *ctx, double *sigma, double *sigmamass, const double *P, double eps) {
  if (!sigma || !sigmamass || !P) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_s = ctx->io, *d_P = d_s + V, *d_out = d_P + V, *d_sm = d_out + V;
    up(E, d_s, sigma, V);
    up(E, d_P, P, V);
    E.sigma_mass(d_s, d_P, eps, d_out, d_sm);
    down(E, sigma, d_out, V);
    down(E, sigmamass, d_sm, V);
    sync(E);
    return GN_OK;
  });
}

int gn_evolve_momenta(gn_context *ctx, double *P, const double *F, double eps) {
  if (!P || !F) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_P = ctx->io, *d_F = d_P + V;
    up(E, d_P, P, V);
    up(E, d_F, F, V);
    E.momenta(d_P, d_F, eps);
    down(E, P, d_P, V);
    sync(E);
    return GN_OK;
  });
}

int gn_condensate(gn_context *ctx, const double *sigmamass, double tol, double *target, double *D,
                  double (*uniform)(void), double *out, double *cg_iterations, long long *cg_calls, int precision) {
  if (!sigmamass || !target || !D || !uniform || !out) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_sm = ctx->io, *d_t = d_sm + V, *d_D = d_t + 2 * V;
    up(E, d_sm, sigmamass, V);
    up(E, d_t, target, 2 * V);
    double it = 0.0;
    long long calls = 0;
    const int st = E.condensate(d_sm, tol, d_t, d_D, uniform, out, &it, &calls, precision);
    down(E, target, d_t, 2 * V);
    down(E, D, d_D, 2 * V);
    sync(E);
    if (cg_iterations) *cg_iterations = it;
    if (cg_calls) *cg_calls = calls;
    return st;
  });
}

int gn_condensate_sigma(gn_context *ctx, const double *sigma, double *out) {
  if (!out) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const double *d = E.sigma();
    if (sigma) {
      up(E, ctx->io, sigma, size_t(E.V()));
      d = ctx->io;
    }
    E.sigma_observables(d, E.u1() ? E.pi() : nullptr, out);
    return GN_OK;
  });
}

int gn_condensate_sigma_device(gn_context *ctx, const double *sigma, double *out) {
  if (!sigma || !out) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    E.sigma_observables(sigma, E.u1() ? E.pi() : nullptr, out);
    return GN_OK;
  });
}

int gn_checkpoint_save(gn_context *ctx, const char *path, const char *path_copy, const gn_hmc_counters *c) {
  if (!path || !c) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) -> int {
    const size_t V = size_t(E.V());
    std::vector<double> sigma(V), sm(V);
    down(E, sigma.data(), E.sigma(), V);
    down(E, sm.data(), E.sm(), V);
    sync(E);
    const int st = gn::write_lattice_file(path, path_copy, E.L(), sigma.data(), sm.data(), nullptr, *c);
    return st == GN_OK ? GN_OK : fail(st, "cannot write the lattice file");
  });
}

int gn_checkpoint_load(gn_context *ctx, const char *path, const char *path_copy, gn_hmc_counters *c) {
  if (!path) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) -> int {
    const size_t V = size_t(E.V());
    double *d_sigma = ctx->io, *d_sm = ctx->io + V;
    auto sm_of = [&](const double *sigma, double *sm) {  // on staging buffers: the resident field stays
      up(E, d_sigma, sigma, V);
      E.sigma_mass(d_sigma, nullptr, 0.0, nullptr, d_sm);
      down(E, sm, d_sm, V);
      sync(E);
    };
    auto accept = [&](const double *sigma) {
      up(E, E.sigma(), sigma, V);
      E.sigma_mass(E.sigma(), nullptr, 0.0, nullptr, E.sm());
      sync(E);
    };
    const int st = gn::load_lattice(path, path_copy, E.L(), c, sm_of, accept);
    if (st == GN_ERR_NOT_FOUND) return fail(st, "no lattice file (a fresh start)");
    if (st != GN_OK) return fail(st, "no lattice file passed its check");
    return GN_OK;
  });
}

// ---- the U(1) model
int gn_set_u1(gn_context *ctx, int on) {
  return guarded(ctx, [&](gn::Engine &E) {
    E.set_u1(on != 0);
    return GN_OK;
  });
}

int gn_load_pi(gn_context *ctx, const double *pi) {
  if (!pi) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    E.set_u1(true);
    up(E, E.pi(), pi, size_t(E.V()));
    E.sigma_mass(E.pi(), nullptr, 0.0, nullptr, E.pm());  // ComputeFullPiMass: the same 8-corner mean
    sync(E);
    return GN_OK;
  });
}

int gn_store_pi(gn_context *ctx, double *pi, double *pimass) {
  return guarded(ctx, [&](gn::Engine &E) -> int {
    if (!E.u1()) return fail(GN_ERR_ARG, "the context is not in the U(1) model");
    if (pi) down(E, pi, E.pi(), size_t(E.V()));
    if (pimass) down(E, pimass, E.pm(), size_t(E.V()));
    sync(E);
    return GN_OK;
  });
}

int gn_dirac_u1(gn_context *ctx, const double *sigmamass, const double *pimass, const double *in, double *out,
                int nsys, int op) {
  if (!sigmamass || !pimass || !in || !out) return fail(GN_ERR_ARG, "null pointer");
  if (nsys < 1 || nsys > 4 || op < 0 || op > 2) return fail(GN_ERR_ARG, "bad nsys / op");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_sm = ctx->io, *d_pm = d_sm + V, *d_in = d_pm + V, *d_out = d_in + 8 * V;
    up(E, d_sm, sigmamass, V);
    up(E, d_pm, pimass, V);
    up(E, d_in, in, 2 * size_t(nsys) * V);
    if (op == GN_OP_SUB_M) up(E, d_out, out, 2 * size_t(nsys) * V);
    E.dirac_cm(d_sm, d_pm, d_in, d_out, nsys, op);
    down(E, out, d_out, 2 * size_t(nsys) * V);
    sync(E);
    return GN_OK;
  });
}

int gn_cg_u1(gn_context *ctx, const double *sigmamass, const double *pimass, const double *b, double *x, int nrhs,
             double tol, int variant, int relative, long long max_iter, int precision, gn_cg_info *info) {
  if (!sigmamass || !pimass || !b || !x) return fail(GN_ERR_ARG, "null pointer");
  if (nrhs < 1 || nrhs > 2) return fail(GN_ERR_ARG, "nrhs must be 1 or 2");
  if (variant < 0 || variant > 1) return fail(GN_ERR_ARG, "bad variant");
  if (precision != GN_PREC_FP64 && precision != GN_PREC_MIXED && precision != GN_PREC_FP64_EXACT)
    return fail(GN_ERR_ARG, "unknown precision");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_sm = ctx->io, *d_pm = d_sm + V, *d_b = d_pm + V, *d_x = d_b + 4 * V;
    up(E, d_sm, sigmamass, V);
    up(E, d_pm, pimass, V);
    up(E, d_b, b, 2 * size_t(nrhs) * V);
    up(E, d_x, x, 2 * size_t(nrhs) * V);
    const double *bs[2] = {d_b, d_b + 2 * V};
    double *xs[2] = {d_x, d_x + 2 * V};
    gn::SolveInfo si[2];
    const int st = E.solve_cm(d_sm, d_pm, bs, xs, nrhs, tol, variant, relative, max_iter, si, precision);
    down(E, x, d_x, 2 * size_t(nrhs) * V);
    sync(E);
    if (info)
      for (int k = 0; k < nrhs; k++) fill_info(si[k], &info[k]);
    return st;
  });
}

static int force_u1(gn_context *ctx, bool pi, double beta_s, const double *field, const double *sigmamass,
                    const double *pimass, const double *phi, double *X, double *Y, double tol, double *force,
                    gn_cg_info *info) {
  if (!field || !sigmamass || !pimass || !phi || !X || !Y || !force) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_f = ctx->io, *d_sm = d_f + V, *d_pm = d_sm + V, *d_phi = d_pm + V, *d_X = d_phi + 4 * V,
           *d_Y = d_X + 4 * V, *d_F = d_Y + 4 * V;
    up(E, d_f, field, V);
    up(E, d_sm, sigmamass, V);
    up(E, d_pm, pimass, V);
    up(E, d_phi, phi, 4 * V);
    up(E, d_X, X, 4 * V);
    const double *bs[2] = {d_phi, d_phi + 2 * V};
    double *xs[2] = {d_X, d_X + 2 * V};
    gn::SolveInfo si[2];
    // parity mode (gn_set_parity_mode): the exact-order solver and M^dagger
    const int st = E.solve_cm(d_sm, d_pm, bs, xs, 2, tol, 0, 0, 0, si, E.exact ? GN_PREC_FP64_EXACT : GN_PREC_FP64);
    if (st == GN_OK) {
      E.dirac_cm(d_sm, d_pm, d_X, d_Y, 2, GN_OP_MT);
      // (NFLAV * beta_scalar / 4.0) for pi (moleculardynamics.c:685), / 2.0 for sigma (:580)
      const double gcoef = pi ? (4 * beta_s / 4.0) : (4 * beta_s / 2.0);
      E.force_cm(pi, d_X, d_Y, d_f, gcoef, d_F, nullptr, 0.0);
      down(E, Y, d_Y, 4 * V);
      down(E, force, d_F, V);
    }
    down(E, X, d_X, 4 * V);
    sync(E);
    if (st != GN_OK) memset(force, 0, V * sizeof(double));  // the force was zeroed first
    if (info)
      for (int k = 0; k < 2; k++) fill_info(si[k], &info[k]);
    return st;
  });
}

int gn_sigma_force_u1(gn_context *ctx, double beta_s, const double *sigma, const double *sigmamass,
                      const double *pimass, const double *phi, double *X, double *Y, double tol, double *force,
                      gn_cg_info *info) {
  return force_u1(ctx, false, beta_s, sigma, sigmamass, pimass, phi, X, Y, tol, force, info);
}

int gn_pi_force(gn_context *ctx, double beta_s, const double *pi, const double *sigmamass, const double *pimass,
                const double *phi, double *X, double *Y, double tol, double *force, gn_cg_info *info) {
  return force_u1(ctx, true, beta_s, pi, sigmamass, pimass, phi, X, Y, tol, force, info);
}

int gn_energy_u1(gn_context *ctx, int which, double beta_s, const double *field, const double *P, const double *phi,
                 const double *X, double *H) {
  if (!field || !P || !phi || !X || !H) return fail(GN_ERR_ARG, "null pointer");
  if (which != 0 && which != 1) return fail(GN_ERR_ARG, "which: 0 sigma, 1 pi");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    double *d_f = ctx->io, *d_P = d_f + V, *d_phi = d_P + V, *d_X = d_phi + 4 * V;
    up(E, d_f, field, V);
    up(E, d_P, P, V);
    up(E, d_phi, phi, 4 * V);
    up(E, d_X, X, 4 * V);
    double e[3];
    E.energy_cm(d_P, d_phi, d_X, d_f, e);
    const double coef = which == 0 ? (4 * beta_s / 4.0) : (4 * beta_s / 8.0);
    *H = (e[0] + e[1]) + coef * e[2];
    return GN_OK;
  });
}

int gn_trajectory_pi(gn_context *ctx, const gn_hmc_params *params, void (*gauss_pair)(double *, double *),
                     double (*gauss)(void), double (*uniform)(void), gn_traj_result *res) {
  if (!params || !res) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) { return E.trajectory_pi(*params, gauss_pair, gauss, uniform, res); });
}

int gn_load_sigma(gn_context *ctx, const double *sigma) {
  if (!sigma) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    up(E, E.sigma(), sigma, size_t(E.V()));
    E.sigma_mass(E.sigma(), nullptr, 0.0, nullptr, E.sm());
    sync(E);
    return GN_OK;
  });
}

int gn_store_sigma(gn_context *ctx, double *sigma, double *sigmamass) {
  return guarded(ctx, [&](gn::Engine &E) {
    if (sigma) down(E, sigma, E.sigma(), size_t(E.V()));
    if (sigmamass) down(E, sigmamass, E.sm(), size_t(E.V()));
    sync(E);
    return GN_OK;
  });
}

static double *field_ptr(gn::Engine &E, int field, size_t &n) {
  const size_t V = size_t(E.V());
  switch (field) {
    case GN_F_P: n = V; return E.P();
    case GN_F_F: n = V; return E.F();
    case GN_F_CHI: n = 2 * V; return E.chi();
    case GN_F_PHI: n = 2 * V; return E.phi();
    case GN_F_X: n = 2 * V; return E.X();
    case GN_F_Y: n = 2 * V; return E.Y();
    default: break;
  }
  if (!E.u1()) throw gn::GnError(GN_ERR_ARG, "unknown field (U(1) fields need gn_load_pi first)");
  switch (field) {
    case GN_F_PI_P: n = V; return E.Ppi();
    case GN_F_PI_F: n = V; return E.Fpi();
    case GN_F_CHI_C: n = 4 * V; return E.chi_c();
    case GN_F_PHI_C: n = 4 * V; return E.phi_c();
    case GN_F_X_C: n = 4 * V; return E.X_c();
    case GN_F_Y_C: n = 4 * V; return E.Y_c();
    default: throw gn::GnError(GN_ERR_ARG, "unknown field");
  }
}

int gn_read_state(gn_context *ctx, int field, double *outp) {
  if (!outp) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    size_t n = 0;
    double *p = field_ptr(E, field, n);
    down(E, outp, p, n);
    sync(E);
    return GN_OK;
  });
}

int gn_write_state(gn_context *ctx, int field, const double *in) {
  if (!in) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    size_t n = 0;
    double *p = field_ptr(E, field, n);
    up(E, p, in, n);
    sync(E);
    return GN_OK;
  });
}

int gn_trajectory(gn_context *ctx, const gn_hmc_params *params, double (*gauss)(void), double (*uniform)(void),
                  gn_traj_result *res) {
  if (!params || !res) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) { return E.trajectory(*params, gauss, uniform, nullptr, nullptr, res); });
}

void *gn_stream(gn_context *ctx) { return (ctx && ctx->eng) ? (void *)ctx->eng->stream() : nullptr; }

double *gn_field_ptr(gn_context *ctx, int field) {
  if (!ctx || !ctx->eng) return nullptr;
  gn::Engine &E = *ctx->eng;
  if (field == GN_F_SIGMA) return E.sigma();
  if (field == GN_F_SM) return E.sm();
  if (field == GN_F_PI) return E.u1() ? E.pi() : nullptr;
  if (field == GN_F_PM) return E.u1() ? E.pm() : nullptr;
  try {
    size_t n = 0;
    return field_ptr(E, field, n);
  } catch (const gn::GnError &e) {
    fail(e.status, e.what());
    return nullptr;
  }
}

int gn_dirac_device(gn_context *ctx, const double *sigmamass, const double *in, double *out, int ncomp, int op) {
  if (!sigmamass || !in || !out) return fail(GN_ERR_ARG, "null pointer");
  if (ncomp < 1 || ncomp > 2 || op < 0 || op > 2) return fail(GN_ERR_ARG, "bad ncomp or op");
  return guarded(ctx, [&](gn::Engine &E) {
    E.dirac(sigmamass, in, out, ncomp, op);
    return GN_OK;
  });
}

int gn_cg_device(gn_context *ctx, const double *sigmamass, const double *b, double *x, int nrhs, int ncomp, double tol,
                 int variant, int relative, long long max_iter, int precision, gn_cg_info *info) {
  if (!sigmamass || !b || !x) return fail(GN_ERR_ARG, "null pointer");
  if (nrhs < 1 || nrhs > gn::kMaxRhs || ncomp < 1 || ncomp > 2) return fail(GN_ERR_ARG, "bad nrhs or ncomp");
  if (variant < 0 || variant > 1 || precision < 0 || precision > 2) return fail(GN_ERR_ARG, "bad variant/precision");
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t V = size_t(E.V());
    const double *bs[gn::kMaxRhs];
    double *xs[gn::kMaxRhs];
    for (int k = 0; k < nrhs; k++) {
      bs[k] = b + size_t(k) * ncomp * V;
      xs[k] = x + size_t(k) * ncomp * V;
    }
    gn::SolveInfo si[gn::kMaxRhs];
    const int st = E.solve(sigmamass, bs, xs, nrhs, ncomp, tol, variant, relative, max_iter, precision, si);
    if (info)
      for (int k = 0; k < nrhs; k++) fill_info(si[k], &info[k]);
    return st;
  });
}

int gn_trajectory_device(gn_context *ctx, const gn_hmc_params *params, const double *P, const double *chi,
                         double (*uniform)(void), gn_traj_result *res) {
  if (!params || !res || !P || !chi) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) { return E.trajectory(*params, nullptr, uniform, P, chi, res); });
}

int gn_md_evolve(gn_context *ctx, const gn_hmc_params *params, gn_traj_result *res) {
  if (!params || !res) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) {
    struct KeepPhi {  // restored on every exit
      bool &flag;
      explicit KeepPhi(bool &f) : flag(f) { flag = true; }
      ~KeepPhi() { flag = false; }
    } keep(E.keep_phi);
    return E.trajectory(*params, nullptr, nullptr, nullptr, nullptr, res);
  });
}

int gn_evolve_sigma_in_time(gn_context *ctx, const gn_hmc_params *params, gn_traj_result *res) {
  if (!params || !res) return fail(GN_ERR_ARG, "null pointer");
  return guarded(ctx, [&](gn::Engine &E) { return E.evolve_in_time(*params, res); });
}

long long gn_launch_count(gn_context *ctx) { return (ctx && ctx->eng) ? ctx->eng->launches : 0; }

int gn_flush_l2(gn_context *ctx) {
  return guarded(ctx, [&](gn::Engine &E) {
    const size_t bytes = size_t(512) << 20;
    if (!ctx->flush) E.check(cudaMalloc(&ctx->flush, bytes), "cudaMalloc flush");
    E.check(cudaMemsetAsync(ctx->flush, ctx->eng->V() & 0xff, bytes, E.stream()), "flush");
    return GN_OK;
  });
}

}  // extern "C"
