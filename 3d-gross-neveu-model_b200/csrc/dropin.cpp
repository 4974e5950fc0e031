// dropin.cpp -- the reference's hot-path functions (names, signatures, struct
// side effects, return values) on top of the C-ABI of gn_b200.h.  Built twice:
// into lib/libgn_dropin.so for the Z2 model (include/gn_dropin.h) and, with
// GN_DROPIN_PI defined, into lib/libgn_dropin_pi.so for a program built with
// PI_INTERACTION (include/gn_dropin_pi.h).
//
// The reference stores fermion fields as double _Complex[VOLUME].  In the Z2
// model their imaginary parts are zero on the sigma path; they are passed to
// the GPU as one real plane, or as two planes when an imaginary part is
// nonzero (the condensate's phase vector), so every function is exact for
// complex input.  In the U(1) model M itself is complex and every field goes
// as two planes.  The solvers' scratch vectors of the reference's Fermionkit
// (r_k, p_k, temp1, temp2) are not written: they carry no result.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef GN_DROPIN_PI
#include "../../include/gn_dropin_pi.h"
#else
#include "../../include/gn_dropin.h"
#endif

namespace {

gn_context *g_ctx = nullptr;
int g_L = 0;
long long g_V = 0;
double (*g_gauss)(void) = nullptr;
double (*g_uniform)(void) = nullptr;
double g_tol_medium = 1e-3;  // MEDIUM_PRECISION_INVERSION, macro.h:135
double g_tol_high = 1e-9;    // HIGH_PRECISION_INVERSION, macro.h:136
int g_precision = GN_PREC_FP64;
std::vector<double> g_a, g_b, g_c, g_d;  // host staging planes (4V each: two complex flavours)
#ifdef GN_DROPIN_PI
void (*g_gauss2)(double *, double *, double, double) = nullptr;
#endif

[[noreturn]] void fatal(const char *what) {
  fprintf(stderr, "gn_dropin: %s: %s\n", what, gn_last_error());
  exit(2);  // the reference's own exit code for a failed inversion (observables.c:199)
}

gn_context *ctx() {
  if (g_ctx) return g_ctx;
  if (g_L == 0) {
    const char *e = getenv("GN_LSPACE");
    if (e) g_L = atoi(e);
  }
  if (g_L == 0) {
    fprintf(stderr, "gn_dropin: lattice size unknown: call GNB200_SetLattice(LSPACE) or set GN_LSPACE\n");
    exit(2);
  }
  if (gn_create(&g_ctx, g_L, 0) != GN_OK) fatal("gn_create");
  g_V = gn_volume(g_ctx);
  g_a.resize(4 * g_V);
  g_b.resize(4 * g_V);
  g_c.resize(4 * g_V);
  g_d.resize(4 * g_V);
  return g_ctx;
}

// the host program's function `name`, unless one was set
template <typename Fn>
Fn resolve(Fn set, const char *name) {
  if (set) return set;
  void *p = dlsym(RTLD_DEFAULT, name);
  if (!p) {
    fprintf(stderr,
            "gn_dropin: the host program's %s was not found (export it, e.g. link with -rdynamic, "
            "or call GNB200_SetRandom)\n",
            name);
    exit(2);
  }
  return reinterpret_cast<Fn>(p);
}

#ifndef GN_DROPIN_PI
bool has_imag(const double _Complex *z) {
  for (long long x = 0; x < g_V; x++)
    if (__imag__ z[x] != 0.0) return true;
  return false;
}
#endif
// complex field -> planes (re, then im when nc == 2)
void to_planes(const double _Complex *z, double *p, int nc) {
  for (long long x = 0; x < g_V; x++) p[x] = __real__ z[x];
  if (nc == 2)
    for (long long x = 0; x < g_V; x++) p[g_V + x] = __imag__ z[x];
}
void from_planes(const double *p, double _Complex *z, int nc) {
  for (long long x = 0; x < g_V; x++) {
    __real__ z[x] = p[x];
    __imag__ z[x] = nc == 2 ? p[g_V + x] : 0.0;
  }
}
#ifndef GN_DROPIN_PI
// flavour pair of a ManyFermions into 2V real values (imaginary parts are zero on the sigma path)
void pair_to_real(const ManyFermions &m, double *p) {
  for (int f = 0; f < 2; f++)
    for (long long x = 0; x < g_V; x++) p[f * g_V + x] = __real__ m.flav[f].fermion[x];
}
void real_to_pair(const double *p, ManyFermions &m, int nflav = 2) {
  for (int f = 0; f < nflav; f++)
    for (long long x = 0; x < g_V; x++) {
      __real__ m.flav[f].fermion[x] = p[f * g_V + x];
      __imag__ m.flav[f].fermion[x] = 0.0;
    }
}
#endif

#ifdef GN_DROPIN_PI
// flavour pair of complex fields <-> 4V planes (flavour f: real plane 2f, imaginary 2f + 1)
void pair_to_planes(const ManyFermions &m, double *p) {
  for (int f = 0; f < 2; f++) to_planes(m.flav[f].fermion, p + 2 * f * g_V, 2);
}
void planes_to_pair(const double *p, ManyFermions &m) {
  for (int f = 0; f < 2; f++) from_planes(p + 2 * f * g_V, m.flav[f].fermion, 2);
}
#endif

void dirac_op(const Lattice *lat, const Fermion *in, Fermion *out, int op) {
  gn_context *c = ctx();
#ifdef GN_DROPIN_PI
  to_planes(in->fermion, g_a.data(), 2);
  if (op == GN_OP_SUB_M) to_planes(out->fermion, g_b.data(), 2);
  if (gn_dirac_u1(c, lat->sigmamass, lat->pimass, g_a.data(), g_b.data(), 1, op) != GN_OK) fatal("gn_dirac_u1");
  from_planes(g_b.data(), out->fermion, 2);
#else
  const int nc = (has_imag(in->fermion) || (op == GN_OP_SUB_M && has_imag(out->fermion))) ? 2 : 1;
  to_planes(in->fermion, g_a.data(), nc);
  if (op == GN_OP_SUB_M) to_planes(out->fermion, g_b.data(), nc);
  if (gn_dirac(c, lat->sigmamass, g_a.data(), g_b.data(), nc, op) != GN_OK) fatal("gn_dirac");
  from_planes(g_b.data(), out->fermion, nc);
#endif
}

bool cg(const Lattice *lat, const Fermion *b, Fermion *x, double tol, Fermionkit *kit, int variant) {
  gn_context *c = ctx();
  gn_cg_info info;
#ifdef GN_DROPIN_PI
  const int nc = 2;
  to_planes(b->fermion, g_a.data(), nc);
  to_planes(x->fermion, g_b.data(), nc);
  const int st = gn_cg_u1(c, lat->sigmamass, lat->pimass, g_a.data(), g_b.data(), 1, tol, variant, 0, 0,
                          g_precision, &info);
  if (st < 0) fatal("gn_cg_u1");
#else
  const int nc = (has_imag(b->fermion) || has_imag(x->fermion)) ? 2 : 1;
  to_planes(b->fermion, g_a.data(), nc);
  to_planes(x->fermion, g_b.data(), nc);
  const int st =
      gn_cg(c, lat->sigmamass, g_a.data(), g_b.data(), 1, nc, tol, variant, 0, 0, g_precision, &info);
  if (st < 0) fatal("gn_cg");
#endif
  from_planes(g_b.data(), x->fermion, nc);
  if (info.counted) {  // conjugategradient.c:92-93
    kit->iterations += double(info.iterations);
    kit->CG_call++;
  }
  return st == GN_OK;
}

// ComputeSigmaForce (or, in the U(1) model, ComputePiForce when pi) with a
// given Gaussian coefficient: F is overwritten when zero_first, otherwise the
// fermion part is added to it.
bool fermion_force(const Lattice *lat, bool pi, double beta_s, double *force, Fermionkit *kit, double tol,
                   bool zero_first) {
  gn_context *c = ctx();
  double *phi = g_a.data(), *X = g_b.data(), *Y = g_c.data(), *F = g_d.data();
  gn_cg_info info[2];
#ifdef GN_DROPIN_PI
  const int nc = 2;
  pair_to_planes(kit->phi, phi);
  pair_to_planes(kit->inverted_phi, X);
  const int st = pi ? gn_pi_force(c, beta_s, lat->pi, lat->sigmamass, lat->pimass, phi, X, Y, tol, F, info)
                    : gn_sigma_force_u1(c, beta_s, lat->sigma, lat->sigmamass, lat->pimass, phi, X, Y, tol, F, info);
  if (st < 0) fatal(pi ? "gn_pi_force" : "gn_sigma_force_u1");
#else
  (void)pi;
  const int nc = 1;
  pair_to_real(kit->phi, phi);
  pair_to_real(kit->inverted_phi, X);
  const int st = gn_sigma_force(c, beta_s, lat->sigma, lat->sigmamass, phi, X, Y, tol, F, g_precision, info);
  if (st < 0) fatal("gn_sigma_force");
#endif
  // counters and X as the reference's flavour loop leaves them (moleculardynamics.c:593-597)
  for (int f = 0; f < 2; f++) {
    if (info[f].counted) {
      kit->iterations += double(info[f].iterations);
      kit->CG_call++;
    }
    from_planes(X + size_t(f) * nc * g_V, kit->inverted_phi.flav[f].fermion, nc);
    if (info[f].status != 1 && info[f].status != 2) break;
  }
  if (st != GN_OK) {
    if (zero_first) memset(force, 0, sizeof(double) * g_V);
    return false;
  }
  for (int f = 0; f < 2; f++) from_planes(Y + size_t(f) * nc * g_V, kit->inverted_phi_obs.flav[f].fermion, nc);
  if (zero_first) memcpy(force, F, sizeof(double) * g_V);
  else
    for (long long x = 0; x < g_V; x++) force[x] += F[x];
  return true;
}

// the fermion fields a trajectory leaves in the kit: chi, phi, X, Y
void read_kit(gn_context *c, Fermionkit *kit) {
  double *tmp = g_a.data();
#ifdef GN_DROPIN_PI
  const int fields[4] = {GN_F_CHI_C, GN_F_PHI_C, GN_F_X_C, GN_F_Y_C};
#else
  const int fields[4] = {GN_F_CHI, GN_F_PHI, GN_F_X, GN_F_Y};
#endif
  ManyFermions *dst[4] = {&kit->chi, &kit->phi, &kit->inverted_phi, &kit->inverted_phi_obs};
  for (int i = 0; i < 4; i++) {
    if (gn_read_state(c, fields[i], tmp) != GN_OK) fatal("gn_read_state");
#ifdef GN_DROPIN_PI
    planes_to_pair(tmp, *dst[i]);
#else
    real_to_pair(tmp, *dst[i]);
#endif
  }
}

// the acceptance file's line (moleculardynamics.c:1426, :1873)
void acceptance_line(FILE *opf, const Info *info, double dH) {
  fprintf(opf, "%.16f\t%.16f\t%.16f\t%.16f\t%d\t%.16f\t%.16f\t%.16f\t%.16f\t%d\t%.16f\t%.16f\t%.16f\n", info->beta,
          info->beta_scalar, info->mass, info->epsilon_link_HMC, info->steps_link_HMC,
          (info->epsilon_link_HMC * info->steps_link_HMC), info->delta_H_link, info->hybrid_done_acceptance_link,
          info->epsilon_sigma_HMC, info->steps_sigma_HMC, (info->epsilon_sigma_HMC * info->steps_sigma_HMC), dH,
          info->hybrid_done_acceptance_sigma);
}

bool trajectory(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta, Fermionkit *kit,
                double epsilon, int step, const char *acceptance_file, int integrator) {
  gn_context *c = ctx();
  g_gauss = resolve(g_gauss, "Gauss1");
  g_uniform = resolve(g_uniform, "Casuale");
  FILE *opf = fopen(acceptance_file, "a");  // moleculardynamics.c:1238
  if (gn_load_sigma(c, lattice->sigma) != GN_OK) fatal("gn_load_sigma");
#ifdef GN_DROPIN_PI
  if (gn_load_pi(c, lattice->pi) != GN_OK) fatal("gn_load_pi");
#endif
  gn_hmc_params hp;
  hp.beta_s = info->beta_scalar;
  hp.eps = epsilon;
  hp.steps = step;
  hp.integrator = integrator;
  hp.tol_medium = g_tol_medium;
  hp.tol_high = g_tol_high;
  hp.relative = 0;
  hp.precision = g_precision;
  gn_traj_result r;
  const int st = gn_trajectory(c, &hp, g_gauss, g_uniform, &r);
  if (st < 0) fatal("gn_trajectory");
  // the state the reference leaves behind
  if (gn_store_sigma(c, lattice->sigma, lattice->sigmamass) != GN_OK) fatal("gn_store_sigma");
  if (gn_read_state(c, GN_F_P, momenta->momenta) != GN_OK || gn_read_state(c, GN_F_F, force->force) != GN_OK)
    fatal("gn_read_state");
  read_kit(c, kit);
  kit->iterations += r.cg_iterations;
  kit->CG_call += int(r.cg_calls);
  lattice->distance_sigma += r.distance;
  if (!r.ok) {
    if (opf) fclose(opf);
    return false;
  }
  // acceptance bookkeeping (moleculardynamics.c:1385-1424)
  if (r.accepted) {
    info->hybrid_accepted_sigma++;
    info->hybrid_done_sigma++;
    info->hybrid_done_acceptance_sigma = double(info->hybrid_accepted_sigma) / double(info->hybrid_done_sigma);
    info->local_accepted_sigma++;
    info->local_done_sigma++;
    info->local_acceptance_sigma = double(info->local_accepted_sigma) / double(info->local_done_sigma);
    lattice->done_sigma++;
    if (info->story_sigma >= 0) info->story_sigma++;
    else info->story_sigma = -1;
  } else {
    info->hybrid_done_sigma++;
    info->hybrid_done_acceptance_sigma = double(info->hybrid_accepted_sigma) / double(info->hybrid_done_sigma);
    info->local_done_sigma++;
    info->local_acceptance_sigma = double(info->local_accepted_sigma) / double(info->local_done_sigma);
    lattice->done_sigma++;
    if (info->story_sigma >= 0) info->story_sigma = -1;
    else info->story_sigma--;
  }
  if (opf) {  // moleculardynamics.c:1426
    acceptance_line(opf, info, r.dH);
    fclose(opf);
  }
  return true;
}

// The reference's EvolveSigmaInTime* helpers (moleculardynamics.c:1460-1625)
// on the GPU: the fields they read go up, gn_evolve_sigma_in_time runs the
// helper's steps, and the fields they write come back.  In the U(1) build
// the fermion fields are complex and M carries the resident pi mass.
void evolve_in_time(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta, Fermionkit *kit,
                    double epsilon, int step, int integrator) {
  gn_context *c = ctx();
  if (gn_load_sigma(c, lattice->sigma) != GN_OK) fatal("gn_load_sigma");
#ifdef GN_DROPIN_PI
  if (gn_load_pi(c, lattice->pi) != GN_OK) fatal("gn_load_pi");
  const int f_phi = GN_F_PHI_C, f_x = GN_F_X_C, f_y = GN_F_Y_C;
  pair_to_planes(kit->phi, g_a.data());
  pair_to_planes(kit->inverted_phi, g_b.data());
#else
  const int f_phi = GN_F_PHI, f_x = GN_F_X, f_y = GN_F_Y;
  pair_to_real(kit->phi, g_a.data());
  pair_to_real(kit->inverted_phi, g_b.data());
#endif
  if (gn_write_state(c, GN_F_P, momenta->momenta) != GN_OK || gn_write_state(c, f_phi, g_a.data()) != GN_OK ||
      gn_write_state(c, f_x, g_b.data()) != GN_OK)
    fatal("gn_write_state");
  gn_hmc_params hp;
  hp.beta_s = info->beta_scalar;
  hp.eps = epsilon;
  hp.steps = step;
  hp.integrator = integrator;
  hp.tol_medium = g_tol_medium;
  hp.tol_high = g_tol_high;
  hp.relative = 0;
  hp.precision = g_precision;
  gn_traj_result r;
  if (gn_evolve_sigma_in_time(c, &hp, &r) < 0) fatal("gn_evolve_sigma_in_time");
  if (gn_store_sigma(c, lattice->sigma, lattice->sigmamass) != GN_OK) fatal("gn_store_sigma");
  if (gn_read_state(c, GN_F_P, momenta->momenta) != GN_OK || gn_read_state(c, GN_F_F, force->force) != GN_OK ||
      gn_read_state(c, f_x, g_a.data()) != GN_OK || gn_read_state(c, f_y, g_b.data()) != GN_OK)
    fatal("gn_read_state");
#ifdef GN_DROPIN_PI
  planes_to_pair(g_a.data(), kit->inverted_phi);
  planes_to_pair(g_b.data(), kit->inverted_phi_obs);
#else
  real_to_pair(g_a.data(), kit->inverted_phi);
  real_to_pair(g_b.data(), kit->inverted_phi_obs);
#endif
  kit->iterations += r.cg_iterations;
  kit->CG_call += int(r.cg_calls);
  lattice->distance_sigma += r.distance;
}

#ifdef GN_DROPIN_PI
void draw_pair(double *a, double *b) { g_gauss2(a, b, 0.0, 1.0); }  // DrawPiMomentaFromGaussianDistribution

// LeapFrog2Pi (moleculardynamics.c:1743-1880) on the GPU, with the reference's
// draws, bookkeeping, printed lines and acceptance line
bool trajectory_pi(Lattice *lattice, Info *info, Forcepi *force, Momentapi *momenta, Fermionkit *kit, double epsilon,
                   int step, const char *acceptance_file) {
  gn_context *c = ctx();
  g_gauss = resolve(g_gauss, "Gauss1");
  g_uniform = resolve(g_uniform, "Casuale");
  g_gauss2 = resolve(g_gauss2, "Gauss2MeanVariance");
  FILE *opf = fopen(acceptance_file, "a");  // moleculardynamics.c:1747
  if (gn_load_sigma(c, lattice->sigma) != GN_OK || gn_load_pi(c, lattice->pi) != GN_OK) fatal("gn_load_pi");
  // the first inversion starts from the kit's X (ConjugateGradientFastDiracAdjFastDiracToTheMinusOne)
  pair_to_planes(kit->inverted_phi, g_a.data());
  if (gn_write_state(c, GN_F_X_C, g_a.data()) != GN_OK) fatal("gn_write_state");
  gn_hmc_params hp;
  hp.beta_s = info->beta_scalar;
  hp.eps = epsilon;
  hp.steps = step;
  hp.integrator = GN_LFMN2VF;  // not used by LeapFrog2Pi
  hp.tol_medium = g_tol_high;
  hp.tol_high = g_tol_high;    // ComputePiForce inverts at HIGH_PRECISION_INVERSION
  hp.relative = 0;
  hp.precision = g_precision;
  gn_traj_result r;
  const int st = gn_trajectory_pi(c, &hp, draw_pair, g_gauss, g_uniform, &r);
  if (st < 0) fatal("gn_trajectory_pi");
  if (gn_store_pi(c, lattice->pi, lattice->pimass) != GN_OK) fatal("gn_store_pi");
  if (gn_read_state(c, GN_F_PI_P, momenta->momenta) != GN_OK || gn_read_state(c, GN_F_PI_F, force->force) != GN_OK)
    fatal("gn_read_state");
  read_kit(c, kit);
  kit->iterations += r.cg_iterations;
  kit->CG_call += int(r.cg_calls);
  if (!r.ok) {
    if (opf) fclose(opf);
    return false;
  }
  printf("Delta energy is %.16f\n", r.dH);
  if (r.accepted) {
    info->hybrid_accepted_pi++;
    info->hybrid_done_pi++;
    info->hybrid_done_acceptance_pi = double(info->hybrid_accepted_pi) / double(info->hybrid_done_pi);
    if (info->story_pi >= 0) info->story_pi++;
    else info->story_pi = -1;
  } else {
    info->hybrid_done_pi++;
    info->hybrid_done_acceptance_pi = double(info->hybrid_accepted_pi) / double(info->hybrid_done_pi);
    if (info->story_pi >= 0) info->story_pi = -1;
    else info->story_pi--;
  }
  printf("%d/%d\n", info->hybrid_accepted_pi, info->hybrid_done_pi);
  if (opf) {  // moleculardynamics.c:1873
    acceptance_line(opf, info, r.dH);
    fclose(opf);
  }
  return true;
}
#endif

}  // namespace

extern "C" {

void GNB200_SetLattice(int L) {
  if (g_ctx && L != g_L) {
    gn_destroy(g_ctx);
    g_ctx = nullptr;
  }
  g_L = L;
}
void GNB200_SetRandom(double (*gauss)(void), double (*uniform)(void)) {
  g_gauss = gauss;
  g_uniform = uniform;
}
void GNB200_SetTolerances(double medium, double high) {
  g_tol_medium = medium;
  g_tol_high = high;
}
void GNB200_SetPrecision(int precision) {
  g_precision = precision;
  // the operators without a precision argument follow the exact mode too
  if (gn_set_parity_mode(ctx(), precision == GN_PREC_FP64_EXACT) != GN_OK) fatal("gn_set_parity_mode");
}
gn_context *GNB200_Context(void) { return ctx(); }

void DiracFermion(const Lattice *lat, const Fermion *fermion, Fermion *target, const Info *, const Fermioncoor *) {
  dirac_op(lat, fermion, target, GN_OP_M);
}
void AdjDiracFermion(const Lattice *lat, const Fermion *fermion, Fermion *target, const Info *, const Fermioncoor *) {
  dirac_op(lat, fermion, target, GN_OP_MT);
}
void SubtractDiracFermion(const Lattice *lat, const Fermion *fermion, Fermion *target, const Info *,
                          const Fermioncoor *) {
  dirac_op(lat, fermion, target, GN_OP_SUB_M);
}

bool ConjugateGradientFastDiracAdjFastDiracToTheMinusOne(const Lattice *lat, const Fermion *fermion,
                                                         Fermion *target_inverted, const Info *, const Fermioncoor *,
                                                         double inversion_precision, Fermionkit *kit, int) {
  return cg(lat, fermion, target_inverted, inversion_precision, kit, 0);
}
bool StartX0ImposedConjugateGradientFastDiracAdjFastDiracToTheMinusOne(const Lattice *lat, const Fermion *fermion,
                                                                       Fermion *target_inverted, const Info *,
                                                                       const Fermioncoor *, double inversion_precision,
                                                                       Fermionkit *kit, int) {
  return cg(lat, fermion, target_inverted, inversion_precision, kit, 1);
}

void ComputeFullSigmaMass(Lattice *lat, const Fermioncoor *, double *sigmamass) {
  if (gn_sigma_mass(ctx(), lat->sigma, sigmamass) != GN_OK) fatal("gn_sigma_mass");
}

void AddForceFromSigmaSector(const Lattice *lat, const Info *info, Forcesigma *force) {
  // F -= (NFLAV beta_s / 2) sigma, as F + sigma * (-c): the same rounding
  const double coef = (4 * info->beta_scalar / 2.0);
  if (gn_evolve_momenta(ctx(), force->force, lat->sigma, -coef) != GN_OK) fatal("gn_evolve_momenta");
}
bool AddForceFromFermionSectorRespectToSigma(const Lattice *lat, const Info *, const Fermioncoor *,
                                             Forcesigma *force, Fermionkit *kit, double inversion_precision) {
  return fermion_force(lat, false, 0.0, force->force, kit, inversion_precision, false);
}
bool ComputeSigmaForce(const Lattice *lat, const Info *info, const Fermioncoor *, Forcesigma *force, Fermionkit *kit,
                       double inversion_precision) {
  return fermion_force(lat, false, info->beta_scalar, force->force, kit, inversion_precision, true);
}

double ComputeFullEnergyForSigma(const Lattice *lattice, const Info *info, const Fermioncoor *,
                                 const Momentasigma *momenta, const Fermionkit *kit) {
  gn_context *c = ctx();
  double H = 0.0;
#ifdef GN_DROPIN_PI
  pair_to_planes(kit->phi, g_a.data());
  pair_to_planes(kit->inverted_phi, g_b.data());
  if (gn_energy_u1(c, 0, info->beta_scalar, lattice->sigma, momenta->momenta, g_a.data(), g_b.data(), &H) != GN_OK)
    fatal("gn_energy_u1");
#else
  pair_to_real(kit->phi, g_a.data());
  pair_to_real(kit->inverted_phi, g_b.data());
  if (gn_energy(c, info->beta_scalar, lattice->sigma, momenta->momenta, g_a.data(), g_b.data(), &H) != GN_OK)
    fatal("gn_energy");
#endif
  return H;
}

void EvolveCoordinatesSigma(Lattice *lat, const Momentasigma *momenta, const Fermioncoor *, double epsilon) {
  if (gn_evolve_sigma(ctx(), lat->sigma, lat->sigmamass, momenta->momenta, epsilon) != GN_OK)
    fatal("gn_evolve_sigma");
  lat->distance_sigma += epsilon;
}
void EvolveMomentaSigma(Momentasigma *momenta, const Forcesigma *force, double epsilon) {
  if (gn_evolve_momenta(ctx(), momenta->momenta, force->force, epsilon) != GN_OK) fatal("gn_evolve_momenta");
}

bool LeapFrog2Sigma(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta, const Fermioncoor *,
                    Fermionkit *kit, double epsilon, const int step, const char *acceptance_file) {
  return trajectory(lattice, info, force, momenta, kit, epsilon, step, acceptance_file, GN_LF2);
}
bool LeapFrog2MinimumNormSigma(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta,
                               const Fermioncoor *, Fermionkit *kit, double epsilon, const int step,
                               const char *acceptance_file) {
  return trajectory(lattice, info, force, momenta, kit, epsilon, step, acceptance_file, GN_LFMN2);
}
bool LeapFrog2MinimumNormSigmaVelocityFirst(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta,
                                            const Fermioncoor *, Fermionkit *kit, double epsilon, const int step,
                                            const char *acceptance_file) {
  return trajectory(lattice, info, force, momenta, kit, epsilon, step, acceptance_file, GN_LFMN2VF);
}
void EvolveSigmaInTimeLF2(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta, const Fermioncoor *,
                          Fermionkit *kit, double epsilon, const int step) {
  evolve_in_time(lattice, info, force, momenta, kit, epsilon, step, GN_LF2);
}
void EvolveSigmaInTimeMinimumNormLF2(Lattice *lattice, Info *info, Forcesigma *force, Momentasigma *momenta,
                                     const Fermioncoor *, Fermionkit *kit, double epsilon, const int step) {
  evolve_in_time(lattice, info, force, momenta, kit, epsilon, step, GN_LFMN2);
}
void EvolveSigmaInTimeMinimumNormSigmaVelocityFirst(Lattice *lattice, Info *info, Forcesigma *force,
                                                    Momentasigma *momenta, const Fermioncoor *, Fermionkit *kit,
                                                    double epsilon, const int step) {
  evolve_in_time(lattice, info, force, momenta, kit, epsilon, step, GN_LFMN2VF);
}

void ComputeCondensateDirac(const Lattice *lat, double *tr1, double *tr1_abs, double *tr2, double *tr4, double *mu2,
                            double *mu4, double *chi, double *chi_abs, double *chip, double *c12_nosigma,
                            double *c12_withsigma, RandomVec *, Fermion *target_inverted, const Info *,
                            const Fermioncoor *, double inversion_precision, Fermionkit *kit, int) {
  gn_context *c = ctx();
  g_uniform = resolve(g_uniform, "Casuale");
#ifdef GN_DROPIN_PI  // the same solves with the complex M: pi (and its mass) resident first
  if (gn_load_pi(c, lat->pi) != GN_OK) fatal("gn_load_pi");
#endif
  double *target = g_a.data(), *D = g_b.data();
  to_planes(target_inverted->fermion, target, 2);
  double out[11], it = 0.0;
  long long calls = 0;
  const int st =
      gn_condensate(c, lat->sigmamass, inversion_precision, target, D, g_uniform, out, &it, &calls, g_precision);
  if (st < 0) fatal("gn_condensate");
  from_planes(target, target_inverted->fermion, 2);
  from_planes(D, kit->Ddag_inverted_phi_obs.fermion, 2);
  kit->iterations += it;
  kit->CG_call += int(calls);
  double *dst[11] = {tr1, tr1_abs, tr2, tr4, mu2, mu4, chi, chi_abs, chip, c12_nosigma, c12_withsigma};
  for (int k = 0; k < 11; k++) *dst[k] = out[k];
}

void CondensateSigmaPi(const Lattice *lat, const Info *, double *condensate_sigma, double *condensate_sigma_abs,
                       double *mu2, double *mu4, double *chi, double *chip, double *chip_pbc1, double *chip_pbc2) {
  double out[8];
#ifdef GN_DROPIN_PI  // the U(1) order parameter |(sigma, pi)| (observables.c:345)
  if (gn_load_pi(ctx(), lat->pi) != GN_OK) fatal("gn_load_pi");
#endif
  if (gn_condensate_sigma(ctx(), lat->sigma, out) != GN_OK) fatal("gn_condensate_sigma");
  double *dst[8] = {condensate_sigma, condensate_sigma_abs, mu2, mu4, chi, chip, chip_pbc1, chip_pbc2};
  for (int k = 0; k < 8; k++) *dst[k] = out[k];
}

#ifdef GN_DROPIN_PI
void GNB200_SetRandomPair(void (*gauss2)(double *, double *, double, double)) { g_gauss2 = gauss2; }

void ComputeFullPiMass(Lattice *lat, const Fermioncoor *, double *pimass) {
  if (gn_sigma_mass(ctx(), lat->pi, pimass) != GN_OK) fatal("gn_sigma_mass");  // the same 8-corner mean
}

void AddForceFromPiSector(const Lattice *lat, const Info *info, Forcepi *force) {
  // F -= (NFLAV beta_s / 4) pi, as F + pi * (-c): the same rounding
  const double coef = (4 * info->beta_scalar / 4.0);
  if (gn_evolve_momenta(ctx(), force->force, lat->pi, -coef) != GN_OK) fatal("gn_evolve_momenta");
}
bool AddForceFromFermionSectorRespectToPi(const Lattice *lat, const Info *, const Fermioncoor *, Forcepi *force,
                                          Fermionkit *kit) {
  return fermion_force(lat, true, 0.0, force->force, kit, g_tol_high, false);
}
bool ComputePiForce(const Lattice *lat, const Info *info, const Fermioncoor *, Forcepi *force, Fermionkit *kit) {
  return fermion_force(lat, true, info->beta_scalar, force->force, kit, g_tol_high, true);
}

double ComputeFullEnergyForPi(const Lattice *lattice, const Info *info, const Fermioncoor *, const Momentapi *momenta,
                              const Fermionkit *kit) {
  gn_context *c = ctx();
  pair_to_planes(kit->phi, g_a.data());
  pair_to_planes(kit->inverted_phi, g_b.data());
  double H = 0.0;
  if (gn_energy_u1(c, 1, info->beta_scalar, lattice->pi, momenta->momenta, g_a.data(), g_b.data(), &H) != GN_OK)
    fatal("gn_energy_u1");
  return H;
}

void EvolveCoordinatesPi(Lattice *lat, const Momentapi *momenta, const Fermioncoor *, double epsilon) {
  // pi += eps P, then ComputeFullPiMass: the sigma step's arithmetic; no distance counter
  if (gn_evolve_sigma(ctx(), lat->pi, lat->pimass, momenta->momenta, epsilon) != GN_OK) fatal("gn_evolve_sigma");
}
void EvolveMomentaPi(Momentapi *momenta, const Forcepi *force, double epsilon) {
  if (gn_evolve_momenta(ctx(), momenta->momenta, force->force, epsilon) != GN_OK) fatal("gn_evolve_momenta");
}

bool LeapFrog2Pi(Lattice *lattice, Info *info, Forcepi *force, Momentapi *momenta, const Fermioncoor *,
                 Fermionkit *kit, double epsilon, const int step, const char *acceptance_file) {
  return trajectory_pi(lattice, info, force, momenta, kit, epsilon, step, acceptance_file);
}
#endif

}  // extern "C"
