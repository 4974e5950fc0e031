/*
 * gn_b200.h -- C-ABI of the B200 (sm_100a) fermion hot path of the Z2
 * Gross-Neveu sigma-HMC code alefrajoe/3D-Gross-Neveu-model.
 *
 * Plain pointers and sizes only.  One gn_context per lattice size L (even,
 * 4 <= L <= 256) and device.  Every field is a real array in the reference's
 * "fermion lexicographic" order (coordinate.c:25-40, :301-313):
 *   lexicographic n = (x0*L + x1)*L + x2, x2 = time fastest,
 *   fermion index   = n/2 + ((x0+x1+x2) % 2) * V/2   (even sites first),
 * V = L^3.  A complex fermion field (the reference stores `double _Complex`)
 * is passed as two planes of V doubles: real parts, then imaginary parts
 * (ncomp = 2); ncomp = 1 passes real fields (every field of the sigma path is
 * real; only the condensate's phase vector is complex).
 *
 * Functions taking host pointers copy in, run on the GPU and copy out before
 * returning.  They replace the reference functions cited beside them with the
 * same argument meaning; the reference's `struct`-based signatures are
 * provided on top of these by gn_dropin.h.
 *
 * Return values: GN_OK (0) or a negative gn_status; the solvers return
 * GN_NOT_CONVERGED (1) where the reference returns `false`.
 * gn_last_error() describes the last failure of the calling thread.
 */
#ifndef GN_B200_H
#define GN_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define GN_API __attribute__((visibility("default")))
#else
#define GN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gn_context gn_context;

enum gn_status {
  GN_OK = 0,
  GN_NOT_CONVERGED = 1, /* CG hit its iteration cap: the reference's `return false` */
  GN_ERR_ARG = -1,      /* bad argument (size, null pointer, L) */
  GN_ERR_CUDA = -2,     /* a CUDA call failed */
  GN_ERR_TIMEOUT = -3,  /* a device-side wait ran out (bounded barrier) */
  GN_ERR_ABORTED = -4,  /* gn_request_abort() stopped a solve */
  GN_ERR_NO_DEVICE = -5, /* no usable sm_100 device */
  GN_ERR_IO = -6,        /* a file could not be written */
  GN_ERR_NOT_FOUND = -7, /* a file could not be opened for reading */
  GN_ERR_FORMAT = -8     /* a file is short or its check value differs */
};

enum gn_op { GN_OP_M = 0, GN_OP_MT = 1, GN_OP_SUB_M = 2 };
/* GN_PREC_FP64: FP64, tree-ordered global sums (fast).  GN_PREC_MIXED: FP32
 * iterations with FP64 reliable updates.  GN_PREC_FP64_EXACT: FP64 in the
 * reference's exact order of operations -- serial sums, M^T in the order of
 * the reference's scatter -- reproducing its results bit for bit (the Z2
 * model's real fields and the U(1) model's complex ones); one block per
 * solve, so meant for parity runs at small L. */
enum gn_precision { GN_PREC_FP64 = 0, GN_PREC_MIXED = 1, GN_PREC_FP64_EXACT = 2 };
enum gn_integrator { GN_LFMN2VF = 0, GN_LF2 = 1, GN_LFMN2 = 2 };

/* Per right-hand side outcome of a solve. */
typedef struct gn_cg_info {
  int status;          /* 1 converged (counted), 2 start vector already good (not counted), 3 cap, 4 error */
  int counted;         /* 1 when the reference adds `iterations` to kit->iterations and bumps kit->CG_call */
  long long iterations;
  double residual;     /* final |r| of the stopping test */
  double b_norm;       /* |b| */
  long long inner_iterations; /* mixed precision: low-precision iterations (else = iterations) */
  long long reliable_updates; /* mixed precision: FP64 true-residual recomputations */
} gn_cg_info;

/* Parameters of one sigma-HMC trajectory (moleculardynamics.c:859, :1018, :1234). */
typedef struct gn_hmc_params {
  double beta_s;       /* info->beta_scalar */
  double eps;          /* info->epsilon_sigma_HMC */
  int steps;           /* info->steps_sigma_HMC (>= 1; the reference's StartInfo rejects 1, info.c:66) */
  int integrator;      /* gn_integrator; the reference default is GN_LFMN2VF (macro.h:71) */
  double tol_medium;   /* MEDIUM_PRECISION_INVERSION (1e-3) for the MD forces */
  double tol_high;     /* HIGH_PRECISION_INVERSION (1e-9) for H0 / H1 */
  int relative;        /* 0: stop at |r| < tol (reference); 1: at |r| < tol |b| */
  int precision;       /* gn_precision of the solver */
} gn_hmc_params;

typedef struct gn_traj_result {
  int ok;              /* 0 when a solve failed (sigma restored, no uniform drawn) */
  int accepted;
  double dH, H0, H1;
  double cg_iterations; /* added to kit->iterations */
  long long cg_calls;   /* added to kit->CG_call */
  double distance;      /* added to lat->distance_sigma */
  long long inner_iterations, reliable_updates;
} gn_traj_result;

/* ---- context ---------------------------------------------------------- */
GN_API int gn_create(gn_context **ctx, int L, int device);
GN_API void gn_destroy(gn_context *ctx);
GN_API const char *gn_last_error(void);
GN_API long long gn_volume(const gn_context *ctx);
/* Ask a running solve on this context to stop (from another host thread).
 * The solve returns GN_ERR_ABORTED within a few iterations; the flag stays
 * set until gn_request_abort(ctx, 0). */
GN_API void gn_request_abort(gn_context *ctx, int on);
/* Failure-detection self-test (no counterpart in the reference): runs the
 * library's bounded team barrier for a team of two blocks of which only one
 * is launched, so the wait runs out after about a second, as a wait on a
 * block or peer that has died would.  Returns GN_ERR_TIMEOUT, with the context
 * still usable; no fault or trap is involved. */
GN_API int gn_selftest_wait_timeout(gn_context *ctx);

/* Parity mode for the operators that take no precision argument (gn_dirac's
 * M^T, gn_energy): on = the reference's exact order of operations. */
GN_API int gn_set_parity_mode(gn_context *ctx, int on);

/* Mixed precision: a reliable update (x folded into FP64, the true residual
 * recomputed) at least every n inner iterations, besides the ones the
 * residual's drop by 100x triggers.  Default 100; n >= 1. */
GN_API int gn_set_reliable_interval(gn_context *ctx, int n);

/* ---- host-buffer operators (one call = one reference function) -------- */

/* ComputeFullSigmaMass, sigma.c:75-94: sm(x) = 1/8 sum of sigma over the 8
 * dual sites of the cube at x. */
GN_API int gn_sigma_mass(gn_context *ctx, const double *sigma, double *sigmamass);

/* op GN_OP_M:     out = M in      (DiracFermion, dirac.c:46-82)
 * op GN_OP_MT:    out = M^T in    (AdjDiracFermion, dirac.c:88-123)
 * op GN_OP_SUB_M: out = out - M in (SubtractDiracFermion, dirac.c:213-247)
 * in/out hold ncomp planes of V doubles. */
GN_API int gn_dirac(gn_context *ctx, const double *sigmamass, const double *in, double *out, int ncomp, int op);

/* CG on A = M M^T (conjugategradient.c:13-107 for variant 0, which first tests
 * the incoming x as the reference does under START_X0_NULL; :115-182 for
 * variant 1, which starts from x = 0).  nrhs independent systems, each of
 * ncomp planes: b and x hold nrhs*ncomp*V doubles; x is in/out.  Stops when
 * |r| < tol (relative = 0, the reference's absolute test) or |r| < tol |b|.
 * max_iter <= 0 means the reference's cap, V + 1 (macro.h:134).
 * Returns GN_OK when every system converged, else GN_NOT_CONVERGED. */
GN_API int gn_cg(gn_context *ctx, const double *sigmamass, const double *b, double *x, int nrhs, int ncomp, double tol,
          int variant, int relative, long long max_iter, int precision, gn_cg_info *info);

/* ComputeSigmaForce (moleculardynamics.c:631-647): for both flavours X_f =
 * (M M^T)^-1 phi_f by variant-0 CG from the incoming X_f (tolerance tol), then
 * Y_f = M^T X_f and F = sum_f 1/8 sum_corners X_f Y_f - (N_f beta_s / 2) sigma.
 * phi, X, Y hold 2*V doubles (flavour 0 then 1); X in/out, Y and force out.
 * info[2] (may be NULL). */
GN_API int gn_sigma_force(gn_context *ctx, double beta_s, const double *sigma, const double *sigmamass, const double *phi,
                   double *X, double *Y, double tol, double *force, int precision, gn_cg_info *info);

/* ComputeFullEnergyForSigma (moleculardynamics.c:299-319):
 * H = 1/2 sum P^2 + 1/2 sum_f phi_f . X_f + (N_f beta_s / 4) sum sigma^2. */
GN_API int gn_energy(gn_context *ctx, double beta_s, const double *sigma, const double *P, const double *phi,
              const double *X, double *H);

/* EvolveCoordinatesSigma (moleculardynamics.c:824-836): sigma += eps P, then
 * sigmamass recomputed.  sigma and sigmamass are in/out and out. */
GN_API int gn_evolve_sigma(gn_context *ctx, double *sigma, double *sigmamass, const double *P, double eps);

/* EvolveMomentaSigma (moleculardynamics.c:843-848): P += eps F. */
GN_API int gn_evolve_momenta(gn_context *ctx, double *P, const double *F, double eps);

/* ComputeCondensateDirac (condensate.c:114-244) with CONDENSATE_PRECISION 1
 * and Z2 noise drawn by uniform() (the reference's Casuale, random.c:28),
 * V draws per noise vector, in the reference's order.
 * target (2V: complex planes) is target_inverted, in/out (each solve first
 * tests it, as the reference does); D (2V) receives kit->Ddag_inverted_phi_obs.
 * out[11] = tr1, |tr1|, tr2, tr4, mu2, mu4, chi, |chi|, chi_p, c12 without
 * sigma, c12 with sigma.  cg_iterations / cg_calls (may be NULL) receive the
 * amounts the reference adds to kit->iterations / kit->CG_call.  In a context
 * holding pi (gn_load_pi) M is the U(1) model's complex M with the resident
 * pimass, as the reference's PI_INTERACTION build runs it; precision
 * GN_PREC_FP64 or GN_PREC_MIXED there. */
GN_API int gn_condensate(gn_context *ctx, const double *sigmamass, double tol, double *target, double *D,
                  double (*uniform)(void), double *out, double *cg_iterations, long long *cg_calls, int precision);

/* CondensateSigmaPi (observables.c:323-369, the Z2 model) of a sigma field:
 * sigma (V doubles, fermion order) on the host, or NULL for the resident
 * sigma (no transfer of the field).  out[8] = condensate_sigma,
 * |condensate_sigma|, mu2, mu4, chi, chip, chip_pbc1, chip_pbc2, the
 * reference's argument order.  The sums run on the device.  In the U(1) model
 * (after gn_load_pi) the order parameter is |(sigma, pi)| with the resident
 * pi, as under PI_INTERACTION (observables.c:354-357). */
GN_API int gn_condensate_sigma(gn_context *ctx, const double *sigma, double *out);
/* The same for a device sigma (V doubles). */
GN_API int gn_condensate_sigma_device(gn_context *ctx, const double *sigma, double *out);

/* ---- the U(1) model (the reference's PI_INTERACTION) --------------------
 * M = D + sigmamass + i eps(x) pimass (dirac.c:65-69; eps = +1 on even, -1 on
 * odd sites), M^dagger = -D + sigmamass - i eps pimass.  Fermion fields are
 * complex: two planes (real, imaginary) per system; a field of both flavours
 * is four planes (flavour f: planes 2f, 2f + 1).  Precisions as for the Z2
 * model; in parity mode (gn_set_parity_mode, or a call with
 * GN_PREC_FP64_EXACT) M^dagger, the solves and the energies follow the
 * reference's order of operations.
 *
 * gn_load_pi sets the resident pi (V doubles, fermion order; pimass =
 * ComputeFullPiMass, pi.c:44-60) and switches the context to the U(1) model:
 * gn_trajectory then runs the sigma integrators with this M on complex
 * fields.  gn_set_u1(ctx, 0) switches back to the Z2 model (real fields). */
GN_API int gn_load_pi(gn_context *ctx, const double *pi);
GN_API int gn_store_pi(gn_context *ctx, double *pi, double *pimass);
GN_API int gn_set_u1(gn_context *ctx, int on);

/* gn_dirac with the complex mass: in/out hold nsys complex systems (2 nsys V). */
GN_API int gn_dirac_u1(gn_context *ctx, const double *sigmamass, const double *pimass, const double *in, double *out,
                       int nsys, int op);
/* CG on M M^dagger for nrhs (1 or 2) complex systems (b, x: 2 nrhs V; x in/out),
 * variant / relative / max_iter as gn_cg; precision GN_PREC_FP64,
 * GN_PREC_MIXED (FP32 inner iterations, FP64 reliable updates, the same
 * true-residual test) or GN_PREC_FP64_EXACT.  info[nrhs] may be NULL. */
GN_API int gn_cg_u1(gn_context *ctx, const double *sigmamass, const double *pimass, const double *b, double *x,
                    int nrhs, double tol, int variant, int relative, long long max_iter, int precision,
                    gn_cg_info *info);
/* ComputeSigmaForce (moleculardynamics.c:631-647) and ComputePiForce
 * (:736-752) in the U(1) model: X_f = (M M^dagger)^-1 phi_f by variant-0 CG
 * from the incoming X_f (tolerance tol), Y_f = M^dagger X_f, then
 *   sigma: F = sum_f 1/8 sum_corners Re(conj X_f Y_f) - (N_f beta_s / 2) sigma
 *   pi:    F = sum_f 1/8 sum_corners Re(i eps conj X_f Y_f) - (N_f beta_s / 4) pi
 * phi, X, Y: 4V (X in/out); field = sigma or pi (V); force out (V).  FP64;
 * the exact-order solver and M^dagger in parity mode. */
GN_API int gn_sigma_force_u1(gn_context *ctx, double beta_s, const double *sigma, const double *sigmamass,
                             const double *pimass, const double *phi, double *X, double *Y, double tol, double *force,
                             gn_cg_info *info);
GN_API int gn_pi_force(gn_context *ctx, double beta_s, const double *pi, const double *sigmamass,
                       const double *pimass, const double *phi, double *X, double *Y, double tol, double *force,
                       gn_cg_info *info);
/* ComputeFullEnergyForSigma (which = 0, moleculardynamics.c:299-319) or
 * ComputeFullEnergyForPi (which = 1, :349-369) with complex phi, X (4V):
 *   H = 1/2 sum P^2 + 1/2 sum_f Re(conj phi_f X_f) + c beta_s-term,
 * c = N_f beta_s / 4 times sum sigma^2, or N_f beta_s / 8 times sum pi^2. */
GN_API int gn_energy_u1(gn_context *ctx, int which, double beta_s, const double *field, const double *P,
                        const double *phi, const double *X, double *H);
/* LeapFrog2Pi (moleculardynamics.c:1743-1870) on the resident sigma and pi.
 * Draws as the reference: the pi momenta in pairs, gauss_pair(&P[x],
 * &P[x + V/2]) for x < V/2 (DrawPiMomentaFromGaussianDistribution calls
 * Gauss2MeanVariance(.., 0, 1), random.c:129), then chi_0, chi_1 from gauss()
 * (Gauss1); phi_f = M chi_f; every inversion a variant-0 CG at
 * params->tol_high; the Metropolis test with uniform().  pi is restored on
 * reject or on a failed solve (res->ok = 0).  params->eps and ->steps are the
 * pi step (epsilon_pi_HMC, steps_pi_HMC); integrator and tol_medium are not
 * used; precision GN_PREC_FP64 or GN_PREC_MIXED.  gauss_pair and gauss NULL: P_pi (GN_F_PI_P)
 * and the real parts of GN_F_CHI_C as they are. */
GN_API int gn_trajectory_pi(gn_context *ctx, const gn_hmc_params *params, void (*gauss_pair)(double *, double *),
                            double (*gauss)(void), double (*uniform)(void), gn_traj_result *res);

/* ---- checkpoints: the reference's lattice file ------------------------- */

/* The HMC bookkeeping the file carries (simulation.c:162-178, struct Info
 * fields, info.h).  The lengths of the HMC trajectories are not in the file,
 * as in the reference. */
typedef struct gn_hmc_counters {
  double epsilon_link, epsilon_pi;
  int story_link, story_sigma, story_pi;
  int accepted_link, done_link;
  int accepted_sigma, done_sigma;
  int accepted_pi, done_pi;
  int measure;
} gn_hmc_counters;

/* The file of WriteBinaryLattice / ReadBinaryLattice (simulation.c:129-401)
 * for the sigma model (SIGMA_INTERACTION without PI_INTERACTION), DIM = 3:
 *   V x 3 complex links (lexicographic site, then direction), V sigma values
 *   (fermion order), the check value sum_x sum_d (carg(link) + sigmamass[x]/3)
 *   accumulated in that order, then the counters: epsilon_link, an 8-byte
 *   slot, accepted_link, done_link, a slot, accepted_sigma, done_sigma,
 *   epsilon_pi, a slot, accepted_pi, done_pi, measure.  The reference writes
 *   the int story fields with sizeof(double), so the three slots hold the
 *   ints {story_link, story_sigma}, {story_sigma, story_pi}, {story_pi, the
 *   struct's padding (written 0 here)}.
 * Host functions, no device needed.  links (6V doubles: re, im per link) may
 * be NULL: unit links, the reference's START_LINK_IDENTITY.
 *
 * write: as WriteBinaryLattice, an existing path_copy is removed and path is
 * renamed to path_copy before path is written (path_copy may be NULL: no
 * rotation).  Returns GN_OK or GN_ERR_IO. */
GN_API int gn_checkpoint_write_file(const char *path, const char *path_copy, int L, const double *sigma,
                                    const double *sigmamass, const double *links, const gn_hmc_counters *c);
/* read one file: sigma (V), links (6V, may be NULL), counters, and the stored
 * check value.  GN_OK, GN_ERR_NOT_FOUND (cannot open) or GN_ERR_FORMAT (short). */
GN_API int gn_checkpoint_read_file(const char *path, int L, double *sigma, double *links, gn_hmc_counters *c,
                                   double *check);
/* The check value of (sigmamass, links) in the reference's order (links NULL: unit). */
GN_API double gn_checkpoint_check_value(int L, const double *sigmamass, const double *links);

/* A context's resident sigma: save writes it (sigmamass computed on the
 * device, links unit).  load follows ReadBinaryLattice with try_copy: path,
 * else path_copy when path cannot be opened or fails (short, or the check
 * value recomputed from the loaded sigma differs bit for bit); on success
 * sigma becomes the resident field and c receives the counters.  Returns
 * GN_OK, GN_ERR_NOT_FOUND (neither file exists: a fresh start) or
 * GN_ERR_FORMAT (every candidate failed). */
GN_API int gn_checkpoint_save(gn_context *ctx, const char *path, const char *path_copy, const gn_hmc_counters *c);
GN_API int gn_checkpoint_load(gn_context *ctx, const char *path, const char *path_copy, gn_hmc_counters *c);

/* ---- resident sigma-HMC state ------------------------------------------ */

/* Upload sigma (V doubles) as the resident field; sigmamass is recomputed. */
GN_API int gn_load_sigma(gn_context *ctx, const double *sigma);
/* Download the resident sigma and sigmamass (either may be NULL). */
GN_API int gn_store_sigma(gn_context *ctx, double *sigma, double *sigmamass);

/* Resident vectors for gn_read_state / gn_write_state. */
enum gn_field { GN_F_P = 0, GN_F_F = 1, GN_F_CHI = 2, GN_F_PHI = 3, GN_F_X = 4, GN_F_Y = 5 };
/* P and F are V doubles; CHI, PHI, X (kit->inverted_phi), Y (kit->inverted_phi_obs) are 2V. */
GN_API int gn_read_state(gn_context *ctx, int field, double *out);
GN_API int gn_write_state(gn_context *ctx, int field, const double *in);

/* One sigma-HMC trajectory on the resident state, the body of
 * LeapFrog2MinimumNormSigmaVelocityFirst (moleculardynamics.c:1234-1434) or of
 * LeapFrog2Sigma (:859-1005) / LeapFrog2MinimumNormSigma (:1018-1221):
 * P and chi_0, chi_1 are drawn on the host with gauss() (V each, in that
 * order; the reference's Gauss1), phi_f = M chi_f, every solve and MD step
 * runs on the device, dH is formed in FP64 and the Metropolis test
 * uniform() <= exp(-dH) is made on the host with the reference's uniform.  On
 * rejection sigma is restored.  If gauss is NULL, P and chi are taken from the
 * resident GN_F_P / GN_F_CHI buffers instead (already on the device).
 * Returns GN_OK, or GN_NOT_CONVERGED when a solve failed (then res->ok = 0 and
 * sigma is restored, as in the reference). */
GN_API int gn_trajectory(gn_context *ctx, const gn_hmc_params *params, double (*gauss)(void), double (*uniform)(void),
                  gn_traj_result *res);

/* The molecular dynamics of one trajectory without draws and without the
 * Metropolis test (a reversibility check in the manner of the reference's
 * DEBUG_LF2_SIGMA): from the resident sigma, P (GN_F_P) and phi (GN_F_PHI;
 * in the U(1) model GN_F_PHI_C), exactly the initial solve, energies and MD
 * schedule gn_trajectory runs for params->integrator.  phi is not formed from
 * chi.  res->H0, H1, dH are the energies before and after; sigma and P are
 * left evolved (res->accepted = 1), or restored when a solve fails
 * (GN_NOT_CONVERGED).  Flipping P and evolving again retraces the trajectory.
 * For the reference's own helpers, with their tolerance pattern, see
 * gn_evolve_sigma_in_time. */
GN_API int gn_md_evolve(gn_context *ctx, const gn_hmc_params *params, gn_traj_result *res);

/* The reference's MD helpers, replaced one for one:
 * EvolveSigmaInTimeLF2 (moleculardynamics.c:1460, params->integrator GN_LF2),
 * EvolveSigmaInTimeMinimumNormLF2 (:1489, GN_LFMN2) and
 * EvolveSigmaInTimeMinimumNormSigmaVelocityFirst (:1551, GN_LFMN2VF), on the
 * resident sigma, P (GN_F_P), phi (GN_F_PHI) and X (GN_F_X, the start of
 * every early-exit solve); in the U(1) model with the complex M on
 * GN_F_PHI_C and GN_F_X_C (Y in GN_F_Y_C), as the PI_INTERACTION build's
 * helpers run.
 * Their step sequences and tolerances are the helpers' own: the LF2 and
 * LFMN2 helpers take their first force at tol_high, the velocity-first one
 * runs an X0-imposed solve before and an early-exit solve after the
 * integrator's MD.  No draws, no energies, no Metropolis test, sigma never
 * restored; as in the reference a force whose solve fails is left at zero and
 * the MD goes on.  Leaves sigma, sigmamass, P, F, X and Y (= M^T X) evolved;
 * res->cg_iterations / cg_calls add up the counted solves, res->distance the
 * sigma steps, res->ok = 0 (and GN_NOT_CONVERGED) if any solve failed. */
GN_API int gn_evolve_sigma_in_time(gn_context *ctx, const gn_hmc_params *params, gn_traj_result *res);

/* ---- device-resident entry points ------------------------------------- */

/* The context's CUDA stream (a cudaStream_t); every device-pointer call below
 * is ordered on it. */
GN_API void *gn_stream(gn_context *ctx);

/* Device pointer of a resident field: GN_F_* above, or GN_F_SIGMA / GN_F_SM
 * (the current sigma and sigmamass, V doubles each).  U(1) model: GN_F_PI /
 * GN_F_PM (pi, pimass), and for gn_read_state / gn_write_state too the pi
 * momenta and force (V) and the complex chi, phi, X, Y of both flavours (4V). */
enum { GN_F_SIGMA = 6, GN_F_SM = 7, GN_F_PI_P = 8, GN_F_PI_F = 9, GN_F_CHI_C = 10, GN_F_PHI_C = 11, GN_F_X_C = 12,
       GN_F_Y_C = 13, GN_F_PI = 14, GN_F_PM = 15 };
GN_API double *gn_field_ptr(gn_context *ctx, int field);

/* gn_dirac on device pointers; asynchronous on gn_stream(ctx). */
GN_API int gn_dirac_device(gn_context *ctx, const double *sigmamass, const double *in, double *out, int ncomp, int op);

/* gn_cg on device pointers (b, x: nrhs*ncomp*V doubles each, not aliased);
 * returns after the solve (it reads the per-system outcome back). */
GN_API int gn_cg_device(gn_context *ctx, const double *sigmamass, const double *b, double *x, int nrhs, int ncomp,
                        double tol, int variant, int relative, long long max_iter, int precision, gn_cg_info *info);

/* gn_trajectory with the draws already on the device: P (V doubles) and
 * chi (2V doubles, flavour 0 then 1) are device pointers, copied into the
 * resident buffers on gn_stream(ctx); the Metropolis uniform still comes from
 * uniform() on the host. */
GN_API int gn_trajectory_device(gn_context *ctx, const gn_hmc_params *params, const double *P, const double *chi,
                                double (*uniform)(void), gn_traj_result *res);

/* Number of kernels this context has launched so far. */
GN_API long long gn_launch_count(gn_context *ctx);

/* Overwrite a device buffer larger than the L2 cache on gn_stream(ctx), so the
 * next kernel starts cold (used by benchmarks). */
GN_API int gn_flush_l2(gn_context *ctx);

/* ---- allocation-free solve --------------------------------------------- */

/* No counterpart in the reference (it is an addition of this library).
 * CG on (M M^T) x = b for one real right-hand side, like gn_cg_device with
 * precision GN_PREC_FP64, for callers that cannot allocate device memory once
 * they run: an HMC driver that sizes all of its buffers once up front, as the
 * reference's Allocate* functions do, or an application that gives this
 * library a fixed budget from its own pool allocator, where a cudaMalloc
 * would escape the budget or fail.  It needs no gn_context and calls no
 * cudaMalloc / cudaFree: the solver's scratch is a static device array of
 * about 1 MiB, sized for L <= 32 (32768 sites), that every GPU loading this
 * library holds until exit.  Larger L returns GN_ERR_ARG.  sigmamass, b
 * (input) and x (in/out) are device pointers of V doubles on the current
 * device; stream is a cudaStream_t (NULL = default).  All calls share the
 * static array: calls that overlap on the GPU race, and so do calls from
 * several host threads on one stream, so serialise whole calls on the host.
 * The first call on each device sets up the array's address and should come
 * before any stream capture.  Returns like gn_cg; gn_cg_noalloc_error()
 * describes the failure of the calling thread's last call ("" after a call
 * that did not fail). */
GN_API int gn_cg_noalloc(int L, const double *sigmamass, const double *b, double *x, double tol, int variant,
                         int relative, long long max_iter, void *stream, gn_cg_info *info);
GN_API const char *gn_cg_noalloc_error(void);
/* The largest V = L^3 gn_cg_noalloc accepts. */
GN_API long long gn_cg_noalloc_max_volume(void);

/* ---- batched chains ------------------------------------------------------ */

/* No counterpart in the reference, which runs one chain per process
 * (observables.c:178 drives one lattice).  An ensemble holds many independent
 * sigma-HMC chains, each with its own lattice size L (even, 4..256) and
 * beta_s, on one GPU.  Every trajectory is the reference's (the integrators of
 * moleculardynamics.c:859 / :1018 / :1234, energy of :299, Metropolis test
 * u <= exp(-dH) with sigma restored on reject); every solve is the
 * CG (mixed precision or FP64) to a true relative residual `tol`, from x = 0.  The
 * random numbers (momenta, pseudofermion sources, the Metropolis uniform) come
 * from the chain's own Philox4x64-10 stream, key (seed, stream id), counter
 * (trajectory number, field, site block): a chain's trajectory depends only on
 * its own state, L, beta_s, stream id and the team layout, not on the chains
 * beside it.  All chains advance together: one persistent kernel per MD step,
 * the trajectory replayed as a CUDA graph. */
typedef struct gn_ensemble gn_ensemble;

typedef struct {
  double eps;     /* MD step size */
  int steps;      /* MD steps per trajectory (>= 1) */
  int integrator; /* GN_LFMN2VF, GN_LF2 or GN_LFMN2 */
  double tol;     /* relative tolerance of every solve, true residual (> 0) */
  int precision;  /* GN_PREC_MIXED or GN_PREC_FP64 */
} gn_ens_params;

typedef struct {
  long long trajectories;       /* since the last reset */
  long long accepted;
  long long failed;             /* trajectories rejected because a solve did not converge */
  long long cg_iterations;      /* inner (FP32) iterations of the counted solves */
  long long reliable_updates;
  double sum_dH, sum_exp_mdH;   /* sums of dH and exp(-dH) */
  double sum_sigma2;            /* sum over trajectories of (1/V) sum_x sigma(x)^2 after the trajectory */
  double last_dH;
  int last_accepted;
  long long total_trajectories; /* since creation (the Philox counter of the next one) */
  /* the reference's struct Info bookkeeping of the chain (moleculardynamics.c:1385-1416) */
  long long total_accepted;     /* hybrid_accepted_sigma; hybrid_done_sigma is total_trajectories */
  int story;                    /* story_sigma: +n after n accepts in a row, -n after n rejects */
  int local_accepted, local_done;
  double epsilon_scale;         /* the chain's epsilon / gn_ens_params.eps (autoregulation) */
} gn_chain_stats;

/* nchains chains: L[c], beta_s[c]; stream_ids[c] (NULL: c) keys each chain's
 * Philox stream together with seed.  sigma starts at 0: load it per chain. */
GN_API int gn_ensemble_create(gn_ensemble **ens, int nchains, const int *L, const double *beta_s,
                              const unsigned long long *stream_ids, unsigned long long seed, int device);
GN_API void gn_ensemble_destroy(gn_ensemble *ens);
/* sigma of chain c (V doubles, fermion order) in and out; sm optional on output. */
GN_API int gn_ensemble_load_sigma(gn_ensemble *ens, int chain, const double *sigma);
GN_API int gn_ensemble_store_sigma(gn_ensemble *ens, int chain, double *sigma, double *sigmamass);
/* Team layout: chains with V >= big_min_volume run on groups of group_blocks
 * blocks, the others on single blocks (group_blocks = 1: all on single blocks).
 * The layout fixes the order of the reductions, hence the last bits. */
GN_API int gn_ensemble_set_layout(gn_ensemble *ens, int group_blocks, long long big_min_volume);
/* Autotuner: times the refresh-and-solve slice (no effect on any chain's
 * results) for every candidate layout, keeps the fastest and returns it. */
GN_API int gn_ensemble_tune(gn_ensemble *ens, const gn_ens_params *p, int *group_blocks, long long *big_min_volume);
/* ntraj trajectories of every chain; use_graph = 1 replays a captured CUDA
 * graph (falls back to direct launches where capture is not possible).
 * GN_ERR_TIMEOUT if a team barrier timed out. */
GN_API int gn_ensemble_run(gn_ensemble *ens, const gn_ens_params *p, int ntraj, int use_graph);
/* Per-chain statistics into out[nchains] (may be NULL); reset = 1 zeroes the
 * accumulators afterwards. */
GN_API int gn_ensemble_stats(gn_ensemble *ens, gn_chain_stats *out, int reset);
/* Per-chain means of the CondensateSigmaPi outputs (gn_condensate_sigma's
 * order) over the trajectories that gn_chain_stats.trajectories counts:
 * out[8 * nchains].  The kernel takes the sums on the device after every
 * trajectory, so no sigma leaves the GPU (TakeMeasures' averaging,
 * observables.c:259-292, with IMEAS = the trajectories since the last reset);
 * gn_ensemble_stats(..., reset = 1) zeroes them with the other accumulators. */
GN_API int gn_ensemble_observables(gn_ensemble *ens, double *out);
/* UpdateHMCParameters (info.c:123-135, the reference's AUTOREGULATION) for
 * chain c (c < 0: every chain), on the device after every trajectory: after
 * 100 trajectories the chain's epsilon is multiplied by 1.15 / 1.08 or
 * divided by 1.08 / 1.15 for a local acceptance >= 0.85 / >= 0.8 / >= 0.75 /
 * below, and the local counters restart.  Switching on restarts them too.
 * The epsilon of chain c is gn_ens_params.eps times its epsilon_scale. */
GN_API int gn_ensemble_set_autoregulation(gn_ensemble *ens, int chain, int on);
/* Checkpoint of chain c in the reference's lattice file (gn_checkpoint_save /
 * gn_checkpoint_load).  save with c == NULL takes the sigma counters from the
 * chain (accepted_sigma = total_accepted, done_sigma = total_trajectories,
 * story_sigma = story; the others 0).  load puts sigma in place of the
 * chain's and sets total_trajectories, total_accepted and story from the
 * file's done_sigma, accepted_sigma and story_sigma: the trajectory count is
 * the chain's Philox counter, so a chain reloaded with the same seed and
 * stream id continues its random stream where it stopped. */
GN_API int gn_ensemble_checkpoint_save(gn_ensemble *ens, int chain, const char *path, const char *path_copy,
                                       const gn_hmc_counters *c);
GN_API int gn_ensemble_checkpoint_load(gn_ensemble *ens, int chain, const char *path, const char *path_copy,
                                       gn_hmc_counters *c);

/* The observables line TakeMeasures appends (observables.c:266-292) with
 * OBS_CONDENSATE and OBS_CONDENSATE_SIGMA defined: measure, L, beta,
 * beta_scalar, mass, average CG iterations, average sigma distance, then
 * cond_dirac[11] (gn_condensate's out; NULL leaves the group out) and
 * cond_sigma[8] (NULL leaves it out), tab-separated, every double "%.16f",
 * and a newline.  Returns the length snprintf reports, or GN_ERR_ARG. */
GN_API int gn_format_measure_line(char *buf, size_t size, int measure, int L, double beta, double beta_scalar,
                                  double mass, double avg_iterations, double avg_distance, const double *cond_dirac,
                                  const double *cond_sigma);
/* The CUDA stream (cudaStream_t) the ensemble's work runs on. */
GN_API void *gn_ensemble_stream(gn_ensemble *ens);
/* The layout in use, whether the last run used the graph, kernel launches per trajectory. */
GN_API int gn_ensemble_info(gn_ensemble *ens, int *group_blocks, long long *big_min_volume, int *graph_used,
                            int *launches_per_trajectory);

/* ---- serving ------------------------------------------------------------- */

/* No counterpart in the reference.  A server keeps chains resident on the GPU
 * (sigma and its mass) and runs requests on them with continuous batching:
 *   GN_REQ_TRAJECTORY  one HMC trajectory of the chain (the ensemble's: the
 *                      parameters given at creation, solves in their precision);
 *   GN_REQ_SOLVE       one solve of (M M^T) x = b at the chain's sigma, b ~ N(0, 1);
 *   GN_REQ_CONDENSATE  the estimate (1/n) sum_k xi_k . M^T (M M^T)^-1 xi_k / V
 *                      of tr M^-1 / V (condensate.c:142-145) from n Z2 vectors.
 * gn_server_step launches the batched kernel once: every running request
 * advances by one slice (a trajectory has one per MD step, a solve one, a
 * condensate one per two noise vectors), finished requests retire, and queued
 * ones are admitted in arrival order when their chain is free and their work
 * arrays (about 196 bytes per site) fit the memory budget.  A request's draws
 * come from its chain's Philox stream with its number among the chain's
 * requests (trajectories: the chain's trajectory number) as the counter, so its
 * result does not depend on the requests running beside it.  Times are seconds on the server's clock
 * (gn_server_clock). */
typedef struct gn_server gn_server;

enum gn_request_type { GN_REQ_TRAJECTORY = 0, GN_REQ_SOLVE = 1, GN_REQ_CONDENSATE = 2 };

typedef struct {
  long long id;
  int type;           /* gn_request_type */
  int status;         /* 0 queued, 1 running, 2 done */
  int chain;
  int noise_vectors;  /* condensate requests */
  int failed;         /* a solve did not converge (a trajectory is then rejected) */
  int accepted;       /* trajectory */
  double t_arrival, t_admit, t_done;
  double dH;          /* trajectory */
  double value;       /* condensate estimate */
  long long cg_iterations;
} gn_request_info;

/* traj: the trajectories' integrator, steps, step size, and the tolerance and
 * precision of every solve.  mem_budget_bytes bounds the running requests'
 * work arrays.
 * Team tiers (0 to 3): a chain with V >= tier_min_volume[t] (and below the
 * earlier tiers' bounds) runs on teams of tier_blocks[t] blocks; sizes >= 2,
 * each dividing the previous one, volumes decreasing; smaller chains run on
 * single blocks.  The top tier's teams grow to share the whole GPU among the
 * running top-tier requests (tier_blocks[0] is their minimum size), so a
 * request's result is bit for bit independent of the load below the top tier
 * and agrees to the solver tolerance in it. */
GN_API int gn_server_create(gn_server **srv, const gn_ens_params *traj, double mem_budget_bytes,
                            unsigned long long seed, int ntiers, const int *tier_blocks,
                            const long long *tier_min_volume, int device);
GN_API void gn_server_destroy(gn_server *srv);
/* A resident chain: returns its index (>= 0) or a negative status. */
GN_API int gn_server_add_chain(gn_server *srv, int L, double beta_s, const double *sigma,
                               unsigned long long stream_id);
GN_API double gn_server_clock(gn_server *srv);
/* Queues a request (noise_vectors: condensate only, even, 2..64); returns its id or a negative status. */
GN_API long long gn_server_submit(gn_server *srv, int chain, int type, int noise_vectors, double t_arrival);
/* One step of the server; *completed = requests finished in it. */
GN_API int gn_server_step(gn_server *srv, int *completed);
GN_API int gn_server_request(gn_server *srv, long long id, gn_request_info *out);
/* A finished solve's x (V doubles). */
GN_API int gn_server_solution(gn_server *srv, long long id, double *x);
GN_API int gn_server_chain_sigma(gn_server *srv, int chain, double *sigma);
GN_API int gn_server_load(gn_server *srv, int *running, int *queued, long long *bytes_in_use);

#ifdef __cplusplus
}
#endif
#endif /* GN_B200_H */
