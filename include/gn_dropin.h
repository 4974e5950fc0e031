/*
 * gn_dropin.h -- the reference's own hot-path functions, with the reference's
 * signatures and struct layouts, implemented on the B200 library
 * (3d-gross-neveu-model_b200/lib/libgn_dropin.so over libgn_b200.so).
 *
 * A program built from the reference's sources links this library ahead of
 * (or instead of) the reference's dirac.c, conjugategradient.c, sigma.c,
 * moleculardynamics.c and condensate.c: every call below then runs on the GPU
 * with the reference's argument meaning, side effects on the structs and
 * return values.  The struct layouts must equal the reference's, so they are
 * restated here member for member (lattice.h:10-56, fermion.h:12-33, :49-52,
 * :77-80, :93-112, info.h:7-61 with HYBRID_MC defined and METROPOLIS_LINK not,
 * as macro.h configures them, link.h:7-10, moleculardynamics.h:65-68, :91-94,
 * condensate.h:11-15).  A program that includes the reference's own headers
 * does not include this file; it only links the library.
 *
 * Set-up: the lattice size is a compile-time macro (LSPACE) in the reference;
 * tell the library once with GNB200_SetLattice(LSPACE) (or set the environment
 * variable GN_LSPACE).  The integrators and the condensate draw their random
 * numbers from the host program's Gauss1 / Casuale (random.c:88 / :28), found
 * by name at the first use, or from functions given to GNB200_SetRandom.
 * Tolerances default to the reference's MEDIUM / HIGH_PRECISION_INVERSION
 * (1e-3 / 1e-9, macro.h:135-136); GNB200_SetTolerances changes them.
 */
#ifndef GN_DROPIN_H
#define GN_DROPIN_H

#include <complex.h>
#include <stdbool.h>

#include "gn_b200.h"

#ifdef __cplusplus
extern "C" {
#define GN_COMPLEX double _Complex
#else
#define GN_COMPLEX double complex
#endif

/* ---- the reference's structs (layouts as listed above) ------------------ */
struct Link { GN_COMPLEX link; };

struct Lattice {
  struct Link *dlink;
  double *sigma, *sigmamass;
  double *pi, *epsilon_pi, *pimass;
  int *site, *lattice_site, *pp, *mm, *fermionsite, *fermionpp, *fermionmm;
  double *eta_pp, *eta_mm, *eta_pbc;
  double distance_link, distance_sigma, distance_pi;
  int done_link, done_sigma, done_pi;
};

struct Fermioncoor {
  int *site, *pp, *mm, *fermionsite, *fermionpp, *fermionmm;
  double *eta_pp, *eta_mm, *eta_pbc;
};

struct Fermion { GN_COMPLEX *fermion; };
struct ManyFermions { struct Fermion *flav; };

struct Fermionkit {
  struct ManyFermions r_k, p_k, chi, phi, inverted_phi, inverted_phi_obs;
  struct Fermion Ddag_inverted_phi_obs, temp1, temp2, tempbminusx0, bminusax0;
  double iterations;
  int CG_call;
};

struct Info {
  double beta, beta_scalar, mass;
  int sosia, measure;
  double epsilon_link_HMC, distance_link_HMC;
  int steps_link_HMC;
  double epsilon_sigma_HMC, distance_sigma_HMC;
  int steps_sigma_HMC;
  double epsilon_pi_HMC, distance_pi_HMC;
  int steps_pi_HMC;
  int hybrid_accepted_link, hybrid_done_link;
  double hybrid_done_acceptance_link;
  int hybrid_accepted_sigma, hybrid_done_sigma;
  double hybrid_done_acceptance_sigma;
  int local_accepted_sigma, local_done_sigma;
  double local_acceptance_sigma;
  int hybrid_accepted_pi, hybrid_done_pi;
  double hybrid_done_acceptance_pi;
  double delta_H_link, delta_H_sigma, delta_H_pi;
  int story_link, story_sigma, story_pi;
};

struct Forcesigma { double *force; };
struct Momentasigma { double *momenta; };
struct RandomVec { struct Fermion *vec; };

/* ---- set-up (no counterpart in the reference) --------------------------- */
GN_API void GNB200_SetLattice(int L);
GN_API void GNB200_SetRandom(double (*gauss)(void), double (*uniform)(void));
GN_API void GNB200_SetTolerances(double medium, double high);
GN_API void GNB200_SetPrecision(int precision); /* GN_PREC_FP64 (default), GN_PREC_MIXED or GN_PREC_FP64_EXACT */
GN_API gn_context *GNB200_Context(void);      /* the library's context (created on first use) */

/* ---- dirac.c ------------------------------------------------------------- */
/* dirac.c:46 */
GN_API void DiracFermion(const struct Lattice *lat, const struct Fermion *fermion, struct Fermion *target,
                         const struct Info *info, const struct Fermioncoor *fermioncoor);
/* dirac.c:88 */
GN_API void AdjDiracFermion(const struct Lattice *lat, const struct Fermion *fermion, struct Fermion *target,
                            const struct Info *info, const struct Fermioncoor *fermioncoor);
/* dirac.c:213 */
GN_API void SubtractDiracFermion(const struct Lattice *lat, const struct Fermion *fermion, struct Fermion *target,
                                 const struct Info *info, const struct Fermioncoor *fermioncoor);

/* ---- conjugategradient.c --------------------------------------------------- */
/* conjugategradient.c:13 */
GN_API bool ConjugateGradientFastDiracAdjFastDiracToTheMinusOne(const struct Lattice *lat, const struct Fermion *fermion,
                                                                struct Fermion *target_inverted,
                                                                const struct Info *info,
                                                                const struct Fermioncoor *fermioncoor,
                                                                double inversion_precision, struct Fermionkit *kit,
                                                                int f);
/* conjugategradient.c:115 */
GN_API bool StartX0ImposedConjugateGradientFastDiracAdjFastDiracToTheMinusOne(
    const struct Lattice *lat, const struct Fermion *fermion, struct Fermion *target_inverted, const struct Info *info,
    const struct Fermioncoor *fermioncoor, double inversion_precision, struct Fermionkit *kit, int f);

/* ---- sigma.c -------------------------------------------------------------- */
/* sigma.c:75 */
GN_API void ComputeFullSigmaMass(struct Lattice *lat, const struct Fermioncoor *fcor, double *sigmamass);

/* ---- moleculardynamics.c (sigma part) -------------------------------------- */
/* :576 */
GN_API void AddForceFromSigmaSector(const struct Lattice *lat, const struct Info *info, struct Forcesigma *force);
/* :590 */
GN_API bool AddForceFromFermionSectorRespectToSigma(const struct Lattice *lat, const struct Info *info,
                                                    const struct Fermioncoor *fcor, struct Forcesigma *force,
                                                    struct Fermionkit *kit, double inversion_precision);
/* :631 */
GN_API bool ComputeSigmaForce(const struct Lattice *lat, const struct Info *info, const struct Fermioncoor *fcor,
                              struct Forcesigma *force, struct Fermionkit *kit, double inversion_precision);
/* :299 */
GN_API double ComputeFullEnergyForSigma(const struct Lattice *lattice, const struct Info *info,
                                        const struct Fermioncoor *fcor, const struct Momentasigma *momenta,
                                        const struct Fermionkit *kit);
/* :824 */
GN_API void EvolveCoordinatesSigma(struct Lattice *lat, const struct Momentasigma *momenta,
                                   const struct Fermioncoor *fcor, double epsilon);
/* :843 */
GN_API void EvolveMomentaSigma(struct Momentasigma *momenta, const struct Forcesigma *force, double epsilon);
/* :859, :1018, :1234 */
GN_API bool LeapFrog2Sigma(struct Lattice *lattice, struct Info *info, struct Forcesigma *force,
                           struct Momentasigma *momenta, const struct Fermioncoor *fermioncoor,
                           struct Fermionkit *kit, double epsilon, const int step, const char *acceptance_file);
GN_API bool LeapFrog2MinimumNormSigma(struct Lattice *lattice, struct Info *info, struct Forcesigma *force,
                                      struct Momentasigma *momenta, const struct Fermioncoor *fermioncoor,
                                      struct Fermionkit *kit, double epsilon, const int step,
                                      const char *acceptance_file);
GN_API bool LeapFrog2MinimumNormSigmaVelocityFirst(struct Lattice *lattice, struct Info *info, struct Forcesigma *force,
                                                   struct Momentasigma *momenta, const struct Fermioncoor *fermioncoor,
                                                   struct Fermionkit *kit, double epsilon, const int step,
                                                   const char *acceptance_file);
/* :1460, :1489, :1551 -- the MD helpers of the reference's reversibility check
 * (DEBUG_LF2_SIGMA): sigma, P and the kit's phi / inverted_phi in, sigma,
 * sigmamass, P, F, inverted_phi and inverted_phi_obs out, kit counters and
 * lat->distance_sigma updated; on the GPU through gn_evolve_sigma_in_time
 * (libgn_dropin_pi.so: with the complex M, on the lattice's sigma and pi). */
GN_API void EvolveSigmaInTimeLF2(struct Lattice *lattice, struct Info *info, struct Forcesigma *force,
                                 struct Momentasigma *momenta, const struct Fermioncoor *fermioncoor,
                                 struct Fermionkit *kit, double epsilon, const int step);
GN_API void EvolveSigmaInTimeMinimumNormLF2(struct Lattice *lattice, struct Info *info, struct Forcesigma *force,
                                            struct Momentasigma *momenta, const struct Fermioncoor *fermioncoor,
                                            struct Fermionkit *kit, double epsilon, const int step);
GN_API void EvolveSigmaInTimeMinimumNormSigmaVelocityFirst(struct Lattice *lattice, struct Info *info,
                                                           struct Forcesigma *force, struct Momentasigma *momenta,
                                                           const struct Fermioncoor *fermioncoor,
                                                           struct Fermionkit *kit, double epsilon, const int step);

/* ---- condensate.c ------------------------------------------------------------ */
/* condensate.c:114 */
GN_API void ComputeCondensateDirac(const struct Lattice *lat, double *condensate_tr1, double *condensate_tr1_abs,
                                   double *condensate_tr2, double *condensate_tr4, double *condensate_mu2,
                                   double *condensate_mu4, double *condensate_chi, double *condensate_chi_abs,
                                   double *condensate_chip, double *condensate12_nosigma,
                                   double *condensate12_withsigma, struct RandomVec *vec,
                                   struct Fermion *target_inverted, const struct Info *info,
                                   const struct Fermioncoor *fermioncoor, double inversion_precision,
                                   struct Fermionkit *kit, int f);

/* ---- observables.c ----------------------------------------------------------- */
/* observables.c:323 (the Z2 model: SIGMA_INTERACTION without PI_INTERACTION);
 * the sums over lat->sigma run on the device */
GN_API void CondensateSigmaPi(const struct Lattice *lat, const struct Info *info, double *condensate_sigma,
                              double *condensate_sigma_abs, double *mu2, double *mu4, double *chi, double *chip,
                              double *chip_pbc1, double *chip_pbc2);

#undef GN_COMPLEX
#ifdef __cplusplus
}
#endif
#endif /* GN_DROPIN_H */
