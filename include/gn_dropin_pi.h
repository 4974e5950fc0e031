/*
 * gn_dropin_pi.h -- the drop-in layer for a program built with PI_INTERACTION
 * (the U(1) Gross-Neveu model): 3d-gross-neveu-model_b200/lib/libgn_dropin_pi.so.
 *
 * It exports every function of gn_dropin.h with the PI build's meaning:
 * M = D + sigmamass + i epsilon_pi pimass on complex fermion fields
 * (dirac.c:65-69), the CG, the sigma force, the sigma integrators and their
 * EvolveSigmaInTime* MD helpers, and
 * ComputeCondensateDirac (condensate.c:114, unchanged by PI_INTERACTION but
 * for its M) with that M, and CondensateSigmaPi of |(sigma, pi)|
 * (observables.c:345).  It adds the pi functions below.  The struct layouts
 * are those of gn_dropin.h (the reference's headers have no PI_INTERACTION
 * switch) plus Forcepi and Momentapi (moleculardynamics.h:64-67, :94-97).
 *
 * LeapFrog2Pi draws the pi momenta in pairs from the host program's
 * Gauss2MeanVariance (random.c:129), found by name like Gauss1 and Casuale,
 * or from the function given to GNB200_SetRandomPair.  Precision:
 * GN_PREC_FP64 (default), GN_PREC_MIXED for the solves and the integrators
 * (the standalone forces run in FP64), or GN_PREC_FP64_EXACT, the reference's
 * order of operations throughout (bit for bit its PI_INTERACTION build).
 */
#ifndef GN_DROPIN_PI_H
#define GN_DROPIN_PI_H

#include "gn_dropin.h"

#ifdef __cplusplus
extern "C" {
#endif

struct Forcepi { double *force; };
struct Momentapi { double *momenta; };

/* Gauss2MeanVariance's signature (random.c:129). */
GN_API void GNB200_SetRandomPair(void (*gauss2)(double *ris1, double *ris2, double mean, double variance));

/* ---- pi.c ---------------------------------------------------------------- */
/* pi.c:49 */
GN_API void ComputeFullPiMass(struct Lattice *lat, const struct Fermioncoor *fcor, double *pimass);

/* ---- moleculardynamics.c (pi part) ----------------------------------------- */
/* :681 */
GN_API void AddForceFromPiSector(const struct Lattice *lat, const struct Info *info, struct Forcepi *force);
/* :695 */
GN_API bool AddForceFromFermionSectorRespectToPi(const struct Lattice *lat, const struct Info *info,
                                                 const struct Fermioncoor *fcor, struct Forcepi *force,
                                                 struct Fermionkit *kit);
/* :736 */
GN_API bool ComputePiForce(const struct Lattice *lat, const struct Info *info, const struct Fermioncoor *fcor,
                           struct Forcepi *force, struct Fermionkit *kit);
/* :349 */
GN_API double ComputeFullEnergyForPi(const struct Lattice *lattice, const struct Info *info,
                                     const struct Fermioncoor *fcor, const struct Momentapi *momenta,
                                     const struct Fermionkit *kit);
/* :1711 */
GN_API void EvolveCoordinatesPi(struct Lattice *lat, const struct Momentapi *momenta, const struct Fermioncoor *fcor,
                                double epsilon);
/* :1727 */
GN_API void EvolveMomentaPi(struct Momentapi *momenta, const struct Forcepi *force, double epsilon);
/* :1743 */
GN_API bool LeapFrog2Pi(struct Lattice *lattice, struct Info *info, struct Forcepi *force, struct Momentapi *momenta,
                        const struct Fermioncoor *fermioncoor, struct Fermionkit *kit, double epsilon, const int step,
                        const char *acceptance_file);

#ifdef __cplusplus
}
#endif
#endif /* GN_DROPIN_PI_H */
