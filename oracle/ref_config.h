/*
 * ref_config.h -- TEST INFRASTRUCTURE (oracle only; never linked into the product).
 *
 * Pre-included (gcc -include) when the reference sources are compiled in place
 * by oracle/build_ref.py.  It defines the include guard MACRO_H before any
 * reference file is read, so the reference's own macro.h body is skipped and
 * the configuration below is used instead.  This is how the oracle varies the
 * lattice size without copying or patching a single reference source file.
 *
 * Every value here restates the reference configuration in macro.h:1-181
 * (same names, same values), except:
 *   - LSPACE comes from -DGN_REF_L (macro.h:21 fixes it at 8);
 *   - the sigma integrator can be switched with -DGN_REF_INTEGRATOR
 *     (0 = LFMN2SIGMAVF, the default of macro.h:71; 1 = LF2SIGMA;
 *      2 = LFMN2SIGMA), so that the alternative integrators of
 *      moleculardynamics.c:859 and :1018 can be pinned as well;
 *   - the CG tolerances can be overridden with -DGN_REF_MEDIUM_TOL /
 *     -DGN_REF_HIGH_TOL (macro.h:135-136), used only by the CPU baseline;
 *   - with -DGN_REF_RELATIVE_TOL=t both tolerances become t |phi|, evaluated
 *     at each solve by gnref_relative_tolerance() (ref_harness.c), so that the
 *     reference's absolute stopping test |r| < tol (conjugategradient.c:94)
 *     is the relative test of the benchmark workload.  The macro is read where
 *     the integrators pass it (moleculardynamics.c:1263, :1279, ...), so the
 *     reference's code is unchanged.
 */
#ifndef MACRO_H
#define MACRO_H

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <complex.h>
#include <time.h>
#include <stdbool.h>
#include <sys/types.h>
#include <sys/stat.h>
#include <unistd.h>

#ifndef GN_REF_L
#define GN_REF_L 8
#endif

/* lattice (macro.h:21-35) */
#define LSPACE (GN_REF_L)
#define LTIME (LSPACE)
#define DIM (3)
#define VOLUME (LSPACE * LSPACE * LTIME)
#define NFLAV (4)
#define Q_CHARGE (1)
#define HALFNFLAV (NFLAV / 2)
#define HALFVOLUME (VOLUME / 2)
#define LATTICE_UPDATE (1)
#define IMEAS (100)
#define MEASURE (10000)
#define COOR(x, d) ((x) * DIM + (d))

/* Hamiltonian (macro.h:47-50) */
#define PSEUDO_FERMION
#define SIGMA_INTERACTION

/* initialisation (macro.h:57-78) */
#define START_LINK_IDENTITY
#define START_WEAK_SIGMA (0.3)
#define START_PI_GAUSSIAN

/* integrator (macro.h:69-72) */
#ifndef GN_REF_INTEGRATOR
#define GN_REF_INTEGRATOR 0
#endif
#if GN_REF_INTEGRATOR == 0
#define LFMN2SIGMAVF
#elif GN_REF_INTEGRATOR == 1
#define LF2SIGMA
#elif GN_REF_INTEGRATOR == 2
#define LFMN2SIGMA
#endif

/* observables (macro.h:82-87) */
#define OBS_CONDENSATE
#define OBS_CONDENSATE_SIGMA
#define CONDENSATE_PRECISION (1)

/* boundary conditions (macro.h:100) */
#define APBC_FERMION_TIME

/* info (macro.h:114-121) */
#define HYBRID_MC
#define TERMALIZATION_STEP (10000)
#define METROPOLIS_LINK_THRESHOLD (100000)
#define METROPOLIS_LINK_ACCEPTANCE (0.3)
#define PRINT_LINK_ACCEPTANCE

/* conjugate gradient (macro.h:129-136) */
#define START_X0_NULL
#define MAX_CONJUGATE_GRADIENT_ITERATION (VOLUME + 1)
#ifdef GN_REF_RELATIVE_TOL
double gnref_relative_tolerance(void);
#define MEDIUM_PRECISION_INVERSION (gnref_relative_tolerance())
#define HIGH_PRECISION_INVERSION (gnref_relative_tolerance())
#else
#ifdef GN_REF_MEDIUM_TOL
#define MEDIUM_PRECISION_INVERSION (GN_REF_MEDIUM_TOL)
#else
#define MEDIUM_PRECISION_INVERSION (1e-3)
#endif
#ifdef GN_REF_HIGH_TOL
#define HIGH_PRECISION_INVERSION (GN_REF_HIGH_TOL)
#else
#define HIGH_PRECISION_INVERSION (1e-9)
#endif
#endif

/* condensate noise (macro.h:146) */
#define Z2_NOISE

/* constants (macro.h:163-178) */
#define PI (3.141592653589793238462643383279502884197169399375105820974944)
#define MAGIC_LAMBDA (0.1931833275037836)
#define LF4MN4_RHO (0.1786178958448091)
#define LF4MN4_THETA (-0.06626458266981843)
#define LF4MN4_LAMBDA (0.7123418310626056)
#define I_UNIT (I)
#define P_MIN ((2 * PI) / LSPACE)
#define P_MIN_APBC ((PI) / LSPACE)

#endif /* MACRO_H */
