/*
 * gn_oracle.c -- TEST INFRASTRUCTURE: CPU restatement of the reference's fermion
 * hot path.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it, and only as the checker.  It is never the product path.
 *
 * Pinned: it reproduces the reference's results bit for bit (tests/test_oracle.py
 * compares it with the reference compiled from its own sources, oracle/_ref/,
 * and with the committed golden fixtures in tests/golden/).  To make that
 * possible it follows the reference's order of floating-point operations
 * exactly, including the scatter form of the transposed operator and the
 * serial order of every sum; it does NOT try to be fast.
 *
 * Differences from the reference, none of which change a result:
 *   - L is a run-time argument (the reference fixes LSPACE at compile time);
 *   - fields are real arrays in the reference's fermion order; a complex field
 *     (only the condensate's phase vector is one) is two real planes, re then im;
 *   - random numbers come from caller-supplied functions (the reference calls
 *     Gauss1 / Casuale of random.c:88 / :28 directly).
 *
 * Layout (coordinate.c:25-40, :301-313): lexicographic n = (x0*L + x1)*L + x2,
 * x2 = time fastest; fermion index = n/2 + ((x0+x1+x2) % 2) * V/2.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GN_PI 3.141592653589793238462643383279502884197169399375105820974944 /* macro.h:163 */
#define GN_LAMBDA 0.1931833275037836                                         /* macro.h:169 */
#define GN_NFLAV 4                                                           /* macro.h:25 */

typedef double (*gno_draw_fn)(void);

/* ------------------------------------------------------------------ geometry */
typedef struct {
    int L;
    long V;
    int *pp; /* fermion index of x + mu, [x*3+mu] (fcor->fermionpp) */
    int *mm; /* fermion index of x - mu (fcor->fermionmm) */
    signed char *eta_pp, *eta_mm; /* +-1 (coordinate.c:133-200) */
    int *x2; /* time coordinate of fermion site x */
} geom_t;

static int lex_to_fermion(int L, int c0, int c1, int c2)
{
    long V = (long)L * L * L;
    long lex = ((long)c0 * L + c1) * L + c2;
    return (int)(lex / 2 + ((c0 + c1 + c2) % 2) * (V / 2));
}

static geom_t *geom_cache = NULL;

static const geom_t *geom(int L)
{
    if (geom_cache && geom_cache->L == L) return geom_cache;
    if (geom_cache) {
        free(geom_cache->pp); free(geom_cache->mm); free(geom_cache->eta_pp); free(geom_cache->eta_mm);
        free(geom_cache->x2); free(geom_cache);
    }
    geom_t *g = calloc(1, sizeof(geom_t));
    long V = (long)L * L * L;
    g->L = L; g->V = V;
    g->pp = malloc(sizeof(int) * 3 * V);
    g->mm = malloc(sizeof(int) * 3 * V);
    g->eta_pp = malloc(3 * V);
    g->eta_mm = malloc(3 * V);
    g->x2 = malloc(sizeof(int) * V);
    for (int c0 = 0; c0 < L; c0++)
        for (int c1 = 0; c1 < L; c1++)
            for (int c2 = 0; c2 < L; c2++) {
                int c[3] = {c0, c1, c2};
                int x = lex_to_fermion(L, c0, c1, c2);
                g->x2[x] = c2;
                for (int d = 0; d < 3; d++) {
                    int up[3] = {c0, c1, c2}, dn[3] = {c0, c1, c2};
                    up[d] = (c[d] + 1) % L;
                    dn[d] = (c[d] + L - 1) % L;
                    g->pp[x * 3 + d] = lex_to_fermion(L, up[0], up[1], up[2]);
                    g->mm[x * 3 + d] = lex_to_fermion(L, dn[0], dn[1], dn[2]);
                    int s = 0;
                    for (int t = 0; t < d; t++) s += c[t];
                    int eta = (s % 2) ? -1 : 1;
                    g->eta_pp[x * 3 + d] = (signed char)((d == 2 && c2 == L - 1) ? -eta : eta);
                    g->eta_mm[x * 3 + d] = (signed char)((d == 2 && c2 == 0) ? -eta : eta);
                }
            }
    geom_cache = g;
    return g;
}

/* Tables for tests of the device index math. */
int gno_tables(int L, int *pp, int *mm, signed char *eta_pp, signed char *eta_mm)
{
    const geom_t *g = geom(L);
    memcpy(pp, g->pp, sizeof(int) * 3 * g->V);
    memcpy(mm, g->mm, sizeof(int) * 3 * g->V);
    memcpy(eta_pp, g->eta_pp, 3 * g->V);
    memcpy(eta_mm, g->eta_mm, 3 * g->V);
    return 0;
}

/* ------------------------------------------------------------------ sigma mass */
/* ComputeFullSigmaMass, sigma.c:75-94 */
void gno_sigma_mass(int L, const double *sigma, double *sm)
{
    const geom_t *g = geom(L);
    const int *mm = g->mm;
    for (long x = 0; x < g->V; x++) {
        double s = sigma[x];
        s += sigma[mm[x * 3 + 0]];
        s += sigma[mm[x * 3 + 1]];
        s += sigma[mm[x * 3 + 2]];
        s += sigma[mm[mm[x * 3 + 0] * 3 + 1]];
        s += sigma[mm[mm[x * 3 + 0] * 3 + 2]];
        s += sigma[mm[mm[x * 3 + 1] * 3 + 2]];
        s += sigma[mm[mm[mm[x * 3 + 0] * 3 + 1] * 3 + 2]];
        sm[x] = s / 8.0;
    }
}

/* ------------------------------------------------------------------ Dirac */
/* which: 0 = M (DiracFermion, dirac.c:46-82, gather);
 *        1 = M^T (AdjDiracFermion, dirac.c:88-123, scatter in the reference's order);
 *        2 = out -= M in (SubtractDiracFermion, dirac.c:213-247).
 * ncomp real planes of length V (2 = complex). */
void gno_dirac(int L, const double *sm, const double *in, double *out, int ncomp, int which)
{
    const geom_t *g = geom(L);
    long V = g->V;
    for (int c = 0; c < ncomp; c++) {
        const double *psi = in + c * V;
        double *t = out + c * V;
        if (which == 0) {
            for (long x = 0; x < V; x++) t[x] = sm[x] * psi[x];
            for (long x = 0; x < V; x++)
                for (int d = 0; d < 3; d++) {
                    t[x] += (0.5 * g->eta_pp[x * 3 + d]) * psi[g->pp[x * 3 + d]];
                    t[x] -= (0.5 * g->eta_mm[x * 3 + d]) * psi[g->mm[x * 3 + d]];
                }
        } else if (which == 1) {
            for (long x = 0; x < V; x++) t[x] = sm[x] * psi[x];
            for (long x = 0; x < V; x++)
                for (int d = 0; d < 3; d++) {
                    t[g->pp[x * 3 + d]] += (0.5 * g->eta_pp[x * 3 + d]) * psi[x];
                    t[g->mm[x * 3 + d]] -= (0.5 * g->eta_mm[x * 3 + d]) * psi[x];
                }
        } else {
            for (long x = 0; x < V; x++) t[x] -= sm[x] * psi[x];
            for (long x = 0; x < V; x++)
                for (int d = 0; d < 3; d++) {
                    t[x] -= (0.5 * g->eta_pp[x * 3 + d]) * psi[g->pp[x * 3 + d]];
                    t[x] += (0.5 * g->eta_mm[x * 3 + d]) * psi[g->mm[x * 3 + d]];
                }
        }
    }
}

/* ------------------------------------------------------------------ BLAS-1 */
/* |z|^2 as the reference's CG computes it: pow(cabs(z), 2.0) (conjugategradient.c:65). */
static double abs2_cabs(const double *v, long V, int ncomp, long x)
{
    double a = (ncomp == 2) ? hypot(v[x], v[V + x]) : fabs(v[x]);
    return a * a;
}
/* NormFermion, fermion.h:67: sqrt via pow(sum creal(conj(z) z), 0.5) */
static double norm_fermion(const double *v, long V, int ncomp)
{
    double total = 0.0;
    for (long x = 0; x < V; x++) {
        double re = v[x], im = (ncomp == 2) ? v[V + x] : 0.0;
        total += re * re - (-im) * im;
    }
    return pow(total, 0.5);
}

/* ------------------------------------------------------------------ CG */
/* variant 0: ConjugateGradientFastDiracAdjFastDiracToTheMinusOne (conjugategradient.c:13-107,
 *            START_X0_NULL: early exit when the incoming x already satisfies tol);
 * variant 1: StartX0ImposedConjugateGradient... (conjugategradient.c:115-182).
 * Solves (M M^T) x = b, absolute stop ||r|| < tol, at most max_iter iterations.
 * A negative tol asks for the relative stop ||r|| < |tol| ||b|| instead (the
 * benchmark's rule; the reference's own callers always pass tol > 0).
 * Returns 1 on convergence.  *iters = iteration+1 and *counted = 1 when the
 * reference would add to kit->iterations / kit->CG_call; 0 on an early exit. */
int gno_cg(int L, const double *sm, const double *b, double *x, int ncomp, double tol, int variant, long max_iter,
           long *iters, int *counted)
{
    const geom_t *g = geom(L);
    long V = g->V, n = V * ncomp;
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
    double *t1 = malloc(sizeof(double) * n), *t2 = malloc(sizeof(double) * n);
    int ok = 0;
    *iters = 0;
    *counted = 0;
    if (tol < 0.0) tol = -tol * norm_fermion(b, V, ncomp);
    if (variant == 0) {
        memcpy(r, b, sizeof(double) * n);
        gno_dirac(L, sm, x, t1, ncomp, 1);
        gno_dirac(L, sm, t1, r, ncomp, 2);
        if (norm_fermion(r, V, ncomp) < tol) { ok = 1; goto done; }
        memset(x, 0, sizeof(double) * n);
        memcpy(r, b, sizeof(double) * n);
        memcpy(p, b, sizeof(double) * n);
    } else {
        memset(x, 0, sizeof(double) * n);
        memcpy(r, b, sizeof(double) * n);
        if (norm_fermion(r, V, ncomp) < tol) { ok = 1; goto done; }
        memcpy(p, b, sizeof(double) * n);
    }
    for (long it = 0; it < max_iter; it++) {
        double rr = 0.0, pAp = 0.0;
        for (long s = 0; s < V; s++) rr += abs2_cabs(r, V, ncomp, s);
        gno_dirac(L, sm, p, t1, ncomp, 1);
        for (long s = 0; s < V; s++) pAp += abs2_cabs(t1, V, ncomp, s);
        double alpha = rr / pAp;
        for (long i = 0; i < n; i++) x[i] += alpha * p[i];
        gno_dirac(L, sm, t1, t2, ncomp, 0);
        for (long i = 0; i < n; i++) r[i] += (-alpha) * t2[i];
        if (norm_fermion(r, V, ncomp) < tol) {
            *iters = it + 1;
            *counted = 1;
            ok = 1;
            goto done;
        }
        double rr1 = 0.0;
        for (long s = 0; s < V; s++) rr1 += abs2_cabs(r, V, ncomp, s);
        double beta = rr1 / rr;
        for (long i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
    }
done:
    free(r); free(p); free(t1); free(t2);
    return ok;
}

/* ------------------------------------------------------------------ sigma MD */
typedef struct {
    int L;
    long V;
    double beta_s;
    double *sigma, *sm, *P, *F;
    double *chi, *phi, *X, *Y; /* 2 flavours x V each (kit->chi, phi, inverted_phi, inverted_phi_obs) */
    double iterations;         /* kit->iterations */
    long calls;                /* kit->CG_call */
    double distance;           /* lat->distance_sigma */
} md_t;

static void cg_count(md_t *m, long it, int counted)
{
    if (counted) { m->iterations += it; m->calls++; }
}

/* AddForceFromFermionSectorRespectToSigma (moleculardynamics.c:590-622) +
 * AddForceFromSigmaSector (:576-581) inside ComputeSigmaForce (:631-647). */
static int md_force(md_t *m, double tol)
{
    const geom_t *g = geom(m->L);
    long V = m->V;
    const int *pp = g->pp;
    for (long x = 0; x < V; x++) m->F[x] = 0.0;
    for (int f = 0; f < 2; f++) {
        long it; int cnt;
        int ok = gno_cg(m->L, m->sm, m->phi + f * V, m->X + f * V, 1, tol, 0, V + 1, &it, &cnt);
        cg_count(m, it, cnt);
        if (!ok) return 0;
    }
    for (int f = 0; f < 2; f++) gno_dirac(m->L, m->sm, m->X + f * V, m->Y + f * V, 1, 1);
    for (int f = 0; f < 2; f++) {
        const double *X = m->X + f * V, *Y = m->Y + f * V;
        for (long x = 0; x < V; x++) {
            long c[8];
            c[0] = x;
            c[1] = pp[pp[x * 3 + 0] * 3 + 1];
            c[2] = pp[pp[x * 3 + 0] * 3 + 2];
            c[3] = pp[pp[x * 3 + 1] * 3 + 2];
            c[4] = pp[x * 3 + 0];
            c[5] = pp[x * 3 + 1];
            c[6] = pp[x * 3 + 2];
            c[7] = pp[pp[pp[x * 3 + 0] * 3 + 1] * 3 + 2];
            for (int k = 0; k < 8; k++) m->F[x] += 0.125 * (X[c[k]] * Y[c[k]]);
        }
    }
    double coef = (GN_NFLAV * m->beta_s / 2.0);
    for (long x = 0; x < V; x++) m->F[x] -= coef * m->sigma[x];
    return 1;
}

/* ComputeFullEnergyForSigma, moleculardynamics.c:299-319 */
static double md_energy(const md_t *m)
{
    long V = m->V;
    double total = 0.0;
    for (long r = 0; r < V; r++) total += (m->P[r] * m->P[r] / 2.0);
    for (int f = 0; f < 2; f++)
        for (long x = 0; x < V; x++) total += (0.5 * (m->phi[f * V + x] * m->X[f * V + x]));
    double s2 = 0.0;
    for (long x = 0; x < V; x++) s2 += m->sigma[x] * m->sigma[x];
    total += ((GN_NFLAV * m->beta_s / 4.0) * s2);
    return total;
}

/* EvolveCoordinatesSigma (:824-836) */
static void md_q(md_t *m, double eps)
{
    for (long x = 0; x < m->V; x++) m->sigma[x] += (eps * m->P[x]);
    gno_sigma_mass(m->L, m->sigma, m->sm);
    m->distance += eps;
}
/* EvolveMomentaSigma (:843-848) */
static void md_p(md_t *m, double eps)
{
    for (long x = 0; x < m->V; x++) m->P[x] += (m->F[x] * eps);
}

/* The integrator schedules, as op lists shared by every implementation:
 *   'F' force (tol M or H), 'P' momentum step, 'Q' sigma step, 'S' X0-imposed
 *   solve of both flavours at H (LeapFrog2MinimumNormSigma's final solve). */
enum { OP_F_MED = 1, OP_F_HIGH, OP_P, OP_Q, OP_S_HIGH };
typedef struct { int op; double c; } md_op_t;

/* Build the op list of an integrator; returns the count (<= cap). */
int gno_schedule(int integrator, double eps, int step, int *ops, double *coefs, int cap)
{
    int n = 0;
#define PUSH(o, cc) do { if (n < cap) { ops[n] = (o); coefs[n] = (cc); } n++; } while (0)
    const double lam = GN_LAMBDA;
    if (integrator == 0) { /* LeapFrog2MinimumNormSigmaVelocityFirst, :1234-1434 */
        PUSH(OP_F_MED, 0); PUSH(OP_P, lam * eps); PUSH(OP_Q, eps / 2.0);
        PUSH(OP_F_MED, 0); PUSH(OP_P, (1.0 - (2.0 * lam)) * eps); PUSH(OP_Q, eps / 2.0);
        for (int s = 1; s < step - 1; s++) {
            PUSH(OP_F_MED, 0); PUSH(OP_P, 2.0 * lam * eps); PUSH(OP_Q, eps / 2.0);
            PUSH(OP_F_MED, 0); PUSH(OP_P, (1.0 - (2.0 * lam)) * eps); PUSH(OP_Q, eps / 2.0);
        }
        PUSH(OP_F_MED, 0); PUSH(OP_P, 2.0 * lam * eps); PUSH(OP_Q, eps / 2.0);
        PUSH(OP_F_MED, 0); PUSH(OP_P, (1.0 - (2.0 * lam)) * eps); PUSH(OP_Q, eps / 2.0);
        PUSH(OP_F_HIGH, 0); PUSH(OP_P, lam * eps);
    } else if (integrator == 1) { /* LeapFrog2Sigma, :859-1005 */
        PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        for (int s = 0; s < step - 1; s++) { PUSH(OP_Q, eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps); }
        PUSH(OP_Q, eps); PUSH(OP_F_HIGH, 0); PUSH(OP_P, eps / 2.0);
    } else { /* LeapFrog2MinimumNormSigma, :1018-1221 */
        PUSH(OP_Q, lam * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        PUSH(OP_Q, (1.0 - (2.0 * lam)) * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        for (int s = 1; s < step - 1; s++) {
            PUSH(OP_Q, 2.0 * lam * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
            PUSH(OP_Q, (1.0 - (2.0 * lam)) * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        }
        PUSH(OP_Q, 2.0 * lam * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        PUSH(OP_Q, (1 - (2.0 * lam)) * eps); PUSH(OP_F_MED, 0); PUSH(OP_P, eps / 2.0);
        PUSH(OP_Q, lam * eps); PUSH(OP_S_HIGH, 0);
    }
#undef PUSH
    return n;
}

/* One sigma-HMC trajectory (the body shared by the three integrators,
 * moleculardynamics.c:1234-1434 for the default one).  Draws P, chi_0, chi_1
 * with gauss() and the Metropolis uniform with uniform(), in the reference's
 * order.  State arrays are in/out: sigma, sm (V), P, F (V), chi, phi, X, Y (2V).
 * out[0] = dH, out[1] = accepted (0/1), out[2] = H0, out[3] = H1.
 * Returns 1, or 0 when a CG failed (sigma and sm restored, no uniform drawn). */
int gno_trajectory(int L, double beta_s, double eps, int step, int integrator, double tol_med, double tol_high,
                   double *sigma, double *sm, double *P, double *F, double *chi, double *phi, double *X, double *Y,
                   gno_draw_fn gauss, gno_draw_fn uniform, double *out, double *iterations, long *calls,
                   double *distance)
{
    md_t m = {L, (long)L * L * L, beta_s, sigma, sm, P, F, chi, phi, X, Y, *iterations, *calls, *distance};
    long V = m.V;
    int ops[512];
    double coefs[512];
    int nops = gno_schedule(integrator, eps, step, ops, coefs, 512);
    if (nops > 512) return -1;
    for (long x = 0; x < V; x++) P[x] = gauss();
    for (int f = 0; f < 2; f++) {
        for (long x = 0; x < V; x++) chi[f * V + x] = gauss();
        gno_dirac(L, sm, chi + f * V, phi + f * V, 1, 0);
    }
    double *copy = malloc(sizeof(double) * V);
    memcpy(copy, sigma, sizeof(double) * V);
    int ok = 1;
    for (int f = 0; f < 2 && ok; f++) {
        long it; int cnt;
        ok = gno_cg(L, sm, phi + f * V, X + f * V, 1, tol_high, 1, V + 1, &it, &cnt);
        cg_count(&m, it, cnt);
    }
    double h0 = ok ? md_energy(&m) : 0.0;
    for (int k = 0; k < nops && ok; k++) {
        switch (ops[k]) {
        case OP_F_MED: ok = md_force(&m, tol_med); break;
        case OP_F_HIGH: ok = md_force(&m, tol_high); break;
        case OP_P: md_p(&m, coefs[k]); break;
        case OP_Q: md_q(&m, coefs[k]); break;
        case OP_S_HIGH:
            for (int f = 0; f < 2 && ok; f++) {
                long it; int cnt;
                ok = gno_cg(L, sm, phi + f * V, X + f * V, 1, tol_high, 1, V + 1, &it, &cnt);
                cg_count(&m, it, cnt);
            }
            break;
        }
    }
    if (!ok) {
        memcpy(sigma, copy, sizeof(double) * V);
        gno_sigma_mass(L, sigma, sm);
    } else {
        double h1 = md_energy(&m);
        double dh = h1 - h0;
        int acc = uniform() <= exp(-(h1 - h0));
        if (!acc) {
            memcpy(sigma, copy, sizeof(double) * V);
            gno_sigma_mass(L, sigma, sm);
        }
        out[0] = dh; out[1] = acc; out[2] = h0; out[3] = h1;
    }
    free(copy);
    *iterations = m.iterations;
    *calls = m.calls;
    *distance = m.distance;
    return ok;
}

/* Force and energy alone, for unit parity (ComputeSigmaForce, ComputeFullEnergyForSigma). */
int gno_force(int L, double beta_s, const double *sigma, const double *sm, const double *phi, double *X, double *Y,
              double tol, double *F, double *iterations, long *calls)
{
    md_t m = {L, (long)L * L * L, beta_s, (double *)sigma, (double *)sm, NULL, F, NULL, (double *)phi, X, Y,
              *iterations, *calls, 0.0};
    int ok = md_force(&m, tol);
    *iterations = m.iterations;
    *calls = m.calls;
    return ok;
}
double gno_energy(int L, double beta_s, const double *sigma, const double *P, const double *phi, const double *X)
{
    md_t m = {L, (long)L * L * L, beta_s, (double *)sigma, NULL, (double *)P, NULL, NULL, (double *)phi,
              (double *)X, NULL, 0.0, 0, 0.0};
    return md_energy(&m);
}
void gno_evolve_sigma(int L, double *sigma, double *sm, const double *P, double eps)
{
    md_t m = {L, (long)L * L * L, 0.0, sigma, sm, (double *)P};
    md_q(&m, eps);
}
void gno_evolve_momenta(int L, double *P, const double *F, double eps)
{
    md_t m = {L, (long)L * L * L, 0.0, NULL, NULL, P, (double *)F};
    md_p(&m, eps);
}

/* ------------------------------------------------------------------ condensate */
/* ComputeCondensateDirac, condensate.c:114-244, with CONDENSATE_PRECISION = 1.
 * target (2V, complex planes) is target_inverted (in/out, used by the early-exit
 * test of every solve); D (2V) is kit->Ddag_inverted_phi_obs (out).
 * out[11] = tr1, |tr1|, tr2, tr4, mu2, mu4, chi, |chi|, chip, c12_nosigma, c12_withsigma. */
int gno_condensate(int L, const double *sm, double tol, double *target, double *D, gno_draw_fn uniform, double *out,
                   double *iterations, long *calls)
{
    const geom_t *g = geom(L);
    long V = g->V;
    int Vi = (int)V;
    double *vec = calloc(2 * V, sizeof(double));
    double *z2 = malloc(sizeof(double) * V);
    int ok_all = 1;
    for (int k = 0; k < 11; k++) out[k] = 0.0;
#define SOLVE(bvec)                                                                             \
    do {                                                                                        \
        long it_; int cnt_;                                                                     \
        ok_all &= gno_cg(L, sm, (bvec), target, 2, tol, 0, V + 1, &it_, &cnt_);                 \
        if (cnt_) { *iterations += it_; (*calls)++; }                                           \
    } while (0)
#define Z2FILL()                                                                                \
    do {                                                                                        \
        for (long x = 0; x < V; x++) { vec[x] = (uniform() <= 0.5) ? 1.0 : -1.0; vec[V + x] = 0.0; } \
    } while (0)
    double temp[4] = {0, 0, 0, 0};
    for (int p = 0; p < 4; p++) {
        Z2FILL();
        SOLVE(vec);
        gno_dirac(L, sm, target, D, 2, 1);
        for (long x = 0; x < V; x++) {
            double re = vec[x] * D[x] - (-vec[V + x]) * D[V + x];
            temp[p] += re / Vi;
        }
    }
    /* Mean over CONDENSATE_PRECISION = 1 element (inputoutput.c:307): 0.0 + a / 1 */
    double tr0 = 0.0 + temp[0] / 1, tr1 = 0.0 + temp[1] / 1, tr2 = 0.0 + temp[2] / 1, tr3 = 0.0 + temp[3] / 1;
    out[0] = (tr0 + tr1 + tr2 + tr3) / 4.0;
    out[1] = fabs(out[0]);
    out[2] = ((tr0 * tr1) + (tr0 * tr2) + (tr0 * tr3) + (tr1 * tr2) + (tr1 * tr3) + (tr2 * tr3)) / 6.0;
    out[3] = (tr0 * tr1 * tr2 * tr3);
    /* mu2 / chi with the 1/V vector (:167-181) */
    for (long x = 0; x < V; x++) { vec[x] = 1.0 / Vi; vec[V + x] = 0.0; }
    SOLVE(vec);
    gno_dirac(L, sm, target, D, 2, 1);
    for (long x = 0; x < V; x++) out[4] += vec[x] * D[x] - (-vec[V + x]) * D[V + x];
    out[5] = out[4] * out[4];
    out[6] = Vi * out[4];
    out[7] = fabs(out[6]);
    /* chi_p with the phase vector e^{i pi/L x_2} / V (:84-89, :185-197) */
    for (long x = 0; x < V; x++) {
        double complex z = cexp(I * ((GN_PI) / L) * g->x2[x]) / Vi;
        vec[x] = creal(z);
        vec[V + x] = cimag(z);
    }
    SOLVE(vec);
    gno_dirac(L, sm, target, D, 2, 1);
    double tchip = 0.0;
    for (long x = 0; x < V; x++) tchip += vec[x] * D[V + x] + (-vec[V + x]) * D[x];
    out[8] = tchip * Vi;
    /* <chibar1 chi2> without sigma (:201-212) */
    Z2FILL();
    for (long x = 0; x < V; x++) z2[x] = vec[x];
    SOLVE(vec);
    gno_dirac(L, sm, target, D, 2, 1);
    SOLVE(D);
    gno_dirac(L, sm, target, D, 2, 1);
    for (long x = 0; x < V; x++) out[9] += D[x] * z2[x] / Vi;
    /* with sigma-mass insertions (:216-230) */
    Z2FILL();
    for (long x = 0; x < V; x++) z2[x] = vec[x];
    for (long x = 0; x < V; x++) { vec[x] = vec[x] * sm[x]; vec[V + x] = vec[V + x] * sm[x]; }
    SOLVE(vec);
    gno_dirac(L, sm, target, D, 2, 1);
    for (long y = 0; y < V; y++) { D[y] = D[y] * sm[y]; D[V + y] = D[V + y] * sm[y]; }
    SOLVE(D);
    gno_dirac(L, sm, target, D, 2, 1);
    for (long x = 0; x < V; x++) out[10] += D[x] * z2[x] / Vi;
#undef SOLVE
#undef Z2FILL
    free(vec);
    free(z2);
    return ok_all;
}

/* ------------------------------------------------------------------ replay RNG */
/* A recorded stream of Gauss1 / Casuale outputs, replayed in order.  Lets the
 * tests drive every implementation with the reference's exact random numbers
 * without the reference's RNG code present. */
static const double *rp_g = NULL, *rp_u = NULL;
static long rp_ng = 0, rp_nu = 0, rp_ig = 0, rp_iu = 0;
void gno_replay_set(const double *g, long ng, const double *u, long nu)
{
    rp_g = g; rp_ng = ng; rp_u = u; rp_nu = nu; rp_ig = rp_iu = 0;
}
double gno_replay_gauss(void) { return (rp_ig < rp_ng) ? rp_g[rp_ig++] : NAN; }
double gno_replay_uniform(void) { return (rp_iu < rp_nu) ? rp_u[rp_iu++] : NAN; }
void gno_replay_pos(long *ig, long *iu) { *ig = rp_ig; *iu = rp_iu; }
