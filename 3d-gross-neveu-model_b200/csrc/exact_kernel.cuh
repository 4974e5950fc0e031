// exact_kernel.cuh -- the FP64 path in the reference's exact order of
// operations, for bit-for-bit parity runs (precision GN_PREC_FP64_EXACT).
//
// Two things make the fast path differ from the reference in the last bits:
// its global sums are trees instead of the reference's serial loops, and its
// M^T gathers the six hopping terms in another order than the reference's
// scatter (dirac.c:88-123).  Here every sum is a serial loop over the sites in
// fermion order, as in conjugategradient.c:64-98, moleculardynamics.c:299-319
// and condensate.c:142-227, and M^T adds the terms of a site in the order the
// reference's scatter delivers them: by increasing index of the source site.
// One block does a whole solve (block barriers between phases; thread 0 runs
// the serial sums), so the mode is meant for the lattice sizes of parity tests.
// Built with --fmad=false.
#pragma once
#include "device_common.cuh"
#include "host_hypot.h"

namespace gn {

constexpr int kExactThreads = 1024;

// M^T psi at site i in the reference's scatter order.  Source x = i - mu
// delivers +1/2 eta_pp(x, mu) psi(x) = +1/2 eta_mm(i, mu) psi(i - mu); source
// x = i + mu delivers -1/2 eta_mm(x, mu) psi(x) = -1/2 eta_pp(i, mu) psi(i + mu)
// (the antiperiodic signs move with the phases).  For L >= 4 the six sources
// are distinct; they are taken by increasing fermion index.
__device__ __forceinline__ double apply_Mt_ref_order(const Site &s, double sm, const double *psi, uint32_t i) {
  uint32_t idx[6];
  int kind[6];  // 0..2: backward source mu (added), 3..5: forward source mu (subtracted)
#pragma unroll
  for (int d = 0; d < 3; d++) {
    idx[d] = s.nb_dn[d];
    kind[d] = d;
    idx[3 + d] = s.nb_up[d];
    kind[3 + d] = 3 + d;
  }
  // insertion sort of six keys
  for (int a = 1; a < 6; a++) {
    const uint32_t ki = idx[a];
    const int kk = kind[a];
    int b = a - 1;
    while (b >= 0 && idx[b] > ki) {
      idx[b + 1] = idx[b];
      kind[b + 1] = kind[b];
      b--;
    }
    idx[b + 1] = ki;
    kind[b + 1] = kk;
  }
  double t = sm * psi[i];
  for (int a = 0; a < 6; a++) {
    const int kd = kind[a];
    const double v = psi[idx[a]];
    if (kd < 3) t = hop_add(t, v, s.neg, 3 + kd);  // +1/2 eta_mm(i, mu) psi(i - mu)
    else t = hop_sub(t, v, s.neg, kd - 3);         // -1/2 eta_pp(i, mu) psi(i + mu)
  }
  return t;
}

// |z|^2 as pow(cabs(z), 2.0) (conjugategradient.c:65; the host library's
// pow(a, 2.0) is a * a) and creal(conj(z) z) (fermion.h:67) for one or two planes.
__device__ __forceinline__ double abs2_cabs(const double *v, uint32_t V, int nc, uint32_t x) {
  const double a = nc == 2 ? gn_host_hypot(v[x], v[V + x]) : fabs(v[x]);
  return a * a;
}
__device__ __forceinline__ double abs2_conj(const double *v, uint32_t V, int nc, uint32_t x) {
  const double re = v[x], im = nc == 2 ? v[V + x] : 0.0;
  return re * re - (-im) * im;
}

struct ExactArgs {
  Geom g;
  const double *sm;
  const double *b;
  double *x, *r, *p, *t, *ap;
  int nc;
  int variant;
  int rel;
  double tol;
  long long max_iter;
  CgState *state;
};

// M^T on all sites of the block's grid-stride share, reference order.
__device__ __forceinline__ void exact_mt(const Geom &g, const double *sm, const double *in, double *out, int nc) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = threadIdx.x; i < V; i += blockDim.x) {
    const Site s = make_site(g, i);
    for (int c = 0; c < nc; c++) out[size_t(c) * V + i] = apply_Mt_ref_order(s, sm[i], in + size_t(c) * V, i);
  }
}

// One CG solve (conjugategradient.c:13-107 / :115-182) in a single block.
__global__ void __launch_bounds__(kExactThreads) cg_exact_kernel(ExactArgs a) {
  __shared__ double s_val;
  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const int nc = a.nc;
  const size_t n = size_t(nc) * V;
  auto serial = [&](int which, const double *v) {  // thread 0: the reference's serial loop
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (uint32_t x = 0; x < V; x++) s += which == 0 ? abs2_cabs(v, V, nc, x) : abs2_conj(v, V, nc, x);
      s_val = s;
    }
    __syncthreads();
    return s_val;
  };
  CgState st;
  st.status = kCgRunning;
  st.reliable = 0;
  st.iters = 0;
  st.r2 = 0.0;
  st.b2 = 0.0;
  double tau = a.tol;
  if (a.variant == 0) {
    // r = b - M (M^T x)
    exact_mt(g, a.sm, a.x, a.t, nc);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < V; i += blockDim.x) {
      const Site s = make_site(g, i);
      for (int c = 0; c < nc; c++) {
        const double *tv = a.t + size_t(c) * V;
        const Nb<double> nb = gather7<double>(s, i, [&](uint32_t j) { return tv[j]; });
        a.r[size_t(c) * V + i] = apply_sub_M<double>(s, a.b[size_t(c) * V + i], a.sm[i], nb);
      }
    }
    __syncthreads();
    const double rn2 = serial(1, a.r);
    if (a.rel) tau = a.tol * sqrt(serial(1, a.b));
    st.r2 = rn2;
    if (sqrt(rn2) < tau) {
      st.status = kCgConvergedStart;
    }
  }
  if (st.status == kCgRunning) {
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) {
      a.x[j] = 0.0;
      a.r[j] = a.b[j];
    }
    __syncthreads();
    if (a.variant == 1) {
      const double rn2 = serial(1, a.r);
      if (a.rel) tau = a.tol * sqrt(rn2);
      st.r2 = rn2;
      if (sqrt(rn2) < tau) st.status = kCgConvergedStart;
    }
    if (st.status == kCgRunning) {
      for (size_t j = threadIdx.x; j < n; j += blockDim.x) a.p[j] = a.b[j];
      __syncthreads();
    }
  }
  long long it = 0;
  for (; st.status == kCgRunning && it < a.max_iter; it++) {
    const double rr = serial(0, a.r);
    exact_mt(g, a.sm, a.p, a.t, nc);
    __syncthreads();
    const double pap = serial(0, a.t);
    const double alpha = rr / pap;
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) a.x[j] = a.x[j] + alpha * a.p[j];
    for (uint32_t i = threadIdx.x; i < V; i += blockDim.x) {
      const Site s = make_site(g, i);
      for (int c = 0; c < nc; c++) {
        const double *tv = a.t + size_t(c) * V;
        const Nb<double> nb = gather7<double>(s, i, [&](uint32_t j) { return tv[j]; });
        a.ap[size_t(c) * V + i] = apply_M<double>(s, a.sm[i], nb);
      }
    }
    __syncthreads();
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) a.r[j] = a.r[j] + (-alpha) * a.ap[j];
    __syncthreads();
    const double rn2 = serial(1, a.r);
    st.r2 = rn2;
    if (sqrt(rn2) < tau) {
      st.status = kCgConverged;
      st.iters = it + 1;
      break;
    }
    const double rr1 = serial(0, a.r);
    const double beta = rr1 / rr;
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) a.p[j] = a.r[j] + beta * a.p[j];
    __syncthreads();
  }
  if (st.status == kCgRunning) {
    st.status = kCgMaxIter;
    st.iters = it;
  }
  if (threadIdx.x == 0) *a.state = st;
}

// M^T on one or more planes in the reference's order (for Y = M^T X and the condensate).
__global__ void __launch_bounds__(256) mt_exact_kernel(Geom g, const double *__restrict__ sm,
                                                      const double *__restrict__ in, double *__restrict__ out) {
  const uint32_t V = uint32_t(g.V);
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const Site s = make_site(g, i);
  out[size_t(blockIdx.y) * V + i] = apply_Mt_ref_order(s, sm[i], in + size_t(blockIdx.y) * V, i);
}

// Serial sums of the energy (moleculardynamics.c:299-319): out[0] = the total
// P^2/2 and 1/2 phi X terms in the reference's order, out[1] = sum sigma^2.
__global__ void energy_exact_kernel(uint32_t V, const double *P, const double *phi, const double *X,
                                    const double *sigma, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double total = 0.0;
  for (uint32_t r = 0; r < V; r++) total += (P[r] * P[r] / 2.0);
  for (int f = 0; f < 2; f++)
    for (uint32_t x = 0; x < V; x++) total += (0.5 * (phi[size_t(f) * V + x] * X[size_t(f) * V + x]));
  double s2 = 0.0;
  for (uint32_t x = 0; x < V; x++) s2 += sigma[x] * sigma[x];
  out[0] = total;
  out[1] = s2;
}

// Serial condensate dot products (condensate.c:142-227) of v with D (both two
// planes): out[0] = sum Re(conj v D)/V, out[1] = sum Re(conj v D),
// out[2] = sum Im(conj v D), out[3] = sum D_re z / V with z = the real plane of v.
__global__ void cond_dot_exact_kernel(uint32_t V, const double *v, const double *D, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int Vi = int(V);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (uint32_t x = 0; x < V; x++) {
    const double vr = v[x], vi = v[V + x], dr = D[x], di = D[V + x];
    const double re = vr * dr - (-vi) * di;
    s0 += re / Vi;
    s1 += re;
    s2 += vr * di + (-vi) * dr;
    s3 += dr * vr / Vi;
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  out[3] = s3;
}

}  // namespace gn
