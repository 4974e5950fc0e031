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
struct MtOrder {
  uint32_t idx[6];
  int kind[6];  // 0..2: backward source mu (added), 3..5: forward source mu (subtracted)
};

__device__ __forceinline__ MtOrder mt_ref_order(const Site &s) {
  MtOrder o;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    o.idx[d] = s.nb_dn[d];
    o.kind[d] = d;
    o.idx[3 + d] = s.nb_up[d];
    o.kind[3 + d] = 3 + d;
  }
  // insertion sort of six keys
  for (int a = 1; a < 6; a++) {
    const uint32_t ki = o.idx[a];
    const int kk = o.kind[a];
    int b = a - 1;
    while (b >= 0 && o.idx[b] > ki) {
      o.idx[b + 1] = o.idx[b];
      o.kind[b + 1] = o.kind[b];
      b--;
    }
    o.idx[b + 1] = ki;
    o.kind[b + 1] = kk;
  }
  return o;
}

// the six hopping terms of one plane added to t (the site's mass term) in that order
__device__ __forceinline__ double mt_hops(const Site &s, const MtOrder &o, const double *psi, double t) {
  for (int a = 0; a < 6; a++) {
    const int kd = o.kind[a];
    const double v = psi[o.idx[a]];
    if (kd < 3) t = hop_add(t, v, s.neg, 3 + kd);  // +1/2 eta_mm(i, mu) psi(i - mu)
    else t = hop_sub(t, v, s.neg, kd - 3);         // -1/2 eta_pp(i, mu) psi(i + mu)
  }
  return t;
}

__device__ __forceinline__ double apply_Mt_ref_order(const Site &s, double sm, const double *psi, uint32_t i) {
  return mt_hops(s, mt_ref_order(s), psi, sm * psi[i]);
}

// The U(1) model's complex mass (dirac.c:66-69, :107-110): sm + i b with
// b = eps_pi pm, eps_pi = +1 on the even half and -1 on the odd one.
__device__ __forceinline__ double eps_pm(const Geom &g, const double *pm, uint32_t i) {
  return i >= uint32_t(g.half) ? -pm[i] : pm[i];
}

// M^dagger of a complex psi (planes re, im) at site i: the mass sm - i b times
// psi as C forms the product, (sm c - (-b) d) + i (sm d + (-b) c), then each
// plane's hopping terms in the scatter order above.
__device__ __forceinline__ void apply_Mt_ref_order_cm(const Site &s, double sm, double b, const double *re,
                                                      const double *im, uint32_t i, double &out_r, double &out_i) {
  const MtOrder o = mt_ref_order(s);
  const double mb = -b, c = re[i], d = im[i];
  out_r = mt_hops(s, o, re, sm * c - mb * d);
  out_i = mt_hops(s, o, im, sm * d + mb * c);
}

// M and out - M psi of a complex psi at one site (gather order, as DiracFermion
// and SubtractDiracFermion add their terms): the mass product first.
__device__ __forceinline__ void apply_M_cm(const Site &s, double sm, double b, const Nb<double> &nr,
                                           const Nb<double> &ni, double &out_r, double &out_i) {
  double tr = sm * nr.c - b * ni.c, ti = sm * ni.c + b * nr.c;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    tr = hop_add(tr, nr.up[d], s.neg, d);
    tr = hop_sub(tr, nr.dn[d], s.neg, 3 + d);
    ti = hop_add(ti, ni.up[d], s.neg, d);
    ti = hop_sub(ti, ni.dn[d], s.neg, 3 + d);
  }
  out_r = tr;
  out_i = ti;
}
__device__ __forceinline__ void apply_sub_M_cm(const Site &s, double sm, double b, const Nb<double> &nr,
                                               const Nb<double> &ni, double &out_r, double &out_i) {
  double tr = out_r - (sm * nr.c - b * ni.c), ti = out_i - (sm * ni.c + b * nr.c);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    tr = hop_sub(tr, nr.up[d], s.neg, d);
    tr = hop_add(tr, nr.dn[d], s.neg, 3 + d);
    ti = hop_sub(ti, ni.up[d], s.neg, d);
    ti = hop_add(ti, ni.dn[d], s.neg, 3 + d);
  }
  out_r = tr;
  out_i = ti;
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
  const double *pm;  // the U(1) model's pi mass (complex mass sm + i eps pm, nc = 2), else null
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
__device__ __forceinline__ void exact_mt(const Geom &g, const double *sm, const double *pm, const double *in,
                                         double *out, int nc) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = threadIdx.x; i < V; i += blockDim.x) {
    const Site s = make_site(g, i);
    if (pm != nullptr) {
      apply_Mt_ref_order_cm(s, sm[i], eps_pm(g, pm, i), in, in + V, i, out[i], out[V + i]);
    } else {
      for (int c = 0; c < nc; c++) out[size_t(c) * V + i] = apply_Mt_ref_order(s, sm[i], in + size_t(c) * V, i);
    }
  }
}

// M (or b - M) on all sites of the block's share, gather order.
__device__ __forceinline__ void exact_m(const Geom &g, const double *sm, const double *pm, const double *in,
                                        const double *b, double *out, int nc) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = threadIdx.x; i < V; i += blockDim.x) {
    const Site s = make_site(g, i);
    if (pm != nullptr) {
      const Nb<double> nr = gather7<double>(s, i, [&](uint32_t j) { return in[j]; });
      const Nb<double> ni = gather7<double>(s, i, [&](uint32_t j) { return in[V + j]; });
      double o_r, o_i;
      if (b != nullptr) {
        o_r = b[i];
        o_i = b[V + i];
        apply_sub_M_cm(s, sm[i], eps_pm(g, pm, i), nr, ni, o_r, o_i);
      } else {
        apply_M_cm(s, sm[i], eps_pm(g, pm, i), nr, ni, o_r, o_i);
      }
      out[i] = o_r;
      out[V + i] = o_i;
    } else {
      for (int c = 0; c < nc; c++) {
        const double *tv = in + size_t(c) * V;
        const Nb<double> nb = gather7<double>(s, i, [&](uint32_t j) { return tv[j]; });
        out[size_t(c) * V + i] = b != nullptr ? apply_sub_M<double>(s, b[size_t(c) * V + i], sm[i], nb)
                                              : apply_M<double>(s, sm[i], nb);
      }
    }
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
    exact_mt(g, a.sm, a.pm, a.x, a.t, nc);
    __syncthreads();
    exact_m(g, a.sm, a.pm, a.t, a.b, a.r, nc);
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
    exact_mt(g, a.sm, a.pm, a.p, a.t, nc);
    __syncthreads();
    const double pap = serial(0, a.t);
    const double alpha = rr / pap;
    for (size_t j = threadIdx.x; j < n; j += blockDim.x) a.x[j] = a.x[j] + alpha * a.p[j];
    exact_m(g, a.sm, a.pm, a.t, nullptr, a.ap, nc);
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

// M^dagger of complex systems with the complex mass, reference order: system
// y = blockIdx.y on planes 2y (real) and 2y + 1 (imaginary).
__global__ void __launch_bounds__(256) mt_exact_cm_kernel(Geom g, const double *__restrict__ sm,
                                                         const double *__restrict__ pm,
                                                         const double *__restrict__ in, double *__restrict__ out) {
  const uint32_t V = uint32_t(g.V);
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const Site s = make_site(g, i);
  const double *re = in + size_t(2 * blockIdx.y) * V;
  double *o = out + size_t(2 * blockIdx.y) * V;
  apply_Mt_ref_order_cm(s, sm[i], eps_pm(g, pm, i), re, re + V, i, o[i], o[V + i]);
}

// Serial sums of the U(1) model's energies (moleculardynamics.c:299-319 and
// :349-367 in the PI_INTERACTION build): out[0] = sum P^2/2, then, in the same
// accumulator, sum_f sum_x 0.5 Re(conj phi_f X_f), formed as C forms it,
// 0.5 (pr Xr - (-pi) Xi); out[1] = sum of the field squared (sigma or pi).
__global__ void energy_cm_exact_kernel(uint32_t V, const double *P, const double *phi, const double *X,
                                       const double *field, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double total = 0.0;
  for (uint32_t r = 0; r < V; r++) total += (P[r] * P[r] / 2.0);
  for (int f = 0; f < 2; f++) {
    const double *pr = phi + size_t(2 * f) * V, *pim = pr + V;
    const double *xr = X + size_t(2 * f) * V, *xi = xr + V;
    for (uint32_t x = 0; x < V; x++) total += (0.5 * (pr[x] * xr[x] - (-pim[x]) * xi[x]));
  }
  double s2 = 0.0;
  for (uint32_t x = 0; x < V; x++) s2 += field[x] * field[x];
  out[0] = total;
  out[1] = s2;
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
