// ops_kernels.cuh -- the non-solver kernels of the sigma-HMC path.  Each one is
// a single sweep over the V sites (grid-stride), HBM-bound.
#pragma once
#include "rowvec.cuh"

namespace gn {

constexpr int kOpThreads = 256;

// Dirac apply on ncomp planes: op 0 = M, 1 = M^T, 2 = out -= M in.
// Algorithmic traffic 3 words per site and plane (in, sm, out; +1 read for op 2).
// One item of W sites per thread (rowvec.cuh: W = 2 with 128-bit loads when
// L/2 is even), a grid covering every item (blockIdx.y = plane) and no
// grid-stride loop: few registers, so all 2048 thread slots of an SM are
// filled and the hardware streams blocks in as others finish -- the stencil's
// seven loads per item need that many requests in flight to cover the memory
// latency.  Items run in row order with both parities of a row together, so
// each value of `in` comes from DRAM once although it is read as a centre and
// as a neighbour.
template <int W, int OP>
__global__ void __launch_bounds__(kOpThreads) dirac_item_kernel(Geom g, const double *__restrict__ sm,
                                                               const double *__restrict__ in,
                                                               double *__restrict__ out) {
  const uint32_t V = uint32_t(g.V);
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= row_items<W>(g)) return;
  const double *pv = in + size_t(blockIdx.y) * V;
  double *ov = out + size_t(blockIdx.y) * V;
  const RowItem it = make_item<W>(g, j);
  Nb<double> n[W];
  gather_item<double, W>(
      it, n, [&](uint32_t i, double(&v)[W]) { vload<double, W>(pv + i, v); }, [&](uint32_t i) { return __ldg(pv + i); });
  double smv[W], o[W];
  vload<double, W>(sm + it.own, smv);
  if (OP == 0) {
    item_M<double, W>(it, smv, n, o);
  } else if (OP == 1) {
    item_Mt<double, W>(it, smv, n, o);
  } else {
    vload<double, W>(ov + it.own, o);
    item_sub_M<double, W>(it, smv, n, o);
  }
  vstore<double, W>(ov + it.own, o);
}

// sigma mass (sigma.c:75-94): sm(x) = 1/8 sum of sigma over the 8 dual sites
// whose cube contains x, i.e. sigma at x - {0, 0^, 1^, 2^, 0^+1^, 0^+2^, 1^+2^,
// 0^+1^+2^}, added in that order.  With eps != 0 it is fused with the sigma
// step of EvolveCoordinatesSigma (moleculardynamics.c:824-836):
// sigma_out = sigma_in + eps P, and sm is built from the updated values (every
// thread forms sigma_in + eps P identically, so the neighbour values agree bit
// for bit with the stored ones).  sigma_out must not alias sigma_in.
// Loads of the per-site helpers: through the read-only cache (RO) when the
// data is constant for the kernel's lifetime (separate launches), plain when
// the same kernel writes it in an earlier phase (the batched kernel).
template <bool RO, typename T>
__device__ __forceinline__ T ld_site(const T *p) {
  if constexpr (RO) return __ldg(p);
  else return *p;
}

template <typename T, bool RO = true>
__device__ __forceinline__ void sigma_mass_site(const Geom &g, uint32_t i, const T *__restrict__ sigma_in,
                                                const T *__restrict__ P, T eps, T *__restrict__ sigma_out,
                                                T *__restrict__ sm) {
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  uint32_t x0, x1, x2, par, row, k;
  site_coords(g, i, x0, x1, x2, par, row, k);
  T s = T(0);
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const uint32_t j = corner_index<-1>(g, x0, x1, x2, off[c][0], off[c][1], off[c][2]);
    T v = ld_site<RO>(sigma_in + j);
    if (P != nullptr) v = v + eps * ld_site<RO>(P + j);
    s = (c == 0) ? v : s + v;
  }
  sm[i] = s / T(8);
  if (sigma_out != nullptr) {
    T v = ld_site<RO>(sigma_in + i);
    if (P != nullptr) v = v + eps * ld_site<RO>(P + i);
    sigma_out[i] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(kOpThreads) sigma_mass_kernel(Geom g, const T *__restrict__ sigma_in,
                                                               const T *__restrict__ P, T eps,
                                                               T *__restrict__ sigma_out, T *__restrict__ sm) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
    sigma_mass_site<T>(g, i, sigma_in, P, eps, sigma_out, sm);
}

// P += eps F (EvolveMomentaSigma, moleculardynamics.c:843-848)
template <typename T>
__global__ void __launch_bounds__(kOpThreads) momenta_kernel(uint32_t V, T *P, const T *__restrict__ F, T eps) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) P[i] = P[i] + F[i] * eps;
}

// Sigma force (moleculardynamics.c:576-647):
//   F(x~) = sum_f sum_{c in corners(x~)} 1/8 X_f(c) Y_f(c) - (N_f beta_s / 2) sigma(x~)
// corners in the reference's order x, x+0^+1^, x+0^+2^, x+1^+2^, x+0^, x+1^,
// x+2^, x+0^+1^+2^; flavour 0 first.  X_f = (M M^T)^-1 phi_f, Y_f = M^T X_f.
// If P != null the momentum step P += pcoef F is fused (the integrators always
// follow a force by one).
template <typename T, bool RO = true>
__device__ __forceinline__ void force_site(const Geom &g, uint32_t i, const T *__restrict__ X, const T *__restrict__ Y,
                                           const T *__restrict__ sigma, T gcoef, T *__restrict__ F, T *P, T pcoef) {
  const uint32_t V = uint32_t(g.V);
  const int off[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
  uint32_t x0, x1, x2, par, row, k;
  site_coords(g, i, x0, x1, x2, par, row, k);
  uint32_t cj[8];
#pragma unroll
  for (int c = 0; c < 8; c++) cj[c] = corner_index<1>(g, x0, x1, x2, off[c][0], off[c][1], off[c][2]);
  T f = T(0);
#pragma unroll
  for (int fl = 0; fl < 2; fl++) {
    const T *Xf = X + size_t(fl) * V;
    const T *Yf = Y + size_t(fl) * V;
#pragma unroll
    for (int c = 0; c < 8; c++) f = f + T(0.125) * (ld_site<RO>(Xf + cj[c]) * ld_site<RO>(Yf + cj[c]));
  }
  f = f - gcoef * ld_site<RO>(sigma + i);
  F[i] = f;
  if (P != nullptr) P[i] = P[i] + f * pcoef;
}

template <typename T>
__global__ void __launch_bounds__(kOpThreads) force_kernel(Geom g, const T *__restrict__ X, const T *__restrict__ Y,
                                                          const T *__restrict__ sigma, T gcoef, T *__restrict__ F,
                                                          T *P, T pcoef) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
    force_site<T>(g, i, X, Y, sigma, gcoef, F, P, pcoef);
}

// Compensated block sums of up to 7 quantities: per thread a Neumaier sum,
// per block a tree of (hi, lo) pairs.  Writes part[q*2*nb + 2*block + {0,1}].
template <int NQ>
__device__ __forceinline__ void publish_compensated(double (&hi)[NQ], double (&lo)[NQ], double *part) {
  __shared__ double s_h[NQ][kOpThreads], s_l[NQ][kOpThreads];
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    s_h[q][threadIdx.x] = hi[q];
    s_l[q][threadIdx.x] = lo[q];
  }
  __syncthreads();
  for (int w = kOpThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        double s, e;
        two_sum(s_h[q][threadIdx.x], s_h[q][threadIdx.x + w], s, e);
        s_h[q][threadIdx.x] = s;
        s_l[q][threadIdx.x] = s_l[q][threadIdx.x] + s_l[q][threadIdx.x + w] + e;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      part[(size_t(q) * gridDim.x + blockIdx.x) * 2 + 0] = s_h[q][0];
      part[(size_t(q) * gridDim.x + blockIdx.x) * 2 + 1] = s_l[q][0];
    }
  }
}

__device__ __forceinline__ void neumaier(double &hi, double &lo, double v) {
  double s, e;
  two_sum(hi, v, s, e);
  hi = s;
  lo += e;
}

// Energy terms (ComputeFullEnergyForSigma, moleculardynamics.c:299-319):
//   q0 = sum P^2 / 2, q1 = sum_f sum 1/2 phi_f X_f, q2 = sum sigma^2
template <typename T>
__global__ void __launch_bounds__(kOpThreads) energy_kernel(uint32_t V, const T *__restrict__ P,
                                                           const T *__restrict__ phi, const T *__restrict__ X,
                                                           const T *__restrict__ sigma, double *part) {
  double hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    const double p = double(P[i]);
    neumaier(hi[0], lo[0], p * p / 2.0);
    neumaier(hi[1], lo[1], 0.5 * (double(phi[i]) * double(X[i])));
    neumaier(hi[1], lo[1], 0.5 * (double(phi[V + i]) * double(X[V + i])));
    const double s = double(sigma[i]);
    neumaier(hi[2], lo[2], s * s);
  }
  publish_compensated<3>(hi, lo, part);
}

// Condensate dot products (condensate.c:142-145, :172, :194, :209, :227) of a
// complex vector v = (vr, vi) with D = (Dr, Di), both as two planes:
//   q0 = sum Re(conj v D) / V, q1 = sum Re(conj v D), q2 = sum Im(conj v D)
static __global__ void __launch_bounds__(kOpThreads) cond_dot_kernel(uint32_t V, const double *__restrict__ v,
                                                             const double *__restrict__ D, double *part) {
  double hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
  const double Vd = double(V);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    const double vr = v[i], vi = v[V + i], dr = D[i], di = D[V + i];
    const double re = vr * dr - (-vi) * di;
    neumaier(hi[0], lo[0], re / Vd);
    neumaier(hi[1], lo[1], re);
    neumaier(hi[2], lo[2], vr * di + (-vi) * dr);
  }
  publish_compensated<3>(hi, lo, part);
}

// Condensate source vectors (condensate.c:52-104), complex planes (re, im):
//   mode 0: Z2 noise from signs[x] (+1 / -1, drawn on the host)
//   mode 1: 1/V everywhere
//   mode 2: phase table[x2] (re, im) indexed by the time coordinate
//   mode 3: v *= sm (pointwise, both planes)
static __global__ void __launch_bounds__(kOpThreads) cond_fill_kernel(Geom g, int mode, const signed char *__restrict__ signs,
                                                              const double *__restrict__ table,
                                                              const double *__restrict__ sm, double *v) {
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    if (mode == 0) {
      v[i] = signs[i] > 0 ? 1.0 : -1.0;
      v[V + i] = 0.0;
    } else if (mode == 1) {
      v[i] = 1.0 / double(int(V));
      v[V + i] = 0.0;
    } else if (mode == 2) {
      uint32_t x0, x1, x2, par, row, k;
      site_coords(g, i, x0, x1, x2, par, row, k);
      v[i] = table[2 * x2];
      v[V + i] = table[2 * x2 + 1];
    } else {
      v[i] = v[i] * sm[i];
      v[V + i] = v[V + i] * sm[i];
    }
  }
}


// ------------------------------------------------------------------ U(1) model
// M, M^dagger or out - M psi with the complex mass sm + i eps pm (rowvec.cuh)
// on complex fields of two planes each: system y = blockIdx.y uses planes 2y
// (real) and 2y + 1 (imaginary).
template <int W, int OP>
__global__ void __launch_bounds__(kOpThreads) dirac_cm_kernel(Geom g, const double *__restrict__ sm,
                                                             const double *__restrict__ pm,
                                                             const double *__restrict__ in, double *__restrict__ out) {
  const uint32_t V = uint32_t(g.V);
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= row_items<W>(g)) return;
  const double *pr = in + size_t(2 * blockIdx.y) * V, *pi = pr + V;
  double *orr = out + size_t(2 * blockIdx.y) * V, *oi = orr + V;
  const RowItem it = make_item<W>(g, j);
  Nb<double> nr[W], ni[W];
  gather_item<double, W>(it, pr, nr);
  gather_item<double, W>(it, pi, ni);
  double smv[W], b[W], o_r[W], o_i[W];
  vload<double, W>(sm + it.own, smv);
  item_eps_pm<double, W>(g, it, pm, b);
  if (OP == 0) {
    item_M_cm<double, W>(it, smv, b, nr, ni, o_r, o_i);
  } else if (OP == 1) {
    item_Mt_cm<double, W>(it, smv, b, nr, ni, o_r, o_i);
  } else {
    vload<double, W>(orr + it.own, o_r);
    vload<double, W>(oi + it.own, o_i);
    item_sub_M_cm<double, W>(it, smv, b, nr, ni, o_r, o_i);
  }
  vstore<double, W>(orr + it.own, o_r);
  vstore<double, W>(oi + it.own, o_i);
}

// The fermion forces of the U(1) model on complex X_f, Y_f (flavour f: planes
// 2f, 2f + 1), over the corners of force_site in its order, flavour 0 first:
//   sigma: F += 1/8 Re(conj X Y)           (moleculardynamics.c:590-622)
//   pi:    F += 1/8 Re(i eps conj X Y)     (moleculardynamics.c:695-733)
// then F -= gcoef field (the quadratic terms, :576-581 / :681-686), and the
// momentum step P += pcoef F when P is given.  C forms Re(conj X Y) as
// Xr Yr - (-Xi) Yi and Re(i eps conj X Y) as (eps Xi) Yr - (eps Xr) Yi.
template <bool PI>
__global__ void __launch_bounds__(kOpThreads) force_cm_kernel(Geom g, const double *__restrict__ X,
                                                             const double *__restrict__ Y,
                                                             const double *__restrict__ field, double gcoef,
                                                             double *__restrict__ F, double *P, double pcoef) {
  const uint32_t V = uint32_t(g.V);
  const int off[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    uint32_t x0, x1, x2, par, row, k;
    site_coords(g, i, x0, x1, x2, par, row, k);
    uint32_t cj[8];
#pragma unroll
    for (int c = 0; c < 8; c++) cj[c] = corner_index<1>(g, x0, x1, x2, off[c][0], off[c][1], off[c][2]);
    double f = 0.0;
#pragma unroll
    for (int fl = 0; fl < 2; fl++) {
      const double *Xr = X + size_t(2 * fl) * V, *Xi = Xr + V;
      const double *Yr = Y + size_t(2 * fl) * V, *Yi = Yr + V;
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const uint32_t j = cj[c];
        const double xr = __ldg(Xr + j), xi = __ldg(Xi + j), yr = __ldg(Yr + j), yi = __ldg(Yi + j);
        double t;
        if constexpr (PI) {
          const double e = j >= uint32_t(g.half) ? -1.0 : 1.0;
          t = (e * xi) * yr - (e * xr) * yi;
        } else {
          t = xr * yr - (-xi) * yi;
        }
        f = f + 0.125 * t;
      }
    }
    f = f - gcoef * __ldg(field + i);
    F[i] = f;
    if (P != nullptr) P[i] = P[i] + f * pcoef;
  }
}

// Energy terms with complex phi_f, X_f (planes 2f, 2f + 1):
//   q0 = sum P^2 / 2, q1 = sum_f sum 1/2 Re(conj phi_f X_f), q2 = sum field^2
// (ComputeFullEnergyForSigma / ForPi, moleculardynamics.c:299-319, :349-369).
static __global__ void __launch_bounds__(kOpThreads) energy_cm_kernel(uint32_t V, const double *__restrict__ P,
                                                              const double *__restrict__ phi,
                                                              const double *__restrict__ X,
                                                              const double *__restrict__ field, double *part) {
  double hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    const double p = P[i];
    neumaier(hi[0], lo[0], p * p / 2.0);
#pragma unroll
    for (int fl = 0; fl < 2; fl++) {
      const double pr = phi[size_t(2 * fl) * V + i], pim = phi[size_t(2 * fl + 1) * V + i];
      const double xr = X[size_t(2 * fl) * V + i], xi = X[size_t(2 * fl + 1) * V + i];
      neumaier(hi[1], lo[1], 0.5 * (pr * xr - (-pim) * xi));
    }
    const double s = field[i];
    neumaier(hi[2], lo[2], s * s);
  }
  publish_compensated<3>(hi, lo, part);
}

// ------------------------------------------------------------------ sigma observables
// CondensateSigmaPi (observables.c:323-369, the Z2 model): with t = sigma(x) / V,
//   s0 = sum_x t,   s1+2d + i s2+2d = sum_x exp(i P_MIN x_d) t   (d = 0, 1, 2),
// P_MIN = 2 PI / L formed as macro.h:178 forms it, the angle as the
// reference's product P_MIN * x_d.  From the sums (sigma_obs_finish):
//   condensate = s0, |condensate|, mu2 = s0^2, mu4 = mu2^2, chi = V mu2,
//   chip = V |box_2|^2, chip_pbc1 = V |box_0|^2, chip_pbc2 = V |box_1|^2.
constexpr double kPi = 3.14159265358979323846;
constexpr int kSigmaObsSums = 7;
constexpr int kSigmaObs = 8;

// pi != null: the U(1) model's order parameter |(sigma, pi)| = pow(sigma^2 +
// pi^2, 0.5) in place of sigma (observables.c:354-357).
__device__ __forceinline__ void sigma_obs_site(const Geom &g, uint32_t i, const double *__restrict__ sigma,
                                               double (&v)[kSigmaObsSums], const double *__restrict__ pi = nullptr) {
  uint32_t x[3], par, row, k;
  site_coords(g, i, x[0], x[1], x[2], par, row, k);
  const double t = (pi == nullptr ? sigma[i] : sqrt(sigma[i] * sigma[i] + pi[i] * pi[i])) / double(g.V);
  const double pmin = (2 * kPi) / double(g.L);
  v[0] = t;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double sn, cs;
    sincos(pmin * double(x[d]), &sn, &cs);
    v[1 + 2 * d] = cs * t;
    v[2 + 2 * d] = sn * t;
  }
}

__host__ __device__ inline void sigma_obs_finish(const double (&s)[kSigmaObsSums], double V, double (&out)[kSigmaObs]) {
  const double c = s[0];
  out[0] = c;
  out[1] = c < 0 ? -c : c;
  out[2] = c * c;
  out[3] = out[2] * out[2];
  out[4] = V * out[2];
  out[5] = V * (s[5] * s[5] + s[6] * s[6]);
  out[6] = V * (s[1] * s[1] + s[2] * s[2]);
  out[7] = V * (s[3] * s[3] + s[4] * s[4]);
}

static __global__ void __launch_bounds__(kOpThreads) sigma_obs_kernel(Geom g, const double *__restrict__ sigma,
                                                                      const double *__restrict__ pi, double *part) {
  double hi[kSigmaObsSums], lo[kSigmaObsSums];
#pragma unroll
  for (int q = 0; q < kSigmaObsSums; q++) hi[q] = lo[q] = 0.0;
  const uint32_t V = uint32_t(g.V);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    double v[kSigmaObsSums];
    sigma_obs_site(g, i, sigma, v, pi);
#pragma unroll
    for (int q = 0; q < kSigmaObsSums; q++) neumaier(hi[q], lo[q], v[q]);
  }
  publish_compensated<kSigmaObsSums>(hi, lo, part);
}

}  // namespace gn
