// ops_kernels.cuh -- the non-solver kernels of the sigma-HMC path.  Each one is
// a single sweep over the V sites (grid-stride), HBM-bound.
#pragma once
#include "device_common.cuh"

namespace gn {

constexpr int kOpThreads = 256;

// Dirac apply on ncomp planes: op 0 = M, 1 = M^T, 2 = out -= M in.
// Algorithmic traffic 3 words per site and plane (in, sm, out; +1 read for op 2).
// One site per thread and a grid covering every site (blockIdx.y = plane), no
// grid-stride loop: few registers, so all 2048 thread slots of an SM are
// filled and the hardware streams blocks in as others finish -- the stencil's
// seven loads per site need that many requests in flight to cover the memory
// latency.
template <typename T, int OP>
__global__ void __launch_bounds__(kOpThreads) dirac_kernel(Geom g, const T *__restrict__ sm, const T *__restrict__ in,
                                                          T *__restrict__ out) {
  const uint32_t V = uint32_t(g.V);
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  const T *pv = in + size_t(blockIdx.y) * V;
  T *ov = out + size_t(blockIdx.y) * V;
  const Site s = make_site(g, i);
  const T smi = __ldg(sm + i);
  const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return __ldg(pv + j); });
  if (OP == 0) ov[i] = apply_M<T>(s, smi, n);
  else if (OP == 1) ov[i] = apply_Mt<T>(s, smi, n);
  else ov[i] = apply_sub_M<T>(s, ov[i], smi, n);
}

// The same apply two sites at a time with 128-bit loads, for L a multiple of
// 4 (L/2 even).  A thread takes the sites (k, k+1), k even, of one parity row:
// their x0 +- 1 and x1 +- 1 neighbours are the pairs (k, k+1) of rows a plane
// or a row away in the other half, 16-byte aligned; their time neighbours are
// the pair (k, k+1) of the same row of the other half plus one more value,
// k-1 or k+2.  With b = (parity + x0 + x1) & 1 the site k sits at x2 = 2k + b:
//   b = 0:  up(k) = q[k], dn(k) = q[k-1], up(k+1) = q[k+1], dn(k+1) = q[k]
//   b = 1:  up(k) = q[k+1], dn(k) = q[k], up(k+1) = q[k+2], dn(k+1) = q[k+1]
// (indices mod L/2); the antiperiodic sign can only fall on dn(k) at x2 = 0
// (b = 0, k = 0) or on up(k+1) at x2 = L-1 (b = 1, k = L/2-2).  Every site is
// computed with the same operation order as dirac_kernel.
template <int OP>
__global__ void __launch_bounds__(kOpThreads) dirac_pair_kernel(Geom g, const double *__restrict__ sm,
                                                               const double *__restrict__ in,
                                                               double *__restrict__ out) {
  const uint32_t V = uint32_t(g.V), half = uint32_t(g.half), quarter = half / 2u;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= half) return;
  const double *pv = in + size_t(blockIdx.y) * V;
  double *ov = out + size_t(blockIdx.y) * V;
  const uint32_t par = t >= quarter ? 1u : 0u;
  const uint32_t h = 2u * (t - par * quarter);  // even half index: the pair (h, h+1)
  const uint32_t row = fdiv(h, g.div_Lh);
  const uint32_t k = h - row * uint32_t(g.Lh);
  const uint32_t x0 = fdiv(row, g.div_L);
  const uint32_t x1 = row - x0 * uint32_t(g.L);
  const uint32_t L = uint32_t(g.L), Lh = uint32_t(g.Lh), P = uint32_t(g.plane);
  const uint32_t b = (par + x0 + x1) & 1u;
  const uint32_t own = par * half + h, qb = (1u - par) * half;
  const double2 psi = __ldg(reinterpret_cast<const double2 *>(pv + own));
  const double2 smv = __ldg(reinterpret_cast<const double2 *>(sm + own));
  const double2 u0 = __ldg(reinterpret_cast<const double2 *>(pv + qb + ((x0 + 1u == L) ? h - (L - 1u) * P : h + P)));
  const double2 d0 = __ldg(reinterpret_cast<const double2 *>(pv + qb + ((x0 == 0u) ? h + (L - 1u) * P : h - P)));
  const double2 u1 = __ldg(reinterpret_cast<const double2 *>(pv + qb + ((x1 + 1u == L) ? h - (L - 1u) * Lh : h + Lh)));
  const double2 d1 = __ldg(reinterpret_cast<const double2 *>(pv + qb + ((x1 == 0u) ? h + (L - 1u) * Lh : h - Lh)));
  const double2 tq = __ldg(reinterpret_cast<const double2 *>(pv + qb + h));
  // the extra time value: k-1 (b = 0) or k+2 (b = 1), wrapping within the row
  const uint32_t rb = qb + row * Lh;
  const uint32_t ke = b ? ((k + 2u == Lh) ? 0u : k + 2u) : ((k == 0u) ? Lh - 1u : k - 1u);
  const double te = __ldg(pv + rb + ke);
  const uint32_t e1 = x0 & 1u, e2 = (x0 + x1) & 1u;
  // sign bits as in Site::neg: bits 0..2 forward, 3..5 backward
  uint32_t negA = (e1 << 1) | (e2 << 2) | (e1 << 4) | (e2 << 5);
  uint32_t negB = negA;
  if (b == 0u && k == 0u) negA ^= 1u << 5;        // dn(k) at x2 = 0
  if (b == 1u && k + 2u == Lh) negB ^= 1u << 2;   // up(k+1) at x2 = L-1
  Site sA, sB;
  sA.neg = negA;
  sB.neg = negB;
  Nb<double> A, B;
  A.c = psi.x;
  B.c = psi.y;
  A.up[0] = u0.x; B.up[0] = u0.y;
  A.dn[0] = d0.x; B.dn[0] = d0.y;
  A.up[1] = u1.x; B.up[1] = u1.y;
  A.dn[1] = d1.x; B.dn[1] = d1.y;
  if (b == 0u) {
    A.up[2] = tq.x; A.dn[2] = te; B.up[2] = tq.y; B.dn[2] = tq.x;
  } else {
    A.up[2] = tq.y; A.dn[2] = tq.x; B.up[2] = te; B.dn[2] = tq.y;
  }
  double2 o;
  if (OP == 0) {
    o.x = apply_M<double>(sA, smv.x, A);
    o.y = apply_M<double>(sB, smv.y, B);
  } else if (OP == 1) {
    o.x = apply_Mt<double>(sA, smv.x, A);
    o.y = apply_Mt<double>(sB, smv.y, B);
  } else {
    const double2 prev = *reinterpret_cast<const double2 *>(ov + own);
    o.x = apply_sub_M<double>(sA, prev.x, smv.x, A);
    o.y = apply_sub_M<double>(sB, prev.y, smv.y, B);
  }
  *reinterpret_cast<double2 *>(ov + own) = o;
}

// sigma mass (sigma.c:75-94): sm(x) = 1/8 sum of sigma over the 8 dual sites
// whose cube contains x, i.e. sigma at x - {0, 0^, 1^, 2^, 0^+1^, 0^+2^, 1^+2^,
// 0^+1^+2^}, added in that order.  With eps != 0 it is fused with the sigma
// step of EvolveCoordinatesSigma (moleculardynamics.c:824-836):
// sigma_out = sigma_in + eps P, and sm is built from the updated values (every
// thread forms sigma_in + eps P identically, so the neighbour values agree bit
// for bit with the stored ones).  sigma_out must not alias sigma_in.
template <typename T>
__global__ void __launch_bounds__(kOpThreads) sigma_mass_kernel(Geom g, const T *__restrict__ sigma_in,
                                                               const T *__restrict__ P, T eps,
                                                               T *__restrict__ sigma_out, T *__restrict__ sm) {
  const uint32_t V = uint32_t(g.V);
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    uint32_t x0, x1, x2, par, row, k;
    site_coords(g, i, x0, x1, x2, par, row, k);
    T s = T(0);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const uint32_t j = site_index(g, int(x0) - off[c][0], int(x1) - off[c][1], int(x2) - off[c][2]);
      T v = __ldg(sigma_in + j);
      if (P != nullptr) v = v + eps * __ldg(P + j);
      s = (c == 0) ? v : s + v;
    }
    sm[i] = s / T(8);
    if (sigma_out != nullptr) {
      T v = __ldg(sigma_in + i);
      if (P != nullptr) v = v + eps * __ldg(P + i);
      sigma_out[i] = v;
    }
  }
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
template <typename T>
__global__ void __launch_bounds__(kOpThreads) force_kernel(Geom g, const T *__restrict__ X, const T *__restrict__ Y,
                                                          const T *__restrict__ sigma, T gcoef, T *__restrict__ F,
                                                          T *P, T pcoef) {
  const uint32_t V = uint32_t(g.V);
  const int off[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    uint32_t x0, x1, x2, par, row, k;
    site_coords(g, i, x0, x1, x2, par, row, k);
    uint32_t cj[8];
#pragma unroll
    for (int c = 0; c < 8; c++) cj[c] = site_index(g, int(x0) + off[c][0], int(x1) + off[c][1], int(x2) + off[c][2]);
    T f = T(0);
#pragma unroll
    for (int fl = 0; fl < 2; fl++) {
      const T *Xf = X + size_t(fl) * V;
      const T *Yf = Y + size_t(fl) * V;
#pragma unroll
      for (int c = 0; c < 8; c++) f = f + T(0.125) * (__ldg(Xf + cj[c]) * __ldg(Yf + cj[c]));
    }
    f = f - gcoef * __ldg(sigma + i);
    F[i] = f;
    if (P != nullptr) P[i] = P[i] + f * pcoef;
  }
}

// Compensated block sums of up to 4 quantities: per thread a Neumaier sum,
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
__global__ void __launch_bounds__(kOpThreads) cond_dot_kernel(uint32_t V, const double *__restrict__ v,
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
__global__ void __launch_bounds__(kOpThreads) cond_fill_kernel(Geom g, int mode, const signed char *__restrict__ signs,
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

}  // namespace gn
