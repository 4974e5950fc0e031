// device_common.cuh -- building blocks shared by every kernel: the staggered
// stencils and deterministic reductions.  (The solvers' grid barrier is in
// phase_sync.cuh.)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "geometry.cuh"

namespace gn {

// ------------------------------------------------------------------ stencils
// The Dirac operator of dirac.c:46-82 on one site, real arithmetic (the
// reference's fields are complex with a zero imaginary part on this path;
// a genuinely complex field is handled as two real planes):
//   (M psi)(x)   = sm(x) psi(x) + sum_mu 1/2 [eta_pp(x,mu) psi(x+mu) - eta_mm(x,mu) psi(x-mu)]
//   (M^T psi)(x) = sm(x) psi(x) - sum_mu 1/2 [eta_pp(x,mu) psi(x+mu) - eta_mm(x,mu) psi(x-mu)]
// M^T is the gather form of the scatter in dirac.c:88-123 (eta_mm(x+mu, mu) =
// eta_pp(x, mu) under antiperiodic time).  The order of the additions of M
// (and of out - M psi) is the reference's: mass term first, then mu = 0, 1, 2
// with the forward term before the backward one.  With FMA contraction off
// (the FP64 translation units are built with --fmad=false) M is therefore bit
// identical to DiracFermion; M^T adds the same seven terms in another order.
template <typename T>
struct Nb {
  T c, up[3], dn[3];
};

template <typename T, typename Load>
__device__ __forceinline__ Nb<T> gather7(const Site &s, uint32_t i, Load ld) {
  Nb<T> n;
  n.c = ld(i);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    n.up[d] = ld(s.nb_up[d]);
    n.dn[d] = ld(s.nb_dn[d]);
  }
  return n;
}

// Each hopping term is (+-1/2) psi, an exact product, so adding the term
// with the sign of eta equals the reference's t += (0.5 eta) psi bit for bit.
template <typename T>
__device__ __forceinline__ T hop_add(T t, T v, uint32_t neg, int bit) {
  const T h = T(0.5) * v;
  return ((neg >> bit) & 1u) ? t - h : t + h;
}
template <typename T>
__device__ __forceinline__ T hop_sub(T t, T v, uint32_t neg, int bit) {
  const T h = T(0.5) * v;
  return ((neg >> bit) & 1u) ? t + h : t - h;
}

template <typename T>
__device__ __forceinline__ T apply_M(const Site &s, T sm, const Nb<T> &n) {
  T t = sm * n.c;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    t = hop_add(t, n.up[d], s.neg, d);
    t = hop_sub(t, n.dn[d], s.neg, 3 + d);
  }
  return t;
}

template <typename T>
__device__ __forceinline__ T apply_Mt(const Site &s, T sm, const Nb<T> &n) {
  T t = sm * n.c;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    t = hop_sub(t, n.up[d], s.neg, d);
    t = hop_add(t, n.dn[d], s.neg, 3 + d);
  }
  return t;
}

// out - M psi in the order of SubtractDiracFermion (dirac.c:213-247)
template <typename T>
__device__ __forceinline__ T apply_sub_M(const Site &s, T out, T sm, const Nb<T> &n) {
  T t = out - sm * n.c;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    t = hop_sub(t, n.up[d], s.neg, d);
    t = hop_add(t, n.dn[d], s.neg, 3 + d);
  }
  return t;
}

// ------------------------------------------------------------------ reductions
// Deterministic: fixed shuffle pattern, fixed warp order.  Every call with the
// same inputs returns the same bits.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums N values over the block; thread 0 gets the totals in v.
// smem needs 32*N doubles.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *smem) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int j = 0; j < N; j++) v[j] = warp_sum(v[j]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < N; j++) smem[j * 32 + w] = v[j];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int j = 0; j < N; j++) {
      double a = lane < nw ? smem[j * 32 + lane] : 0.0;
      v[j] = warp_sum(a);
    }
  }
  __syncthreads();
}

// Error-free two-sum (Knuth), for compensated energy sums.
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

}  // namespace gn
