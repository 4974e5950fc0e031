// cg_kernel.cuh -- conjugate gradient on A = M M^T as ONE persistent,
// cooperative kernel per solve (conjugategradient.c:13-107 and :115-182).
//
// Why persistent: at the reference's lattice sizes a CG iteration is a few µs
// of memory traffic (the whole working set of L = 64 sits in the 126 MB L2),
// so kernel launches and host round trips would dominate.  The kernel runs all
// iterations; the grid synchronises with a bounded barrier between phases, and
// every block reduces the per-block partial sums itself (same order in every
// block, so every block computes bit-identical scalars and takes the same
// branches).  Up to kMaxRhs independent right-hand sides run in lock step (the
// two pseudofermion flavours share one sweep of sm and of the geometry), each
// with its own alpha, beta and stopping test, exactly as separate solves.
//
// Per iteration, two phases (12 words of traffic per site and RHS):
//   A: p <- r + beta p (on the fly at the 7 stencil points), t = M^T p, sum t^2
//   B: x += alpha p, r -= alpha M t, sum r^2 ; stop when sqrt(sum r^2) < tol
// The update formulas and their rounding follow the reference (x += a p,
// r += (-a) Ap, p = r + b p; no FMA in the FP64 build); only the order of the
// global sums differs (tree instead of serial).
#pragma once
#include "device_common.cuh"

namespace gn {

constexpr int kMaxRhs = 4;
constexpr int kCgThreads = 256;

enum CgStatus : int {
  kCgRunning = 0,
  kCgConverged = 1,      // converged inside the loop: counted by the reference
  kCgConvergedStart = 2, // the start vector already satisfied tol: not counted
  kCgMaxIter = 3,        // iteration cap reached: the reference returns false
  kCgError = 4           // barrier timeout or abort
};

struct CgState {
  int status;
  int reliable;  // mixed precision: reliable updates done
  long long iters;
  double r2;  // last |r|^2 seen by the stopping test
  double b2;  // |b|^2
};

template <typename T>
struct CgArgs {
  Geom g;
  const T *sm;
  const T *b[kMaxRhs];
  T *x[kMaxRhs];
  T *r[kMaxRhs];
  T *p0[kMaxRhs];
  T *p1[kMaxRhs];
  T *t[kMaxRhs];
  int nrhs;
  int variant;  // 0: test the incoming x first (START_X0_NULL form); 1: x = 0
  int rel;      // 0: stop at |r| < tol; 1: stop at |r| < tol |b|
  double tol;
  long long max_iter;
  double *partials;  // [2 slots][2 quantities][kMaxRhs][gridDim.x]
  GridBar *bar;
  int *err;
  const int *abort_flag;  // host-mapped; nonzero asks the kernel to stop
  CgState *state;         // [kMaxRhs]
};

// Every block sums the partials of one slot (8 values per block) and leaves the
// totals in s_val[0..7].  Warp j sums quantity j; fixed order.
__device__ __forceinline__ void collect8(const double *part, int nb, double *s_val) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (w < 2 * kMaxRhs) {
    const double *p = part + size_t(w) * nb;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int b = lane;
    for (; b + 96 < nb; b += 128) {
      s0 += p[b];
      s1 += p[b + 32];
      s2 += p[b + 64];
      s3 += p[b + 96];
    }
    for (; b < nb; b += 32) s0 += p[b];
    double s = warp_sum((s0 + s1) + (s2 + s3));
    if (lane == 0) s_val[w] = s;
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ void publish8(double (&v)[2 * kMaxRhs], double *smem, double *part, int nb) {
  block_sum<2 * kMaxRhs>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) part[size_t(j) * nb + blockIdx.x] = v[j];
  }
}

template <typename T, int NC>
__global__ void __launch_bounds__(kCgThreads) cg_kernel(CgArgs<T> a) {
  __shared__ double s_red[32 * 2 * kMaxRhs];
  __shared__ double s_val[2 * kMaxRhs];
  __shared__ double s_alpha[kMaxRhs], s_beta[kMaxRhs], s_rr[kMaxRhs], s_tau[kMaxRhs];
  __shared__ int s_active[kMaxRhs], s_status[kMaxRhs];
  __shared__ long long s_iters[kMaxRhs];
  __shared__ double s_r2[kMaxRhs], s_b2[kMaxRhs];

  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const int nb = gridDim.x;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  double *part0 = a.partials;
  double *part1 = a.partials + size_t(2 * kMaxRhs) * nb;
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = ld_acquire(&a.bar->gen);
  const T *__restrict__ sm = a.sm;

  if (threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    s_active[k] = k < a.nrhs;
    s_status[k] = k < a.nrhs ? kCgRunning : kCgConverged;
    s_iters[k] = 0;
    s_alpha[k] = s_beta[k] = s_rr[k] = s_r2[k] = s_b2[k] = 0.0;
    s_tau[k] = a.tol;
  }
  __syncthreads();
  bool ok = true;

  // ---------------------------------------------------------------- start
  if (a.variant == 0) {
    // t = M^T x_in
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const T smi = sm[i];
#pragma unroll
      for (int k = 0; k < kMaxRhs; k++) {
        if (k >= a.nrhs) break;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const T *xv = a.x[k] + size_t(c) * V;
          const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return xv[j]; });
          a.t[k][size_t(c) * V + i] = apply_Mt<T>(s, smi, n);
        }
      }
    }
    ok = grid_barrier(a.bar, gen, a.err);
    // r = b - M t ; sums r^2 and b^2
    double acc[2 * kMaxRhs];
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    if (ok) {
      for (uint32_t i = i0; i < V; i += stride) {
        const Site s = make_site(g, i);
        const T smi = sm[i];
#pragma unroll
        for (int k = 0; k < kMaxRhs; k++) {
          if (k >= a.nrhs) break;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const T *tv = a.t[k] + size_t(c) * V;
            const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return tv[j]; });
            const T bi = a.b[k][size_t(c) * V + i];
            const T ri = apply_sub_M<T>(s, bi, smi, n);
            a.r[k][size_t(c) * V + i] = ri;
            acc[k] += double(ri) * double(ri);
            acc[kMaxRhs + k] += double(bi) * double(bi);
          }
        }
      }
    }
    publish8<T>(acc, s_red, part0, nb);
    ok = grid_barrier(a.bar, gen, a.err) && ok;
    collect8(part0, nb, s_val);
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs) {
        const double bb = s_val[kMaxRhs + k];
        s_b2[k] = bb;
        s_r2[k] = s_val[k];
        s_tau[k] = a.rel ? a.tol * sqrt(bb) : a.tol;
        if (sqrt(s_val[k]) < s_tau[k]) {
          s_active[k] = 0;
          s_status[k] = kCgConvergedStart;
        }
      }
    }
    __syncthreads();
  }
  // x = 0, r = b, p = b ; rr = sum b^2
  {
    double acc[2 * kMaxRhs];
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    if (ok) {
      for (uint32_t i = i0; i < V; i += stride) {
#pragma unroll
        for (int k = 0; k < kMaxRhs; k++) {
          if (k >= a.nrhs || !s_active[k]) continue;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t j = size_t(c) * V + i;
            const T bi = a.b[k][j];
            a.x[k][j] = T(0);
            a.r[k][j] = bi;
            a.p0[k][j] = bi;
            acc[k] += double(bi) * double(bi);
          }
        }
      }
    }
    publish8<T>(acc, s_red, part1, nb);
    ok = grid_barrier(a.bar, gen, a.err) && ok;
    collect8(part1, nb, s_val);
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs && s_active[k]) {
        s_rr[k] = s_val[k];
        s_r2[k] = s_val[k];
        s_b2[k] = s_val[k];
        if (a.variant == 1) {
          s_tau[k] = a.rel ? a.tol * sqrt(s_val[k]) : a.tol;
          if (sqrt(s_val[k]) < s_tau[k]) {
            s_active[k] = 0;
            s_status[k] = kCgConvergedStart;
          }
        }
      }
    }
    __syncthreads();
  }

  // ---------------------------------------------------------------- iterations
  long long it = 0;
  for (; ok && it < a.max_iter; it++) {
    int any = 0;
#pragma unroll
    for (int k = 0; k < kMaxRhs; k++) any |= (k < a.nrhs) ? s_active[k] : 0;
    if (!any) break;
    // phase A: p = r + beta p_old (it > 0), t = M^T p, sum t^2
    double acc[2 * kMaxRhs];
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const T smi = sm[i];
#pragma unroll
      for (int k = 0; k < kMaxRhs; k++) {
        if (k >= a.nrhs || !s_active[k]) continue;
        const T beta = T(s_beta[k]);
        T *const pn = (it & 1) ? a.p1[k] : a.p0[k];
        const T *const po = (it & 1) ? a.p0[k] : a.p1[k];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          Nb<T> n;
          if (it == 0) {
            const T *pv = pn + off;
            n = gather7<T>(s, i, [&](uint32_t j) { return pv[j]; });
          } else {
            const T *rv = a.r[k] + off;
            const T *pov = po + off;
            n = gather7<T>(s, i, [&](uint32_t j) { return rv[j] + beta * pov[j]; });
            pn[off + i] = n.c;
          }
          const T ti = apply_Mt<T>(s, smi, n);
          a.t[k][off + i] = ti;
          acc[k] += double(ti) * double(ti);
        }
      }
    }
    publish8<T>(acc, s_red, part0, nb);
    ok = grid_barrier(a.bar, gen, a.err);
    if (!ok) break;
    collect8(part0, nb, s_val);
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs && s_active[k]) s_alpha[k] = s_rr[k] / s_val[k];
    }
    __syncthreads();
    // phase B: Ap = M t, x += alpha p, r -= alpha Ap, sum r^2
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const T smi = sm[i];
#pragma unroll
      for (int k = 0; k < kMaxRhs; k++) {
        if (k >= a.nrhs || !s_active[k]) continue;
        const T alpha = T(s_alpha[k]);
        const T malpha = -alpha;
        const T *const pn = (it & 1) ? a.p1[k] : a.p0[k];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          const T *tv = a.t[k] + off;
          const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return tv[j]; });
          const T ap = apply_M<T>(s, smi, n);
          const T pi = pn[off + i];
          a.x[k][off + i] = a.x[k][off + i] + alpha * pi;
          const T ri = a.r[k][off + i] + malpha * ap;
          a.r[k][off + i] = ri;
          acc[k] += double(ri) * double(ri);
        }
      }
    }
    publish8<T>(acc, s_red, part1, nb);
    ok = grid_barrier(a.bar, gen, a.err);
    if (!ok) break;
    collect8(part1, nb, s_val);
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs && s_active[k]) {
        const double r2 = s_val[k];
        if (sqrt(r2) < s_tau[k]) {
          s_active[k] = 0;
          s_status[k] = kCgConverged;
          s_iters[k] = it + 1;
        } else {
          s_beta[k] = r2 / s_rr[k];
          s_rr[k] = r2;
        }
        s_r2[k] = r2;
      }
    }
    // host abort request: block 0's view decides for everyone at the next phase
    __syncthreads();
    if (a.abort_flag != nullptr) {
      if (threadIdx.x == 0 && blockIdx.x == 0 && *(volatile const int *)a.abort_flag) atomicExch(a.err, 2);
    }
  }
  // ---------------------------------------------------------------- results
  if (blockIdx.x == 0 && threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    if (k < a.nrhs) {
      CgState st;
      st.status = s_status[k];
      if (!ok) st.status = kCgError;
      else if (st.status == kCgRunning) st.status = kCgMaxIter;
      st.reliable = 0;
      st.iters = (s_status[k] == kCgRunning) ? it : s_iters[k];
      st.r2 = s_r2[k];
      st.b2 = s_b2[k];
      a.state[k] = st;
    }
  }
}

}  // namespace gn
