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
#include "phase_sync.cuh"

namespace gn {

constexpr int kMaxRhs = 4;

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
  double *partials;  // [2 slots][kSyncQ][gridDim.x]
  PhaseBar *bar;
  int *err;
  const int *abort_flag;  // host-mapped; nonzero asks the kernel to stop
  CgState *state;         // [kMaxRhs]
};

// NR: right-hand-side slots unrolled (>= nrhs); BS: threads per block.
template <typename T, int NC, int NR, int BS>
__global__ void __launch_bounds__(BS, 1) cg_kernel(CgArgs<T> a) {
  __shared__ SyncShared sh;
  double *const s_val = sh.val;
  __shared__ double s_alpha[kMaxRhs], s_beta[kMaxRhs], s_rr[kMaxRhs], s_tau[kMaxRhs];
  __shared__ int s_active[kMaxRhs], s_status[kMaxRhs];
  __shared__ long long s_iters[kMaxRhs];
  __shared__ double s_r2[kMaxRhs], s_b2[kMaxRhs];

  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  double *part0 = a.partials;
  double *part1 = a.partials + size_t(kSyncQ + 1) * gridDim.x;
  unsigned long long nph = 0;  // phases ended so far (same count in every block)
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
      for (int k = 0; k < NR; k++) {
        if (k >= a.nrhs) break;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const T *xv = a.x[k] + size_t(c) * V;
          const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return xv[j]; });
          a.t[k][size_t(c) * V + i] = apply_Mt<T>(s, smi, n);
        }
      }
    }
    double acc[2 * kMaxRhs];
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    ok = end_phase<1>(acc, sh, part1, a.bar, nph++, a.err);
    // r = b - M t ; sums r^2 and b^2
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    if (ok) {
      for (uint32_t i = i0; i < V; i += stride) {
        const Site s = make_site(g, i);
        const T smi = sm[i];
#pragma unroll
        for (int k = 0; k < NR; k++) {
          if (k >= a.nrhs) break;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const T *tv = a.t[k] + size_t(c) * V;
            const Nb<T> n = gather7<T>(s, i, [&](uint32_t j) { return tv[j]; });
            const T bi = a.b[k][size_t(c) * V + i];
            const T ri = apply_sub_M<T>(s, bi, smi, n);
            a.r[k][size_t(c) * V + i] = ri;
            acc[k] += double(ri) * double(ri);
            acc[NR + k] += double(bi) * double(bi);
          }
        }
      }
    }
    ok = end_phase<2 * NR>(acc, sh, part0, a.bar, nph++, a.err) && ok;
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs) {
        const double bb = s_val[NR + k];
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
        for (int k = 0; k < NR; k++) {
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
    ok = end_phase<NR>(acc, sh, part1, a.bar, nph++, a.err) && ok;
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
    // the host's abort request lives in mapped host memory: one thread reads it
    // every 16 iterations, and the value is only used at the end of phase B
    int abort_req = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.abort_flag != nullptr && (it & 15) == 0)
      abort_req = *(volatile const int *)a.abort_flag;
    // phase A: p = r + beta p_old (it > 0), t = M^T p, sum t^2
    double acc[2 * kMaxRhs];
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const T smi = sm[i];
#pragma unroll
      for (int k = 0; k < NR; k++) {
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
    ok = end_phase<NR>(acc, sh, part0, a.bar, nph++, a.err);
    if (!ok) break;
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
      for (int k = 0; k < NR; k++) {
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
    ok = end_phase<NR>(acc, sh, part1, a.bar, nph++, a.err, abort_req);
    if (!ok) break;
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
    if (sh.flag != 0) {  // block 0 saw the host's abort request at the last phase end
      if (threadIdx.x == 0 && blockIdx.x == 0) atomicExch(a.err, 2);
      ok = false;
      break;
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
