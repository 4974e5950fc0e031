// mixed_kernel.cuh -- mixed-precision CG on A = M M^T with reliable updates,
// one persistent cooperative kernel per solve.
//
// The bulk of the iterations runs in FP32 (vectors and stencils; half the
// bytes of FP64), with every global sum accumulated in FP64.  The solution is
// accumulated in FP64: the FP32 iterate x^ collects the steps since the last
// reliable update and is folded into the FP64 x at every update, where the
// true residual r = b - A x is recomputed in FP64 and becomes the new FP32
// residual (reliable updates: Sleijpen & van der Vorst 1996; as used for
// lattice solvers by Clark et al., Comput. Phys. Commun. 181 (2010) 1517).
// An update happens when the iterated residual has dropped by a factor delta
// since the last one, after n_ru iterations, or when the iterated residual
// passes the tolerance; the solve stops only on the FP64 true residual, so its
// stopping rule is the same as the FP64 solver's.
//
// Inner iteration, two phases (12 FP32 words per site and RHS):
//   A: p^ <- r^ + beta p^ (on the fly at the 7 points), t^ = M^T p^, sum t^2
//   B: x^ += alpha p^, r^ -= alpha M t^, sum r^2
// Reliable update, two phases (FP64):
//   C: t = M^T (x + x^) (on the fly at the 7 points)
//   D: x += x^, x^ = 0, r = b - M t, r^ = (float) r, sum r^2
#pragma once
#include "cg_kernel.cuh"

namespace gn {

struct MixedArgs {
  Geom g;
  const double *sm;
  float *sm32;
  const double *b[kMaxRhs];
  double *x[kMaxRhs];
  double *t64[kMaxRhs];
  float *rh[kMaxRhs];
  float *ph0[kMaxRhs];
  float *ph1[kMaxRhs];
  float *th[kMaxRhs];
  float *xh[kMaxRhs];
  int nrhs;
  int variant;
  int rel;
  double tol;
  long long max_iter;
  double delta;  // reliable update when |r^| < delta * max |r^| since the last one
  int n_ru;      // ... or after this many inner iterations
  double *partials;
  PhaseBar *bar;
  int *err;
  const int *abort_flag;
  CgState *state;
};

template <int NC, int NR, int BS>
__global__ void __launch_bounds__(BS, 1) cg_mixed_kernel(MixedArgs a) {
  __shared__ SyncShared sh;
  double *const s_val = sh.val;
  __shared__ double s_alpha[kMaxRhs], s_beta[kMaxRhs], s_rr[kMaxRhs], s_tau[kMaxRhs], s_rmax[kMaxRhs];
  __shared__ double s_r2[kMaxRhs], s_b2[kMaxRhs];
  __shared__ int s_active[kMaxRhs], s_status[kMaxRhs], s_ru[kMaxRhs], s_since[kMaxRhs], s_nru[kMaxRhs];
  __shared__ long long s_iters[kMaxRhs];
  __shared__ int s_any_ru;

  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  double *part0 = a.partials;
  double *part1 = a.partials + size_t(kSyncQ + 1) * gridDim.x;
  unsigned long long nph = 0;  // phases ended so far (same count in every block)
  const double *__restrict__ sm = a.sm;

  if (threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    s_active[k] = k < a.nrhs;
    s_status[k] = k < a.nrhs ? kCgRunning : kCgConverged;
    s_iters[k] = 0;
    s_alpha[k] = s_beta[k] = s_rr[k] = s_r2[k] = s_b2[k] = s_rmax[k] = 0.0;
    s_tau[k] = a.tol;
    s_ru[k] = 0;
    s_since[k] = 0;
    s_nru[k] = 0;
  }
  __syncthreads();
  bool ok = true;
  double acc[2 * kMaxRhs];

  // ---------------------------------------------------------------- start (FP64)
  if (a.variant == 0) {
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const double smi = sm[i];
#pragma unroll
      for (int k = 0; k < NR; k++) {
        if (k >= a.nrhs) break;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const double *xv = a.x[k] + size_t(c) * V;
          const Nb<double> n = gather7<double>(s, i, [&](uint32_t j) { return xv[j]; });
          a.t64[k][size_t(c) * V + i] = apply_Mt<double>(s, smi, n);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    ok = end_phase<1>(acc, sh, part1, a.bar, nph++, a.err);
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    if (ok) {
      for (uint32_t i = i0; i < V; i += stride) {
        const Site s = make_site(g, i);
        const double smi = sm[i];
#pragma unroll
        for (int k = 0; k < NR; k++) {
          if (k >= a.nrhs) break;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const double *tv = a.t64[k] + size_t(c) * V;
            const Nb<double> n = gather7<double>(s, i, [&](uint32_t j) { return tv[j]; });
            const double bi = a.b[k][size_t(c) * V + i];
            const double ri = apply_sub_M<double>(s, bi, smi, n);
            acc[k] += ri * ri;
            acc[NR + k] += bi * bi;
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
  // x = 0, x^ = 0, r^ = p^ = (float) b, sm32 = (float) sm ; sums r^2 (FP32 values), b^2
#pragma unroll
  for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
  if (ok) {
    for (uint32_t i = i0; i < V; i += stride) {
      a.sm32[i] = float(sm[i]);
#pragma unroll
      for (int k = 0; k < NR; k++) {
        if (k >= a.nrhs || !s_active[k]) continue;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t j = size_t(c) * V + i;
          const double bi = a.b[k][j];
          const float bf = float(bi);
          a.x[k][j] = 0.0;
          a.xh[k][j] = 0.f;
          a.rh[k][j] = bf;
          a.ph0[k][j] = bf;
          acc[k] += double(bf) * double(bf);
          acc[NR + k] += bi * bi;
        }
      }
    }
  }
  ok = end_phase<2 * NR>(acc, sh, part1, a.bar, nph++, a.err) && ok;
  if (threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    if (k < a.nrhs && s_active[k]) {
      s_rr[k] = s_val[k];
      s_rmax[k] = sqrt(s_val[k]);
      s_r2[k] = s_val[NR + k];
      s_b2[k] = s_val[NR + k];
      if (a.variant == 1) {
        s_tau[k] = a.rel ? a.tol * sqrt(s_val[NR + k]) : a.tol;
        if (sqrt(s_val[NR + k]) < s_tau[k]) {
          s_active[k] = 0;
          s_status[k] = kCgConvergedStart;
        }
      }
    }
  }
  __syncthreads();

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
    // A: p^ = r^ + beta p^, t^ = M^T p^
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const float smi = a.sm32[i];
#pragma unroll
      for (int k = 0; k < NR; k++) {
        if (k >= a.nrhs || !s_active[k]) continue;
        const float beta = float(s_beta[k]);
        float *const pn = (it & 1) ? a.ph1[k] : a.ph0[k];
        const float *const po = (it & 1) ? a.ph0[k] : a.ph1[k];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          Nb<float> n;
          if (it == 0) {
            const float *pv = pn + off;
            n = gather7<float>(s, i, [&](uint32_t j) { return pv[j]; });
          } else {
            const float *rv = a.rh[k] + off;
            const float *pov = po + off;
            n = gather7<float>(s, i, [&](uint32_t j) { return fmaf(beta, pov[j], rv[j]); });
            pn[off + i] = n.c;
          }
          const float ti = apply_Mt<float>(s, smi, n);
          a.th[k][off + i] = ti;
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
    // B: x^ += alpha p^, r^ -= alpha M t^
#pragma unroll
    for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
    for (uint32_t i = i0; i < V; i += stride) {
      const Site s = make_site(g, i);
      const float smi = a.sm32[i];
#pragma unroll
      for (int k = 0; k < NR; k++) {
        if (k >= a.nrhs || !s_active[k]) continue;
        const float alpha = float(s_alpha[k]);
        const float *const pn = (it & 1) ? a.ph1[k] : a.ph0[k];
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          const float *tv = a.th[k] + off;
          const Nb<float> n = gather7<float>(s, i, [&](uint32_t j) { return tv[j]; });
          const float ap = apply_M<float>(s, smi, n);
          a.xh[k][off + i] = fmaf(alpha, pn[off + i], a.xh[k][off + i]);
          const float ri = fmaf(-alpha, ap, a.rh[k][off + i]);
          a.rh[k][off + i] = ri;
          acc[k] += double(ri) * double(ri);
        }
      }
    }
    ok = end_phase<NR>(acc, sh, part1, a.bar, nph++, a.err, abort_req);
    if (!ok) break;
    if (threadIdx.x == 0) s_any_ru = 0;
    __syncthreads();
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      s_ru[k] = 0;
      if (k < a.nrhs && s_active[k]) {
        const double r2 = s_val[k];
        const double rn = sqrt(r2);
        s_since[k]++;
        if (rn > s_rmax[k]) s_rmax[k] = rn;
        if (rn < s_tau[k] || rn < a.delta * s_rmax[k] || s_since[k] >= a.n_ru || !(rn == rn)) {
          s_ru[k] = 1;
          atomicOr(&s_any_ru, 1);
          s_r2[k] = r2;  // beta is formed from the true residual below
        } else {
          s_beta[k] = r2 / s_rr[k];
          s_rr[k] = r2;
          s_r2[k] = r2;
        }
      }
    }
    __syncthreads();
    if (s_any_ru) {
      // C: t = M^T (x + x^) in FP64
      for (uint32_t i = i0; i < V; i += stride) {
        const Site s = make_site(g, i);
        const double smi = sm[i];
#pragma unroll
        for (int k = 0; k < NR; k++) {
          if (k >= a.nrhs || !s_ru[k]) continue;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V;
            const double *xv = a.x[k] + off;
            const float *xhv = a.xh[k] + off;
            const Nb<double> n = gather7<double>(s, i, [&](uint32_t j) { return xv[j] + double(xhv[j]); });
            a.t64[k][off + i] = apply_Mt<double>(s, smi, n);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
      ok = end_phase<1>(acc, sh, part0, a.bar, nph++, a.err);
      if (!ok) break;
      // D: x += x^, x^ = 0, r = b - M t, r^ = (float) r
#pragma unroll
      for (int j = 0; j < 2 * kMaxRhs; j++) acc[j] = 0.0;
      for (uint32_t i = i0; i < V; i += stride) {
        const Site s = make_site(g, i);
        const double smi = sm[i];
#pragma unroll
        for (int k = 0; k < NR; k++) {
          if (k >= a.nrhs || !s_ru[k]) continue;
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V;
            a.x[k][off + i] = a.x[k][off + i] + double(a.xh[k][off + i]);
            a.xh[k][off + i] = 0.f;
            const double *tv = a.t64[k] + off;
            const Nb<double> n = gather7<double>(s, i, [&](uint32_t j) { return tv[j]; });
            const double ri = apply_sub_M<double>(s, a.b[k][off + i], smi, n);
            a.rh[k][off + i] = float(ri);
            acc[k] += ri * ri;
          }
        }
      }
      ok = end_phase<NR>(acc, sh, part1, a.bar, nph++, a.err);
      if (!ok) break;
      if (threadIdx.x < kMaxRhs) {
        const int k = threadIdx.x;
        if (k < a.nrhs && s_ru[k]) {
          const double r2 = s_val[k];
          s_nru[k]++;
          s_since[k] = 0;
          s_r2[k] = r2;
          s_rmax[k] = sqrt(r2);
          if (sqrt(r2) < s_tau[k]) {
            s_active[k] = 0;
            s_status[k] = kCgConverged;
            s_iters[k] = it + 1;
          } else {
            s_beta[k] = r2 / s_rr[k];
            s_rr[k] = r2;
          }
        }
      }
      __syncthreads();
    }
    if (sh.flag != 0) {  // block 0 saw the host's abort request at the last phase end
      if (threadIdx.x == 0 && blockIdx.x == 0) atomicExch(a.err, 2);
      ok = false;
      break;
    }
  }
  // ---------------------------------------------------------------- results
  // On the iteration cap x holds the solution of the last reliable update.
  if (blockIdx.x == 0 && threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    if (k < a.nrhs) {
      CgState st;
      st.status = s_status[k];
      if (!ok) st.status = kCgError;
      else if (st.status == kCgRunning) st.status = kCgMaxIter;
      st.reliable = s_nru[k];
      st.iters = (s_status[k] == kCgRunning) ? it : s_iters[k];
      st.r2 = s_r2[k];
      st.b2 = s_b2[k];
      a.state[k] = st;
    }
  }
}

}  // namespace gn
