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
// Two inner iterations, chosen per solve by MixedArgs::scheme:
//
// kMixedSplit -- Chronopoulos & Gear's CG (J. Comput. Appl. Math. 25 (1989)
// 153), whose two global sums g = (r,r) and d = (r, A r) = |M^T r|^2 are taken
// together, with A = M M^T applied as two stencil sweeps:
//   S1: u^ = M^T r^, sums (r^,r^), (u^,u^)                   -> phase end with sums
//       beta = g / g_old, alpha = g / (d - beta g / alpha_old)   (beta = 0 first;
//       a non-positive denominator restarts the direction)
//   S2: a^ <- M u^ + beta a^ (= A p^), p^ <- r^ + beta p^,
//       x^ += alpha p^, r^ -= alpha a^                         -> team barrier
// One phase end with sums and one plain barrier per iteration (about 1.5 us
// against 3.2 - 3.7 us for a phase end with sums on B200): the faster scheme
// while the FP32 vectors stay in L2 and the iteration is latency-bound.
//
// kMixedTwoPhase -- the CG of the FP64 solver, two phase ends with sums:
//   A: p^ <- r^ + beta p^, t^ <- M^T r^ + beta t^ (= M^T p^), sum t^2
//   B: x^ += alpha p^, r^ -= alpha M t^, sum r^2
// Four FP32 vectors instead of five (t^ lives in u^'s array): the faster
// scheme once the working set no longer fits in L2.  Both move 13 FP32 words
// per site and RHS per iteration.
//
// Reliable update (FP64), when the iterated residual has dropped far enough
// (in kMixedSplit S2 is then skipped for that system):
//   C: t = M^T (x + x^) (on the fly at the 7 points)
//   D: x += x^, x^ = 0, r = b - M t, r^ = (float) r, sum r^2
// and the iteration goes on from the true residual, keeping p^ (and a^), as
// the reliable-update CG of Clark et al. keeps p.
// The FP32 phases sweep row items of W sites (rowvec.cuh; W = 4, one float4
// per vector, when 4 divides L/2), the FP64 phases items of min(W, 2) sites;
// a work unit is one (system, item) pair, as in cg_kernel.cuh.
#pragma once
#include "cg_kernel.cuh"

namespace gn {

enum MixedScheme : int { kMixedTwoPhase = 0, kMixedSplit = 1 };

// The split iteration while its FP32 vectors (five per system and plane, and
// sm) take at most 48 MB: measured on B200 with two systems, it is faster at
// L = 96 (39 MB; 17.9 against 18.3 us per iteration) and slower at L = 128
// (92 MB, a working set the 126 MB L2 no longer holds across the sweeps; 33.4
// against 29.1 us).
constexpr double kMixedSplitMaxBytes = 48.0 * (1 << 20);
__host__ __device__ inline int mixed_scheme(int64_t V, int nrhs, int ncomp) {
  const double bytes = double(5 * nrhs * ncomp + 1) * double(V) * 4.0;
  return bytes <= kMixedSplitMaxBytes ? kMixedSplit : kMixedTwoPhase;
}

struct MixedArgs {
  Geom g;
  const double *sm;
  float *sm32;
  const double *pm;  // U(1) model (CM solves): the pi mass, and its FP32 copy
  float *pm32;
  const double *b[kMaxRhs];
  double *x[kMaxRhs];
  double *t64[kMaxRhs];
  float *rh[kMaxRhs];  // r^
  float *ph[kMaxRhs];  // p^
  float *uh[kMaxRhs];  // u^ = M^T r^ (kMixedSplit) or t^ = M^T p^ (kMixedTwoPhase)
  float *ah[kMaxRhs];  // a^ = A p^
  float *xh[kMaxRhs];  // x^
  int nrhs;
  int variant;
  int rel;
  int scheme;      // MixedScheme
  int sm32_ready;  // sm32 (and pm32) already hold the FP32 masses: the start skips forming them
  // a two-team solve's second team starts once *lead (the first team's
  // arrival counter) reaches lead_count: half an iteration behind (null: at once)
  const unsigned long long *lead;
  unsigned long long lead_count;
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

// Block-shared state of one solve (the same values in every block of the team).
struct MixedShared {
  double alpha[kMaxRhs], beta[kMaxRhs], rr[kMaxRhs], tau[kMaxRhs], rmax[kMaxRhs], r2[kMaxRhs], b2[kMaxRhs];
  int active[kMaxRhs], status[kMaxRhs], ru[kMaxRhs], since[kMaxRhs], nru[kMaxRhs], all[kMaxRhs];
  int first[kMaxRhs], step[kMaxRhs];
  long long iters[kMaxRhs];
  SysList run, every, upd, stp;  // systems iterating / all / taking a reliable update / taking a CG step
};

// One mixed-precision solve by a team (all its threads call it; a.bar,
// a.partials and a.err are not used: the team's own are).
//
// CM (NC = 2): the U(1) model's complex mass sm + i eps pm, as in cg_solve;
// always the split inner iteration.
template <int NC, int NR, int W, bool CM = false>
__device__ __forceinline__ void mixed_solve(const MixedArgs &a, Team &team, SyncShared &sh, MixedShared &ms) {
  static_assert(!CM || NC == 2, "the complex mass couples the two planes of a system");
  constexpr int W64 = W >= 2 ? 2 : 1;
  double *const s_val = sh.val;
  double *const s_alpha = ms.alpha, *const s_beta = ms.beta, *const s_rr = ms.rr, *const s_tau = ms.tau;
  double *const s_rmax = ms.rmax, *const s_r2 = ms.r2, *const s_b2 = ms.b2;
  int *const s_active = ms.active, *const s_status = ms.status, *const s_ru = ms.ru, *const s_since = ms.since;
  int *const s_nru = ms.nru, *const s_all = ms.all, *const s_first = ms.first, *const s_step = ms.step;
  long long *const s_iters = ms.iters;
  SysList &s_run = ms.run, &s_every = ms.every, &s_upd = ms.upd, &s_stp = ms.stp;

  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const uint32_t NI = row_items<W>(g), NI64 = row_items<W64>(g);
  const double *__restrict__ sm = a.sm;

  if (team.btid < kMaxRhs) {
    const int k = team.btid;
    s_active[k] = k < a.nrhs;
    s_all[k] = k < a.nrhs;
    s_status[k] = k < a.nrhs ? kCgRunning : kCgConverged;
    s_iters[k] = 0;
    s_alpha[k] = s_beta[k] = s_rr[k] = s_r2[k] = s_b2[k] = s_rmax[k] = 0.0;
    s_tau[k] = a.tol;
    s_ru[k] = 0;
    s_since[k] = 0;
    s_nru[k] = 0;
    s_first[k] = 1;
    s_step[k] = 0;
  }
  team_sync(team);
  if (team.btid == 0) {
    sys_list_from(s_every, s_all, a.nrhs);
    sys_list_from(s_run, s_active, a.nrhs);
  }
  team_sync(team);
  bool ok = true;
  double acc[2 * kMaxRhs];
  auto zero_acc = [&]() {
#pragma unroll
    for (int q = 0; q < 2 * kMaxRhs; q++) acc[q] = 0.0;
  };

  // ---------------------------------------------------------------- start (FP64)
  if (a.variant == 0) {
    for_units(NI64, s_every, team, [&](int k, uint32_t j) {
      const RowItem it = make_item<W64>(g, j);
      double smi[W64];
      vload<double, W64>(sm + it.own, smi);
      const double *xk = pick<NR>(a.x, k);
      double *tk = pick<NR>(a.t64, k);
      if constexpr (CM) {
        Nb<double> nr[W64], ni[W64];
        double b[W64], o_r[W64], o_i[W64];
        gather_item<double, W64>(it, xk, nr);
        gather_item<double, W64>(it, xk + V, ni);
        item_eps_pm<double, W64>(g, it, a.pm, b);
        item_Mt_cm<double, W64>(it, smi, b, nr, ni, o_r, o_i);
        vstore<double, W64>(tk + it.own, o_r);
        vstore<double, W64>(tk + V + it.own, o_i);
      } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
          Nb<double> n[W64];
          double o[W64];
          gather_item<double, W64>(it, xk + size_t(c) * V, n);
          item_Mt<double, W64>(it, smi, n, o);
          vstore<double, W64>(tk + size_t(c) * V + it.own, o);
        }
      }
    });
    ok = team_barrier(sh, team);  // t is complete: no sums needed
    zero_acc();
    if (ok) {
      for_units(NI64, s_every, team, [&](int k, uint32_t j) {
        const RowItem it = make_item<W64>(g, j);
        double smi[W64];
        vload<double, W64>(sm + it.own, smi);
        const double *tk = pick<NR>(a.t64, k);
        const double *bk = pick<NR>(a.b, k);
        if constexpr (CM) {
          Nb<double> nr[W64], ni[W64];
          double b[W64], br[W64], bim[W64], rr[W64], rim[W64];
          gather_item<double, W64>(it, tk, nr);
          gather_item<double, W64>(it, tk + V, ni);
          item_eps_pm<double, W64>(g, it, a.pm, b);
          vload<double, W64>(bk + it.own, br);
          vload<double, W64>(bk + V + it.own, bim);
#pragma unroll
          for (int e = 0; e < W64; e++) {
            rr[e] = br[e];
            rim[e] = bim[e];
          }
          item_sub_M_cm<double, W64>(it, smi, b, nr, ni, rr, rim);
          double sr = 0.0, sb = 0.0;
#pragma unroll
          for (int e = 0; e < W64; e++) {
            sr += rr[e] * rr[e] + rim[e] * rim[e];
            sb += br[e] * br[e] + bim[e] * bim[e];
          }
          acc_add<NR>(acc, k, sr);
          acc_add<NR>(acc, NR + k, sb);
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            Nb<double> n[W64];
            double bi[W64], ri[W64];
            gather_item<double, W64>(it, tk + size_t(c) * V, n);
            vload<double, W64>(bk + size_t(c) * V + it.own, bi);
#pragma unroll
            for (int e = 0; e < W64; e++) ri[e] = bi[e];
            item_sub_M<double, W64>(it, smi, n, ri);
            double sr = 0.0, sb = 0.0;
#pragma unroll
            for (int e = 0; e < W64; e++) {
              sr += ri[e] * ri[e];
              sb += bi[e] * bi[e];
            }
            acc_add<NR>(acc, k, sr);
            acc_add<NR>(acc, NR + k, sb);
          }
        }
      });
    }
    ok = end_phase<2 * NR>(acc, sh, team) && ok;
    if (team.btid < kMaxRhs) {
      const int k = team.btid;
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
    team_sync(team);
    if (team.btid == 0) sys_list_from(s_run, s_active, a.nrhs);
    team_sync(team);
  }
  const bool split = CM || a.scheme == kMixedSplit;
  // x = 0, x^ = 0, r^ = (float) b, p^ = (float) b (two-phase) or 0 (split),
  // a^ = 0, sm32 = (float) sm; sums r^2 (FP32 values), b^2
  zero_acc();
  if (ok) {
    for (uint32_t j = team.tid; !a.sm32_ready && j < NI64; j += team.nthreads) {
      const uint32_t own = make_item<W64>(g, j).own;
      double s64[W64];
      float s32[W64];
      vload<double, W64>(sm + own, s64);
#pragma unroll
      for (int e = 0; e < W64; e++) s32[e] = float(s64[e]);
      vstore<float, W64>(a.sm32 + own, s32);
      if constexpr (CM) {
        vload<double, W64>(a.pm + own, s64);
#pragma unroll
        for (int e = 0; e < W64; e++) s32[e] = float(s64[e]);
        vstore<float, W64>(a.pm32 + own, s32);
      }
    }
    for_units(NI64, s_run, team, [&](int k, uint32_t j) {
      const uint32_t own = make_item<W64>(g, j).own;
      const double *bk = pick<NR>(a.b, k);
      double *xk = pick<NR>(a.x, k);
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const size_t off = size_t(c) * V + own;
        double bi[W64], z64[W64];
        float bf[W64], z32[W64];
        vload<double, W64>(bk + off, bi);
        double sf = 0.0, sb = 0.0;
#pragma unroll
        for (int e = 0; e < W64; e++) {
          bf[e] = float(bi[e]);
          z64[e] = 0.0;
          z32[e] = 0.f;
          sf += double(bf[e]) * double(bf[e]);
          sb += bi[e] * bi[e];
        }
        acc_add<NR>(acc, k, sf);
        acc_add<NR>(acc, NR + k, sb);
        vstore<double, W64>(xk + off, z64);
        vstore<float, W64>(pick<NR>(a.xh, k) + off, z32);
        vstore<float, W64>(pick<NR>(a.ph, k) + off, split ? z32 : bf);
        vstore<float, W64>(pick<NR>(a.ah, k) + off, z32);
        vstore<float, W64>(pick<NR>(a.rh, k) + off, bf);
      }
    });
  }
  ok = end_phase<2 * NR>(acc, sh, team) && ok;
  if (team.btid < kMaxRhs) {
    const int k = team.btid;
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
  team_sync(team);
  if (team.btid == 0) sys_list_from(s_run, s_active, a.nrhs);
  team_sync(team);

  // ---------------------------------------------------------------- iterations
  long long it = 0;
  for (; ok && it < a.max_iter; it++) {
    if (s_run.n == 0) break;
    // the host's abort request lives in mapped host memory: one thread reads it
    // every 16 passes, and the value is only used at the end of the pass's
    // last phase with sums
    int abort_req = 0;
    if (team.brank == 0 && team.btid == 0 && a.abort_flag != nullptr && (it & 15) == 0)
      abort_req = *(volatile const int *)a.abort_flag;
    if (split) {
      // S1: u^ = M^T r^, sums (r^,r^), (u^,u^)
      zero_acc();
      for_units(NI, s_run, team, [&](int k, uint32_t j) {
        const RowItem ri = make_item<W>(g, j);
        float smi[W];
        vload<float, W>(a.sm32 + ri.own, smi);
        const float *rk = pick<NR>(a.rh, k);
        float *uk = pick<NR>(a.uh, k);
        if constexpr (CM) {
          Nb<float> nr[W], ni[W];
          float b[W], u_r[W], u_i[W];
          gather_item<float, W>(ri, rk, nr);
          gather_item<float, W>(ri, rk + V, ni);
          item_eps_pm<float, W>(g, ri, a.pm32, b);
          item_Mt_cm<float, W>(ri, smi, b, nr, ni, u_r, u_i);
          vstore<float, W>(uk + ri.own, u_r);
          vstore<float, W>(uk + V + ri.own, u_i);
          double sg = 0.0, sd = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            sg += double(nr[e].c) * double(nr[e].c) + double(ni[e].c) * double(ni[e].c);
            sd += double(u_r[e]) * double(u_r[e]) + double(u_i[e]) * double(u_i[e]);
          }
          acc_add<NR>(acc, k, sg);
          acc_add<NR>(acc, NR + k, sd);
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V;
            Nb<float> n[W];
            float u[W];
            gather_item<float, W>(ri, rk + off, n);
            item_Mt<float, W>(ri, smi, n, u);
            vstore<float, W>(uk + off + ri.own, u);
            double sg = 0.0, sd = 0.0;
#pragma unroll
            for (int e = 0; e < W; e++) {
              sg += double(n[e].c) * double(n[e].c);
              sd += double(u[e]) * double(u[e]);
            }
            acc_add<NR>(acc, k, sg);
            acc_add<NR>(acc, NR + k, sd);
          }
        }
      });
      // the step parameters of system k from the pass's totals
      auto book = [&](int k) {
        s_ru[k] = 0;
        s_step[k] = 0;
        if (k < a.nrhs && s_active[k]) {
          const double gn = s_val[k], dn = s_val[NR + k];
          const double rn = sqrt(gn);
          s_r2[k] = gn;
          if (rn > s_rmax[k]) s_rmax[k] = rn;
          if (rn < s_tau[k] || !(rn == rn)) {
            // r^ says converged (or is not finite): the true residual decides,
            // and this pass takes no step.  (A step from u^ of the drifted r^
            // after the refresh would leave a^ != A p^ by A (r - r^), an error
            // that a^ and p^ carry on and that grows from one refresh to the next.)
            s_ru[k] = 1;
          } else {
            double bt = 0.0, den = dn;
            if (!s_first[k]) {
              bt = gn / s_rr[k];
              den = dn - bt * gn / s_alpha[k];
              if (!(den > 0.0)) {
                bt = 0.0;
                den = dn;
              }
            }
            s_first[k] = 0;
            s_beta[k] = bt;
            s_alpha[k] = gn / den;
            s_rr[k] = gn;
            s_since[k]++;
            s_step[k] = 1;
            // a scheduled refresh runs after this pass's step (S2 comes before
            // C, D in the split scheme), so the next S1 starts from the true r
            if (rn < a.delta * s_rmax[k] || s_since[k] >= a.n_ru) s_ru[k] = 1;
          }
        }
        if (NR == 1 && k == 0) {  // one system: its lists too, saving a barrier below
          sys_list_from(s_upd, s_ru, a.nrhs);
          sys_list_from(s_stp, s_step, a.nrhs);
        }
      };
      ok = end_phase<2 * NR>(acc, sh, team, abort_req);
      if (ok && team.btid < kMaxRhs) book(int(team.btid));
      if (!ok) break;
    } else {
      // A: p^ = r^ + beta p^, t^ = M^T p^ = M^T r^ + beta t^ (linearity: only r^
      // is gathered; p^ and t^ are updated in place at the unit's own sites)
      zero_acc();
      for_units(NI, s_run, team, [&](int k, uint32_t j) {
        const RowItem ri = make_item<W>(g, j);
        float smi[W];
        vload<float, W>(a.sm32 + ri.own, smi);
        const float beta = float(s_beta[k]);
        float *const pk = pick<NR>(a.ph, k);
        const float *rk = pick<NR>(a.rh, k);
        float *tk = pick<NR>(a.uh, k);
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          Nb<float> n[W];
          float ti[W];
          if (it == 0) {  // p^ = b^ (set above): t^ = M^T p^
            gather_item<float, W>(ri, pk + off, n);
            item_Mt<float, W>(ri, smi, n, ti);
          } else {
            float u[W], told[W], pold[W];
            gather_item<float, W>(ri, rk + off, n);
            vload<float, W>(tk + off + ri.own, told);
            vload<float, W>(pk + off + ri.own, pold);
            item_Mt<float, W>(ri, smi, n, u);
#pragma unroll
            for (int e = 0; e < W; e++) {
              ti[e] = fmaf(beta, told[e], u[e]);
              pold[e] = fmaf(beta, pold[e], n[e].c);
            }
            vstore<float, W>(pk + off + ri.own, pold);
          }
          vstore<float, W>(tk + off + ri.own, ti);
          double st = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) st += double(ti[e]) * double(ti[e]);
          acc_add<NR>(acc, k, st);
        }
      });
      ok = end_phase<NR>(acc, sh, team);
      if (!ok) break;
      if (team.btid < kMaxRhs) {
        const int k = team.btid;
        if (k < a.nrhs && s_active[k]) s_alpha[k] = s_rr[k] / s_val[k];
      }
      team_sync(team);
      // B: x^ += alpha p^, r^ -= alpha M t^
      zero_acc();
      for_units(NI, s_run, team, [&](int k, uint32_t j) {
        const RowItem ri = make_item<W>(g, j);
        float smi[W];
        vload<float, W>(a.sm32 + ri.own, smi);
        const float alpha = float(s_alpha[k]);
        const float *const pn = pick<NR>(a.ph, k);
        const float *tk = pick<NR>(a.uh, k);
        float *xhk = pick<NR>(a.xh, k);
        float *rk = pick<NR>(a.rh, k);
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V + ri.own;
          Nb<float> n[W];
          float ap[W], pv[W], xv[W], rv[W];
          gather_item<float, W>(ri, tk + size_t(c) * V, n);
          vload<float, W>(pn + off, pv);
          vload<float, W>(xhk + off, xv);
          vload<float, W>(rk + off, rv);
          item_M<float, W>(ri, smi, n, ap);
          double sr = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            xv[e] = fmaf(alpha, pv[e], xv[e]);
            rv[e] = fmaf(-alpha, ap[e], rv[e]);
            sr += double(rv[e]) * double(rv[e]);
          }
          acc_add<NR>(acc, k, sr);
          vstore<float, W>(xhk + off, xv);
          vstore<float, W>(rk + off, rv);
        }
      });
      ok = end_phase<NR>(acc, sh, team, abort_req);
      if (!ok) break;
      if (team.btid < kMaxRhs) {
        const int k = team.btid;
        s_ru[k] = 0;
        if (k < a.nrhs && s_active[k]) {
          const double r2 = s_val[k];
          const double rn = sqrt(r2);
          s_since[k]++;
          s_r2[k] = r2;
          if (rn > s_rmax[k]) s_rmax[k] = rn;
          if (rn < s_tau[k] || rn < a.delta * s_rmax[k] || s_since[k] >= a.n_ru || !(rn == rn)) {
            s_ru[k] = 1;  // beta is formed from the true residual below
          } else {
            s_beta[k] = r2 / s_rr[k];
            s_rr[k] = r2;
          }
        }
      }
    }
    const int abort_seen = sh.flag;  // block 0's abort flag (the next phase ends overwrite sh.flag)
    team_sync(team);
    if (!(NR == 1 && split)) {
      if (team.btid == 0) {
        sys_list_from(s_upd, s_ru, a.nrhs);
        if (split) sys_list_from(s_stp, s_step, a.nrhs);
      }
      team_sync(team);
    }
    if (abort_seen != 0) {  // block 0 saw the host's abort request
      if (team.btid == 0 && team.brank == 0) atomicExch(team.err, 2);
      ok = false;
      break;
    }
    if (split && s_stp.n > 0) {
      // S2: a^ = M u^ + beta a^, p^ = r^ + beta p^, x^ += alpha p^, r^ -= alpha a^
      for_units(NI, s_stp, team, [&](int k, uint32_t j) {
        const RowItem ri = make_item<W>(g, j);
        float smi[W];
        vload<float, W>(a.sm32 + ri.own, smi);
        const float alpha = float(s_alpha[k]), beta = float(s_beta[k]);
        const float *uk = pick<NR>(a.uh, k);
        if constexpr (CM) {
          Nb<float> nr[W], ni[W];
          float b[W], w[2][W];
          gather_item<float, W>(ri, uk, nr);
          gather_item<float, W>(ri, uk + V, ni);
          item_eps_pm<float, W>(g, ri, a.pm32, b);
          item_M_cm<float, W>(ri, smi, b, nr, ni, w[0], w[1]);
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const size_t o = size_t(c) * V + ri.own;
            float av[W], pv[W], xv[W], rv[W];
            float *const ak = pick<NR>(a.ah, k) + o;
            float *const pk = pick<NR>(a.ph, k) + o;
            float *const xk = pick<NR>(a.xh, k) + o;
            float *const rk = pick<NR>(a.rh, k) + o;
            vload<float, W>(ak, av);
            vload<float, W>(pk, pv);
            vload<float, W>(xk, xv);
            vload<float, W>(rk, rv);
#pragma unroll
            for (int e = 0; e < W; e++) {
              av[e] = fmaf(beta, av[e], w[c][e]);
              pv[e] = fmaf(beta, pv[e], rv[e]);
              xv[e] = fmaf(alpha, pv[e], xv[e]);
              rv[e] = fmaf(-alpha, av[e], rv[e]);
            }
            vstore<float, W>(ak, av);
            vstore<float, W>(pk, pv);
            vstore<float, W>(xk, xv);
            vstore<float, W>(rk, rv);
          }
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V;
            const size_t o = off + ri.own;
            Nb<float> n[W];
            float w[W], av[W], pv[W], xv[W], rv[W];
            gather_item<float, W>(ri, uk + off, n);
            float *const ak = pick<NR>(a.ah, k) + o;
            float *const pk = pick<NR>(a.ph, k) + o;
            float *const xk = pick<NR>(a.xh, k) + o;
            float *const rk = pick<NR>(a.rh, k) + o;
            vload<float, W>(ak, av);
            vload<float, W>(pk, pv);
            vload<float, W>(xk, xv);
            vload<float, W>(rk, rv);
            item_M<float, W>(ri, smi, n, w);
#pragma unroll
            for (int e = 0; e < W; e++) {
              av[e] = fmaf(beta, av[e], w[e]);
              pv[e] = fmaf(beta, pv[e], rv[e]);
              xv[e] = fmaf(alpha, pv[e], xv[e]);
              rv[e] = fmaf(-alpha, av[e], rv[e]);
            }
            vstore<float, W>(ak, av);
            vstore<float, W>(pk, pv);
            vstore<float, W>(xk, xv);
            vstore<float, W>(rk, rv);
          }
        }
      });
      ok = team_barrier(sh, team);
      if (!ok) break;
    }
    if (s_upd.n > 0) {
      // C: t = M^T (x + x^) in FP64
      for_units(NI64, s_upd, team, [&](int k, uint32_t j) {
        const RowItem it = make_item<W64>(g, j);
        double smi[W64];
        vload<double, W64>(sm + it.own, smi);
        const double *xk = pick<NR>(a.x, k);
        const float *xhk = pick<NR>(a.xh, k);
        double *tk = pick<NR>(a.t64, k);
        if constexpr (CM) {
          Nb<double> n[2][W64];
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const double *xv = xk + size_t(c) * V;
            const float *xhv = xhk + size_t(c) * V;
            gather_item<double, W64>(
                it, n[c],
                [&](uint32_t i, double(&v)[W64]) {
                  double xx[W64];
                  float hh[W64];
                  vload<double, W64>(xv + i, xx);
                  vload<float, W64>(xhv + i, hh);
#pragma unroll
                  for (int e = 0; e < W64; e++) v[e] = xx[e] + double(hh[e]);
                },
                [&](uint32_t i) { return xv[i] + double(xhv[i]); });
          }
          double b[W64], o_r[W64], o_i[W64];
          item_eps_pm<double, W64>(g, it, a.pm, b);
          item_Mt_cm<double, W64>(it, smi, b, n[0], n[1], o_r, o_i);
          vstore<double, W64>(tk + it.own, o_r);
          vstore<double, W64>(tk + V + it.own, o_i);
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V;
            const double *xv = xk + off;
            const float *xhv = xhk + off;
            Nb<double> n[W64];
            gather_item<double, W64>(
                it, n,
                [&](uint32_t i, double(&v)[W64]) {
                  double xx[W64];
                  float hh[W64];
                  vload<double, W64>(xv + i, xx);
                  vload<float, W64>(xhv + i, hh);
#pragma unroll
                  for (int e = 0; e < W64; e++) v[e] = xx[e] + double(hh[e]);
                },
                [&](uint32_t i) { return xv[i] + double(xhv[i]); });
            double o[W64];
            item_Mt<double, W64>(it, smi, n, o);
            vstore<double, W64>(tk + off + it.own, o);
          }
        }
      });
      ok = team_barrier(sh, team);  // t is complete: no sums needed
      if (!ok) break;
      // D: x += x^, x^ = 0, r = b - M t, r^ = (float) r
      zero_acc();
      for_units(NI64, s_upd, team, [&](int k, uint32_t j) {
        const RowItem it = make_item<W64>(g, j);
        double smi[W64];
        vload<double, W64>(sm + it.own, smi);
        const double *bk = pick<NR>(a.b, k);
        const double *tk = pick<NR>(a.t64, k);
        double *xk = pick<NR>(a.x, k);
        float *xhk = pick<NR>(a.xh, k);
        float *rhk = pick<NR>(a.rh, k);
        if constexpr (CM) {
          Nb<double> nr[W64], ni[W64];
          double b[W64], rv[2][W64];
          gather_item<double, W64>(it, tk, nr);
          gather_item<double, W64>(it, tk + V, ni);
          item_eps_pm<double, W64>(g, it, a.pm, b);
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const size_t off = size_t(c) * V + it.own;
            double xx[W64];
            float hh[W64], z32[W64];
            vload<double, W64>(xk + off, xx);
            vload<float, W64>(xhk + off, hh);
#pragma unroll
            for (int e = 0; e < W64; e++) {
              xx[e] = xx[e] + double(hh[e]);
              z32[e] = 0.f;
            }
            vstore<double, W64>(xk + off, xx);
            vstore<float, W64>(xhk + off, z32);
            vload<double, W64>(bk + off, rv[c]);
          }
          item_sub_M_cm<double, W64>(it, smi, b, nr, ni, rv[0], rv[1]);
          double sr = 0.0;
#pragma unroll
          for (int c = 0; c < 2; c++) {
            float rf[W64];
#pragma unroll
            for (int e = 0; e < W64; e++) {
              rf[e] = float(rv[c][e]);
              sr += rv[c][e] * rv[c][e];
            }
            vstore<float, W64>(rhk + size_t(c) * V + it.own, rf);
          }
          acc_add<NR>(acc, k, sr);
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V + it.own;
            double xx[W64], ri[W64];
            float hh[W64], z32[W64], rf[W64];
            vload<double, W64>(xk + off, xx);
            vload<float, W64>(xhk + off, hh);
#pragma unroll
            for (int e = 0; e < W64; e++) {
              xx[e] = xx[e] + double(hh[e]);
              z32[e] = 0.f;
            }
            vstore<double, W64>(xk + off, xx);
            vstore<float, W64>(xhk + off, z32);
            Nb<double> n[W64];
            gather_item<double, W64>(it, tk + size_t(c) * V, n);
            vload<double, W64>(bk + off, ri);
            item_sub_M<double, W64>(it, smi, n, ri);
            double sr = 0.0;
#pragma unroll
            for (int e = 0; e < W64; e++) {
              rf[e] = float(ri[e]);
              sr += ri[e] * ri[e];
            }
            acc_add<NR>(acc, k, sr);
            vstore<float, W64>(rhk + off, rf);
          }
        }
      });
      ok = end_phase<NR>(acc, sh, team);
      if (!ok) break;
      if (team.btid < kMaxRhs) {
        const int k = team.btid;
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
          } else if (!split) {
            s_beta[k] = r2 / s_rr[k];
            s_rr[k] = r2;
          }
        }
      }
      team_sync(team);
      if (team.btid == 0) sys_list_from(s_run, s_active, a.nrhs);
      team_sync(team);
    }
  }
  // ---------------------------------------------------------------- results
  // On the iteration cap x holds the solution of the last reliable update.
  if (team.brank == 0 && team.btid < kMaxRhs) {
    const int k = team.btid;
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

// The single-lattice solve: the whole cooperative grid is the team.
template <int NC, int NR, int BS, int W, bool CM = false>
__global__ void __launch_bounds__(BS, 1) cg_mixed_kernel(MixedArgs a) {
  __shared__ SyncShared sh;
  __shared__ MixedShared ms;
  Team team = grid_team(a.bar, a.partials, a.err);
  mixed_solve<NC, NR, W, CM>(a, team, sh, ms);
}

// Two independent systems in one cooperative launch (the two pseudofermion
// flavours of a force): system h runs on the threads [h BS/2, (h+1) BS/2) of
// every block, as a team of its own -- its own arrival counter, partial sums,
// phase count and named barrier 1 + h.  The systems never wait for each other,
// so while one system's blocks wait at a phase end the other system's stencil
// sweep has the SM's load/store path to itself; and each system stops on its
// own convergence instead of running in lock step with the other.  To set the
// two teams half an iteration apart, team 1 starts when team 0 has ended its
// first phase (a1.lead; the wait is bounded and only a matter of timing).
// Measured on B200 at L = 64, two flavours from x = 0 to 1e-10: 10.1 us per
// iteration in lock step, 9.6 with two teams started together, 8.8 with the
// offset.  a0 and a1 are the two systems' solves (nrhs = 1 each).  Each half
// runs its own inlined copy of the solver, which reads its argument struct
// from the kernel's parameters at fixed offsets, as the single-team kernel
// does.
template <int NC, int BS, int W, int H, bool CM>
__device__ __forceinline__ void duo_half(const MixedArgs &a, SyncShared &sh, MixedShared &ms) {
  Team team;
  team.tid = blockIdx.x * (BS / 2) + (threadIdx.x - H * (BS / 2));
  team.nthreads = gridDim.x * (BS / 2);
  team.brank = int(blockIdx.x);
  team.nblocks = int(gridDim.x);
  team.bar = a.bar;
  team.partials = a.partials;
  team.err = a.err;
  team.nph = 0;
  set_block_share(team, threadIdx.x - H * (BS / 2), BS / 2, 1 + H);
  if (H == 1 && a.lead != nullptr) {
    if (team.btid == 0) {
      unsigned spins = 0;
      while (ld_relaxed64(a.lead) < a.lead_count && ++spins < (1u << 20)) {
      }
    }
    team_sync(team);
  }
  mixed_solve<NC, 1, W, CM>(a, team, sh, ms);
}

// CM: the U(1) model's two complex systems (NC = 2), as cg_mixed_kernel's CM.
template <int NC, int BS, int W, bool CM = false>
__global__ void __launch_bounds__(BS, 1) cg_mixed_duo_kernel(MixedArgs a0, MixedArgs a1) {
  static_assert(BS % 64 == 0, "each half holds whole warps");
  __shared__ SyncShared sh[2];
  __shared__ MixedShared ms[2];
  if (threadIdx.x < BS / 2) duo_half<NC, BS, W, 0, CM>(a0, sh[0], ms[0]);
  else duo_half<NC, BS, W, 1, CM>(a1, sh[1], ms[1]);
}

}  // namespace gn
