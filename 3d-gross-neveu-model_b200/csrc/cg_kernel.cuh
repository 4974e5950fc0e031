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
// two pseudofermion flavours share every barrier), each with its own alpha,
// beta and stopping test, exactly as separate solves.
//
// Per iteration, two phases (12 words of traffic per site and RHS):
//   A: p <- r + beta p (on the fly at the 7 stencil points), t = M^T p, sum t^2
//   B: x += alpha p, r -= alpha M t, sum r^2 ; stop when sqrt(sum r^2) < tol
// The update formulas and their rounding follow the reference (x += a p,
// r += (-a) Ap, p = r + b p; no FMA in the FP64 build); only the order of the
// global sums differs (tree instead of serial).
//
// A sweep's work unit is one (system, row item) pair (rowvec.cuh; items of
// W = 2 sites with 128-bit loads when L/2 is even), one unit per thread where
// the grid allows: the systems' loads are then all in flight at once instead
// of one system after the other, and a phase is one latency round.
#pragma once
#include "phase_sync.cuh"
#include "rowvec.cuh"

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
  const T *pm;  // U(1) model: the pi mass of the complex diagonal (CM solves only)
  int nrhs;
  int variant;  // 0: test the incoming x first (START_X0_NULL form); 1: x = 0
  int rel;      // 0: stop at |r| < tol; 1: stop at |r| < tol |b|
  double tol;
  long long max_iter;
  double *partials;  // [2 banks][kSyncQ + 1][gridDim.x]
  PhaseBar *bar;
  int *err;
  const int *abort_flag;  // host-mapped; nonzero asks the kernel to stop
  CgState *state;         // [kMaxRhs]
};

// ------------------------------------------------------------------ work units
// The systems a sweep covers (block-shared, the same in every block).
struct SysList {
  int n;
  int k[kMaxRhs];
};

// Rebuilds the list from a per-system flag (thread 0; the caller synchronises).
__device__ __forceinline__ void sys_list_from(SysList &sl, const int *flag, int nrhs) {
  int n = 0;
  for (int k = 0; k < nrhs; k++)
    if (flag[k]) sl.k[n++] = k;
  sl.n = n;
}

// f(k, j) for every (system k of the list, item j < NI), spread over the
// team's threads: the items of one system are contiguous in the unit
// numbering, so a warp reads contiguous vectors of one system.
template <typename F>
__device__ __forceinline__ void for_units(uint32_t NI, const SysList &sl, const Team &t, F f) {
  // the team's indices in registers: when the team is held in memory (a solver
  // called with a reference to its caller's), the stores of f() could alias it
  // and would make every step of the loop reload them
  const uint32_t tid = t.tid, nthreads = t.nthreads;
  const uint32_t total = uint32_t(sl.n) * NI;
  for (uint32_t u = tid; u < total; u += nthreads) {
    uint32_t j = u;
    int ka = 0;
    while (j >= NI) {
      j -= NI;
      ka++;
    }
    f(sl.k[ka], j);
  }
}

// Per-system selections without dynamic indexing (which would move the
// kernel's argument arrays and the accumulators to local memory).
template <int NR, typename P>
__device__ __forceinline__ P pick(const P (&arr)[kMaxRhs], int k) {
  P p = arr[0];
#pragma unroll
  for (int q = 1; q < NR; q++)
    if (q == k) p = arr[q];
  return p;
}
template <int NR>
__device__ __forceinline__ void acc_add(double (&acc)[2 * kMaxRhs], int slot, double v) {
#pragma unroll
  for (int q = 0; q < 2 * NR; q++)
    if (q == slot) acc[q] += v;
}

// Block-shared state of one FP64 solve (the same values in every block of the team).
struct CgShared {
  double alpha[kMaxRhs], beta[kMaxRhs], rr[kMaxRhs], tau[kMaxRhs], r2[kMaxRhs], b2[kMaxRhs];
  int active[kMaxRhs], status[kMaxRhs], all[kMaxRhs];
  long long iters[kMaxRhs];
  SysList run, every;  // systems still iterating / all systems
};

// One solve by a team (all its threads call it; a.bar, a.partials and a.err
// are not used: the team's own are).  NR: right-hand-side slots unrolled
// (>= nrhs); W: sites per item (divides L/2).
//
// CM (NC = 2): the U(1) model's complex mass sm + i eps pm (rowvec.cuh), the
// two planes of a system coupled through it; the CG formulas are the same,
// with the global sums running over both planes (the real form of the
// reference's complex CG).
template <typename T, int NC, int NR, int W, bool CM = false>
__device__ __forceinline__ void cg_solve(const CgArgs<T> &a, Team &team, SyncShared &sh, CgShared &cs) {
  double *const s_val = sh.val;
  double *const s_alpha = cs.alpha, *const s_beta = cs.beta, *const s_rr = cs.rr, *const s_tau = cs.tau;
  double *const s_r2 = cs.r2, *const s_b2 = cs.b2;
  int *const s_active = cs.active, *const s_status = cs.status, *const s_all = cs.all;
  long long *const s_iters = cs.iters;
  SysList &s_run = cs.run, &s_every = cs.every;

  const Geom g = a.g;
  const uint32_t V = uint32_t(g.V);
  const uint32_t NI = row_items<W>(g);
  const T *__restrict__ sm = a.sm;
  static_assert(!CM || NC == 2, "the complex mass couples the two planes of a system");

  if (threadIdx.x < kMaxRhs) {
    const int k = threadIdx.x;
    s_active[k] = k < a.nrhs;
    s_all[k] = k < a.nrhs;
    s_status[k] = k < a.nrhs ? kCgRunning : kCgConverged;
    s_iters[k] = 0;
    s_alpha[k] = s_beta[k] = s_rr[k] = s_r2[k] = s_b2[k] = 0.0;
    s_tau[k] = a.tol;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sys_list_from(s_every, s_all, a.nrhs);
    sys_list_from(s_run, s_active, a.nrhs);
  }
  __syncthreads();
  bool ok = true;
  double acc[2 * kMaxRhs];
  auto zero_acc = [&]() {
#pragma unroll
    for (int q = 0; q < 2 * kMaxRhs; q++) acc[q] = 0.0;
  };

  // ---------------------------------------------------------------- start
  if (a.variant == 0) {
    // t = M^T x_in
    for_units(NI, s_every, team, [&](int k, uint32_t j) {
      const RowItem it = make_item<W>(g, j);
      T smi[W];
      vload<T, W>(sm + it.own, smi);
      const T *xk = pick<NR>(a.x, k);
      T *tk = pick<NR>(a.t, k);
      if constexpr (CM) {
        Nb<T> nr[W], ni[W];
        T b[W], o_r[W], o_i[W];
        gather_item<T, W>(it, xk, nr);
        gather_item<T, W>(it, xk + V, ni);
        item_eps_pm<T, W>(g, it, a.pm, b);
        item_Mt_cm<T, W>(it, smi, b, nr, ni, o_r, o_i);
        vstore<T, W>(tk + it.own, o_r);
        vstore<T, W>(tk + V + it.own, o_i);
      } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
          Nb<T> n[W];
          T o[W];
          gather_item<T, W>(it, xk + size_t(c) * V, n);
          item_Mt<T, W>(it, smi, n, o);
          vstore<T, W>(tk + size_t(c) * V + it.own, o);
        }
      }
    });
    zero_acc();
    ok = end_phase<1>(acc, sh, team);
    // r = b - M t ; sums r^2 and b^2
    zero_acc();
    if (ok) {
      for_units(NI, s_every, team, [&](int k, uint32_t j) {
        const RowItem it = make_item<W>(g, j);
        T smi[W];
        vload<T, W>(sm + it.own, smi);
        const T *tk = pick<NR>(a.t, k);
        const T *bk = pick<NR>(a.b, k);
        T *rk = pick<NR>(a.r, k);
        if constexpr (CM) {
          Nb<T> nr[W], ni[W];
          T b[W], br[W], bim[W], rr[W], rim[W];
          gather_item<T, W>(it, tk, nr);
          gather_item<T, W>(it, tk + V, ni);
          item_eps_pm<T, W>(g, it, a.pm, b);
          vload<T, W>(bk + it.own, br);
          vload<T, W>(bk + V + it.own, bim);
#pragma unroll
          for (int e = 0; e < W; e++) {
            rr[e] = br[e];
            rim[e] = bim[e];
          }
          item_sub_M_cm<T, W>(it, smi, b, nr, ni, rr, rim);
          vstore<T, W>(rk + it.own, rr);
          vstore<T, W>(rk + V + it.own, rim);
          double sr = 0.0, sb = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            sr += double(rr[e]) * double(rr[e]) + double(rim[e]) * double(rim[e]);
            sb += double(br[e]) * double(br[e]) + double(bim[e]) * double(bim[e]);
          }
          acc_add<NR>(acc, k, sr);
          acc_add<NR>(acc, NR + k, sb);
        } else {
#pragma unroll
          for (int c = 0; c < NC; c++) {
            const size_t off = size_t(c) * V + it.own;
            Nb<T> n[W];
            T bi[W], ri[W];
            gather_item<T, W>(it, tk + size_t(c) * V, n);
            vload<T, W>(bk + off, bi);
#pragma unroll
            for (int e = 0; e < W; e++) ri[e] = bi[e];
            item_sub_M<T, W>(it, smi, n, ri);
            vstore<T, W>(rk + off, ri);
            double sr = 0.0, sb = 0.0;
#pragma unroll
            for (int e = 0; e < W; e++) {
              sr += double(ri[e]) * double(ri[e]);
              sb += double(bi[e]) * double(bi[e]);
            }
            acc_add<NR>(acc, k, sr);
            acc_add<NR>(acc, NR + k, sb);
          }
        }
      });
    }
    ok = end_phase<2 * NR>(acc, sh, team) && ok;
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
    if (threadIdx.x == 0) sys_list_from(s_run, s_active, a.nrhs);
    __syncthreads();
  }
  // x = 0, r = b, p = b ; rr = sum b^2
  zero_acc();
  if (ok) {
    for_units(NI, s_run, team, [&](int k, uint32_t j) {
      const uint32_t own = make_item<W>(g, j).own;
      const T *bk = pick<NR>(a.b, k);
      T *xk = pick<NR>(a.x, k);
      T *rk = pick<NR>(a.r, k);
      T *pk = pick<NR>(a.p0, k);
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const size_t off = size_t(c) * V + own;
        T bi[W], zero[W];
        vload<T, W>(bk + off, bi);
        double sb = 0.0;
#pragma unroll
        for (int e = 0; e < W; e++) {
          zero[e] = T(0);
          sb += double(bi[e]) * double(bi[e]);
        }
        acc_add<NR>(acc, k, sb);
        vstore<T, W>(xk + off, zero);
        vstore<T, W>(rk + off, bi);
        vstore<T, W>(pk + off, bi);
      }
    });
  }
  ok = end_phase<NR>(acc, sh, team) && ok;
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
  if (threadIdx.x == 0) sys_list_from(s_run, s_active, a.nrhs);
  __syncthreads();

  // ---------------------------------------------------------------- iterations
  long long it = 0;
  for (; ok && it < a.max_iter; it++) {
    if (s_run.n == 0) break;
    // the host's abort request lives in mapped host memory: one thread reads it
    // every 16 iterations, and the value is only used at the end of phase B
    int abort_req = 0;
    if (team.brank == 0 && threadIdx.x == 0 && a.abort_flag != nullptr && (it & 15) == 0)
      abort_req = *(volatile const int *)a.abort_flag;
    const bool odd = (it & 1) != 0;
    // phase A: p = r + beta p_old (it > 0), t = M^T p, sum t^2
    zero_acc();
    for_units(NI, s_run, team, [&](int k, uint32_t j) {
      const RowItem ri = make_item<W>(g, j);
      T smi[W];
      vload<T, W>(sm + ri.own, smi);
      const T beta = T(s_beta[k]);
      T *const pn = odd ? pick<NR>(a.p1, k) : pick<NR>(a.p0, k);
      const T *const po = odd ? pick<NR>(a.p0, k) : pick<NR>(a.p1, k);
      const T *rk = pick<NR>(a.r, k);
      T *tk = pick<NR>(a.t, k);
      if constexpr (CM) {
        Nb<T> n[2][W];
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const size_t off = size_t(c) * V;
          if (it == 0) {
            gather_item<T, W>(ri, pn + off, n[c]);
          } else {
            const T *rv = rk + off;
            const T *pov = po + off;
            gather_item<T, W>(
                ri, n[c],
                [&](uint32_t i, T(&v)[W]) {
                  T rr[W], pp[W];
                  vload<T, W>(rv + i, rr);
                  vload<T, W>(pov + i, pp);
#pragma unroll
                  for (int e = 0; e < W; e++) v[e] = rr[e] + beta * pp[e];
                },
                [&](uint32_t i) { return rv[i] + beta * pov[i]; });
            T pc[W];
#pragma unroll
            for (int e = 0; e < W; e++) pc[e] = n[c][e].c;
            vstore<T, W>(pn + off + ri.own, pc);
          }
        }
        T b[W], t_r[W], t_i[W];
        item_eps_pm<T, W>(g, ri, a.pm, b);
        item_Mt_cm<T, W>(ri, smi, b, n[0], n[1], t_r, t_i);
        vstore<T, W>(tk + ri.own, t_r);
        vstore<T, W>(tk + V + ri.own, t_i);
        double st = 0.0;
#pragma unroll
        for (int e = 0; e < W; e++) st += double(t_r[e]) * double(t_r[e]) + double(t_i[e]) * double(t_i[e]);
        acc_add<NR>(acc, k, st);
      } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          Nb<T> n[W];
          if (it == 0) {
            gather_item<T, W>(ri, pn + off, n);
          } else {
            const T *rv = rk + off;
            const T *pov = po + off;
            gather_item<T, W>(
                ri, n,
                [&](uint32_t i, T(&v)[W]) {
                  T rr[W], pp[W];
                  vload<T, W>(rv + i, rr);
                  vload<T, W>(pov + i, pp);
#pragma unroll
                  for (int e = 0; e < W; e++) v[e] = rr[e] + beta * pp[e];
                },
                [&](uint32_t i) { return rv[i] + beta * pov[i]; });
            T pc[W];
#pragma unroll
            for (int e = 0; e < W; e++) pc[e] = n[e].c;
            vstore<T, W>(pn + off + ri.own, pc);
          }
          T ti[W];
          item_Mt<T, W>(ri, smi, n, ti);
          vstore<T, W>(tk + off + ri.own, ti);
          double st = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) st += double(ti[e]) * double(ti[e]);
          acc_add<NR>(acc, k, st);
        }
      }
    });
    ok = end_phase<NR>(acc, sh, team);
    if (!ok) break;
    if (threadIdx.x < kMaxRhs) {
      const int k = threadIdx.x;
      if (k < a.nrhs && s_active[k]) s_alpha[k] = s_rr[k] / s_val[k];
    }
    __syncthreads();
    // phase B: Ap = M t, x += alpha p, r -= alpha Ap, sum r^2
    zero_acc();
    for_units(NI, s_run, team, [&](int k, uint32_t j) {
      const RowItem ri = make_item<W>(g, j);
      T smi[W];
      vload<T, W>(sm + ri.own, smi);
      const T alpha = T(s_alpha[k]);
      const T malpha = -alpha;
      const T *const pn = odd ? pick<NR>(a.p1, k) : pick<NR>(a.p0, k);
      const T *tk = pick<NR>(a.t, k);
      T *xk = pick<NR>(a.x, k);
      T *rk = pick<NR>(a.r, k);
      if constexpr (CM) {
        Nb<T> nr[W], ni[W];
        T b[W], ap[2][W];
        gather_item<T, W>(ri, tk, nr);
        gather_item<T, W>(ri, tk + V, ni);
        item_eps_pm<T, W>(g, ri, a.pm, b);
        item_M_cm<T, W>(ri, smi, b, nr, ni, ap[0], ap[1]);
        double sr = 0.0;
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const size_t off = size_t(c) * V;
          T pv[W], xv[W], rv[W];
          vload<T, W>(pn + off + ri.own, pv);
          vload<T, W>(xk + off + ri.own, xv);
          vload<T, W>(rk + off + ri.own, rv);
#pragma unroll
          for (int e = 0; e < W; e++) {
            xv[e] = xv[e] + alpha * pv[e];
            rv[e] = rv[e] + malpha * ap[c][e];
            sr += double(rv[e]) * double(rv[e]);
          }
          vstore<T, W>(xk + off + ri.own, xv);
          vstore<T, W>(rk + off + ri.own, rv);
        }
        acc_add<NR>(acc, k, sr);
      } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
          const size_t off = size_t(c) * V;
          Nb<T> n[W];
          T ap[W], pv[W], xv[W], rv[W];
          gather_item<T, W>(ri, tk + off, n);
          vload<T, W>(pn + off + ri.own, pv);
          vload<T, W>(xk + off + ri.own, xv);
          vload<T, W>(rk + off + ri.own, rv);
          item_M<T, W>(ri, smi, n, ap);
          double sr = 0.0;
#pragma unroll
          for (int e = 0; e < W; e++) {
            xv[e] = xv[e] + alpha * pv[e];
            rv[e] = rv[e] + malpha * ap[e];
            sr += double(rv[e]) * double(rv[e]);
          }
          acc_add<NR>(acc, k, sr);
          vstore<T, W>(xk + off + ri.own, xv);
          vstore<T, W>(rk + off + ri.own, rv);
        }
      }
    });
    ok = end_phase<NR>(acc, sh, team, abort_req);
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
    __syncthreads();
    if (threadIdx.x == 0) sys_list_from(s_run, s_active, a.nrhs);
    __syncthreads();
    // host abort request: block 0's view decides for everyone at the next phase
    if (sh.flag != 0) {  // block 0 saw the host's abort request at the last phase end
      if (threadIdx.x == 0 && team.brank == 0) atomicExch(team.err, 2);
      ok = false;
      break;
    }
  }
  // ---------------------------------------------------------------- results
  if (team.brank == 0 && threadIdx.x < kMaxRhs) {
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

// The single-lattice solve: the whole cooperative grid is the team.
template <typename T, int NC, int NR, int BS, int W, bool CM = false>
__global__ void __launch_bounds__(BS, 1) cg_kernel(CgArgs<T> a) {
  __shared__ SyncShared sh;
  __shared__ CgShared cs;
  Team team = grid_team(a.bar, a.partials, a.err);
  cg_solve<T, NC, NR, W, CM>(a, team, sh, cs);
}

}  // namespace gn
