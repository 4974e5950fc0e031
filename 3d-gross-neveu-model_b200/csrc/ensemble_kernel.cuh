// ensemble_kernel.cuh -- many independent sigma-HMC chains of mixed lattice
// sizes in one persistent kernel per slice of a trajectory.
//
// A launch runs one slice of the trajectory's op list (an MD step, or the
// refresh / initial solve / energy at either end) for every chain.  Chains
// come in tiers, each taken from its own work queue, largest first: a tier's
// chains run on teams of that tier's size, groups of blocks that synchronise
// with a team barrier (phase_sync.cuh); the last tier's on single blocks that
// need only __syncthreads.  Tier sizes divide each other (e.g. 16, 4, 1), so a
// block's team in a later tier lies inside its team of the earlier one and no
// block waits on a block outside its current team.  Every chain's
// work is a fixed sequence of team phases, so every block of a team takes the
// same branches.  Momenta, pseudofermion sources and the Metropolis uniform
// come from the chain's own Philox stream (philox.cuh) with the trajectory
// number as the counter, so a chain's results do not depend on the chains
// beside it or on which team ran it (for a fixed team size).
#pragma once
#include <cstdlib>
#include "../../include/gn_b200.h"
#include "mixed_kernel.cuh"
#include "ops_kernels.cuh"
#include "philox.cuh"

namespace gn {

constexpr int kEnsThreads = 1024;
constexpr int kMaxTiers = 4;

// Ops of the batched trajectory (the schedule of schedule.h, translated).
enum EnsOpCode : int {
  E_REFRESH = 1,  // save sigma; P, chi_0, chi_1 ~ N(0, 1) from the chain's stream
  E_PHI,          // phi_f = M chi_f
  E_SOLVE,        // X_f = (M M^T)^-1 phi_f, both flavours, mixed precision
  E_FORCE,        // Y_f = M^T X_f; F = sigma force; P += c F
  E_P,            // P += c F
  E_Q,            // sigma += c P, sm recomputed
  E_ENERGY0,      // H0
  E_ENERGY1,      // H1
  E_METROPOLIS,   // accept if u <= exp(-(H1 - H0)), else restore sigma; statistics
  E_RHS,          // phi_0 ~ N(0, 1), phi_1 = 0 (a solve request's right-hand side)
  E_Z2,           // phi_0, phi_1 = Z2 noise vectors 2c, 2c+1 of the request
  E_TRACE         // Y_f = M^T X_f; result += sum_f phi_f . Y_f / V (condensate estimate)
};

struct EnsOp {
  int code;
  double c;
};

struct EnsState;

// One chain's arrays (device pointers, 256-byte aligned) and constants.
struct EnsChain {
  struct EnsState *state;     // the chain's mutable state
  int op_begin, op_end;       // the chain's own op range (used when the launch gives none)
  Geom g;
  int w;  // sites per FP32 item (4, 2 or 1); the FP64 sweeps use min(w, 2)
  double beta_s;
  unsigned long long stream;  // Philox key word of the chain
  double *sigma[2];           // current / other (ping-pong of the sigma steps)
  double *sm, *P, *F, *sigma_save;
  double *chi, *phi, *X, *Y;  // two flavour planes each
  double *t64;                // solver FP64 scratch, two planes
  float *sm32, *rh, *ph, *uh, *ah, *xh;  // solver FP32 vectors, two planes each
  double *r64, *pa64, *pb64;  // FP64 solver vectors (with t64), two planes each
  int precision;              // GN_PREC_MIXED or GN_PREC_FP64
};

// One chain's mutable state (device).
struct EnsState {
  int cur;     // which sigma buffer is current
  int failed;  // a solve of the current trajectory did not converge
  double H0, H1;
  long long ntraj;  // trajectories done: the Philox counter of the next one
  // accumulated since the last reset
  long long n, nacc, iters, reliable, fails;
  double sum_dH, sum_exp_mdH, sum_sigma2, last_dH;
  double sum_obs[kSigmaObs];  // CondensateSigmaPi outputs after each trajectory
  int last_acc;
  // HMC bookkeeping of the reference's struct Info (moleculardynamics.c:1385-1416)
  long long total_acc;  // hybrid_accepted_sigma (total_acc of ntraj trajectories)
  int story;            // story_sigma: +n after n accepts in a row, -n after n rejects
  int local_acc, local_done;
  int autoreg;          // UpdateHMCParameters (info.c:123-135) after every trajectory
  double eps_scale;     // the chain's epsilon / the launch's (0 stands for 1)
  // the current request of a served chain
  unsigned long long serial;  // Philox counter of the request's draws
  double result;              // E_TRACE accumulator
};

struct EnsLaunch {
  const EnsChain *chains;
  int nchains;
  const int *order;  // chain indices, tier by tier
  int ntier;
  int tier_gs[kMaxTiers];   // blocks per team of tier t (decreasing; each divides the previous)
  int tier_end[kMaxTiers];  // tier t runs order[tier_end[t-1] .. tier_end[t])
  const EnsOp *ops;
  int op_begin, op_end;  // op range of every chain; op_begin < 0: each chain's own
  int *queue;         // [kMaxTiers] next task of each tier; zero before the launch
  PhaseBar *bars;     // [kMaxTiers][gridDim.x] team barrier counters; zero before the launch
  double *partials;   // [kMaxTiers][gridDim.x][2][kSyncQ + 1]
  double *partials2;  // the same again, for the second flavour of a two-team solve
  int duo;            // solve the two flavours as two teams of half blocks
  CgState *cg_state;  // [gridDim.x][kMaxRhs] solver status scratch
  int *err;
  unsigned long long seed;
  double tol;     // relative tolerance of every solve
  double delta;   // reliable-update threshold
  int n_ru;       // reliable update at least every n_ru iterations
};

// Sweep of (plane, item) units of W sites over the team: M or M^T of two planes.
template <int W, int OP>
__device__ __forceinline__ void team_dirac2(const Geom &g, const Team &t, const double *sm, const double *in,
                                            double *out) {
  const uint32_t NI = row_items<W>(g), V = uint32_t(g.V);
  for (uint32_t u = t.tid; u < 2u * NI; u += t.nthreads) {
    const uint32_t f = u >= NI ? 1u : 0u, j = u - f * NI;
    const RowItem it = make_item<W>(g, j);
    Nb<double> n[W];
    double smv[W], o[W];
    gather_item<double, W>(it, in + size_t(f) * V, n);
    vload<double, W>(sm + it.own, smv);
    if (OP == 0) item_M<double, W>(it, smv, n, o);
    else item_Mt<double, W>(it, smv, n, o);
    vstore<double, W>(out + size_t(f) * V + it.own, o);
  }
}

// The solvers of one chain, one function per item width (each gets its own
// register allocation instead of sharing the caller's).  The argument structs
// live in shared memory, written by one thread of the block: read through a
// reference to the caller's stack, every access of the sweeps was a
// local-memory load (ncu: more local than global load requests in this
// kernel).
template <int W>
__device__ __noinline__ void ens_solve(const MixedArgs &a, Team &t, SyncShared &sh, MixedShared &ms) {
  mixed_solve<1, 2, W>(a, t, sh, ms);
}
template <int W>
__device__ __noinline__ void ens_solve64(const CgArgs<double> &a, Team &t, SyncShared &sh, CgShared &cs) {
  cg_solve<double, 1, 2, W>(a, t, sh, cs);
}
template <int W>
__device__ __noinline__ void ens_solve_half(const MixedArgs &a, Team &t, SyncShared &sh, MixedShared &ms) {
  mixed_solve<1, 1, W>(a, t, sh, ms);
}

// The second flavour's team state of a two-team solve: its own arrival
// counter and partial sums (the first flavour uses the team's), and its phase
// count, kept from one solve of the launch to the next.
struct DuoSync {
  PhaseBar *bar;
  double *partials;
  unsigned long long nph;
};

// Shared memory of a chain's solves: the argument structs and the two half
// teams' state.
struct DuoShared {
  SyncShared sh[2];
  MixedShared ms[2];
  unsigned long long nph[2];
  MixedArgs args[2];  // the solve (args[0]), or one flavour per half team
  CgArgs<double> args64;
};

// Both flavours of a mixed-precision solve as two teams of half blocks, as in
// cg_mixed_duo_kernel: flavour h runs on the threads [h B/2, (h+1) B/2) of
// every block of the team, with named barrier 1 + h, so one flavour's phase
// ends overlap the other's sweeps; on a team of several blocks flavour 1
// starts half an iteration behind.  ds.args[h] holds flavour h's solve
// (nrhs = 1, sm32 already formed by the whole team).  On return every thread
// of the team holds both phase counts.  Measured on the 256-chain benchmark
// mix: 372 chain trajectories/s against 336 in lock step (without the offset).
__device__ __forceinline__ void ens_duo_solve(int w, Team &t, DuoSync &d, DuoShared &ds) {
  const uint32_t half = blockDim.x / 2;
  const int h = threadIdx.x >= half ? 1 : 0;
  Team ht = t;
  ht.tid = uint32_t(t.brank) * half + (threadIdx.x - h * half);
  ht.nthreads = uint32_t(t.nblocks) * half;
  set_block_share(ht, threadIdx.x - h * half, half, 1 + h);
  if (h) {
    ht.bar = d.bar;
    ht.partials = d.partials;
    ht.nph = d.nph;
  }
  if (h == 1 && t.nblocks > 1) {
    // start half an iteration behind flavour 0: after its first phase end on
    // the team's counter (a bounded wait; only a matter of timing)
    if (ht.btid == 0) {
      const unsigned long long target = (t.nph + 1ull) * t.nblocks;
      unsigned spins = 0;
      while (ld_relaxed64(&t.bar->arrived) < target && ++spins < (1u << 20)) {
      }
    }
    team_sync(ht);
  }
  if (w == 4) ens_solve_half<4>(ds.args[h], ht, ds.sh[h], ds.ms[h]);
  else if (w == 2) ens_solve_half<2>(ds.args[h], ht, ds.sh[h], ds.ms[h]);
  else ens_solve_half<1>(ds.args[h], ht, ds.sh[h], ds.ms[h]);
  if (ht.btid == 0) ds.nph[h] = ht.nph;
  __syncthreads();  // the whole block again
  t.nph = ds.nph[0];
  d.nph = ds.nph[1];
}

// Box-Muller on two uniforms: two N(0, 1) values.
__device__ __forceinline__ void box_muller(uint64_t a, uint64_t b, double &z0, double &z1) {
  const double r = sqrt(-2.0 * log(phx_unit_open0(a)));
  double s, c;
  sincospi(2.0 * phx_unit(b), &s, &c);
  z0 = r * c;
  z1 = r * s;
}

// The factor of the chain's own step size on the launch's step coefficients.
__device__ __forceinline__ double eps_scale(const EnsState *st) { return st->eps_scale > 0.0 ? st->eps_scale : 1.0; }

// The chain's ops [op_begin, op_end) by team t.  Returns false on a barrier timeout.
static __device__ __noinline__ bool ens_run_chain(const EnsLaunch &L, int c, Team &t, SyncShared &sh, MixedShared &ms,
                                                  CgShared &cs, DuoSync &duo, DuoShared &ds) {
  const EnsChain &ch = L.chains[c];
  EnsState *st = ch.state;
  const int op_begin = L.op_begin >= 0 ? L.op_begin : ch.op_begin;
  const int op_end = L.op_begin >= 0 ? L.op_end : ch.op_end;
  const Geom g = ch.g;
  const uint32_t V = uint32_t(g.V);
  const bool leader = t.brank == 0 && threadIdx.x == 0;
  int cur = st->cur;  // every thread tracks the ping-pong index itself
  double acc[kSyncQ];
  auto zero_acc = [&]() {
#pragma unroll
    for (int q = 0; q < kSyncQ; q++) acc[q] = 0.0;
  };
  for (int o = op_begin; o < op_end; o++) {
    const EnsOp op = L.ops[o];
    double *const sig = ch.sigma[cur];
    double *const sig_o = ch.sigma[cur ^ 1];
    zero_acc();
    bool ok = true;
    if (op.code == E_REFRESH) {
      const unsigned long long traj = (unsigned long long)st->ntraj;
      for (uint32_t i = t.tid; i < V; i += t.nthreads) ch.sigma_save[i] = sig[i];
      // four sites per Philox block: P, chi_0, chi_1
      for (uint32_t u = t.tid; u < 3u * (V / 4u); u += t.nthreads) {
        const uint32_t f = u / (V / 4u), q = u - f * (V / 4u);
        const Philox4x64 r = phx_draw(L.seed, ch.stream, traj, f, q);
        double z[4];
        box_muller(r.v[0], r.v[1], z[0], z[1]);
        box_muller(r.v[2], r.v[3], z[2], z[3]);
        double *dst = f == 0 ? ch.P : ch.chi + size_t(f - 1) * V;
#pragma unroll
        for (int e = 0; e < 4; e++) dst[4 * q + e] = z[e];
      }
      if (leader) st->failed = 0;
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_PHI) {
      if (ch.w >= 2) team_dirac2<2, 0>(g, t, ch.sm, ch.chi, ch.phi);
      else team_dirac2<1, 0>(g, t, ch.sm, ch.chi, ch.phi);
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_SOLVE) {
      const int nrhs = op.c > 0.0 ? int(op.c) : 2;
      const int *status;
      const long long *iters;
      const bool two = ch.precision != GN_PREC_FP64 && L.duo && nrhs == 2;
      if (ch.precision == GN_PREC_FP64) {
        CgArgs<double> &a = ds.args64;
        if (threadIdx.x == 0) {
          a.g = g;
          a.sm = ch.sm;
          for (int k = 0; k < kMaxRhs; k++) {
            const size_t off = size_t(k < 2 ? k : 1) * V;
            a.b[k] = ch.phi + off;
            a.x[k] = ch.X + off;
            a.r[k] = ch.r64 + off;
            a.p0[k] = ch.pa64 + off;
            a.p1[k] = ch.pb64 + off;
            a.t[k] = ch.t64 + off;
          }
          a.nrhs = nrhs;
          a.variant = 1;
          a.rel = 1;
          a.tol = L.tol;
          a.max_iter = (long long)V + 1;
          a.partials = nullptr;
          a.bar = nullptr;
          a.err = t.err;
          a.abort_flag = nullptr;
          a.state = L.cg_state + size_t(blockIdx.x) * kMaxRhs;
        }
        __syncthreads();
        if (ch.w >= 2) ens_solve64<2>(a, t, sh, cs);
        else ens_solve64<1>(a, t, sh, cs);
        status = cs.status;
        iters = cs.iters;
      } else {
        if (two) {  // sm32 by the whole team, then one flavour per half of every block
          for (uint32_t i = t.tid; i < V; i += t.nthreads) ch.sm32[i] = float(ch.sm[i]);
          ok = end_phase<0>(acc, sh, t);
        }
        if (threadIdx.x == 0) {
          MixedArgs &a = ds.args[0];
          a.g = g;
          a.sm = ch.sm;
          a.sm32 = ch.sm32;
          a.pm = nullptr;
          a.pm32 = nullptr;
          for (int k = 0; k < kMaxRhs; k++) {
            const size_t off = size_t(k < 2 ? k : 1) * V;
            a.b[k] = ch.phi + off;
            a.x[k] = ch.X + off;
            a.t64[k] = ch.t64 + off;
            a.rh[k] = ch.rh + off;
            a.ph[k] = ch.ph + off;
            a.uh[k] = ch.uh + off;
            a.ah[k] = ch.ah + off;
            a.xh[k] = ch.xh + off;
          }
          a.nrhs = nrhs;
          a.variant = 1;
          a.rel = 1;
          a.scheme = mixed_scheme(g.V, nrhs, 1);
          a.sm32_ready = two ? 1 : 0;
          a.lead = nullptr;
          a.lead_count = 0;
          a.tol = L.tol;
          a.max_iter = (long long)V + 1;
          a.delta = L.delta;
          a.n_ru = L.n_ru;
          a.partials = nullptr;
          a.bar = nullptr;
          a.err = t.err;
          a.abort_flag = nullptr;
          a.state = L.cg_state + size_t(blockIdx.x) * kMaxRhs;
          if (two) {  // flavour 1 in args[1], flavour 0 alone in args[0]
            MixedArgs &a1 = ds.args[1];
            a1 = a;
            a1.b[0] = a.b[1];
            a1.x[0] = a.x[1];
            a1.t64[0] = a.t64[1];
            a1.rh[0] = a.rh[1];
            a1.ph[0] = a.ph[1];
            a1.uh[0] = a.uh[1];
            a1.ah[0] = a.ah[1];
            a1.xh[0] = a.xh[1];
            a1.state = a.state + 1;
            a.nrhs = a1.nrhs = 1;
          }
        }
        __syncthreads();
        if (two) {
          if (ok) ens_duo_solve(ch.w, t, duo, ds);
        } else {
          if (ch.w == 4) ens_solve<4>(ds.args[0], t, sh, ms);
          else if (ch.w == 2) ens_solve<2>(ds.args[0], t, sh, ms);
          else ens_solve<1>(ds.args[0], t, sh, ms);
        }
        status = ms.status;
        iters = ms.iters;
      }
      if (leader) {
        for (int k = 0; k < nrhs; k++) {
          const int s = two ? ds.ms[k].status[0] : status[k];
          if (s != kCgConverged && s != kCgConvergedStart) st->failed = 1;
          st->iters += (s == kCgConverged) ? (two ? ds.ms[k].iters[0] : iters[k]) : 0;
          if (ch.precision != GN_PREC_FP64) st->reliable += two ? ds.ms[k].nru[0] : ms.nru[k];
        }
      }
      ok = ok && ld_relaxed_int(t.err) == 0;
    } else if (op.code == E_FORCE) {
      if (ch.w >= 2) team_dirac2<2, 1>(g, t, ch.sm, ch.X, ch.Y);
      else team_dirac2<1, 1>(g, t, ch.sm, ch.X, ch.Y);
      ok = end_phase<0>(acc, sh, t);
      const double gcoef = (4 * ch.beta_s / 2.0);  // (NFLAV * beta_scalar / 2.0), moleculardynamics.c:580
      const double pc = op.c * eps_scale(st);
      for (uint32_t i = t.tid; i < V && ok; i += t.nthreads)
        force_site<double, false>(g, i, ch.X, ch.Y, sig, gcoef, ch.F, ch.P, pc);
      ok = end_phase<0>(acc, sh, t) && ok;
    } else if (op.code == E_P) {
      const double pc = op.c * eps_scale(st);
      for (uint32_t i = t.tid; i < V; i += t.nthreads) ch.P[i] = ch.P[i] + ch.F[i] * pc;
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_Q) {
      const double qc = op.c * eps_scale(st);
      for (uint32_t i = t.tid; i < V; i += t.nthreads)
        sigma_mass_site<double, false>(g, i, sig, ch.P, qc, sig_o, ch.sm);
      cur ^= 1;
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_ENERGY0 || op.code == E_ENERGY1) {
      // ComputeFullEnergyForSigma, moleculardynamics.c:299-319
      for (uint32_t i = t.tid; i < V; i += t.nthreads) {
        const double p = ch.P[i];
        acc[0] += p * p / 2.0;
        acc[1] += 0.5 * (ch.phi[i] * ch.X[i]) + 0.5 * (ch.phi[V + i] * ch.X[V + i]);
        acc[2] += sig[i] * sig[i];
      }
      ok = end_phase<3>(acc, sh, t);
      const double h = (sh.val[0] + sh.val[1]) + (4 * ch.beta_s / 4.0) * sh.val[2];
      if (leader) {
        if (op.code == E_ENERGY0) st->H0 = h;
        else st->H1 = h;
      }
      ok = end_phase<0>(acc, sh, t) && ok;  // H stored before anyone reads it
    } else if (op.code == E_METROPOLIS) {
      const double dH = st->H1 - st->H0;
      const Philox4x64 r = phx_draw(L.seed, ch.stream, (unsigned long long)st->ntraj, kPhxMetropolis, 0);
      const int failed = st->failed;
      const int accept = !failed && (phx_unit(r.v[0]) <= exp(-dH));
      if (!accept) {  // restore sigma and its mass (moleculardynamics.c:1404-1416)
        for (uint32_t i = t.tid; i < V; i += t.nthreads)
          sigma_mass_site<double, false>(g, i, ch.sigma_save, (const double *)nullptr, 0.0, sig_o, ch.sm);
        cur ^= 1;
      }
      ok = end_phase<0>(acc, sh, t);
      // sum sigma^2 and the CondensateSigmaPi sums of the chain's sigma
      const double *fin = ch.sigma[cur];
      for (uint32_t i = t.tid; i < V; i += t.nthreads) {
        double v[kSigmaObsSums];
        sigma_obs_site(g, i, fin, v);
        acc[0] += fin[i] * fin[i];
#pragma unroll
        for (int q = 0; q < kSigmaObsSums; q++) acc[1 + q] += v[q];
      }
      ok = end_phase<1 + kSigmaObsSums>(acc, sh, t) && ok;
      if (leader) {
        double sums[kSigmaObsSums], o[kSigmaObs];
        for (int q = 0; q < kSigmaObsSums; q++) sums[q] = sh.val[1 + q];
        sigma_obs_finish(sums, double(V), o);
        for (int q = 0; q < kSigmaObs; q++) st->sum_obs[q] += o[q];
        st->n++;
        st->nacc += accept;
        st->fails += failed;
        st->sum_dH += dH;
        st->sum_exp_mdH += exp(-dH);
        st->sum_sigma2 += sh.val[0] / double(V);
        st->last_dH = dH;
        st->last_acc = accept;
        st->ntraj++;
        // acceptance bookkeeping and epsilon autoregulation (a failed solve
        // counts as a reject here; the reference exits instead)
        st->total_acc += accept;
        st->local_acc += accept;
        st->local_done++;
        if (accept) st->story = st->story >= 0 ? st->story + 1 : -1;
        else st->story = st->story >= 0 ? -1 : st->story - 1;
        if (st->autoreg && st->local_done == 100) {
          const double a = double(st->local_acc) / double(st->local_done);
          double sc = eps_scale(st);
          if (a >= 0.85) sc = sc * 1.15;
          else if (a >= 0.8) sc = sc * 1.08;
          else if (a >= 0.75) sc = sc / 1.08;
          else sc = sc / 1.15;
          st->eps_scale = sc;
          st->local_acc = 0;
          st->local_done = 0;
        }
      }
    } else if (op.code == E_RHS) {
      const unsigned long long serial = st->serial;
      for (uint32_t q = t.tid; q < V / 4u; q += t.nthreads) {
        const Philox4x64 r = phx_draw(L.seed, ch.stream, serial, kPhxRhs, q);
        double z[4];
        box_muller(r.v[0], r.v[1], z[0], z[1]);
        box_muller(r.v[2], r.v[3], z[2], z[3]);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          ch.phi[4 * q + e] = z[e];
          ch.phi[V + 4 * q + e] = 0.0;
        }
      }
      if (leader) st->failed = 0;
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_Z2) {
      // one Philox block gives the signs of 256 sites: noise vector n, block q
      const unsigned long long serial = st->serial;
      const int n0 = 2 * int(op.c);
      for (uint32_t u = t.tid; u < 2u * V; u += t.nthreads) {
        const uint32_t f = u >= V ? 1u : 0u, i = u - f * V;
        const Philox4x64 r = phx_draw(L.seed, ch.stream, serial, kPhxZ2 + uint64_t(n0 + int(f)), i >> 8);
        const uint64_t bits = r.v[(i >> 6) & 3u];
        ch.phi[u] = ((bits >> (i & 63u)) & 1ull) ? 1.0 : -1.0;
      }
      if (leader) st->failed = 0;
      ok = end_phase<0>(acc, sh, t);
    } else if (op.code == E_TRACE) {
      // tr M^{-1} estimate of condensate.c:142-145 for two real noise vectors:
      // xi . M^T (M M^T)^-1 xi / V
      if (ch.w >= 2) team_dirac2<2, 1>(g, t, ch.sm, ch.X, ch.Y);
      else team_dirac2<1, 1>(g, t, ch.sm, ch.X, ch.Y);
      ok = end_phase<0>(acc, sh, t);
      for (uint32_t u = t.tid; u < 2u * V; u += t.nthreads) acc[0] += ch.phi[u] * ch.Y[u];
      ok = end_phase<1>(acc, sh, t) && ok;
      if (leader) st->result += sh.val[0] / double(V);
    }
    if (!ok) return false;
  }
  // every block of the team has passed the last barrier (after reading st->cur)
  if (leader) st->cur = cur;
  return true;
}

// Whether the batched kernel solves the two flavours as two teams of half
// blocks (default), or in lock step on the whole team (GN_ENS_DUO=0).
inline int ens_duo_enabled() {
  const char *e = getenv("GN_ENS_DUO");
  return (e != nullptr && e[0] == '0') ? 0 : 1;
}

// Defined in one translation unit (ensemble.cu, which sets
// GN_DEFINE_ENSEMBLE_KERNEL); the others launch it through this declaration.
__global__ void __launch_bounds__(kEnsThreads, 1) ens_node_kernel(EnsLaunch L);

#ifdef GN_DEFINE_ENSEMBLE_KERNEL
__global__ void __launch_bounds__(kEnsThreads, 1) ens_node_kernel(EnsLaunch L) {
  __shared__ SyncShared sh;
  __shared__ MixedShared ms;
  __shared__ CgShared cs;
  __shared__ DuoShared ds;
  __shared__ int s_task;
  int tb = 0;  // first order index of the tier
  for (int tier = 0; tier < L.ntier; tier++) {
    const int gs = L.tier_gs[tier], te = L.tier_end[tier];
    if (gs > 1) {
      // teams of gs blocks; blocks beyond the last whole team go straight on
      const int group = int(blockIdx.x) / gs, grank = int(blockIdx.x) % gs;
      if (group < int(gridDim.x) / gs && te > tb) {
        Team gt;
        gt.tid = uint32_t(grank) * blockDim.x + threadIdx.x;
        gt.nthreads = uint32_t(gs) * blockDim.x;
        gt.brank = grank;
        gt.nblocks = gs;
        gt.bar = L.bars + size_t(tier) * gridDim.x + group;
        gt.partials = L.partials + (size_t(tier) * gridDim.x + size_t(group) * gs) * 2 * (kSyncQ + 1);
        gt.err = L.err;
        gt.nph = 0;
        whole_block(gt);
        // the second flavour's counter: past the tier's gridDim.x / gs team counters
        DuoSync duo{L.bars + size_t(tier) * gridDim.x + gridDim.x / gs + group,
                    L.partials2 + (size_t(tier) * gridDim.x + size_t(group) * gs) * 2 * (kSyncQ + 1), 0ull};
        for (;;) {
          int task = 0;
          if (grank == 0 && threadIdx.x == 0) task = tb + atomicAdd(&L.queue[tier], 1);
          double acc[kSyncQ];
#pragma unroll
          for (int q = 0; q < kSyncQ; q++) acc[q] = 0.0;
          if (!end_phase<0>(acc, sh, gt, task)) return;  // the team leader's task, to every block
          task = sh.flag;
          if (task >= te) break;
          if (!ens_run_chain(L, L.order[task], gt, sh, ms, cs, duo, ds)) return;
        }
      }
    } else {
      Team bt;
      bt.tid = threadIdx.x;
      bt.nthreads = blockDim.x;
      bt.brank = 0;
      bt.nblocks = 1;
      bt.bar = nullptr;
      bt.partials = nullptr;
      bt.err = L.err;
      bt.nph = 0;
      whole_block(bt);
      DuoSync duo{nullptr, nullptr, 0ull};  // one-block teams need no counters
      for (;;) {
        if (threadIdx.x == 0) s_task = tb + atomicAdd(&L.queue[tier], 1);
        __syncthreads();
        const int task = s_task;
        __syncthreads();
        if (task >= te) break;
        if (!ens_run_chain(L, L.order[task], bt, sh, ms, cs, duo, ds)) return;
      }
    }
    tb = te;
  }
}
#endif

}  // namespace gn
