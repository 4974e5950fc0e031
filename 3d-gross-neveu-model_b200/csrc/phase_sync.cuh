// phase_sync.cuh -- end-of-phase synchronisation of the persistent solvers:
// every block's partial sums are reduced, the grid waits until every block has
// finished the phase, and every block gets the grid totals.
//
// Costs measured on B200 that shaped it: a block reduction of 8 doubles with
// three block barriers took 1.1 us, a __threadfence 0.4 us, and every block
// arriving on the barrier word adds about 8 ns (arrivals serialise on one
// address).  So: only the quantities a phase needs are reduced, with one block
// barrier; the grid barrier is a 64-bit monotonic arrival counter written with
// red.release, polled with relaxed loads and followed by one acquire fence;
// and the solvers run few, large blocks.  Every order is fixed, so all blocks
// compute the same totals bit for bit.  The barrier and the totals are two
// calls, so that a solver can start the next phase's stencil loads before it
// reads the other blocks' partial sums.
#pragma once
#include "device_common.cuh"

namespace gn {

constexpr int kSyncQ = 8;  // largest number of quantities reduced at one phase end

// Monotonic arrival counter: phase n is complete when it reaches
// (n+1) * gridDim.x.  (Spreading arrivals over several counters polled by
// several lanes was measured slower: every acquire load is a fence.)
struct PhaseBar {
  unsigned long long arrived;
  unsigned long long pad[15];
};

__device__ __forceinline__ void red_release_add64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_int(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

struct SyncShared {
  double red[32 * kSyncQ];  // per-warp sums
  double val[kSyncQ];       // grid totals of the last phase
  int ok;
  int flag;                 // block 0's flag word of the last phase
};

// A team: the blocks that sweep one lattice together and synchronise among
// themselves -- the whole grid of a single-lattice solve, or a group of
// blocks of the batched kernel.  A one-block team needs no global memory.
//
// A block normally gives all its threads to one team.  It can also hold two
// teams side by side (cg_mixed_duo_kernel): each then owns a contiguous,
// warp-aligned share of the block's threads and synchronises that share with
// a named barrier of its own, so the two teams never wait for each other.
struct Team {
  uint32_t tid;       // thread index within the team
  uint32_t nthreads;  // threads in the team
  int brank;          // this block's index within the team
  int nblocks;        // blocks in the team
  PhaseBar *bar;      // arrival counter (nblocks > 1)
  double *partials;   // [2][kSyncQ + 1][nblocks] partial sums (nblocks > 1)
  int *err;           // set to 1 by a wait that timed out
  unsigned long long nph;  // phases ended so far (the same count in every block of the team)
  uint32_t btid;      // thread index within this block's share of the team
  uint32_t bsize;     // threads of this block in the team (a multiple of 32)
  int bid;            // named barrier of that share: 0 = the whole block (__syncthreads)
};

// The team's threads in this block: the whole block, or a share of it given
// by (btid, bsize, bid).
__device__ __forceinline__ void set_block_share(Team &t, uint32_t btid, uint32_t bsize, int bid) {
  t.btid = btid;
  t.bsize = bsize;
  t.bid = bid;
}
__device__ __forceinline__ void whole_block(Team &t) { set_block_share(t, threadIdx.x, blockDim.x, 0); }

// Barrier of the team's threads in this block.
__device__ __forceinline__ void team_sync(const Team &t) {
  if (t.bid == 0) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(t.bid), "r"(t.bsize) : "memory");
}

// The whole grid as one team.
__device__ __forceinline__ Team grid_team(PhaseBar *bar, double *partials, int *err) {
  Team t;
  t.tid = blockIdx.x * blockDim.x + threadIdx.x;
  t.nthreads = gridDim.x * blockDim.x;
  t.brank = int(blockIdx.x);
  t.nblocks = int(gridDim.x);
  t.bar = bar;
  t.partials = partials;
  t.err = err;
  t.nph = 0;
  whole_block(t);
  return t;
}

// End of the team's next phase, first half: publishes this block's partial
// sums of NQ quantities (acc[]) and the flag word, and waits until every block
// of the team has done the same.  The team's writes of the phase are visible
// to this block on return.  Returns false if this block's wait timed out (it
// then sets *err; the other blocks time out at their next wait).  Slots
// alternate between two banks: [NQ][nblocks] partials, then one flag word.
template <int NQ>
__device__ __forceinline__ bool phase_arrive_wait(double (&acc)[kSyncQ], SyncShared &sh, const Team &t,
                                                  int flag = 0) {
  const int lane = t.btid & 31, w = t.btid >> 5, nw = t.bsize >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) sh.red[q * 32 + w] = v;
  }
  team_sync(t);
  if (w == 0) {
    double tot[NQ > 0 ? NQ : 1];
#pragma unroll
    for (int q = 0; q < NQ; q++) tot[q] = warp_sum(lane < nw ? sh.red[q * 32 + lane] : 0.0);
    if (lane == 0) {
      if (t.nblocks == 1) {  // the block is the team: its sums are the totals
#pragma unroll
        for (int q = 0; q < NQ; q++) sh.val[q] = tot[q];
        sh.flag = flag;
        sh.ok = 1;
      } else {
        double *slot = t.partials + (t.nph & 1ull) * size_t(kSyncQ + 1) * t.nblocks;
#pragma unroll
        for (int q = 0; q < NQ; q++) slot[size_t(q) * t.nblocks + t.brank] = tot[q];
        if (t.brank == 0) reinterpret_cast<int *>(slot + size_t(NQ) * t.nblocks)[0] = flag;
        // arrive (release: the block's writes of this phase, ordered before by
        // the block barrier, become visible with it), poll with relaxed loads,
        // and acquire once the count is complete
        red_release_add64(&t.bar->arrived, 1ull);
        const unsigned long long target = (t.nph + 1ull) * t.nblocks;
        unsigned spins = 0;
        int ok = 1;
        while (ld_relaxed64(&t.bar->arrived) < target) {
          if (++spins > (1u << 22)) {  // ~ a second: give up, report, return
            atomicExch(t.err, 1);
            ok = 0;
            break;
          }
        }
        fence_acquire();
        sh.ok = ok;
      }
    }
  }
  team_sync(t);
  return sh.ok != 0;
}

// Second half: the team totals into sh.val[0..NQ) and the flag word of the
// team's block 0 into sh.flag, summed by every block in the same order (so
// every block holds the same bits).  Advances the team's phase count.
template <int NQ>
__device__ __forceinline__ void phase_totals(SyncShared &sh, Team &t) {
  if (t.nblocks > 1) {
    const double *slot = t.partials + (t.nph & 1ull) * size_t(kSyncQ + 1) * t.nblocks;
    const int lane = t.btid & 31, w = t.btid >> 5;
    if (w < NQ) {
      const double *p = slot + size_t(w) * t.nblocks;
      double s = 0.0;
      for (int b = lane; b < t.nblocks; b += 32) s += p[b];
      s = warp_sum(s);
      if (lane == 0) sh.val[w] = s;
    } else if (t.btid == t.bsize - 1) {
      sh.flag = reinterpret_cast<const int *>(slot + size_t(NQ) * t.nblocks)[0];
    }
    team_sync(t);
  }
  t.nph++;
}

// Both halves: on return sh.val[0..NQ) holds the team totals in every block
// and sh.flag the word the team's block 0 put in `flag`.
template <int NQ>
__device__ __forceinline__ bool end_phase(double (&acc)[kSyncQ], SyncShared &sh, Team &t, int flag = 0) {
  const bool ok = phase_arrive_wait<NQ>(acc, sh, t, flag);
  phase_totals<NQ>(sh, t);
  return ok;
}

// A team barrier without sums: on return the team's writes before the call
// are visible to this block.  About 1.5 us on B200 for a grid of 64 - 148
// blocks of 1024 threads, against 3.2 - 3.7 us for an end_phase with sums
// (the block and team reductions and the read of the partials are what it
// saves); 0.28 us for a one-block team.  Counts as one phase of the team.
__device__ __forceinline__ bool team_barrier(SyncShared &sh, Team &t) {
  team_sync(t);
  if (t.btid == 0) {
    int ok = 1;
    if (t.nblocks > 1) {
      red_release_add64(&t.bar->arrived, 1ull);
      const unsigned long long target = (t.nph + 1ull) * t.nblocks;
      unsigned spins = 0;
      while (ld_relaxed64(&t.bar->arrived) < target) {
        if (++spins > (1u << 22)) {  // ~ a second: give up, report, return
          atomicExch(t.err, 1);
          ok = 0;
          break;
        }
      }
      fence_acquire();
    }
    sh.ok = ok;
  }
  t.nph++;
  team_sync(t);
  return sh.ok != 0;
}

}  // namespace gn
