// launch.h -- cooperative launches of the persistent solvers and the rule that
// sizes their grid.  Shared by every entry point so that a solve gets the same
// grid, hence the same summation order, whichever entry point launched it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "cg_kernel.cuh"
#include "rowvec.cuh"

namespace gn {

// Threads per block of the solvers: one large block per SM (launch bounds
// (BS, 1)), because every block arriving at a grid barrier costs about 8 ns
// (measured).  The hot shapes (one real plane, up to two systems: the two
// pseudofermion flavours) use 1024 threads (64 registers), so that a sweep of
// the mixed solver at L = 64 gives every thread one work unit; the rarely
// used shapes 512 (up to 128 registers).
constexpr int kWideThreads = 1024;
constexpr int kSolverThreads = 512;

// Instantiated solver kernels: (planes, RHS slots) = (1, 1), (1, 2), (1, 4), (2, 1), (2, 2).
inline int rhs_slots(int nrhs) { return nrhs <= 1 ? 1 : (nrhs <= 2 ? 2 : 4); }
inline int threads_for(int ncomp, int nrhs) { return (ncomp == 1 && nrhs <= 2) ? kWideThreads : kSolverThreads; }

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Sites per item of the FP64 sweeps (rowvec.cuh): 2, with 16-byte loads, when
// L/2 is even and every array the caller passed is 16-byte aligned; else 1.
inline int fp64_width(int L, const void *const *ptrs, int n) {
  if (row_width(L, 2) != 2) return 1;
  for (int i = 0; i < n; i++)
    if (ptrs[i] != nullptr && !aligned16(ptrs[i])) return 1;
  return 2;
}

// Largest co-resident grid (in blocks) for `fn` launched with bs threads; 0 on error.
inline int coop_capacity(const void *fn, int bs) {
  int dev = 0, per_sm = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bs, 0) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return per_sm * sms;
}

// Work units of a sweep: (system, item) pairs, items of w sites.
inline int64_t solver_units(int64_t V, int w, int nrhs) { return int64_t(nrhs) * (V / w); }

// Grid of a solve with `units` work units: one unit per thread at most, within
// the co-resident capacity and cap_blocks.
inline int solver_grid(int64_t units, int capacity, int cap_blocks, int bs) {
  int64_t want = (units + bs - 1) / bs;
  int64_t cap = capacity < cap_blocks ? capacity : cap_blocks;
  return int(want < cap ? want : cap);
}

// Cooperative launch of a persistent solver taking one argument struct.
template <typename Args>
inline cudaError_t launch_solver(const void *fn, int nblocks, int bs, Args &a, cudaStream_t st) {
  void *args[] = {(void *)&a};
  return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(bs), args, 0, st);
}

}  // namespace gn
