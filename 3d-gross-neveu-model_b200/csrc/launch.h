// launch.h -- cooperative launches of the persistent solvers and the rule that
// sizes their grid.  Shared by every entry point so that a solve gets the same
// grid, hence the same summation order, whichever entry point launched it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "cg_kernel.cuh"

namespace gn {

// Threads per block of the solvers: one large block per SM (launch bounds
// (BS, 1)), because every block arriving at a grid barrier costs about 8 ns
// (measured).  Two shapes are built: 512 threads (up to 128 registers) and 768
// (80 registers).  solver_threads() picks one for every entry point alike: the
// environment variable GN_SOLVER_THREADS (512 or 768, for tuning sweeps) or
// else kDefaultSolverThreads, the shape measured fastest at every L from 8 to
// 128 (bench.py --case cgscan).
constexpr int kDefaultSolverThreads = 768;
constexpr int kSolverThreads = 512;  // shape of the rarely used instantiations

inline int solver_threads() {
  static const int bs = [] {
    const char *e = getenv("GN_SOLVER_THREADS");
    const int v = e ? atoi(e) : kDefaultSolverThreads;
    return (v == 512 || v == 768) ? v : kDefaultSolverThreads;
  }();
  return bs;
}

// Largest co-resident grid (in blocks) for `fn` launched with bs threads; 0 on error.
inline int coop_capacity(const void *fn, int bs) {
  int dev = 0, per_sm = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bs, 0) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return per_sm * sms;
}

// Grid of a solve over V sites: one site per thread at most, within the
// co-resident capacity and cap_blocks.
inline int solver_grid(int64_t V, int capacity, int cap_blocks, int bs) {
  int64_t want = (V + bs - 1) / bs;
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
