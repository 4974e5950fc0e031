// noalloc.cu -- a CG solve on (M M^T) x = b that allocates no memory.
//
// Who needs it: callers that must not allocate device memory once they are
// running.  An HMC driver written like the reference sizes every buffer once,
// from the lattice size, in its Allocate* functions, and owns all of its
// device memory from then on; an application that hands this library a fixed
// budget from its own pool allocator cannot have it call cudaMalloc behind
// the pool's back, where the allocation would escape the budget, or fail
// when the pool has taken the rest of the GPU.  gn_create() needs cudaMalloc
// for its per-lattice buffers; this entry point does not.
//
// The solver's scratch (residual, two search directions, M^T p, the per-block
// partial sums and the grid barrier) lives in the file-scope array below,
// sized for lattices up to kNoAllocMaxL^3 sites (about 1 MiB).  Every GPU that
// loads the library holds it until the process exits.  All calls share it:
// calls that overlap on the GPU race on it, and so do calls from several host
// threads even on one stream, because one call's read-back of its outcome can
// pick up another call's.  Serialise whole calls on the host (one thread at a
// time, or a lock around the call).  The array keeps the last call's contents;
// what must start at zero (barrier counter, error flag, outcome) is cleared by
// every call.
//
// Set-up: the host cannot use the array's name as a device address (in host
// code it is only a stand-in).  The first call on each device, with that
// device current, asks cudaGetSymbolAddress for the address and the occupancy
// API for the cooperative grid size and caches both; that first call should
// come before any stream capture.  Later calls only clear the control words,
// launch the kernel and read the outcome back.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/gn_b200.h"
#include "launch.h"

namespace {

using gn::CgArgs;
using gn::CgState;
using gn::PhaseBar;

constexpr int kNoAllocMaxL = 32;
constexpr size_t kMaxV = size_t(kNoAllocMaxL) * kNoAllocMaxL * kNoAllocMaxL;  // 32768 sites
constexpr int kMaxBlocks = int((kMaxV + 511) / 512);  // one site per thread at most (blocks of >= 512 threads)
// the same solver instantiations, block shape and grid rule as gn_cg_device
// for one real system; w = sites per item (1 or 2)
constexpr int kThreads = gn::kWideThreads;
inline const void *solver_kernel(int w) {
  return w == 2 ? (const void *)gn::cg_kernel<double, 1, 1, kThreads, 2>
                : (const void *)gn::cg_kernel<double, 1, 1, kThreads, 1>;
}
constexpr size_t kVecWords = 4 * kMaxV;                                         // r, p0, p1, t
constexpr size_t kPartialWords = size_t(2 * (gn::kSyncQ + 1)) * kMaxBlocks;      // 2 slots x (8 sums + flag) per block
constexpr size_t kBarWords = sizeof(gn::PhaseBar) / sizeof(double);
constexpr size_t kControlWords = kBarWords + 8;                                 // barrier, error flag, state
constexpr size_t kScratchWords = kVecWords + kPartialWords + kControlWords;

static __device__ __align__(256) double g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
struct DeviceSetup {
  double *scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int capacity[2] = {0, 0};  // co-resident blocks of the solver kernel, 1 and 2 sites per item
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

thread_local char g_msg[256];

int err(int status, const char *msg) {
  strncpy(g_msg, msg, sizeof g_msg - 1);
  return status;
}

}  // namespace

extern "C" GN_API const char *gn_cg_noalloc_error(void) { return g_msg; }

extern "C" GN_API long long gn_cg_noalloc_max_volume(void) { return (long long)kMaxV; }

extern "C" GN_API int gn_cg_noalloc(int L, const double *sigmamass, const double *b, double *x, double tol, int variant,
                                    int relative, long long max_iter, void *stream, gn_cg_info *info) {
  g_msg[0] = '\0';  // a message describes the failure of the last call only
  if (L < 4 || (L & 1)) return err(GN_ERR_ARG, "gn_cg_noalloc: L must be even and >= 4");
  if (L > kNoAllocMaxL)
    return err(GN_ERR_ARG, "gn_cg_noalloc: L exceeds the static scratch limit of 32 (32768 sites); use gn_cg_device");
  if (!sigmamass || !b || !x) return err(GN_ERR_ARG, "gn_cg_noalloc: null pointer");
  if (b == x) return err(GN_ERR_ARG, "gn_cg_noalloc: b and x must not alias");
  if (variant < 0 || variant > 1) return err(GN_ERR_ARG, "gn_cg_noalloc: variant must be 0 or 1");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return err(GN_ERR_NO_DEVICE, "gn_cg_noalloc: no current CUDA device");
  const gn::Geom g = gn::make_geom(L);
  const size_t V = size_t(g.V);
  if (max_iter <= 0) max_iter = (long long)V + 1;  // MAX_CONJUGATE_GRADIENT_ITERATION, macro.h:134

  // ---- once per device: the scratch address and the cooperative grid size
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &s = g_setup[dev];
    if (s.scratch == nullptr) {
      cudaDeviceProp prop;
      if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10)
        return err(GN_ERR_NO_DEVICE, "gn_cg_noalloc: this library is built for sm_100a (B200) only");
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) return err(GN_ERR_CUDA, "gn_cg_noalloc: cudaGetSymbolAddress failed");
      for (int w = 1; w <= 2; w++) {
        const int capacity = gn::coop_capacity(solver_kernel(w), kThreads);
        if (capacity < 1) return err(GN_ERR_CUDA, "gn_cg_noalloc: occupancy query failed");
        s.capacity[w - 1] = capacity;
      }
      s.scratch = static_cast<double *>(p);
    }
  }
  const DeviceSetup &s = g_setup[dev];
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // ---- carve the static array
  double *base = s.scratch;
  double *vec = base;
  double *partials = base + kVecWords;
  double *control = base + kVecWords + kPartialWords;
  PhaseBar *bar = reinterpret_cast<PhaseBar *>(control);
  int *errflag = reinterpret_cast<int *>(control + kBarWords);
  CgState *state = reinterpret_cast<CgState *>(control + kBarWords + 2);
  if (cudaMemsetAsync(control, 0, kControlWords * sizeof(double), st) != cudaSuccess)
    return err(GN_ERR_CUDA, "gn_cg_noalloc: clearing the control words failed");

  CgArgs<double> a;
  memset(&a, 0, sizeof a);
  a.g = g;
  a.sm = sigmamass;
  a.b[0] = b;
  a.x[0] = x;
  a.r[0] = vec;
  a.p0[0] = vec + V;
  a.p1[0] = vec + 2 * V;
  a.t[0] = vec + 3 * V;
  a.nrhs = 1;
  a.variant = variant;
  a.rel = relative;
  a.tol = tol;
  a.max_iter = max_iter;
  a.partials = partials;
  a.bar = bar;
  a.err = errflag;
  a.abort_flag = nullptr;
  a.state = state;
  const void *ptrs[3] = {sigmamass, b, x};
  const int w = gn::fp64_width(L, ptrs, 3);
  const int nb = gn::solver_grid(gn::solver_units(int64_t(V), w, 1), s.capacity[w - 1], kMaxBlocks, kThreads);
  if (gn::launch_solver(solver_kernel(w), nb, kThreads, a, st) != cudaSuccess)
    return err(GN_ERR_CUDA, "gn_cg_noalloc: kernel launch failed");

  // ---- outcome (into host stack memory; no allocation)
  CgState h_state;
  int h_err = 0;
  if (cudaMemcpyAsync(&h_state, state, sizeof h_state, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&h_err, errflag, sizeof h_err, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return err(GN_ERR_CUDA, "gn_cg_noalloc: reading the outcome failed");
  if (h_err == 1) return err(GN_ERR_TIMEOUT, "gn_cg_noalloc: grid barrier timed out");
  if (info) {
    info->status = h_state.status;
    info->counted = h_state.status == gn::kCgConverged;
    info->iterations = h_state.iters;
    info->residual = std::sqrt(h_state.r2);
    info->b_norm = std::sqrt(h_state.b2);
    info->inner_iterations = h_state.iters;
    info->reliable_updates = 0;
  }
  if (h_state.status == gn::kCgConverged || h_state.status == gn::kCgConvergedStart) return GN_OK;
  return GN_NOT_CONVERGED;
}
