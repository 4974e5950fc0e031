// selftest.cu -- failure-detection self-test of the bounded device waits.
//
// Every wait of the library's kernels on other blocks (the grid and team
// barriers of phase_sync.cuh) gives up after a bounded number of polls, sets
// the error word and returns, and the host reports GN_ERR_TIMEOUT with the
// context still usable.  This self-test makes such a wait run out on purpose
// without any fault: one block runs the barrier of a team of two blocks whose
// second block is never launched, so the arrival count never completes.
#include "engine.h"
#include "errors.h"
#include "phase_sync.cuh"

namespace gn {

// One block, the first of a team of two: its team_barrier waits for a block
// that does not exist, gives up after its poll limit and sets *err.
__global__ void selftest_timeout_kernel(PhaseBar *bar, int *err) {
  __shared__ SyncShared sh;
  Team t;
  t.tid = threadIdx.x;
  t.nthreads = blockDim.x;
  t.brank = 0;
  t.nblocks = 2;
  t.bar = bar;
  t.partials = nullptr;
  t.err = err;
  t.nph = 0;
  whole_block(t);
  team_barrier(sh, t);
}

int Engine::selftest_wait_timeout() {
  check(cudaMemsetAsync(bar_, 0, sizeof(PhaseBar), stream_), "memset");
  check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  selftest_timeout_kernel<<<1, 32, 0, stream_>>>(bar_, err_);
  check(cudaGetLastError(), "selftest_timeout_kernel");
  launches++;
  int h_err = 0;
  check(cudaMemcpyAsync(&h_err, err_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "selftest sync");
  // leave the barrier state as every solve expects to find it
  check(cudaMemsetAsync(bar_, 0, sizeof(PhaseBar), stream_), "memset");
  check(cudaMemsetAsync(err_, 0, sizeof(int), stream_), "memset");
  check(cudaStreamSynchronize(stream_), "selftest sync");
  if (h_err != 1) throw GnError(GN_ERR_CUDA, "self-test: the barrier did not report its timeout");
  return GN_ERR_TIMEOUT;
}

}  // namespace gn
