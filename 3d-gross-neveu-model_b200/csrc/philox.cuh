// philox.cuh -- counter-based random numbers for the batched chains:
// Philox4x64-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11), restated from the paper.
//
// One call maps a 256-bit counter and a 128-bit key to 256 random bits, with
// no state: every (chain, trajectory, field, site block) has its own counter,
// so any thread can draw any site's numbers in any order and every chain's
// stream is independent of how many chains run beside it.  The block function
// equals numpy.random.Philox's (its counter is incremented before the first
// block; tests/test_philox.py pins the two against each other).
//
// Host and device: the same code, so the host tests check the device's bits.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define GN_PHX_HD __host__ __device__ __forceinline__
#else
#define GN_PHX_HD static inline
#endif

namespace gn {

struct Philox4x64 {
  uint64_t v[4];
};

GN_PHX_HD void phx_mulhilo(uint64_t a, uint64_t b, uint64_t &hi, uint64_t &lo) {
#if defined(__CUDA_ARCH__)
  hi = __umul64hi(a, b);
  lo = a * b;
#else
  const unsigned __int128 p = (unsigned __int128)a * b;
  hi = uint64_t(p >> 64);
  lo = uint64_t(p);
#endif
}

// Ten rounds of the Philox S-P network with the paper's 4x64 constants.
GN_PHX_HD Philox4x64 philox4x64(Philox4x64 c, uint64_t k0, uint64_t k1) {
  const uint64_t M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
  const uint64_t W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t hi0, lo0, hi1, lo1;
    phx_mulhilo(M0, c.v[0], hi0, lo0);
    phx_mulhilo(M1, c.v[2], hi1, lo1);
    Philox4x64 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Uniform double in (0, 1] from 53 random bits (never 0: Box-Muller takes its log).
GN_PHX_HD double phx_unit_open0(uint64_t x) { return double((x >> 11) + 1ull) * (1.0 / 9007199254740992.0); }
// Uniform double in [0, 1).
GN_PHX_HD double phx_unit(uint64_t x) { return double(x >> 11) * (1.0 / 9007199254740992.0); }

// Streams of one chain: what a counter's words mean.
// (Trajectory draws take the chain's trajectory number as the counter word;
// a served request's own draws take its serial number: a solve's right-hand
// side, and Z2 noise vector n at kPhxZ2 + n.)
enum PhxField : uint64_t {
  kPhxMomenta = 0,
  kPhxChi0 = 1,
  kPhxChi1 = 2,
  kPhxMetropolis = 3,
  kPhxRhs = 4,
  kPhxZ2 = 16
};

// Four random words for (field, block) of trajectory `traj` of the chain with
// key (seed, chain).
GN_PHX_HD Philox4x64 phx_draw(uint64_t seed, uint64_t chain, uint64_t traj, uint64_t field, uint64_t block) {
  Philox4x64 c;
  c.v[0] = block;
  c.v[1] = field;
  c.v[2] = traj;
  c.v[3] = 0;
  return philox4x64(c, seed, chain);
}

}  // namespace gn

#undef GN_PHX_HD
