// geometry.cuh -- site indexing of the L^3 staggered lattice, computed from
// coordinates on the device (no neighbour or phase tables are stored).
//
// Layout (the reference's "fermion lexicographic" order, coordinate.c:25-40 and
// :301-313): lexicographic n = (x0*L + x1)*L + x2 with x2 = time fastest; the
// fermion index of a site is n/2 + parity*V/2, parity = (x0+x1+x2) % 2, so the
// even sites come first.  For even L this is an even/odd checkerboard in which
// each parity half is a sequence of "rows" (x0, x1) of L/2 sites along time:
//     h = (x0*L + x1)*(L/2) + k,     x2 = 2k + ((parity + x0 + x1) & 1).
// The x0 and x1 neighbours of a site therefore sit at the same k in an
// adjacent row of the other parity half (coalesced), and the two time
// neighbours are at k or k +- 1 in the same row.
//
// Staggered phases (coordinate.c:133-200): eta_0 = 1, eta_1 = (-1)^x0,
// eta_2 = (-1)^(x0+x1); with antiperiodic time the forward phase eta_pp(x, 2)
// flips sign at x2 = L-1 and the backward phase eta_mm(x, 2) at x2 = 0.
#pragma once
#include <cstdint>

namespace gn {

// Exact division by a small constant via one 64-bit multiply: q = (n*m) >> 36,
// m = ceil(2^36 / d).  Exact for n * d < 2^36, i.e. for every index used here
// (n < 2^27, d <= 512).
struct FastDiv {
  uint64_t m;
  uint32_t d;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  f.m = ((uint64_t(1) << 36) + d - 1) / d;
  return f;
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  return uint32_t((uint64_t(n) * f.m) >> 36);
}

// Lattice constants passed by value to every kernel.
struct Geom {
  int L;         // spatial and temporal extent (even)
  int Lh;        // L / 2
  int64_t V;     // L^3
  int64_t half;  // V / 2
  int plane;     // L * Lh: sites of one parity in an x0-slice
  FastDiv div_Lh, div_L;
};

inline Geom make_geom(int L) {
  Geom g;
  g.L = L;
  g.Lh = L / 2;
  g.V = int64_t(L) * L * L;
  g.half = g.V / 2;
  g.plane = L * (L / 2);
  g.div_Lh = make_fastdiv(uint32_t(L / 2));
  g.div_L = make_fastdiv(uint32_t(L));
  return g;
}

// Everything the stencils need about one site.
struct Site {
  uint32_t x0, x1, x2, par;
  uint32_t qbase;             // first index of the opposite parity half
  uint32_t nb_up[3], nb_dn[3];  // fermion indices of x + mu, x - mu
  float eta_up[3], eta_dn[3];   // +-1: eta_pp(x, mu), eta_mm(x, mu)
};

__host__ __device__ __forceinline__ void site_coords(const Geom &g, uint32_t i, uint32_t &x0, uint32_t &x1, uint32_t &x2,
                                            uint32_t &par, uint32_t &row, uint32_t &k) {
  par = i >= uint32_t(g.half) ? 1u : 0u;
  uint32_t h = i - par * uint32_t(g.half);
  row = fdiv(h, g.div_Lh);
  k = h - row * uint32_t(g.Lh);
  x0 = fdiv(row, g.div_L);
  x1 = row - x0 * uint32_t(g.L);
  x2 = 2u * k + ((par + x0 + x1) & 1u);
}

__host__ __device__ __forceinline__ Site make_site(const Geom &g, uint32_t i) {
  Site s;
  uint32_t row, k;
  site_coords(g, i, s.x0, s.x1, s.x2, s.par, row, k);
  const uint32_t L = uint32_t(g.L), Lh = uint32_t(g.Lh);
  s.qbase = (1u - s.par) * uint32_t(g.half);
  // x0 +- 1
  const uint32_t x0u = (s.x0 + 1u == L) ? 0u : s.x0 + 1u;
  const uint32_t x0d = (s.x0 == 0u) ? L - 1u : s.x0 - 1u;
  const uint32_t x1u = (s.x1 + 1u == L) ? 0u : s.x1 + 1u;
  const uint32_t x1d = (s.x1 == 0u) ? L - 1u : s.x1 - 1u;
  const uint32_t x2u = (s.x2 + 1u == L) ? 0u : s.x2 + 1u;
  const uint32_t x2d = (s.x2 == 0u) ? L - 1u : s.x2 - 1u;
  s.nb_up[0] = s.qbase + (x0u * L + s.x1) * Lh + k;
  s.nb_dn[0] = s.qbase + (x0d * L + s.x1) * Lh + k;
  s.nb_up[1] = s.qbase + (s.x0 * L + x1u) * Lh + k;
  s.nb_dn[1] = s.qbase + (s.x0 * L + x1d) * Lh + k;
  s.nb_up[2] = s.qbase + row * Lh + (x2u >> 1);
  s.nb_dn[2] = s.qbase + row * Lh + (x2d >> 1);
  const float e1 = (s.x0 & 1u) ? -1.f : 1.f;
  const float e2 = ((s.x0 + s.x1) & 1u) ? -1.f : 1.f;
  s.eta_up[0] = 1.f;
  s.eta_dn[0] = 1.f;
  s.eta_up[1] = e1;
  s.eta_dn[1] = e1;
  s.eta_up[2] = (s.x2 == L - 1u) ? -e2 : e2;
  s.eta_dn[2] = (s.x2 == 0u) ? -e2 : e2;
  return s;
}

// Fermion index of the site at lattice coordinates (any values mod L).
__host__ __device__ __forceinline__ uint32_t site_index(const Geom &g, int c0, int c1, int c2) {
  const int L = g.L;
  c0 = (c0 % L + L) % L;
  c1 = (c1 % L + L) % L;
  c2 = (c2 % L + L) % L;
  const uint32_t par = uint32_t(c0 + c1 + c2) & 1u;
  return par * uint32_t(g.half) + (uint32_t(c0) * L + uint32_t(c1)) * uint32_t(g.Lh) + uint32_t(c2 >> 1);
}

}  // namespace gn
