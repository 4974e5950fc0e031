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

// Exact division by a small constant d <= 512 for n < 2^24: a float
// reciprocal estimate (n is exact in float) corrected by one step, so the
// quotient is exact.
struct FastDiv {
  float inv;
  uint32_t d;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  f.inv = 1.0f / float(d);
  return f;
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  uint32_t q = uint32_t(float(n) * f.inv);
  const int32_t r = int32_t(n) - int32_t(q * f.d);
  if (r < 0) q--;
  else if (r >= int32_t(f.d)) q++;
  return q;
}

// Lattice constants passed by value to every kernel.
struct Geom {
  int L;         // spatial and temporal extent (even)
  int Lh;        // L / 2
  int64_t V;     // L^3
  int64_t half;  // V / 2
  int plane;     // L * Lh: sites of one parity in an x0-slice
  FastDiv div_Lh, div_L, div_Lq;  // division by L/2, L, L/4 (the last only for L % 4 == 0)
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
  g.div_Lq = make_fastdiv(uint32_t(L % 4 == 0 ? L / 4 : 1));
  return g;
}

// Everything the stencils need about one site.  The staggered phases are
// kept as sign bits: bit mu of neg set <=> eta_pp(x, mu) = -1, bit 3+mu set
// <=> eta_mm(x, mu) = -1.
struct Site {
  uint32_t x0, x1, x2, par;
  uint32_t nb_up[3], nb_dn[3];  // fermion indices of x + mu, x - mu
  uint32_t neg;
};

__host__ __device__ __forceinline__ void site_coords(const Geom &g, uint32_t i, uint32_t &x0, uint32_t &x1, uint32_t &x2,
                                                     uint32_t &par, uint32_t &row, uint32_t &k) {
  par = i >= uint32_t(g.half) ? 1u : 0u;
  const uint32_t h = i - par * uint32_t(g.half);
  row = fdiv(h, g.div_Lh);
  k = h - row * uint32_t(g.Lh);
  x0 = fdiv(row, g.div_L);
  x1 = row - x0 * uint32_t(g.L);
  x2 = 2u * k + ((par + x0 + x1) & 1u);
}

// Neighbours as offsets from the half index h = row*(L/2) + k: x0 +- 1 is a
// whole plane (L*L/2) away, x1 +- 1 one row (L/2), the time neighbours are at
// k or k +- 1 of the same row; each wraps periodically.
__host__ __device__ __forceinline__ Site make_site(const Geom &g, uint32_t i) {
  Site s;
  uint32_t row, k;
  site_coords(g, i, s.x0, s.x1, s.x2, s.par, row, k);
  const uint32_t L = uint32_t(g.L), Lh = uint32_t(g.Lh), P = uint32_t(g.plane);
  const uint32_t h = row * Lh + k;
  const uint32_t qb = (1u - s.par) * uint32_t(g.half);
  s.nb_up[0] = qb + ((s.x0 + 1u == L) ? h - (L - 1u) * P : h + P);
  s.nb_dn[0] = qb + ((s.x0 == 0u) ? h + (L - 1u) * P : h - P);
  s.nb_up[1] = qb + ((s.x1 + 1u == L) ? h - (L - 1u) * Lh : h + Lh);
  s.nb_dn[1] = qb + ((s.x1 == 0u) ? h + (L - 1u) * Lh : h - Lh);
  if ((s.x2 & 1u) == 0u) {  // x2 = 2k: x2+1 -> k, x2-1 -> k-1
    s.nb_up[2] = qb + h;
    s.nb_dn[2] = qb + ((k == 0u) ? h + Lh - 1u : h - 1u);
  } else {  // x2 = 2k+1: x2+1 -> k+1, x2-1 -> k
    s.nb_up[2] = qb + ((k + 1u == Lh) ? h + 1u - Lh : h + 1u);
    s.nb_dn[2] = qb + h;
  }
  const uint32_t e1 = s.x0 & 1u, e2 = (s.x0 + s.x1) & 1u;
  const uint32_t up2 = e2 ^ (s.x2 == L - 1u ? 1u : 0u);
  const uint32_t dn2 = e2 ^ (s.x2 == 0u ? 1u : 0u);
  s.neg = (e1 << 1) | (up2 << 2) | (e1 << 4) | (dn2 << 5);
  return s;
}

__host__ __device__ __forceinline__ float eta_up(const Site &s, int d) { return (s.neg >> d) & 1u ? -1.f : 1.f; }
__host__ __device__ __forceinline__ float eta_dn(const Site &s, int d) { return (s.neg >> (3 + d)) & 1u ? -1.f : 1.f; }

// Fermion index of the site at lattice coordinates (any values mod L).
__host__ __device__ __forceinline__ uint32_t site_index(const Geom &g, int c0, int c1, int c2) {
  const int L = g.L;
  c0 = (c0 % L + L) % L;
  c1 = (c1 % L + L) % L;
  c2 = (c2 % L + L) % L;
  const uint32_t par = uint32_t(c0 + c1 + c2) & 1u;
  return par * uint32_t(g.half) + (uint32_t(c0) * L + uint32_t(c1)) * uint32_t(g.Lh) + uint32_t(c2 >> 1);
}

// Index of the corner x + S*(d0, d1, d2) of a cube, d in {0, 1}^3 and S = +1
// or -1, for 0 <= x < L: each coordinate wraps with one compare instead of
// site_index's three divisions (the 8-corner gathers: the sigma mass takes
// S = -1, the sigma force S = +1).  Equal to site_index for these offsets.
template <int S>
__host__ __device__ __forceinline__ uint32_t corner_index(const Geom &g, uint32_t x0, uint32_t x1, uint32_t x2,
                                                          int d0, int d1, int d2) {
  const uint32_t L = uint32_t(g.L);
  auto step = [L](uint32_t x, int d) -> uint32_t {
    if (d == 0) return x;
    if constexpr (S > 0) return x + 1u == L ? 0u : x + 1u;
    else return x == 0u ? L - 1u : x - 1u;
  };
  const uint32_t c0 = step(x0, d0), c1 = step(x1, d1), c2 = step(x2, d2);
  const uint32_t par = (c0 + c1 + c2) & 1u;
  return par * uint32_t(g.half) + (c0 * L + c1) * uint32_t(g.Lh) + (c2 >> 1);
}

}  // namespace gn
