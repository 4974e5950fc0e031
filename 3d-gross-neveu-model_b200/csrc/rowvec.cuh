// rowvec.cuh -- the staggered stencil on W consecutive sites at a time, with
// 8- or 16-byte vector loads, and the site order every sweep follows.
//
// Work item: W consecutive sites k0 .. k0+W-1 of one parity half of one
// lattice row (x0, x1) (see geometry.cuh for the layout).  W divides L/2.
// Items are numbered row by row, and within a row the even half's items come
// before the odd half's:
//     j = row * (L/W) + par * (L/2)/W + k0/W.
// So a sweep over j visits both parities of a row together.  The time
// neighbours of a row's sites sit in the other parity half of the same row,
// so they are read from DRAM once for both uses (as a centre and as a
// neighbour).  The x0 +- 1 and x1 +- 1 rows are at most L rows away, well
// inside the window of rows a sweep has in flight.
//
// Neighbours of the item (all in the other parity half):
//   x0 +- 1, x1 +- 1: the sites k0 .. k0+W-1 of the adjacent rows, one aligned
//                     vector each;
//   time:             the vector k0 .. k0+W-1 of the same row (q) plus one
//                     value e.  With b = (par + x0 + x1) & 1, site k sits at
//                     x2 = 2k + b:
//                       b = 0: up(k) = q[k],   dn(k) = q[k-1]  (e = q[k0-1])
//                       b = 1: up(k) = q[k+1], dn(k) = q[k]    (e = q[k0+W])
//                     indices mod L/2.  The antiperiodic sign falls on
//                     dn(k0) when b = 0 and k0 = 0 (x2 = 0), and on
//                     up(k0+W-1) when b = 1 and k0+W = L/2 (x2 = L-1).
// Every site gets the same Nb<T> and sign bits as make_site() gives it, so
// the stencils of device_common.cuh produce the same bits on either path.
#pragma once
#include "device_common.cuh"

namespace gn {

template <typename T, int W>
struct VecT;
template <>
struct VecT<double, 1> {
  using type = double;
};
template <>
struct VecT<double, 2> {
  using type = double2;
};
template <>
struct VecT<float, 1> {
  using type = float;
};
template <>
struct VecT<float, 2> {
  using type = float2;
};
template <>
struct VecT<float, 4> {
  using type = float4;
};

// Aligned vector load / store of W values (index a multiple of W).
template <typename T, int W>
__device__ __forceinline__ void vload(const T *p, T (&v)[W]) {
  using VT = typename VecT<T, W>::type;
  const VT x = *reinterpret_cast<const VT *>(p);
  if constexpr (W == 1) {
    v[0] = x;
  } else if constexpr (W == 2) {
    v[0] = x.x;
    v[1] = x.y;
  } else {
    v[0] = x.x;
    v[1] = x.y;
    v[2] = x.z;
    v[3] = x.w;
  }
}
template <typename T, int W>
__device__ __forceinline__ void vstore(T *p, const T (&v)[W]) {
  using VT = typename VecT<T, W>::type;
  VT x;
  if constexpr (W == 1) {
    x = v[0];
  } else if constexpr (W == 2) {
    x.x = v[0];
    x.y = v[1];
  } else {
    x.x = v[0];
    x.y = v[1];
    x.z = v[2];
    x.w = v[3];
  }
  *reinterpret_cast<VT *>(p) = x;
}

// Largest W in {1, 2, 4} (at most wmax) that divides L/2.
__host__ __device__ __forceinline__ int row_width(int L, int wmax) {
  const int Lh = L / 2;
  if (wmax >= 4 && Lh % 4 == 0) return 4;
  if (wmax >= 2 && Lh % 2 == 0) return 2;
  return 1;
}

struct RowItem {
  uint32_t own;    // fermion index of the first site
  uint32_t nb[4];  // first-site indices of the x0+1, x0-1, x1+1, x1-1 vectors (other half)
  uint32_t tq;     // first-site index of the time vector q (other half, same row)
  uint32_t te;     // index of the extra time value
  uint32_t b;      // (par + x0 + x1) & 1
  uint32_t neg;    // sign bits shared by the W sites (Site::neg without the antiperiodic flips)
  uint32_t flip;   // 1: dn(time) of the first site flips; 2: up(time) of the last site flips
};

// Number of items of a sweep over all V sites.
template <int W>
__host__ __device__ __forceinline__ uint32_t row_items(const Geom &g) {
  return uint32_t(g.V / W);
}

template <int W>
__host__ __device__ __forceinline__ RowItem make_item(const Geom &g, uint32_t j) {
  const uint32_t L = uint32_t(g.L), Lh = uint32_t(g.Lh), P = uint32_t(g.plane);
  const uint32_t per_row = L / W, C = Lh / W;
  uint32_t row;
  if constexpr (W == 1) row = fdiv(j, g.div_L);
  else if constexpr (W == 2) row = fdiv(j, g.div_Lh);
  else row = fdiv(j, g.div_Lq);
  const uint32_t rem = j - row * per_row;
  const uint32_t par = rem >= C ? 1u : 0u;
  const uint32_t k0 = (rem - par * C) * W;
  const uint32_t x0 = fdiv(row, g.div_L);
  const uint32_t x1 = row - x0 * L;
  const uint32_t h = row * Lh + k0;
  const uint32_t qb = (1u - par) * uint32_t(g.half);
  RowItem it;
  it.own = par * uint32_t(g.half) + h;
  it.nb[0] = qb + ((x0 + 1u == L) ? h - (L - 1u) * P : h + P);
  it.nb[1] = qb + ((x0 == 0u) ? h + (L - 1u) * P : h - P);
  it.nb[2] = qb + ((x1 + 1u == L) ? h - (L - 1u) * Lh : h + Lh);
  it.nb[3] = qb + ((x1 == 0u) ? h + (L - 1u) * Lh : h - Lh);
  it.tq = qb + h;
  it.b = (par + x0 + x1) & 1u;
  const uint32_t rb = qb + row * Lh;
  it.te = rb + (it.b ? ((k0 + W == Lh) ? 0u : k0 + W) : ((k0 == 0u) ? Lh - 1u : k0 - 1u));
  const uint32_t e1 = x0 & 1u, e2 = (x0 + x1) & 1u;
  it.neg = (e1 << 1) | (e2 << 2) | (e1 << 4) | (e2 << 5);
  it.flip = (it.b == 0u && k0 == 0u) ? 1u : ((it.b == 1u && k0 + W == Lh) ? 2u : 0u);
  return it;
}

// Sign bits of site e of the item.
template <int W>
__host__ __device__ __forceinline__ uint32_t item_neg(const RowItem &it, int e) {
  uint32_t n = it.neg;
  if (e == 0 && it.flip == 1u) n ^= 1u << 5;
  if (e == W - 1 && it.flip == 2u) n ^= 1u << 2;
  return n;
}

// The seven stencil values of the W sites.  ldv(index, T(&)[W]) loads an
// aligned vector, lds(index) one value; both may transform what they read
// (e.g. r + beta p), applied the same way to every value.
template <typename T, int W, typename LoadV, typename LoadS>
__device__ __forceinline__ void gather_item(const RowItem &it, Nb<T> (&n)[W], LoadV ldv, LoadS lds) {
  T c[W], u0[W], d0[W], u1[W], d1[W], q[W];
  ldv(it.own, c);
  ldv(it.nb[0], u0);
  ldv(it.nb[1], d0);
  ldv(it.nb[2], u1);
  ldv(it.nb[3], d1);
  ldv(it.tq, q);
  const T e = lds(it.te);
#pragma unroll
  for (int s = 0; s < W; s++) {
    n[s].c = c[s];
    n[s].up[0] = u0[s];
    n[s].dn[0] = d0[s];
    n[s].up[1] = u1[s];
    n[s].dn[1] = d1[s];
    if (it.b == 0u) {
      n[s].up[2] = q[s];
      n[s].dn[2] = s == 0 ? e : q[s - 1];
    } else {
      n[s].up[2] = s == W - 1 ? e : q[s + 1];
      n[s].dn[2] = q[s];
    }
  }
}

// Plain gather from one field.
template <typename T, int W>
__device__ __forceinline__ void gather_item(const RowItem &it, const T *f, Nb<T> (&n)[W]) {
  gather_item<T, W>(
      it, n, [&](uint32_t j, T(&v)[W]) { vload<T, W>(f + j, v); }, [&](uint32_t j) { return f[j]; });
}

// The stencils on the W sites (same operation order as the one-site forms).
template <typename T, int W>
__device__ __forceinline__ void item_M(const RowItem &it, const T (&sm)[W], const Nb<T> (&n)[W], T (&out)[W]) {
  Site s;
#pragma unroll
  for (int e = 0; e < W; e++) {
    s.neg = item_neg<W>(it, e);
    out[e] = apply_M<T>(s, sm[e], n[e]);
  }
}
template <typename T, int W>
__device__ __forceinline__ void item_Mt(const RowItem &it, const T (&sm)[W], const Nb<T> (&n)[W], T (&out)[W]) {
  Site s;
#pragma unroll
  for (int e = 0; e < W; e++) {
    s.neg = item_neg<W>(it, e);
    out[e] = apply_Mt<T>(s, sm[e], n[e]);
  }
}
// out <- out - M psi
template <typename T, int W>
__device__ __forceinline__ void item_sub_M(const RowItem &it, const T (&sm)[W], const Nb<T> (&n)[W], T (&out)[W]) {
  Site s;
#pragma unroll
  for (int e = 0; e < W; e++) {
    s.neg = item_neg<W>(it, e);
    out[e] = apply_sub_M<T>(s, out[e], sm[e], n[e]);
  }
}

// ------------------------------------------------------------------ U(1) model
// The complex mass of the U(1) Gross-Neveu model (PI_INTERACTION): the
// diagonal of M is sm + i eps(x) pm (dirac.c:65-69), of M^dagger sm - i eps pm
// (dirac.c:106-109), with eps = +1 on even and -1 on odd sites (the item's
// parity) and pm the pi field's mass.  A complex field is two planes (real,
// imaginary).  The mass product is formed as C forms (a + ib)(c + id):
// (ac - bd) + i(ad + bc); the hopping terms are added to each plane in the
// order of the real stencils.  b = eps pm is exact (eps = +-1).
template <typename T, int W>
__device__ __forceinline__ void item_eps_pm(const Geom &g, const RowItem &it, const T *pm, T (&b)[W]) {
  vload<T, W>(pm + it.own, b);
  if (it.own >= uint32_t(g.half)) {
#pragma unroll
    for (int e = 0; e < W; e++) b[e] = -b[e];
  }
}

template <typename T, int W>
__device__ __forceinline__ void item_M_cm(const RowItem &it, const T (&sm)[W], const T (&b)[W],
                                          const Nb<T> (&nr)[W], const Nb<T> (&ni)[W], T (&out_r)[W],
                                          T (&out_i)[W]) {
#pragma unroll
  for (int e = 0; e < W; e++) {
    const uint32_t neg = item_neg<W>(it, e);
    T tr = sm[e] * nr[e].c - b[e] * ni[e].c;
    T ti = sm[e] * ni[e].c + b[e] * nr[e].c;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      tr = hop_add(tr, nr[e].up[d], neg, d);
      tr = hop_sub(tr, nr[e].dn[d], neg, 3 + d);
      ti = hop_add(ti, ni[e].up[d], neg, d);
      ti = hop_sub(ti, ni[e].dn[d], neg, 3 + d);
    }
    out_r[e] = tr;
    out_i[e] = ti;
  }
}

// M^dagger: the mass sm - i b, formed as (sm c - (-b) d) + i(sm d + (-b) c)
template <typename T, int W>
__device__ __forceinline__ void item_Mt_cm(const RowItem &it, const T (&sm)[W], const T (&b)[W],
                                           const Nb<T> (&nr)[W], const Nb<T> (&ni)[W], T (&out_r)[W],
                                           T (&out_i)[W]) {
#pragma unroll
  for (int e = 0; e < W; e++) {
    const uint32_t neg = item_neg<W>(it, e);
    const T mb = -b[e];
    T tr = sm[e] * nr[e].c - mb * ni[e].c;
    T ti = sm[e] * ni[e].c + mb * nr[e].c;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      tr = hop_sub(tr, nr[e].up[d], neg, d);
      tr = hop_add(tr, nr[e].dn[d], neg, 3 + d);
      ti = hop_sub(ti, ni[e].up[d], neg, d);
      ti = hop_add(ti, ni[e].dn[d], neg, 3 + d);
    }
    out_r[e] = tr;
    out_i[e] = ti;
  }
}

// out <- out - M psi (SubtractDiracFermion with the complex mass, dirac.c:213-247:
// the mass product first, then the hopping terms)
template <typename T, int W>
__device__ __forceinline__ void item_sub_M_cm(const RowItem &it, const T (&sm)[W], const T (&b)[W],
                                              const Nb<T> (&nr)[W], const Nb<T> (&ni)[W], T (&out_r)[W],
                                              T (&out_i)[W]) {
#pragma unroll
  for (int e = 0; e < W; e++) {
    const uint32_t neg = item_neg<W>(it, e);
    T tr = out_r[e] - (sm[e] * nr[e].c - b[e] * ni[e].c);
    T ti = out_i[e] - (sm[e] * ni[e].c + b[e] * nr[e].c);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      tr = hop_sub(tr, nr[e].up[d], neg, d);
      tr = hop_add(tr, nr[e].dn[d], neg, 3 + d);
      ti = hop_sub(ti, ni[e].up[d], neg, d);
      ti = hop_add(ti, ni[e].dn[d], neg, 3 + d);
    }
    out_r[e] = tr;
    out_i[e] = ti;
  }
}

}  // namespace gn
