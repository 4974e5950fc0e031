// Host check of the row-item geometry (3d-gross-neveu-model_b200/csrc/rowvec.cuh)
// against make_site (geometry.cuh) for every site: every site is covered once,
// the item neighbours and sign bits equal the one-site ones, vectors are
// aligned and every index is inside the lattice; and the 8-corner index of
// geometry.cuh against the general one.  Built and run by
// tests/test_item_geometry.py; prints the mismatch count per L and W.
#include <cstdio>
#include <vector>
#include "rowvec.cuh"
using namespace gn;
template <int W>
int check(int L) {
  Geom g = make_geom(L);
  const uint32_t V = uint32_t(g.V);
  if ((L / 2) % W) return 0;
  std::vector<int> seen(V, 0);
  int bad = 0;
  for (uint32_t j = 0; j < row_items<W>(g); j++) {
    RowItem it = make_item<W>(g, j);
    if (it.own % W || it.tq % W) bad++;
    for (int d = 0; d < 4; d++) if (it.nb[d] % W || it.nb[d] >= V) bad++;
    if (it.te >= V || it.own + W > V || it.tq + W > V) bad++;
    for (int e = 0; e < W; e++) {
      const uint32_t i = it.own + e;
      seen[i]++;
      Site s = make_site(g, i);
      if (s.nb_up[0] != it.nb[0] + e || s.nb_dn[0] != it.nb[1] + e || s.nb_up[1] != it.nb[2] + e || s.nb_dn[1] != it.nb[3] + e) bad++;
      uint32_t up2, dn2;
      if (it.b == 0) { up2 = it.tq + e; dn2 = e == 0 ? it.te : it.tq + e - 1; }
      else { up2 = e == W - 1 ? it.te : it.tq + e + 1; dn2 = it.tq + e; }
      if (s.nb_up[2] != up2 || s.nb_dn[2] != dn2) { if (bad < 5) printf("L=%d W=%d j=%u e=%d time mismatch\n", L, W, j, e); bad++; }
      if (s.neg != item_neg<W>(it, e)) { if (bad < 5) printf("L=%d W=%d j=%u e=%d neg %u vs %u\n", L, W, j, e, s.neg, item_neg<W>(it, e)); bad++; }
    }
  }
  for (uint32_t i = 0; i < V; i++) if (seen[i] != 1) bad++;
  return bad;
}
// corner_index (the 8-corner gathers) against site_index for every site and
// corner offset, in both directions
int check_corners(int L) {
  Geom g = make_geom(L);
  int bad = 0;
  for (uint32_t i = 0; i < uint32_t(g.V); i++) {
    uint32_t x0, x1, x2, par, row, k;
    site_coords(g, i, x0, x1, x2, par, row, k);
    for (int c = 0; c < 8; c++) {
      const int d0 = c & 1, d1 = (c >> 1) & 1, d2 = (c >> 2) & 1;
      if (corner_index<1>(g, x0, x1, x2, d0, d1, d2) != site_index(g, int(x0) + d0, int(x1) + d1, int(x2) + d2)) bad++;
      if (corner_index<-1>(g, x0, x1, x2, d0, d1, d2) != site_index(g, int(x0) - d0, int(x1) - d1, int(x2) - d2)) bad++;
    }
  }
  return bad;
}
int main() {
  int tot = 0;
  for (int L : {4, 6, 8, 10, 12, 16, 24, 32, 48, 64, 128, 256}) {
    int b1 = check<1>(L), b2 = check<2>(L), b4 = check<4>(L);
    int bc = L <= 64 ? check_corners(L) : 0;
    printf("L=%d bad W1 %d W2 %d W4 %d corners %d\n", L, b1, b2, b4, bc);
    tot += b1 + b2 + b4 + bc;
  }
  printf("total bad %d\n", tot);
  return tot != 0;
}
