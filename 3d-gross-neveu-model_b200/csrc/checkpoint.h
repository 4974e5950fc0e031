// checkpoint.h -- the reference's lattice file (WriteBinaryLattice /
// ReadBinaryLattice, simulation.c:129-401) for the sigma model, shared by the
// context and ensemble entry points.
#pragma once
#include <vector>

#include "../../include/gn_b200.h"

namespace gn {

struct LatticeFile {
  std::vector<double> sigma;  // V, fermion order
  std::vector<double> links;  // 6V: (re, im) per (lexicographic site, direction)
  gn_hmc_counters c;
  double check = 0.0;  // the stored check value
};

// GN_OK, GN_ERR_NOT_FOUND (cannot open) or GN_ERR_FORMAT (short file).
int read_lattice_file(const char *path, int L, LatticeFile &f);
// GN_OK or GN_ERR_IO; rotates path to copy first when copy is given.
int write_lattice_file(const char *path, const char *copy, int L, const double *sigma, const double *sm,
                       const double *links, const gn_hmc_counters &c);
// sum_x sum_d (carg(link) + sm[x] / 3), the order of TestWriteReadLattice
// (simulation.c:101-120); links NULL: unit links.
double lattice_check_value(int L, const double *sm, const double *links);

// ReadBinaryLattice with try_copy: path, then copy.  A candidate is taken
// when it reads in full and the check value recomputed from its sigma
// (sm_of(sigma, sm) computes the sigma mass) equals the stored one bit for
// bit; then accept(sigma) installs it and c receives the counters.  Returns
// GN_OK, GN_ERR_NOT_FOUND (no candidate could be opened) or GN_ERR_FORMAT.
template <typename SmOf, typename Accept>
int load_lattice(const char *path, const char *copy, int L, gn_hmc_counters *c, SmOf sm_of, Accept accept) {
  const size_t V = size_t(L) * L * L;
  const char *cand[2] = {path, copy};
  bool opened = false;
  for (const char *p : cand) {
    if (p == nullptr) continue;
    LatticeFile f;
    const int st = read_lattice_file(p, L, f);
    if (st == GN_ERR_NOT_FOUND) continue;
    opened = true;
    if (st != GN_OK) continue;
    std::vector<double> sm(V);
    sm_of(f.sigma.data(), sm.data());
    if (lattice_check_value(L, sm.data(), f.links.data()) != f.check) continue;
    accept(f.sigma.data());
    if (c) *c = f.c;
    return GN_OK;
  }
  return opened ? GN_ERR_FORMAT : GN_ERR_NOT_FOUND;
}

}  // namespace gn
