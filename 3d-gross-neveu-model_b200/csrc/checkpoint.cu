// checkpoint.cu -- host code: the reference's lattice file and the
// TakeMeasures output line.  No device code.
//
// File layout (simulation.c:129-185, SIGMA_INTERACTION without
// PI_INTERACTION, DIM = 3), native byte order as fwrite leaves it:
//   double complex link[V][3]   lexicographic site, then direction
//   double sigma[V]             the reference's storage (fermion) order
//   double check                sum_x sum_d (carg(link[x][d]) + sigmamass[x] / 3)
//   double epsilon_link; slot;  int accepted_link, done_link;
//   slot;                       int accepted_sigma, done_sigma;
//   double epsilon_pi;   slot;  int accepted_pi, done_pi;   int measure
// where each slot is the 8 bytes that fwrite(&info.story_X, sizeof(double))
// takes from struct Info (info.h:57-59, three consecutive ints): {story_link,
// story_sigma}, {story_sigma, story_pi}, {story_pi, padding}.  Read back the
// same way, the later slot sets story_sigma and story_pi last, so each field
// ends as the first int of its own slot.
// The reader recomputes the check value from the sigma mass of the sigma it
// read and compares it for equality, so the writer forms it in the
// reference's order of additions (TestWriteReadLattice, simulation.c:101-120)
// from a sigma mass computed as ComputeFullSigmaMass computes it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>

#include "checkpoint.h"
#include "errors.h"

namespace gn {

namespace {

struct File {
  FILE *f;
  explicit File(FILE *p) : f(p) {}
  ~File() {
    if (f) fclose(f);
  }
};

template <typename T>
bool put(FILE *f, const T *v, size_t n) {
  return fwrite(v, sizeof(T), n, f) == n;
}
template <typename T>
bool get(FILE *f, T *v, size_t n) {
  return fread(v, sizeof(T), n, f) == n;
}

}  // namespace

double lattice_check_value(int L, const double *sm, const double *links) {
  const size_t V = size_t(L) * L * L;
  double total = 0.0;
  for (size_t x = 0; x < V; x++)
    for (int d = 0; d < 3; d++) {
      total += links ? std::atan2(links[(3 * x + d) * 2 + 1], links[(3 * x + d) * 2]) : 0.0;
      total += sm[x] / 3;
    }
  return total;
}

int write_lattice_file(const char *path, const char *copy, int L, const double *sigma, const double *sm,
                       const double *links, const gn_hmc_counters &c) {
  const size_t V = size_t(L) * L * L;
  if (copy != nullptr) {  // keep the previous file as the copy (simulation.c:131-136)
    struct stat st;
    if (stat(copy, &st) == 0) remove(copy);
    rename(path, copy);
  }
  File out(fopen(path, "wb"));
  if (out.f == nullptr) return GN_ERR_IO;
  std::vector<double> unit;
  if (links == nullptr) {
    unit.assign(6 * V, 0.0);
    for (size_t i = 0; i < 3 * V; i++) unit[2 * i] = 1.0;
    links = unit.data();
  }
  const double check = lattice_check_value(L, sm, links);
  const int slot_link[2] = {c.story_link, c.story_sigma}, slot_sigma[2] = {c.story_sigma, c.story_pi},
            slot_pi[2] = {c.story_pi, 0};
  bool ok = put(out.f, links, 6 * V) && put(out.f, sigma, V) && put(out.f, &check, 1);
  ok = ok && put(out.f, &c.epsilon_link, 1) && put(out.f, slot_link, 2) && put(out.f, &c.accepted_link, 1) &&
       put(out.f, &c.done_link, 1);
  ok = ok && put(out.f, slot_sigma, 2) && put(out.f, &c.accepted_sigma, 1) && put(out.f, &c.done_sigma, 1);
  ok = ok && put(out.f, &c.epsilon_pi, 1) && put(out.f, slot_pi, 2) && put(out.f, &c.accepted_pi, 1) &&
       put(out.f, &c.done_pi, 1);
  ok = ok && put(out.f, &c.measure, 1);
  ok = (fclose(out.f) == 0) && ok;
  out.f = nullptr;
  return ok ? GN_OK : GN_ERR_IO;
}

int read_lattice_file(const char *path, int L, LatticeFile &f) {
  const size_t V = size_t(L) * L * L;
  File in(fopen(path, "rb"));
  if (in.f == nullptr) return GN_ERR_NOT_FOUND;
  f.links.assign(6 * V, 0.0);
  f.sigma.assign(V, 0.0);
  memset(&f.c, 0, sizeof f.c);
  gn_hmc_counters &c = f.c;
  int slot_link[2], slot_sigma[2], slot_pi[2];
  bool ok = get(in.f, f.links.data(), 6 * V) && get(in.f, f.sigma.data(), V) && get(in.f, &f.check, 1);
  ok = ok && get(in.f, &c.epsilon_link, 1) && get(in.f, slot_link, 2) && get(in.f, &c.accepted_link, 1) &&
       get(in.f, &c.done_link, 1);
  ok = ok && get(in.f, slot_sigma, 2) && get(in.f, &c.accepted_sigma, 1) && get(in.f, &c.done_sigma, 1);
  ok = ok && get(in.f, &c.epsilon_pi, 1) && get(in.f, slot_pi, 2) && get(in.f, &c.accepted_pi, 1) &&
       get(in.f, &c.done_pi, 1);
  ok = ok && get(in.f, &c.measure, 1);
  c.story_link = slot_link[0];
  c.story_sigma = slot_sigma[0];
  c.story_pi = slot_pi[0];
  return ok ? GN_OK : GN_ERR_FORMAT;
}

}  // namespace gn

extern "C" {

int gn_checkpoint_write_file(const char *path, const char *path_copy, int L, const double *sigma,
                             const double *sigmamass, const double *links, const gn_hmc_counters *c) {
  if (!path || !sigma || !sigmamass || !c || L < 2 || (L & 1)) return gn::set_last_error(GN_ERR_ARG, "bad argument");
  const int st = gn::write_lattice_file(path, path_copy, L, sigma, sigmamass, links, *c);
  return st == GN_OK ? GN_OK : gn::set_last_error(st, "cannot write the lattice file");
}

int gn_checkpoint_read_file(const char *path, int L, double *sigma, double *links, gn_hmc_counters *c,
                            double *check) {
  if (!path || !sigma || L < 2 || (L & 1)) return gn::set_last_error(GN_ERR_ARG, "bad argument");
  gn::LatticeFile f;
  const int st = gn::read_lattice_file(path, L, f);
  if (st == GN_ERR_NOT_FOUND) return gn::set_last_error(st, "cannot open the lattice file");
  if (st != GN_OK) return gn::set_last_error(st, "the lattice file is short");
  memcpy(sigma, f.sigma.data(), f.sigma.size() * sizeof(double));
  if (links) memcpy(links, f.links.data(), f.links.size() * sizeof(double));
  if (c) *c = f.c;
  if (check) *check = f.check;
  return GN_OK;
}

double gn_checkpoint_check_value(int L, const double *sigmamass, const double *links) {
  if (!sigmamass || L < 2) return 0.0;
  return gn::lattice_check_value(L, sigmamass, links);
}

int gn_format_measure_line(char *buf, size_t size, int measure, int L, double beta, double beta_scalar, double mass,
                           double avg_iterations, double avg_distance, const double *cond_dirac,
                           const double *cond_sigma) {
  std::string s;
  char tmp[400];  // "%.16f" of the largest double is 326 characters
  snprintf(tmp, sizeof tmp, "%d\t%d", measure, L);
  s += tmp;
  auto add = [&](double v) {
    snprintf(tmp, sizeof tmp, "\t%.16f", v);
    s += tmp;
  };
  for (double v : {beta, beta_scalar, mass, avg_iterations, avg_distance}) add(v);
  if (cond_dirac)
    for (int i = 0; i < 11; i++) add(cond_dirac[i]);
  if (cond_sigma)
    for (int i = 0; i < 8; i++) add(cond_sigma[i]);
  s += "\n";
  if (buf != nullptr && size > 0) {
    const size_t n = s.size() < size - 1 ? s.size() : size - 1;
    memcpy(buf, s.data(), n);
    buf[n] = '\0';
  }
  return int(s.size());
}

}  // extern "C"
