// Prints the op lists of csrc/schedule.h (the sigma integrators and the
// reference's MD helpers) for tests/test_schedule.py: one line per list,
// "<kind> <integrator> <step>: op:coef op:coef ...".
#include <cstdio>

#include "schedule.h"
using namespace gn;

static void dump(const char *kind, int integrator, int step, const std::vector<Op> &v) {
  std::printf("%s %d %d:", kind, integrator, step);
  for (const Op &o : v) std::printf(" %d:%.17g", o.op, o.c);
  std::printf("\n");
}

int main() {
  const double eps = 0.05;
  for (int integrator = 0; integrator < 3; integrator++)
    for (int step : {1, 2, 3, 4, 10}) {
      dump("traj", integrator, step, schedule(integrator, eps, step));
      dump("evolve", integrator, step, evolve_schedule(integrator, eps, step));
    }
  return 0;
}
