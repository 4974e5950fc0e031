/* Compares gn_host_hypot (3d-gross-neveu-model_b200/csrc/host_hypot.h) with
 * this host's libm hypot, and pow(a, 2.0) with a * a, on random pairs over a
 * wide range of magnitudes and ratios.  Prints the two mismatch counts.
 * Built by tests/test_host_hypot.py with -ffp-contract=off. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "host_hypot.h"

static uint64_t state = 0x9E3779B97F4A7C15ull;
static double unit(void) {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return (double)(state >> 11) * (1.0 / 9007199254740992.0);
}

int main(int argc, char **argv) {
  const long n = argc > 1 ? atol(argv[1]) : 1000000;
  long bad_h = 0, bad_p = 0;
  for (long i = 0; i < n; i++) {
    double x, y;
    switch (i % 4) {
      case 0:
        x = (unit() - 0.5) * ldexp(1.0, (int)(unit() * 80) - 60);
        y = (unit() - 0.5) * ldexp(1.0, (int)(unit() * 80) - 60);
        break;
      case 1:
        x = unit() - 0.5;
        y = x * (2 * unit() - 1) * ldexp(1.0, -(int)(unit() * 60));
        break;
      case 2:
        x = unit();
        y = unit();
        break;
      default:
        x = (unit() - 0.5) * 1e-6;
        y = (unit() - 0.5) * 1e-6;
    }
    const double h = hypot(x, y);
    if (gn_host_hypot(x, y) != h) bad_h++;
    if (pow(h, 2.0) != h * h) bad_p++;
  }
  printf("%ld %ld\n", bad_h, bad_p);
  return 0;
}
