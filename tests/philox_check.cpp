// Prints Philox4x64-10 blocks of csrc/philox.cuh (host build of the device
// code) for the (key, counter) pairs read from stdin, one block per line as
// four hexadecimal words.  Used by tests/test_philox.py.
#include <cstdio>

#include "philox.cuh"

int main() {
  unsigned long long k0, k1, c0, c1, c2, c3;
  while (std::scanf("%llx %llx %llx %llx %llx %llx", &k0, &k1, &c0, &c1, &c2, &c3) == 6) {
    gn::Philox4x64 c;
    c.v[0] = c0;
    c.v[1] = c1;
    c.v[2] = c2;
    c.v[3] = c3;
    const gn::Philox4x64 r = gn::philox4x64(c, k0, k1);
    std::printf("%016llx %016llx %016llx %016llx\n", (unsigned long long)r.v[0], (unsigned long long)r.v[1],
                (unsigned long long)r.v[2], (unsigned long long)r.v[3]);
  }
  return 0;
}
