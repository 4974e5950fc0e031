// schedule.h -- the sigma integrators as op lists, shared by the single-lattice
// trajectory (engine.cu) and the batched chains (ensemble.cu).
#pragma once
#include <vector>

#include "../../include/gn_b200.h"

namespace gn {

// Integrator schedules (moleculardynamics.c:859-1005, :1018-1221, :1234-1434)
// as op lists: F force (medium / high tolerance), P momentum step, Q sigma
// step, S X0-imposed solve at high tolerance, C early-exit solve
// (conjugategradient.c:13, from the current X) at high tolerance.
enum { OP_F_MED = 1, OP_F_HIGH, OP_P, OP_Q, OP_S_HIGH, OP_C_HIGH };
struct Op {
  int op;
  double c;
};

inline std::vector<Op> schedule(int integrator, double eps, int step) {
  std::vector<Op> v;
  const double lam = 0.1931833275037836;  // MAGIC_LAMBDA, macro.h:169
  auto push = [&](int o, double c) { v.push_back({o, c}); };
  if (integrator == GN_LFMN2VF) {
    push(OP_F_MED, 0); push(OP_P, lam * eps); push(OP_Q, eps / 2.0);
    push(OP_F_MED, 0); push(OP_P, (1.0 - (2.0 * lam)) * eps); push(OP_Q, eps / 2.0);
    for (int s = 1; s < step - 1; s++) {
      push(OP_F_MED, 0); push(OP_P, 2.0 * lam * eps); push(OP_Q, eps / 2.0);
      push(OP_F_MED, 0); push(OP_P, (1.0 - (2.0 * lam)) * eps); push(OP_Q, eps / 2.0);
    }
    push(OP_F_MED, 0); push(OP_P, 2.0 * lam * eps); push(OP_Q, eps / 2.0);
    push(OP_F_MED, 0); push(OP_P, (1.0 - (2.0 * lam)) * eps); push(OP_Q, eps / 2.0);
    push(OP_F_HIGH, 0); push(OP_P, lam * eps);
  } else if (integrator == GN_LF2) {
    push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    for (int s = 0; s < step - 1; s++) { push(OP_Q, eps); push(OP_F_MED, 0); push(OP_P, eps); }
    push(OP_Q, eps); push(OP_F_HIGH, 0); push(OP_P, eps / 2.0);
  } else {
    push(OP_Q, lam * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    push(OP_Q, (1.0 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    for (int s = 1; s < step - 1; s++) {
      push(OP_Q, 2.0 * lam * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
      push(OP_Q, (1.0 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    }
    push(OP_Q, 2.0 * lam * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    push(OP_Q, (1 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    push(OP_Q, lam * eps); push(OP_S_HIGH, 0);
  }
  return v;
}

// The reference's MD helpers EvolveSigmaInTimeLF2 (moleculardynamics.c:1460),
// EvolveSigmaInTimeMinimumNormLF2 (:1489) and
// EvolveSigmaInTimeMinimumNormSigmaVelocityFirst (:1551) -- the MD of the
// integrators without draws, energies or Metropolis test, used by the
// reference's reversibility check.  Their tolerance pattern differs from the
// integrators': the LF2 and LFMN2 helpers take their first force at the high
// tolerance and the others at the medium one; the velocity-first helper wraps
// the integrator's MD in an X0-imposed solve before and an early-exit solve
// after, both at the high tolerance.
inline std::vector<Op> evolve_schedule(int integrator, double eps, int step) {
  const double lam = 0.1931833275037836;  // MAGIC_LAMBDA, macro.h:169
  if (integrator == GN_LFMN2VF) {
    std::vector<Op> v{{OP_S_HIGH, 0.0}};
    for (const Op &o : schedule(GN_LFMN2VF, eps, step)) v.push_back(o);
    v.push_back({OP_C_HIGH, 0.0});
    return v;
  }
  std::vector<Op> v;
  auto push = [&](int o, double c) { v.push_back({o, c}); };
  if (integrator == GN_LF2) {
    push(OP_F_HIGH, 0); push(OP_P, eps / 2.0);
    for (int s = 0; s < step - 1; s++) { push(OP_Q, eps); push(OP_F_MED, 0); push(OP_P, eps); }
    push(OP_Q, eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
  } else {
    push(OP_Q, lam * eps); push(OP_F_HIGH, 0); push(OP_P, eps / 2.0);
    push(OP_Q, (1.0 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    for (int s = 1; s < step - 1; s++) {
      push(OP_Q, 2.0 * lam * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
      push(OP_Q, (1.0 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    }
    push(OP_Q, 2.0 * lam * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    push(OP_Q, (1.0 - (2.0 * lam)) * eps); push(OP_F_MED, 0); push(OP_P, eps / 2.0);
    push(OP_Q, lam * eps);
  }
  return v;
}

}  // namespace gn
