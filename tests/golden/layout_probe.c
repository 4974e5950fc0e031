/* Prints the struct layout of include/gn_dropin.h and gn_dropin_pi.h in the
 * order of gnref_layout (oracle/ref_harness.c); compiled and run by
 * tests/test_capi.py. */
#include <stddef.h>
#include <stdio.h>
#include "gn_dropin_pi.h"
int main(void)
{
    long v[] = {
        sizeof(struct Lattice), offsetof(struct Lattice, sigma), offsetof(struct Lattice, sigmamass),
        offsetof(struct Lattice, eta_pbc), offsetof(struct Lattice, distance_sigma), offsetof(struct Lattice, done_sigma),
        sizeof(struct Fermioncoor), sizeof(struct Fermionkit), offsetof(struct Fermionkit, chi),
        offsetof(struct Fermionkit, phi), offsetof(struct Fermionkit, inverted_phi),
        offsetof(struct Fermionkit, inverted_phi_obs), offsetof(struct Fermionkit, Ddag_inverted_phi_obs),
        offsetof(struct Fermionkit, iterations), offsetof(struct Fermionkit, CG_call), sizeof(struct Info),
        offsetof(struct Info, beta_scalar), offsetof(struct Info, epsilon_link_HMC), offsetof(struct Info, steps_link_HMC),
        offsetof(struct Info, epsilon_sigma_HMC), offsetof(struct Info, steps_sigma_HMC),
        offsetof(struct Info, hybrid_done_acceptance_link), offsetof(struct Info, hybrid_accepted_sigma),
        offsetof(struct Info, hybrid_done_acceptance_sigma), offsetof(struct Info, local_acceptance_sigma),
        offsetof(struct Info, delta_H_link), offsetof(struct Info, story_sigma), sizeof(struct Forcesigma),
        sizeof(struct Momentasigma), sizeof(struct RandomVec), offsetof(struct Lattice, pi),
        offsetof(struct Lattice, epsilon_pi), offsetof(struct Lattice, pimass), offsetof(struct Lattice, distance_pi),
        offsetof(struct Lattice, done_pi), offsetof(struct Info, epsilon_pi_HMC), offsetof(struct Info, steps_pi_HMC),
        offsetof(struct Info, hybrid_accepted_pi), offsetof(struct Info, hybrid_done_acceptance_pi),
        offsetof(struct Info, story_pi), sizeof(struct Forcepi), sizeof(struct Momentapi)};
    for (size_t i = 0; i < sizeof v / sizeof v[0]; i++) printf("%ld\n", v[i]);
    return 0;
}
