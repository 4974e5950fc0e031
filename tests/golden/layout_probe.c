/* Prints the struct layout of include/gn_dropin.h in the order of
 * gnref_layout (oracle/ref_harness.c); compiled and run by tests/test_capi.py. */
#include <stddef.h>
#include <stdio.h>
#include "gn_dropin.h"
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
        sizeof(struct Momentasigma), sizeof(struct RandomVec)};
    for (size_t i = 0; i < sizeof v / sizeof v[0]; i++) printf("%ld\n", v[i]);
    return 0;
}
