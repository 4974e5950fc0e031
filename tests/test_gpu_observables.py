"""GPU tests of the sigma observables (CondensateSigmaPi, observables.c:323)
and of checkpoints of device-resident fields (the reference's lattice file,
simulation.c:129-401), through the C-ABI.

Reference values: the fixtures made by the reference's own code
(tests/golden/make_observables.py) and, where its compiled harness is present
(oracle/_ref), the reference run live on the same sigma.  Tolerances: the
observables are sums over V sites in another order than the reference's
serial loop (a compensated tree): relative 1e-12; files and fields exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUNTERS = dict(epsilon_link=0.5, epsilon_pi=0.25, story_link=4, story_sigma=-6, story_pi=3, accepted_link=1,
                done_link=2, accepted_sigma=77, done_sigma=90, accepted_pi=5, done_pi=8, measure=17)


def ref_lattice(L):
    from oracle import build_ref
    from oracle.oracle import Ref
    if not build_ref.lib_path(L).exists() and not build_ref.available():
        pytest.skip("no compiled reference harness")
    r = Ref(L)
    r.init(1231, 0.85, 0.2, 2)
    return r


@pytest.fixture(scope="module")
def lattices():
    import gn_b200
    cache = {}

    def get(L):
        if L not in cache:
            cache[L] = gn_b200.Lattice(L)
        return cache[L]
    yield get
    for lat in cache.values():
        lat.close()


@pytest.mark.parametrize("L", [4, 8])
def test_condensate_sigma_vs_golden(lattices, golden, L):
    g = golden(f"golden_L{L}_sigma_obs.npz")
    lat = lattices(L)
    for name in ("centred", "shifted"):
        got = lat.condensate_sigma(g[f"sigma_{name}"])
        np.testing.assert_allclose(got, g[f"obs_{name}"], rtol=1e-12, atol=1e-16)
        lat.load_sigma(g[f"sigma_{name}"])  # the resident field, no transfer
        np.testing.assert_allclose(lat.condensate_sigma(), g[f"obs_{name}"], rtol=1e-12, atol=1e-16)


@pytest.mark.parametrize("L", [16, 32])
def test_condensate_sigma_vs_reference(lattices, L):
    ref = ref_lattice(L)
    rng = np.random.default_rng(L)
    sigma = rng.normal(0.1, 0.77, L ** 3)
    ref.set_sigma(sigma)
    np.testing.assert_allclose(lattices(L).condensate_sigma(sigma), ref.condensate_sigma(), rtol=1e-12, atol=1e-16)


def test_checkpoint_save_is_the_reference_file(lattices, golden, tmp_path):
    """A context's resident sigma saved: the reference's file byte for byte
    (the sigma mass of the check value comes from the device, bit-exact)."""
    from conftest import GOLDEN
    g = golden("golden_L4_lattice.npz")
    counters = {str(k): v for k, v in zip(g["counter_names"], g["counters"])}
    lat = lattices(4)
    lat.load_sigma(g["sigma"])
    path = tmp_path / "terma.bin"
    lat.checkpoint_save(path, None, counters)
    assert path.read_bytes() == (GOLDEN / "golden_L4_lattice.bin").read_bytes()


def test_checkpoint_load_and_fallback(lattices, golden, tmp_path):
    """ReadBinaryLattice's rules: the file, else its copy; a file that is short
    or whose check value does not match is passed over; neither file: a fresh
    start; nothing acceptable: GN_ERR_FORMAT with the resident sigma kept."""
    import gn_b200 as G
    from conftest import GOLDEN
    g = golden("golden_L4_lattice.npz")
    good = (GOLDEN / "golden_L4_lattice.bin").read_bytes()
    lat = lattices(4)
    lat.load_sigma(np.zeros(64))
    path, copy = tmp_path / "t.bin", tmp_path / "t_copy.bin"
    path.write_bytes(good)
    st, c = lat.checkpoint_load(path, copy)
    assert st == G.GN_OK and c["measure"] == 42
    assert np.array_equal(lat.store_sigma()[0], g["sigma"])
    # a short primary: the copy
    path.write_bytes(good[:-5])
    copy.write_bytes(good)
    lat.load_sigma(np.zeros(64))
    assert lat.checkpoint_load(path, copy)[0] == G.GN_OK
    assert np.array_equal(lat.store_sigma()[0], g["sigma"])
    # one sigma value changed: the check value no longer matches
    bad = bytearray(good)
    bad[3072 + 8 * 5 + 6] ^= 0x40  # a high mantissa bit of sigma[5]
    path.write_bytes(bytes(bad))
    copy.unlink()
    keep = np.arange(64, dtype=np.float64)
    lat.load_sigma(keep)
    assert lat.checkpoint_load(path, copy)[0] == G.GN_ERR_FORMAT
    assert np.array_equal(lat.store_sigma()[0], keep)
    path.unlink()
    assert lat.checkpoint_load(path, copy)[0] == G.GN_ERR_NOT_FOUND


def test_checkpoint_round_trip_with_reference(lattices, tmp_path):
    """A saved L = 8 context read by the reference's ReadBinaryLattice, and a
    file written by the reference loaded into a context."""
    import gn_b200 as G
    ref = ref_lattice(8)
    sigma = np.random.default_rng(3).normal(0.0, 0.77, 512)
    lat = lattices(8)
    lat.load_sigma(sigma)
    ours = tmp_path / "ours.bin"
    lat.checkpoint_save(ours, None, COUNTERS)
    s, c, check_ref = ref.read_lattice(ours, tmp_path / "absent.bin")
    assert np.array_equal(s, sigma) and all(float(c[k]) == float(COUNTERS[k]) for k in COUNTERS)
    assert G.checkpoint_read_file(ours, 8)[3] == check_ref
    theirs = tmp_path / "theirs.bin"
    ref.set_sigma(-sigma)
    ref.write_lattice(theirs, tmp_path / "theirs_copy.bin", COUNTERS)
    lat.load_sigma(np.zeros(512))
    assert lat.checkpoint_load(theirs)[0] == G.GN_OK
    assert np.array_equal(lat.store_sigma()[0], -sigma)


def test_ensemble_observables_and_checkpoint(tmp_path):
    """Per-chain means of CondensateSigmaPi over trajectories, taken on the
    device after every trajectory, against the reference's CondensateSigmaPi
    of each chain's sigma read back after each trajectory; a chain's checkpoint
    saved and loaded back."""
    import gn_b200 as G
    Ls, betas = [8, 12], [0.85, 1.0]
    refs = {L: ref_lattice(L) for L in Ls}
    with G.Ensemble(Ls, betas, seed=77) as ens:
        rng = np.random.default_rng(9)
        for c, L in enumerate(Ls):
            ens.load_sigma(c, rng.normal(0.2, 0.77, L ** 3))
        p = ens.params(0.08, 4, tol=1e-10)
        ens.stats(reset=True)
        want = np.zeros((len(Ls), 8))
        ntraj = 3
        for _ in range(ntraj):
            ens.run(p, 1)
            for c, L in enumerate(Ls):
                refs[L].set_sigma(ens.store_sigma(c)[0])
                want[c] += refs[L].condensate_sigma()
        want /= ntraj
        st = ens.stats()
        assert [s["trajectories"] for s in st] == [ntraj] * len(Ls)
        np.testing.assert_allclose(ens.observables(), want, rtol=1e-11, atol=1e-16)
        # checkpoint of chain 1: the file holds its sigma; loading it back restores it
        s1, sm1 = ens.store_sigma(1)
        path = tmp_path / "chain1.bin"
        ens.checkpoint_save(1, path, None, COUNTERS)
        s, links, c, check = G.checkpoint_read_file(path, 12)
        assert np.array_equal(s, s1) and c["measure"] == COUNTERS["measure"]
        assert G.checkpoint_check_value(12, sm1) == check
        ens.load_sigma(1, np.zeros(12 ** 3))
        assert ens.checkpoint_load(1, path)[0] == G.GN_OK
        assert np.array_equal(ens.store_sigma(1)[0], s1)
        # an L = 12 file read as L = 8 has a sigma value where the check value
        # should be: rejected, and chain 0 keeps its sigma
        s0 = ens.store_sigma(0)[0]
        assert ens.checkpoint_load(0, path)[0] == G.GN_ERR_FORMAT
        assert np.array_equal(ens.store_sigma(0)[0], s0)
