"""CPU tests of the reference's lattice file (WriteBinaryLattice /
ReadBinaryLattice, simulation.c:129-401) and of TakeMeasures' output line,
through the library's host functions (no device needed).

Parity: against the committed fixture written by the reference
(tests/golden/golden_L4_lattice.bin, make_observables.py), and, where the
reference tree is present, live against the reference's own reader and writer
(oracle/ref_harness.c).  The check value, which the reference's reader compares
for equality, must match bit for bit; sigma and every counter exactly.
"""
import numpy as np
import pytest

from oracle import build_ref

have_ref = build_ref.available()

COUNTERS = dict(epsilon_link=0.5, epsilon_pi=0.25, story_link=4, story_sigma=-6, story_pi=3, accepted_link=1,
                done_link=2, accepted_sigma=77, done_sigma=90, accepted_pi=5, done_pi=8, measure=17)


def golden_file(golden):
    g = golden("golden_L4_lattice.npz")
    counters = {str(k): v for k, v in zip(g["counter_names"], g["counters"])}
    return g["sigma"], g["sigmamass"], counters


def same_counters(a, b):
    return all(float(a[k]) == float(b[k]) for k in COUNTERS)


def test_reads_the_reference_file(golden, port):
    """The fixture the reference wrote reads back in full: sigma, unit links,
    every counter (the int story fields from their 8-byte slots), and the
    stored check value equals the one recomputed from the sigma mass."""
    import gn_b200 as G
    from conftest import GOLDEN
    sigma, sm, counters = golden_file(golden)
    s, links, c, check = G.checkpoint_read_file(GOLDEN / "golden_L4_lattice.bin", 4)
    assert np.array_equal(s, sigma)
    assert np.array_equal(links[..., 0], np.ones((64, 3))) and np.array_equal(links[..., 1], np.zeros((64, 3)))
    assert same_counters(c, counters)
    assert np.array_equal(port.sigma_mass(4, s), sm)
    assert G.checkpoint_check_value(4, sm) == check
    assert G.checkpoint_check_value(4, sm, links) == check


def test_writes_the_reference_file(golden, tmp_path):
    """Written from the same sigma, sigma mass and counters, the file is the
    reference's byte for byte."""
    import gn_b200 as G
    from conftest import GOLDEN
    sigma, sm, counters = golden_file(golden)
    path = tmp_path / "terma.bin"
    G.checkpoint_write_file(path, None, 4, sigma, sm, counters)
    assert path.read_bytes() == (GOLDEN / "golden_L4_lattice.bin").read_bytes()


@pytest.mark.skipif(not have_ref, reason="needs the reference tree")
@pytest.mark.parametrize("L", [4, 8])
def test_round_trips_with_the_reference(tmp_path, L):
    """Ours -> the reference's ReadBinaryLattice, and the reference's
    WriteBinaryLattice -> ours, on a fresh seeded sigma."""
    import gn_b200 as G
    from oracle.oracle import Ref
    ref = Ref(L)
    ref.init(1231, 0.85, 0.2, 2)
    V = L ** 3
    sigma = np.random.default_rng(L).normal(0.0, 0.77, V)
    ref.set_sigma(sigma)
    sm = ref.sigmamass()
    ours = tmp_path / "ours.bin"
    G.checkpoint_write_file(ours, None, L, sigma, sm, COUNTERS)
    ref.set_sigma(np.zeros(V))
    s, c, check_ref = ref.read_lattice(ours, tmp_path / "absent.bin")
    assert np.array_equal(s, sigma)
    assert same_counters(c, COUNTERS)
    assert G.checkpoint_read_file(ours, L)[3] == check_ref  # the reference's reader accepts the file
    theirs = tmp_path / "theirs.bin"
    ref.set_sigma(sigma)
    ref.write_lattice(theirs, tmp_path / "theirs_copy.bin", COUNTERS)
    s2, links, c2, check = G.checkpoint_read_file(theirs, L)
    assert np.array_equal(s2, sigma) and same_counters(c2, COUNTERS)
    assert G.checkpoint_check_value(L, sm, links) == check
    assert theirs.read_bytes() == ours.read_bytes()


def test_rotation_and_errors(tmp_path, golden):
    """WriteBinaryLattice's rotation (the previous file becomes the copy); a
    missing file is GN_ERR_NOT_FOUND, a short one GN_ERR_FORMAT."""
    import gn_b200 as G
    sigma, sm, counters = golden_file(golden)
    path, copy = tmp_path / "t.bin", tmp_path / "t_copy.bin"
    G.checkpoint_write_file(path, copy, 4, sigma, sm, counters)
    assert not copy.exists()
    c2 = dict(counters, measure=counters["measure"] + 1)
    G.checkpoint_write_file(path, copy, 4, 2 * sigma, 2 * sm, c2)
    assert G.checkpoint_read_file(copy, 4)[2]["measure"] == counters["measure"]
    assert G.checkpoint_read_file(path, 4)[2]["measure"] == c2["measure"]
    assert np.array_equal(G.checkpoint_read_file(path, 4)[0], 2 * sigma)
    with pytest.raises(G.GnError) as e:
        G.checkpoint_read_file(tmp_path / "absent.bin", 4)
    assert e.value.status == G.GN_ERR_NOT_FOUND
    short = tmp_path / "short.bin"
    short.write_bytes(path.read_bytes()[:-3])
    with pytest.raises(G.GnError) as e:
        G.checkpoint_read_file(short, 4)
    assert e.value.status == G.GN_ERR_FORMAT


def test_measure_line_format():
    """TakeMeasures' line (observables.c:266-292): two ints, then tab-separated
    "%.16f" values, the OBS_CONDENSATE group (11) and OBS_CONDENSATE_SIGMA (8)."""
    import gn_b200 as G
    rng = np.random.default_rng(5)
    head = [0.0, 0.85, 0.0, 123.456789, 0.5]
    cd, cs = rng.normal(size=11) * 1e3, rng.normal(size=8) * 1e-3
    line = G.format_measure_line(7, 16, *head, cond_dirac=cd, cond_sigma=cs)
    expect = "%d\t%d" % (7, 16) + "".join("\t%.16f" % v for v in [*head, *cd, *cs]) + "\n"
    assert line == expect
    assert G.format_measure_line(1, 8, *head) == "%d\t%d" % (1, 8) + "".join("\t%.16f" % v for v in head) + "\n"
    assert G.format_measure_line(1, 8, *head, cond_sigma=cs).count("\t") == 1 + 5 + 8
