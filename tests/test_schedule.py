"""The integrators' op lists (csrc/schedule.h), checked on the host.

schedule() restates the reference's three sigma integrators
(moleculardynamics.c:859-1005 LeapFrog2Sigma, :1018-1221
LeapFrog2MinimumNormSigma, :1234-1434 LeapFrog2MinimumNormSigmaVelocityFirst)
and evolve_schedule() its MD helpers (:1460-1625) as lists of force (F,
medium or high tolerance), momentum (P), sigma (Q) and solve steps.  The GPU
tests replay the reference's trajectories through them; these checks need no
GPU:

- for step >= 2 the sigma and momentum steps each add up to step x eps;
- the P/Q coefficient sequence is a palindrome (the integrators are
  time-reversible);
- the number of forces: 2 step + 1 (velocity first), step + 1 (LF2), 2 step
  (position-first minimum norm, then an X0-imposed solve);
- every force is followed by its momentum step; the tolerance pattern is the
  reference's (the last force of LF2 and of the velocity-first integrator at
  the high tolerance, the others medium; the helpers: the first force high in
  LF2 and LFMN2, the velocity-first helper wrapped in an X0-imposed and an
  early-exit solve).
For step = 1 the reference peels the first and the last MD step of its
minimum-norm integrators out of the loop, so both run; the lists do the same.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "3d-gross-neveu-model_b200" / "csrc"
F_MED, F_HIGH, P, Q, S_HIGH, C_HIGH = 1, 2, 3, 4, 5, 6
EPS = 0.05
LFMN2VF, LF2, LFMN2 = 0, 1, 2


@pytest.fixture(scope="module")
def lists(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    exe = tmp_path_factory.mktemp("sched") / "schedule_check"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{CSRC}", str(ROOT / "tests" / "schedule_check.cpp"), "-o",
                    str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        head, ops = line.split(":", 1)
        kind, integ, step = head.split()
        out[(kind, int(integ), int(step))] = [(int(a), float(b)) for a, b in (t.split(":") for t in ops.split())]
    return out


def pq(v):
    return [(o, c) for o, c in v if o in (P, Q)]


@pytest.mark.parametrize("integ", [LFMN2VF, LF2, LFMN2])
@pytest.mark.parametrize("step", [2, 3, 4, 10])
def test_integrator_invariants(lists, integ, step):
    v = lists[("traj", integ, step)]
    assert abs(sum(c for o, c in v if o == Q) - step * EPS) < 1e-15 * step
    assert abs(sum(c for o, c in v if o == P) - step * EPS) < 1e-15 * step
    seq = pq(v)
    assert all(a[0] == b[0] and abs(a[1] - b[1]) < 1e-17 for a, b in zip(seq, reversed(seq))), "not reversible"
    forces = [o for o, _ in v if o in (F_MED, F_HIGH)]
    assert len(forces) == {LFMN2VF: 2 * step + 1, LF2: step + 1, LFMN2: 2 * step}[integ]
    for k, (o, _) in enumerate(v):
        if o in (F_MED, F_HIGH):
            assert v[k + 1][0] == P  # a force is followed by its momentum step
    if integ == LFMN2:
        assert forces == [F_MED] * len(forces) and v[-1] == (S_HIGH, 0.0)
    else:
        assert forces == [F_MED] * (len(forces) - 1) + [F_HIGH] and v[-1][0] == P


@pytest.mark.parametrize("step", [1, 2, 4, 10])
def test_helpers_against_integrators(lists, step):
    t0, e0 = lists[("traj", LFMN2VF, step)], lists[("evolve", LFMN2VF, step)]
    assert e0 == [(S_HIGH, 0.0)] + t0 + [(C_HIGH, 0.0)]
    for integ in (LF2, LFMN2):
        t, e = lists[("traj", integ, step)], lists[("evolve", integ, step)]
        assert pq(e) == pq(t)  # the same MD
        fe = [o for o, _ in e if o in (F_MED, F_HIGH)]
        assert fe == [F_HIGH] + [F_MED] * (len(fe) - 1)
        assert not any(o in (S_HIGH, C_HIGH) for o, _ in e)


def test_single_step_peels_like_the_reference(lists):
    v = lists[("traj", LFMN2VF, 1)]
    # first and last MD step both run: four half sigma steps
    assert [c for o, c in v if o == Q] == [EPS / 2] * 4
    assert len([o for o, _ in v if o in (F_MED, F_HIGH)]) == 5
