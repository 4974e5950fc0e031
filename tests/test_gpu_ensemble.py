"""Batched chains (gn_ensemble_*): many independent sigma-HMC chains of mixed
lattice sizes in persistent kernels per MD step, replayed as a CUDA graph,
with device Philox random numbers.

- Statistics agree with the reference's own chains within statistical errors
  (tests/golden/ensemble_reference_L{8,12,16}.json, made by
  tests/golden/make_ensemble_stats.py) for three beta_s: acceptance,
  <sigma^2>, <|sigma_bar|> and the condensate oriented by the sign of
  sigma_bar (the Z2 symmetry sigma -> -sigma flips tr1 with it; a chain in the
  broken phase stays in one vacuum, so the GPU chains, started independently,
  populate both).  <exp(-dH)> = 1, the identity of a reversible
  area-preserving integrator, holds within the GPU chains' error.
- A chain's trajectory does not depend on the chains beside it: the same chain
  alone and in a mixed ensemble ends bit for bit the same, with and without
  the CUDA graph.
- Chains spread over shards (gn_shard, one rank's chains per shard) end bit
  for bit as they do in one ensemble.
- The autotuner returns a layout and the benchmark's mix of sizes runs.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"


def _sigma0(L, beta, seed):
    return np.random.default_rng(seed).normal(0.0, np.sqrt(2.0 / (4 * beta)), L ** 3)


def test_chain_alone_equals_chain_in_mix():
    import gn_b200 as G
    p = G.Ensemble.params(0.08, 8)
    L0, b0 = 12, 0.85
    s0 = _sigma0(L0, b0, 1)
    with G.Ensemble([L0], [b0], seed=99, stream_ids=[7]) as e:
        e.load_sigma(0, s0)
        e.run(p, 5)
        alone, _ = e.store_sigma(0)
        st_alone = e.stats()[0]
    Ls = [8, 16, L0, 24, 8, 12]
    betas = [0.6, 1.0, b0, 0.7, 1.1, 0.9]
    ids = [3, 4, 7, 5, 6, 8]
    for graph in (True, False):
        with G.Ensemble(Ls, betas, seed=99, stream_ids=ids) as e:
            for c, (L, b) in enumerate(zip(Ls, betas)):
                e.load_sigma(c, s0 if c == 2 else _sigma0(L, b, 10 + c))
            e.run(p, 5, graph=graph)
            mixed, _ = e.store_sigma(2)
            st = e.stats()[2]
            if graph:
                assert e.info()["graph"] == 1
        assert np.array_equal(mixed, alone)
        assert st["accepted"] == st_alone["accepted"] and st["sum_dH"] == st_alone["sum_dH"]


def test_shards_equal_the_whole_ensemble():
    """The chains split over two shards, run one after the other on this GPU
    as two ranks would run them on two, end as the same chains do in one
    ensemble: each shard keys its chains by their global indices."""
    import gn_b200 as G
    import gn_shard as S
    p = G.Ensemble.params(0.08, 8)
    Ls = [8, 16, 12, 24, 8, 12, 16]
    betas = [0.6, 1.0, 0.85, 0.7, 1.1, 0.9, 0.75]
    sig = [_sigma0(L, b, 20 + c) for c, (L, b) in enumerate(zip(Ls, betas))]

    def run(rank, world):
        with S.ShardedEnsemble(Ls, betas, seed=99, rank=rank, world=world) as e:
            for c in range(len(Ls)):
                e.load_sigma(c, sig[c])
            e.run(p, 3)
            return e.mine, {c: e.store_sigma(c)[0] for c in e.mine}, e.stats()

    _, whole, st_whole = run(0, 1)
    seen = []
    for r in range(2):
        mine, part, st = run(r, 2)
        seen += mine
        for c in mine:
            assert np.array_equal(part[c], whole[c]), c
            assert st[c]["accepted"] == st_whole[c]["accepted"] and st[c]["sum_dH"] == st_whole[c]["sum_dH"]
    assert sorted(seen) == list(range(len(Ls)))


@pytest.mark.parametrize("L0", [8, 12, 16])
def test_ensemble_statistics_vs_reference(L0):
    import gn_b200 as G
    ref = json.loads((GOLD / f"ensemble_reference_L{L0}.json").read_text())
    L, nper = ref["L"], 32
    betas = [float(b) for b in ref["betas"]]
    Ls = [L] * (nper * len(betas))
    bet = [b for b in betas for _ in range(nper)]
    p = G.Ensemble.params(ref["eps"], ref["steps"])
    n = len(Ls)
    nchunk, per = 15, 10
    s2 = np.zeros((n, nchunk))
    sbar = np.zeros((n, nchunk))
    acc, emdh = np.zeros(n), np.zeros(n)
    with G.Ensemble(Ls, bet, seed=2024) as e:
        for c, b in enumerate(bet):
            e.load_sigma(c, _sigma0(L, b, 1000 + c))
        e.run(p, 100 if L <= 8 else 200)  # thermalisation
        e.stats(reset=True)
        for k in range(nchunk):
            e.run(p, per)
            st = e.stats(reset=True)
            assert all(s["failed"] == 0 for s in st)
            s2[:, k] = [s["sum_sigma2"] / per for s in st]
            acc += [s["accepted"] for s in st]
            emdh += [s["sum_exp_mdH"] for s in st]
            sbar[:, k] = [abs(np.mean(e.store_sigma(c)[0])) for c in range(n)]
        ntot = nchunk * per
        sigmas = [e.store_sigma(c)[0] for c in range(n)]
    # condensate tr1 on each chain's final configuration (single-lattice path,
    # Z2 noise), oriented by the sign of that configuration's sigma_bar
    rng = np.random.default_rng(5)
    cond = []
    with G.Lattice(L) as lat:
        for s in sigmas:
            out, *_ = lat.condensate(lat.sigma_mass(s), 1e-9, np.zeros(L ** 3, complex),
                                     lambda: float(rng.uniform()))
            cond.append(out[0] * np.sign(np.mean(s)))
    cond = np.array(cond)
    for i, b in enumerate(betas):
        r = ref["betas"][str(b)]
        sl = slice(i * nper, (i + 1) * nper)
        for name, per_chain in (("acceptance", acc[sl] / ntot), ("sigma2", s2[sl].mean(axis=1)),
                                ("abs_sigma_bar", sbar[sl].mean(axis=1)), ("cond_tr1_oriented", cond[sl])):
            m, err = per_chain.mean(), per_chain.std(ddof=1) / np.sqrt(nper)
            tol = 4.0 * np.hypot(err, r[name + "_err"]) + 1e-12
            assert abs(m - r[name]) <= tol, (b, name, m, err, r[name], r[name + "_err"])
        m = (emdh[sl] / ntot).mean()
        err = (emdh[sl] / ntot).std(ddof=1) / np.sqrt(nper)
        assert abs(m - 1.0) <= 5.0 * err + 1e-5, (b, m, err)


def test_autotuner_and_mixed_sizes():
    """The benchmark's mix of lattice sizes: the tuner returns a valid layout,
    every chain runs, dH stays small."""
    import gn_b200 as G
    rng = np.random.default_rng(3)
    Ls = [int(x) for x in rng.choice([8, 12, 16, 24, 32, 48], size=24)]
    bet = list(np.linspace(0.5, 1.2, 24))
    p = G.Ensemble.params(0.08, 8)
    with G.Ensemble(Ls, bet, seed=11) as e:
        for c, (L, b) in enumerate(zip(Ls, bet)):
            e.load_sigma(c, _sigma0(L, b, c))
        gs, vmin = e.tune(p)
        assert gs >= 1
        e.run(p, 3)
        st = e.stats()
    assert all(s["trajectories"] == 3 and s["failed"] == 0 for s in st)
    assert max(abs(s["last_dH"]) for s in st) < 5.0
    assert all(s["cg_iterations"] > 0 for s in st)


@pytest.mark.parametrize("Ls", [[8, 12, 16], [6, 10, 26]])
def test_fp64_and_mixed_chains_agree(Ls):
    """The same chains with FP64 and with mixed-precision solves (both to a
    true relative residual of 1e-10): the trajectories agree to the solver
    tolerance.  The second set has odd half-rows (one-site items), L = 26 on a
    team of several blocks."""
    import gn_b200 as G
    betas = [0.7, 0.9, 1.1]
    out = {}
    for prec in (G.GN_PREC_FP64, G.GN_PREC_MIXED):
        p = G.Ensemble.params(0.08, 8, precision=prec)
        with G.Ensemble(Ls, betas, seed=3) as e:
            for c, (L, b) in enumerate(zip(Ls, betas)):
                e.load_sigma(c, _sigma0(L, b, 50 + c))
            e.run(p, 2)
            out[prec] = ([e.store_sigma(c)[0] for c in range(3)], [s["sum_dH"] for s in e.stats()])
    for a, b in zip(out[G.GN_PREC_FP64][0], out[G.GN_PREC_MIXED][0]):
        assert np.max(np.abs(a - b)) / np.max(np.abs(a)) < 1e-7
    assert np.allclose(out[G.GN_PREC_FP64][1], out[G.GN_PREC_MIXED][1], rtol=0, atol=1e-6)


def test_two_teams_and_lock_step_chains_agree(monkeypatch):
    """A chain's two flavours solved as two teams of half blocks (the
    default) and in lock step on the whole team (GN_ENS_DUO=0): the same
    trajectories to the solver tolerance, on single-block teams (L = 8, 12)
    and on a team of several blocks (L = 24)."""
    import gn_b200 as G
    Ls, betas = [8, 12, 24], [0.7, 0.9, 1.1]
    p = G.Ensemble.params(0.08, 8)
    out = {}
    for duo in ("1", "0"):
        monkeypatch.setenv("GN_ENS_DUO", duo)
        with G.Ensemble(Ls, betas, seed=4) as e:
            e.set_layout(4, 16 ** 3)
            for c, (L, b) in enumerate(zip(Ls, betas)):
                e.load_sigma(c, _sigma0(L, b, 80 + c))
            e.run(p, 2)
            st = e.stats()
            assert all(s["failed"] == 0 for s in st)
            out[duo] = ([e.store_sigma(c)[0] for c in range(3)], [s["sum_dH"] for s in st],
                        [s["accepted"] for s in st])
    for a, b in zip(out["1"][0], out["0"][0]):
        assert np.max(np.abs(a - b)) / np.max(np.abs(a)) < 1e-7
    assert np.allclose(out["1"][1], out["0"][1], rtol=0, atol=1e-6)
    assert out["1"][2] == out["0"][2]


def test_checkpoint_resume_is_exact(tmp_path):
    """Two trajectories, a checkpoint of every chain (the chain's own counters),
    a new ensemble with the same seed and stream ids loading them, two more
    trajectories: bit for bit the chain that ran four trajectories without a
    stop.  The file's done_sigma is the chain's Philox counter."""
    import gn_b200 as G
    Ls, betas = [8, 12], [0.85, 1.0]
    p = G.Ensemble.params(0.08, 4, tol=1e-10)

    def fresh():
        e = G.Ensemble(Ls, betas, seed=2024)
        for c, L in enumerate(Ls):
            e.load_sigma(c, _sigma0(L, betas[c], 31 + c))
        return e

    with fresh() as whole:
        whole.run(p, 4)
        want = [whole.store_sigma(c)[0] for c in range(len(Ls))]
        want_stats = whole.stats()
    with fresh() as first:
        first.run(p, 2)
        for c in range(len(Ls)):
            first.checkpoint_save(c, tmp_path / f"chain{c}.bin")
    with G.Ensemble(Ls, betas, seed=2024) as second:
        for c in range(len(Ls)):
            st, cnt = second.checkpoint_load(c, tmp_path / f"chain{c}.bin")
            assert st == G.GN_OK and cnt["done_sigma"] == 2
        second.run(p, 2)
        for c in range(len(Ls)):
            assert np.array_equal(second.store_sigma(c)[0], want[c])
        got = second.stats()
        for c in range(len(Ls)):
            assert got[c]["total_trajectories"] == 4
            assert got[c]["total_accepted"] == want_stats[c]["total_accepted"]
            assert got[c]["story"] == want_stats[c]["story"]


def test_autoregulation_follows_update_hmc_parameters():
    """UpdateHMCParameters (info.c:123-135) after 100 trajectories: the step
    grows by 1.15 at local acceptance >= 0.85 (a small step) and shrinks by
    1.15 below 0.75 (a large one); the local counters restart."""
    import gn_b200 as G
    Ls, betas = [4, 4], [0.85, 0.85]
    with G.Ensemble(Ls, betas, seed=5) as ens:
        for c in range(2):
            ens.load_sigma(c, _sigma0(4, 0.85, 70 + c))
        ens.set_autoregulation(True)
        acc = [[], []]  # a small step: acceptance near 1
        for _ in range(100):
            ens.run(G.Ensemble.params(0.05, 4, tol=1e-10), 1)
            for c, s in enumerate(ens.stats()):
                acc[c].append(s["last_accepted"])
        st = ens.stats()
        for c in range(2):
            a = sum(acc[c]) / 100.0
            want = 1.15 if a >= 0.85 else 1.08 if a >= 0.8 else 1 / 1.08 if a >= 0.75 else 1 / 1.15
            assert st[c]["epsilon_scale"] == pytest.approx(want, rel=1e-15)
            assert st[c]["local_done"] == 0 and st[c]["local_accepted"] == 0
            assert st[c]["total_trajectories"] == 100
    with G.Ensemble([4], [0.85], seed=6) as ens:  # a large step: acceptance low
        ens.load_sigma(0, _sigma0(4, 0.85, 80))
        ens.set_autoregulation(True)
        acc = []
        for _ in range(100):
            ens.run(G.Ensemble.params(1.5, 4, tol=1e-10), 1)
            acc.append(ens.stats()[0]["last_accepted"])
        a = sum(acc) / 100.0
        want = 1.15 if a >= 0.85 else 1.08 if a >= 0.8 else 1 / 1.08 if a >= 0.75 else 1 / 1.15
        assert a < 0.75
        assert ens.stats()[0]["epsilon_scale"] == pytest.approx(want, rel=1e-15)
