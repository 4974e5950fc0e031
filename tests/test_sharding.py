"""Chains and requests spread over ranks (gn_shard), on CPU ranks.

The batched chains and the server shard with no exchange on the data path:
every rank computes the same owner map and keeps its own chains; the ranks
meet only to gather host-side results.  These tests check the owner maps and
run that logic as two gloo processes, with stand-ins for the GPU ensemble
and server that record what each rank was given; and bench.py's serving on
N GPUs the same way, with a server that only keeps time.
"""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "3d-gross-neveu-model_b200"))

import gn_shard as S  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_chains_partitions_and_balances():
    rng = np.random.default_rng(3)
    Ls = [int(x) for x in rng.choice([8, 12, 16, 24, 32, 48], size=256)]
    for world in (1, 2, 3, 4, 8):
        owner = S.shard_chains(Ls, world)
        assert owner == S.shard_chains(list(Ls), world)  # a function of the list alone
        assert sorted(set(owner)) == list(range(world))
        load = [sum(S.chain_cost(L) for L, r in zip(Ls, owner) if r == q) for q in range(world)]
        # longest processing time first: no rank exceeds another by more than one chain
        assert max(load) - min(load) <= max(S.chain_cost(L) for L in Ls)
    assert S.shard_chains([], 4) == []
    assert S.shard_chains([8, 8], 4) == [0, 1]


def test_online_balancer_is_deterministic():
    Ls = [8, 64, 16, 16, 32, 8, 48, 24]
    a, b = S.OnlineBalancer(3), S.OnlineBalancer(3)
    ra = [a.add(L) for L in Ls]
    assert ra == [b.add(L) for L in Ls] == a.owner
    assert ra[:3] == [0, 1, 2]  # the first chains fill the empty ranks in order
    assert ra[3] == 0  # then the least loaded (rank 0 holds only an L = 8 chain)


class FakeEnsemble:
    """Records its chains; stats and observables name each chain's stream."""

    def __init__(self, Ls, betas, seed, stream_ids, device):
        self.Ls, self.betas, self.ids = list(Ls), list(betas), list(stream_ids)
        self.loaded, self.runs = {}, 0

    def load_sigma(self, c, sigma):
        self.loaded[self.ids[c]] = float(sigma[0])

    def run(self, p, ntraj, graph=True):
        self.runs += ntraj

    def stats(self, reset=False):
        return [{"stream": i, "L": L, "accepted": self.runs} for i, L in zip(self.ids, self.Ls)]

    def observables(self):
        return np.array([[float(i)] * 8 for i in self.ids])

    def close(self):
        pass


class FakeServer:
    def __init__(self, traj_params, mem_budget_bytes, seed, device, **kw):
        self.chains, self.reqs = [], []

    def add_chain(self, L, beta_s, sigma, stream_id):
        self.chains.append((L, stream_id))
        return len(self.chains) - 1

    def submit(self, chain, rtype, noise_vectors, t_arrival):
        self.reqs.append((chain, rtype))
        return len(self.reqs) - 1

    def request(self, rid):
        c, t = self.reqs[rid]
        return {"id": rid, "chain": c, "type": t, "status": 2}

    def close(self):
        pass


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank))
    sys.path.insert(0, str(ROOT / "3d-gross-neveu-model_b200"))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2)
    import gn_shard as S2
    Ls = [8, 48, 16, 32, 12, 24, 8, 16]
    betas = np.linspace(0.5, 1.2, len(Ls))
    out = {}
    with S2.ShardedEnsemble(Ls, betas, seed=5, ensemble_factory=FakeEnsemble) as e:
        for c in range(len(Ls)):  # every rank makes every call; the owner acts
            e.load_sigma(c, np.full(Ls[c] ** 3, float(c)))
        e.run(None, 3)
        out["mine"] = e.mine
        out["loaded"] = e.ens.loaded
        out["stats"] = e.stats()
        out["obs"] = e.observables().tolist()
    srv = S2.ShardedServer(None, server_factory=FakeServer)
    for c, L in enumerate(Ls):
        assert srv.add_chain(L, 0.8, None) == c
    rids = [srv.submit(c % len(Ls), c % 3) for c in range(20)]
    out["rids"] = rids
    out["server_chains"] = srv.srv.chains
    out["owner"] = srv.owner
    out["requests"] = {str(k): v for k, v in srv.gather_requests(rids).items()}
    (Path(out_dir) / f"rank{rank}.json").write_text(json.dumps(out))
    dist.destroy_process_group()


def test_sharded_ensemble_and_server_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(free_port(), str(tmp_path)), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    Ls = [8, 48, 16, 32, 12, 24, 8, 16]
    owner = S.shard_chains(Ls, 2)
    for r in range(2):
        g = got[r]
        assert g["mine"] == [c for c in range(len(Ls)) if owner[c] == r]
        # each chain's sigma reached its owner only, under its global stream
        assert {int(k): v for k, v in g["loaded"].items()} == {c: float(c) for c in g["mine"]}
        # gathered results: every chain, global order, the same on both ranks
        assert [s["stream"] for s in g["stats"]] == list(range(len(Ls)))
        assert [s["L"] for s in g["stats"]] == Ls
        assert all(s["accepted"] == 3 for s in g["stats"])
        assert [row[0] for row in g["obs"]] == list(range(len(Ls)))
        # the server: chains by the online map, streams = global indices
        assert [c for c, q in enumerate(g["owner"]) if q == r] == [s for _, s in g["server_chains"]]
        assert g["rids"] == list(range(20))
        assert sorted(int(k) for k in g["requests"]) == list(range(20))
        for k, rec in g["requests"].items():
            assert rec["id"] == int(k) and rec["chain"] == int(k) % len(Ls) and rec["type"] == int(k) % 3
    assert got[0]["requests"] == got[1]["requests"]
    assert got[0]["owner"] == got[1]["owner"]
    assert set(got[0]["mine"]).isdisjoint(got[1]["mine"])


def test_explicit_shard_without_a_group():
    Ls = [8, 16, 24]
    e = S.ShardedEnsemble(Ls, [0.6, 0.8, 1.0], ensemble_factory=FakeEnsemble, rank=1, world=2)
    mine = e.mine
    assert mine == [c for c, r in enumerate(S.shard_chains(Ls, 2)) if r == 1]
    st = e.stats()
    assert [s is None for s in st] == [c not in mine for c in range(3)]
    obs = e.observables()
    assert np.isnan(obs[[c for c in range(3) if c not in mine]]).all()


class ClockServer:
    """A server stand-in with a host clock: a step completes every running
    request and admits the queued ones."""

    def __init__(self, traj_params, mem_budget_bytes, seed, device, **kw):
        import time
        self.t0 = time.perf_counter()
        self.chains, self.reqs, self.queue, self.running = [], [], [], []

    def clock(self):
        import time
        return time.perf_counter() - self.t0

    def add_chain(self, L, beta_s, sigma, stream_id):
        assert np.asarray(sigma).size == L ** 3  # built on the owner only
        self.chains.append(L)
        return len(self.chains) - 1

    def submit(self, chain, rtype, noise_vectors, t_arrival):
        self.reqs.append({"chain": chain, "type": rtype, "t_arrival": t_arrival, "t_done": None, "failed": 0})
        self.queue.append(len(self.reqs) - 1)
        return len(self.reqs) - 1

    def load(self):
        return {"running": len(self.running), "queued": len(self.queue), "bytes_in_use": 0}

    def step(self):
        for r in self.running:
            self.reqs[r]["t_done"] = self.clock()
        self.running, self.queue = self.queue, []
        return 0

    def request(self, rid):
        return dict(self.reqs[rid])

    def close(self):
        pass


def _fake_gn():
    import types
    G = types.SimpleNamespace(GN_REQ_TRAJECTORY=0, GN_REQ_SOLVE=1, GN_REQ_CONDENSATE=2, Server=ClockServer)
    G.Ensemble = types.SimpleNamespace(params=lambda eps, steps: (eps, steps))
    return G


def _serve_rank(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK="0")
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    world, r, _ = bench.dist_setup("gloo")
    out = bench.serve_sharded_bench(_fake_gn(), world, rate_per_gpu=400.0, nreq_per_gpu=200)
    (Path(out_dir) / f"serve{r}.json").write_text(json.dumps(out))
    dist.destroy_process_group()


def test_sharded_serving_bench_gloo(tmp_path):
    """bench.py's serving on N GPUs, as two gloo ranks with a clock-only
    server: every request is served once, on its chain's owner, and both
    ranks report the same gathered figures."""
    import torch.multiprocessing as mp
    mp.spawn(_serve_rank, args=(free_port(), str(tmp_path)), nprocs=2, join=True)
    got = [json.loads((tmp_path / f"serve{r}.json").read_text()) for r in range(2)]
    for g in got:
        assert g["n_gpus"] == 2 and g["requests"] == 400 and g["failed"] == 0
        assert sum(g["requests_per_rank"]) == 400 and min(g["requests_per_rank"]) > 0
        assert g["throughput_req_per_s"] > 0 and g["p99_ms"] >= g["p50_ms"] >= 0
    assert got[0] == got[1]
