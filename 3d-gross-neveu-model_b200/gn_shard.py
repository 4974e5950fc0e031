"""Batched chains and served requests spread over the GPUs of one node.

One process per GPU (torch.distributed, NCCL or gloo, set up by the caller;
with NCCL the rank's device must be current, torch.cuda.set_device, since the
gathers stage their bytes there).
Chains shard without a collective on the data path: a chain lives on one rank
for its whole life and keeps its global index as its Philox stream, so its
trajectories are the same on any rank and beside any other chains (the
batched kernel's chains never read each other's data).  Every rank computes
the same owner map from the chain list alone; ranks exchange only host-side
summaries after a run (all_gather_object), never lattice fields.

The reference runs one lattice per process (its chains are separate runs of
the program, simulation.c's main loop); this layer is the batched path's
counterpart of starting those runs on several GPUs at once.
"""
from __future__ import annotations

import heapq

import numpy as np


def chain_cost(L: int) -> int:
    """Relative cost of one trajectory of an L^3 chain: V sites times a solve
    length that grows about like L."""
    return int(L) ** 4


def shard_chains(Ls, world: int) -> list[int]:
    """Owner rank of every chain.  Longest processing time first: chains by
    falling cost (ties by index) each go to the rank with the least cost so
    far (ties by rank), so the map depends only on the chain list and every
    rank computes the same one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    owner = [0] * len(Ls)
    heap = [(0, r) for r in range(world)]
    for c in sorted(range(len(Ls)), key=lambda c: (-chain_cost(Ls[c]), c)):
        load, r = heapq.heappop(heap)
        owner[c] = r
        heapq.heappush(heap, (load + chain_cost(Ls[c]), r))
    return owner


class OnlineBalancer:
    """Owner ranks for chains that arrive one at a time (a server's
    add_chain): each goes to the rank with the least cost so far, ties by
    rank.  The same call sequence gives the same map on every rank."""

    def __init__(self, world: int):
        if world < 1:
            raise ValueError("world must be >= 1")
        self.load = [0] * world
        self.owner: list[int] = []

    def add(self, L: int) -> int:
        r = min(range(len(self.load)), key=lambda q: (self.load[q], q))
        self.load[r] += chain_cost(L)
        self.owner.append(r)
        return r


def rank_world(group=None) -> tuple[int, int]:
    """(rank, world size) of the process group, (0, 1) without one."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def gather_objects(obj, group=None) -> list:
    """Every rank's obj, in rank order, on every rank (host objects only)."""
    import torch.distributed as dist
    rank, world = rank_world(group)
    if world == 1:
        return [obj]
    out = [None] * world
    dist.all_gather_object(out, obj, group=group)
    return out


class ShardedEnsemble:
    """An ensemble of chains over the ranks of a process group, one GPU each.

    Rank r runs the chains `shard_chains` gives it as one Ensemble, keyed by
    their global indices.  Calls that name a chain (load_sigma, store_sigma,
    set_autoregulation, checkpoints) may be made on every rank and act only
    on the owner; run, tune and set_layout act on each rank's own chains;
    stats and observables are collective and return every chain's entry, in
    global order, on every rank.

    rank and world, when given, name a shard without a process group (one
    process running the shards one after another; stats and observables then
    fill only its own chains' entries: None, or a row of NaN, for the rest)."""

    def __init__(self, Ls, betas, seed=1231, device=0, group=None, ensemble_factory=None, rank=None, world=None):
        if len(Ls) != len(betas):
            raise ValueError("Ls and betas differ in length")
        self.group = group
        self.rank, self.world = rank_world(group) if world is None else (int(rank), int(world))
        if not 0 <= self.rank < self.world:
            raise ValueError("rank outside [0, world)")
        self._solo = world is not None
        self.Ls = [int(x) for x in Ls]
        self.n = len(self.Ls)
        self.owner = shard_chains(self.Ls, self.world)
        self.mine = [c for c in range(self.n) if self.owner[c] == self.rank]
        self._local = {c: i for i, c in enumerate(self.mine)}
        if ensemble_factory is None:
            import gn_b200 as G
            ensemble_factory = G.Ensemble
        self.ens = None
        if self.mine:
            self.ens = ensemble_factory([self.Ls[c] for c in self.mine], [float(betas[c]) for c in self.mine],
                                        seed=seed, stream_ids=list(self.mine), device=device)

    def close(self):
        if self.ens is not None:
            self.ens.close()
            self.ens = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def owns(self, c: int) -> bool:
        return c in self._local

    def local_index(self, c: int):
        """Index of chain c in this rank's Ensemble, None if another rank owns it."""
        return self._local.get(c)

    def load_sigma(self, c, sigma):
        if self.owns(c):
            self.ens.load_sigma(self._local[c], sigma)

    def store_sigma(self, c):
        """(sigma, sigmamass) of chain c on its owner, None elsewhere."""
        return self.ens.store_sigma(self._local[c]) if self.owns(c) else None

    def set_layout(self, group_blocks, big_min_volume):
        if self.ens is not None:
            self.ens.set_layout(group_blocks, big_min_volume)

    def tune(self, p):
        """Each rank tunes the layout of its own chains; returns this rank's."""
        return self.ens.tune(p) if self.ens is not None else None

    def run(self, p, ntraj, graph=True):
        if self.ens is not None:
            self.ens.run(p, ntraj, graph)

    def set_autoregulation(self, on=True, chain=-1):
        if self.ens is None:
            return
        if chain < 0:
            self.ens.set_autoregulation(on, -1)
        elif self.owns(chain):
            self.ens.set_autoregulation(on, self._local[chain])

    def checkpoint_save(self, c, path, path_copy=None, counters=None):
        if self.owns(c):
            self.ens.checkpoint_save(self._local[c], path, path_copy, counters)

    def checkpoint_load(self, c, path, path_copy=None):
        return self.ens.checkpoint_load(self._local[c], path, path_copy) if self.owns(c) else None

    def _gathered(self, local):
        parts = [(self.mine, local)] if self._solo else gather_objects((self.mine, local), self.group)
        out = [None] * self.n
        for chains, vals in parts:
            for c, v in zip(chains, vals):
                out[c] = v
        return out

    def stats(self, reset=False):
        """Every chain's statistics (Ensemble.stats entries), global order."""
        return self._gathered(self.ens.stats(reset) if self.ens is not None else [])

    def observables(self):
        """(nchains, 8) per-chain means of the sigma observables, global order."""
        local = [np.asarray(v, np.float64) for v in self.ens.observables()] if self.ens is not None else []
        return np.array([np.full(8, np.nan) if v is None else v for v in self._gathered(local)], dtype=np.float64)


class ShardedServer:
    """A request server over the ranks of a process group, one GPU each.

    Every rank makes the same add_chain and submit calls in the same order
    (the request stream is the input, replicated); a rank keeps only the
    chains that an OnlineBalancer gives it and the requests on them, so
    routing needs no message.  Chains and requests are named by global
    indices: the add_chain order and the submit order.

    rank and world, when given, name a shard without a process group (as for
    ShardedEnsemble; gather_requests then returns only its own requests)."""

    def __init__(self, traj_params, mem_budget_bytes=8e9, seed=1231, tiers=None, device=0, group=None,
                 server_factory=None, rank=None, world=None):
        self.group = group
        self.rank, self.world = rank_world(group) if world is None else (int(rank), int(world))
        if not 0 <= self.rank < self.world:
            raise ValueError("rank outside [0, world)")
        self._solo = world is not None
        self.balancer = OnlineBalancer(self.world)
        if server_factory is None:
            import gn_b200 as G
            server_factory = G.Server
        kw = {} if tiers is None else {"tiers": tiers}
        self.srv = server_factory(traj_params, mem_budget_bytes=mem_budget_bytes, seed=seed, device=device, **kw)
        self.chain_local: dict[int, int] = {}
        self.chain_global: dict[int, int] = {}
        self.req_local: dict[int, int] = {}
        self.nreq = 0

    def close(self):
        if self.srv is not None:
            self.srv.close()
            self.srv = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def owner(self):
        return self.balancer.owner

    def add_chain(self, L, beta_s, sigma, stream_id=None):
        """Global chain index; the chain's Philox stream defaults to it.
        sigma may be a callable returning the field, called on the owner only
        (the other ranks need not build it)."""
        c = len(self.balancer.owner)
        r = self.balancer.add(L)
        if r == self.rank:
            if callable(sigma):
                sigma = sigma()
            lc = self.srv.add_chain(L, beta_s, sigma, c if stream_id is None else stream_id)
            self.chain_local[c] = lc
            self.chain_global[lc] = c
        return c

    def clock(self):
        return self.srv.clock()

    def submit(self, chain, rtype, noise_vectors=0, t_arrival=None):
        """Global request id (taken on every rank, kept by the chain's owner)."""
        rid = self.nreq
        self.nreq += 1
        if chain in self.chain_local:
            self.req_local[rid] = self.srv.submit(self.chain_local[chain], rtype, noise_vectors, t_arrival)
        return rid

    def step(self):
        return self.srv.step() if self.chain_local else 0

    def load(self):
        return self.srv.load()

    def drain(self, max_steps=100000):
        if self.chain_local:
            self.srv.drain(max_steps)

    def request(self, rid):
        """The request's record on the owner rank (its id and chain global),
        None elsewhere."""
        if rid not in self.req_local:
            return None
        rec = dict(self.srv.request(self.req_local[rid]))
        rec["id"], rec["chain"] = rid, self.chain_global[rec["chain"]]
        return rec

    def solution(self, rid):
        return self.srv.solution(self.req_local[rid]) if rid in self.req_local else None

    def chain_sigma(self, c):
        return self.srv.chain_sigma(self.chain_local[c]) if c in self.chain_local else None

    def gather_requests(self, rids):
        """{rid: record} for the given global ids, from their owners, on every
        rank (collective)."""
        local = {rid: self.request(rid) for rid in rids if rid in self.req_local}
        out = {}
        for part in [local] if self._solo else gather_objects(local, self.group):
            out.update(part)
        return out
