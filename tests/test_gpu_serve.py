"""The request server (gn_server_*): continuous batching of trajectory, solve
and condensate requests on resident chains.

- A request's result does not depend on the requests beside it: the same
  chain's requests give the same bits alone and inside a mixed load, and on
  one server or on the shard (gn_shard) that owns its chain.
- A solve request solves (M M^T) x = b for its b ~ N(0, 1): b regenerated on
  the host from the same Philox counters gives a true relative residual
  below 1e-9 with the CPU restatement's operator.
- The condensate estimate is unbiased: its mean over requests at fixed sigma
  agrees with tr M^-1 / V from a dense inverse at L = 8.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 77


def _sigma0(L, beta, seed):
    return np.random.default_rng(seed).normal(0.0, np.sqrt(2.0 / (4 * beta)), L ** 3)


M64 = (1 << 64) - 1


def _philox(ctr, key):
    c, k = list(ctr), list(key)
    for _ in range(10):
        p0 = 0xD2E7470EE14C6C93 * c[0]
        p1 = 0xCA5A826395121157 * c[2]
        c = [(p1 >> 64) ^ c[1] ^ k[0], p1 & M64, (p0 >> 64) ^ c[3] ^ k[1], p0 & M64]
        k = [(k[0] + 0x9E3779B97F4A7C15) & M64, (k[1] + 0xBB67AE8584CAA73B) & M64]
    return c


def _rhs(V, seed, stream, serial):
    """The solve request's right-hand side: Philox field 4, four sites per block."""
    b = np.empty(V)
    for q in range(V // 4):
        r = _philox([q, 4, serial, 0], [seed, stream])
        for h in range(2):
            u1 = ((r[2 * h] >> 11) + 1) / 9007199254740992.0
            u2 = (r[2 * h + 1] >> 11) / 9007199254740992.0
            rad = math.sqrt(-2.0 * math.log(u1))
            b[4 * q + 2 * h] = rad * math.cos(2 * math.pi * u2)
            b[4 * q + 2 * h + 1] = rad * math.sin(2 * math.pi * u2)
    return b


def _server(G, **kw):
    return G.Server(G.Ensemble.params(0.08, 8), seed=SEED, **kw)


def _target_requests(G, s, c):
    ids = [s.submit(c, G.GN_REQ_TRAJECTORY), s.submit(c, G.GN_REQ_SOLVE), s.submit(c, G.GN_REQ_CONDENSATE, 16),
           s.submit(c, G.GN_REQ_TRAJECTORY)]
    return ids


def _results(s, ids, c):
    info = [s.request(i) for i in ids]
    assert all(x["status"] == 2 and x["failed"] == 0 for x in info)
    return {"dH": [info[0]["dH"], info[3]["dH"]], "acc": [info[0]["accepted"], info[3]["accepted"]],
            "x": s.solution(ids[1]), "cond": info[2]["value"], "sigma": s.chain_sigma(c)}


def test_request_alone_equals_request_in_mix():
    import gn_b200 as G
    L0, b0 = 16, 0.8
    with _server(G) as s:
        c = s.add_chain(L0, b0, _sigma0(L0, b0, 1), stream_id=42)
        ids = _target_requests(G, s, c)
        s.drain()
        alone = _results(s, ids, c)
    rng = np.random.default_rng(9)
    with _server(G) as s:
        others = []
        for k, L in enumerate([8, 24, 32, 12, 16, 48, 8]):
            b = float(rng.uniform(0.6, 1.1))
            others.append(s.add_chain(L, b, _sigma0(L, b, 100 + k), stream_id=1000 + k))
        for o in others[:4]:
            s.submit(o, G.GN_REQ_TRAJECTORY)
        c = s.add_chain(L0, b0, _sigma0(L0, b0, 1), stream_id=42)
        ids = []
        for k, rtype in enumerate([G.GN_REQ_TRAJECTORY, G.GN_REQ_SOLVE, G.GN_REQ_CONDENSATE, G.GN_REQ_TRAJECTORY]):
            ids.append(s.submit(c, rtype, 16 if rtype == G.GN_REQ_CONDENSATE else 0))
            s.submit(others[k % len(others)], G.GN_REQ_SOLVE)
            s.submit(others[(k + 3) % len(others)], G.GN_REQ_CONDENSATE, 8)
            s.step()
        s.drain()
        mixed = _results(s, ids, c)
    assert mixed["dH"] == alone["dH"] and mixed["acc"] == alone["acc"]
    assert np.array_equal(mixed["x"], alone["x"])
    assert mixed["cond"] == alone["cond"]
    assert np.array_equal(mixed["sigma"], alone["sigma"])


def test_sharded_server_equals_one_server():
    """The same request stream on one server and on two shards (run one after
    the other on this GPU, as two ranks would on two): every request ends
    with the same bits on the shard that owns its chain."""
    import gn_b200 as G
    import gn_shard as S
    Ls = [8, 24, 16, 12, 32, 16]
    rng = np.random.default_rng(13)
    betas = [float(b) for b in rng.uniform(0.6, 1.1, len(Ls))]
    kinds = [(G.GN_REQ_TRAJECTORY, 0), (G.GN_REQ_SOLVE, 0), (G.GN_REQ_CONDENSATE, 8)]
    stream = [(int(c), kinds[int(k)]) for c, k in zip(rng.integers(0, len(Ls), 18), rng.integers(0, 3, 18))]

    def serve(rank, world):
        with S.ShardedServer(G.Ensemble.params(0.08, 8), seed=SEED, rank=rank, world=world) as s:
            for c, (L, b) in enumerate(zip(Ls, betas)):
                s.add_chain(L, b, _sigma0(L, b, 200 + c))
            rids = []
            for k, (c, (t, nv)) in enumerate(stream):
                rids.append(s.submit(c, t, nv))
                if k % 4 == 3:
                    s.step()
            s.drain()
            recs = s.gather_requests(rids)
            sol = {r: s.solution(r) for r in recs if recs[r]["type"] == G.GN_REQ_SOLVE}
            sig = {c: s.chain_sigma(c) for c in range(len(Ls)) if c in s.chain_local}
            return recs, sol, sig

    whole, wsol, wsig = serve(0, 1)
    assert len(whole) == len(stream) and all(r["status"] == 2 and r["failed"] == 0 for r in whole.values())
    got = {}
    for r in range(2):
        recs, sol, sig = serve(r, 2)
        got.update(recs)
        for rid, rec in recs.items():
            w = whole[rid]
            assert rec["chain"] == w["chain"] and rec["type"] == w["type"]
            assert (rec["dH"], rec["accepted"], rec["value"]) == (w["dH"], w["accepted"], w["value"]), rid
        for rid, x in sol.items():
            assert np.array_equal(x, wsol[rid])
        for c, sg in sig.items():
            assert np.array_equal(sg, wsig[c])
    assert sorted(got) == sorted(whole)


def test_solve_request_residual(port):
    import gn_b200 as G
    L, beta = 16, 0.85
    sigma = _sigma0(L, beta, 3)
    with _server(G) as s:
        c = s.add_chain(L, beta, sigma, stream_id=5)
        rid = s.submit(c, G.GN_REQ_SOLVE)
        s.drain()
        info = s.request(rid)
        x = s.solution(rid)
    assert info["cg_iterations"] > 0
    b = _rhs(L ** 3, SEED, 5, 0)  # the chain's first request: serial 0
    sm = port.sigma_mass(L, sigma)
    Ax = port.dirac(L, sm, port.dirac(L, sm, x, 1), 0)
    assert np.linalg.norm(b - Ax) / np.linalg.norm(b) < 1e-9


def test_condensate_request_unbiased(port):
    import gn_b200 as G
    L, beta = 8, 0.85
    V = L ** 3
    sigma = _sigma0(L, beta, 4)
    sm = port.sigma_mass(L, sigma)
    M = np.stack([port.dirac(L, sm, np.eye(V)[j], 0) for j in range(V)], axis=1)
    exact = np.trace(np.linalg.inv(M)) / V
    with _server(G) as s:
        c = s.add_chain(L, beta, sigma, stream_id=6)
        ids = [s.submit(c, G.GN_REQ_CONDENSATE, 64) for _ in range(12)]
        s.drain()
        vals = np.array([s.request(i)["value"] for i in ids])
    err = vals.std(ddof=1) / np.sqrt(len(vals))
    assert abs(vals.mean() - exact) < 5 * err + 1e-12, (vals.mean(), err, exact)
