"""Multi-rank host logic on CPU ranks (gloo): sharding of independent
products, max-over-ranks timing, and the cross-rank Chudnovsky merge
(ranks.py), whose root must equal the one-process tree over the same terms
and the reference's own root hash (tests/golden/chudnovsky.json). The
transport and merge order are the ones the GPUs use; the node store is
Python integers here and device-resident b2m_pqt nodes there."""
import hashlib
import json
import multiprocessing as mp
import os
import socket
import traceback

import numpy as np
import pytest

import oracle
import ranks
from golden_util import sha_limbs

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _to_int(sign, mag):
    v = int.from_bytes(np.ascontiguousarray(mag, dtype="<u4").tobytes(), "little")
    return -v if sign < 0 else v


def _limbs(v: int) -> np.ndarray:
    v = abs(v)
    n = (v.bit_length() + 31) // 32
    return np.frombuffer(v.to_bytes(4 * n, "little"), dtype="<u4").copy() if n else np.zeros(0, np.uint32)


class IntBackend:
    """(P, Q, T) as Python integers; subtrees from the oracle's C port of
    chudnovsky_bs; nodes cross ranks as int32 CPU tensors."""

    def bs(self, a, b):
        return tuple(_to_int(s, m) for s, m in oracle.bs_port(a, b))

    def merge(self, left, right):
        pl, ql, tl = left
        pr, qr, tr = right
        return (pl * pr, ql * qr, tl * qr + pl * tr)

    def send(self, r, node, dst):
        import torch

        arrs = [_limbs(v) for v in node]
        sign = (node[2] > 0) - (node[2] < 0)
        r.dist.send(torch.tensor([a.size for a in arrs] + [sign], dtype=torch.int64), dst)
        for a in arrs:
            if a.size:
                r.dist.send(torch.from_numpy(a.view(np.int32)), dst)

    def recv(self, r, src):
        import torch

        h = torch.empty(4, dtype=torch.int64)
        r.dist.recv(h, src)
        lens, sign = [int(x) for x in h[:3]], int(h[3])
        vals = []
        for n in lens:
            t = torch.empty(n, dtype=torch.int32)
            if n:
                r.dist.recv(t, src)
            vals.append(int.from_bytes(t.numpy().view("<u4").tobytes(), "little"))
        return (vals[0], vals[1], -vals[2] if sign < 0 else vals[2])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_terms, q):
    try:
        os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                           "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
        r = ranks.from_env("gloo", timeout_s=60)
        mx = ranks.max_over_ranks(r, float(rank) + 0.5, -float(rank))
        root = ranks.chudnovsky_bs_ranks(r, n_terms, IntBackend())
        ranks.barrier(r)
        ranks.close(r)
        q.put((rank, mx, root))
    except Exception:
        q.put((rank, "error", traceback.format_exc()))


def _run(world, n_terms):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_terms, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, mx, root = q.get(timeout=240)
        assert mx != "error", root
        out[rank] = (mx, root)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_lpt_shard_covers_every_job_once_and_balances():
    rng = np.random.default_rng(5)
    sizes = [(int(2 ** (6 + 10 * x)), int(2 ** (6 + 10 * y))) for x, y in rng.random((4096, 2))]
    costs = [ranks.product_cost(a, b) for a, b in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = ranks.lpt_shard(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        bound = max(sum(costs) / world, max(costs))
        assert max(loads) <= 4 / 3 * bound
        assert parts == ranks.lpt_shard(costs, world)  # every rank computes the same partition


def test_term_ranges_and_schedule():
    for world in range(1, 9):
        rg = ranks.term_ranges(100, world)
        assert rg[0][0] == 0 and rg[-1][1] == 100
        assert all(rg[i][1] == rg[i + 1][0] and rg[i][0] < rg[i][1] for i in range(world - 1))
        # every rank but 0 sends exactly once, always to a lower rank, and a
        # receiving rank has already received everything right of it
        sends = [src for step in ranks.merge_schedule(world) for _, src in step]
        assert sorted(sends) == list(range(1, world))
        held = {r: [r] for r in range(world)}
        for step in ranks.merge_schedule(world):
            for dst, src in step:
                assert held[dst][-1] + 1 == held[src][0]   # adjacent ranges, left then right
                held[dst] += held.pop(src)
        assert held == {0: list(range(world))}
    with pytest.raises(ValueError):
        ranks.term_ranges(2, 3)


def test_ntt_length_matches_the_library_rule():
    assert ranks.ntt_length(60000, 60000) == 1 << 18
    assert ranks.ntt_length(1 << 24, 1 << 24) == 1 << 26
    assert ranks.ntt_length(1, 1) == 4


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_max_and_chudnovsky_merge(world):
    tree = next(t for t in json.load(open(os.path.join(GOLD, "chudnovsky.json")))["trees"] if t["digits"] == 1000)
    n = tree["terms"]
    out = _run(world, n)
    for rank, (mx, root) in out.items():
        assert mx == [world - 1 + 0.5, 0.0]
        assert (root is None) == (rank != 0)
    p, q, t = out[0][1]
    whole = tuple(_to_int(s, m) for s, m in oracle.bs_port(0, n))
    assert (p, q, t) == whole
    for v, nm in zip((p, q, t), "PQT"):
        assert sha_limbs(_limbs(v)) == tree[nm]["sha256"], nm
    assert (1 if t > 0 else -1) == tree["T"]["sign"]
