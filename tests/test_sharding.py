"""Multi-GPU host logic on the CPU: the first-index partition and the one exchange step
(two MIN all-reduces), run as world_size-2 gloo process groups.  Each rank's shard
result comes from the oracle restricted to that rank's first indices, so the exchange
must reproduce the oracle's global best (lowest score, ties to the lowest index)."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "cross-dpc-episdet_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from epik2 import sharding as SH  # noqa: E402


def _tri(m):
    return m * (m - 1) * (m - 2) // 6 if m >= 3 else 0


@pytest.mark.parametrize("m", [0, 1, 3, 4, 5, 10, 100, 1000, 4096])
@pytest.mark.parametrize("parts", [1, 2, 3, 8, 64, 200])
def test_shard_bounds_cover_and_balance(m, parts):
    b = SH.shard_bounds(m, parts)
    assert len(b) == parts
    assert b[0][0] == 0 and b[-1][1] == m
    for (lo, hi), (lo2, _) in zip(b, b[1:]):
        assert lo <= hi == lo2
    work = [SH.triplets_in(m, lo, hi) for lo, hi in b]
    assert sum(work) == _tri(m)
    biggest = SH.triplets_of_first(m, 0)
    assert max(work) <= _tri(m) / parts + biggest


def test_key_orders():
    rng = np.random.default_rng(0)
    xs = np.sort(rng.uniform(0, 1e6, 500).astype(np.float32))
    bits = [SH.score_bits(float(x)) for x in xs]
    assert bits == sorted(bits)
    assert SH.score_bits(float(np.finfo(np.float32).max)) < SH.NO_SCORE_BITS
    trip = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3), (2, 3, 2000000), (2000000, 2000001, 2000002)]
    keys = [SH.pack_index(*t) for t in trip]
    assert keys == sorted(keys) and all(SH.unpack_index(k) == t for k, t in zip(keys, trip))
    assert max(keys) < SH.NO_INDEX


class OracleShardContext:
    """Stands in for a device context on the CPU: `scan` over a first-index range answers
    from the oracle's full score list restricted to that range (lowest index on ties)."""

    def __init__(self, g, p):
        import oracle as O
        self.m = g.shape[1]
        r = O.scan(g, p, with_tables=True)
        self.scores = r["scores"]
        self.trip = O.triplet_list(self.m)
        self.first = np.array([t[0] for t in self.trip], dtype=np.int64)
        self.calls = []

    def info(self, dataset):
        return {"n_snps": self.m}

    def scan(self, dataset, snp_begin=0, snp_end=0, **opts):
        self.calls.append((snp_begin, snp_end))
        sel = np.nonzero((self.first >= snp_begin) & (self.first < snp_end))[0]
        t = sel[np.argmin(self.scores[sel])]

        class B:
            score = float(self.scores[t])
            ijk = self.trip[t]
        return B()


def _rank_main(rank, world, port, cases, q):
    import torch.distributed as dist
    import oracle as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        out = []
        for kind, arg in cases:
            if kind == "scan":
                seed, S, M, cases_n, parts, planted = arg
                g, p = O.gen_hwe(seed, S, M, cases_n, planted=planted, effects=[0.8] * len(planted))
                ctx = OracleShardContext(g, p)
                out.append((SH.scan_sharded(ctx, 0, rank, world, parts=parts), ctx.calls))
            else:  # explicit per-rank candidates
                cand = arg[rank]
                out.append((SH.exchange_best(*(cand if cand else (None, None))), None))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _run_world(cases, world=2):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, out = q.get(timeout=300)
        res[r] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


SCAN_CASES = [
    ("scan", (11, 300, 16, 140, 2, [])),
    ("scan", (12, 500, 20, 250, 5, [(3, 9, 17)])),
    ("scan", (13, 200, 9, 80, 8, [])),       # more parts than useful first indices: empty shards
    ("scan", (14, 64, 3, 32, 2, [])),        # one triplet: rank 1 holds nothing
]
FIXED_CASES = [
    ("fixed", [(5.5, (5, 6, 7)), (5.5, (1, 2, 3))]),    # tie: lowest index wins
    ("fixed", [(5.25, (1, 2, 9)), (5.5, (0, 1, 2))]),   # lower score beats lower index
    ("fixed", [None, (7.0, (2, 3, 4))]),                # a rank with no triplet
    ("fixed", [None, None]),
]


def test_exchange_world2_matches_oracle():
    import oracle as O
    res = _run_world(SCAN_CASES + FIXED_CASES)
    for t, (kind, arg) in enumerate(SCAN_CASES):
        seed, S, M, n_cases, parts, planted = arg
        g, p = O.gen_hwe(seed, S, M, n_cases, planted=planted, effects=[0.8] * len(planted))
        ref = O.scan(g, p)
        for rank in (0, 1):
            (score, ijk), calls = res[rank][t]
            assert ijk == ref["ijk"]
            assert SH.score_bits(score) == SH.score_bits(ref["score"])
        # the two ranks together scanned every non-empty shard exactly once
        scanned = sorted(res[0][t][1] + res[1][t][1])
        bounds = [b for b in SH.shard_bounds(M, parts) if SH.triplets_in(M, *b) > 0]
        assert scanned == sorted(bounds)
    expect = [(5.5, (1, 2, 3)), (5.25, (1, 2, 9)), (7.0, (2, 3, 4)), (None, None)]
    for t, e in enumerate(expect):
        for rank in (0, 1):
            assert res[rank][len(SCAN_CASES) + t][0] == e
