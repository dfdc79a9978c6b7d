"""Serving form: continuous-batching request server (GPU).

Each request's results must be the same alone and in the mix (bit-exact FP32 scores,
identical triplets), and equal the plain search / oracle on the same phenotype."""
import threading

import numpy as np
import pytest

import epik2
import oracle as O
from conftest import f32_bits

pytestmark = pytest.mark.gpu


def _perms(p, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.permutation(p) for _ in range(n)])


def test_request_same_alone_and_in_the_mix():
    gA, pA = O.gen_hwe(91, 700, 90, 300, planted=[(3, 40, 77)], effects=[0.8])
    gB, pB = O.gen_hwe(92, 1200, 60, 600)
    reps = _perms(pA, 6, 1)
    with epik2.Server(0, rescore_fp64=1, batch_work=5e9) as srv:
        A = srv.add_matrix(gA, pA)
        B = srv.add_matrix(gB, pB)
        st, alone, lat = srv.wait(srv.submit_replicates(A, reps))
        assert st == epik2.OK and len(alone) == 6 and lat > 0
        # the same request among others submitted from several threads
        ids, lock = [], threading.Lock()

        def client(seed):
            rng = np.random.default_rng(seed)
            for t in range(4):
                if t % 2:
                    rid = srv.submit_replicates(B, _perms(pB, int(rng.integers(2, 6)), seed * 10 + t))
                else:
                    g, p = O.gen_hwe(seed * 100 + t, 400, int(rng.integers(20, 50)), 200)
                    rid = srv.submit_scan(g, p)
                with lock:
                    ids.append(rid)

        threads = [threading.Thread(target=client, args=(s,)) for s in range(3)]
        for t in threads:
            t.start()
        mine = srv.submit_replicates(A, reps)
        for t in threads:
            t.join()
        st, mixed, _ = srv.wait(mine)
        others = [srv.wait(r) for r in ids]
        stats = srv.stats()
    assert st == epik2.OK
    for a, b in zip(alone, mixed):
        assert a.ijk == b.ijk and f32_bits(a.score) == f32_bits(b.score) and a.score_fp64 == b.score_fp64
    assert all(o[0] == epik2.OK for o in others)
    assert stats["completed"] == 2 + len(ids) and stats["launches"] >= 2
    for r, a in zip(reps, alone):
        ref = O.scan(gA, r)
        assert a.ijk == ref["ijk"] and f32_bits(a.score) == f32_bits(ref["score"])
        assert abs(a.score - a.score_fp64) / a.score_fp64 <= 1e-5


def test_replicate_dataset_shares_genotypes():
    g, p = O.gen_hwe(93, 800, 70, 300)
    q = np.random.default_rng(5).permutation(p)
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        rep = ctx.load_replicate(base, q)
        b = ctx.scan(rep)
        with pytest.raises(epik2.Epik2Error) as e:
            ctx.unload(base)  # still shared
        assert e.value.status == epik2.E_BUSY
        ctx.unload(rep)
        ctx.unload(base)
    r = O.scan(g, q)
    assert b.ijk == r["ijk"] and f32_bits(b.score) == f32_bits(r["score"])
    assert epik2.library().epik2_replicate_bytes(800, 70) < epik2.dataset_bytes(800, 70)


def test_cancel_refuse_and_unknown():
    g, p = O.gen_hwe(94, 500, 40, 200)
    with epik2.Server(0, max_queued=8) as srv:
        m = srv.add_matrix(g, p)
        with pytest.raises(epik2.Epik2Error) as e:
            srv.submit_replicates(m, _perms(p, 9, 2))  # more scans than the queue allows
        assert e.value.status == epik2.E_BUSY
        with pytest.raises(epik2.Epik2Error) as e:
            srv.submit_replicates(99, _perms(p, 1, 2))
        assert e.value.status == epik2.E_NOT_FOUND
        rid = srv.submit_replicates(m, _perms(p, 4, 3))
        srv.cancel(rid)
        st, res, _ = srv.wait(rid)
        assert st in (epik2.OK, epik2.E_CANCELLED)  # may have run before the cancel landed
        stats = srv.stats()
    assert stats["rejected"] == 1
