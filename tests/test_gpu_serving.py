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


def test_permutation_pvalue_through_the_server_matches_oracle():
    """Permutation test end to end: the observed phenotype and R = 64 permutation replicates
    of one resident matrix run through the server; every replicate's best triplet and FP32
    score equal the oracle's scan of that permuted phenotype bit for bit, and the p-value
    (1 + #{replicate best <= observed}) / (1 + R) equals the one from the oracle's scores."""
    # common alleles (MAF 0.3..0.5) make the planted triplet's carriers frequent, so its
    # association clearly beats every permutation's best (checked against the oracle)
    g, p = O.gen_hwe(95, 600, 36, 300, maf=(0.3, 0.5), planted=[(4, 17, 30)], effects=[0.85])
    R = 64
    reps = _perms(p, R, 7)
    with epik2.Server(0, batch_work=2e9) as srv:
        m = srv.add_matrix(g, p)
        rid_obs = srv.submit_replicates(m, p[None, :])
        rid = srv.submit_replicates(m, reps)
        st_obs, obs, _ = srv.wait(rid_obs)
        st, res, _ = srv.wait(rid)
    assert st_obs == epik2.OK and st == epik2.OK and len(res) == R
    ref_obs = O.scan(g, p)
    assert obs[0].ijk == ref_obs["ijk"] and f32_bits(obs[0].score) == f32_bits(ref_obs["score"])
    ref_scores = []
    for r, a in zip(reps, res):
        ref = O.scan(g, r)
        assert a.ijk == ref["ijk"] and f32_bits(a.score) == f32_bits(ref["score"])
        ref_scores.append(np.float32(ref["score"]))
    pv = epik2.perm_pvalue(obs[0].score, [a.score for a in res])
    pv_ref = (1 + sum(1 for s in ref_scores if s <= np.float32(ref_obs["score"]))) / (1 + R)
    assert pv == pv_ref
    assert pv == 1.0 / (1 + R)  # the planted triplet beats every permutation


def test_admission_by_free_device_memory():
    """Admission control on the host: with a reserve that leaves room for about three and a
    half replicate datasets (each replicate holds its own planes, margins and tables, ~22 MB
    here), no launch takes more than three scans, every scan still completes with the result
    of a plain run of its phenotype, and a fresh matrix that could never fit is refused with
    EPIK2_E_NOMEM."""
    S, M = 20000, 1000
    g, p = epik2.generate_hwe(96, S, M, S // 2)
    reps = _perms(p, 10, 11)
    page = 2 << 20
    per = -(-epik2.library().epik2_replicate_bytes(S, M) // page) * page
    with epik2.Context(0) as probe:  # a context like the server's, to measure what is free
        free, total = probe.mem_info()
    reserve = free - epik2.dataset_bytes(S, M) - int(3.5 * per)
    with epik2.Server(0, batch_work=1e16, hbm_reserve_bytes=reserve) as srv:
        m = srv.add_matrix(g, p)
        rid = srv.submit_replicates(m, reps)
        big_m = 64
        while epik2.dataset_bytes(4000, big_m) <= total - reserve:
            big_m *= 2
        gb = np.zeros((4000, big_m), dtype=np.uint8)
        pb = np.zeros(4000, dtype=np.uint8)
        pb[:2000] = 1
        rid_big = srv.submit_scan(gb, pb)
        st, res, _ = srv.wait(rid)
        st_big, _, _ = srv.wait(rid_big)
        stats = srv.stats()
    assert st == epik2.OK and len(res) == 10
    assert st_big == epik2.E_NOMEM
    assert 1 <= stats["max_active"] <= 3 and stats["launches"] >= 4
    with epik2.Context(0) as ctx:
        did = ctx.load(g, p)
        for r, a in zip(reps, res):
            ctx.set_pheno(did, r)
            b = ctx.scan(did)
            assert a.ijk == b.ijk and f32_bits(a.score) == f32_bits(b.score)
