"""Batched form: one persistent, graph-captured tensor-core launch over many datasets
(GPU).  Each dataset's result must equal a separate plain run's (and the oracle's)."""
import numpy as np
import pytest

import epik2
import oracle as O
from conftest import f32_bits
from epik2 import workloads as W

pytestmark = pytest.mark.gpu

MIXED = [  # (seed, samples, SNPs, cases): uneven sizes, class splits and tile counts
    (71, 300, 20, 140), (72, 1000, 45, 333), (73, 64, 3, 32), (74, 2047, 70, 1500), (75, 500, 130, 250),
    (76, 40, 12, 5), (77, 3001, 33, 1500), (78, 129, 257, 64), (79, 777, 64, 400), (80, 1500, 100, 600),
]


@pytest.mark.parametrize("engine,stage_words,pair_tile,overlap",
                         [(2, 4, 32, 1), (2, 8, 32, 1), (3, 8, 32, 1), (3, 16, 64, 1), (3, 8, 64, 1), (3, 16, 32, 1),
                          (3, 4, 64, 2), (3, 8, 64, 2)],
                         ids=["tc-4", "tc-8", "fp4-8", "fp4-16-pair", "fp4-8-pair", "fp4-16", "fp4-4-overlap",
                              "fp4-8-overlap"])
def test_batch_equals_separate_runs_and_oracle(engine, stage_words, pair_tile, overlap):
    data = [O.gen_hwe(sd, S, M, c) for sd, S, M, c in MIXED]
    kw = dict(engine=engine, stage_words=stage_words, pair_tile=pair_tile, overlap=overlap)
    with epik2.Context(0) as ctx:
        ids = [ctx.load(g, p) for g, p in data]
        batched = ctx.scan_batch(ids, **kw)
        again = ctx.scan_batch(ids, **kw)  # graph replay
        single = [ctx.scan(d, **kw) for d in ids]
        single_int = [ctx.scan(d, engine=epik2.ENGINE_INT) for d in ids]
    for (g, p), b, b2, s, si in zip(data, batched, again, single, single_int):
        ref = O.scan(g, p) if g.shape[1] <= 140 else None
        assert b.ijk == s.ijk == si.ijk == b2.ijk
        assert f32_bits(b.score) == f32_bits(s.score) == f32_bits(si.score) == f32_bits(b2.score)
        if ref is not None:
            assert b.ijk == ref["ijk"] and f32_bits(b.score) == f32_bits(ref["score"])


def test_batch_follows_phenotype_reencoding():
    g, p = O.gen_hwe(81, 900, 60, 400)
    g2, p2 = O.gen_hwe(82, 600, 80, 300)
    with epik2.Context(0) as ctx:
        a, b = ctx.load(g, p), ctx.load(g2, p2)
        first = ctx.scan_batch([a, b])
        q = np.random.default_rng(3).permutation(p)
        ctx.set_pheno(a, q)
        second = ctx.scan_batch([a, b])  # same plan, new class split of dataset a
    assert second[1].ijk == first[1].ijk
    r = O.scan(g, q)
    assert second[0].ijk == r["ijk"] and f32_bits(second[0].score) == f32_bits(r["score"])


@pytest.mark.slow
def test_batched_workload_96_datasets_equals_one_by_one():
    specs = W.batched_specs()
    with epik2.Context(0) as ctx:
        ids = []
        for sp in specs:
            g, p = W.generate(sp)
            ids.append(ctx.load(g, p))
        batched = ctx.scan_batch(ids)
        one_by_one = [ctx.scan(d) for d in ids]
    for sp, b, s in zip(specs, batched, one_by_one):
        assert b.ijk == s.ijk, sp["name"]
        assert f32_bits(b.score) == f32_bits(s.score), sp["name"]


def test_autotune_reports_all_candidates():
    g, p = O.gen_hwe(83, 2000, 300, 1000)
    with epik2.Context(0) as ctx:
        d = ctx.load(g, p)
        t = ctx.autotune(d)
        b = ctx.scan(d)  # AUTO engine uses the cached choice
    assert t["engine"] in (epik2.ENGINE_INT, epik2.ENGINE_TC, epik2.ENGINE_TC_FP4)
    assert t["stage_words"] in ((8, 16) if t["engine"] == epik2.ENGINE_TC_FP4 else (4, 8))
    assert t["pair_tile"] in ((32, 64) if t["engine"] == epik2.ENGINE_TC_FP4 else (32,))
    assert min(t["rate_int"], t["rate_tc4"], t["rate_tc8"], t["rate_fp4_8"], t["rate_fp4_16"], t["rate_fp4_8_pair"],
               t["rate_fp4_16_single"], t["rate_fp4_4_overlap"], t["rate_fp4_8_overlap"]) > 0
    rates = {(epik2.ENGINE_INT, 0, 32, 0): t["rate_int"], (epik2.ENGINE_TC, 4, 32, 0): t["rate_tc4"],
             (epik2.ENGINE_TC, 8, 32, 0): t["rate_tc8"], (epik2.ENGINE_TC_FP4, 8, 32, 0): t["rate_fp4_8"],
             (epik2.ENGINE_TC_FP4, 8, 64, 0): t["rate_fp4_8_pair"],
             (epik2.ENGINE_TC_FP4, 16, 32, 0): t["rate_fp4_16_single"],
             (epik2.ENGINE_TC_FP4, 16, 64, 0): t["rate_fp4_16"], (epik2.ENGINE_TC_FP4, 4, 64, 1): t["rate_fp4_4_overlap"],
             (epik2.ENGINE_TC_FP4, 8, 64, 1): t["rate_fp4_8_overlap"]}
    chosen = (t["engine"], 0 if t["engine"] == epik2.ENGINE_INT else t["stage_words"], t["pair_tile"], t["overlap"])
    assert rates[chosen] == max(rates.values())
    r = O.scan(g, p)
    assert b.ijk == r["ijk"]


def test_fp4_refuses_classes_of_2_24_samples():
    """FP32 accumulators hold exact counts below 2^24 per class: the FP4 engine refuses a
    larger class; the int8 engine (int32 accumulators) and the autotuner's choice serve it."""
    n = (1 << 24) + 64
    rng = np.random.default_rng(9)
    g = rng.integers(0, 3, size=(n, 3), dtype=np.uint8)
    p = np.zeros(n, dtype=np.uint8)
    p[:64] = 1  # 2^24 controls
    with epik2.Context(0) as ctx:
        d = ctx.load(g, p)
        with pytest.raises(epik2.Epik2Error) as e:
            ctx.scan(d, engine=epik2.ENGINE_TC_FP4)
        assert e.value.status == epik2.E_TOO_LARGE
        b8 = ctx.scan(d, engine=epik2.ENGINE_TC)
        bi = ctx.scan(d, engine=epik2.ENGINE_INT)
    assert b8.ijk == bi.ijk == (0, 1, 2) and f32_bits(b8.score) == f32_bits(bi.score)


def test_batch_limit_and_tiny_datasets():
    """512 datasets fit one batched launch (the tile descriptors name the dataset in 9
    bits); 513 are refused.  Tiny datasets (3..5 SNPs) still match the oracle."""
    data = [O.gen_hwe(2000 + t, 64, 3 + t % 3, 32) for t in range(513)]
    with epik2.Context(0) as ctx:
        ids = [ctx.load(g, p) for g, p in data]
        got = ctx.scan_batch(ids[:512])
        with pytest.raises(epik2.Epik2Error) as e:
            ctx.scan_batch(ids)
        assert e.value.status == epik2.E_TOO_LARGE
    for (g, p), b in list(zip(data, got))[::37]:
        r = O.scan(g, p)
        assert b.ijk == r["ijk"] and f32_bits(b.score) == f32_bits(r["score"])
