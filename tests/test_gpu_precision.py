"""Precision form: FP32 search, per-warp top-32 candidates rescored in FP64 on the GPU
(GPU).  Counts stay exact; FP32 scores are bit-exact against the oracle; FP64 scores
equal the FP64 oracle (same table, same summation order); the FP64 top-32 (set and
order) equals the oracle's; relative FP32-vs-FP64 error <= 1e-5."""
import numpy as np
import pytest

import epik2
import oracle as O
from conftest import f32_bits, ref_best

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


@pytest.mark.parametrize("seed,S,M,cases", [(61, 1500, 60, 700), (62, 2049, 45, 1100), (63, 513, 33, 100)])
def test_top32_fp64_matches_oracle(ctx, seed, S, M, cases):
    g, p = O.gen_hwe(seed, S, M, cases, maf=(0.01, 0.5), planted=[(2, 20, 40), (5, 9, 31)], effects=[0.7, 0.8])
    s64 = O.scan_fp64(g, p)
    r = O.scan(g, p, with_tables=True)
    trip = O.triplet_list(M)
    order = np.lexsort((np.arange(len(s64)), s64))[:32]
    did = ctx.load(g, p)
    try:
        top = ctx.scan_topk(did, 32, rescore_fp64=1)
        assert [t.ijk for t in top] == [trip[x] for x in order]
        for t, x in zip(top, order):
            assert t.score_fp64 == s64[x]                       # FP64 bit-exact vs oracle
            assert f32_bits(t.score) == f32_bits(r["scores"][x])  # FP32 bit-exact vs reference arithmetic
            assert abs(t.score - t.score_fp64) / t.score_fp64 <= REL_TOL
        best = ctx.scan(did, rescore_fp64=1)
        assert best.ijk == trip[order[0]] and best.score_fp64 == s64[order[0]]
    finally:
        ctx.unload(did)


def test_precision_workload_top1_matches_reference():
    rec = ref_best()["precision"]
    g, p = epik2.generate_hwe(rec["seed"], rec["n_samples"], rec["n_snps"], rec["n_cases"], rec["maf"],
                              rec["planted"], rec["effects"])
    with epik2.Context(0) as ctx:
        did = ctx.load(g, p)
        top = ctx.scan_topk(did, 32, rescore_fp64=1)
        plain = ctx.scan(did)
        tables = ctx.tables(did, [t.ijk for t in top])
    assert list(top[0].ijk) == rec["ijk"]
    assert list(plain.ijk) == rec["ijk"] and f32_bits(plain.score) == rec["score_bits"]
    errs = [abs(t.score - t.score_fp64) / t.score_fp64 for t in top]
    assert max(errs) <= REL_TOL
    for t, tab in zip(top, tables):
        assert t.score_fp64 == O.k2_fp64(tab)
        assert f32_bits(t.score) == f32_bits(O.k2(tab, O.lut(rec["n_samples"] + 1)))


def test_precision_workload_top32_matches_fp64_oracle():
    """The full precision workload (2048 SNPs x 8192 samples, three planted triplets): the GPU's
    FP64 top-32 -- per-warp FP32 top-32 lists, every candidate rescored in FP64 on the GPU,
    ranked by FP64 score -- equals the FP64 oracle's top-32 over all 1.43e9 triplets in set and
    order, with bit-identical FP64 scores, the reference's FP32 scores and the oracle's tables
    (tests/golden/precision_top32.json, made by tests/golden/make_golden.py --only top32)."""
    import hashlib
    import json
    import os
    from conftest import GOLDEN
    from epik2 import workloads as W
    fx = json.load(open(os.path.join(GOLDEN, "precision_top32.json")))
    g, p = W.generate(W.PRECISION)
    assert hashlib.sha256(np.ascontiguousarray(g).tobytes()).hexdigest() == fx["geno_sha256"]
    with epik2.Context(0) as ctx:
        did = ctx.load(g, p)
        top = ctx.scan_topk(did, 32, rescore_fp64=1)
        tables = ctx.tables(did, [t.ijk for t in top])
    assert [list(t.ijk) for t in top] == [x["ijk"] for x in fx["top"]]
    for t, x, tab in zip(top, fx["top"], tables):
        assert t.score_fp64 == float.fromhex(x["s64"])
        assert f32_bits(t.score) == x["s32_bits"]
        assert tab.tolist() == x["table"]
        assert abs(t.score - t.score_fp64) / t.score_fp64 <= REL_TOL
