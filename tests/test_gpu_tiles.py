"""Per-cell tables of searches that span many tensor-core tiles, and classes far beyond the
sizes of the other fixtures (GPU).

The tensor-core engines cut a search into tiles of 32 pairs j x 128 SNPs k (int8), 32 x 112
(FP4) or 64 x 112 (FP4 on CTA pairs).  With 150 to 300 SNPs every search here has many
first indices, several pair blocks and several k blocks per pair block, the odd CTA's half of
a CTA-pair tile beyond the first, and tile descriptors over many (i, j-block) pairs.  Every
one of the C(M,3) tables and FP32 scores must equal the oracle's (GPU/v2.cpp:288-540 restated)
bit for bit, and on two shapes also the reference's own recorded tables (sha256 of the
tables and scores that oracle/ref_tap_tables recorded from CPU/v2.cpp, tile_taps.json).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import epik2
import oracle as O
from conftest import GOLDEN, f32_bits

pytestmark = pytest.mark.gpu

# (seed, samples, SNPs, cases)
SHAPES = [(101, 300, 150, 140), (102, 1000, 257, 333), (103, 300, 300, 170)]

_oracle_cache = {}


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _oracle(seed, S, M, cases):
    """Input matrix and the oracle's best, with sha256 digests of its tables and scores (the
    arrays themselves are up to 1 GB, so only their digests are kept between engines)."""
    key = (seed, S, M, cases)
    if key not in _oracle_cache:
        g, p = O.gen_hwe(seed, S, M, cases)
        r = O.scan(g, p, with_tables=True)
        _oracle_cache[key] = dict(g=g, p=p, ijk=r["ijk"], score=r["score"], tables=_sha(r["tables"]),
                                  scores=_sha(r["scores"].view(np.uint32)), T=r["T"])
    return _oracle_cache[key]


def _first_mismatch(g, p, tables, scores):
    r = O.scan(g, p, with_tables=True)
    bad = np.flatnonzero((tables != r["tables"]).any(axis=1) | (scores.view(np.uint32) != r["scores"].view(np.uint32)))
    M = g.shape[1]
    return [(O.triplet_of(M, int(t)), tables[t].tolist(), r["tables"][t].tolist()) for t in bad[:3]], len(bad)


@pytest.mark.parametrize("seed,S,M,cases", SHAPES)
def test_every_table_across_many_tiles_vs_oracle(ctx, seed, S, M, cases):
    o = _oracle(seed, S, M, cases)
    did = ctx.load(o["g"], o["p"])
    try:
        tables, scores = ctx.dump_tables(did)
        b = ctx.scan(did)
    finally:
        ctx.unload(did)
    assert tables.shape == (o["T"], 54)
    if _sha(tables) != o["tables"] or _sha(scores.view(np.uint32)) != o["scores"]:
        first, n_bad = _first_mismatch(o["g"], o["p"], tables, scores)
        pytest.fail(f"{n_bad} of {o['T']} triplets differ from the oracle; first: {first}")
    assert b.ijk == o["ijk"] and f32_bits(b.score) == f32_bits(o["score"])
    taps = json.load(open(os.path.join(GOLDEN, "tile_taps.json")))
    rec = taps.get(f"hwe_{S}x{M}_{cases}cases")
    if rec is not None:  # the reference's own tables and scores of this input
        assert _sha(o["g"]) == rec["geno_sha256"] and _sha(o["p"]) == rec["pheno_sha256"]
        assert _sha(tables.astype("<u4")) == rec["tables_sha256"]
        assert _sha(scores.view(np.uint32).astype("<u4")) == rec["scores_sha256"]


_big_class = {}


def _big_class_case():
    """2^23 + 12345 controls, 4099 cases, 8 SNPs (about 70 MB of genotypes)."""
    if not _big_class:
        n0, n1 = (1 << 23) + 12345, 4099
        g, p = O.gen_hwe(111, n0 + n1, 8, n1)
        r = O.scan(g, p, with_tables=True)
        _big_class.update(g=g, p=p, r=r)
    return _big_class


def test_class_of_2_23_samples_tables_and_margins(ctx):
    """Pair margins come from the FP4 tensor-core kernel (FP32 accumulators) whenever every
    class has fewer than 2^24 samples.  A class of 2^23 + 12345 samples puts the counts where
    FP32 integers are sparsest below that limit: every table, score and the best triplet
    must still equal the oracle's on every engine."""
    c = _big_class_case()
    did = ctx.load(c["g"], c["p"])
    try:
        if ctx.config[3] == 2:  # the overlapped kernel stages counts in 16 bits: it refuses
            with pytest.raises(epik2.Epik2Error) as e:
                ctx.scan(did)
            assert e.value.status == epik2.E_TOO_LARGE
            return
        tables, scores = ctx.dump_tables(did)
        b = ctx.scan(did)
    finally:
        ctx.unload(did)
    assert np.array_equal(tables, c["r"]["tables"])
    assert np.array_equal(scores.view(np.uint32), c["r"]["scores"].view(np.uint32))
    assert b.ijk == c["r"]["ijk"] and f32_bits(b.score) == f32_bits(c["r"]["score"])
