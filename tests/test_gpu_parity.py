"""CUDA search path against the reference-recorded fixtures and the oracle (GPU).

Tables and FP32 scores must be bit-exact; the best triplet must be identical, ties
broken by the lowest (i, j, k).
"""
import numpy as np
import pytest

import epik2
import oracle as O
from conftest import TAP_CASES, f32_bits, load_tap, ref_kat

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", TAP_CASES)
def test_every_table_and_score_bit_exact_vs_reference(ctx, case):
    t = load_tap(case)
    did = ctx.load(t["geno"], t["pheno"])
    try:
        tables, scores = ctx.dump_tables(did)
        assert np.array_equal(tables, t["tables"])
        assert np.array_equal(scores.view(np.uint32), t["scores"].view(np.uint32))
        b = ctx.scan(did)
        # lowest score, ties to the lowest lexicographic index
        order = np.lexsort((np.arange(len(scores)), scores))
        best_t = order[0]
        M = t["geno"].shape[1]
        trip = [(i, j, k) for i in range(M) for j in range(i + 1, M) for k in range(j + 1, M)]
        assert b.ijk == trip[best_t]
        assert f32_bits(b.score) == int(t["scores"].view(np.uint32)[best_t])
    finally:
        ctx.unload(did)


@pytest.mark.parametrize("case", TAP_CASES)
def test_direct_27_cell_kernel_matches_reference(ctx, case):
    t = load_tap(case)
    did = ctx.load(t["geno"], t["pheno"])
    try:
        M = t["geno"].shape[1]
        trip = np.array([(i, j, k) for i in range(M) for j in range(i + 1, M) for k in range(j + 1, M)])
        sel = np.arange(0, len(trip), max(1, len(trip) // 300))
        got = ctx.tables(did, trip[sel])
        assert np.array_equal(got, t["tables"][sel])
    finally:
        ctx.unload(did)


@pytest.mark.parametrize("key", ["2048x128", "2000x100", "2048x512", "100x7", "33x5"])
def test_reference_generator_known_answers(ctx, key):
    k = ref_kat()[key]
    g, p = epik2.generate_reference(k["n_samples"], k["n_snps"])
    b = ctx.scan_u8(g, p)
    assert list(b.ijk) == k["ijk"]
    assert f32_bits(b.score) == k["score_bits"]


RAGGED = [
    # (seed, samples, snps, cases): sample counts off multiples of 32/64, SNP counts off
    # multiples of 32, tiny classes, empty-ish shapes
    (31, 1, 3, 0), (32, 2, 5, 1), (33, 31, 33, 7), (34, 33, 64, 16), (35, 65, 65, 1), (36, 100, 97, 99),
    (37, 129, 40, 64), (38, 1000, 35, 333), (39, 77, 3, 40), (40, 4096, 36, 2048), (41, 3001, 70, 1500),
]


@pytest.mark.parametrize("seed,S,M,cases", RAGGED)
def test_ragged_shapes_vs_oracle(ctx, seed, S, M, cases):
    g, p = O.gen_hwe(seed, S, M, cases)
    r = O.scan(g, p, with_tables=(M <= 64))
    did = ctx.load(g, p)
    try:
        b = ctx.scan(did)
        assert b.ijk == r["ijk"]
        assert f32_bits(b.score) == f32_bits(r["score"])
        if M <= 64:
            tables, scores = ctx.dump_tables(did)
            assert np.array_equal(tables, r["tables"])
            assert np.array_equal(scores.view(np.uint32), r["scores"].view(np.uint32))
    finally:
        ctx.unload(did)


@pytest.mark.parametrize("seed,S,M", [(61, 23742, 40), (62, 23743, 36), (63, 40000, 40)])
def test_large_sample_counts_vs_oracle(ctx, seed, S, M):
    """Up to 23,742 samples the tensor-core epilogue reads the ln n! table from a shared-memory
    copy, beyond it from global memory: both sides of that limit, tables included."""
    g, p = O.gen_hwe(seed, S, M, S // 2)
    r = O.scan(g, p, with_tables=True)
    did = ctx.load(g, p)
    try:
        b = ctx.scan(did)
        assert b.ijk == r["ijk"]
        assert f32_bits(b.score) == f32_bits(r["score"])
        tables, scores = ctx.dump_tables(did)
        assert np.array_equal(tables, r["tables"])
        assert np.array_equal(scores.view(np.uint32), r["scores"].view(np.uint32))
    finally:
        ctx.unload(did)


def test_one_call_entry_point_reuses_its_allocation(ctx):
    """epik2_scan_u8 keeps one dataset allocation for its next call; nothing of the previous
    dataset may show through (same shape, smaller within 2x, much smaller, larger)."""
    for seed, S, M, cases in [(51, 2000, 80, 1000), (52, 2000, 80, 700), (53, 1900, 76, 1000), (54, 64, 10, 30),
                              (55, 2100, 84, 1050)]:
        g, p = O.gen_hwe(seed, S, M, cases)
        r = O.scan(g, p)
        b = ctx.scan_u8(g, p)
        assert b.ijk == r["ijk"]
        assert f32_bits(b.score) == f32_bits(r["score"])


def test_planted_ties_break_to_lowest_index(ctx):
    # Duplicate SNP columns make many triplets share an exact score.
    g, p = O.gen_hwe(50, 500, 12, 250)
    g = g.copy()
    g[:, 7] = g[:, 2]
    g[:, 9] = g[:, 4]
    g[:, 11] = g[:, 2]
    r = O.scan(g, p, with_tables=True)
    did = ctx.load(g, p)
    try:
        b = ctx.scan(did)
        assert b.ijk == r["ijk"]
        _, scores = ctx.dump_tables(did)
        assert np.array_equal(scores.view(np.uint32), r["scores"].view(np.uint32))
    finally:
        ctx.unload(did)


def test_set_pheno_reencodes(ctx):
    g, p = O.gen_hwe(51, 700, 40, 300)
    did = ctx.load(g, p)
    try:
        rng = np.random.default_rng(0)
        for _ in range(3):
            q = rng.permutation(p)
            ctx.set_pheno(did, q)
            r = O.scan(g, q)
            b = ctx.scan(did)
            assert b.ijk == r["ijk"] and f32_bits(b.score) == f32_bits(r["score"])
        # more cases than before: the class split changes size
        q = np.zeros_like(p)
        q[:650] = 1
        ctx.set_pheno(did, q)
        r = O.scan(g, q)
        b = ctx.scan(did)
        assert b.ijk == r["ijk"] and f32_bits(b.score) == f32_bits(r["score"])
    finally:
        ctx.unload(did)


def test_first_index_range_partitions_the_search(ctx):
    g, p = O.gen_hwe(52, 900, 150, 450)
    did = ctx.load(g, p)
    try:
        full = ctx.scan(did)
        parts = [ctx.scan(did, snp_begin=a, snp_end=b) for a, b in [(0, 7), (7, 40), (40, 150)]]
        best = min(parts, key=lambda x: (x.score, x.ijk))
        assert best.ijk == full.ijk and best.score == full.score
    finally:
        ctx.unload(did)


def test_errors_are_statuses(ctx):
    with pytest.raises(epik2.Epik2Error) as e:
        ctx.scan(12345)
    assert e.value.status == epik2.E_NOT_FOUND
    g, p = O.gen_hwe(53, 50, 2, 25)
    did = ctx.load(g, p)
    with pytest.raises(epik2.Epik2Error) as e:
        ctx.scan(did)
    assert e.value.status == epik2.E_INVALID
    ctx.unload(did)
    with pytest.raises(epik2.Epik2Error):
        ctx.tables(did, [(0, 1, 2)])


def test_topk_matches_oracle_ranking(ctx):
    g, p = O.gen_hwe(54, 1500, 60, 700, planted=[(4, 20, 50)], effects=[0.8])
    r = O.scan(g, p, with_tables=True)
    did = ctx.load(g, p)
    try:
        top = ctx.scan_topk(did, 32)
        order = np.lexsort((np.arange(len(r["scores"])), r["scores"]))[:32]
        M = 60
        trip = [(i, j, k) for i in range(M) for j in range(i + 1, M) for k in range(j + 1, M)]
        assert [t.ijk for t in top] == [trip[x] for x in order]
        assert [f32_bits(t.score) for t in top] == [f32_bits(r["scores"][x]) for x in order]
    finally:
        ctx.unload(did)
