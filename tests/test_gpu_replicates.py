"""Replicate form: permutation replicates of one resident matrix searched with shared
all-sample counts (GPU).

Every tile counts the base matrix's all-sample cells once and then, per replicate, only the
replicate's cases; controls are the totals minus the cases.  Each replicate's best triplet and
FP32 score must equal a plain search of the matrix with that phenotype (and the oracle's), bit
for bit, including replicates with no cases or no controls, ragged sample and SNP counts, and
more replicates than one launch takes (256)."""
import numpy as np
import pytest

import epik2
import oracle as O
from conftest import f32_bits

pytestmark = pytest.mark.gpu


def _perms(p, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.permutation(p) for _ in range(n)])


@pytest.mark.parametrize("seed,S,M,cases,R", [(131, 1000, 150, 400, 1), (132, 777, 97, 300, 7), (133, 2049, 70, 1500, 32)])
def test_replicates_equal_plain_searches_and_oracle(seed, S, M, cases, R):
    g, p = O.gen_hwe(seed, S, M, cases, planted=[(3, 40, M - 5)], effects=[0.8])
    reps = _perms(p, R, seed)
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps)
        plain = []
        for r in reps:
            ctx.set_pheno(base, r)
            plain.append(ctx.scan(base, engine=epik2.ENGINE_TC_FP4, stage_words=16, pair_tile=64, overlap=1))
        ctx.unload(base)
    assert len(got) == R
    for a, b in zip(got, plain):
        assert a.ijk == b.ijk and f32_bits(a.score) == f32_bits(b.score)
    for r, a in list(zip(reps, got))[:3]:
        ref = O.scan(g, r)
        assert a.ijk == ref["ijk"] and f32_bits(a.score) == f32_bits(ref["score"])


def test_replicates_without_cases_or_controls():
    """A replicate whose phenotype has no cases (its cases' accumulators are never written in
    that pass) or only cases (no controls) still gets the oracle's result."""
    g, p = O.gen_hwe(134, 600, 40, 300)
    reps = np.stack([np.zeros(600, np.uint8), np.ones(600, np.uint8), p, np.roll(p, 7)])
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps)
        ctx.unload(base)
    for r, a in zip(reps, got):
        ref = O.scan(g, r)
        assert a.ijk == ref["ijk"] and f32_bits(a.score) == f32_bits(ref["score"])


def test_more_replicates_than_one_launch():
    g, p = O.gen_hwe(135, 200, 20, 90)
    reps = _perms(p, 300, 135)
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps)
        plain = []
        for r in reps:
            ctx.set_pheno(base, r)
            plain.append(ctx.scan(base, engine=epik2.ENGINE_TC_FP4, stage_words=16, pair_tile=64, overlap=1))
        ctx.unload(base)
    assert [a.ijk for a in got] == [b.ijk for b in plain]
    assert [f32_bits(a.score) for a in got] == [f32_bits(b.score) for b in plain]


def test_early_tiles_of_the_queue_are_searched():
    """The replicates' own loads compute pair margins with the tensor-core kernel, which uses a
    descriptor buffer of its own kind: the search's tiles must be laid down after them.  A
    triplet planted in the first tiles of the queue (first index 2, SNPs 5 and 40) on a 700-SNP
    matrix is the best of the unpermuted replicate, as a plain search finds."""
    g, p = O.gen_hwe(136, 1000, 700, 500, maf=(0.3, 0.5), planted=[(2, 5, 40)], effects=[0.9])
    reps = np.concatenate([p[None, :], _perms(p, 3, 136)])
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps)
        plain = []
        for r in reps:
            ctx.set_pheno(base, r)
            plain.append(ctx.scan(base, engine=epik2.ENGINE_TC_FP4, stage_words=16, pair_tile=64, overlap=1))
        ctx.unload(base)
    assert got[0].ijk == (2, 5, 40)
    for a, b in zip(got, plain):
        assert a.ijk == b.ijk and f32_bits(a.score) == f32_bits(b.score)


def test_fp64_rescore_of_each_replicate_equals_oracle():
    """With rescore_fp64 each replicate's best carries its FP64 K2 score, computed on the GPU
    from the replicate's own tables: equal bit for bit to the oracle's FP64 K2 of that
    triplet's table under the replicate's phenotype, and to the plain search's rescore."""
    g, p = O.gen_hwe(137, 900, 60, 420, planted=[(4, 30, 55)], effects=[0.7])
    reps = np.concatenate([p[None, :], _perms(p, 5, 137)])
    with epik2.Context(0) as ctx:
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps, rescore_fp64=1)
        plain = []
        for r in reps:
            ctx.set_pheno(base, r)
            plain.append(ctx.scan(base, engine=epik2.ENGINE_TC_FP4, stage_words=16, pair_tile=64, overlap=1,
                                  rescore_fp64=1))
        ctx.unload(base)
    for r, a, b in zip(reps, got, plain):
        assert a.ijk == b.ijk and f32_bits(a.score) == f32_bits(b.score)
        assert a.score_fp64 == b.score_fp64
        assert a.score_fp64 == O.k2_fp64(O.table(g, r, *a.ijk))


def test_spare_allocation_shared_with_the_one_call_entry_point():
    """The replicates' allocation stays with the context as its spare (reported as free) and
    serves or yields to the next allocation: one-call scans before and after a replicate call,
    and a second replicate call of another shape, all keep their results, and the context's
    free memory (spare included) returns to where it was."""
    g, p = O.gen_hwe(138, 800, 50, 380)
    g2, p2 = O.gen_hwe(139, 1500, 90, 700)
    reps = _perms(p, 12, 138)
    with epik2.Context(0) as ctx:
        free0 = ctx.mem_info()[0]
        a = ctx.scan_u8(g, p)
        base = ctx.load(g, p)
        got = ctx.scan_replicates(base, reps)
        b = ctx.scan_u8(g2, p2)
        base2 = ctx.load(g2, p2)
        got2 = ctx.scan_replicates(base2, _perms(p2, 3, 139))
        ctx.unload(base2)
        again = ctx.scan_replicates(base, reps[:5])
        ctx.unload(base)
        free1 = ctx.mem_info()[0]
    ref, ref2 = O.scan(g, p), O.scan(g2, p2)
    assert a.ijk == ref["ijk"] and f32_bits(a.score) == f32_bits(ref["score"])
    assert b.ijk == ref2["ijk"] and f32_bits(b.score) == f32_bits(ref2["score"])
    for r, x in zip(reps[:3], got[:3]):
        rr = O.scan(g, r)
        assert x.ijk == rr["ijk"] and f32_bits(x.score) == f32_bits(rr["score"])
    assert [x.ijk for x in again] == [x.ijk for x in got[:5]]
    assert [f32_bits(x.score) for x in again] == [f32_bits(x.score) for x in got[:5]]
    assert len(got2) == 3
    assert abs(free1 - free0) < (64 << 20)  # scratch of a few MiB may stay allocated
