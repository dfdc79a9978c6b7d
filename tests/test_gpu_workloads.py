"""Full-size workloads against the reference CPU search's recorded answers (GPU).

ref_best.json holds, for each seeded Hardy-Weinberg workload, the best triplet and the
exact FP32 score bits printed by the reference's v4_popc_avx512 search on the same
matrix (and the matrix's sha256, so the product generator is pinned too).
"""
import hashlib

import numpy as np
import pytest

import epik2
from conftest import f32_bits, ref_best

pytestmark = pytest.mark.gpu


def _matrix(rec):
    g, p = epik2.generate_hwe(rec["seed"], rec["n_samples"], rec["source_snps"], rec["n_cases"], rec["maf"],
                              rec["planted"], rec["effects"])
    if rec["n_snps"] < rec["source_snps"]:
        g = np.ascontiguousarray(g[:, :rec["n_snps"]])
    assert hashlib.sha256(g.tobytes()).hexdigest() == rec["geno_sha256"]
    assert hashlib.sha256(p.tobytes()).hexdigest() == rec["pheno_sha256"]
    return g, p


CASES = sorted(ref_best().keys())


@pytest.mark.parametrize("name", CASES)
def test_best_triplet_identical_to_reference(ctx, name):
    rec = ref_best()[name]
    g, p = _matrix(rec)
    did = ctx.load(g, p)
    try:
        b = ctx.scan(did)
        assert list(b.ijk) == rec["ijk"], (name, b.ijk, rec["ijk"])
        assert f32_bits(b.score) == rec["score_bits"], (name, b.score, rec["score"])
    finally:
        ctx.unload(did)


def test_planted_triplet_tables_sum_to_class_sizes(ctx):
    rec = ref_best()["plain-small"]
    g, p = _matrix(rec)
    did = ctx.load(g, p)
    try:
        t = ctx.tables(did, [rec["ijk"]])[0]
        assert t[:27].sum() == rec["n_samples"] - rec["n_cases"]
        assert t[27:].sum() == rec["n_cases"]
    finally:
        ctx.unload(did)
