"""The C oracle pinned against fixtures recorded from the reference itself (CPU only)."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import TAP_CASES, addlog_bits, f32_bits, load_tap, ref_kat


@pytest.fixture(scope="module", autouse=True)
def built():
    if not O.os.path.exists(O.LIB_PATH):
        O.build()


@pytest.mark.parametrize("case", TAP_CASES)
def test_oracle_tables_and_scores_match_reference(case):
    t = load_tap(case)
    r = O.scan(t["geno"], t["pheno"], with_tables=True)
    assert r["T"] == len(t["tables"])
    assert np.array_equal(r["tables"], t["tables"])
    assert np.array_equal(r["scores"].view(np.uint32), t["scores"].view(np.uint32))
    line = str(t["best_line"])
    ijk = tuple(int(x) for x in line.split(":")[1].split("-")[0].split(","))
    assert r["ijk"] == ijk


def test_oracle_lut_matches_reference_addlog():
    ref = addlog_bits()
    assert np.array_equal(O.lut(len(ref) - 1).view(np.uint32), ref)


@pytest.mark.parametrize("key", ["100x7", "33x5", "2000x100"])
def test_oracle_reference_generator_kat(key):
    k = ref_kat()[key]
    A, B = O.gen_reference(k["n_samples"], k["n_snps"])
    r = O.scan(A, B)
    assert list(r["ijk"]) == k["ijk"]
    assert f32_bits(r["score"]) == k["score_bits"]


def test_mt19937_64_check_value():
    # C++ [rand.predef]: the 10000th output of a default-seeded mt19937_64
    assert O.mt64_nth(5489, 10000) == 9981545732273789042


def test_triplet_index_is_lexicographic():
    M = 9
    seen = []
    for i in range(M):
        for j in range(i + 1, M):
            for k in range(j + 1, M):
                seen.append(O.triplet_index(M, i, j, k))
    assert seen == list(range(M * (M - 1) * (M - 2) // 6))


def test_table_margins_sum_to_class_sizes():
    A, B = O.gen_hwe(3, 517, 9, 200)
    ft = O.table(A, B, 1, 4, 7)
    assert ft[:27].sum() == 517 - 200 and ft[27:].sum() == 200
    # definitional count
    gi, gj, gk = A[:, 1].astype(int), A[:, 4].astype(int), A[:, 7].astype(int)
    cell = 9 * gi + 3 * gj + gk
    for cls, off in ((0, 0), (1, 27)):
        sel = (B == 1) if cls else (B != 1)
        assert np.array_equal(np.bincount(cell[sel], minlength=27), ft[off:off + 27])


def test_fp64_oracle_close_to_fp32_and_lgamma():
    A, B = O.gen_hwe(4, 2000, 6, 1000)
    ft = O.table(A, B, 0, 2, 5)
    f32 = O.k2(ft, O.lut(2001))
    f64 = O.k2_fp64(ft)
    lg = O.k2_lgamma(ft)
    assert abs(f32 - f64) / f64 < 1e-5
    assert abs(f64 - lg) / lg < 1e-3


def test_hwe_generator_case_count_and_planted_signal():
    A, B = O.gen_hwe(5, 3000, 20, 1234, planted=[(2, 9, 15)], effects=[0.9])
    assert int(B.sum()) == 1234
    carrier = (A[:, 2] >= 1) & (A[:, 9] >= 1) & (A[:, 15] >= 1)
    assert B[carrier].mean() > B[~carrier].mean() + 0.2


@pytest.mark.parametrize("seed,S,M,cases", [(61, 1500, 60, 700), (63, 513, 33, 100), (64, 70, 5, 33), (65, 200, 3, 100)])
def test_fp64_topk_oracle_matches_exhaustive_fp64_scan(seed, S, M, cases):
    """oracle_topk_fp64_u8 (pair planes hoisted, 64-bit words) ranks exactly like the
    per-triplet FP64 scan, and its tables equal oracle_table's."""
    g, p = O.gen_hwe(seed, S, M, cases, maf=(0.01, 0.5))
    s64 = O.scan_fp64(g, p)
    order = np.lexsort((np.arange(len(s64)), s64))[:32]
    r = O.topk_fp64(g, p, 32)
    trip = O.triplet_list(M)
    assert r["ijk"] == [trip[x] for x in order]
    assert np.array_equal(r["s64"], s64[order])
    full = O.scan(g, p, with_tables=True)
    assert np.array_equal(r["tables"], full["tables"][order])


def test_precision_top32_fixture_is_self_consistent():
    """Each recorded table scores to its recorded FP64 and FP32 values, the list is sorted by
    (FP64 score, index), and its first triplet is the reference's best on that workload."""
    import json
    from conftest import GOLDEN, ref_best
    fx = json.load(open(os.path.join(GOLDEN, "precision_top32.json")))
    assert len(fx["top"]) == 32
    lut = O.lut(8192 + 1)
    keys = []
    for x in fx["top"]:
        t = np.array(x["table"], dtype=np.uint32)
        assert O.k2_fp64(t) == float.fromhex(x["s64"])
        assert int(np.float32(O.k2(t, lut)).view(np.uint32)) == x["s32_bits"]
        keys.append((float.fromhex(x["s64"]), O.triplet_index(2048, *x["ijk"])))
    assert keys == sorted(keys)
    assert fx["top"][0]["ijk"] == ref_best()["precision"]["ijk"]
