"""Regenerates the golden fixtures in this directory from the reference itself.

Needs the reference sources (the harness binaries under oracle/_ref are built from
them by oracle/Makefile); run in a container that has them:

    python tests/golden/make_golden.py            # fixtures that take seconds
    python tests/golden/make_golden.py --long     # + full-size reference searches (minutes to ~1 h)

Fixtures:
  ref_kat.json        best triplet + exact score bits of the reference's own programs on
                      the reference's srand(100) data (ref_v4popc and ref_v2 "gen" mode)
  tap_<case>.npz      every triplet's 54-count table and FP32 score, recorded from the
                      reference's unblocked search (CPU/v2.cpp) by oracle/ref_tap_tables,
                      together with the input matrix
  addlog.npz          the reference's addlog(n) (its ln n! with Stirling tail) for
                      n in [0, 70000], as float32 bit patterns
  ref_best.json       best triplet + exact score bits of the reference's CPU search
                      (v4_popc_avx512 through oracle/ref_harness) on the seeded
                      Hardy-Weinberg workloads, with a sha256 of each input matrix
  tile_taps.json      sha256 of every triplet's 54-count table and of every FP32 score
                      recorded from the reference's unblocked search (oracle/ref_tap_tables)
                      on shapes that span many tensor-core tiles (too large to commit as
                      arrays), checked here against the oracle
  precision_top32.json  the 32 lowest FP64 K2 scores of the precision workload (2048 SNPs x
                      8192 samples) from the FP64 oracle (oracle_topk_fp64_u8), with their
                      tables; the FP64 top-1 is checked against the reference's best

    python tests/golden/make_golden.py --only tiles     # just tile_taps.json
    python tests/golden/make_golden.py --only top32     # just precision_top32.json (~6 min)
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle as O  # noqa: E402

REF = os.path.join(REPO, "oracle", "_ref")
# the reference sources the harness binaries are built from
REF_SRC = os.environ.get("EPIK2_REF_DIR", "/root/reference")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tap_case(name, A, B, mode_gen=None):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "tap.bin")
        if mode_gen:
            cmd = [os.path.join(REF, "ref_tap_tables"), "gen", str(mode_gen[0]), str(mode_gen[1]), out]
        else:
            gp = os.path.join(td, "geno.bin")
            O.write_geno_file(gp, A, B)
            cmd = [os.path.join(REF, "ref_tap_tables"), "file", gp, str(A.shape[0]), str(A.shape[1]), out]
        r = subprocess.run(cmd, check=True, capture_output=True, text=True)
        raw = open(out, "rb").read()
    N, M, T = (int(x) for x in np.frombuffer(raw[:24], dtype=np.int64))
    off = 24
    A2 = np.frombuffer(raw[off:off + N * M], dtype=np.uint8).reshape(N, M)
    off += N * M
    B2 = np.frombuffer(raw[off:off + N], dtype=np.uint8)
    off += N
    tables = np.frombuffer(raw[off:off + T * 216], dtype=np.uint32).reshape(T, 54)
    off += T * 216
    scores = np.frombuffer(raw[off:off + T * 4], dtype=np.float32)
    best_line = [l for l in r.stdout.splitlines() if l.startswith("Best SNPs")][0]
    np.savez_compressed(os.path.join(HERE, f"tap_{name}.npz"), geno=A2, pheno=B2, tables=tables, scores=scores,
                        best_line=np.array(best_line))
    print(f"tap_{name}: N={N} M={M} T={T} {best_line}")


# shapes whose searches span many 64-pair x 112-SNP (and 32 x 128) tensor-core tiles:
# (seed, samples, SNPs, cases) of O.gen_hwe
TILE_SHAPES = [(102, 1000, 257, 333), (103, 300, 300, 170)]


def tap_raw(A, B):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "tap.bin")
        gp = os.path.join(td, "geno.bin")
        O.write_geno_file(gp, A, B)
        r = subprocess.run([os.path.join(REF, "ref_tap_tables"), "file", gp, str(A.shape[0]), str(A.shape[1]), out],
                           check=True, capture_output=True, text=True)
        raw = open(out, "rb").read()
    N, M, T = (int(x) for x in np.frombuffer(raw[:24], dtype=np.int64))
    off = 24 + N * M + N
    tables = np.frombuffer(raw[off:off + T * 216], dtype=np.uint32).reshape(T, 54)
    scores = np.frombuffer(raw[off + T * 216:off + T * 220], dtype=np.float32)
    best_line = [l for l in r.stdout.splitlines() if l.startswith("Best SNPs")][0]
    return tables, scores, best_line


def make_tile_taps():
    out = {}
    for seed, S, M, cases in TILE_SHAPES:
        A, B = O.gen_hwe(seed, S, M, cases)
        tables, scores, best_line = tap_raw(A, B)
        r = O.scan(A, B, with_tables=True)
        assert np.array_equal(r["tables"], tables) and np.array_equal(r["scores"].view(np.uint32),
                                                                      scores.view(np.uint32)), (seed, S, M)
        out[f"hwe_{S}x{M}_{cases}cases"] = {
            "seed": seed, "n_samples": S, "n_snps": M, "n_cases": cases, "triplets": int(len(scores)),
            "geno_sha256": sha(A), "pheno_sha256": sha(B), "tables_sha256": sha(tables.astype("<u4")),
            "scores_sha256": sha(scores.view(np.uint32).astype("<u4")), "ref_best_line": best_line}
        print("tile tap", seed, S, M, best_line)
    json.dump(out, open(os.path.join(HERE, "tile_taps.json"), "w"), indent=1)


def make_precision_top32():
    sys.path.insert(0, os.path.join(REPO, "cross-dpc-episdet_b200"))
    from epik2 import workloads as W
    cfg = W.PRECISION
    A, B = O.gen_hwe(cfg["seed"], cfg["n_samples"], cfg["n_snps"], cfg["n_cases"], cfg["maf"], cfg["planted"],
                     cfg["effects"])
    r = O.topk_fp64(A, B, 32)
    rb = json.load(open(os.path.join(HERE, "ref_best.json")))["precision"]
    assert rb["geno_sha256"] == sha(A) and list(r["ijk"][0]) == rb["ijk"], (r["ijk"][0], rb["ijk"])
    lut = O.lut(cfg["n_samples"] + 1)
    top = [{"ijk": list(ijk), "s64": float(s).hex(), "s32_bits": int(np.float32(O.k2(t, lut)).view(np.uint32)),
            "table": [int(x) for x in t]} for ijk, s, t in zip(r["ijk"], r["s64"], r["tables"])]
    json.dump({"workload": cfg["name"], "seed": cfg["seed"], "geno_sha256": sha(A), "pheno_sha256": sha(B),
               "source": "oracle_topk_fp64_u8 (27-cell AND3+popcount tables, K2 in double)", "top": top},
              open(os.path.join(HERE, "precision_top32.json"), "w"), indent=0)
    print("precision top32:", [t["ijk"] for t in top[:4]], "...")


def main(long_runs, only=None):
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), f"REF_DIR={REF_SRC}"], check=True)
    if only == "tiles":
        return make_tile_taps()
    if only == "top32":
        return make_precision_top32()

    # 1. reference programs on their own srand(100) data
    kat = {}
    for S, M in [(2048, 128), (2000, 100), (2048, 512), (100, 7), (33, 5)]:
        r4 = O.run_ref_gen("ref_v4popc", S, M, 32, 16)
        r2 = O.run_ref_gen("ref_v2", S, M, threads=1)
        assert r4["ijk"] == r2["ijk"] and r4["score_bits"] == r2["score_bits"], (S, M, r4, r2)
        kat[f"{S}x{M}"] = {"n_samples": S, "n_snps": M, "ijk": list(r2["ijk"]), "score_bits": r2["score_bits"],
                           "score": r2["score"]}
        print("kat", S, M, r2["ijk"], r2["score"])
    json.dump(kat, open(os.path.join(HERE, "ref_kat.json"), "w"), indent=1)

    # 2. per-triplet tables from the reference's own code
    tap_case("refgen_256x20", None, None, mode_gen=(256, 20))
    A, B = O.gen_hwe(7, 300, 24, 37)
    tap_case("hwe_300x24_37cases", A, B)
    A, B = O.gen_hwe(8, 40, 12, 5)
    tap_case("hwe_40x12_5cases", A, B)
    A, B = O.gen_hwe(9, 64, 3, 32)
    tap_case("hwe_64x3", A, B)
    A, B = O.gen_hwe(10, 1000, 30, 500, planted=[(3, 17, 29)], effects=[0.9])
    tap_case("hwe_1000x30_planted", A, B)
    # values outside {0,1} count as genotype 2; phenotype values other than 1 are controls
    A, B = O.gen_hwe(11, 100, 10, 50)
    rng = np.random.default_rng(11)
    A = A.copy()
    A[rng.random(A.shape) < 0.05] = 3
    A[rng.random(A.shape) < 0.02] = 255
    B = B.copy()
    B[(B == 0) & (rng.random(B.shape) < 0.2)] = 2
    tap_case("odd_values_100x10", A, B)

    # 3. the reference's ln n!
    with tempfile.TemporaryDirectory() as td:
        p4, p2 = os.path.join(td, "a4"), os.path.join(td, "a2")
        subprocess.run([os.path.join(REF, "ref_v4popc"), "addlog", "70000", p4], check=True)
        subprocess.run([os.path.join(REF, "ref_v2"), "addlog", "70000", p2], check=True)
        a4, a2 = np.fromfile(p4, dtype=np.uint32), np.fromfile(p2, dtype=np.uint32)
    assert (a4 == a2).all()
    np.savez_compressed(os.path.join(HERE, "addlog.npz"), bits=a4)

    # 4. reference CPU search on the seeded Hardy-Weinberg workloads
    sys.path.insert(0, os.path.join(REPO, "cross-dpc-episdet_b200"))
    from epik2 import workloads as W
    path = os.path.join(HERE, "ref_best.json")
    best = json.load(open(path)) if os.path.exists(path) else {}
    cases = [
        ("hwe_3000x150", dict(seed=21, n_snps=150, n_samples=3000, n_cases=1000, maf=(0.05, 0.5), planted=[],
                              effects=[]), None, 32, 16),
        ("hwe_2500x97_planted", dict(seed=22, n_snps=97, n_samples=2500, n_cases=1400, maf=(0.05, 0.5),
                                     planted=[(5, 50, 90)], effects=[0.7]), None, 32, 16),
        ("plain-small", W.PLAIN_SMALL, None, 32, 16),
        ("plain-large-first512", W.PLAIN_LARGE, 512, 64, 16),
    ]
    if long_runs:
        cases += [("precision", W.PRECISION, None, 64, 16), ("plain-large", W.PLAIN_LARGE, None, 64, 16)]
    for name, cfg, sub, bp, bs in cases:
        if name in best:
            continue
        A, B = O.gen_hwe(cfg["seed"], cfg["n_samples"], cfg["n_snps"], cfg["n_cases"], cfg["maf"], cfg["planted"],
                         cfg["effects"])
        if sub:
            A = np.ascontiguousarray(A[:, :sub])
        with tempfile.TemporaryDirectory() as td:
            gp = os.path.join(td, "geno.bin")
            O.write_geno_file(gp, A, B)
            r = O.run_ref_file("ref_v4popc", gp, A.shape[0], A.shape[1], bp, bs)
        best[name] = {"seed": cfg["seed"], "n_samples": int(A.shape[0]), "n_snps": int(A.shape[1]),
                      "source_snps": int(cfg["n_snps"]), "n_cases": int(cfg["n_cases"]), "maf": list(cfg["maf"]),
                      "planted": [list(t) for t in cfg["planted"]], "effects": list(cfg["effects"]),
                      "geno_sha256": sha(A), "pheno_sha256": sha(B), "ijk": list(r["ijk"]),
                      "score_bits": r["score_bits"], "score": r["score"], "ref_wall_search_s": r["wall_search_s"],
                      "ref_threads": r["threads"], "ref_binary": "v4_popc_avx512", "block_pac": bp, "block_snp": bs}
        print("ref_best", name, best[name]["ijk"], best[name]["score"], r["wall_search_s"])
        json.dump(best, open(path, "w"), indent=1)


if __name__ == "__main__":
    main("--long" in sys.argv, sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None)
