"""ctypes binding of the C oracle (oracle.c) and runners for the reference harnesses.

TEST INFRASTRUCTURE ONLY: imported by the test suite, the smoke check and the
CPU-baseline leg of the benchmark, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    """Compile the oracle (and the reference harnesses when the sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        i64, u64, p = ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p
        L.oracle_gen_reference.argtypes = [i64, i64, p, p]
        L.oracle_mt64_nth.argtypes = [u64, i64]
        L.oracle_mt64_nth.restype = u64
        L.oracle_gen_hwe.argtypes = [u64, i64, i64, i64, ctypes.c_double, ctypes.c_double, ctypes.c_int, p, p, p, p]
        L.oracle_encode.argtypes = [p, p, i64, i64, p, p, p]
        L.oracle_masks.argtypes = [i64, i64, p, p]
        L.oracle_table.argtypes = [p, p, i64, i64, i64, i64, i64, p]
        L.oracle_lut.argtypes = [i64, p]
        L.oracle_k2.argtypes = [p, p]
        L.oracle_k2.restype = ctypes.c_float
        L.oracle_k2_fp64.argtypes = [p]
        L.oracle_k2_fp64.restype = ctypes.c_double
        L.oracle_k2_lgamma.argtypes = [p]
        L.oracle_k2_lgamma.restype = ctypes.c_double
        L.oracle_lnfact_fp64.argtypes = [i64]
        L.oracle_lnfact_fp64.restype = ctypes.c_double
        L.oracle_triplet_index.argtypes = [i64, i64, i64, i64]
        L.oracle_triplet_index.restype = i64
        L.oracle_scan.argtypes = [p, p, i64, i64, i64, p, p, p, p, p, ctypes.c_int]
        L.oracle_scan.restype = i64
        L.oracle_scan_u8.argtypes = [p, p, i64, i64, p, p, p, p, ctypes.c_int]
        L.oracle_scan_u8.restype = i64
        L.oracle_scan_fp64_u8.argtypes = [p, p, i64, i64, p, ctypes.c_int]
        L.oracle_scan_fp64_u8.restype = i64
        L.oracle_topk_fp64_u8.argtypes = [p, p, i64, i64, ctypes.c_int, p, p, p, ctypes.c_int]
        L.oracle_topk_fp64_u8.restype = i64
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def gen_reference(n_samples, n_snps):
    """The reference's srand(100)/rand() data: geno [S][M] uint8, pheno [S] uint8."""
    A = np.zeros((n_samples, n_snps), dtype=np.uint8)
    B = np.zeros(n_samples + 1, dtype=np.uint8)
    lib().oracle_gen_reference(n_samples, n_snps, _ptr(A), _ptr(B))
    return A, B[:n_samples].copy()


def gen_hwe(seed, n_samples, n_snps, n_cases, maf=(0.05, 0.5), planted=(), effects=()):
    A = np.zeros((n_samples, n_snps), dtype=np.uint8)
    B = np.zeros(max(n_samples, 1), dtype=np.uint8)
    pl = np.ascontiguousarray(np.array(planted, dtype=np.int64).reshape(-1, 3))
    ef = np.ascontiguousarray(np.array(effects, dtype=np.float64).reshape(-1))
    assert len(pl) == len(ef)
    lib().oracle_gen_hwe(seed, n_samples, n_snps, n_cases, float(maf[0]), float(maf[1]), len(pl),
                         _ptr(pl), _ptr(ef), _ptr(A), _ptr(B))
    return A, B[:n_samples].copy()


def mt64_nth(seed, n):
    return int(lib().oracle_mt64_nth(seed, n))


def encode(A, B):
    """Reference planes per class, layout [snp][word][2] (CPU/v2.cpp:122-150)."""
    A = np.ascontiguousarray(A, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    S, M = A.shape
    n1 = int((B == 1).sum())
    n0 = S - n1
    W0, W1 = (n0 + 31) // 32, (n1 + 31) // 32
    z = np.zeros(M * W0 * 2 + 1, dtype=np.uint32)
    o = np.zeros(M * W1 * 2 + 1, dtype=np.uint32)
    out = ctypes.c_int64(0)
    lib().oracle_encode(_ptr(A), _ptr(B), S, M, _ptr(z), _ptr(o), ctypes.byref(out))
    return z[: M * W0 * 2].reshape(M, W0, 2), o[: M * W1 * 2].reshape(M, W1, 2), n0, n1


def lut(n_max):
    out = np.zeros(n_max + 1, dtype=np.float32)
    lib().oracle_lut(n_max, _ptr(out))
    return out


def table(A, B, i, j, k):
    z, o, n0, n1 = encode(A, B)
    ft = np.zeros(54, dtype=np.uint32)
    lib().oracle_table(_ptr(np.ascontiguousarray(z)), _ptr(np.ascontiguousarray(o)), n0, n1, i, j, k, _ptr(ft))
    return ft


def k2(ft54, lut_arr):
    ft = np.ascontiguousarray(ft54, dtype=np.uint32)
    return float(lib().oracle_k2(_ptr(ft), _ptr(np.ascontiguousarray(lut_arr, dtype=np.float32))))


def k2_fp64(ft54):
    return float(lib().oracle_k2_fp64(_ptr(np.ascontiguousarray(ft54, dtype=np.uint32))))


def k2_lgamma(ft54):
    return float(lib().oracle_k2_lgamma(_ptr(np.ascontiguousarray(ft54, dtype=np.uint32))))


def triplet_index(M, i, j, k):
    return int(lib().oracle_triplet_index(M, i, j, k))


def scan(A, B, with_tables=False, n_threads=0):
    """Exhaustive scan: returns dict(score, ijk, tables?, scores?)."""
    A = np.ascontiguousarray(A, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    S, M = A.shape
    T = M * (M - 1) * (M - 2) // 6 if M >= 3 else 0
    tables = np.zeros((max(T, 1), 54), dtype=np.uint32) if with_tables else None
    scores = np.zeros(max(T, 1), dtype=np.float32) if with_tables else None
    bs = ctypes.c_float(0)
    ijk = np.zeros(3, dtype=np.int64)
    lib().oracle_scan_u8(_ptr(A), _ptr(B), S, M, ctypes.byref(bs), _ptr(ijk),
                         _ptr(tables) if with_tables else None, _ptr(scores) if with_tables else None, n_threads)
    out = {"score": float(np.float32(bs.value)), "ijk": tuple(int(x) for x in ijk), "T": T}
    if with_tables:
        out["tables"] = tables[:T]
        out["scores"] = scores[:T]
    return out


def scan_fp64(A, B, n_threads=0):
    """FP64 K2 of every triplet, in lexicographic order."""
    A = np.ascontiguousarray(A, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    S, M = A.shape
    T = M * (M - 1) * (M - 2) // 6 if M >= 3 else 0
    out = np.zeros(max(T, 1), dtype=np.float64)
    lib().oracle_scan_fp64_u8(_ptr(A), _ptr(B), S, M, _ptr(out), n_threads)
    return out[:T]


def topk_fp64(A, B, k=32, n_threads=0):
    """The k lowest FP64 K2 scores over all triplets (ties to the lowest index), in order:
    dict(ijk=[(i,j,k)...], s64=float64 array, tables=uint32 [k][54])."""
    A = np.ascontiguousarray(A, dtype=np.uint8)
    B = np.ascontiguousarray(B, dtype=np.uint8)
    S, M = A.shape
    t = np.zeros(k, dtype=np.int64)
    s64 = np.zeros(k, dtype=np.float64)
    ft = np.zeros((k, 54), dtype=np.uint32)
    n = lib().oracle_topk_fp64_u8(_ptr(A), _ptr(B), S, M, k, _ptr(t), _ptr(s64), _ptr(ft), n_threads)
    ijk = [triplet_of(M, int(x)) for x in t[:n]]
    return {"ijk": ijk, "s64": s64[:n].copy(), "tables": ft[:n].copy(), "t": t[:n].copy()}


def triplet_of(M, t):
    """(i, j, k) of lexicographic triplet index t among C(M,3)."""
    i = 0
    while i + 1 < M - 2 and triplet_index(M, i + 1, i + 2, i + 3) <= t:
        i += 1
    j = i + 1
    while j + 1 < M - 1 and triplet_index(M, i, j + 1, j + 2) <= t:
        j += 1
    return (i, j, j + 1 + (t - triplet_index(M, i, j, j + 1)))


def triplet_list(M):
    return [(i, j, k) for i in range(M) for j in range(i + 1, M) for k in range(j + 1, M)]


# ---------------------------------------------------------------- reference harnesses

def ref_available(name="ref_v4popc"):
    return os.path.exists(os.path.join(REF_DIR, name))


def write_geno_file(path, A, B):
    with open(path, "wb") as f:
        f.write(np.ascontiguousarray(A, dtype=np.uint8).tobytes())
        f.write(np.ascontiguousarray(B, dtype=np.uint8).tobytes())


def parse_harness_output(text):
    res = {}
    for line in text.splitlines():
        parts = line.split()
        if line.startswith("EXACT"):
            res["ijk"] = (int(parts[1]), int(parts[2]), int(parts[3]))
            bits = int(parts[5], 16)
            res["score_bits"] = bits
            res["score"] = float(np.array([bits], dtype=np.uint32).view(np.float32)[0])
        elif line.startswith("WALL_SEARCH_S"):
            res["wall_search_s"] = float(parts[1])
        elif line.startswith("WALL_ENCODE_S"):
            res["wall_encode_s"] = float(parts[1])
        elif line.startswith("THREADS"):
            res["threads"] = int(parts[1])
    return res


def run_ref_file(binary, geno_path, S, M, block_pac=None, block_snp=None, threads=None, timeout=None):
    cmd = [os.path.join(REF_DIR, binary), "file", geno_path, str(S), str(M)]
    if block_pac is not None:
        cmd += [str(block_pac), str(block_snp)]
    env = dict(os.environ)
    if threads is not None:
        env["REF_THREADS"] = str(threads)
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env, timeout=timeout)
    return parse_harness_output(r.stdout)


def run_ref_gen(binary, S, M, block_pac=None, block_snp=None, threads=None):
    cmd = [os.path.join(REF_DIR, binary), "gen", str(S), str(M)]
    if block_pac is not None:
        cmd += [str(block_pac), str(block_snp)]
    env = dict(os.environ)
    if threads is not None:
        env["REF_THREADS"] = str(threads)
    r = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env)
    return parse_harness_output(r.stdout)


def host_cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def best_ref_binary():
    """v4_popc_avx512 if the host has VPOPCNTDQ, else v4_avx512, else v4_avx."""
    fl = host_cpu_flags()
    if {"avx512_vpopcntdq", "avx512f", "avx512bw"} <= fl and ref_available("ref_v4popc"):
        return "ref_v4popc"
    if {"avx512f", "avx512bw"} <= fl and ref_available("ref_v4avx512"):
        return "ref_v4avx512"
    if ref_available("ref_v4avx"):
        return "ref_v4avx"
    return None
