"""Python host binding of libepik2 (the C ABI in include/epik2.h).

The compute path is the CUDA library; this module only marshals arguments.  There is
no CPU fallback: if the shared library is missing or no sm_100 GPU is visible, the
calls raise.
"""
import ctypes
import math
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(HERE, "lib", "libepik2.so")
CLI_PATH = os.path.join(HERE, "bin", "epik2_v4")
HEADER = os.path.join(REPO_ROOT, "include", "epik2.h")

OK = 0
E_INVALID = -1
E_CUDA = -2
E_NOMEM = -3
E_NOT_FOUND = -4
E_TOO_LARGE = -5
E_TIMEOUT = -6
E_NO_DEVICE = -7
E_BUSY = -8
E_CANCELLED = -9

ENGINE_AUTO = 0
ENGINE_INT = 1
ENGINE_TC = 2
ENGINE_TC_FP4 = 3


class Epik2Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"epik2 status {status}: {msg}")
        self.status = status


class Best(ctypes.Structure):
    _fields_ = [("score", ctypes.c_float), ("_pad", ctypes.c_float), ("score_fp64", ctypes.c_double),
                ("i", ctypes.c_uint32), ("j", ctypes.c_uint32), ("k", ctypes.c_uint32), ("_pad2", ctypes.c_uint32)]

    @property
    def ijk(self):
        return (int(self.i), int(self.j), int(self.k))

    def __repr__(self):
        return f"Best(score={self.score!r}, score_fp64={self.score_fp64!r}, ijk={self.ijk})"


class Stats(ctypes.Structure):
    _fields_ = [("kernel_launches", ctypes.c_uint64), ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("last_scan_kernel_ms", ctypes.c_double), ("last_scan_triplets", ctypes.c_int64),
                ("last_scan_words", ctypes.c_int64), ("last_load_ms", ctypes.c_double),
                ("last_upload_ms", ctypes.c_double), ("last_prepare_ms", ctypes.c_double),
                ("last_scan_wall_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Tune(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int32), ("stage_words", ctypes.c_int32), ("rate_int", ctypes.c_double),
                ("rate_tc4", ctypes.c_double), ("rate_tc8", ctypes.c_double), ("rate_fp4_8", ctypes.c_double),
                ("rate_fp4_16", ctypes.c_double), ("rate_fp4_8_pair", ctypes.c_double),
                ("rate_fp4_16_single", ctypes.c_double), ("pair_tile", ctypes.c_int32), ("overlap", ctypes.c_int32),
                ("rate_fp4_4_overlap", ctypes.c_double), ("rate_fp4_8_overlap", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_reserve_bytes", ctypes.c_int64), ("batch_work", ctypes.c_double), ("max_active", ctypes.c_int32),
                ("max_queued", ctypes.c_int32), ("rescore_fp64", ctypes.c_int32), ("stage_words", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("rejected", ctypes.c_int64),
                ("cancelled", ctypes.c_int64), ("scans_queued", ctypes.c_int64), ("scans_active", ctypes.c_int64),
                ("scans_done", ctypes.c_int64), ("launches", ctypes.c_int64), ("triplet_samples", ctypes.c_double),
                ("busy_seconds", ctypes.c_double), ("max_active", ctypes.c_int64),
                ("kernel_seconds", ctypes.c_double), ("replicate_scans", ctypes.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Opts(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int32), ("top_k", ctypes.c_int32), ("rescore_fp64", ctypes.c_int32),
                ("pair_tile", ctypes.c_int32), ("stage_words", ctypes.c_int32), ("overlap", ctypes.c_int32),
                ("snp_begin", ctypes.c_int64), ("snp_end", ctypes.c_int64)]


_lib = None


PROBE_LIB_PATH = os.path.join(HERE, "lib", "libepik2_probe.so")
PROBE_HEADER = os.path.join(REPO_ROOT, "include", "epik2_probe.h")


def exported_symbols(header=HEADER):
    """Function names declared in a header of include/."""
    with open(header) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(epik2_[a-z0-9_]+)\s*\(", text)))


def library():
    """Load libepik2.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise Epik2Error(E_NO_DEVICE, f"{LIB_PATH} not built (run __graft_entry__.build() or make -C {PKG_ROOT})")
    L = ctypes.CDLL(LIB_PATH)
    p, i32, i64, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64
    sig = {
        "epik2_create": ([ctypes.POINTER(p), ctypes.c_int], ctypes.c_int),
        "epik2_destroy": ([p], None),
        "epik2_strerror": ([ctypes.c_int], ctypes.c_char_p),
        "epik2_last_error": ([p], ctypes.c_char_p),
        "epik2_device_name": ([p, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "epik2_mem_info": ([p, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
        "epik2_generate_reference": ([i64, i64, p, p], ctypes.c_int),
        "epik2_generate_hwe": ([u64, i64, i64, i64, ctypes.c_double, ctypes.c_double, i32, p, p, p, p], ctypes.c_int),
        "epik2_load_u8": ([p, p, p, i64, i64, ctypes.POINTER(i32)], ctypes.c_int),
        "epik2_set_pheno": ([p, i32, p], ctypes.c_int),
        "epik2_unload": ([p, i32], ctypes.c_int),
        "epik2_dataset_info": ([p, i32, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                ctypes.POINTER(i64)], ctypes.c_int),
        "epik2_dataset_bytes": ([i64, i64], i64),
        "epik2_scan": ([p, i32, ctypes.POINTER(Opts), ctypes.POINTER(Best)], ctypes.c_int),
        "epik2_scan_topk": ([p, i32, ctypes.POINTER(Opts), ctypes.POINTER(Best), i32, ctypes.POINTER(i32)],
                            ctypes.c_int),
        "epik2_scan_u8": ([p, p, p, i64, i64, ctypes.POINTER(Opts), ctypes.POINTER(Best)], ctypes.c_int),
        "epik2_dump_tables": ([p, i32, p, p], ctypes.c_int),
        "epik2_tables": ([p, i32, p, i64, p], ctypes.c_int),
        "epik2_k2_lut": ([i64, p], ctypes.c_int),
        "epik2_set_stream": ([p, p], ctypes.c_int),
        "epik2_get_stream": ([p, ctypes.POINTER(p)], ctypes.c_int),
        "epik2_get_stats": ([p, ctypes.POINTER(Stats)], ctypes.c_int),
        "epik2_reset_stats": ([p], ctypes.c_int),
        "epik2_scan_u8_noalloc": ([p, p, i64, i64, p, ctypes.POINTER(Best)], ctypes.c_int),
        "epik2_set_engine": ([p, ctypes.c_int], ctypes.c_int),
        "epik2_set_stage_words": ([p, ctypes.c_int], ctypes.c_int),
        "epik2_set_wait_limit": ([p, i64], ctypes.c_int),
        "epik2_set_pair_tile": ([p, ctypes.c_int], ctypes.c_int),
        "epik2_set_overlap": ([p, ctypes.c_int], ctypes.c_int),
        "epik2_test_withhold_arrival": ([p], ctypes.c_int),
        "epik2_plink_dims": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
                             ctypes.c_int),
        "epik2_read_plink": ([ctypes.c_char_p, ctypes.c_uint8, p, p], ctypes.c_int),
        "epik2_perm_pvalue": ([ctypes.c_float, p, ctypes.c_int64], ctypes.c_double),
        "epik2_scan_batch": ([p, p, i32, ctypes.POINTER(Opts), ctypes.POINTER(Best)], ctypes.c_int),
        "epik2_scan_replicates": ([p, i32, p, i32, ctypes.POINTER(Opts), ctypes.POINTER(Best)], ctypes.c_int),
        "epik2_autotune": ([p, i32, ctypes.POINTER(Tune)], ctypes.c_int),
        "epik2_load_replicate": ([p, i32, p, ctypes.POINTER(i32)], ctypes.c_int),
        "epik2_replicate_bytes": ([i64, i64], i64),
        "epik2_server_create": ([ctypes.POINTER(p), ctypes.c_int, ctypes.POINTER(ServerOpts)], ctypes.c_int),
        "epik2_server_destroy": ([p], None),
        "epik2_server_add_matrix": ([p, p, p, i64, i64, ctypes.POINTER(i32)], ctypes.c_int),
        "epik2_server_submit_replicates": ([p, i32, p, i32, ctypes.POINTER(i64)], ctypes.c_int),
        "epik2_server_submit_scan": ([p, p, p, i64, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "epik2_server_poll": ([p, i64, ctypes.POINTER(Best), i32, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_double)],
                              ctypes.c_int),
        "epik2_server_cancel": ([p, i64], ctypes.c_int),
        "epik2_server_get_stats": ([p, ctypes.POINTER(ServerStats)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def strerror(status):
    return library().epik2_strerror(status).decode()


def generate_reference(n_samples, n_snps):
    """The reference's srand(100) synthetic data: (geno [S][M] uint8, pheno [S] uint8)."""
    g = np.empty((n_samples, n_snps), dtype=np.uint8)
    ph = np.empty(n_samples, dtype=np.uint8)
    r = library().epik2_generate_reference(n_samples, n_snps, _ptr(g), _ptr(ph))
    if r:
        raise Epik2Error(r, strerror(r))
    return g, ph


def generate_hwe(seed, n_samples, n_snps, n_cases, maf=(0.05, 0.5), planted=(), effects=()):
    """Seeded Hardy-Weinberg matrix with planted triplets: (geno [S][M] uint8, pheno [S] uint8)."""
    g = np.empty((n_samples, n_snps), dtype=np.uint8)
    ph = np.empty(n_samples, dtype=np.uint8)
    pl = np.ascontiguousarray(np.array(planted, dtype=np.int64).reshape(-1, 3))
    ef = np.ascontiguousarray(np.array(effects, dtype=np.float64).reshape(-1))
    if len(pl) != len(ef):
        raise ValueError("planted and effects differ in length")
    r = library().epik2_generate_hwe(seed, n_samples, n_snps, n_cases, float(maf[0]), float(maf[1]), len(pl),
                                     _ptr(pl), _ptr(ef), _ptr(g), _ptr(ph))
    if r:
        raise Epik2Error(r, strerror(r))
    return g, ph


NOALLOC_SCRATCH_BYTES = 64 << 20


def scan_u8_noalloc(geno, pheno, stream=None):
    """Allocation-free one-call search on the current device (epik2_scan_u8_noalloc).

    For callers that cannot allocate device memory: all intermediates live in the
    library's fixed 64 MiB static device array.  Raises Epik2Error on failure."""
    geno = np.ascontiguousarray(geno, dtype=np.uint8)
    pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
    b = Best()
    r = library().epik2_scan_u8_noalloc(_ptr(geno), _ptr(pheno), geno.shape[0], geno.shape[1],
                                        ctypes.c_void_p(stream or None), ctypes.byref(b))
    if r:
        raise Epik2Error(r, strerror(r))
    return b


def k2_lut(n_max):
    out = np.empty(n_max + 1, dtype=np.float32)
    r = library().epik2_k2_lut(n_max, _ptr(out))
    if r:
        raise Epik2Error(r, strerror(r))
    return out


def dataset_bytes(n_samples, n_snps):
    return int(library().epik2_dataset_bytes(n_samples, n_snps))


def read_plink(prefix, missing_genotype=0):
    """PLINK 1 binary fileset -> (geno uint8 [samples, SNPs], pheno uint8 [samples])."""
    L = library()
    n, m = ctypes.c_int64(), ctypes.c_int64()
    r = L.epik2_plink_dims(prefix.encode(), ctypes.byref(n), ctypes.byref(m))
    if r:
        raise Epik2Error(r, f"{strerror(r)}: {prefix}")
    geno = np.zeros((n.value, m.value), dtype=np.uint8)
    pheno = np.zeros(n.value, dtype=np.uint8)
    r = L.epik2_read_plink(prefix.encode(), missing_genotype, _ptr(geno), _ptr(pheno))
    if r:
        raise Epik2Error(r, f"{strerror(r)}: {prefix}")
    return geno, pheno


def perm_pvalue(observed, replicate_best):
    """Permutation p-value: (1 + #{replicate best <= observed}) / (1 + replicates)."""
    rb = np.ascontiguousarray(np.asarray(replicate_best, dtype=np.float32))
    return float(library().epik2_perm_pvalue(np.float32(observed), _ptr(rb), len(rb)))


def n_triplets(m):
    return m * (m - 1) * (m - 2) // 6 if m >= 3 else 0


class Context:
    """One device context: owns a CUDA stream and the resident datasets."""

    def __init__(self, device=0, engine=ENGINE_AUTO, stage_words=0, pair_tile=0, overlap=0):
        self._lib = library()
        h = ctypes.c_void_p()
        r = self._lib.epik2_create(ctypes.byref(h), device)
        if r:
            raise Epik2Error(r, strerror(r))
        self._h = h
        if engine:
            self.set_engine(engine)
        if stage_words:
            self.set_stage_words(stage_words)
        if pair_tile:
            self.set_pair_tile(pair_tile)
        if overlap:
            self.set_overlap(overlap)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.epik2_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, r):
        if r:
            msg = self._lib.epik2_last_error(self._h)
            raise Epik2Error(r, f"{strerror(r)}: {msg.decode() if msg else ''}")

    @property
    def handle(self):
        return self._h

    def set_engine(self, engine):
        """Default engine of this context: ENGINE_AUTO, ENGINE_INT, ENGINE_TC or ENGINE_TC_FP4."""
        self._check(self._lib.epik2_set_engine(self._h, engine))

    def set_stage_words(self, stage_words):
        """Default tensor-core stage depth (0 = autotuned; int8 4/8, FP4 8/16)."""
        self._check(self._lib.epik2_set_stage_words(self._h, stage_words))

    def set_pair_tile(self, pair_tile):
        """Default tensor-core pair tile (0 = autotuned; 32, or 64 = FP4 on CTA pairs)."""
        self._check(self._lib.epik2_set_pair_tile(self._h, pair_tile))

    def set_overlap(self, overlap):
        """Default overlapped-kernel choice (0 = tuned, 1 = off, 2 = on; FP4 on CTA pairs)."""
        self._check(self._lib.epik2_set_overlap(self._h, overlap))

    def set_wait_limit(self, sm_clocks):
        """SM clocks a bounded device-side wait lasts before the search gives up (0 = ~2 s)."""
        self._check(self._lib.epik2_set_wait_limit(self._h, int(sm_clocks)))

    def test_withhold_arrival(self):
        """Test hook: the next single-CTA tensor-core search times out (EPIK2_E_TIMEOUT)."""
        self._check(self._lib.epik2_test_withhold_arrival(self._h))

    def stats(self):
        st = Stats()
        self._check(self._lib.epik2_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        self._check(self._lib.epik2_reset_stats(self._h))

    def stream(self):
        """The cudaStream_t (as an int) the context launches on."""
        v = ctypes.c_void_p()
        self._check(self._lib.epik2_get_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    def set_stream(self, stream_ptr):
        self._check(self._lib.epik2_set_stream(self._h, ctypes.c_void_p(stream_ptr or None)))

    def device_name(self):
        buf = ctypes.create_string_buffer(256)
        self._check(self._lib.epik2_device_name(self._h, buf, 256))
        return buf.value.decode()

    def mem_info(self):
        fr, tot = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(self._lib.epik2_mem_info(self._h, ctypes.byref(fr), ctypes.byref(tot)))
        return fr.value, tot.value

    def load(self, geno, pheno):
        geno = np.ascontiguousarray(geno, dtype=np.uint8)
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        if geno.ndim != 2 or pheno.shape != (geno.shape[0],):
            raise ValueError("geno must be [n_samples][n_snps] and pheno [n_samples]")
        did = ctypes.c_int32()
        self._check(self._lib.epik2_load_u8(self._h, _ptr(geno), _ptr(pheno), geno.shape[0], geno.shape[1],
                                            ctypes.byref(did)))
        return did.value

    def set_pheno(self, dataset, pheno):
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        self._check(self._lib.epik2_set_pheno(self._h, dataset, _ptr(pheno)))

    def unload(self, dataset):
        self._check(self._lib.epik2_unload(self._h, dataset))

    def info(self, dataset):
        s, m, c, b = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(self._lib.epik2_dataset_info(self._h, dataset, ctypes.byref(s), ctypes.byref(m), ctypes.byref(c),
                                                 ctypes.byref(b)))
        return {"n_samples": s.value, "n_snps": m.value, "n_cases": c.value, "device_bytes": b.value}

    @staticmethod
    def _opts(**kw):
        o = Opts()
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def scan(self, dataset, **opts):
        o = self._opts(**opts)
        b = Best()
        self._check(self._lib.epik2_scan(self._h, dataset, ctypes.byref(o), ctypes.byref(b)))
        return b

    def scan_topk(self, dataset, k=32, **opts):
        o = self._opts(top_k=k, **opts)
        arr = (Best * k)()
        n = ctypes.c_int32()
        self._check(self._lib.epik2_scan_topk(self._h, dataset, ctypes.byref(o), arr, k, ctypes.byref(n)))
        return [arr[t] for t in range(n.value)]

    def scan_u8(self, geno, pheno, **opts):
        geno = np.ascontiguousarray(geno, dtype=np.uint8)
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        o = self._opts(**opts)
        b = Best()
        self._check(self._lib.epik2_scan_u8(self._h, _ptr(geno), _ptr(pheno), geno.shape[0], geno.shape[1],
                                            ctypes.byref(o), ctypes.byref(b)))
        return b

    def scan_batch(self, datasets, **opts):
        """Best triplet of each dataset from one batched, graph-captured launch."""
        ids = np.ascontiguousarray(np.asarray(datasets, dtype=np.int32))
        o = self._opts(**opts)
        arr = (Best * len(ids))()
        self._check(self._lib.epik2_scan_batch(self._h, _ptr(ids), len(ids), ctypes.byref(o), arr))
        return [arr[t] for t in range(len(ids))]

    def scan_replicates(self, dataset, phenos, **opts):
        """Best triplet of each phenotype-permutation replicate (rows of phenos) of a resident
        dataset, the all-sample counts shared across replicates (epik2_scan_replicates)."""
        phenos = np.ascontiguousarray(np.atleast_2d(phenos), dtype=np.uint8)
        arr = (Best * len(phenos))()
        o = self._opts(**opts)
        self._check(self._lib.epik2_scan_replicates(self._h, dataset, _ptr(phenos), len(phenos), ctypes.byref(o),
                                                    arr))
        return [arr[t] for t in range(len(phenos))]

    def autotune(self, dataset):
        t = Tune()
        self._check(self._lib.epik2_autotune(self._h, dataset, ctypes.byref(t)))
        return t.as_dict()

    def load_replicate(self, dataset, pheno):
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        did = ctypes.c_int32()
        self._check(self._lib.epik2_load_replicate(self._h, dataset, _ptr(pheno), ctypes.byref(did)))
        return did.value

    def dump_tables(self, dataset):
        m = self.info(dataset)["n_snps"]
        T = n_triplets(m)
        tables = np.zeros((T, 54), dtype=np.uint32)
        scores = np.zeros(T, dtype=np.float32)
        self._check(self._lib.epik2_dump_tables(self._h, dataset, _ptr(tables), _ptr(scores)))
        return tables, scores

    def tables(self, dataset, triplets):
        t = np.ascontiguousarray(np.asarray(triplets, dtype=np.uint32).reshape(-1, 3))
        out = np.zeros((len(t), 54), dtype=np.uint32)
        self._check(self._lib.epik2_tables(self._h, dataset, _ptr(t), len(t), _ptr(out)))
        return out


def probe_int_peaks(device=0):
    """Measured POPC / LOP3 / IADD rates of the device (operations per second) and the dense
    int8 and FP4 tensor-core rates (multiply-accumulates per second)."""
    if not os.path.exists(PROBE_LIB_PATH):
        raise Epik2Error(E_NO_DEVICE, f"{PROBE_LIB_PATH} not built")
    L = ctypes.CDLL(PROBE_LIB_PATH)
    d = ctypes.POINTER(ctypes.c_double)
    L.epik2_probe_int_peaks.argtypes = [ctypes.c_int, d, d, d]
    L.epik2_probe_int_peaks.restype = ctypes.c_int
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    r = L.epik2_probe_int_peaks(device, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    if r:
        raise Epik2Error(r, "probe failed")
    out = {"popc_per_s": a.value, "lop3_per_s": b.value, "iadd_per_s": c.value}
    L.epik2_probe_tc_i8.argtypes = [ctypes.c_int, d]
    L.epik2_probe_tc_i8.restype = ctypes.c_int
    m = ctypes.c_double()
    if L.epik2_probe_tc_i8(device, ctypes.byref(m)) == 0:
        out["tc_i8_mac_per_s"] = m.value
    L.epik2_probe_tc_fp4.argtypes = [ctypes.c_int, d]
    L.epik2_probe_tc_fp4.restype = ctypes.c_int
    if L.epik2_probe_tc_fp4(device, ctypes.byref(m)) == 0:
        out["tc_fp4_mac_per_s"] = m.value
    return out


class Server:
    """Continuous-batching request server (epik2_server_*): one device context, one
    worker thread, requests from any thread."""

    def __init__(self, device=0, **opts):
        self._lib = library()
        o = ServerOpts()
        for k, v in opts.items():
            setattr(o, k, v)
        h = ctypes.c_void_p()
        r = self._lib.epik2_server_create(ctypes.byref(h), device, ctypes.byref(o))
        if r:
            raise Epik2Error(r, strerror(r))
        self._h = h
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.epik2_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_matrix(self, geno, pheno):
        geno = np.ascontiguousarray(geno, dtype=np.uint8)
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        mid = ctypes.c_int32()
        r = self._lib.epik2_server_add_matrix(self._h, _ptr(geno), _ptr(pheno), geno.shape[0], geno.shape[1],
                                              ctypes.byref(mid))
        if r:
            raise Epik2Error(r, strerror(r))
        self._sizes[mid.value] = geno.shape[0]
        return mid.value

    def submit_replicates(self, matrix, phenos):
        phenos = np.ascontiguousarray(phenos, dtype=np.uint8)
        rid = ctypes.c_int64()
        r = self._lib.epik2_server_submit_replicates(self._h, matrix, _ptr(phenos), phenos.shape[0], ctypes.byref(rid))
        if r:
            raise Epik2Error(r, strerror(r))
        return rid.value

    def submit_scan(self, geno, pheno):
        geno = np.ascontiguousarray(geno, dtype=np.uint8)
        pheno = np.ascontiguousarray(pheno, dtype=np.uint8)
        rid = ctypes.c_int64()
        r = self._lib.epik2_server_submit_scan(self._h, _ptr(geno), _ptr(pheno), geno.shape[0], geno.shape[1],
                                               ctypes.byref(rid))
        if r:
            raise Epik2Error(r, strerror(r))
        return rid.value

    def poll(self, request, capacity=1024):
        """None while running; (status, [Best], latency_s) once done (record released)."""
        arr = (Best * capacity)()
        n = ctypes.c_int32()
        lat = ctypes.c_double()
        r = self._lib.epik2_server_poll(self._h, request, arr, capacity, ctypes.byref(n), ctypes.byref(lat))
        if r == E_BUSY:
            return None
        if r == E_NOT_FOUND:
            raise Epik2Error(r, "unknown request")
        return r, [arr[t] for t in range(n.value)], lat.value

    def wait(self, request, timeout=600.0, capacity=1024):
        import time
        t0 = time.time()
        while True:
            res = self.poll(request, capacity)
            if res is not None:
                return res
            if time.time() - t0 > timeout:
                raise TimeoutError(f"request {request} not done after {timeout} s")
            time.sleep(0.002)

    def cancel(self, request):
        return self._lib.epik2_server_cancel(self._h, request)

    def stats(self):
        st = ServerStats()
        self._lib.epik2_server_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()
