"""The allocation-free entry point epik2_scan_u8_noalloc (GPU).

It serves callers that cannot allocate device memory -- for example a plugin running
inside a host application that owns the device heap -- by keeping every intermediate
in the library's fixed 64 MiB static device array.  Its results must equal the
regular one-call entry point epik2_scan_u8 bit for bit (the tolerance of every search
test here), on consecutive calls that reuse the same array.

Named test_zz_* so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import epik2
from conftest import f32_bits, ref_best

pytestmark = pytest.mark.gpu


def _regular(geno, pheno):
    with epik2.Context(0) as ctx:
        return ctx.scan_u8(geno, pheno)


def _cases():
    rb = ref_best()
    out = []
    for name in ("plain-small", "hwe_3000x150"):
        rec = rb[name]
        g, p = epik2.generate_hwe(rec["seed"], rec["n_samples"], rec["source_snps"], rec["n_cases"], rec["maf"],
                                  rec["planted"], rec["effects"])
        out.append((name, g, p, rec))
    return out


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    lib = epik2.library()
    cases = _cases()
    for name, g, p, rec in cases + cases[:1]:  # A, B, then A again on the same scratch
        ours = epik2.scan_u8_noalloc(g, p)
        reg = _regular(g, p)
        assert ours.ijk == reg.ijk, name
        assert f32_bits(ours.score) == f32_bits(reg.score), name
        assert list(ours.ijk) == rec["ijk"] and f32_bits(ours.score) == rec["score_bits"], name
    # through the raw C ABI as well, on a caller-supplied default stream (NULL)
    name, g, p, rec = cases[1]
    b = epik2.Best()
    g = np.ascontiguousarray(g)
    r = lib.epik2_scan_u8_noalloc(g.ctypes.data_as(ctypes.c_void_p), p.ctypes.data_as(ctypes.c_void_p),
                                  g.shape[0], g.shape[1], None, ctypes.byref(b))
    assert r == epik2.OK
    assert list(b.ijk) == rec["ijk"] and f32_bits(b.score) == rec["score_bits"]


def test_noalloc_rejects_shapes_beyond_its_array():
    lib = epik2.library()
    b = epik2.Best()
    g = np.zeros((16, 8), dtype=np.uint8)
    p = np.zeros(16, dtype=np.uint8)
    # 5000 SNPs is over the 4096-SNP limit; 4096 SNPs x 16384 samples needs far more than 64 MiB
    assert lib.epik2_scan_u8_noalloc(g.ctypes.data_as(ctypes.c_void_p), p.ctypes.data_as(ctypes.c_void_p), 16, 5000,
                                     None, ctypes.byref(b)) == epik2.E_TOO_LARGE
    big = np.zeros((16384, 4096), dtype=np.uint8)
    pb = np.zeros(16384, dtype=np.uint8)
    assert lib.epik2_scan_u8_noalloc(big.ctypes.data_as(ctypes.c_void_p), pb.ctypes.data_as(ctypes.c_void_p),
                                     16384, 4096, None, ctypes.byref(b)) == epik2.E_TOO_LARGE
