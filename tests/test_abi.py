"""The C-ABI library: it loads, exports every declared symbol, and its host-only entry
points (data sources, K2 table, status strings) agree with the oracle and the
reference fixtures.  No GPU needed."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import epik2
import oracle as O
from conftest import ROOT, addlog_bits, ref_best


def test_library_exports_every_declared_symbol():
    lib = epik2.library()
    declared = epik2.exported_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", epik2.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {l.split()[-1] for l in out.stdout.splitlines() if " T " in l}
    assert set(declared) <= exported


def test_probe_library_exports_every_declared_symbol():
    import ctypes as C
    lib = C.CDLL(epik2.PROBE_LIB_PATH)
    declared = epik2.exported_symbols(epik2.PROBE_HEADER)
    assert declared == ["epik2_probe_int_peaks", "epik2_probe_tc_fp4", "epik2_probe_tc_i8"]
    assert all(hasattr(lib, s) for s in declared)


def test_strerror_and_invalid_arguments():
    lib = epik2.library()
    assert epik2.strerror(0) == "ok"
    assert "invalid" in epik2.strerror(epik2.E_INVALID)
    assert lib.epik2_create(None, 0) == epik2.E_INVALID
    assert lib.epik2_generate_reference(0, 5, None, None) == epik2.E_INVALID
    assert lib.epik2_dataset_bytes(0, 10) < 0
    assert lib.epik2_k2_lut(-1, None) == epik2.E_INVALID


def test_no_device_is_reported_not_faked():
    # In a container without a GPU the context must refuse, never fall back to the CPU.
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    assert epik2.library().epik2_create(ctypes.byref(h), 0) == epik2.E_NO_DEVICE


def test_reference_generator_matches_oracle():
    for S, M in [(2000, 100), (33, 5), (257, 31)]:
        g, p = epik2.generate_reference(S, M)
        g2, p2 = O.gen_reference(S, M)
        assert np.array_equal(g, g2) and np.array_equal(p, p2)


def test_hwe_generator_matches_oracle_and_fixtures():
    for name, rec in ref_best().items():
        if rec["n_samples"] * rec["source_snps"] > 3e7:
            continue
        g, p = epik2.generate_hwe(rec["seed"], rec["n_samples"], rec["source_snps"], rec["n_cases"], rec["maf"],
                                  rec["planted"], rec["effects"])
        g = np.ascontiguousarray(g[:, :rec["n_snps"]])
        import hashlib
        assert hashlib.sha256(g.tobytes()).hexdigest() == rec["geno_sha256"], name
        assert hashlib.sha256(p.tobytes()).hexdigest() == rec["pheno_sha256"], name


def test_k2_lut_matches_reference_addlog():
    ref = addlog_bits()
    assert np.array_equal(epik2.k2_lut(len(ref) - 1).view(np.uint32), ref)


def test_dataset_bytes_accounts_for_every_buffer():
    s, m = 16384, 4096
    b = epik2.dataset_bytes(s, m)
    m_pad = 4096
    planes = ((s + 31) // 32 + 1) * m_pad * 8
    pairs = 2 * (m_pad * (m_pad - 1) // 2) * 16
    assert b >= s * m + planes + pairs + (s + 2) * 4
    assert b < (s * m + planes + pairs) * 1.01 + (1 << 20)


def test_cli_usage_errors():
    if not os.path.exists(epik2.CLI_PATH):
        pytest.skip("CLI not built")
    r = subprocess.run([epik2.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_cli_file_input_errors(tmp_path):
    """Reading the --file matrix fails before any device is touched."""
    if not os.path.exists(epik2.CLI_PATH):
        pytest.skip("CLI not built")
    path = tmp_path / "short.bin"
    path.write_bytes(bytes(100))
    r = subprocess.run([epik2.CLI_PATH, "--file", str(path), "50", "10"], capture_output=True, text=True)
    assert r.returncode != 0 and "short read" in r.stderr
    r = subprocess.run([epik2.CLI_PATH, "--file", str(tmp_path / "absent.bin"), "50", "10"], capture_output=True,
                       text=True)
    assert r.returncode != 0 and "cannot open" in r.stderr
