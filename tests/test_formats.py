"""Input files and permutation statistics around the search: the PLINK 1 binary fileset
reader (host code, CPU tests; the GPU test runs the command-line drop-in on a fileset) and
the permutation p-value."""
import os
import subprocess

import numpy as np
import pytest

import epik2

CODE = {2: 0b00, 1: 0b10, 0: 0b11}  # count of the first allele -> PLINK 2-bit code; 0b01 missing


def write_plink(prefix, geno, status, missing=None):
    """geno [N, M] in {0,1,2}; status per sample: 'case', 'control' or 'missing';
    missing: boolean [N, M] of missing genotypes."""
    n, m = geno.shape
    with open(prefix + ".fam", "w") as f:
        for s in range(n):
            ph = {"case": "2", "control": "1", "missing": "-9"}[status[s]]
            f.write(f"FAM{s}\tIND{s} 0 0 {1 + s % 2} {ph}\n")
        f.write("\n")  # a trailing blank line is ignored
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"1 rs{j} 0 {1000 + j} A G\n")
    with open(prefix + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        row = (n + 3) // 4
        for j in range(m):
            b = bytearray(row)
            for s in range(n):
                c = 0b01 if (missing is not None and missing[s, j]) else CODE[int(geno[s, j])]
                b[s // 4] |= c << (2 * (s % 4))
            f.write(bytes(b))


def make_case(tmp_path, seed=3, n=203, m=17):
    rng = np.random.default_rng(seed)
    geno = rng.integers(0, 3, size=(n, m), dtype=np.uint8)
    status = rng.choice(["case", "control", "missing"], size=n, p=[0.45, 0.45, 0.10])
    missing = rng.random((n, m)) < 0.03
    prefix = str(tmp_path / "study")
    write_plink(prefix, geno, status, missing)
    return prefix, geno, status, missing


def test_plink_reader_maps_genotypes_samples_and_missing(tmp_path):
    prefix, geno, status, missing = make_case(tmp_path)
    keep = np.array([s != "missing" for s in status])
    for missing_value in (0, 1, 2, 3):
        g, p = epik2.read_plink(prefix, missing_genotype=missing_value)
        want = geno.copy()
        want[missing] = missing_value
        assert g.shape == (keep.sum(), geno.shape[1])
        assert np.array_equal(g, want[keep])
        assert np.array_equal(p, np.array([s == "case" for s in status[keep]], dtype=np.uint8))


def test_plink_reader_errors(tmp_path):
    prefix, geno, status, _ = make_case(tmp_path, n=20, m=5)
    with pytest.raises(epik2.Epik2Error) as e:
        epik2.read_plink(str(tmp_path / "absent"))
    assert e.value.status == epik2.E_NOT_FOUND
    data = open(prefix + ".bed", "rb").read()
    open(prefix + ".bed", "wb").write(data[:-3])  # truncated
    with pytest.raises(epik2.Epik2Error) as e:
        epik2.read_plink(prefix)
    assert e.value.status == epik2.E_INVALID
    open(prefix + ".bed", "wb").write(bytes([0x6C, 0x1B, 0x00]) + data[3:])  # sample-major mode
    with pytest.raises(epik2.Epik2Error) as e:
        epik2.read_plink(prefix)
    assert e.value.status == epik2.E_INVALID


def test_perm_pvalue():
    assert epik2.perm_pvalue(10.0, []) == 1.0
    assert epik2.perm_pvalue(10.0, [11.0, 12.0, 13.0]) == 0.25
    assert epik2.perm_pvalue(10.0, [9.0, 10.0, 13.0]) == 0.75  # ties count as at least as good
    rng = np.random.default_rng(1)
    reps = rng.normal(1000, 5, 999).astype(np.float32)
    obs = np.float32(990.0)
    assert epik2.perm_pvalue(obs, reps) == pytest.approx((1 + np.sum(reps <= obs)) / 1000)


@pytest.mark.gpu
def test_cli_reads_plink_fileset(tmp_path):
    import oracle as O
    g0, p0 = O.gen_hwe(55, 600, 40, 300, planted=[(4, 11, 30)], effects=[0.85])
    status = np.where(p0 == 1, "case", "control")
    prefix = str(tmp_path / "planted")
    write_plink(prefix, g0, status)
    out = subprocess.run([epik2.CLI_PATH, "--plink", prefix], capture_output=True, text=True, check=True).stdout
    sol = [l for l in out.splitlines() if l.startswith("Solution:")][0].split()[1:]
    ref = O.scan(g0, p0)
    assert tuple(int(x) for x in sol) == ref["ijk"] == (4, 11, 30)
