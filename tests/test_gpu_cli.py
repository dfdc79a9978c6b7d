"""The process-level drop-in: `epik2_v4` with the reference's own arguments prints the
reference's four lines (GPU/v4.cpp:251, 610-612) with its known answers, and `--file` reads
a raw matrix (GPU)."""
import os
import subprocess

import numpy as np
import pytest

import epik2
import oracle as O
from conftest import ref_kat

pytestmark = pytest.mark.gpu


def run_cli(*args):
    if not os.path.exists(epik2.CLI_PATH):
        pytest.fail("CLI not built: " + epik2.CLI_PATH)
    r = subprocess.run([epik2.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout.splitlines()


def parse(lines):
    assert len(lines) == 4
    assert lines[0].startswith("Selected device: ")
    assert lines[1].startswith("Time: ") and float(lines[1].split()[1]) >= 0.0
    assert lines[2].startswith("Score: ") and lines[3].startswith("Solution: ")
    return lines[2].split(" ", 1)[1], tuple(int(x) for x in lines[3].split()[1:])


@pytest.mark.parametrize("key", ["2048x128", "2000x100", "2048x512"])
@pytest.mark.parametrize("form", ["v4", "v1-v3"])
def test_reference_arguments_print_reference_answers(key, form):
    k = ref_kat()[key]
    args = [k["n_samples"], k["n_snps"]] + ([32] if form == "v4" else [])
    score, ijk = parse(run_cli(*args))
    assert list(ijk) == k["ijk"]
    # std::cout of a float: default stream precision, 6 significant digits
    assert score == "%g" % np.float32(k["score"])


def test_file_input_matches_oracle(tmp_path):
    g, p = O.gen_hwe(71, 1500, 60, 700)
    path = tmp_path / "geno.bin"
    path.write_bytes(np.ascontiguousarray(g).tobytes() + np.ascontiguousarray(p).tobytes())
    score, ijk = parse(run_cli("--file", path, g.shape[0], g.shape[1]))
    r = O.scan(g, p)
    assert ijk == r["ijk"]
    assert score == "%g" % np.float32(r["score"])

