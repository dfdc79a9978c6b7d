import ctypes
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "cross-dpc-episdet_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; runs the CUDA path")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def cuda_device_count():
    for name in ("libcudart.so", "libcudart.so.12"):
        try:
            rt = ctypes.CDLL(name)
            break
        except OSError:
            rt = None
    if rt is None:
        try:
            import torch  # the venv's torch ships a cudart
            return torch.cuda.device_count()
        except Exception:
            return 0
    n = ctypes.c_int(0)
    if rt.cudaGetDeviceCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


HAS_GPU = None


def has_gpu():
    global HAS_GPU
    if HAS_GPU is None:
        HAS_GPU = cuda_device_count() > 0
    return HAS_GPU


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


ENGINES = {1: "int", 2: "tc", 3: "fp4"}


@pytest.fixture(scope="session", params=[(1, 0, 0, 0), (2, 0, 0, 0), (3, 8, 32, 1), (3, 16, 64, 1), (3, 8, 64, 1),
                                        (3, 16, 32, 1), (3, 4, 64, 2), (3, 8, 64, 2)],
                ids=["int", "tc", "fp4", "fp4pair", "fp4pair8", "fp4w16", "fp4ov4", "fp4ov8"])
def ctx(request):
    """A device context per search engine: integer pipe; int8 tensor cores; FP4 tensor cores
    on single CTAs (32 SNPs j per tile) at 8 and 16 words per stage; FP4 on CTA pairs (64 SNPs
    j per tile) at 16 and 8 words per stage; the overlapped FP4 CTA-pair kernel at 4 and 8
    words per stage.  Every test that takes `ctx` runs on all eight.  A configuration a
    dataset cannot take (the overlapped kernel for classes above 65535 samples) is refused with
    EPIK2_E_TOO_LARGE."""
    import epik2
    c = epik2.Context(0, engine=request.param[0], stage_words=request.param[1], pair_tile=request.param[2],
                      overlap=request.param[3])
    c.config = request.param
    yield c
    c.close()


def load_tap(name):
    z = np.load(os.path.join(GOLDEN, f"tap_{name}.npz"))
    return {k: z[k] for k in z.files}


TAP_CASES = ["refgen_256x20", "hwe_300x24_37cases", "hwe_40x12_5cases", "hwe_64x3", "hwe_1000x30_planted",
             "odd_values_100x10"]


def ref_kat():
    return json.load(open(os.path.join(GOLDEN, "ref_kat.json")))


def ref_best():
    return json.load(open(os.path.join(GOLDEN, "ref_best.json")))


def addlog_bits():
    return np.load(os.path.join(GOLDEN, "addlog.npz"))["bits"]


def f32_bits(x):
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])
