import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from addingdoublingrt_b200 import _abi  # noqa: E402
from addingdoublingrt_b200.workloads import Batch  # noqa: E402

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(path):
    """(name, Batch, reference outputs) from one tests/golden fixture."""
    z = np.load(path)
    fields = {}
    for key in z.files:
        if key.startswith("desc_"):
            v = z[key]
            fields[key[5:]] = float(v) if v.dtype.kind == "f" else int(v)
    desc = _abi.make_desc(**fields)
    b = Batch(desc)
    for key in z.files:
        if key.startswith("in_"):
            b.set(key[3:], z[key])
    out = {key[4:]: z[key] for key in z.files if key.startswith("out_")}
    return os.path.basename(path)[:-4], b, out


def golden_paths():
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


@pytest.fixture(scope="session")
def golden():
    return [load_golden(p) for p in golden_paths()]


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
