import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


# the reflection symmetry of the golden grids (grid = box octant / bitant)
GOLDEN_SYMMETRY = {"bssn_punc_octant": 7, "bssn_fourier_bitant": 4}


def golden_level(g, symmetry=0):
    from baum_b200 import abi
    boxes = [(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in g["boxes"]]
    return abi.Level(boxes, float(g["dx"]), g["boundary"], symmetry=symmetry)


def relerr(a, b, floor=1e-8):
    """Per-variable max |a-b| / max(max|b|, floor)."""
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for v in range(b.shape[0]):
        scale = max(np.abs(b[v]).max(), floor)
        out.append(np.abs(a[v] - b[v]).max() / scale)
    return np.array(out)


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from baum_b200 import abi, build
    build.build()
    abi.lib()
    return torch.device("cuda:0")
