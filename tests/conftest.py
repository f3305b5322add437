import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests proper")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


@pytest.fixture(scope="session")
def golden_edge():
    return dict(np.load(os.path.join(GOLDEN, "edge_4x4x4.npz")))


@pytest.fixture(scope="session")
def golden_small_1ppc():
    return dict(np.load(os.path.join(GOLDEN, "gem_small_1ppc.npz")))


def edge_workload(d):
    """The GemWorkload the edge fixture was made with (grid row of the npz)."""
    from sputnipic_b200 import workload as W
    g = d["grid"]
    return W.GemWorkload(name="edge-4x4x4", nxc=int(g[0]), nyc=int(g[1]), nzc=int(g[2]),
                         Lx=float(g[3]), Ly=float(g[4]), Lz=float(g[5]), dt=float(g[6]),
                         c=float(g[7]), niter=int(g[8]), n_sub_cycles=int(g[9]),
                         periodic=tuple(bool(int(v)) for v in g[10:13]))


@pytest.fixture(scope="session")
def cuda():
    """Skip unless a CUDA device is present; returns torch."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
