import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the hand-written sm_100a kernels")


@pytest.fixture(scope="session")
def golden_indexer():
    return np.load(GOLDEN / "indexer_ref.npz")


@pytest.fixture(scope="session")
def golden_math():
    return np.load(GOLDEN / "math_ref.npz")


@pytest.fixture(scope="session")
def golden_flips():
    return np.load(GOLDEN / "flips_ref.npz")


@pytest.fixture(scope="session")
def ref():
    import oracle

    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the compiled reference) is not built here")
    return oracle


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.c_lib()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    return torch.device("cuda:0")
