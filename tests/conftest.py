import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


@pytest.fixture(scope="session")
def port():
    from oracle.loader import PortOracle
    return PortOracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.loader import ReferenceOracle, reference_available
    if not reference_available():
        pytest.skip("reference oracle library not built on this host")
    return ReferenceOracle()


@pytest.fixture(scope="session")
def lib():
    import photorealisticrender4610_b200 as prr
    return prr.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
