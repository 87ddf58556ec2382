import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU case")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return {name: np.load(GOLDEN / f"{name}.npz") for name in ("manufactured", "checks", "cube")}


@pytest.fixture(scope="session")
def cube_system():
    from hsc_reimpl_b200.systems import make_cube_system
    return make_cube_system(seed=0)


@pytest.fixture(scope="session")
def vehicle_system():
    from hsc_reimpl_b200.systems import make_vehicle_system
    return make_vehicle_system(seed=0)
