import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")
FULL_CASES = ("city36", "city24x40_s05", "dem_bush", "bush24")
SVF_CASES = FULL_CASES + ("strip1x16", "lowveg16")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def golden_location(d):
    return {"latitude": float(d["latitude"]), "longitude": float(d["longitude"]),
            "altitude": float(d["site_altitude"])}


@pytest.fixture(scope="session", autouse=True)
def native_library():
    """The host table builders (sw100_march_tables) and every kernel live in
    the in-tree library: build it once per session when it is missing or
    older than its sources."""
    from solweig_project_b200 import build
    build.build()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    from solweig_project_b200 import build
    build.build()
    return torch.device("cuda")
