import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLD = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = ["potential_field_source_surface", "potential_field_current_sheet", "open_field"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs (set POT3D_SLOW=1)")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("POT3D_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle run; set POT3D_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


def load_case(case):
    with open(os.path.join(GOLD, f"{case}.json")) as fh:
        meta = json.load(fh)
    z = np.load(os.path.join(GOLD, f"{case}_br.npz"))
    return meta, z


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    return torch.device("cuda:0")
