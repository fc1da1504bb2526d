import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "ref_gll_gmtk.npz")


@pytest.fixture(scope="session")
def ctx():
    from geoflow_b200 import Context
    # problems keep a reference to their context; it is released after them
    return Context(0)


@pytest.fixture(scope="session")
def refpath():
    """Inputs and outputs of the reference's own grid, GGFX, GHelmholtz,
    GAdvect, GCG and GBurgers/GExRKStepper code
    (tests/golden/make_path_golden.py)."""
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "ref_path.npz")
