import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "egg-sync_b200"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests" / "golden"))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    O = Oracle()
    O.set_box_mode(False)
    return O


@pytest.fixture(scope="session")
def eggsync_lib():
    """The built libeggsync.so (built here when missing)."""
    from eggsync import _lib, build

    if not _lib.LIB_PATH.exists():
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def gpu():
    import torch

    assert torch.cuda.is_available()
    torch.cuda.init()
    return torch.device("cuda:0")


def load_golden(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip("golden fixture %s not present" % name)
    return dict(np.load(p, allow_pickle=False))
