import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "uni-dock_b200"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def pytest_sessionstart(session):
    """Build the engine library, the CLI and the oracle libraries when a fresh
    checkout lacks them (nvcc cross-compiles for sm_100a without a GPU)."""
    import subprocess
    need = [ROOT / "uni-dock_b200" / "lib" / "libunidock_b200.so", ROOT / "uni-dock_b200" / "bin" / "unidock",
            ROOT / "oracle" / "_ref" / "liboracle32.so", ROOT / "oracle" / "_ref" / "liboracle64.so"]
    if all(x.exists() for x in need):
        return
    for d in ("uni-dock_b200", "oracle"):
        subprocess.run(["make", "-C", str(ROOT / d)], check=True, stdout=subprocess.DEVNULL)


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
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("ud")


@pytest.fixture(scope="session")
def receptor():
    from unidock_tools import synth
    return synth.make_receptor(3000, seed=1)


BOX_CENTER = np.zeros(3, np.float32)
BOX_SIZE = np.full(3, 22.5, np.float32)
