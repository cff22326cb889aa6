import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # Build the library and the checkers if they are missing (a fresh checkout).
    if not (ROOT / "cwbvh_b200" / "librq.so").exists():
        subprocess.run([sys.executable, str(ROOT / "cwbvh_b200" / "build.py")], check=True)
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True)


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def rq():
    import cwbvh_b200
    return cwbvh_b200


@pytest.fixture(scope="session")
def po():
    from oracle import pyoracle
    return pyoracle
