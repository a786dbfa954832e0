"""Shared pytest setup: the `gpu` marker and the repository root on sys.path."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(autouse=True, scope="session")
def _tune_cache_in_tmp(tmp_path_factory):
    """Autotuner choices made by the tests go to a file of the test session,
    not to the user's cache."""
    import os
    os.environ["CUDATREE_B200_TUNE_CACHE"] = str(tmp_path_factory.mktemp("tune") / "autotune.json")
    yield


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from cudatree_b200 import _lib
    _lib.load()  # raises when the library is missing: no fallback
    return torch.device("cuda", 0)
