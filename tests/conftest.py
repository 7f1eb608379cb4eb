"""Test configuration.

Markers: `gpu` tests need a CUDA device and run the library's kernels;
everything else runs on a CPU-only machine (oracle, host logic, the C ABI's
validation paths, golden fixtures).
"""

import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs libcuhc kernels")


def _has_gpu():
    try:
        import torch  # noqa: PLC0415
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="needs a CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _pruning_mode():
    """CUHC_TEST_PRUNING=always|never runs every test with that pruning mode
    (results must not change); the mode is reset after each test."""
    mode = os.environ.get("CUHC_TEST_PRUNING")
    if mode:
        from cuhc_b200 import _lib  # noqa: PLC0415
        _lib.set_pruning(mode)
    yield
    if mode:
        from cuhc_b200 import _lib  # noqa: PLC0415
        _lib.set_pruning("auto")
