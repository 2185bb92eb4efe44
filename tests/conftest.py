"""pytest configuration: the ``gpu`` marker, repo path, shared fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle, build

    build()
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle.pyoracle import RefLib, build

    build()
    if not RefLib.available():
        pytest.skip("oracle/_ref not built: reference sources absent")
    return RefLib()


@pytest.fixture(scope="session")
def lib():
    from blackhole_b200 import _abi
    from blackhole_b200.build import build_library

    if not _abi.LIB_PATH.exists():
        build_library(quiet=True)
    return _abi.load_library()


@pytest.fixture(scope="session")
def cuda(lib):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch.device("cuda", 0)


def load_golden(name: str):
    import numpy as np

    path = GOLDEN / name
    if not path.exists():
        pytest.fail(f"golden fixture {path} missing: run tests/golden/make_golden.py")
    return dict(np.load(path, allow_pickle=False))
