"""Shared test configuration.

* ``@pytest.mark.gpu`` tests need a CUDA device and the in-tree libqnd_b200.so;
  they are skipped (not failed) on machines without a GPU.
* The CPU oracle (oracle/libqnd_oracle.so) is built on demand with gcc.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if any("gpu" in item.keywords for item in items) and not _has_gpu():
        skip = pytest.mark.skip(reason="no CUDA device")
        for item in items:
            if "gpu" in item.keywords:
                item.add_marker(skip)


@pytest.fixture(scope="session")
def qnd_lib():
    """The CUDA engine library; built in-tree if missing (nvcc is part of the image)."""
    from tdse_nd_mpi_b200 import _lib, build

    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    d = os.path.join(ROOT, "tests", "golden")
    return {f[:-4]: dict(np.load(os.path.join(d, f))) for f in os.listdir(d) if f.endswith(".npz")}
