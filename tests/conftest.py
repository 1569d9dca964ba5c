"""Shared fixtures: import paths, the `gpu` marker, and in-tree builds of the library and oracle."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from mrsim_acq_b200 import build as product_build
    from oracle import oracle as oracle_mod
    if not product_build.LIB.exists():
        product_build.build()
    if not oracle_mod.LIB.exists():
        oracle_mod.build()
    yield


@pytest.fixture(scope="session")
def gpu_ctx():
    from mrsim_acq_b200 import api
    return api.default_context(0)
