"""Shared fixtures.  Tests marked `gpu` need a B200 and the in-tree
libpsycles_cuda.so; everything else runs on CPU (the oracle, host tables,
the C ABI surface, host logic)."""

import json
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_vectors.json"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and libpsycles_cuda.so")


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    return oracle.load()


@pytest.fixture(scope="session")
def backend():
    from psycles_b200.backend import CudaPathTracerBackend
    return CudaPathTracerBackend(0)
