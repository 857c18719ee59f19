import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import __graft_entry__ as graft_entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def pkg():
    return graft_entry.load_package()


@pytest.fixture(scope="session")
def oracle(pkg):
    return graft_entry.load_oracle().Oracle(pkg.abi)


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def device_api(pkg):
    """The CUDA library through its C ABI; built on demand (nvcc is part of
    the image on every machine this suite runs on)."""
    import importlib

    importlib.import_module("lsmps3d_b200.build").build_all()
    api = importlib.import_module("lsmps3d_b200.api")
    return api
