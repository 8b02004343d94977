import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the engine on the device)")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return lib


@pytest.fixture(scope="session")
def oracle():
    from tests._oracle import Oracle
    return Oracle(_ensure_oracle())


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "perft_golden.json")) as f:
        return json.load(f)["positions"]


@pytest.fixture(scope="session")
def engine():
    """The GPU engine, initialised once per session with an 8 GiB arena."""
    import perft_gpu_b200 as pg
    pg.init(device=0, arena_bytes=8 << 30)
    yield pg
    pg.shutdown()
