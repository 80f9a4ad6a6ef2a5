import os
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PKG = REPO / "flock-challenge-multi_b200"
for p in (str(PKG), str(REPO / "tests"), str(REPO / "tests" / "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _build_oracle():
    lib = REPO / "oracle/_build/libflockref.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(REPO / "oracle")], check=True, capture_output=True)
    return lib


@pytest.fixture(scope="session")
def oracle():
    _build_oracle()
    import oracle_lib
    return oracle_lib.Oracle()


@pytest.fixture(scope="session")
def gpu_ctx():
    import flockgpu
    ctx = flockgpu.Context(int(os.environ.get("FLOCK_DEVICE", "0")))
    yield ctx
    ctx.close()
