"""Shared test setup: the `gpu` marker, import paths and fixtures.

`-m "not gpu"` runs on any machine (oracle against the golden fixtures, host logic, the
C-ABI library's exports). `-m gpu` runs the CUDA device against the oracle and needs a GPU.
"""
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG = ROOT / "oidn-protoray_b200"
GOLDEN = ROOT / "tests" / "golden"
for p in (PKG, ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    register_sunsky_fixtures()


def register_sunsky_fixtures():
    """The reference's sun-sky products for the sun-sky parameters the tests use (fixtures made
    by golden/make_golden.py from the reference's SunSkyLight), handed to the scene generators."""
    import prt_scenes

    for path in sorted(GOLDEN.glob("sunsky_*.npz")):
        z = np.load(path)
        prt_scenes.register_sunsky_products(z["params"], z["sun_color"], float(z["sun_angle"]), z["sky"])


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(GOLDEN / name)

    return load


@pytest.fixture(scope="session")
def device():
    import prt_cuda

    dev = prt_cuda.DeviceCuda(0)
    yield dev
    dev.close()


def rel_mse(x, ref):
    """Per-pixel relative MSE, mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2)."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))
