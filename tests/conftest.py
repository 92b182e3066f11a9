import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built libdft_b200.so")
    config.addinivalue_line("markers", "slow: minutes of CPU time")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def port():
    from oracle.bindings import Port
    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.bindings import Ref, ref_available
    if not ref_available():
        pytest.skip("reference library oracle/_ref/libdft_ref.so not built here")
    return Ref()


@pytest.fixture(scope="session")
def engine():
    import dft_b200
    e = dft_b200.Engine(0)
    yield e
    e.close()


def grid_coords(n, b):
    x = np.linspace(b[0], b[1], n[0])
    y = np.linspace(b[2], b[3], n[1])
    z = np.linspace(b[4], b[5], n[2])
    Zc, Yc, Xc = np.meshgrid(z, y, x, indexing="ij")
    return Xc.ravel(), Yc.ravel(), Zc.ravel()


def gaussian_density(n, b, seed, scale=1.0):
    """Two seeded Gaussian spin densities with floored and fully polarised points."""
    rng = np.random.default_rng(seed)
    X, Y, Z = grid_coords(n, b)
    r2 = X ** 2 + Y ** 2 + Z ** 2
    na = scale * (0.8 * np.exp(-0.9 * r2) + 1e-3 * rng.random(r2.size))
    nb = scale * (0.5 * np.exp(-0.6 * (r2 + 0.3 * X)) + 1e-3 * rng.random(r2.size))
    nb[::17] = 0.0
    na[::23] = 0.0
    na[5::41] = 0.0
    nb[5::41] = 0.0
    return na, nb
