"""Shared fixtures: grids, seeded random fields in the reference layout, and
the oracle / GPU context factories.

``-m gpu`` tests need a CUDA device and the in-tree ``libfugu_gpu.so``; they
compare the CUDA path with the CPU oracle (``oracle/``) on identical inputs.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from coupled_codefort_2d_b200.layout import Grid  # noqa: E402
from coupled_codefort_2d_b200.params import Params  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libfugu_gpu.so")
    config.addinivalue_line("markers", "slow: long CPU oracle run")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


# grids covering walls / periodic combinations and odd sizes
GRIDS = {
    "walls_13x9": Grid(13, 9, 1.0, 0.7),
    "walls_32x24": Grid(32, 24),
    "px_16x12": Grid(16, 12, periodic_x=True),
    "py_12x16": Grid(12, 16, periodic_y=True),
    "pxy_10x14": Grid(10, 14, periodic_x=True, periodic_y=True),
}


def rfield(rng, g, kind, lo=-1.0, hi=1.0):
    return np.asfortranarray(rng.uniform(lo, hi, size=g.shape(kind)))


def colour(rng, g):
    """smooth-ish colour field in [0,1] with a few out-of-range values"""
    c = rng.uniform(-0.05, 1.05, size=g.shape("cell"))
    return np.asfortranarray(c)


def two_phase_params(**kw):
    base = dict(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98)
    base.update(kw)
    return Params(**base)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from coupled_codefort_2d_b200 import build

    build.build()
    from coupled_codefort_2d_b200 import _lib

    _lib.lib()
    return _lib
