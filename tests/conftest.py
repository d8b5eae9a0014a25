"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (B200); the rest
run on the CPU (oracle, host setup, C-ABI loading)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    from fmm3dbie_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def sphere4(built):
    """Sphere: icosahedron x2 refinements, order 4, npts 4800."""
    from fmm3dbie_b200 import surface as S
    return S.icosa_sphere(2, 4)


@pytest.fixture(scope="session")
def sphere_lap_setup(sphere4):
    from fmm3dbie_b200 import surface as S
    return S.setup(sphere4, 0, 1e-6, (1.0, 1.0))


@pytest.fixture(scope="session")
def ellipsoid_small(built):
    """Reduced ellipsoid (1,2,3): 80 order-6 patches, npts 2240."""
    from fmm3dbie_b200 import surface as S
    return S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0))


@pytest.fixture(scope="session")
def ellipsoid_helm_setup(ellipsoid_small):
    from fmm3dbie_b200 import surface as S
    zk = 2.0
    return S.setup(ellipsoid_small, 1, 1e-7, (zk, -1j * zk, 1.0))


def wnorm(w, x):
    return float(np.sqrt(np.sum(w * np.abs(x) ** 2)))
