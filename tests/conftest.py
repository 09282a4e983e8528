import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: builds a full-size basis")


@pytest.fixture(scope="session")
def basis_cache(tmp_path_factory):
    """Directory for bases built during the session (reuses the repo cache if present)."""
    repo_cache = os.path.join(ROOT, ".basis_cache")
    if os.path.isdir(repo_cache) and os.access(repo_cache, os.W_OK):
        return repo_cache
    return str(tmp_path_factory.mktemp("bases"))


def _device():
    try:
        import torch

        return "cuda" if torch.cuda.is_available() else "cpu"
    except Exception:
        return "cpu"


@pytest.fixture(scope="session")
def make_basis(basis_cache):
    from parallelspectralfluids3d_b200.fixture import cached_basis

    def make(domain, n_modes):
        return cached_basis(domain, n_modes, cache_dir=basis_cache, device=_device())

    return make


@pytest.fixture(scope="session")
def c1_basis(make_basis):
    """16^3 all-wall box, N = 64 (the single-instance FP64/FP32 parity workload)."""
    from parallelspectralfluids3d_b200.domain import box_domain

    return make_basis(box_domain(16), 64)


@pytest.fixture(scope="session")
def small_bases(make_basis):
    """Small domains covering obstacles, non-cubic grids and odd mode counts."""
    from parallelspectralfluids3d_b200.domain import box_domain, sphere_obstacle_domain

    return {
        "box6": make_basis(box_domain(6), 12),
        "sphere10": make_basis(sphere_obstacle_domain(10, 2.5), 16),
        "box576": make_basis(box_domain((5, 7, 6)), 13),
        "sphere12x10x9": make_basis(sphere_obstacle_domain((12, 10, 9), 3.0), 37),
    }


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def medium_basis(make_basis):
    """12^3 box with N = 160: two 128-row tiles per mode and three 64-wide K chunks in the GEMMs."""
    from parallelspectralfluids3d_b200.domain import box_domain

    return make_basis(box_domain(12), 160)
