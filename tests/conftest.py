"""Test configuration: import paths, the gpu marker and shared seeded grids."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "sal-fort_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def rel_l2(ax, ay, bx, by):
    """||[a_x; a_y] - [b_x; b_y]||_2 / ||[b_x; b_y]||_2."""
    num = np.sqrt(np.sum((np.asarray(ax) - bx) ** 2) + np.sum((np.asarray(ay) - by) ** 2))
    den = np.sqrt(np.sum(np.asarray(bx) ** 2) + np.sum(np.asarray(by) ** 2))
    return float(num / den)


_GRIDS = {}


def grid_and_ssh(name, nfields=1, seed=11):
    """Seeded synthetic grid + SSH (F, N), built on the CPU and cached."""
    from salgpu import synth
    key = (name, nfields, seed)
    if key not in _GRIDS:
        g = synth.config_grid(name, device="cpu")
        h = synth.config_ssh(name, g, nfields=nfields, seed=seed, device="cpu")
        _GRIDS[key] = (g, h)
    return _GRIDS[key]


@pytest.fixture(scope="session")
def small_grid():
    return grid_and_ssh("small_3000")


@pytest.fixture(scope="session")
def cfg0_grid():
    return grid_and_ssh("cfg0")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
