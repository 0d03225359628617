import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / 'golden'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


@pytest.fixture(scope='session')
def golden():
    return dict(np.load(GOLDEN / 'golden.npz'))


@pytest.fixture(scope='session')
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope='session')
def gpu():
    if not gpu_available():
        pytest.fail('GPU test collected on a machine without a CUDA device')
    from damask_b200 import build
    build.build()
    return True


def rel(a, b):
    """Field-maximum metric: max|a - b| / max|b| over the whole field."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


# Floor of the per-voxel metric, as a fraction of the field maximum: a voxel whose own values
# are all below 1e-3 of the largest value in the field (an elastic voxel's L_p, a slip system
# that has not slipped) is measured against that level instead of its own near-zero size.
PV_FLOOR = 1.0e-3


def rel_pv(a, b, floor=PV_FLOOR):
    """Per-voxel metric: max over voxels v of max_k|a_vk - b_vk| / max(max_k|b_vk|, floor * max|b|),
    for fields stored voxel-major (N, k).  Every voxel is held to the tolerance in its own terms
    (down to the floor), which the field-maximum metric does not do for low-stress voxels."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    if a.ndim == 1:
        a, b = a[:, None], b[:, None]
    a, b = a.reshape(a.shape[0], -1), b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), floor * max(np.abs(b).max(), 1e-300))
    return float((np.abs(a - b).max(axis=1) / scale).max())


def assert_fields(g, o, names, tol, floor=PV_FLOOR):
    """Fields of two solvers agree within tol under both metrics (field maximum and per voxel)."""
    for name in names:
        a, b = g.get_field(name), o.get_field(name)
        assert rel(a, b) < tol, (name, 'field max', rel(a, b))
        assert rel_pv(a, b, floor) < tol, (name, 'per voxel', rel_pv(a, b, floor))


os.environ.setdefault('OMP_NUM_THREADS', str(min(8, os.cpu_count() or 1)))
