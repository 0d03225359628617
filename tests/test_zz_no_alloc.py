"""dmk_field_mean_noalloc: the volume average for callers that may not allocate device
memory when they need it (their field already lives in device memory they own, e.g.
in an arena their framework manages).  It must give the same <P> as the context-based
constitutive response, call after call, without allocating.  Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from damask_b200 import _lib, synthetic, workloads
from damask_b200.grid import SpectralBasic

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _mean_noalloc(lib, planes_ptr, n):
    out = np.zeros(9)
    rc = lib.dmk_field_mean_noalloc(C.c_void_p(planes_ptr), n, out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == 0, lib.dmk_last_error()
    return out


def test_noalloc_mean_matches_constitutive_response(gpu):
    import torch
    lib = _lib.load()
    rve = synthetic.voronoi_rve((8, 8, 6), workloads.SIZE_1MM, 5, 0)
    g = SpectralBasic(rve.cells, rve.size, rve.material, rve.quaternions, workloads.fcc_al(),
                      workloads.numerics_default())
    rng = np.random.default_rng(3)
    results = []
    for strain in (3e-3, 5e-3):                  # two calls in a row on different fields
        F = np.tile((np.eye(3) + np.diag([strain, -0.4 * strain, -0.4 * strain])).reshape(-1, order='F'), (g.N, 1))
        F += 1e-4 * rng.normal(size=F.shape)
        P, P_av, _, _, st = g.constitutive_response(F, 1.0)
        assert st == 0
        planes = torch.tensor(np.ascontiguousarray(P.T), dtype=torch.float64, device='cuda')   # [9][N] on the device
        torch.cuda.synchronize()
        mean = _mean_noalloc(lib, planes.data_ptr(), g.N)
        assert np.abs(mean - P_av).max() / np.abs(P_av).max() < TOL
        results.append(mean)
    assert not np.allclose(results[0], results[1])   # the second call did not return the first result
    g.close()


def test_noalloc_many_blocks_and_tail_allocates_nothing(gpu):
    """A 33^3 field spans 36 partial-sum blocks of 1024 voxels, the last one partly filled:
    the final sum over several block slots and the tail are exercised.  Repeated calls leave
    the device's free memory unchanged (no allocation), and give the same mean each time."""
    import torch
    lib = _lib.load()
    n = 33 ** 3
    rng = np.random.default_rng(5)
    host = rng.normal(size=(9, n)) * 1e8 + np.arange(9)[:, None] * 1e7
    planes = torch.tensor(host, dtype=torch.float64, device='cuda')
    torch.cuda.synchronize()
    first = _mean_noalloc(lib, planes.data_ptr(), n)         # set-up happens here, before measuring
    free0 = torch.cuda.mem_get_info()[0]
    means = [_mean_noalloc(lib, planes.data_ptr(), n) for _ in range(20)]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ref = host.mean(axis=1)
    assert np.abs(first - ref).max() / np.abs(ref).max() < TOL
    assert all(np.array_equal(m, first) for m in means)      # fixed summation order


def test_noalloc_rejects_oversized_grid(gpu):
    lib = _lib.load()
    out = np.zeros(9)
    rc = lib.dmk_field_mean_noalloc(C.c_void_p(1), 256 ** 3 + 1, out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == -4                              # DMK_ERR_ARG, nothing launched
    assert b'16777216' in lib.dmk_last_error()
