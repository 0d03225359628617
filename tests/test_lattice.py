"""Lattice constants of the product (host code of libdamask_b200.so) and of the oracle,
pinned against the reference's own Python (golden.npz, made by tests/golden/make_golden.py)."""
import ctypes as C

import numpy as np
import pytest

from damask_b200 import _lib, workloads
from damask_b200.config import Phase

from conftest import rel


def phase(lattice, N_sl, h=None, nonschmid=None):
    n = len(N_sl)
    d = {'lattice': lattice,
         'mechanical': {'elastic': {'type': 'Hooke', 'C_11': 100e9, 'C_12': 60e9, 'C_44': 30e9},
                        'plastic': {'type': 'phenopowerlaw', 'N_sl': N_sl, 'a_sl': [2.0] * n,
                                    'dot_gamma_0_sl': [1e-3] * n, 'h_0_sl-sl': [1e8] * n,
                                    'h_sl-sl': h or list(range(1, 29)), 'n_sl': [20] * n,
                                    'xi_0_sl': [1e8] * n, 'xi_inf_sl': [2e8] * n}}}
    if nonschmid:
        d['mechanical']['plastic']['a_non-Schmid'] = [nonschmid]
    return Phase.from_dict(d)


def product_schmid(ph, sense=1):
    lib = _lib.load()
    ps = ph.to_struct()
    out = np.zeros((ph.n_slip, 9))
    n = lib.dmk_phase_schmid(C.byref(ps), sense, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert n == ph.n_slip
    return out.reshape(n, 3, 3).transpose(0, 2, 1)      # column-major -> [s, i, j]


def product_interaction(ph):
    lib = _lib.load()
    ps = ph.to_struct()
    out = np.zeros((ph.n_slip, ph.n_slip))
    assert lib.dmk_phase_interaction(C.byref(ps), out.ctypes.data_as(C.POINTER(C.c_double))) == ph.n_slip
    return out


@pytest.mark.parametrize('lattice,N_sl,key', [('cF', [12, 6], 'schmid_cF'), ('cI', [12, 12, 24], 'schmid_cI')])
def test_schmid_matches_reference(golden, oracle_lib, lattice, N_sl, key):
    ph = phase(lattice, N_sl)
    ref = golden[key]
    assert rel(product_schmid(ph), ref) < 1e-15
    assert rel(oracle_lib.schmid(ph), ref) < 1e-15
    # the opposite sense flips the slip direction
    assert rel(product_schmid(ph, -1), -ref) < 1e-15


def test_schmid_properties():
    for lattice, N_sl in (('cF', [12, 6]), ('cI', [12, 12, 24])):
        P = product_schmid(phase(lattice, N_sl))
        assert np.abs(np.trace(P, axis1=1, axis2=2)).max() < 1e-15
        assert np.allclose(np.linalg.norm(P, axis=(1, 2)), 1.0, atol=1e-15)


def test_nonschmid_product_vs_oracle(oracle_lib):
    ph = phase('cI', [12], h=[1, 1.4, 1, 1.4, 1.4, 1.4, 1.4], nonschmid=[0.1] * 6)
    for sense in (1, -1):
        assert rel(product_schmid(ph, sense), oracle_lib.schmid(ph, sense)) < 1e-15
    P = product_schmid(phase('cI', [12], h=[1, 1.4, 1, 1.4, 1.4, 1.4, 1.4]))
    Pns = product_schmid(ph)
    assert np.abs(Pns - P).max() > 1e-3          # the non-Schmid terms are active


@pytest.mark.parametrize('ph', [workloads.fcc_al(), workloads.bcc_24(), phase('cF', [12, 6]),
                                phase('cI', [12, 12, 24]), phase('cF', [6]), phase('cI', [12, 12, 12])])
def test_interaction_product_vs_oracle(oracle_lib, ph):
    h = product_interaction(ph)
    assert np.array_equal(h, oracle_lib.interaction(ph))
    assert np.all(np.diag(h) == ph.h_sl_sl[0])   # type 1 = self interaction on the diagonal


def test_interaction_fcc_values():
    # examples/grid/material.yaml: h_sl-sl [1, 1, 1.4, 1.4, 1.4, 1.4, 1.4] over 12 {111}<110> systems:
    # self and coplanar = 1, all other types 1.4
    h = product_interaction(workloads.fcc_al())
    assert h.shape == (12, 12)
    coplanar = np.zeros((12, 12), bool)
    for g in range(4):
        coplanar[3 * g:3 * g + 3, 3 * g:3 * g + 3] = True
    assert np.all(h[coplanar] == 1.0) and np.all(h[~coplanar] == 1.4)


def test_interaction_too_few_values_rejected():
    ph = phase('cI', [12, 12], h=[1, 1.4, 1, 1.4, 1.4, 1.4])   # types up to 24 are needed
    ps = ph.to_struct()
    out = np.zeros((24, 24))
    lib = _lib.load()
    assert lib.dmk_phase_interaction(C.byref(ps), out.ctypes.data_as(C.POINTER(C.c_double))) < 0
    assert b'h_sl-sl' in lib.dmk_last_error()
