"""The Fortran drop-in module (damask_b200/fortran/grid_mech_spectral_b200.f90) binds the C-ABI with
bind(C) derived types.  No Fortran compiler exists on the build or GPU machines, so its types are
checked here against include/damask_b200.h field by field (order, C type, array length), and its
five plugin procedures against the argument lists of the reference's grid_mechanical_spectral_basic
procedures (src/grid/grid_mech_spectral_basic.f90:103,243,284,361,378)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
F90 = (ROOT / 'damask_b200' / 'fortran' / 'grid_mech_spectral_b200.f90').read_text()
HDR = (ROOT / 'include' / 'damask_b200.h').read_text()


def c_fields(name):
    body = re.search(r'typedef struct \{([^{}]*)\}\s*' + name + ';', HDR).group(1)
    body = re.sub(r'/\*.*?\*/', '', body, flags=re.S)
    out = []
    for decl in body.split(';'):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r'(double\*|double|int)\s+(.*)', decl)
        ctype, names = m.group(1), m.group(2)
        for n in names.split(','):
            n = n.strip()
            star = n.startswith('*')
            n = n.lstrip('*')
            dim = re.search(r'\[(\d+)\]', n)
            base = re.sub(r'\[.*', '', n)
            kind = 'ptr' if (ctype == 'double*' or star) else ctype
            out.append((base.lower(), kind, int(dim.group(1)) if dim else 1))
    return out


def f_fields(name):
    body = re.search(r'type, bind\(C\) :: ' + name + r'\n(.*?)end type ' + name, F90, re.S).group(1)
    out = []
    kinds = {'real(C_DOUBLE)': 'double', 'integer(C_INT)': 'int', 'type(C_PTR)': 'ptr'}
    for line in body.splitlines():
        line = line.split('!')[0].strip()
        if not line:
            continue
        t, names = [x.strip() for x in line.split('::')]
        for n in re.split(r',(?![^(]*\))', names):
            n = n.strip()
            dim = re.search(r'\((\d+)\)', n)
            out.append((re.sub(r'\(.*', '', n).lower(), kinds[t], int(dim.group(1)) if dim else 1))
    return out


@pytest.mark.parametrize('name', ['dmk_phase', 'dmk_numerics', 'dmk_bc', 'dmk_solution_state', 'dmk_restart'])
def test_bind_c_types_match_the_header(name):
    assert f_fields(name) == c_fields(name)


def test_plugin_procedures_keep_the_reference_signatures():
    sigs = {
        'init': r'subroutine grid_mechanical_spectral_b200_init\(num_grid_mech\)',
        'solution': r'function grid_mechanical_spectral_b200_solution\(incInfoIn\) result\(solution\)',
        'forward': r'subroutine grid_mechanical_spectral_b200_forward\(cutBack,guess,Delta_t,Delta_t_old,t_remaining,&\s*'
                   r'deformation_BC,stress_BC,rotation_BC\)',
        'updateCoords': r'subroutine grid_mechanical_spectral_b200_updateCoords\(\)',
        'restartWrite': r'subroutine grid_mechanical_spectral_b200_restartWrite\(\)',
    }
    for k, pat in sigs.items():
        assert re.search(pat, F90), k
    assert 'type(tDict), pointer, intent(in) :: num_grid_mech' in F90
    assert 'type(tSolutionState)         :: solution' in F90
    for decl in ('type(tBCmech),   intent(in)', 'type(tRotation), intent(in)', 'logical,         intent(in)'):
        assert decl in F90


def test_every_bound_function_is_exported():
    from damask_b200 import _lib
    bound = set(re.findall(r"bind\(C, name='(dmk_\w+)'\)", F90))
    assert bound and bound <= set(_lib.EXPORTS)
