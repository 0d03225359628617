"""Generate ``golden_17grains_bcc.npz`` from the reference's regression resources.

Run here (where the reference tree is mounted), not on the test machines:

    python tests/golden/make_golden_17grains.py <path of the reference's source tree>

Source: ``tests/integration/resources/plastic_detect_changes/`` of the reference, the
inputs and stored result of ``tests/integration/test_plastic_detect_changes.py`` for
the ``phenopowerlawbcc`` model: a 10x16x12 grid of 17 grains (``17grains.vti``), the
bcc phenopowerlaw phase with non-Schmid terms (``material.yaml``), tension along x with
mixed boundary conditions over 150 increments (``tensionX.yaml``), ``N_iter_min: 4``
(``numerics.yaml``), and the reference's result file
``17grains_tensionX_phenopowerlawbcc.hdf5`` (read with ``dadf5.py``).  The reference test
compares every dataset at rtol 2.5 %, atol = max(1e-5 max|x|, 1e-6).

Fixture contents: ``material`` (0-based material index per cell, x fastest), ``cells``,
``size``, ``quaternions`` (one per material), the phase, load and numerics dictionaries
as JSON strings, and ``xi_sl_<inc>`` / ``gamma_sl_<inc>`` for the stored increments
0, 75 and 150 (shape (cells, N_sl)), ``u_p_<inc>`` / ``u_n_<inc>`` (displacements of cell
centres and nodes) for 75 and 150, and ``layout_json``: the result file's group tree for the
written phase (groups, datasets with shape, dtype and the attributes other than
creator/created, the t/s of each increment, the root and geometry attributes).  Also ``vti_known``: the base64 known answers of
the reference's VTI decoder tests (``tests/unit_cpp/test_VTI.cpp``) with their decoded
bytes, for the reader in ``damask_b200/vti.py``.
"""
import json
import re
import sys
from pathlib import Path

import numpy as np
import yaml

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

from damask_b200.h5read import DADF5         # noqa: E402
from damask_b200 import vti                  # noqa: E402


def vti_known_answers(root: Path) -> dict:
    """The base64 strings and expected byte sequences of test_VTI.cpp."""
    src = (root / 'tests' / 'unit_cpp' / 'test_VTI.cpp').read_text()
    consts = {}
    for name in ('B64_UC32', 'B64_UC64', 'B64_COMP32', 'B64_COMP64'):
        m = re.search(name + r'\s*=\s*((?:"[^"]*"\s*)+);', src)
        consts[name] = ''.join(re.findall(r'"([^"]*)"', m.group(1)))
    exp = {}
    for name in ('EXPECTED_UNCOMPRESSED', 'EXPECTED_COMPRESSED'):
        m = re.search(name + r'\s*=\s*\{([^}]*)\}', src)
        exp[name] = [int(x) for x in m.group(1).split(',')]
    return {'uc32': (consts['B64_UC32'], 4, False, exp['EXPECTED_UNCOMPRESSED']),
            'uc64': (consts['B64_UC64'], 8, False, exp['EXPECTED_UNCOMPRESSED']),
            'comp32': (consts['B64_COMP32'], 4, True, exp['EXPECTED_COMPRESSED']),
            'comp64': (consts['B64_COMP64'], 8, True, exp['EXPECTED_COMPRESSED'])}


def _plain(v):
    return v.tolist() if isinstance(v, np.ndarray) else (v.item() if isinstance(v, np.generic) else v)


def layout(f: DADF5, phase: str) -> dict:
    """Group tree of the reference's result file restricted to one phase."""
    def attrs(path):
        return {k: _plain(v) for k, v in f.attrs(path).items() if k not in ('creator', 'created', 'call')}

    def walk(path):
        out = {}
        for k in f.keys(path):
            p = f'{path}/{k}'.strip('/')
            if p.count('/') == 2 and p.split('/')[1] == 'phase' and k != phase:
                continue                                          # other phases of the file
            try:
                out[k] = {'groups': walk(p), 'attrs': attrs(p)}
            except KeyError:
                d = f.read(p)
                out[k] = {'shape': list(d.shape), 'dtype': str(d.dtype) if not d.dtype.names else list(d.dtype.names),
                          'attrs': attrs(p)}
        return out

    return {'root_attrs': sorted(f.attrs('')), 'tree': walk('')}


def main(root: str) -> None:
    root = Path(root)
    res = root / 'tests' / 'integration' / 'resources' / 'plastic_detect_changes'
    geom = vti.load(res / '17grains.vti')
    mat = yaml.safe_load((res / 'material.yaml').read_text())
    quats = np.array([m['constituents'][0]['O'] for m in mat['material']], dtype=np.float64)
    phase = mat['phase']['phenopowerlawbcc']
    load = yaml.safe_load((res / 'tensionX.yaml').read_text())
    numerics = yaml.safe_load((res / 'numerics.yaml').read_text())
    out = {'material': geom.material, 'cells': np.array(geom.cells), 'size': np.array(geom.size),
           'quaternions': quats, 'phase_json': json.dumps(phase), 'load_json': json.dumps(load),
           'numerics_json': json.dumps(numerics),
           'vti_known_json': json.dumps(vti_known_answers(root))}
    f = DADF5(res / '17grains_tensionX_phenopowerlawbcc.hdf5')
    for inc in (0, 75, 150):
        for name in ('xi_sl', 'gamma_sl'):
            out[f'{name}_{inc}'] = f.read(f'increment_{inc}/phase/phenopowerlawbcc/mechanical/{name}')
    for inc in (75, 150):
        for name in ('u_p', 'u_n'):
            out[f'{name}_{inc}'] = f.read(f'increment_{inc}/geometry/{name}')
    out['layout_json'] = json.dumps(layout(f, 'phenopowerlawbcc'))
    np.savez_compressed(HERE / 'golden_17grains_bcc.npz', **out)
    print('wrote', HERE / 'golden_17grains_bcc.npz', sorted(out))


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit(f'usage: python {sys.argv[0]} <path of the reference source tree>')
    main(sys.argv[1])
