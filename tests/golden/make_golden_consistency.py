"""Generate ``golden_mech_consistency.npz`` from the reference's cross-solver test inputs.

Run here (where the reference tree is mounted), not on the test machines:

    python tests/golden/make_golden_consistency.py <path of the reference's source tree>

Source: ``tests/integration/resources/grid_mech_consistency/`` of the reference, the inputs
of ``tests/integration/test_grid_mech_consistency.py`` for the plastic case: the 4x4x4 grid of
8 grains ``g_444.vti``, ``material_plast.yaml`` (phenopowerlaw Al, outputs F, F_e, F_p, L_p, O)
and ``tensionX.yaml`` (tension along x, 100 increments over 15 s, output every 10).  The
reference runs the same job with each grid solver and requires every output dataset to agree
at rtol 1e-5, atol 1e-2 (its ``assert_allclose`` fixture).

Fixture contents: ``material`` (0-based per cell, x fastest), ``cells``, ``size``,
``quaternions`` (one per material), the phase and load dictionaries as JSON strings.
"""
import json
import sys
from pathlib import Path

import numpy as np
import yaml

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from damask_b200 import vti                  # noqa: E402


def main(root: str) -> None:
    res = Path(root) / 'tests' / 'integration' / 'resources' / 'grid_mech_consistency'
    geom = vti.load(res / 'g_444.vti')
    mat = yaml.safe_load((res / 'material_plast.yaml').read_text())
    out = {'material': geom.material, 'cells': np.array(geom.cells), 'size': np.array(geom.size),
           'quaternions': np.array([m['constituents'][0]['O'] for m in mat['material']], dtype=np.float64),
           'phase_json': json.dumps(mat['phase']['Aluminum']),
           'load_json': json.dumps(yaml.safe_load((res / 'tensionX.yaml').read_text()))}
    np.savez_compressed(HERE / 'golden_mech_consistency.npz', **out)
    print('wrote', HERE / 'golden_mech_consistency.npz', sorted(out))


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit(f'usage: python {sys.argv[0]} <path of the reference source tree>')
    main(sys.argv[1])
