"""Generate ``golden.npz`` from the reference's own Python package.

Run here (where the reference tree is mounted), not on the test machines:

    python tests/golden/make_golden.py <path of the reference's source tree>

The reference package is imported piecewise: its optional I/O dependencies
(h5py, vtk, matplotlib) are replaced by inert stand-ins because none of the
functions used here touches them.  Fixtures written:

* ``schmid_cF``, ``schmid_cI``: Schmid matrices ``Crystal.Schmid(N_slip='*')``
  (``python/damask/_crystal.py``), all slip systems, shape (n, 3, 3);
* ``seeds_0``, ``quats_0``: 20 seed points in a 1 mm cube and 20 orientations drawn
  from one generator ``default_rng(0)`` (``seeds.from_random``, ``Rotation.from_random``);
* ``div_field``, ``div_rms``: a seeded random tensor field on an 8x6x4 grid of size
  (1, 2, 3) mm and the RMS of its spectral divergence ``grid.divergence``
  (``python/damask/grid.py:143-167``);
* ``coords_<case>_{F,size,ip,nodes}``: deformation gradient fields and their current
  cell-centre and node coordinates ``grid.coordinates_point`` / ``grid.coordinates_node``
  (``python/damask/grid.py:298-330,445-470``, the Python form of ``utilities_updateCoords``),
  case ``odd`` a random field on 5x7x9 and case ``smooth`` a band-limited field on 8x6x4 (no
  content at the Nyquist frequencies, where the Python form transforms a different axis).
"""
import importlib
import sys
import types
from pathlib import Path

import numpy as np


def import_reference(root: str):
    sys.path.insert(0, str(Path(root) / 'python'))

    class _Inert(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith('__'):
                raise AttributeError(name)
            return type(name, (), {})

    for name in ('h5py', 'vtk', 'vtkmodules', 'matplotlib', 'matplotlib.pyplot', 'PIL'):
        m = _Inert(name)
        m.__path__ = []
        sys.modules[name] = m
    pkg = types.ModuleType('damask')
    pkg.__path__ = [str(Path(root) / 'python' / 'damask')]
    pkg.version = '0'
    sys.modules['damask'] = pkg
    rot = importlib.import_module('damask._rotation')
    pkg.Rotation = rot.Rotation
    return (rot, importlib.import_module('damask.seeds'), importlib.import_module('damask._crystal'),
            importlib.import_module('damask.grid'))


def main(root: str) -> None:
    rot, seeds, crystal, grid = import_reference(root)
    out = {}
    out['schmid_cF'] = crystal.Crystal(lattice='cF').Schmid(N_slip='*')
    out['schmid_cI'] = crystal.Crystal(lattice='cI').Schmid(N_slip='*')
    rng = np.random.default_rng(0)
    out['seeds_0'] = seeds.from_random([1.0e-3] * 3, 20, rng=rng)
    out['quats_0'] = rot.Rotation.from_random(20, rng=rng).quaternion
    size = np.array([1.0e-3, 2.0e-3, 3.0e-3])
    f = np.random.default_rng(7).normal(size=(8, 6, 4, 3, 3)) * 1.0e8
    d = grid.divergence(size, f)
    out['div_field'] = f
    out['div_size'] = size
    out['div_rms'] = np.sqrt(np.mean(np.sum(d ** 2, axis=-1)))
    for case, cells in (('odd', (5, 7, 9)), ('smooth', (8, 6, 4))):
        size = np.array([1.0e-3, 2.0e-3, 1.5e-3])
        g = np.random.default_rng(3)
        if case == 'odd':
            F = np.eye(3) + 0.05 * g.normal(size=cells + (3, 3))
        else:
            X = np.stack(np.meshgrid(*[np.arange(c) / c for c in cells], indexing='ij'), -1)
            F = np.broadcast_to(np.eye(3) + 0.02 * g.normal(size=(3, 3)), cells + (3, 3)).copy()
            for _ in range(3):
                A = 0.03 * g.normal(size=(3, 3))
                kv = g.integers(-1, 2, size=3)
                F += A * np.cos(2 * np.pi * (X @ kv) + g.uniform())[..., None, None]
        out[f'coords_{case}_F'] = F
        out[f'coords_{case}_size'] = size
        out[f'coords_{case}_ip'] = grid.coordinates_point(size, F)
        out[f'coords_{case}_nodes'] = grid.coordinates_node(size, F)
    np.savez_compressed(Path(__file__).with_name('golden.npz'), **out)
    print({k: np.shape(v) for k, v in out.items()})


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit(f'usage: python {sys.argv[0]} <path of the reference source tree>')
    main(sys.argv[1])
