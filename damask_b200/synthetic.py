"""Seeded synthetic microstructures in the reference's own recipe.

* seed points: uniform in the box, ``rng.random((N,3)) * size``
  (``python/damask/seeds.py:30-66``, ``from_random`` without ``cells``);
* orientations: normalised Gaussian quaternions, standardised to q0 >= 0
  (``python/damask/_rotation.py:1252-1282``, ``Rotation.from_random``);
* grains: periodic nearest-seed Voronoi tessellation of the cell centres with a
  periodic KD-tree (``python/damask/_geomgrid.py:580-636``,
  ``GeomGrid.from_Voronoi_tessellation``).

One generator ``numpy.random.default_rng(seed)`` draws the seed points first and
then the orientations, so a (cells, size, grains, seed) tuple names one RVE.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def seeds_from_random(size, n_seeds: int, rng: np.random.Generator) -> np.ndarray:
    """Seed coordinates, shape (n_seeds, 3), uniform in [0, size)."""
    return rng.random((n_seeds, 3)) * np.asarray(size, float)


def rotations_from_random(n: int, rng: np.random.Generator) -> np.ndarray:
    """Unit quaternions (w, x, y, z), shape (n, 4), uniform on SO(3), w >= 0."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    q[q[:, 0] < 0.0] *= -1.0
    return q


def cell_centres(cells, size) -> np.ndarray:
    """Cell-centre coordinates, shape (cells0, cells1, cells2, 3), indexed [x, y, z]."""
    cells = np.asarray(cells, int)
    size = np.asarray(size, float)
    delta = size / cells
    axes = [np.linspace(delta[i] * 0.5, size[i] - delta[i] * 0.5, cells[i]) for i in range(3)]
    return np.stack(np.meshgrid(*axes, indexing='ij'), axis=-1)


def voronoi(cells, size, seeds: np.ndarray, periodic: bool = True) -> np.ndarray:
    """Material index per cell, shape (cells0, cells1, cells2), indexed [x, y, z]."""
    from scipy import spatial
    coords = cell_centres(cells, size).reshape(-1, 3)
    tree = spatial.KDTree(seeds, boxsize=np.asarray(size, float) if periodic else None)
    return np.asarray(tree.query(coords, workers=-1)[1]).reshape(tuple(cells))


@dataclass
class RVE:
    cells: tuple[int, int, int]
    size: tuple[float, float, float]
    material: np.ndarray          # int32, shape (N,), x fastest (Fortran order of [x,y,z])
    quaternions: np.ndarray       # (n_materials, 4)

    @property
    def n_cells(self) -> int:
        return int(np.prod(self.cells))


def voronoi_rve(cells, size, n_grains: int, seed: int) -> RVE:
    rng = np.random.default_rng(seed)
    seeds = seeds_from_random(size, n_grains, rng)
    quats = rotations_from_random(n_grains, rng)
    mat = voronoi(cells, size, seeds)
    return RVE(tuple(int(c) for c in cells), tuple(float(s) for s in size),
               np.ascontiguousarray(mat.reshape(-1, order='F').astype(np.int32)), quats)
