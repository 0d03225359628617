"""The benchmark workloads (material, load case, microstructure) in DAMASK's terms.

Each workload is a seeded synthetic Voronoi RVE built with the reference's own
recipe (see :mod:`damask_b200.synthetic`) and a material/load definition written
with the same keys as DAMASK's ``material.yaml`` / ``load.yaml``.

* ``fcc_al``: Aluminum-like phenopowerlaw, 12 {111}<110> systems
  (the ``examples/grid/material.yaml`` phase; C11/C12/C44 = 106.75/60.41/28.34 GPa).
* ``bcc_24``: bcc phenopowerlaw on {110}<111> + {112}<111> (N_sl [12,12], 24 systems),
  C11/C12/C44 = 233.3/135.5/118.0 GPa, xi_0 95/97 MPa, xi_inf 222/412 MPa,
  h_0 1 GPa, n 20, a 2; the 24 interaction values start [1,1.4,1,1.4] and are
  padded with 1.4 (the reference needs one value per interaction type present).
* ``bcc_48``: the same with the third cI family {123}<111> (N_sl [12,12,24], 48 systems), which
  takes the {112} parameters (xi_0 97 MPa, xi_inf 412 MPa); 28 interaction values
  [1,1.4,1,1.4] + 24 x 1.4, as the reference's phenopowerlaw_polygonal-ferrite.yaml.
"""
from __future__ import annotations

import numpy as np

from .config import LoadCase, Numerics, Phase, parse_load
from .synthetic import RVE, voronoi_rve

SIZE_1MM = (1.0e-3, 1.0e-3, 1.0e-3)


def fcc_al(xi_0=31.0e6, xi_inf=63.0e6, h_0=75.0e6, n=20.0, a=2.25) -> Phase:
    return Phase.from_dict({
        'lattice': 'cF',
        'mechanical': {
            'elastic': {'type': 'Hooke', 'C_11': 106.75e9, 'C_12': 60.41e9, 'C_44': 28.34e9},
            'plastic': {'type': 'phenopowerlaw', 'N_sl': [12], 'a_sl': [a], 'atol_xi': 1.0,
                        'dot_gamma_0_sl': [0.001], 'h_0_sl-sl': [h_0], 'h_sl-sl': [1, 1, 1.4, 1.4, 1.4, 1.4, 1.4],
                        'n_sl': [n], 'xi_0_sl': [xi_0], 'xi_inf_sl': [xi_inf]}}})


def bcc_24() -> Phase:
    h = [1, 1.4, 1, 1.4] + [1.4] * 20
    return Phase.from_dict({
        'lattice': 'cI',
        'mechanical': {
            'elastic': {'type': 'Hooke', 'C_11': 233.3e9, 'C_12': 135.5e9, 'C_44': 118.0e9},
            'plastic': {'type': 'phenopowerlaw', 'N_sl': [12, 12], 'a_sl': [2.0, 2.0],
                        'dot_gamma_0_sl': [0.001, 0.001], 'h_0_sl-sl': [1.0e9, 1.0e9], 'h_sl-sl': h,
                        'n_sl': [20, 20], 'xi_0_sl': [95.0e6, 97.0e6], 'xi_inf_sl': [222.0e6, 412.0e6]}}})


def bcc_48() -> Phase:
    h = [1, 1.4, 1, 1.4] + [1.4] * 24
    return Phase.from_dict({
        'lattice': 'cI',
        'mechanical': {
            'elastic': {'type': 'Hooke', 'C_11': 233.3e9, 'C_12': 135.5e9, 'C_44': 118.0e9},
            'plastic': {'type': 'phenopowerlaw', 'N_sl': [12, 12, 24], 'a_sl': [2.0, 2.0, 2.0],
                        'dot_gamma_0_sl': [0.001] * 3, 'h_0_sl-sl': [1.0e9] * 3, 'h_sl-sl': h,
                        'n_sl': [20, 20, 20], 'xi_0_sl': [95.0e6, 97.0e6, 97.0e6],
                        'xi_inf_sl': [222.0e6, 412.0e6, 412.0e6]}}})


def tension_x(t: float, N: int, f_out: int = 1) -> list[LoadCase]:
    """Uniaxial tension dot_F_xx = 1e-3/s with P_yy = P_zz = 0 (examples/grid/tensionX.yaml)."""
    return parse_load({'loadstep': [{
        'boundary_conditions': {'mechanical': {
            'dot_F': [[1.0e-3, 0, 0], [0, 'x', 0], [0, 0, 'x']],
            'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]]}},
        'discretization': {'t': t, 'N': N}, 'f_out': f_out}]})


def numerics_default() -> Numerics:
    n = Numerics()
    n.eps_rel_div = 5.0e-4
    n.eps_rel_P = 1.0e-3
    return n


WORKLOADS = {
    # name: (cells, grains, seed, phase, t, N)
    'grid16_fcc_20g': ((16, 16, 16), 20, 0, 'fcc_al', 60.0, 60),
    'grid64_fcc_200g': ((64, 64, 64), 200, 1, 'fcc_al', 100.0, 100),
    'grid32_fcc_50g': ((32, 32, 32), 50, 2, 'fcc_al', 50.0, 50),
    'grid256_bcc24_2000g': ((256, 256, 256), 2000, 3, 'bcc_24', 100.0, 100),
    'grid256_bcc48_2000g': ((256, 256, 256), 2000, 3, 'bcc_48', 100.0, 100),
}
PHASES = {'fcc_al': lambda: fcc_al(), 'bcc_24': lambda: bcc_24(), 'bcc_48': lambda: bcc_48()}


def make(name: str, cells=None) -> tuple[RVE, Phase, list[LoadCase], Numerics]:
    c, grains, seed, ph, t, N = WORKLOADS[name]
    cells = tuple(cells) if cells is not None else c
    rve = voronoi_rve(cells, SIZE_1MM, grains, seed)
    phase = PHASES[ph]()
    return rve, phase, tension_x(t, N), numerics_default()


def make_cut(name: str, cells) -> tuple[RVE, Phase, list[LoadCase], Numerics]:
    """A smaller RVE of a workload at the workload's grain density (grains scaled by the cell
    count, at least 2) with its seed, material, load and numerics: e.g. a 64^3 cut of the
    256^3/2000-grain RVE has 31 grains."""
    c, grains, seed, ph, t, N = WORKLOADS[name]
    cells = tuple(int(x) for x in cells)
    g = max(2, int(round(grains * np.prod(cells) / np.prod(c))))
    rve = voronoi_rve(cells, SIZE_1MM, g, seed)
    return rve, PHASES[ph](), tension_x(t, N), numerics_default()


def material_yaml(rve: RVE, phase_name: str, phase: dict) -> dict:
    """material.yaml content (one constituent per material, isostrain homogenization)."""
    return {'homogenization': {'direct': {'N_constituents': 1, 'mechanical': {'type': 'isostrain'}}},
            'phase': {phase_name: phase},
            'material': [{'homogenization': 'direct',
                          'constituents': [{'phase': phase_name, 'v': 1.0, 'O': [float(x) for x in q]}]}
                         for q in np.asarray(rve.quaternions)]}


def simple_shear_xy(t: float, N: int, rate: float = 1.0e-3) -> list[LoadCase]:
    """Simple shear dot_F_xy = rate, every component deformation-controlled."""
    return parse_load({'loadstep': [{
        'boundary_conditions': {'mechanical': {'dot_F': [[0, rate, 0], [0, 0, 0], [0, 0, 0]]}},
        'discretization': {'t': t, 'N': N}}]})


def tension_along(axis, t: float, N: int) -> list[LoadCase]:
    """Uniaxial tension along a unit axis: the x-tension load case with the load-case rotation
    R (DAMASK_grid.f90:524) that takes x to the axis."""
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    ang = float(np.degrees(np.arccos(np.clip(a[0], -1.0, 1.0))))
    rot = np.cross([1.0, 0.0, 0.0], a)
    n = np.linalg.norm(rot)
    ax = rot / n if n > 1e-12 else np.array([0.0, 0.0, 1.0])
    lcs = parse_load({'loadstep': [{
        'boundary_conditions': {'mechanical': {
            'dot_F': [[1.0e-3, 0, 0], [0, 'x', 0], [0, 0, 'x']],
            'P': [['x', 'x', 'x'], ['x', 0, 'x'], ['x', 'x', 0]],
            'R': [float(ax[0]), float(ax[1]), float(ax[2]), ang]}},
        'discretization': {'t': t, 'N': N}}]})
    return lcs


def batched_jobs(n: int = 512, seed: int = 4, t: float = 40.0, N: int = 40):
    """The batched workload: n independent RVEs, edge uniform in {8, 12, 16, 24, 32}, grain count
    uniform in [5, 100], orientations uniform on SO(3), the fcc material; each RVE gets uniaxial
    tension along a random unit axis or simple shear dot_F_xy = 1e-3/s, 40 increments to 4 %.
    Returns [(rve, phase, loadcases, numerics)]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n):
        edge = int(rng.choice([8, 12, 16, 24, 32]))
        grains = int(rng.integers(5, 101))
        rve = voronoi_rve((edge, edge, edge), SIZE_1MM, grains, int(rng.integers(2 ** 31)))
        if rng.random() < 0.5:
            axis = rng.normal(size=3)
            lcs = tension_along(axis / np.linalg.norm(axis), t, N)
        else:
            lcs = simple_shear_xy(t, N)
        jobs.append((rve, fcc_al(), lcs, numerics_default()))
    return jobs
