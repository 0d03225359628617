"""damask_b200 — DAMASK's grid mechanical hot path (basic spectral scheme with the
phenopowerlaw/Hooke constitutive update) on NVIDIA B200 (sm_100a).

The compute lives in ``libdamask_b200.so`` (C-ABI in ``include/damask_b200.h``);
the Python modules marshal inputs in DAMASK's formats and drive the increment loop.
"""
from .config import LoadCase, Numerics, Phase, parse_load
from .grid import NotConverged, SpectralBasic, SpectralPolarization, run_load_cases

__all__ = ['LoadCase', 'Numerics', 'Phase', 'parse_load', 'SpectralBasic', 'SpectralPolarization', 'run_load_cases', 'NotConverged']
