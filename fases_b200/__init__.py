"""fases_b200 -- B200-native (sm_100a) stepper for the FASES time-domain room-acoustics solver.

The hot path of vitorotri/fases (3D-solver/core/main3D.cu:1280-1417 with the kernels of
3D-solver/core/functions3D.cuh): WENO-Z reconstruction, Godunov fluxes for linear acoustics,
SSP-RK3 stages, CFS-cPML and ADE pole-residue impedance boundaries on the immersed band, as
hand-written CUDA behind the C ABI of include/fz.h (libfz.so).
"""
from ._abi import FzError, lib  # noqa: F401
from .solver import Group, Solver, params, source_waveform  # noqa: F401

__all__ = ["Solver", "Group", "params", "source_waveform", "FzError", "lib"]
