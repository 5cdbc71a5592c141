"""nlos_lbm -- B200 D3Q19 lattice-Boltzmann acoustic solver.

Python side of the C-ABI in include/nlos_lbm.h.  ``abi`` describes the ABI
(ctypes, no GPU needed); ``solver`` wraps a handle and mirrors the reference
LBMSolver interface; ``build`` compiles liblbm_b200.so in-tree.
"""
from . import abi  # noqa: F401
from .solver import (DroneSource, LBMError, LBMSolver, Probe, SlabGroup, Solver, city_triangles,  # noqa: F401
                     library, stl_write, voxelize)
