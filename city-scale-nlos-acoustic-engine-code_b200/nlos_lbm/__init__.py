"""nlos_lbm -- B200 D3Q19 lattice-Boltzmann acoustic solver (Python mirror)."""
from . import abi  # noqa: F401
