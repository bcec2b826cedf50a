"""gell_b200: the Gell per-timestep hot path (Morton-sorted cell-list mechanics, LOD
reaction-diffusion, Ki-67 birth/death) as hand-written CUDA for one NVIDIA B200 (sm_100a), behind
a C ABI (include/gell.h).  This package is the Python mirror of that ABI."""
from .cells import CELL_DTYPE, empty_cells, lattice_spheroid, live_cells, seed_ki67_states, uniform_ball
from .api import (GELL_RNG_PHILOX, GELL_RNG_XORWOW, Ensemble, GellError, GellParams, Simulation, Substrate,
                  default_params, drug, load_library, oxygen, reference_spheroid, write_cells_csv)

__all__ = [
    "CELL_DTYPE", "empty_cells", "lattice_spheroid", "live_cells", "uniform_ball",
    "GELL_RNG_PHILOX", "GELL_RNG_XORWOW", "Ensemble", "GellError", "GellParams", "Simulation", "Substrate",
    "default_params", "drug", "load_library", "oxygen", "reference_spheroid", "seed_ki67_states",
    "write_cells_csv",
]
