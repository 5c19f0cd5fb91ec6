"""fivo2d — host side of the B200 finite-volume stage for FiVoHydro's 2+1D solver.

Mirrors the reference's Julia interface (main2D.jl, src2d/*.jl) over the C ABI
of include/fivo2d.h, implemented by csrc/libfivo2d.so (CUDA, sm_100a).
"""
from .model import (Grid2D, make_grid2d, make_grid_2d, make_layout2d, ConformalHQEOS, LatticeHRGEOS,
                    build_model_2d, allocate_state, IdealDiffVisc2DModel, eos_params)
from . import ic
from .fields_io import save_fields, load_fields
from ._abi import FivoError, load_library

__all__ = ["Grid2D", "make_grid2d", "make_grid_2d", "make_layout2d", "ConformalHQEOS", "LatticeHRGEOS",
           "build_model_2d", "allocate_state", "IdealDiffVisc2DModel", "eos_params", "ic", "FivoError",
           "load_library", "save_fields", "load_fields"]
