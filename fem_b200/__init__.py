"""fem_b200 -- B200-native periodic voxel-FEM homogenization (C^H and dC^H/drho).

The engine is libfemh.so (C++ host + sm_100a CUDA kernels behind the C ABI of
include/femh.h); this package is its Python binding and a torch autograd
wrapper.  See femh.py.
"""
from .femh import (Config, Engine, FemhError, load_library, LIB_PATH, EXPORTS,  # noqa: F401
                   INTERP_SIMP, INTERP_RAMP3, INTERP_BINARY, FP64, MIXED, MIXED_PC, JACOBI_PCG, GMG_PCG,
                   FEMH_OK, FEMH_E_ARG, FEMH_E_CUDA, FEMH_E_OOM, FEMH_E_NOT_CONVERGED, FEMH_E_BREAKDOWN,
                   FEMH_E_STATE)
