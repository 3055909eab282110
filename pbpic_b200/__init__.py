"""pbpic_b200: the 2-D electromagnetic PIC time step of xiaocanli/pbpic
(src/programs/pic2d.f90) as hand-written CUDA kernels for the B200 (sm_100a),
behind a C ABI (include/pbpic.h). This package is the Python view of that ABI.
"""
from ._lib import (BC_CONDUCTING, BC_PERIODIC, COMPAT_BORIS, COMPAT_FOLD, COMPAT_RHO, FP32_MIXED, FP64_PLAIN,
                   LOAD_DOUBLE_HARRIS, LOAD_HARRIS, LOAD_TWO_STREAM, LOAD_UNIFORM, LOAD_WEIBEL, PARTICLE_F32,
                   PARTICLE_F64,
                   FILTER_CERENKOV, FILTER_MARDER, OPT_EXACT_FP64, OPT_NO_AUTOSORT, STATUS_CELL_JUMP, STATUS_NAN, STATUS_UNSORTED,
                   PbpicError, lib)
from .sim import Simulation, counting_sort_keys, kernel_launches

__all__ = [
    "Simulation", "counting_sort_keys", "kernel_launches", "PbpicError", "lib",
    "PARTICLE_F32", "PARTICLE_F64", "OPT_NO_AUTOSORT", "OPT_EXACT_FP64", "FILTER_MARDER", "FILTER_CERENKOV",
    "BC_PERIODIC", "BC_CONDUCTING", "FP64_PLAIN", "FP32_MIXED",
    "COMPAT_BORIS", "COMPAT_FOLD", "COMPAT_RHO",
    "STATUS_CELL_JUMP", "STATUS_NAN", "STATUS_UNSORTED",
    "LOAD_UNIFORM", "LOAD_HARRIS", "LOAD_TWO_STREAM", "LOAD_WEIBEL", "LOAD_DOUBLE_HARRIS",
]
