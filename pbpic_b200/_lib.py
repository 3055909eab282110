"""ctypes declarations of the C ABI in include/pbpic.h.

The library is the in-tree pbpic_b200/libpbpic.so built by pbpic_b200.build.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbpic.so")

PBPIC_OK = 0
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ECAPACITY", -5: "ESTATE"}
ERR_INVAL, ERR_CUDA, ERR_NOMEM, ERR_CAPACITY, ERR_STATE = -1, -2, -3, -4, -5

BC_PERIODIC, BC_CONDUCTING = 0, 1
FP64_PLAIN, FP32_MIXED = 0, 1
COMPAT_BORIS, COMPAT_FOLD, COMPAT_RHO = 1, 2, 4
STATUS_CELL_JUMP, STATUS_NAN, STATUS_UNSORTED = 1, 2, 4
LOAD_UNIFORM, LOAD_HARRIS, LOAD_TWO_STREAM, LOAD_WEIBEL, LOAD_DOUBLE_HARRIS = 0, 1, 2, 3, 4
FILTER_MARDER, FILTER_CERENKOV = 1, 2
OPT_NO_AUTOSORT = 1
OPT_EXACT_FP64 = 2


class Config(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dt", ctypes.c_double),
        ("cva", ctypes.c_double), ("mime", ctypes.c_double), ("in0", ctypes.c_double),
        ("ybc", ctypes.c_int32), ("precision", ctypes.c_int32), ("compat", ctypes.c_int32),
        ("track_pid", ctypes.c_int32), ("capacity", ctypes.c_int64),
        ("tile_rows", ctypes.c_int32), ("options", ctypes.c_int32),
    ]


class Loader(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("ppc", ctypes.c_int32),
        ("vthe", ctypes.c_double), ("vthi", ctypes.c_double),
        ("vdrift_e", ctypes.c_double), ("vdrift_i", ctypes.c_double),
        ("lambda_", ctypes.c_double), ("nb", ctypes.c_double), ("psi0", ctypes.c_double),
        ("bguide", ctypes.c_double), ("b0z", ctypes.c_double), ("anisotropy", ctypes.c_double),
        ("seed", ctypes.c_uint64), ("immobile_ions", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("vthe_bg", ctypes.c_double), ("vthi_bg", ctypes.c_double),
    ]


class DiffConfig(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("ppc", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("dx", ctypes.c_double), ("mime", ctypes.c_double), ("wpe_wce", ctypes.c_double),
        ("lambda_", ctypes.c_double), ("nb0", ctypes.c_double), ("cfl", ctypes.c_double),
        ("nsteps", ctypes.c_int32), ("checkpoint_every", ctypes.c_int32), ("loss", ctypes.c_int32),
        ("reserved", ctypes.c_int32), ("seed", ctypes.c_uint64),
    ]


class DiffParams(ctypes.Structure):
    _fields_ = [("psi0", ctypes.c_double), ("nb", ctypes.c_double), ("ti_te", ctypes.c_double)]


LOSS_MAGNETIC, LOSS_JDOTE = 0, 1

# The reference's `type particle` (pic2d.f90:47-50) and its double-precision twin.
PARTICLE_F32 = np.dtype([("dx", "<f4"), ("dy", "<f4"), ("ux", "<f4"), ("uy", "<f4"), ("uz", "<f4"),
                         ("grid", "<i4"), ("q", "<i4"), ("pid", "<i4")])
PARTICLE_F64 = np.dtype([("dx", "<f8"), ("dy", "<f8"), ("ux", "<f8"), ("uy", "<f8"), ("uz", "<f8"),
                         ("grid", "<i4"), ("q", "<i4"), ("pid", "<i4"), ("pad", "<i4")])
assert PARTICLE_F32.itemsize == 32 and PARTICLE_F64.itemsize == 56

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_PI32 = ctypes.POINTER(ctypes.c_int32)
_PI64 = ctypes.POINTER(ctypes.c_int64)
_PD = ctypes.POINTER(ctypes.c_double)

# name -> (argtypes); every function returns int
SIGNATURES = {
    "pbpic_create": [ctypes.POINTER(Config), ctypes.POINTER(_P)],
    "pbpic_destroy": [_P],
    "pbpic_set_stream": [_P, _P],
    "pbpic_get_config": [_P, ctypes.POINTER(Config)],
    "pbpic_init_plasma": [_P, ctypes.POINTER(Loader)],
    "pbpic_loader_count": [_P, ctypes.POINTER(Loader), _PI64],
    "pbpic_load_particles_f32": [_P, _P, _I64],
    "pbpic_load_particles_f64": [_P, _P, _I64],
    "pbpic_store_particles_f32": [_P, _P, _I64, _PI64],
    "pbpic_store_particles_f64": [_P, _P, _I64, _PI64],
    "pbpic_load_particles_soa_f64": [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P],
    "pbpic_store_particles_soa_f64": [_P, _I64, _PI64, _P, _P, _P, _P, _P, _P, _P, _P],
    "pbpic_num_particles": [_P, _PI64],
    "pbpic_load_fields_f64": [_P, _P],
    "pbpic_store_fields_f64": [_P, _P],
    "pbpic_store_emfgrid_f64": [_P, _P],
    "pbpic_store_denjr_f64": [_P, _P],
    "pbpic_push": [_P],
    "pbpic_fieldsolve": [_P],
    "pbpic_sort": [_P],
    "pbpic_step": [_P, _I32, _I32],
    "pbpic_synchronize": [_P],
    "pbpic_energies": [_P, _P],
    "pbpic_energy_history": [_P, _P, _I32, _PI32],
    "pbpic_time_step": [_P, _PI32],
    "pbpic_cell_counts": [_P, _P],
    "pbpic_gauss_residual": [_P, _PD],
    "pbpic_gauss_residual_rows": [_P, _I32, _I32, _PD],
    "pbpic_reconnected_flux": [_P, _PD],
    "pbpic_status": [_P, _PI32],
    "pbpic_counting_sort_keys": [_P, _I64, _I32, _P, _P, _P],
    "pbpic_kernel_launches": [_PI64],
    "pbpic_counting_sort_keys_static": [_P, _I64, _I32, _P, _P, _P],
    "pbpic_energy_spectra": [_P, ctypes.c_double, ctypes.c_double, _I32, _P],
    "pbpic_field_cuts": [_P, _P, _I32, _P, _I32, _P],
    "pbpic_set_field_filters": [_P, _I32, ctypes.c_double, ctypes.c_double],
    "pbpic_dump": [_P, ctypes.c_char_p],
    "pbpic_dump_h5": [_P, ctypes.c_char_p, ctypes.c_double, ctypes.c_double, _I32],
    "pbpic_band_extract": [_P, _I32, _I32, _I32, _I32, _P, _I64, _PI64],
    "pbpic_band_keep": [_P, _I32, _I32],
    "pbpic_band_append": [_P, _P, _I64, _I32, _I32],
    "pbpic_band_replace": [_P, _I32, _I32, _P, _I64, _I32, _P, _I64, _I32, _I32],
    "pbpic_field_rows_get": [_P, _I32, _I32, _P],
    "pbpic_field_rows_set": [_P, _I32, _I32, _P],
    "pbpic_energies_rows": [_P, _I32, _I32, _I32, _I32, _P],
    "pbpic_restart": [_P, ctypes.c_char_p],
    "pbpic_batch_create": [ctypes.POINTER(Config), ctypes.POINTER(Loader), _I32, ctypes.POINTER(_P)],
    "pbpic_batch_destroy": [_P],
    "pbpic_batch_num_domains": [_P, _PI32],
    "pbpic_batch_domain": [_P, _I32, ctypes.POINTER(_P)],
    "pbpic_batch_set_tiles": [_P, _P, _I32],
    "pbpic_batch_get_tiles": [_P, _P, _PI32],
    "pbpic_batch_step": [_P, _I32],
    "pbpic_batch_stream": [_P, ctypes.POINTER(_P)],
    "pbpic_batch_synchronize": [_P],
    "pbpic_batch_autotune": [_P, _I32, _P, _PI32, _PD],
    "pbpic_batch_energies": [_P, _P],
    "pbpic_diff_create": [ctypes.POINTER(DiffConfig), ctypes.POINTER(_P)],
    "pbpic_diff_destroy": [_P],
    "pbpic_diff_forward": [_P, ctypes.POINTER(DiffParams), _PD],
    "pbpic_diff_backward": [_P, _PD],
}

STATIC_SORT_MAX_KEYS = 1048576  # PBPIC_STATIC_SORT_MAX_KEYS

_lib = None


class PbpicError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pbpic error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def lib():
    """Load libpbpic.so once and declare its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m pbpic_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.pbpic_last_error.argtypes = []
    L.pbpic_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc):
    if rc != PBPIC_OK:
        raise PbpicError(rc, lib().pbpic_last_error().decode())
    return rc


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None
