"""ORACLE -- TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), and the
CPU-baseline legs of bench.py).

ctypes view of oracle/liboracle.so, the CPU restatement of the reference step
(src/programs/pic2d.f90). Parity unpinned: the reference has no golden vectors
and cannot be built here; tests/golden pins this restatement against an
independent line-by-line Python transcription.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

PARTICLE = np.dtype([("dx", "<f8"), ("dy", "<f8"), ("ux", "<f8"), ("uy", "<f8"), ("uz", "<f8"),
                     ("grid", "<i4"), ("q", "<i4"), ("pid", "<i4"), ("pad", "<i4")])


class OrcParams(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dt", ctypes.c_double), ("cva", ctypes.c_double), ("mime", ctypes.c_double),
                ("in0", ctypes.c_double), ("ybc", ctypes.c_int32), ("compat", ctypes.c_int32)]


class LoadParams(ctypes.Structure):  # pic::LoadParams in pbpic_b200/csrc/pic_common.h
    _fields_ = [("kind", ctypes.c_int32), ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("npairs", ctypes.c_int64), ("nsheet", ctypes.c_int64), ("ppc", ctypes.c_int32),
                ("uthe", ctypes.c_double), ("uthi", ctypes.c_double), ("uthe_perp", ctypes.c_double),
                ("udrift_e", ctypes.c_double), ("udrift_i", ctypes.c_double), ("lambda_", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("uthe_bg", ctypes.c_double), ("uthi_bg", ctypes.c_double)]


class FieldInit(ctypes.Structure):  # pic::FieldInit in pbpic_b200/csrc/pic_fields_init.h
    _fields_ = [("kind", ctypes.c_int32), ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("lambda_", ctypes.c_double),
                ("psi0", ctypes.c_double), ("bguide", ctypes.c_double), ("b0z", ctypes.c_double)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int]
        L.orc_create.restype = P
        L.orc_destroy.argtypes = [P]
        L.orc_load_particles.argtypes = [P, P, ctypes.c_int64, ctypes.c_int64]
        L.orc_get_particles.argtypes = [P, P, ctypes.c_int64]
        L.orc_get_particles.restype = ctypes.c_int64
        L.orc_nptl.argtypes = [P]
        L.orc_nptl.restype = ctypes.c_int64
        for f in ("orc_set_yee", "orc_get_yee", "orc_get_j", "orc_get_grid", "orc_energies"):
            getattr(L, f).argtypes = [P, P]
        for f in ("orc_pusher", "orc_fieldsolver"):
            getattr(L, f).argtypes = [P]
        L.orc_countingsort.argtypes = [P, P]
        L.orc_set_filters.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.orc_omp_pusher.argtypes = [P, ctypes.c_int]
        L.orc_omp_countingsort.argtypes = [P, ctypes.c_int]
        L.orc_omp_max_threads.restype = ctypes.c_int
        L.orc_load_pairs.argtypes = [ctypes.POINTER(LoadParams), ctypes.c_int64, ctypes.c_int64, P]
        L.orc_philox.argtypes = [ctypes.c_uint64] * 6 + [P]
        L.orc_log.argtypes = [ctypes.c_double]
        L.orc_log.restype = ctypes.c_double
        L.orc_init_fields.argtypes = [ctypes.POINTER(FieldInit), P]
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """One domain of the CPU restatement. precision: 'f64' or 'f32'."""

    def __init__(self, mx, my, dx, dy, dt, cva, mime, in0, ybc=0, compat=0, precision="f64", **_ignored):
        self.L = lib()
        self.mx, self.my = mx, my
        self.params = OrcParams(mx, my, dx, dy, dt, cva, mime, in0, ybc, compat)
        self.h = self.L.orc_create(ctypes.byref(self.params), 0 if precision == "f64" else 1)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def load_particles(self, p, capacity=None):
        p = np.ascontiguousarray(p.astype(PARTICLE, copy=False))
        cap = len(p) if capacity is None else capacity
        self.L.orc_load_particles(self.h, _p(p), len(p), cap)

    def particles(self):
        n = self.L.orc_nptl(self.h)
        out = np.zeros(n, dtype=PARTICLE)
        self.L.orc_get_particles(self.h, _p(out), n)
        return out

    def set_fields(self, yee6):
        a = np.ascontiguousarray(yee6, dtype=np.float64)
        assert a.shape == (6, self.mx, self.my + 1)
        self.L.orc_set_yee(self.h, _p(a))

    def fields(self):
        a = np.zeros((6, self.mx, self.my + 1))
        self.L.orc_get_yee(self.h, _p(a))
        return a

    def current(self):
        a = np.zeros((4, self.mx, self.my + 1))
        self.L.orc_get_j(self.h, _p(a))
        return a

    def emfgrid(self):
        a = np.zeros((self.mx + 1, self.my + 1, 8))
        self.L.orc_get_grid(self.h, _p(a))
        return a

    def pusher(self):
        self.L.orc_pusher(self.h)

    def fieldsolver(self):
        self.L.orc_fieldsolver(self.h)

    def set_filters(self, flags, marder_d=0.001, cerenkov_tau=0.125):
        """Enable the Marder (bit 0) and Cherenkov (bit 1) field filters."""
        self.L.orc_set_filters(self.h, flags, marder_d, cerenkov_tau)

    def countingsort(self):
        c = np.zeros(self.mx * self.my, dtype=np.int32)
        self.L.orc_countingsort(self.h, _p(c))
        return c

    def omp_pusher(self, nthreads=0):
        self.L.orc_omp_pusher(self.h, nthreads)

    def omp_countingsort(self, nthreads=0):
        self.L.orc_omp_countingsort(self.h, nthreads)

    def energies(self):
        a = np.zeros(4)
        self.L.orc_energies(self.h, _p(a))
        return a


def max_threads():
    return lib().orc_omp_max_threads()


def philox(c, k):
    out = np.zeros(4, dtype=np.uint64)
    lib().orc_philox(*[int(x) for x in c], *[int(x) for x in k], _p(out))
    return out


def pic_log(x):
    return lib().orc_log(float(x))


# ------------------------------------------------------------------ loaders
def load_params(cfg, ld):
    """pic::LoadParams for a handle configuration and a loader, computed the
    way the library does (pbpic_api.cu loader_params)."""
    u = lambda v: v / math.sqrt(1.0 - v * v)
    kind = ld.get("kind", 0)
    ppc = ld["ppc"]
    npairs = ppc * cfg["mx"] * cfg["my"]
    uthe, uthi = u(ld.get("vthe", 0.0)), u(ld.get("vthi", 0.0))
    uthe_perp = uthe
    if kind == 3:
        a = ld.get("anisotropy", 1.0) or 1.0
        uthe_perp = u(ld["vthe"])
        uthe = u(ld["vthe"] / math.sqrt(a))
    nsheet = 0
    if kind == 1:
        ly = cfg["my"] * cfg["dy"]
        fs = 2.0 * ld["lambda_"] / (2.0 * ld["lambda_"] + ld["nb"] * ly)
        nsheet = int(round(npairs * fs))
    if kind == 4:  # double Harris: an even number of sheet pairs, half in each sheet
        lx = cfg["mx"] * cfg["dx"]
        fs = 4.0 * ld["lambda_"] / (4.0 * ld["lambda_"] + ld["nb"] * lx)
        nsheet = 2 * _round_half_away(0.5 * npairs * fs)
    return LoadParams(kind, cfg["mx"], cfg["my"], cfg["dx"], cfg["dy"], npairs, nsheet, ppc, uthe, uthi, uthe_perp,
                      u(ld.get("vdrift_e", 0.0)), u(ld.get("vdrift_i", 0.0)), ld.get("lambda_", 0.0),
                      ld.get("seed", 0), u(ld.get("vthe_bg", 0.0)), u(ld.get("vthi_bg", 0.0)))


def _round_half_away(x):
    """llround: halves away from zero (Python's round takes them to even)."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def load_plasma(cfg, ld):
    """(particles, yee6) of a loader on the CPU: the same bits as pbpic_init_plasma
    before its sort (pairs in load order)."""
    L = lib()
    lp = load_params(cfg, ld)
    out = np.zeros(2 * lp.npairs, dtype=PARTICLE)
    L.orc_load_pairs(ctypes.byref(lp), 0, lp.npairs, _p(out))
    if ld.get("immobile_ions", 0):
        out = out[1::2].copy()
    fi = FieldInit(ld.get("kind", 0), cfg["mx"], cfg["my"], cfg["dx"], cfg["dy"], ld.get("lambda_", 0.0),
                   ld.get("psi0", 0.0), ld.get("bguide", 0.0), ld.get("b0z", 0.0))
    yee = np.zeros((6, cfg["mx"], cfg["my"] + 1))
    L.orc_init_fields(ctypes.byref(fi), _p(yee))
    return out, yee
