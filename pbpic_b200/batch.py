"""Batched form: many independent FP32 domains of uneven size stepped
together (persistent kernels over one (domain, tile) table, the counting
sort every step, pairs of steps replayed from a CUDA graph).

    with Batch(domains) as b:          # domains: [(config dict, loader dict), ...]
        b.autotune(8)                  # tile rows and particles per thread
        b.step(2000)
        e = b.energies()               # (ndomains, 4)
        sim = b.domain(3)              # Simulation view of one domain

The reference runs one domain per MPI job; this form has no counterpart there.
"""
import ctypes

import numpy as np

from . import _lib as L
from .sim import Simulation


def _config(cfg):
    c = L.Config()
    for k, v in cfg.items():
        setattr(c, k, v)
    c.precision = L.FP32_MIXED
    return c


class Batch:
    def __init__(self, domains):
        self._lib = L.lib()
        n = len(domains)
        cfgs = (L.Config * n)()
        loaders = (L.Loader * n)()
        for i, (cfg, ld) in enumerate(domains):
            cfgs[i] = _config(cfg)
            loaders[i] = Simulation.loader(**ld)
        self.n = n
        self._b = ctypes.c_void_p()
        L.check(self._lib.pbpic_batch_create(cfgs, loaders, n, ctypes.byref(self._b)))

    def close(self):
        if self._b:
            self._lib.pbpic_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def domain(self, d):
        h = ctypes.c_void_p()
        L.check(self._lib.pbpic_batch_domain(self._b, d, ctypes.byref(h)))
        return Simulation._borrow(h.value)

    def set_tiles(self, tile_rows=None, groups=2):
        tr = None if tile_rows is None else np.ascontiguousarray(tile_rows, dtype=np.int32)
        if tr is not None:
            assert tr.shape == (self.n,)
        L.check(self._lib.pbpic_batch_set_tiles(self._b, L.ptr(tr), groups))

    def tiles(self):
        tr = np.zeros(self.n, dtype=np.int32)
        g = ctypes.c_int32()
        L.check(self._lib.pbpic_batch_get_tiles(self._b, L.ptr(tr), ctypes.byref(g)))
        return tr, g.value

    def step(self, nsteps=1):
        L.check(self._lib.pbpic_batch_step(self._b, nsteps))

    @property
    def stream(self):
        """The batch's cudaStream_t as an integer (torch.cuda.ExternalStream takes it)."""
        s = ctypes.c_void_p()
        L.check(self._lib.pbpic_batch_stream(self._b, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        L.check(self._lib.pbpic_batch_synchronize(self._b))

    def autotune(self, trial_steps=8):
        """Try each tiling for trial_steps real steps; keep the fastest.
        Returns (tile rows per domain, groups, ms per step)."""
        tr = np.zeros(self.n, dtype=np.int32)
        g = ctypes.c_int32()
        ms = ctypes.c_double()
        L.check(self._lib.pbpic_batch_autotune(self._b, trial_steps, L.ptr(tr), ctypes.byref(g), ctypes.byref(ms)))
        return tr, g.value, ms.value

    def energies(self):
        a = np.zeros((self.n, 4))
        L.check(self._lib.pbpic_batch_energies(self._b, L.ptr(a)))
        return a
