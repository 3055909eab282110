"""Host-side view of one pbpic domain on the GPU, over the C ABI.

The methods keep the names of the reference's subroutines
(src/programs/pic2d.f90): `pusher` (912-1217), `fieldsolver` (678-860),
`countingsort` (1303-1329), and the time loop body `step` (171-188). Errors
of the library raise PbpicError with the library's message.
"""
import ctypes

import numpy as np

from . import _lib as L


class Simulation:
    def __init__(self, mx, my, dx, dy, dt, cva, mime, in0, ybc=L.BC_PERIODIC, precision="fp64",
                 compat=0, track_pid=False, capacity=0, tile_rows=0, options=0):
        self._lib = L.lib()
        prec = {"fp64": L.FP64_PLAIN, "plain": L.FP64_PLAIN, "fp32": L.FP32_MIXED, "mixed": L.FP32_MIXED}[precision]
        self.cfg = L.Config(mx=mx, my=my, dx=dx, dy=dy, dt=dt, cva=cva, mime=mime, in0=in0, ybc=ybc,
                            precision=prec, compat=compat, track_pid=int(bool(track_pid)),
                            capacity=int(capacity), tile_rows=tile_rows, options=options)
        self.mx, self.my = mx, my
        self.precision = precision
        self._h = ctypes.c_void_p()
        L.check(self._lib.pbpic_create(ctypes.byref(self.cfg), ctypes.byref(self._h)))

    @classmethod
    def _borrow(cls, handle):
        """A view of a handle owned elsewhere (a domain of a Batch); closing
        the view leaves the handle alive."""
        self = cls.__new__(cls)
        self._lib = L.lib()
        self._h = ctypes.c_void_p(handle)
        self._owned = False
        self.cfg = L.Config()
        L.check(self._lib.pbpic_get_config(self._h, ctypes.byref(self.cfg)))
        self.mx, self.my = self.cfg.mx, self.cfg.my
        self.precision = "fp32" if self.cfg.precision == L.FP32_MIXED else "fp64"
        return self

    @classmethod
    def from_config(cls, cfg, **kw):
        args = dict(cfg)
        args.update(kw)
        return cls(**args)

    # --------------------------------------------------------------- lifecycle
    def close(self):
        if self._h and getattr(self, "_owned", True):
            self._lib.pbpic_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr):
        L.check(self._lib.pbpic_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # ----------------------------------------------------------------- loading
    @staticmethod
    def loader(**kw):
        ld = L.Loader()
        for k, v in kw.items():
            setattr(ld, k, v)
        return ld

    def loader_count(self, **kw):
        n = ctypes.c_int64()
        L.check(self._lib.pbpic_loader_count(self._h, ctypes.byref(self.loader(**kw)), ctypes.byref(n)))
        return n.value

    def init_plasma(self, **kw):
        L.check(self._lib.pbpic_init_plasma(self._h, ctypes.byref(self.loader(**kw))))

    def load_particles(self, p):
        p = np.ascontiguousarray(p)
        if p.dtype == L.PARTICLE_F32:
            L.check(self._lib.pbpic_load_particles_f32(self._h, L.ptr(p), len(p)))
        elif p.dtype == L.PARTICLE_F64:
            L.check(self._lib.pbpic_load_particles_f64(self._h, L.ptr(p), len(p)))
        else:
            raise TypeError("particles must have dtype PARTICLE_F32 or PARTICLE_F64")

    def num_particles(self):
        n = ctypes.c_int64()
        L.check(self._lib.pbpic_num_particles(self._h, ctypes.byref(n)))
        return n.value

    def particles(self, dtype=L.PARTICLE_F64):
        n = self.num_particles()
        out = np.zeros(n, dtype=dtype)
        got = ctypes.c_int64()
        fn = self._lib.pbpic_store_particles_f64 if dtype == L.PARTICLE_F64 else self._lib.pbpic_store_particles_f32
        L.check(fn(self._h, L.ptr(out), n, ctypes.byref(got)))
        return out

    def load_fields(self, yee6):
        a = np.ascontiguousarray(yee6, dtype=np.float64)
        assert a.shape == (6, self.mx, self.my + 1)
        L.check(self._lib.pbpic_load_fields_f64(self._h, L.ptr(a)))

    def fields(self):
        a = np.zeros((6, self.mx, self.my + 1))
        L.check(self._lib.pbpic_store_fields_f64(self._h, L.ptr(a)))
        return a

    def emfgrid(self):
        a = np.zeros((self.mx + 1, self.my + 1, 8))
        L.check(self._lib.pbpic_store_emfgrid_f64(self._h, L.ptr(a)))
        return a

    def denjr(self):
        a = np.zeros((4, self.mx, self.my + 1))
        L.check(self._lib.pbpic_store_denjr_f64(self._h, L.ptr(a)))
        return a

    # -------------------------------------------------------------------- step
    def pusher(self):
        L.check(self._lib.pbpic_push(self._h))

    def fieldsolver(self):
        L.check(self._lib.pbpic_fieldsolve(self._h))

    def countingsort(self):
        L.check(self._lib.pbpic_sort(self._h))

    def step(self, nsteps=1, sort_every=50):
        L.check(self._lib.pbpic_step(self._h, nsteps, sort_every))

    def synchronize(self):
        L.check(self._lib.pbpic_synchronize(self._h))

    def energy_spectra(self, de_electron=0.005, de_ion=None, nbins=1000, ti_te=1.0):
        """(2, nbins) counts, electrons then ions, of (gamma-1) ms in ((k-1) de, k de]
        (energyspectra, pic2d.f90:1957-1990; ion bins de * Ti/Te by default)."""
        de_ion = de_electron * ti_te if de_ion is None else de_ion
        out = np.zeros((2, nbins), dtype=np.int64)
        L.check(self._lib.pbpic_energy_spectra(self._h, de_electron, de_ion, nbins, L.ptr(out)))
        return out

    def field_cuts(self, rows=None, cols=None):
        """Node values (ex ey ez bx by bz) along node rows (all x) and node columns
        (all y), as dispersioninfo keeps them (pic2d.f90:2124-2142). Default cuts
        are the reference's diagnostic indices (initspectdens, pic2d.f90:318-350)."""
        if rows is None:
            rows = [(self.my * i // 2 - self.my // 4 - 2 - 1) % self.my for i in (1, 2)]
        if cols is None:
            cols = [self.mx * i // 2 - self.mx // 4 - 1 for i in (1, 2)]
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.zeros(len(r) * self.mx * 6 + len(c) * self.my * 6)
        L.check(self._lib.pbpic_field_cuts(self._h, L.ptr(r), len(r), L.ptr(c), len(c), L.ptr(out)))
        nr = len(r) * self.mx * 6
        return out[:nr].reshape(len(r), self.mx, 6), out[nr:].reshape(len(c), self.my, 6)

    def set_field_filters(self, flags, marder_d=0.0, cerenkov_tau=0.0):
        """Marder cleaning (bit 0) and the Cherenkov filter (bit 1); 0 = reference constants."""
        L.check(self._lib.pbpic_set_field_filters(self._h, flags, marder_d, cerenkov_tau))

    # ---------------------------------------------------------- dump / restart
    def dump(self, directory):
        """Write the state as .npy files named like the reference's dump datasets."""
        L.check(self._lib.pbpic_dump(self._h, str(directory).encode()))

    def dump_h5(self, directory, de_electron=0.0, de_ion=0.0, nbins=0):
        """Write the reference's HDF5 dump files (particles.h5, fields%05d.h5,
        spectra.h5 with one group per call, energy_tot.h5) into `directory`;
        0 selects the default bins (0.005, de_electron, 1000)."""
        L.check(self._lib.pbpic_dump_h5(self._h, str(directory).encode(), de_electron, de_ion, nbins))

    def restart(self, directory):
        """Load a dump written by dump() (same grid, boundary and precision)."""
        L.check(self._lib.pbpic_restart(self._h, str(directory).encode()))

    # ------------------------------------------------------------- diagnostics
    def energies(self):
        a = np.zeros(4)
        L.check(self._lib.pbpic_energies(self._h, L.ptr(a)))
        return a

    def energy_history(self):
        n = ctypes.c_int32()
        L.check(self._lib.pbpic_energy_history(self._h, None, 0, ctypes.byref(n)))
        a = np.zeros((n.value, 4))
        L.check(self._lib.pbpic_energy_history(self._h, L.ptr(a), n.value, ctypes.byref(n)))
        return a

    def itime(self):
        t = ctypes.c_int32()
        L.check(self._lib.pbpic_time_step(self._h, ctypes.byref(t)))
        return t.value

    def cell_counts(self):
        a = np.zeros(self.mx * self.my, dtype=np.int32)
        L.check(self._lib.pbpic_cell_counts(self._h, L.ptr(a)))
        return a

    def gauss_residual(self):
        v = ctypes.c_double()
        L.check(self._lib.pbpic_gauss_residual(self._h, ctypes.byref(v)))
        return v.value

    def reconnected_flux(self):
        v = ctypes.c_double()
        L.check(self._lib.pbpic_reconnected_flux(self._h, ctypes.byref(v)))
        return v.value

    def status(self):
        v = ctypes.c_int32()
        L.check(self._lib.pbpic_status(self._h, ctypes.byref(v)))
        return v.value


def counting_sort_keys(keys_ptr, n, ncells, perm_ptr, counts_ptr, stream_ptr=0):
    """Stateless stable counting sort on device buffers (raw pointers)."""
    lib = L.lib()
    L.check(lib.pbpic_counting_sort_keys(ctypes.c_void_p(keys_ptr), n, ncells, ctypes.c_void_p(perm_ptr),
                                         ctypes.c_void_p(counts_ptr), ctypes.c_void_p(stream_ptr)))


def kernel_launches():
    """Kernels launched by the library in this process so far."""
    n = ctypes.c_int64()
    L.check(L.lib().pbpic_kernel_launches(ctypes.byref(n)))
    return n.value
