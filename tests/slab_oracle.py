"""A slab engine over the CPU oracle (test infrastructure): the same
interface as pbpic_b200.slab.GpuEngine, with host arrays, so the slab driver
and its torch.distributed transport can run as gloo ranks without a GPU."""
import numpy as np
import torch

from pbpic_b200 import _lib as L


class OracleEngine:
    def __init__(self, O, cfg, lay):
        self.O = O
        self.lay = lay
        self.cfg = dict(cfg, my=lay.my_local)
        self.o = O.Oracle(**self.cfg)
        self.mx = cfg["mx"]

    def load(self, p, f):
        self.o.load_particles(p, capacity=4 * len(p) + 64)
        self.o.set_fields(f)

    def _rows(self, p):
        g = p["grid"].astype(np.int64) - 1
        return g // self.lay.my_local, g % self.lay.my_local

    def extract(self, y_lo, y_hi, slot=0):
        p = self.o.particles()
        ix, iy = self._rows(p)
        m = (iy >= y_lo) & (iy < y_hi)
        q = p[m].copy()
        q["grid"] = (ix[m] * self.lay.my + iy[m] + self.lay.row_offset + 1).astype(np.int32)
        return torch.from_numpy(q.view(np.uint8).copy())

    def keep(self, y_lo, y_hi):
        p = self.o.particles()
        _, iy = self._rows(p)
        self.o.load_particles(p[(iy >= y_lo) & (iy < y_hi)], capacity=4 * len(p) + 64)

    def replace(self, y_lo, y_hi, bottom, off_bottom, top, off_top):
        self.keep(y_lo, y_hi)
        if bottom is not None:
            self.append(bottom, off_bottom)
        if top is not None:
            self.append(top, off_top)

    def append(self, band, row_offset):
        q = band.numpy().view(self.O.PARTICLE).copy()
        if len(q) == 0:
            return
        g = q["grid"].astype(np.int64) - 1
        ix, gy = g // self.lay.my, g % self.lay.my
        iy = gy - row_offset
        assert ((iy >= 0) & (iy < self.lay.my_local)).all()
        q["grid"] = (ix * self.lay.my_local + iy + 1).astype(np.int32)
        p = np.concatenate([self.o.particles(), q])
        self.o.load_particles(p, capacity=4 * len(p) + 64)

    def field_rows(self, j0, nrows):
        f = self.o.fields()[:, :, j0:j0 + nrows]
        return torch.from_numpy(np.ascontiguousarray(f).reshape(-1).copy())

    def set_field_rows(self, j0, nrows, buf):
        f = self.o.fields()
        f[:, :, j0:j0 + nrows] = buf.numpy().reshape(6, self.mx, nrows)
        self.o.set_fields(f)

    def push(self):
        self.o.pusher()

    def fieldsolve(self):
        self.o.fieldsolver()

    def sort(self):
        self.o.countingsort()

    def gauss_residual(self):
        """max |div E / cva^2 - in0 rho| over the slab's own node rows (walls:
        interior rows), rho the bilinear charge of the particles -- the
        definition of pbpic_gauss_residual_rows."""
        c = self.cfg
        mx, my = self.mx, self.lay.my_local
        p = self.o.particles()
        g = p["grid"].astype(np.int64) - 1
        ix, iy = g // my, g % my
        ax, ay = 0.5 + p["dx"], 0.5 + p["dy"]
        q = p["q"].astype(np.float64)
        rho = np.zeros((mx, my + 1))
        ip = (ix + 1) % mx
        jp = iy + 1
        if c["ybc"] == 0:
            jp = np.where(jp == my, 0, jp)
        for xi, yj, w in ((ix, iy, (1 - ax) * (1 - ay)), (ip, iy, ax * (1 - ay)), (ix, jp, (1 - ax) * ay),
                          (ip, jp, ax * ay)):
            np.add.at(rho, (xi, yj), q * w)
        f = self.o.fields()
        ex, ey = f[0], f[1]
        j0 = max(self.lay.lo, 0 if c["ybc"] == 0 else 1)
        j1 = min(self.lay.hi, my)
        j = np.arange(j0, j1)
        dive = (ex[:, j] - np.roll(ex, 1, axis=0)[:, j]) / c["dx"] + (ey[:, j] - ey[:, (j - 1) % my]) / c["dy"]
        return float(np.abs(dive / c["cva"] ** 2 - c["in0"] * rho[:, j]).max()) if len(j) else 0.0

    def own_count(self):
        return len(self.own_particles())

    def own_particles(self):
        p = self.o.particles()
        ix, iy = self._rows(p)
        m = (iy >= self.lay.lo) & (iy < self.lay.hi)
        q = p[m].copy()
        q["grid"] = (ix[m] * self.lay.my + iy[m] - self.lay.gl + self.lay.y0 + 1).astype(np.int32)
        return q

    def energies(self):
        """Electron KE, ion KE, E and B energy of the own rows, summed as the
        oracle sums them (kinetic energy pic2d.f90:1055-1062 from the particles'
        momenta, fieldsenergy pic2d.f90:653-673 over the own node rows with the
        trapezoid weight 1/2 on global wall rows)."""
        q = self.own_particles()
        gm1 = np.sqrt(1.0 + q["ux"] ** 2 + q["uy"] ** 2 + q["uz"] ** 2) - 1.0
        mime, cva2, in0 = self.cfg["mime"], self.cfg["cva"] ** 2, self.cfg["in0"]
        lo, hi = self.lay.energy_rows()
        g = self.o.emfgrid()[:self.mx, lo:hi]
        w = np.ones(hi - lo)
        for r in (self.lay.wall_lo, self.lay.wall_hi):
            if r >= 0 and lo <= r < hi:
                w[r - lo] = 0.5
        se = float(((g[..., 0] ** 2 + g[..., 1] ** 2 + g[..., 2] ** 2) * w).sum())
        sb = float(((g[..., 4] ** 2 + g[..., 5] ** 2 + g[..., 6] ** 2) * w).sum())
        return np.array([gm1[q["q"] == -1].sum(), mime * gm1[q["q"] == 1].sum(),
                         0.5 * se * mime / (cva2 * cva2 * in0), 0.5 * sb * mime / (cva2 * in0)])

    def own_fields(self):
        f = self.o.fields()
        out = f[:, :, self.lay.lo:self.lay.hi]
        return out, (f[:, :, self.lay.my_local] if self.lay.wall_hi >= 0 else None)
