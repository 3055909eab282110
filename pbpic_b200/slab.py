"""y-slab decomposition: the reference's 1-D domain decomposition along y
(src/programs/pic2d.f90:206-212), one slab of cell rows per rank.

Each rank steps an *extended* domain: its own rows [y0, y1) of the global
grid plus ghost bands of G rows on each side copied from the neighbouring
slabs (no ghost band against a global conducting wall). The extended domain
uses the single-domain kernels unchanged, with its own outer edges closed by
a wrap (periodic global y) or a wall (conducting global y). What those fake
edges do to fields, currents and particles travels inward by at most three
rows per step (three field half-updates, one-cell particle moves and a
one-row deposit stencil) and stays inside the ghost bands, which are
refreshed every step:

  1. push and field solve on every slab;
  2. particles: each slab drops everything outside its own rows and receives
     its neighbours' particles within G rows of the boundary as ghosts (on the
     GPU one pass that writes the own rows and both bands in cell order). A
     particle that crosses a slab boundary was pushed, bit for bit, by both
     slabs (as an own particle on one side, a ghost on the other: same state,
     same fields); it now sits in the other slab's own rows and is kept
     there, so migration needs no separate message;
  3. fields: each slab receives its neighbours' G rows next to the boundary
     into its ghost rows (the reference's ghost-row exchange, pic2d.f90:701-835);
  4. counting sort.
The current needs no exchange: every particle that deposits into a slab's
own rows is pushed on that slab (as an own particle or a ghost). Energies sum
the own rows of every slab and the Gauss residual takes the largest over the
own rows, both reduced over the ranks by the transport (an all-reduce, as the
reference's MPI_Allreduce of its energy sums, pic2d.f90:653-673).

Transports: `InProcess` steps several slabs in one process (tests, or
several domains on one GPU); `TorchDist` exchanges over torch.distributed
between ranks, one slab per rank (NCCL between GPUs, gloo on CPU).
"""
import ctypes

import numpy as np

from . import _lib as L
from .sim import Simulation

GHOST = 4  # ghost rows per side: the fake edges disturb at most 3 rows per step


class Layout:
    """Rows of slab `rank` of `world` on a global grid of `my` rows."""

    def __init__(self, my, world, rank, ybc, ghost=GHOST):
        self.my, self.world, self.rank, self.ybc, self.g = my, world, rank, ybc, ghost
        self.y0, self.y1 = my * rank // world, my * (rank + 1) // world
        self.own = self.y1 - self.y0
        if self.own < ghost:
            raise ValueError(f"slab {rank} has {self.own} rows, fewer than the {ghost} ghost rows")
        walls = ybc == L.BC_CONDUCTING
        self.has_down = not (walls and rank == 0)
        self.has_up = not (walls and rank == world - 1)
        self.gl = ghost if self.has_down else 0
        self.gh = ghost if self.has_up else 0
        self.my_local = self.own + self.gl + self.gh
        self.lo, self.hi = self.gl, self.gl + self.own  # own local rows
        self.row_offset = self.y0 - self.gl  # global row of local row 0 (before the wrap)
        self.down = (rank - 1) % world
        self.up = (rank + 1) % world
        # offsets turning global rows of received bands into local ghost rows
        self.off_down = (self.y0 - self.gl) % my if self.has_down else 0
        self.off_up = (self.y1 % my) - (self.gl + self.own) if self.has_up else 0
        # node rows on global walls (weight 1/2 in the field energy)
        self.wall_lo = 0 if walls and rank == 0 else -1
        self.wall_hi = self.my_local if walls and rank == world - 1 else -1

    def energy_rows(self):
        hi = self.hi + (1 if self.wall_hi >= 0 else 0)  # the top wall's node row
        return self.lo, hi


class GpuEngine:
    """One slab on the GPU: a Simulation handle and device buffers for the bands."""

    def __init__(self, cfg, layout, precision, capacity, track_pid=False, tile_rows=0):
        import torch
        self.torch = torch
        self.lay = layout
        self.precision = precision
        c = dict(cfg, my=layout.my_local)
        self.sim = Simulation(**c, precision=precision, capacity=capacity, track_pid=track_pid, tile_rows=tile_rows)
        self.rec = L.PARTICLE_F32 if precision in ("fp32", "mixed") else L.PARTICLE_F64
        self.ftype = torch.float32 if precision in ("fp32", "mixed") else torch.float64
        self.lib = L.lib()
        self.bands = {}  # outgoing band buffers, one per direction, grown as needed

    # particles
    def extract(self, y_lo, y_hi, slot=0):
        """The particles of rows [y_lo, y_hi) as reference records in a device
        buffer kept for `slot` (one per direction), valid until the next
        extract into the same slot. A band holds a few rows' particles, so the
        buffer is sized from the band's own count (the library reports it when
        the buffer is too small) with a quarter to spare, not from the slab."""
        n = ctypes.c_int64()
        size = self.rec.itemsize
        buf = self.bands.get(slot)
        cap = 0 if buf is None else buf.numel() // size
        dst = ctypes.c_void_p(buf.data_ptr()) if cap else None
        rc = self.lib.pbpic_band_extract(self.sim.handle, y_lo, y_hi, self.lay.my, self.lay.row_offset, dst, cap,
                                         ctypes.byref(n))
        if rc == L.ERR_CAPACITY:
            cap = n.value + n.value // 4 + 256
            buf = self.torch.empty(cap * size, dtype=self.torch.uint8, device="cuda")
            self.bands[slot] = buf
            rc = self.lib.pbpic_band_extract(self.sim.handle, y_lo, y_hi, self.lay.my, self.lay.row_offset,
                                             ctypes.c_void_p(buf.data_ptr()), cap, ctypes.byref(n))
        L.check(rc)
        if n.value == 0:
            return self.empty_band()
        return buf[: n.value * size]

    def keep(self, y_lo, y_hi):
        L.check(self.lib.pbpic_band_keep(self.sim.handle, y_lo, y_hi))

    def replace(self, y_lo, y_hi, bottom, off_bottom, top, off_top):
        """Own rows plus both received bands, in cell order, in one pass."""
        n_b = 0 if bottom is None else bottom.numel() // self.rec.itemsize
        n_t = 0 if top is None else top.numel() // self.rec.itemsize
        p_b = ctypes.c_void_p(bottom.contiguous().data_ptr()) if n_b else None
        p_t = ctypes.c_void_p(top.contiguous().data_ptr()) if n_t else None
        L.check(self.lib.pbpic_band_replace(self.sim.handle, y_lo, y_hi, p_b, n_b, off_bottom, p_t, n_t, off_top,
                                            self.lay.my))

    def append(self, band, row_offset):
        n = band.numel() // self.rec.itemsize
        if n:
            band = band.contiguous()
            L.check(self.lib.pbpic_band_append(self.sim.handle, ctypes.c_void_p(band.data_ptr()), n, self.lay.my,
                                               row_offset))

    # fields
    def field_rows(self, j0, nrows):
        buf = self.torch.empty(6 * self.sim.mx * nrows, dtype=self.ftype, device="cuda")
        L.check(self.lib.pbpic_field_rows_get(self.sim.handle, j0, nrows, ctypes.c_void_p(buf.data_ptr())))
        return buf

    def set_field_rows(self, j0, nrows, buf):
        buf = buf.contiguous()
        L.check(self.lib.pbpic_field_rows_set(self.sim.handle, j0, nrows, ctypes.c_void_p(buf.data_ptr())))

    def empty_band(self):
        return self.torch.empty(0, dtype=self.torch.uint8, device="cuda")

    # step
    def push(self):
        self.sim.pusher()

    def fieldsolve(self):
        self.sim.fieldsolver()

    def sort(self):
        self.sim.countingsort()

    def energies(self):
        lo, hi = self.lay.energy_rows()
        out = np.zeros(4)
        L.check(self.lib.pbpic_energies_rows(self.sim.handle, lo, hi, self.lay.wall_lo, self.lay.wall_hi, L.ptr(out)))
        return out

    def gauss_residual(self):
        v = ctypes.c_double()
        L.check(self.lib.pbpic_gauss_residual_rows(self.sim.handle, self.lay.lo, self.lay.hi, ctypes.byref(v)))
        return v.value

    def own_count(self):
        """Particles in the slab's own rows (ghosts excluded)."""
        c = self.sim.cell_counts().reshape(self.sim.mx, self.lay.my_local)
        return int(c[:, self.lay.lo:self.lay.hi].sum())


class InProcess:
    """All slabs in this process; an exchange hands each band to its neighbour."""

    def allreduce(self, values, op):
        """Every slab is here: the process's own reduction is the whole one."""
        return np.asarray(values, dtype=np.float64)

    def exchange(self, slabs, outgoing):
        """outgoing[r] = (to_down, to_up); returns incoming[r] = (from_down, from_up)."""
        incoming = {}
        for r, s in slabs.items():
            lay = s.lay
            from_down = outgoing[lay.down][1] if lay.has_down else None
            from_up = outgoing[lay.up][0] if lay.has_up else None
            incoming[r] = (from_down, from_up)
        return incoming


class TorchDist:
    """One slab per rank over torch.distributed: sizes first, then payloads.
    Between two ranks that are each other's upper and lower neighbour (two
    periodic slabs) point-to-point messages match in posting order, so every
    rank posts its sends as (up, down) and its receives as (down, up)."""

    def __init__(self, dist, device):
        self.dist, self.device = dist, device

    def allreduce(self, values, op):
        """values (float64) reduced over the ranks with op "sum" or "max"."""
        import torch
        t = torch.tensor(np.asarray(values, dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM if op == "sum" else self.dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def _sendrecv(self, lay, sends, recvs):
        ops = []
        for buf, peer in sends:
            if buf.numel():
                ops.append(self.dist.P2POp(self.dist.isend, buf, peer))
        for buf, peer in recvs:
            if buf.numel():
                ops.append(self.dist.P2POp(self.dist.irecv, buf, peer))
        if ops:
            for q in self.dist.batch_isend_irecv(ops):
                q.wait()

    def exchange(self, slabs, outgoing):
        import torch
        (r, s), = slabs.items()
        lay = s.lay
        to_down, to_up = outgoing[r]
        if not (lay.has_down or lay.has_up):
            return {r: (None, None)}
        dtype = (to_down if to_down is not None else to_up).dtype
        i64 = dict(dtype=torch.int64, device=self.device)
        n_up = torch.tensor([to_up.numel() if lay.has_up else 0], **i64)
        n_down = torch.tensor([to_down.numel() if lay.has_down else 0], **i64)
        m_down, m_up = torch.zeros(1, **i64), torch.zeros(1, **i64)
        sends, recvs = [], []
        if lay.has_up:
            sends.append((n_up, lay.up))
        if lay.has_down:
            sends.append((n_down, lay.down))
            recvs.append((m_down, lay.down))
        if lay.has_up:
            recvs.append((m_up, lay.up))
        self._sendrecv(lay, sends, recvs)
        from_down = torch.empty(int(m_down.item()), dtype=dtype, device=self.device) if lay.has_down else None
        from_up = torch.empty(int(m_up.item()), dtype=dtype, device=self.device) if lay.has_up else None
        sends, recvs = [], []
        if lay.has_up:
            sends.append((to_up.contiguous(), lay.up))
        if lay.has_down:
            sends.append((to_down.contiguous(), lay.down))
            recvs.append((from_down, lay.down))
        if lay.has_up:
            recvs.append((from_up, lay.up))
        self._sendrecv(lay, sends, recvs)
        return {r: (from_down, from_up)}


class SlabRun:
    """Steps the slabs held by this process (a dict rank -> engine)."""

    def __init__(self, slabs, transport):
        self.slabs = slabs
        self.t = transport

    def exchange(self):
        # particles: own bands next to the neighbours, then keep the own rows
        out = {}
        for r, e in self.slabs.items():
            lay = e.lay
            to_down = e.extract(lay.lo, lay.lo + lay.g, 0) if lay.has_down else None
            to_up = e.extract(lay.hi - lay.g, lay.hi, 1) if lay.has_up else None
            out[r] = (to_down, to_up)
        inc = self.t.exchange(self.slabs, out)
        for r, e in self.slabs.items():
            lay = e.lay
            if not (lay.has_down or lay.has_up):
                continue  # a slab with no neighbours (one slab between walls) has no ghost rows
            from_down, from_up = inc[r]
            e.replace(lay.lo, lay.hi, from_down, lay.off_down, from_up, lay.off_up)
        # fields: own rows next to the neighbours into their ghost rows
        out = {}
        for r, e in self.slabs.items():
            lay = e.lay
            to_down = e.field_rows(lay.lo, lay.g) if lay.has_down else None
            to_up = e.field_rows(lay.hi - lay.g, lay.g) if lay.has_up else None
            out[r] = (to_down, to_up)
        inc = self.t.exchange(self.slabs, out)
        for r, e in self.slabs.items():
            lay = e.lay
            from_down, from_up = inc[r]
            if from_down is not None:
                e.set_field_rows(0, lay.gl, from_down)
            if from_up is not None:
                e.set_field_rows(lay.hi, lay.gh, from_up)

    def energies(self):
        """Electron KE, ion KE, E and B energy of the whole domain (every rank
        calls it: an all-reduce)."""
        local = np.zeros(4)
        for e in self.slabs.values():
            local += e.energies()
        return self.t.allreduce(local, "sum")

    def gauss_residual(self):
        """Largest Gauss's-law residual over the own rows of every slab (every
        rank calls it: an all-reduce)."""
        local = max(e.gauss_residual() for e in self.slabs.values())
        return float(self.t.allreduce([local], "max")[0])

    def start(self):
        """Fill the ghost bands of freshly loaded slabs and sort."""
        for e in self.slabs.values():
            e.sort()  # bands leave in cell order
        self.exchange()
        for e in self.slabs.values():
            e.sort()

    def step(self, nsteps=1):
        for _ in range(nsteps):
            for e in self.slabs.values():
                e.push()
                e.fieldsolve()
            self.exchange()
            for e in self.slabs.values():
                e.sort()


def scatter_plasma(particles, yee, lay):
    """The own part of a global plasma for slab `lay`: the particles (reference
    records of the global grid) in its own rows with grid renumbered to the
    extended domain, and Yee planes (6, mx, my_local+1) holding the own rows
    (and, against a global top wall, the wall's node row). The ghost bands are
    filled by a first exchange (SlabRun.start)."""
    my, myl = lay.my, lay.my_local
    g = particles["grid"].astype(np.int64) - 1
    ix, gy = g // my, g % my
    keep = (gy >= lay.y0) & (gy < lay.y1)
    p = particles[keep].copy()
    p["grid"] = (ix[keep] * myl + (gy[keep] - lay.y0 + lay.gl) + 1).astype(np.int32)
    f = np.zeros((6, yee.shape[1], myl + 1))
    f[:, :, lay.lo:lay.hi] = yee[:, :, lay.y0:lay.y1]
    if lay.ybc == L.BC_CONDUCTING and lay.rank == lay.world - 1:
        f[:, :, myl] = yee[:, :, my]
    return p, f
