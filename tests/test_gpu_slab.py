"""The y-slab decomposition against the single-domain run of the same
plasma: W slabs (W = 1, 2, 3, stepped in one process on one GPU, exchanging
their ghost bands between steps) reproduce the single domain's particles
(matched by id), fields and energies. FP64 plain: within 1e-12 relative (the
order of the FP64 current sums differs); FP32 mixed: within FP32 rounding. The
slab run's energies and Gauss residual (reduced over the slabs) give the
single domain's."""
import numpy as np
import pytest

from pbpic_b200 import _lib as L
from pbpic_b200 import configs

pytestmark = pytest.mark.gpu


def global_case(kind):
    if kind == "uniform":
        cfg, ld = configs.uniform_c1(seed=21, mx=24, my=30, ppc=4)
        ld = dict(ld, vthe=0.3, vthi=0.1)
        return cfg, ld
    return configs.harris(24, 30, 4, seed=22)


def run_single(cfg, ld, precision, steps):
    from pbpic_b200.sim import Simulation
    n = 2 * ld["ppc"] * cfg["mx"] * cfg["my"]
    s = Simulation(**cfg, precision=precision, capacity=n, track_pid=True)
    s.init_plasma(**ld)
    p0, f0 = s.particles(), s.fields()
    for _ in range(steps):
        s.pusher()
        s.fieldsolver()
        s.countingsort()
    return s, p0, f0


def run_slabs(cfg, p0, f0, precision, world, steps):
    from pbpic_b200.slab import GpuEngine, InProcess, Layout, SlabRun, scatter_plasma
    slabs = {}
    for r in range(world):
        lay = Layout(cfg["my"], world, r, cfg["ybc"])
        e = GpuEngine(cfg, lay, precision, capacity=2 * len(p0), track_pid=True)  # own rows + ghost bands
        p, f = scatter_plasma(p0, f0, lay)
        e.sim.load_particles(p)
        e.sim.load_fields(f)
        slabs[r] = e
    run = SlabRun(slabs, InProcess())
    run.start()
    run.step(steps)
    return slabs, run


@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("kind", ["uniform", "harris"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slabs_match_single_domain(gpu_lib, kind, world, precision):
    cfg, ld = global_case(kind)
    steps = 5
    single, p0, f0 = run_single(cfg, ld, precision, steps)
    slabs, run = run_slabs(cfg, p0, f0, precision, world, steps)
    ps = single.particles()
    n_own = 0
    for e in slabs.values():
        g = e.sim.particles()["grid"].astype(np.int64) - 1
        iy = g % e.lay.my_local
        n_own += int(((iy >= e.lay.lo) & (iy < e.lay.hi)).sum())
    assert n_own == len(ps)  # every particle in exactly one slab's own rows
    own = []
    for e in slabs.values():
        p = e.sim.particles()
        g = p["grid"].astype(np.int64) - 1
        ix, iy = g // e.lay.my_local, g % e.lay.my_local
        m = (iy >= e.lay.lo) & (iy < e.lay.hi)
        q = p[m].copy()
        q["grid"] = (ix[m] * cfg["my"] + iy[m] - e.lay.gl + e.lay.y0 + 1).astype(np.int32)
        own.append(q)
    pg = np.concatenate(own)
    pg, ps = pg[np.argsort(pg["pid"])], ps[np.argsort(ps["pid"])]
    assert np.array_equal(pg["pid"], ps["pid"])
    tol = 1e-12 if precision == "fp64" else 2e-5
    bad = pg["grid"] != ps["grid"]
    assert bad.sum() <= (0 if precision == "fp64" else 2)
    for c in ("dx", "dy", "ux", "uy", "uz"):
        d = np.abs(pg[c][~bad] - ps[c][~bad]).max()
        assert d <= tol * max(1.0, np.abs(ps[c]).max()), (c, d)
    fs = single.fields()
    fg = np.zeros_like(fs)
    my = cfg["my"]
    for e in slabs.values():
        lay = e.lay
        fl = e.sim.fields()
        fg[:, :, lay.y0:lay.y1] = fl[:, :, lay.lo:lay.hi]
        if lay.wall_hi >= 0:
            fg[:, :, my] = fl[:, :, lay.my_local]
    rows = my + 1 if cfg["ybc"] == L.BC_CONDUCTING else my
    ftol = 1e-12 if precision == "fp64" else 1e-5
    assert np.abs(fg[:, :, :rows] - fs[:, :, :rows]).max() <= ftol * np.abs(fs).max()
    es = single.energies()
    eg = sum(e.energies() for e in slabs.values())
    etol = 1e-11 if precision == "fp64" else 1e-5
    assert np.allclose(eg, es, rtol=etol, atol=etol * np.abs(es).max())
    assert np.array_equal(run.energies(), eg)  # the slab run's reduction over its slabs
    # Gauss's law over the own rows of every slab: the single domain's residual
    gs, gg = single.gauss_residual(), run.gauss_residual()
    if precision == "fp64":
        assert abs(gg - gs) <= 1e-12
    else:
        assert max(gg, gs) <= 1e-5


@pytest.mark.parametrize("kind", ["uniform", "harris"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_field_rows_set_refreshes_the_rows_it_feeds(gpu_lib, kind, precision):
    """Setting field rows recomputes only the node averages and gather records
    those rows feed: a handle loaded with other values in the rows, then set
    to the reference fields there, has the reference handle's node averages
    bit for bit, and one push of the same plasma gives the same particles
    (the mixed form gathers from the records). Rows at the bottom edge, the
    top edge and inside, periodic y and walls."""
    import ctypes

    import torch

    from pbpic_b200.sim import Simulation
    cfg, ld = global_case(kind)
    mx, my = cfg["mx"], cfg["my"]
    n = 2 * ld["ppc"] * mx * my
    ref = Simulation(**cfg, precision=precision, capacity=n)
    ref.init_plasma(**ld)
    f = ref.fields()
    top = my + 1 if cfg["ybc"] == L.BC_CONDUCTING else my  # rows of the field planes the API addresses
    ftype = torch.float64 if precision == "fp64" else torch.float32
    lib = L.lib()
    for j0, nrows in [(0, 4), (top - 4, 4), (12, 3)]:
        g = f.copy()
        rng = np.random.default_rng(j0)
        g[:, :, j0:j0 + nrows] += rng.normal(size=(6, mx, nrows))
        s = Simulation(**cfg, precision=precision, capacity=n)
        s.init_plasma(**ld)
        s.load_fields(g)
        buf = torch.empty(6 * mx * nrows, dtype=ftype, device="cuda")
        L.check(lib.pbpic_field_rows_get(ref.handle, j0, nrows, ctypes.c_void_p(buf.data_ptr())))
        L.check(lib.pbpic_field_rows_set(s.handle, j0, nrows, ctypes.c_void_p(buf.data_ptr())))
        torch.cuda.synchronize()
        assert np.array_equal(s.fields(), f), (j0, nrows)
        assert np.array_equal(s.emfgrid(), ref.emfgrid()), (j0, nrows)
        s.pusher()
        ref2 = Simulation(**cfg, precision=precision, capacity=n)
        ref2.init_plasma(**ld)
        ref2.pusher()
        a, b = s.particles(), ref2.particles()
        for c in ("grid", "dx", "dy", "ux", "uy", "uz"):
            assert np.array_equal(a[c], b[c]), (j0, nrows, c)
        s.close()
        ref2.close()
    ref.close()
