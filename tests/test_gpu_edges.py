"""GPU edge cases against the CPU oracle: no particles at all, very dense cells
(a tile beyond the 32767 particles of the split 32-bit crossing sums, runs of
one cell across whole warps), very sparse cells (several cells inside one
thread's pass), crafted crossings (diagonal moves through cell corners, both x
edges, both walls, offsets exactly on a cell face) and the largest grids the
32-bit cell word encodes (mx = 32767, my = 65535).

Bars as in test_gpu_parity.py: FP64 plain bit-identical particle state and
current within 1e-12 of its maximum; FP32 mixed particles within 2e-5 and
current within 2e-4 of its maximum against the FP64 oracle started from the
same FP32 state; the fused sort's order equal to the oracle's stable sort."""
import numpy as np
import pytest

import pbpic_b200
from pbpic_b200 import configs
from test_gpu_parity import assert_particles, field_err, new_sim, plasma, random_fields

pytestmark = pytest.mark.gpu


def rows_of(cfg):
    return cfg["my"] if cfg["ybc"] == 0 else cfg["my"] + 1


def check_one_step(oracle_mod, cfg, p, yee, precision, jtol64=1e-12):
    """Sort, push and sort again (the push without its own sort, so that the
    pushed order is visible); compare the particles and the current with the
    oracle's step and the second sort with the stable sort of the pushed order."""
    with new_sim(cfg, max(len(p), 1), precision=precision, options=pbpic_b200.OPT_NO_AUTOSORT) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.countingsort()
        o = oracle_mod.Oracle(**cfg)
        if precision == "fp64":
            o.load_particles(p)
            o.set_fields(yee)
        else:  # the FP32 state of the input, so that only the step's arithmetic differs
            o.load_particles(s.particles())
            o.set_fields(s.fields())
        o.countingsort()
        assert np.array_equal(s.particles()["pid"], o.particles()["pid"])
        o.pusher()
        s.pusher()
        pre = s.particles()
        tol, jtol = (1e-12, jtol64) if precision == "fp64" else (2e-5, 2e-4)
        assert_particles(pre, o.particles(), tol)
        rows = rows_of(cfg)
        jg, jo = s.denjr()[:, :, :rows], o.current()[:, :, :rows]
        assert np.abs(jg - jo).max() <= jtol * max(np.abs(jo).max(), 1e-300)
        s.countingsort()  # the fused counting sort from the push's new-cell counts
        post = s.particles()
        order = np.argsort(pre["grid"], kind="stable")
        assert np.array_equal(post["pid"], pre["pid"][order])
        for c in ("grid", "dx", "dy", "ux", "uy", "uz"):
            assert np.array_equal(post[c], pre[c][order]), c
        assert np.array_equal(s.cell_counts(), np.bincount(pre["grid"] - 1, minlength=cfg["mx"] * cfg["my"]))
        assert s.status() & ~pbpic_b200.STATUS_UNSORTED == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("ybc", [0, 1])
def test_no_particles(gpu_lib, oracle_mod, precision, ybc):
    """An empty plasma steps its fields like the oracle; the kinetic energies are zero."""
    cfg, _, _, _ = plasma(oracle_mod, ybc, mx=16, my=12, ppc=1)
    yee = random_fields(cfg, 11)
    empty = np.zeros(0, dtype=oracle_mod.PARTICLE)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(empty)
    o.set_fields(yee)
    with new_sim(cfg, 1, precision=precision) as s:
        s.load_particles(empty)
        s.load_fields(yee)
        fin = s.fields()
        o32 = oracle_mod.Oracle(**cfg)
        o32.load_particles(empty)
        o32.set_fields(fin)
        for _ in range(3):
            o32.pusher()
            o32.fieldsolver()
            o32.countingsort()
        s.step(3, sort_every=1)
        fo = o32.fields()
        tol = 1e-12 if precision == "fp64" else 1e-5
        assert field_err(s.fields(), fo, cfg) <= tol * np.abs(fo).max()
        e = s.energies()
        assert e[0] == 0.0 and e[1] == 0.0
        assert np.allclose(e[2:], o32.energies()[2:], rtol=tol)
        assert len(s.particles()) == 0
        assert s.status() & ~pbpic_b200.STATUS_UNSORTED == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dense_cell(gpu_lib, oracle_mod, precision):
    """40,960 particles with 36,000 of them in two neighbouring cells of one
    tile: the mixed form takes the 64-bit crossing window (tile > 32767
    particles) and the run sums span whole warps of one cell."""
    cfg, _, p, _ = plasma(oracle_mod, 1, mx=8, my=8, ppc=320, vthe=0.3)
    p = p.copy()
    my = cfg["my"]
    dense = np.arange(len(p)) < 36000
    p["grid"][dense] = 3 * my + 4 + 1 + (np.arange(len(p))[dense] % 2)  # cells (3, 4) and (3, 5)
    yee = random_fields(cfg, 12)
    check_one_step(oracle_mod, cfg, p, yee, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("ybc", [0, 1])
def test_sparse_cells(gpu_lib, oracle_mod, precision, ybc):
    """One particle per cell and species on a 64 x 48 grid, fast electrons: a
    thread's 8 consecutive particles span several cells."""
    cfg, _, p, _ = plasma(oracle_mod, ybc, mx=64, my=48, ppc=1, vthe=0.6)
    yee = random_fields(cfg, 13)
    check_one_step(oracle_mod, cfg, p, yee, precision)


def crafted_particles(oracle_mod, cfg):
    """Particles near the four corners of corner and middle cells, moving
    diagonally out of them (each crosses a cell corner), plus particles with
    an offset exactly on the lower cell faces, at the domain's edges."""
    mx, my = cfg["mx"], cfg["my"]
    cells = [(0, 0), (mx - 1, 0), (0, my - 1), (mx - 1, my - 1), (mx // 2, my // 2), (0, my // 2), (mx - 1, 1)]
    recs = []
    for ix, iy in cells:
        for sx in (-1, 1):
            for sy in (-1, 1):
                for q in (1, -1):
                    recs.append((0.45 * sx, 0.45 * sy, 0.6 * sx, 0.6 * sy, 0.1 * q, ix * my + iy + 1, q))
        for q in (1, -1):
            recs.append((-0.5, -0.5, -0.3, -0.3, 0.0, ix * my + iy + 1, q))
            recs.append((-0.5, 0.2, 0.0, 0.0, 0.2, ix * my + iy + 1, q))
    p = np.zeros(len(recs), dtype=oracle_mod.PARTICLE)
    for k, r in enumerate(recs):
        p["dx"][k], p["dy"][k], p["ux"][k], p["uy"][k], p["uz"][k], p["grid"][k], p["q"][k] = r
    p["pid"] = np.arange(1, len(p) + 1)
    return p


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("ybc", [0, 1])
def test_crafted_crossings(gpu_lib, oracle_mod, precision, ybc):
    cfg, _, _, _ = plasma(oracle_mod, ybc, mx=12, my=10, ppc=1)
    p = crafted_particles(oracle_mod, cfg)
    yee = random_fields(cfg, 14, amp=0.02)
    check_one_step(oracle_mod, cfg, p, yee, precision)
    # every diagonal mover left its cell through the corner
    with new_sim(cfg, len(p), precision=precision) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.pusher()
        g = s.particles()
        g = g[np.argsort(g["pid"])]
        diag = np.abs(p["ux"]) == 0.6
        assert np.all(g["grid"][diag] != p["grid"][diag])


@pytest.mark.parametrize("mx,my", [(32767, 4), (3, 65535)])
def test_largest_grids(gpu_lib, oracle_mod, mx, my):
    """The widest and the tallest grid the cell word holds (15 bits of ix, 16
    of iy), conducting walls, one particle per cell and species, FP64.

    The reference's currentdeposit (pic2d.f90:1239-1252), which the oracle
    follows, forms the relay point from absolute cell indices (i1 + i2 + dx1 +
    dx2 + 1) / 2, so its rounding grows with the cell index: near index 32766
    it loses about 32766 ulp of a position, i.e. ~1e-11 of the current. The
    CUDA push works in cell-relative positions. The current is therefore
    compared within 8 ulp times the largest index (the particle state is still
    bit-identical)."""
    cfg, ld = configs.uniform_c1(mx=mx, my=my, ppc=1, seed=15)
    cfg["ybc"] = 1
    ld["vthe"], ld["vthi"] = 0.5, 0.1
    p, _ = oracle_mod.load_plasma(cfg, ld)
    yee = random_fields(cfg, 16, amp=0.02)
    check_one_step(oracle_mod, cfg, p, yee, "fp64", jtol64=8 * np.finfo(np.float64).eps * max(mx, my))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_readers_after_a_permuted_sort(gpu_lib, precision, tmp_path):
    """After steps that end with the sort's permutation (the particle data not
    moved), every reader sees the cell-sorted arrays: two identical runs, one
    read first through particles() and one through gauss_residual(), give the
    same particles (bit for bit in the mixed form; FP64 runs differ by the order
    of their atomic current sums, within 1e-12), spectra and cell counts, the
    same Gauss residual within 1e-12 absolute (its charge density is summed with
    FP64 atomics), and a dump of one restarts into the same state."""
    cfg, ld = configs.harris(48, 32, 12, seed=17)
    n = pbpic_b200.Simulation(**cfg, precision=precision, capacity=1).loader_count(**ld)
    out = []
    for first in ("particles", "gauss"):
        with pbpic_b200.Simulation(**cfg, precision=precision, capacity=n, track_pid=True) as s:
            s.init_plasma(**ld)
            s.step(2, sort_every=1)
            if first == "particles":
                p = s.particles()
                g = s.gauss_residual()
            else:
                g = s.gauss_residual()
                p = s.particles()
            out.append((p, g, s.energy_spectra(nbins=64), s.cell_counts()))
            if first == "gauss":
                s.dump(str(tmp_path / "d"))
                with pbpic_b200.Simulation(**cfg, precision=precision, capacity=n, track_pid=True) as r:
                    r.restart(str(tmp_path / "d"))
                    assert np.array_equal(r.particles(), p)
                    s.step(1, sort_every=1)
                    r.step(1, sort_every=1)
                    assert np.array_equal(r.particles(), s.particles())
    (pa, ga, sa, ca), (pb, gb, sb, cb) = out
    if precision == "fp32":  # bit-reproducible run to run
        assert np.array_equal(pa, pb)
    else:  # two FP64 runs differ by the order of their FP64 current sums
        assert_particles(pa, pb, 1e-12)
    assert np.all(np.diff(pa["grid"]) >= 0)  # cell order
    assert abs(ga - gb) <= 1e-12  # a small difference of O(1) terms, summed with FP64 atomics
    assert np.array_equal(sa, sb) and np.array_equal(ca, cb)
    assert np.array_equal(ca, np.bincount(pa["grid"] - 1, minlength=cfg["mx"] * cfg["my"]))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_handles_of_different_tile_heights(gpu_lib, precision):
    """Handles on one device whose tiles differ in height step in turn: the
    push's shared-memory size is a limit of the kernel function, which every
    handle shares (the plain form's exceeds the 48 KB a launch gets without
    opting in), so a handle with short tiles must not lower it below another's.
    The runs agree (FP64: within 1e-12, the order of the atomic current sums)."""
    cfg, ld = configs.harris(32, 80, 8, seed=3)
    n = pbpic_b200.Simulation(**cfg, precision=precision, capacity=1).loader_count(**ld)
    sims = [pbpic_b200.Simulation(**cfg, precision=precision, capacity=n, track_pid=True, tile_rows=ty)
            for ty in (64, 4, 16)]
    try:
        for s in sims:
            s.init_plasma(**ld)
        for _ in range(3):
            for s in sims:
                s.step(1, sort_every=1)
        ps = [s.particles() for s in sims]
        for p in ps[1:]:
            assert_particles(p, ps[0], 1e-12 if precision == "fp64" else 2e-5)
    finally:
        for s in sims:
            s.close()
