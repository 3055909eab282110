"""Dump and restart: a run dumped right after a counting sort and continued
from the dump in a new handle matches the run that went on without stopping
(particles, fields, energy history), for both y boundaries: bit for bit in
the FP32 mixed form (its fixed-point current does not depend on the order of
the atomics), within 1e-12 relative in the FP64 plain form (its FP64 atomic
sums round in the order the atomics land). The dump files are plain .npy
arrays named like the datasets of the reference's particle and field dumps."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def case(kind):
    from pbpic_b200 import configs
    if kind == "uniform":
        return configs.uniform_c1(seed=5, mx=32, my=16, ppc=8)
    return configs.harris(32, 16, 8, seed=6)


def new_sim(cfg, ld, precision):
    from pbpic_b200.sim import Simulation
    return Simulation.from_config(cfg, precision=precision, track_pid=True,
                                  capacity=2 * ld["ppc"] * cfg["mx"] * cfg["my"])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("kind", ["uniform", "harris"])
def test_restart_continues_bit_for_bit(gpu_lib, tmp_path, precision, kind):
    cfg, ld = case(kind)
    d = tmp_path / "dump"
    with new_sim(cfg, ld, precision) as a:
        a.init_plasma(**ld)
        a.step(4, sort_every=1)
        a.dump(d)
        n = a.num_particles()
        a.step(3, sort_every=1)
        pa, fa, ha = a.particles(), a.fields(), a.energy_history()
    with new_sim(cfg, ld, precision) as b:
        b.restart(d)
        assert b.itime() == 4
        b.step(3, sort_every=1)
        pb, fb, hb = b.particles(), b.fields(), b.energy_history()
    assert np.array_equal(pa["grid"], pb["grid"]) and np.array_equal(pa["pid"], pb["pid"])
    if precision == "fp32":
        for k in ("dx", "dy", "ux", "uy", "uz"):
            assert np.array_equal(pa[k], pb[k]), k
        assert np.array_equal(fa, fb)
        assert np.array_equal(ha, hb)
    else:
        for k in ("dx", "dy", "ux", "uy", "uz"):
            assert np.abs(pa[k] - pb[k]).max() <= 1e-12 * np.abs(pa[k]).max(), k
        assert np.abs(fa - fb).max() <= 1e-12 * np.abs(fa).max()
        assert np.allclose(ha, hb, rtol=1e-12, atol=0)
    # the files
    dt = np.float32 if precision == "fp32" else np.float64
    dx = np.load(d / "particles" / "dx.npy")
    assert dx.dtype == dt and dx.shape == (n,)
    assert np.load(d / "particles" / "grid.npy").dtype == np.int32
    assert np.load(d / "fields" / "ex.npy").shape == (cfg["mx"], cfg["my"] + 1)
    assert np.load(d / "fields" / "rho.npy").dtype == np.float64
    assert np.load(d / "totene.npy").shape == (5, 4)
    st = json.load(open(d / "state.json"))
    assert st["itime"] == 4 and st["particles"] == n and st["mx"] == cfg["mx"]


def test_restart_rejects_another_grid(gpu_lib, tmp_path):
    import pbpic_b200
    cfg, ld = case("uniform")
    with new_sim(cfg, ld, "fp32") as a:
        a.init_plasma(**ld)
        a.dump(tmp_path / "d")
    other = dict(cfg, mx=cfg["mx"] + 2)
    with new_sim(other, ld, "fp32") as b:
        with pytest.raises(pbpic_b200.PbpicError) as e:
            b.restart(tmp_path / "d")
        assert "differ" in str(e.value)
    with new_sim(cfg, ld, "fp64") as c:
        with pytest.raises(pbpic_b200.PbpicError):
            c.restart(tmp_path / "d")


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("kind", ["uniform", "harris"])
def test_hdf5_dumps_hold_the_state(gpu_lib, tmp_path, precision, kind):
    """pbpic_dump_h5 writes the reference's HDF5 files: particles.h5 (the
    particle records, zeros up to the capacity, nptlact), fields%05d.h5 (E, B,
    J, rho, div E and the particles per cell over the reference's index range
    (0:mx+1, 1:my+1), as float32 / int32), spectra.h5 (a group per call) and
    energy_tot.h5; read back with the test reader of the file format."""
    from h5_reader import read

    from pbpic_b200 import PARTICLE_F32
    cfg, ld = case(kind)
    mx, my = cfg["mx"], cfg["my"]
    d = tmp_path / "h5"
    with new_sim(cfg, ld, precision) as s:
        s.init_plasma(**ld)
        s.step(2, sort_every=1)
        s.dump_h5(d, nbins=200)
        s.step(3, sort_every=1)
        s.dump_h5(d, nbins=200)
        p32 = s.particles(PARTICLE_F32)
        yee, jj, n = s.fields(), s.denjr(), s.num_particles()
        hist, counts = s.energy_history(), s.cell_counts()
        spect = s.energy_spectra(nbins=200)
        cap = 2 * ld["ppc"] * mx * my
    pf = read(str(d / "particles.h5"))
    assert int(pf["nptlact"][0]) == n
    for c in ("dx", "dy", "ux", "uy", "uz", "grid", "q", "pid"):
        assert pf[c].shape == (cap,)
        assert np.array_equal(pf[c][:n], p32[c]), c
        assert not pf[c][n:].any()
    ff = read(str(d / "fields00005.h5"))
    assert (d / "fields00002.h5").exists()
    ix = (np.arange(mx + 2) - 1) % mx  # reference column 0..mx+1 -> 0-based column
    iy = np.arange(my + 1)             # reference row 1..my+1 -> 0-based row
    if cfg["ybc"] == 0:
        iy[my] = 0
    for k, c in enumerate(("ex", "ey", "ez", "bx", "by", "bz")):
        want = yee[k][ix][:, iy].T.astype(np.float32)
        assert ff[c].shape == (my + 1, mx + 2) and np.array_equal(ff[c], want), c
    for k, c in enumerate(("jx", "jy", "jz", "rho")):
        assert np.array_equal(ff[c], jj[k][ix][:, iy].T.astype(np.float32)), c
    num = np.zeros((my + 1, mx + 2), dtype=np.int32)
    num[:my, 1:mx + 1] = counts.reshape(mx, my).T
    assert np.array_equal(ff["num"], num)
    assert ff["dive"].dtype == np.float32 and ff["dive"].shape == (my + 1, mx + 2)
    sf = read(str(d / "spectra.h5"))
    assert sorted(sf) == ["00002", "00005", "ebins"]
    assert np.array_equal(sf["00005"]["spectra"], spect.T.astype(np.int32))
    assert np.allclose(sf["ebins"][:, 0], 0.005 * np.arange(1, 201), rtol=1e-6)
    tf = read(str(d / "energy_tot.h5"))
    assert np.array_equal(tf["tote"], hist.astype(np.float32))
