"""Diagnostics around the step: energy spectra (energyspectra,
pic2d.f90:1957-1990) against a numpy statement on the same particles, exact;
field cuts (dispersioninfo, pic2d.f90:2124-2142) against the node grid."""
import numpy as np
import pytest

from pbpic_b200 import configs

pytestmark = pytest.mark.gpu


def spectra_numpy(p, mime, de_e, de_i, nbins):
    g = np.sqrt(1.0 + p["ux"] * p["ux"] + p["uy"] * p["uy"] + p["uz"] * p["uz"])
    out = np.zeros((2, nbins), dtype=np.int64)
    for sp, q, ms, de in ((0, -1, 1.0, de_e), (1, 1, mime, de_i)):
        ene = (g[p["q"] == q] - 1.0) * ms
        ene = ene[ene < de * nbins]
        k = np.clip(np.ceil(ene / de).astype(np.int64), 1, nbins)
        np.add.at(out[sp], k - 1, 1)
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_energy_spectra_match_numpy(gpu_lib, precision):
    from pbpic_b200.sim import Simulation
    cfg, ld = configs.uniform_c1(seed=8, mx=32, my=16, ppc=16)
    ld = dict(ld, vthe=0.3, vthi=0.1)
    with Simulation(**cfg, precision=precision, capacity=2 * 16 * 32 * 16) as s:
        s.init_plasma(**ld)
        s.step(2, sort_every=1)
        p = s.particles()
        for de_e, de_i, nb in ((0.005, 0.005, 1000), (0.002, 0.05, 37), (1.0, 1.0, 1)):
            got = s.energy_spectra(de_e, de_i, nb)
            want = spectra_numpy(p, cfg["mime"], de_e, de_i, nb)
            assert np.array_equal(got, want), (de_e, de_i, nb)
        assert s.energy_spectra(1.0, 1.0, 1).sum() <= len(p)
        assert s.energy_spectra(10.0, 100.0, 10).sum() == len(p)


def test_field_cuts_match_node_grid(gpu_lib):
    from pbpic_b200.sim import Simulation
    cfg, ld = configs.harris(32, 16, 4, seed=9)
    with Simulation(**cfg, precision="fp32", capacity=2 * 4 * 32 * 16) as s:
        s.init_plasma(**ld)
        s.step(3, sort_every=1)
        g = s.emfgrid()  # (mx+1, my+1, 8)
        comps = [0, 1, 2, 4, 5, 6]
        rows, cols = [0, 7, 16], [3, 32]
        xr, yc = s.field_cuts(rows, cols)
        for a, j in enumerate(rows):
            assert np.array_equal(xr[a], g[:32, j][:, comps])
        for a, i in enumerate(cols):
            assert np.array_equal(yc[a], g[i, :16][:, comps])
        dr, dc = s.field_cuts()  # the reference's default diagnostic indices
        assert dr.shape == (2, 32, 6) and dc.shape == (2, 16, 6)
