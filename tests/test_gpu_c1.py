"""The uniform periodic plasma at its full size against the oracle.

Workload: 128x128 cells, dx = dy = 0.05 d_e, CFL 0.5, 32 particles per cell per
species (1,048,576 particles), mi/me = 25, Ti = Te, electron thermal speed
0.1 c, uniform Bz with wpe/wce = 2, seed 0 (configs.uniform_c1 with its
defaults). The reference loop is pic2d.f90:171-188: pusher, fieldsolver and
countingsort every 50 steps (pic2d.f90:180-182).

Bars (FP64 plain form):
- after loading: the stable counting sort (pic2d.f90:1303-1329) gives the same
  permutation and per-cell counts, bit for bit;
- after step 1: particles keyed by pid, the Yee fields, the node averages
  (emfgrid) and the folded current (denjr) within 1e-12 relative; the step's
  sort is the stable counting sort of the step's input order by the new cells
  (same permutation and counts, bit for bit);
- over 500 steps with the reference's sort cadence: the energy history within
  the bound stated in HISTORY_TOL.

The oracle's pusher moves the particles that wrap in y to the end of the array
(the 1-rank exchange, pic2d.f90:1072-1146) while the GPU keeps them in place,
so the arrays after step 1 are compared in the GPU's order: the oracle's
counting sort applied to the oracle's pushed particles arranged in the step's
input order.
"""
import numpy as np
import pytest

import pbpic_b200
from pbpic_b200 import configs

pytestmark = pytest.mark.gpu

COMPS = ("dx", "dy", "ux", "uy", "uz")
# Largest difference of each energy (field E, field B, kinetic e, kinetic i)
# between the GPU and the oracle over 500 steps, relative to the total energy.
# Both are FP64 but add the current in different orders (the GPU's atomics
# land in any order, the oracle's OpenMP threads fold private arrays), so the
# two histories part by rounding. Two orderings of the oracle itself (serial
# and OpenMP) part by at most 5.3e-15 over these 500 steps (measured on the
# CPU); the bound leaves a factor of about 200 for the GPU's order.
HISTORY_TOL = 1e-12


def by_pid(a):
    return a[np.argsort(a["pid"], kind="stable")]


@pytest.fixture(scope="module")
def c1(oracle_mod):
    cfg, ld = configs.uniform_c1()
    assert (cfg["mx"], cfg["my"], ld["ppc"], ld["seed"]) == (128, 128, 32, 0)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    assert len(p) == 2 * 32 * 128 * 128
    return cfg, ld, p, yee


def test_c1_sort_and_step1_match_oracle(gpu_lib, oracle_mod, c1):
    cfg, ld, p, yee = c1
    n = len(p)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    counts0 = o.countingsort()
    with pbpic_b200.Simulation(**cfg, precision="fp64", track_pid=True, capacity=n) as s:
        s.init_plasma(**ld)
        # the loader's plasma, sorted: same permutation and counts
        g0 = s.particles()
        o0 = o.particles()
        assert np.array_equal(g0["pid"], o0["pid"])
        assert np.array_equal(g0["grid"], o0["grid"])
        assert np.array_equal(s.cell_counts(), counts0)
        for c in COMPS:
            assert np.array_equal(g0[c], o0[c]), c
        assert np.array_equal(s.fields(), o.fields())

        # step 1: push + field solve
        o.pusher()
        o.fieldsolver()
        s.pusher()
        s.fieldsolver()
        g1, o1 = s.particles(), o.particles()
        gp, op = by_pid(g1), by_pid(o1)
        assert np.array_equal(gp["pid"], op["pid"])
        assert np.array_equal(gp["grid"], op["grid"])
        for c in COMPS:
            err = np.abs(gp[c] - op[c]).max() / max(1.0, np.abs(op[c]).max())
            assert err <= 1e-12, (c, err)
        jg, jo = s.denjr(), o.current()
        my = cfg["my"]
        assert np.abs(jg[:, :, :my] - jo[:, :, :my]).max() <= 1e-12 * np.abs(jo[:, :, :my]).max()
        fg, fo = s.fields(), o.fields()
        assert np.abs(fg[:, :, :my] - fo[:, :, :my]).max() <= 1e-12 * np.abs(fo[:, :, :my]).max()
        eg, eo = s.emfgrid(), o.emfgrid()
        assert np.abs(eg - eo).max() <= 1e-12 * np.abs(eo).max()
        assert np.allclose(s.energies(), o.energies(), rtol=1e-12, atol=0)

        # the step's sort: the stable counting sort of the step's input order
        # (g0's order) by the new cells, done by the oracle
        pos = np.empty(int(g0["pid"].max()) + 1, dtype=np.int64)
        pos[g0["pid"]] = np.arange(n)
        in_order = o1[np.argsort(pos[o1["pid"]], kind="stable")]
        o2 = oracle_mod.Oracle(**cfg)
        o2.load_particles(in_order)
        counts1 = o2.countingsort()
        want = o2.particles()
        o2.close()
        assert np.array_equal(g1["pid"], want["pid"])
        assert np.array_equal(g1["grid"], want["grid"])
        assert np.array_equal(s.cell_counts(), counts1)
        assert s.status() == 0


def test_c1_energy_history_500_steps(gpu_lib, oracle_mod, c1):
    cfg, ld, p, yee = c1
    n = len(p)
    steps, sort_every = 500, 50
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    o.omp_countingsort()
    hist_o = []
    for it in range(1, steps + 1):
        o.omp_pusher()
        o.fieldsolver()
        hist_o.append(o.energies())
        if it % sort_every == 0:
            o.omp_countingsort()
    hist_o = np.array(hist_o)
    with pbpic_b200.Simulation(**cfg, precision="fp64", capacity=n) as s:
        s.init_plasma(**ld)
        s.step(steps, sort_every=sort_every)
        hist_g = s.energy_history()[1:]
        assert hist_g.shape == hist_o.shape
        tot = hist_o.sum(axis=1)
        err = np.abs(hist_g - hist_o).max(axis=0) / np.abs(tot).max()
        assert (err <= HISTORY_TOL).all(), err
        # total energy drift of both within the same bound
        drift_o = abs(tot[-1] / tot[0] - 1.0)
        drift_g = abs(hist_g[-1].sum() / hist_g[0].sum() - 1.0)
        assert abs(drift_g - drift_o) <= HISTORY_TOL, (drift_g, drift_o)
        assert s.gauss_residual() < 1e-11
        assert s.status() == 0
