"""Size-independent properties at the benchmark's full size (GEM Harris
sheet, 1024x512 cells, 100 particles per cell per species, 104,857,600
particles, FP32 mixed): after three steps no status bit is set, the Gauss
residual stays below 1e-6, the total energy changes by less than 1e-5, the
particles are sorted by cell (the fused counting sort) and none is lost, and a
second run gives the same bits (fields and energy history)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(steps):
    from pbpic_b200 import configs
    from pbpic_b200.sim import Simulation
    cfg, ld = configs.harris_c2()
    n = Simulation(**cfg, precision="fp32", capacity=1).loader_count(**ld)
    s = Simulation(**cfg, precision="fp32", capacity=n)
    s.init_plasma(**ld)
    s.step(steps, sort_every=1)
    return s, n, cfg


def test_fullsize_properties_and_determinism(gpu_lib):
    import pbpic_b200
    a, n, cfg = run(3)
    assert a.status() == 0
    assert a.gauss_residual() < 1e-6
    h = a.energy_history()
    tot = h.sum(axis=1)
    assert np.all(np.isfinite(h)) and abs(tot[-1] / tot[0] - 1) < 1e-5
    assert a.cell_counts().sum() == n
    p = a.particles(dtype=pbpic_b200.PARTICLE_F32)
    assert len(p) == n and np.all(np.diff(p["grid"]) >= 0)
    fa, ha = a.fields(), h
    del p
    a.close()
    b, _, _ = run(3)
    assert np.array_equal(b.fields(), fa)
    assert np.array_equal(b.energy_history(), ha)
    b.close()
