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
