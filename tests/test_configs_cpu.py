"""Host-side pieces that need no GPU: the reference's own run as a named
configuration (module parameters, pic2d.f90:12-43) and the benchmark's CPU
baseline helpers."""
import math

import pytest


def test_double_harris_has_the_reference_parameters():
    from pbpic_b200 import _lib as L
    from pbpic_b200 import configs
    cfg, ld = configs.double_harris()
    assert (cfg["mx"], cfg["my"]) == (256, 256)                       # nx, ny (pic2d.f90:12)
    assert cfg["dx"] == cfg["dy"] == 0.04                             # dx, dy (pic2d.f90:15)
    assert (cfg["mime"], cfg["cva"]) == (25.0, 15.0)                  # mime, cva (pic2d.f90:19-20)
    assert cfg["dt"] == pytest.approx(0.045 / 25.0)                   # dt (pic2d.f90:42)
    assert cfg["ybc"] == L.BC_PERIODIC
    assert ld["kind"] == L.LOAD_DOUBLE_HARRIS and ld["ppc"] == 64      # ppg (pic2d.f90:30)
    assert ld["lambda_"] == 0.5 and ld["nb"] == 0.2                   # dcs, nbgcs (pic2d.f90:24, 29)
    assert ld["vthe"] == 0.092                                        # vthec (pic2d.f90:22)
    assert ld["vthi"] == pytest.approx(0.092 * math.sqrt(5.0 / 25.0))  # tiecs (pic2d.f90:26, 381)
    assert ld["vthe_bg"] == pytest.approx(0.092 * math.sqrt(0.1))     # tbgcs (pic2d.f90:28, 380)
    assert ld["vthi_bg"] == pytest.approx(ld["vthe_bg"] * math.sqrt(1.0 / 25.0))  # tiebg (pic2d.f90:27, 382)
    assert ld["vdrift_i"] == pytest.approx(1.0 / 15.0) and ld["vdrift_e"] == -ld["vdrift_i"]  # vdrift (pic2d.f90:23)
    # in0 = 1/(n0 dx dy) for the sheet peak density: the formula of pic2d.f90:32-33
    lx = 256 * 0.04
    assert cfg["in0"] == pytest.approx((lx * 0.2 + 2.0) / (64 * lx))
    assert 1.0 / cfg["in0"] == pytest.approx(161.897, rel=1e-4)


def test_bench_cpu_helpers():
    import bench
    h = bench.host_cpu()
    assert h["nproc"] >= 1 and isinstance(h["cpu_model"], str)
    r = bench.run_cpu_single_f32(steps=1)
    assert r["cores"] == 1 and r["value"] > 0 and "compat" in r["sample"]
