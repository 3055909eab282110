"""Known-answer tests of the loader's random numbers and math (CPU).

Philox4x64-10 is pinned against numpy.random.Philox, an independent
implementation of the same published generator; numpy pre-increments its
counter, so its block c is philox4x64(counter = c + 1)."""
import math

import numpy as np
import pytest


@pytest.mark.parametrize("key", [(0, 0), (5, 7), (0xDEADBEEF, 0x5049434C4F414431), (2**64 - 1, 12345)])
def test_philox_matches_numpy(oracle_mod, key):
    g = np.random.Philox(key=np.array(key, dtype=np.uint64), counter=np.zeros(4, dtype=np.uint64))
    ref = g.random_raw(4 * 6).reshape(6, 4)
    for c in range(6):
        got = oracle_mod.philox((c + 1, 0, 0, 0), key)
        assert np.array_equal(got, ref[c].astype(np.uint64)), (c, got, ref[c])


def test_philox_high_counter_words(oracle_mod):
    # numpy's 256-bit counter carries into the upper words; start just below a carry
    g = np.random.Philox(key=np.array([3, 4], dtype=np.uint64), counter=np.array([2**64 - 2, 7, 0, 0], dtype=np.uint64))
    ref = g.random_raw(8).reshape(2, 4)
    assert np.array_equal(oracle_mod.philox((2**64 - 1, 7, 0, 0), (3, 4)), ref[0])
    assert np.array_equal(oracle_mod.philox((0, 8, 0, 0), (3, 4)), ref[1])


def test_pic_log_accuracy(oracle_mod):
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.random(2000), 10.0 ** rng.uniform(-300, 300, 2000), [1.0, 2.0, 0.5, 1e-300, 1e300]])
    for x in xs:
        if x <= 0:
            continue
        got = oracle_mod.pic_log(x)
        ref = math.log(x)
        assert abs(got - ref) <= 4e-16 * max(1.0, abs(ref)), (x, got, ref)


def test_uniform_loader_statistics(oracle_mod):
    from pbpic_b200 import configs
    cfg, ld = configs.uniform_c1(mx=16, my=8, ppc=64, seed=11)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    assert len(p) == 2 * 64 * 16 * 8
    # stratified: every cell holds ppc pairs, ion and electron co-located
    counts = np.bincount(p["grid"] - 1, minlength=16 * 8)
    assert np.all(counts == 2 * 64)
    ions, els = p[0::2], p[1::2]
    assert np.all(ions["q"] == 1) and np.all(els["q"] == -1)
    assert np.array_equal(ions["dx"], els["dx"]) and np.array_equal(ions["dy"], els["dy"])
    assert np.all(np.abs(p["dx"]) <= 0.5) and np.all(np.abs(p["dy"]) <= 0.5)
    ue = ld["vthe"] / math.sqrt(1 - ld["vthe"] ** 2)
    for c in ("ux", "uy", "uz"):
        assert abs(els[c].std() / ue - 1) < 0.03
        assert abs(els[c].mean()) < 0.05 * ue
    assert np.all(yee[5] == 1.0) and np.all(yee[:5] == 0.0)


def test_harris_loader_profile(oracle_mod):
    from pbpic_b200 import configs
    cfg, ld = configs.harris(64, 64, 64, seed=2)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    iy = (p["grid"] - 1) % cfg["my"]
    y = (iy + 0.5 + p["dy"]) * cfg["dy"]
    ly = cfg["my"] * cfg["dy"]
    hist, edges = np.histogram(y, bins=32, range=(0, ly))
    centres = 0.5 * (edges[1:] + edges[:-1])
    lam, nb = ld["lambda_"], ld["nb"]
    # expected density n0 sech^2((y - Ly/2)/lambda) + nb n0, in units of macro particles per bin
    p0 = 1.0 / cfg["in0"]
    bin_cells = cfg["mx"] * (ly / 32) / cfg["dy"]
    model = 2 * p0 * bin_cells / cfg["mx"] * cfg["mx"] * (
        np.array([np.mean(1 / np.cosh((np.linspace(a, b, 64) - ly / 2) / lam) ** 2) for a, b in zip(edges[:-1], edges[1:])])
        + nb)
    assert np.allclose(hist, model, rtol=0.08)
    # sheet drifts: ions along -z, electrons along +z at the sheet centre
    core = np.abs(y - ly / 2) < 0.2
    assert p["uz"][core & (p["q"] == 1)].mean() < 0 < p["uz"][core & (p["q"] == -1)].mean()
    # Harris field: Bx = tanh((y - Ly/2)/lambda) on node rows plus a small perturbation
    j = np.arange(cfg["my"] + 1)
    bx_mean = yee[3].mean(axis=0)
    assert np.allclose(bx_mean, np.tanh((j * cfg["dy"] - ly / 2) / lam), atol=1e-12)
