"""Physics known-answer tests of the CPU oracle (the restatement of
src/programs/pic2d.f90 that the GPU parity tests compare against)."""
import math

import numpy as np
import pytest

from pbpic_b200 import configs


def fast_plasma(O, ybc, mx=16, my=12, ppc=4, seed=3, vthe=0.6):
    cfg, ld = configs.uniform_c1(mx=mx, my=my, ppc=ppc, seed=seed)
    cfg["ybc"] = ybc
    ld["vthe"], ld["vthi"] = vthe, vthe / 2
    p, yee = O.load_plasma(cfg, ld)
    return cfg, p, yee


def div_j(cfg, j):
    mx, my, ybc = cfg["mx"], cfg["my"], cfg["ybc"]
    jx, jy = j[0][:, :my + 1], j[1]
    d = (jx - np.roll(jx, 1, axis=0)) / cfg["dx"]
    if ybc == 0:
        d = d[:, :my] + (jy[:, :my] - np.roll(jy[:, :my], 1, axis=1)) / cfg["dy"]
        return d
    dyt = np.zeros_like(jx)
    dyt[:, 1:my] = (jy[:, 1:my] - jy[:, 0:my - 1]) / cfg["dy"]
    return d + dyt


@pytest.mark.parametrize("ybc", [0, 1])
def test_zigzag_charge_conservation(oracle_mod, ybc):
    """rho^{n+1} - rho^n + dt div J^{n+1/2} = 0 at every interior node (Umeda 2003),
    including cell crossings, the x wrap, the y wrap and wall reflections."""
    cfg, p, yee = fast_plasma(oracle_mod, ybc)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(0 * yee)
    o.pusher()
    j1 = o.current()
    o.pusher()
    r2 = o.current()[3]
    res = r2 - j1[3] + cfg["dt"] * np.pad(div_j(cfg, j1), ((0, 0), (0, 1 if ybc == 0 else 0)))
    rows = slice(0, cfg["my"]) if ybc == 0 else slice(1, cfg["my"])
    scale = np.abs(r2).max()
    assert scale > 1e-3
    assert np.abs(res[:, rows]).max() < 1e-13 * max(1.0, scale)


def test_compat_fold_leaks_charge(oracle_mod):
    """With the reference's unfolded jy column (quirk Q3) charge is not conserved."""
    cfg, p, yee = fast_plasma(oracle_mod, 0)
    o = oracle_mod.Oracle(**cfg, compat=2)
    o.load_particles(p)
    o.set_fields(0 * yee)
    o.pusher()
    j1 = o.current()
    o.pusher()
    r2 = o.current()[3]
    res = r2 - j1[3] + cfg["dt"] * np.pad(div_j(cfg, j1), ((0, 0), (0, 1)))
    assert np.abs(res[:, :cfg["my"]]).max() > 1e-6


def test_countingsort_is_stable(oracle_mod):
    cfg, p, _ = fast_plasma(oracle_mod, 0, mx=8, my=6, ppc=5)
    rng = np.random.default_rng(1)
    p = p[rng.permutation(len(p))]
    p["grid"] = rng.integers(1, 8 * 6 + 1, len(p))  # many equal keys, random order
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    counts = o.countingsort()
    s = o.particles()
    order = np.argsort(p["grid"], kind="stable")
    assert np.array_equal(s["pid"], p["pid"][order])
    assert np.array_equal(counts, np.bincount(p["grid"] - 1, minlength=48))


def one_particle(O, cfg, q, u, bz=1.0, e=(0.0, 0.0, 0.0)):
    p = np.zeros(1, dtype=O.PARTICLE)
    p["grid"] = cfg["my"] * 3 + 4
    p["q"] = q
    p["pid"] = 1
    p["ux"], p["uy"], p["uz"] = u
    yee = np.zeros((6, cfg["mx"], cfg["my"] + 1))
    yee[5] = bz
    yee[0], yee[1], yee[2] = e
    return p, yee


@pytest.mark.parametrize("q", [1, -1])
def test_boris_rotation_uniform_b(oracle_mod, q):
    """E = 0, uniform Bz: |u| is conserved and u rotates by 2 atan(|c0| Bz / gamma) per step."""
    cfg, _ = configs.uniform_c1(mx=8, my=8)
    cfg["dt"] *= 0.5
    u = (0.3, -0.2, 0.1)
    p, yee = one_particle(oracle_mod, cfg, q, u)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    o.pusher()
    s = o.particles()[0]
    gamma = math.sqrt(1 + sum(x * x for x in u))
    ms = cfg["mime"] if q > 0 else 1.0
    c0 = q * cfg["dt"] * cfg["mime"] / ms / 2
    theta = 2 * math.atan(abs(c0) / gamma)
    a0 = math.atan2(u[1], u[0])
    a1 = math.atan2(s["uy"], s["ux"])
    dtheta = (a1 - a0 + math.pi) % (2 * math.pi) - math.pi
    assert abs(abs(dtheta) - theta) < 1e-13
    # positive charges gyrate clockwise about +z
    assert np.sign(dtheta) == -np.sign(q)
    assert abs(math.hypot(s["ux"], s["uy"]) - math.hypot(u[0], u[1])) < 1e-15
    assert s["uz"] == u[2]


def test_boris_compat_matches_when_e_is_zero(oracle_mod):
    cfg, _ = configs.uniform_c1(mx=8, my=8)
    p, yee = one_particle(oracle_mod, cfg, -1, (0.3, 0.1, -0.2))
    outs = []
    for compat in (0, 1):
        o = oracle_mod.Oracle(**cfg, compat=compat)
        o.load_particles(p)
        o.set_fields(yee)
        o.pusher()
        outs.append(o.particles())
    assert np.array_equal(outs[0], outs[1])
    yee[0] = 0.3  # with E != 0 the reference's pre-kick rotation (quirk Q1) differs
    outs = []
    for compat in (0, 1):
        o = oracle_mod.Oracle(**cfg, compat=compat)
        o.load_particles(p)
        o.set_fields(yee)
        o.pusher()
        outs.append(o.particles())
    assert not np.array_equal(outs[0]["ux"], outs[1]["ux"])


@pytest.mark.parametrize("ybc", [0, 1])
def test_fdtd_vacuum_dispersion(oracle_mod, ybc):
    """A standing Ez wave in vacuum oscillates at the Yee dispersion frequency
    sin(w dt/2) = c dt sqrt(sin^2(kx dx/2)/dx^2 + sin^2(ky dy/2)/dy^2)."""
    mx, my = 32, 16
    cfg, _ = configs.uniform_c1(mx=mx, my=my)
    cfg["ybc"] = ybc
    dx, dy, dt, c = cfg["dx"], cfg["dy"], cfg["dt"], cfg["cva"]
    kx = 2 * math.pi * 2 / (mx * dx)
    ky = (2 * math.pi if ybc == 0 else math.pi) / (my * dy)  # walls: Ez = 0 on the walls
    xc = (np.arange(mx) + 0.5) * dx
    yc = (np.arange(my + 1) + 0.5) * dy
    yee = np.zeros((6, mx, my + 1))
    shape = np.cos(kx * xc)[:, None] * (np.cos(ky * yc) if ybc == 0 else np.sin(ky * yc))[None, :]
    yee[2] = shape
    yee[2][:, my] = 0.0
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(np.zeros(0, dtype=oracle_mod.PARTICLE))
    o.set_fields(yee)
    w = 2 / dt * math.asin(c * dt * math.sqrt(math.sin(kx * dx / 2) ** 2 / dx ** 2 + math.sin(ky * dy / 2) ** 2 / dy ** 2))
    for n in range(1, 121):
        o.pusher()
        o.fieldsolver()
    ez = o.fields()[2][:, :my]
    amp = (ez * shape[:, :my]).sum() / (shape[:, :my] ** 2).sum()
    assert abs(amp - math.cos(w * 120 * dt)) < 1e-9


def test_omp_baseline_matches_serial(oracle_mod):
    """The OpenMP pusher (CPU baseline) follows the same arithmetic as the serial restatement."""
    cfg, ld = configs.harris(32, 16, 16, seed=5)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    a = oracle_mod.Oracle(**cfg)
    b = oracle_mod.Oracle(**cfg)
    for o in (a, b):
        o.load_particles(p)
        o.set_fields(yee)
    a.countingsort()
    b.omp_countingsort(4)
    assert np.array_equal(a.particles(), b.particles())
    for _ in range(3):
        a.pusher()
        a.fieldsolver()
        b.omp_pusher(4)
        b.fieldsolver()
    pa, pb = a.particles(), b.particles()
    pa, pb = pa[np.argsort(pa["pid"])], pb[np.argsort(pb["pid"])]
    assert np.array_equal(pa["grid"], pb["grid"])
    for c in ("dx", "dy", "ux", "uy", "uz"):
        assert np.abs(pa[c] - pb[c]).max() < 1e-12
    assert np.allclose(a.fields(), b.fields(), rtol=0, atol=1e-12)


def test_energy_conservation_uniform(oracle_mod):
    cfg, ld = configs.uniform_c1(mx=32, my=32, ppc=16)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    tot = []
    for _ in range(50):
        o.pusher()
        o.fieldsolver()
        tot.append(o.energies().sum())
    tot = np.array(tot)
    assert np.abs(tot / tot[0] - 1).max() < 1e-2


def filter_corrections(cfg, yee, j4, marder_d=0.001, tau=0.125):
    """Independent numpy statement of divergenceclean (F:867-886) and
    suppresscerenkov (F:889-907) for periodic y: the E changes they make,
    from E before the field solve's update and rho of the push."""
    mx, my = cfg["mx"], cfg["my"]
    idx, idy, dt, cva2 = 1 / cfg["dx"], 1 / cfg["dy"], cfg["dt"], cfg["cva"] ** 2
    ex, ey, ez = (yee[c][:, :my] for c in range(3))
    rho = j4[3][:, :my]
    r = np.roll
    f = (ex - r(ex, 1, 0)) * idx + (ey - r(ey, 1, 1)) * idy - cva2 * rho
    mex = dt * marder_d / cfg["dx"] * (r(f, -1, 0) - f)
    mey = dt * marder_d / cfg["dy"] * (r(f, -1, 1) - f)
    cdx, cdy = dt * cva2 * tau * dt / cfg["dx"], dt * cva2 * tau * dt / cfg["dy"]
    dexdy, deydx = (r(ex, -1, 1) - ex) * idy, (r(ey, -1, 0) - ey) * idx
    dezdx, dezdy = (ez - r(ez, 1, 0)) * idx, (ez - r(ez, 1, 1)) * idy
    cex = cdy * (deydx - r(deydx, 1, 1) - dexdy + r(dexdy, 1, 1))
    cey = cdx * (-deydx + r(deydx, 1, 0) + dexdy - r(dexdy, 1, 0))
    cez = cdx * (r(dezdx, -1, 0) - dezdx) + cdy * (r(dezdy, -1, 1) - dezdy)
    return mex - cex, mey - cey, cez


@pytest.mark.parametrize("flags", [1, 2, 3])
def test_field_filters_match_numpy(oracle_mod, flags):
    """The oracle's Marder and Cherenkov filters change E by exactly the
    corrections an independent numpy statement computes."""
    cfg, p, _ = fast_plasma(oracle_mod, 0, mx=16, my=12)
    rng = np.random.default_rng(4)
    yee = rng.normal(size=(6, 16, 13)) * 0.3
    out = []
    for fl in (0, flags):
        o = oracle_mod.Oracle(**cfg)
        o.load_particles(p)
        o.set_fields(yee)
        o.set_filters(fl, 0.02, 0.4)  # larger than the reference's constants, to be visible
        e0 = o.fields()
        o.pusher()
        j4 = o.current()
        o.fieldsolver()
        out.append((e0, j4, o.fields()))
    (e0, j4, off), (_, _, on) = out
    want = filter_corrections(cfg, e0, j4, 0.02 if flags & 1 else 0.0, 0.4 if flags & 2 else 0.0)
    my = cfg["my"]
    for c in range(3):
        got = on[c][:, :my] - off[c][:, :my]
        assert np.abs(got - want[c]).max() <= 1e-12 * max(1.0, np.abs(want[c]).max()), (c, np.abs(got - want[c]).max(), np.abs(want[c]).max())
        if c < 2 or flags & 2:
            assert np.abs(want[c]).max() > 1e-6



def test_double_harris_loader(oracle_mod):
    """The reference's own plasma (pic2d.f90:357-648): co-located pairs, an even
    number of sheet pairs alternating between the sheets at Lx/4 and 3Lx/4 with
    a sech^2 profile in x (mean |x - xc| = lambda ln 2), drifts of opposite sign
    in the two sheets and none in the background, no thermal motion along z,
    and By = tanh((x - Lx/4)/lambda) - tanh((x - 3Lx/4)/lambda) - 1 on the node
    columns with every other field component zero."""
    from pbpic_b200 import configs
    cfg, ld = configs.double_harris(mx=256, my=8, ppc=8, seed=11)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    lp = oracle_mod.load_params(cfg, ld)
    mx, my, dx, lam = cfg["mx"], cfg["my"], cfg["dx"], ld["lambda_"]
    lx = mx * dx
    npairs = ld["ppc"] * mx * my
    assert len(p) == 2 * npairs and lp.nsheet % 2 == 0
    assert abs(lp.nsheet - npairs * 4 * lam / (4 * lam + ld["nb"] * lx)) <= 1.0
    ion, ele = p[0::2], p[1::2]
    assert np.all(ion["q"] == 1) and np.all(ele["q"] == -1)
    for c in ("grid", "dx", "dy"):
        assert np.array_equal(ion[c], ele[c])  # zero initial charge density
    ix = (ion["grid"] - 1) // my
    x = (ix + 0.5 + ion["dx"]) * dx
    k = np.arange(npairs)
    sheet = k < lp.nsheet
    for parity, xc in ((0, 0.25 * lx), (1, 0.75 * lx)):
        m = sheet & (k % 2 == parity)
        assert abs(np.mean(np.abs(x[m] - xc)) - lam * math.log(2.0)) < 0.02
        sgn = 1.0 if parity == 0 else -1.0
        assert np.allclose(ion["uz"][m], sgn * lp.udrift_i, rtol=0, atol=1e-15)
        assert np.allclose(ele["uz"][m], sgn * lp.udrift_e, rtol=0, atol=1e-15)
    assert lp.udrift_i > 0 > lp.udrift_e
    assert np.all(ion["uz"][~sheet] == 0) and np.all(ele["uz"][~sheet] == 0)
    # thermal spread in x and y: sheet and background temperatures
    assert abs(np.std(ele["ux"][sheet]) / lp.uthe - 1) < 0.05
    assert abs(np.std(ion["uy"][~sheet]) / lp.uthi_bg - 1) < 0.05
    xs = np.arange(mx) * dx
    by = np.tanh((xs - 0.25 * lx) / lam) - np.tanh((xs - 0.75 * lx) / lam) - 1.0
    assert np.allclose(yee[4], by[:, None], rtol=0, atol=1e-15)
    assert not yee[[0, 1, 2, 3, 5]].any()
