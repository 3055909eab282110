"""GPU parity: the CUDA library (through the C ABI) against the CPU oracle.

Bars: FP64 plain -- particles and fields after one step within 1e-12
relative (bit-identical particle state when the push evaluates the
reference's quotients and square roots in its order, PBPIC_OPT_EXACT_FP64),
sort permutation and per-cell counts exact; FP32 mixed -- particles within 2e-5 relative and current within
2e-4 of its maximum against the FP64 oracle after one step, bit-reproducible
run to run."""
import numpy as np
import pytest

import pbpic_b200
from pbpic_b200 import configs

pytestmark = pytest.mark.gpu

COMPS = ("dx", "dy", "ux", "uy", "uz")


def plasma(O, ybc, mx=16, my=12, ppc=8, seed=5, vthe=0.3, kind="uniform"):
    if kind == "harris":
        cfg, ld = configs.harris(mx, my, ppc, seed=seed)
        cfg["ybc"] = ybc
    elif kind == "double_harris":
        cfg, ld = configs.double_harris(mx, my, ppc, seed=seed)
        cfg["ybc"] = ybc
    else:
        cfg, ld = configs.uniform_c1(mx=mx, my=my, ppc=ppc, seed=seed)
        cfg["ybc"] = ybc
        ld["vthe"], ld["vthi"] = vthe, vthe / 3
    p, yee = O.load_plasma(cfg, ld)
    return cfg, ld, p, yee


def random_fields(cfg, seed, amp=0.05, bz=1.0):
    mx, my = cfg["mx"], cfg["my"]
    rng = np.random.default_rng(seed)
    yee = amp * rng.standard_normal((6, mx, my + 1))
    yee[5] += bz
    if cfg["ybc"] == 1:
        yee[0][:, 0] = yee[0][:, my] = 0.0  # tangential E vanishes on the walls
        yee[[1, 2, 4, 5], :, my] = 0.0
    else:
        yee[:, :, my] = 0.0
    return yee


def field_err(fg, fo, cfg):
    """Max difference over the stored Yee values: node-row components (ex, bx)
    on rows 0..my with walls, half-row components and periodic rows 0..my-1."""
    my = cfg["my"]
    node_rows = my + 1 if cfg["ybc"] == 1 else my
    e = max(np.abs(fg[c, :, :node_rows] - fo[c, :, :node_rows]).max() for c in (0, 3))
    e = max(e, max(np.abs(fg[c, :, :my] - fo[c, :, :my]).max() for c in (1, 2, 4, 5)))
    return e


def by_pid(a):
    return a[np.argsort(a["pid"], kind="stable")]


def assert_particles(g, o, tol, rel=True):
    g, o = by_pid(g), by_pid(o)
    assert np.array_equal(g["pid"], o["pid"])
    assert np.array_equal(g["q"], o["q"])
    bad = np.nonzero(g["grid"] != o["grid"])[0]
    assert len(bad) == 0, (len(bad), g[bad[:3]], o[bad[:3]])
    worst = 0.0
    for c in COMPS:
        scale = max(1.0, np.abs(o[c]).max()) if rel else 1.0
        err = np.abs(g[c] - o[c]).max() / scale
        worst = max(worst, err)
        assert err <= tol, (c, err)
    return worst


def new_sim(cfg, n, precision="fp64", compat=0, **kw):
    return pbpic_b200.Simulation(**cfg, precision=precision, compat=compat, track_pid=True, capacity=n, **kw)


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("ybc,compat,presort", [(0, 0, False), (0, 0, True), (0, 7, True), (1, 0, True),
                                                (1, 0, False)])
def test_plain_one_step_matches_oracle(gpu_lib, oracle_mod, ybc, compat, presort, exact):
    """exact: the push's quotients and square roots correctly rounded in the
    reference's order (PBPIC_OPT_EXACT_FP64, implied by any compat switch), the
    particle state bit-identical to the oracle's; otherwise 1/gamma from rsqrt,
    within 1e-12."""
    cfg, ld, p, _ = plasma(oracle_mod, ybc)
    rng = np.random.default_rng(7)
    p = p[rng.permutation(len(p))]
    yee = random_fields(cfg, 3)
    o = oracle_mod.Oracle(**cfg, compat=compat)
    o.load_particles(p)
    o.set_fields(yee)
    with new_sim(cfg, len(p), compat=compat, options=pbpic_b200.OPT_EXACT_FP64 if exact else 0) as s:
        s.load_particles(p)
        s.load_fields(yee)
        assert np.allclose(s.emfgrid(), o.emfgrid(), rtol=0, atol=1e-15)
        if presort:
            counts_o = o.countingsort()
            s.countingsort()
            assert np.array_equal(s.particles()["pid"], o.particles()["pid"])
            assert np.array_equal(s.cell_counts(), counts_o)
        o.pusher()
        s.pusher()
        err = assert_particles(s.particles(), o.particles(), 1e-12)
        if exact or compat:
            assert err == 0.0  # same operation order: bit-identical particle state
        jg, jo = s.denjr(), o.current()
        rows = cfg["my"] if ybc == 0 else cfg["my"] + 1
        jscale = np.abs(jo[:, :, :rows]).max()
        assert np.abs(jg[:, :, :rows] - jo[:, :, :rows]).max() <= 1e-12 * jscale
        o.fieldsolver()
        s.fieldsolver()
        fg, fo = s.fields(), o.fields()
        assert field_err(fg, fo, cfg) <= 1e-12 * np.abs(fo).max()
        gg, go = s.emfgrid(), o.emfgrid()
        assert np.abs(gg - go).max() <= 1e-12 * np.abs(go).max()
        assert np.allclose(s.energies(), o.energies(), rtol=1e-12)
        assert s.status() & ~pbpic_b200.STATUS_UNSORTED == 0


@pytest.mark.parametrize("ybc", [0, 1])
def test_mixed_one_step_within_fp32_of_fp64_oracle(gpu_lib, oracle_mod, ybc):
    cfg, ld, p, _ = plasma(oracle_mod, ybc, mx=32, my=16, ppc=8)
    yee = random_fields(cfg, 4)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    o.countingsort()
    with new_sim(cfg, len(p), precision="fp32") as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.countingsort()
        # the FP32 state of the oracle's input, to separate storage rounding from the step
        o32 = oracle_mod.Oracle(**cfg)
        o32.load_particles(s.particles())
        o32.set_fields(s.fields())
        o32.countingsort()
        o32.pusher()
        s.pusher()
        assert_particles(s.particles(), o32.particles(), 2e-5)
        jg, jo = s.denjr(), o32.current()
        rows = cfg["my"] if ybc == 0 else cfg["my"] + 1
        assert np.abs(jg[:, :, :rows] - jo[:, :, :rows]).max() <= 2e-4 * np.abs(jo[:, :, :rows]).max()


def test_mixed_is_bit_reproducible(gpu_lib):
    cfg, ld = configs.harris(64, 32, 32, seed=9)
    outs = []
    for _ in range(2):
        with pbpic_b200.Simulation(**cfg, precision="fp32", capacity=2 * 32 * 64 * 32) as s:
            s.init_plasma(**ld)
            s.step(6, sort_every=1)
            outs.append((s.particles(), s.fields(), s.denjr(), s.energy_history()))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_loader_matches_cpu_loader(gpu_lib, oracle_mod, precision):
    for cfg, ld in (configs.uniform_c1(mx=16, my=8, ppc=8, seed=2), configs.harris(32, 16, 8, seed=6),
                    configs.double_harris(64, 16, 8, seed=9), configs.two_stream(32, 16, 8, seed=11),
                    configs.weibel(32, 16, 8, seed=12), configs.two_stream(64, 64, 16, seed=13, vdrift=0.24),
                    configs.weibel(128, 64, 16, seed=14, anisotropy=6.4)):
        p, yee = oracle_mod.load_plasma(cfg, ld)
        ref = p[np.argsort(p["grid"], kind="stable")]
        with new_sim(cfg, len(p), precision=precision) as s:
            s.init_plasma(**ld)
            g = s.particles()
            assert np.array_equal(g["grid"], ref["grid"]) and np.array_equal(g["pid"], ref["pid"])
            for c in COMPS:
                want = ref[c] if precision == "fp64" else ref[c].astype(np.float32).astype(np.float64)
                assert np.array_equal(g[c], want), c
            f = s.fields()
            want = yee if precision == "fp64" else yee.astype(np.float32).astype(np.float64)
            rows = cfg["my"] if cfg["ybc"] == 0 else cfg["my"] + 1
            assert np.array_equal(f[:, :, :rows], want[:, :, :rows])


@pytest.mark.parametrize("ybc,kind", [(0, "uniform"), (1, "harris"), (0, "double_harris")])
def test_plain_energy_history_matches_oracle(gpu_lib, oracle_mod, ybc, kind):
    cfg, ld, p, yee = plasma(oracle_mod, ybc, mx=32, my=16, ppc=8, kind=kind)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    o.countingsort()
    hist_o = []
    with new_sim(cfg, len(p)) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.countingsort()
        for it in range(1, 21):
            o.pusher()
            o.fieldsolver()
            hist_o.append(o.energies())
            if it % 5 == 0:
                o.countingsort()
        s.step(20, sort_every=5)
        hist_g = s.energy_history()[1:]
        assert np.allclose(hist_g, np.array(hist_o), rtol=1e-10, atol=1e-12)
        assert_particles(s.particles(), o.particles(), 1e-9)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gauss_law_preserved(gpu_lib, precision):
    cfg, ld = configs.harris(64, 32, 16, seed=8)
    with pbpic_b200.Simulation(**cfg, precision=precision, capacity=2 * 16 * 64 * 32) as s:
        s.init_plasma(**ld)
        r0 = s.gauss_residual()
        s.step(10, sort_every=1)
        r1 = s.gauss_residual()
        tol = 1e-11 if precision == "fp64" else 2e-4
        assert r0 < 1e-12
        assert r1 < tol, r1
        assert s.status() == 0


def test_sort_matches_oracle_permutation_random_keys(gpu_lib, oracle_mod):
    cfg, ld, p, yee = plasma(oracle_mod, 0, mx=40, my=30, ppc=3)
    rng = np.random.default_rng(12)
    p["grid"] = rng.integers(1, 40 * 30 + 1, len(p))
    p = p[rng.permutation(len(p))]
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    counts = o.countingsort()
    with new_sim(cfg, len(p)) as s:
        s.load_particles(p)
        s.countingsort()
        assert np.array_equal(s.particles()["pid"], o.particles()["pid"])
        assert np.array_equal(s.cell_counts(), counts)


@pytest.mark.parametrize("n,ncells", [(0, 5), (1, 1), (1000, 1), (5000, 7), (100000, 1 << 20), (300000, 70000),
                                      (4097, 300)])
def test_counting_sort_keys_stateless(gpu_lib, n, ncells):
    import torch
    g = torch.Generator().manual_seed(n + ncells)
    keys = torch.randint(0, ncells, (n,), generator=g, dtype=torch.int32)
    if n > 10:
        keys[: n // 3] = ncells - 1  # a heavy cell
    kd = keys.cuda()
    perm = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    counts = torch.empty(ncells, dtype=torch.int32, device="cuda")
    pbpic_b200.counting_sort_keys(kd.data_ptr(), n, ncells, perm.data_ptr(), counts.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = np.argsort(keys.numpy(), kind="stable")
    assert np.array_equal(perm[:n].cpu().numpy(), ref)
    assert np.array_equal(counts.cpu().numpy(), np.bincount(keys.numpy(), minlength=ncells))


def test_counting_sort_keys_rejects_bad_keys(gpu_lib):
    import torch
    kd = torch.tensor([0, 3, 9, 1], dtype=torch.int32, device="cuda")
    perm = torch.empty(4, dtype=torch.int32, device="cuda")
    counts = torch.empty(5, dtype=torch.int32, device="cuda")
    with pytest.raises(pbpic_b200.PbpicError):
        pbpic_b200.counting_sort_keys(kd.data_ptr(), 4, 5, perm.data_ptr(), counts.data_ptr(), 0)


def test_status_flags_report_injected_faults(gpu_lib, oracle_mod):
    """A corrupt offset (|dx| > 1.5 after the move) and a NaN momentum are
    reported through pbpic_status; the step itself stays in bounds."""
    cfg, ld, p, yee = plasma(oracle_mod, 0, mx=8, my=8, ppc=2)
    p = p[:8].copy()
    p["dx"][0] = 1.45
    p["ux"][0] = 0.9
    p["uy"][1] = np.nan
    with new_sim(cfg, len(p)) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.pusher()
        st = s.status()
        assert st & pbpic_b200.STATUS_CELL_JUMP
        assert st & pbpic_b200.STATUS_NAN
        assert s.status() == 0  # cleared by the read


def test_bad_particle_records_are_rejected(gpu_lib, oracle_mod):
    cfg, ld, p, yee = plasma(oracle_mod, 0, mx=8, my=8, ppc=1)
    p = p.copy()
    p["grid"][3] = 8 * 8 + 1
    with new_sim(cfg, len(p)) as s:
        with pytest.raises(pbpic_b200.PbpicError):
            s.load_particles(p)
        with pytest.raises(pbpic_b200.PbpicError):
            s.load_particles(np.concatenate([p, p]))  # over capacity


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("ybc,mx,my,ty", [(0, 16, 12, 0), (0, 9, 20, 6), (1, 16, 12, 0), (1, 7, 13, 5), (1, 8, 40, 64),
                                         (1, 5, 70, 0), (0, 4, 80, 0)])
def test_fused_sort_is_the_stable_sort(gpu_lib, oracle_mod, precision, ybc, mx, my, ty):
    """After a push on a sorted array, the counting sort from the push's
    per-tile histograms gives exactly the stable sort by cell (array order
    within a cell) of the pushed particles, and the per-cell counts."""
    cfg, ld, p, _ = plasma(oracle_mod, ybc, mx=mx, my=my, ppc=6, vthe=0.6)
    yee = random_fields(cfg, 5, amp=0.2)
    # the push leaves its output in pushed order; countingsort runs the fused sort
    with new_sim(cfg, len(p), precision=precision, tile_rows=ty, options=pbpic_b200.OPT_NO_AUTOSORT) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.countingsort()
        for _ in range(3):
            s.pusher()
            pre = s.particles()
            s.fieldsolver()
            s.countingsort()
            post = s.particles()
            order = np.argsort(pre["grid"], kind="stable")
            assert np.array_equal(post["pid"], pre["pid"][order])
            assert np.array_equal(post["grid"], pre["grid"][order])
            for c in COMPS:
                assert np.array_equal(post[c], pre[c][order])
            assert np.array_equal(s.cell_counts(), np.bincount(pre["grid"] - 1, minlength=mx * my))
        assert s.status() == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sort_of_whole_cell_runs(gpu_lib, oracle_mod, precision):
    """Particles whose cells each form one contiguous run, the runs in shuffled
    order (as after a slab exchange: sorted pieces with disjoint cells), sort
    by the single-scatter path to the stable counting sort's order."""
    cfg, ld, p, _ = plasma(oracle_mod, 0, mx=16, my=12, ppc=6)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p)
    o.countingsort()
    ps = o.particles()
    starts = np.flatnonzero(np.r_[True, ps["grid"][1:] != ps["grid"][:-1]])
    runs = np.split(ps, starts[1:])
    rng = np.random.default_rng(9)
    q = np.concatenate([runs[k] for k in rng.permutation(len(runs))])
    assert not np.array_equal(q["pid"], ps["pid"])
    with new_sim(cfg, len(q), precision=precision) as s:
        s.load_particles(q)
        s.countingsort()
        got = s.particles()
        assert np.array_equal(got["pid"], ps["pid"])
        assert np.array_equal(s.cell_counts(), np.bincount(ps["grid"] - 1, minlength=cfg["mx"] * cfg["my"]))
