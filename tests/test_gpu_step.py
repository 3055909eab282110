"""pbpic_step runs the field solve on a second stream beside the counting sort
(the two read disjoint results of the push). Its state after every step must
be the state of the three calls made in order on one stream, which keep the
reference's sequence pusher, fieldsolver, countingsort (pic2d.f90:177-182):
bit for bit in the mixed form (exact current sums), within 1e-12 in the plain
form (its atomic current sums round in the order they land). Checked with the
sort every step (the library's default) and every 5 steps (the push leaves the
sort to the caller, and the pushes between sorts take the path for unsorted
particles), periodic and conducting y."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(cfg, ld, precision, nsteps, sort_every, options, overlapped):
    import pbpic_b200
    from pbpic_b200.sim import Simulation
    n = Simulation(**cfg, precision=precision, capacity=1).loader_count(**ld)
    with Simulation(**cfg, precision=precision, capacity=n, track_pid=True, options=options) as s:
        s.init_plasma(**ld)
        if overlapped:
            s.step(nsteps, sort_every=sort_every)
        else:
            for _ in range(nsteps):
                s.pusher()
                s.fieldsolver()
                if s.itime() % sort_every == 0:
                    s.countingsort()
        p = s.particles(dtype=pbpic_b200.PARTICLE_F64)
        return dict(p=p[np.argsort(p["pid"])], fields=s.fields(), emfgrid=s.emfgrid(), denjr=s.denjr(),
                    hist=s.energy_history(), counts=s.cell_counts(), status=s.status())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("sort_every,autosort", [(1, True), (5, False)])
@pytest.mark.parametrize("kind", ["harris", "uniform"])
def test_step_equals_separate_calls(gpu_lib, precision, sort_every, autosort, kind):
    import pbpic_b200
    from pbpic_b200 import configs
    cfg, ld = configs.harris(64, 48, 16, seed=7) if kind == "harris" else configs.uniform_c1(seed=8, mx=48, my=40, ppc=12)
    opts = 0 if autosort else pbpic_b200.OPT_NO_AUTOSORT
    a = run(cfg, ld, precision, 12, sort_every, opts, overlapped=True)
    b = run(cfg, ld, precision, 12, sort_every, opts, overlapped=False)
    # the pushes between sorts meet particles outside their tiles (informational bit)
    assert a["status"] == b["status"] and (a["status"] & ~pbpic_b200.STATUS_UNSORTED) == 0
    assert np.array_equal(a["counts"], b["counts"])
    assert np.array_equal(a["p"]["grid"], b["p"]["grid"])
    for key in ("fields", "emfgrid", "denjr", "hist"):
        if precision == "fp32":
            assert np.array_equal(a[key], b[key]), key
        else:
            scale = max(1.0, float(np.abs(b[key]).max()))
            assert np.abs(a[key] - b[key]).max() <= 1e-12 * scale, key
    for c in ("dx", "dy", "ux", "uy", "uz"):
        if precision == "fp32":
            assert np.array_equal(a["p"][c], b["p"][c]), c
        else:
            assert np.abs(a["p"][c] - b["p"][c]).max() <= 1e-12 * max(1.0, float(np.abs(b["p"][c]).max())), c
