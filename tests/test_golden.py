"""The CPU oracle against golden fixtures from an independent line-by-line
Python transcription of src/programs/pic2d.f90 (tests/golden/make_golden.py):
countingsort permutation and counts, particles after pusher, the folded
current, fields and node averages after fieldsolver, and the energies. Both
evaluate the reference's expressions in the same order in IEEE double, so the
results agree bit for bit."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_step.npz")


@pytest.mark.parametrize("case", ["a", "b"])
def test_oracle_matches_golden(oracle_mod, case):
    g = np.load(GOLDEN)
    mx, my, dx, dy, dt, cva, mime, in0, compat = g[f"{case}_params"]
    mx, my, compat = int(mx), int(my), int(compat)
    o = oracle_mod.Oracle(mx, my, dx, dy, dt, cva, mime, in0, ybc=0, compat=compat)
    inp = g[f"{case}_inputs"]
    p = np.zeros(len(inp), dtype=oracle_mod.PARTICLE)
    for f in inp.dtype.names:
        p[f] = inp[f]
    o.load_particles(p)
    o.set_fields(g[f"{case}_yee"])
    counts = o.countingsort()
    assert np.array_equal(counts, g[f"{case}_counts"])
    assert np.array_equal(o.particles()["pid"], g[f"{case}_sorted_pid"])
    o.pusher()
    got = o.particles()
    want = g[f"{case}_pushed"]
    assert np.array_equal(got["pid"], want["pid"]) and np.array_equal(got["grid"], want["grid"])
    for f in ("dx", "dy", "ux", "uy", "uz"):
        assert np.array_equal(got[f], want[f]), f
    assert np.array_equal(o.current()[:, :, :my], g[f"{case}_j4"][:, :, :my])
    o.fieldsolver()
    assert np.array_equal(o.fields()[:, :, :my], g[f"{case}_fields"][:, :, :my])
    assert np.array_equal(o.emfgrid(), g[f"{case}_emfgrid"])
    assert np.allclose(o.energies(), g[f"{case}_energies"], rtol=1e-14, atol=0)
