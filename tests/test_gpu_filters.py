"""The optional field filters (Marder divergence cleaning, the Cherenkov
filter) against the oracle: FP64 plain within 1e-12 relative of the oracle's
fields after a push and a field solve with the filters on, over three steps;
FP32 mixed within 2e-5 of its maximum. The filters exist for periodic y only."""
import numpy as np
import pytest

import pbpic_b200
from test_gpu_parity import field_err, new_sim, plasma, random_fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_filters_match_oracle(gpu_lib, oracle_mod, flags, precision):
    cfg, ld, p, _ = plasma(oracle_mod, 0, mx=16, my=12, ppc=8)
    yee = random_fields(cfg, 6, amp=0.3)
    o = oracle_mod.Oracle(**cfg)
    with new_sim(cfg, len(p), precision=precision) as s:
        s.load_particles(p)
        s.load_fields(yee)
        s.countingsort()
        o.load_particles(s.particles() if precision == "fp32" else p)
        o.set_fields(s.fields())
        o.countingsort()
        o.set_filters(flags, 0.02, 0.4)
        s.set_field_filters(flags, 0.02, 0.4)
        off = None
        for _ in range(3):
            o.pusher()
            o.fieldsolver()
            s.pusher()
            s.fieldsolver()
        fg, fo = s.fields(), o.fields()
        tol = 1e-12 if precision == "fp64" else 2e-5
        assert field_err(fg, fo, cfg) <= tol * np.abs(fo).max(), field_err(fg, fo, cfg)
        # the filters changed the fields: a run without them differs
        with new_sim(cfg, len(p), precision=precision) as u:
            u.load_particles(p)
            u.load_fields(yee)
            u.countingsort()
            for _ in range(3):
                u.pusher()
                u.fieldsolver()
            off = u.fields()
        assert field_err(fg, off, cfg) > 100 * tol * np.abs(fo).max()


def test_filters_need_periodic_y(gpu_lib, oracle_mod):
    cfg, ld, p, _ = plasma(oracle_mod, 1, mx=16, my=12, ppc=2)
    with new_sim(cfg, len(p)) as s:
        with pytest.raises(pbpic_b200.PbpicError):
            s.set_field_filters(1)
        s.set_field_filters(0)
        with pytest.raises(pbpic_b200.PbpicError):
            s.set_field_filters(4)
