"""The long-run comparison tool on a small workload: the FP32 mixed and FP64
plain forms stay within 1e-5 relative in total energy over 20 steps of the
uniform periodic plasma, and the mixed form keeps the Gauss residual below
1e-5 (the uniform plasma is loaded as co-located pairs, so it starts at 0)."""
import pytest

pytestmark = pytest.mark.gpu


def test_longrun_compare_small(gpu_lib):
    from pbpic_b200 import longrun
    r = longrun.compare("uniform_128x128_ppc32", 20, 10)
    assert r["fp32_mixed"]["status"] == 0 and r["fp64_plain"]["status"] == 0
    assert len(r["fp32_mixed"]["gauss"]) == 3
    assert r["total_energy_rel_diff_max"] < 1e-5
    assert r["gauss_mixed_max"] < 1e-5 and r["gauss_fp64_max"] < 1e-12
