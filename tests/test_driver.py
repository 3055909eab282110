"""The C++ time-loop driver (pbpic_b200/csrc/pic2d_driver.cpp): the reference's
main program on the C ABI, run end to end."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "pbpic_b200", "pic2d_driver")


@pytest.mark.gpu
@pytest.mark.parametrize("args", [["--uniform", "--mx", "32", "--my", "32", "--ppc", "8", "--fp64"],
                                  ["--harris", "--mx", "64", "--my", "32", "--ppc", "16", "--fp32"],
                                  ["--double-harris", "--mx", "256", "--my", "16", "--ppc", "16", "--fp64"],
                                  []])  # the reference's own run: double Harris, 256x256, 64 pairs per cell
def test_driver_time_loop(gpu_lib, args):
    r = subprocess.run([DRIVER, *args, "--ntime", "30", "--ntdiag", "10", "--sort-every", "5"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rows = np.array([[float(x) for x in ln.split()] for ln in r.stdout.strip().splitlines()])
    assert rows.shape == (4, 5) and list(rows[:, 0]) == [0, 10, 20, 30]
    tot = rows[:, 1:].sum(axis=1)
    assert np.all(np.abs(tot / tot[0] - 1) < 1e-2)


def test_driver_rejects_unknown_options():
    from pbpic_b200 import build
    build.build()
    r = subprocess.run([DRIVER, "--bogus"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown option" in r.stderr
