"""Long run of a workload in the FP32 mixed and FP64 plain forms, side by side.

    python -m pbpic_b200.longrun --workload harris_1024x512_ppc100 --steps 20000

Both forms start from the same seeded plasma and step with the counting sort
every step. Every `--every` steps the run records the reconnected flux and the
Gauss residual max|div E / cva^2 - rho| of each form; the energy history
(electron KE, ion KE, E, B) is kept on the device for every step. The output
(one JSON object) gives, per form, the total-energy drift |E(t)/E(0) - 1| at
the end and its maximum, the Gauss residuals and the flux series, and the
differences between the forms: the largest relative difference of the total
energy and of the flux, and the largest Gauss residual of each form. With
--control a second FP64 run gives the same differences between two FP64 runs
(their FP64 atomic sums round in the order the atomics land, so they are not
bit-identical), the spread that chaotic dynamics alone produce.
"""
import argparse
import json
import time

import numpy as np

from . import configs
from .sim import Simulation


def run(workload, steps, every, precision, seed_offset=0):
    cfg, ld = configs.WORKLOADS[workload]()
    ld = dict(ld, seed=ld["seed"] + seed_offset)
    n = Simulation(**cfg, precision=precision, capacity=1).loader_count(**ld)
    out = {"precision": precision, "particles": n, "steps": steps, "flux": [], "gauss": [], "t": []}
    with Simulation(**cfg, precision=precision, capacity=n) as s:
        s.init_plasma(**ld)
        out["flux"].append(s.reconnected_flux())
        out["gauss"].append(s.gauss_residual())
        out["t"].append(0)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(every, steps - done)
            s.step(k, sort_every=1)
            done += k
            out["flux"].append(s.reconnected_flux())
            out["gauss"].append(s.gauss_residual())
            out["t"].append(done)
        s.synchronize()
        out["seconds"] = time.perf_counter() - t0
        hist = s.energy_history()
        out["status"] = s.status()
    tot = hist.sum(axis=1)
    out["energy_total"] = tot
    out["drift_end"] = float(abs(tot[-1] / tot[0] - 1.0))
    out["drift_max"] = float(np.max(np.abs(tot / tot[0] - 1.0)))
    return out


def differences(a, b):
    ea, eb = a["energy_total"], b["energy_total"]
    rows = min(len(ea), len(eb))
    rel_e = np.abs(ea[:rows] - eb[:rows]) / np.abs(eb[:rows])
    fa, fb = np.array(a["flux"]), np.array(b["flux"])
    scale = max(float(np.max(np.abs(fb))), 1e-300)
    return {"total_energy_rel_diff_max": float(rel_e.max()),
            "flux_diff_rel_to_max_flux": [float(x) for x in np.abs(fa - fb) / scale]}


def compare(workload, steps, every, control=False):
    m = run(workload, steps, every, "fp32")
    d = run(workload, steps, every, "fp64")
    extra = {}
    if control:
        d2 = run(workload, steps, every, "fp64")
        extra["fp64_vs_fp64"] = differences(d2, d)
        extra["fp32_vs_fp64_flux"] = differences(m, d)["flux_diff_rel_to_max_flux"]
        d2.pop("energy_total")
    em, ed = m.pop("energy_total"), d.pop("energy_total")
    rows = min(len(em), len(ed))
    rel_e = np.abs(em[:rows] - ed[:rows]) / np.abs(ed[:rows])
    fm, fd = np.array(m["flux"]), np.array(d["flux"])
    scale = max(float(np.max(np.abs(fd))), 1e-300)
    return {
        "workload": workload, "steps": steps, "record_every": every,
        "fp32_mixed": m, "fp64_plain": d,
        "total_energy_rel_diff_max": float(rel_e.max()),
        "total_energy_rel_diff_end": float(rel_e[-1]),
        "flux_diff_max_rel_to_max_flux": float(np.max(np.abs(fm - fd)) / scale),
        "gauss_mixed_max": float(max(m["gauss"])), "gauss_fp64_max": float(max(d["gauss"])),
        **extra,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="harris_1024x512_ppc100", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--control", action="store_true", help="a second FP64 run for the chaotic spread")
    args = ap.parse_args()
    print(json.dumps(compare(args.workload, args.steps, args.every, args.control)), flush=True)


if __name__ == "__main__":
    main()
