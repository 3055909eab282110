"""Gradient check of the differentiable form on the GEM Harris sheet.

    python -m pbpic_b200.diffcheck --mx 256 --my 128 --ppc 64 --steps 400 --every 20 --seed 3

For each loss (time-integrated magnetic energy; time-integrated work j.E of
the electric field on the particles) and each horizon (number of steps), the
run takes the gradient of the loss with respect to (psi0, nb, Ti/Te) at
(0.1, 0.2, 5) three ways:
  - the adjoint with the FP32 forward (checkpoints every `--every` steps),
  - the adjoint with the FP64 forward,
  - central finite differences of the FP64 forward at the relative steps
    `--fd` (1e-3, the workload's stated step, and smaller ones),
and reports their relative differences and the time of one FP32 forward plus
adjoint (wall time with the device synchronised on both sides, after one
untimed gradient; both calls end synchronised). The
loss of a reconnecting sheet is piecewise smooth in the parameters (every
cell-crossing decision is a jump), so a finite-difference quotient over many
steps averages over the jumps its step covers; the table shows up to which
horizon the adjoint (the derivative of the smooth pieces) and the quotients
agree. Output: one JSON object.
"""
import argparse
import json
import time

import numpy as np

from .autograd import DiffEngine

BASE = dict(psi0=0.1, nb=0.2, ti_te=5.0)
KEYS = ("psi0", "nb", "ti_te")


def central_fd(eng, rel):
    out = []
    for k in KEYS:
        h = rel * BASE[k]
        lp = eng.forward(**dict(BASE, **{k: BASE[k] + h}))
        lm = eng.forward(**dict(BASE, **{k: BASE[k] - h}))
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def gradient(mx, my, ppc, steps, every, precision, loss, seed, timed=False):
    """(open engine, loss, adjoint gradient, ms of one timed forward + adjoint)."""
    import torch
    e = DiffEngine(mx, my, ppc, nsteps=steps, checkpoint_every=min(every, steps), precision=precision, seed=seed,
                   loss=loss)
    value = e.forward(**BASE)
    g = np.array(e.backward())
    ms = None
    if timed:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.forward(**BASE)
        e.backward()
        torch.cuda.synchronize()
        ms = 1e3 * (time.perf_counter() - t0)
    return e, value, g, ms


def check(mx, my, ppc, horizons, every, fds, seed, losses):
    out = {"grid": f"{mx}x{my}", "ppc_per_species": ppc, "particles": 2 * ppc * mx * my, "checkpoint_every": every,
           "seed": seed, "at": BASE, "losses": {}}
    for loss in losses:
        rows = []
        for steps in horizons:
            e32, v32, g32, ms = gradient(mx, my, ppc, steps, every, "fp32", loss, seed, timed=True)
            e32.close()
            e64, v64, g64, _ = gradient(mx, my, ppc, steps, every, "fp64", loss, seed)
            with e64:
                fd = {str(r): central_fd(e64, r) for r in fds}
            row = {"steps": steps, "loss_fp32": v32, "loss_fp64": v64, "adjoint_fp32": g32.tolist(),
                   "adjoint_fp64": g64.tolist(),
                   "fp32_vs_fp64": (np.abs(g32 - g64) / np.abs(g64)).tolist(),
                   "fd": {r: v.tolist() for r, v in fd.items()},
                   "adjoint_fp64_vs_fd": {r: (np.abs(g64 - v) / np.abs(v)).tolist() for r, v in fd.items()},
                   "forward_plus_adjoint_ms_fp32": ms}
            rows.append(row)
            print(json.dumps({"loss": loss, **row}), flush=True)
        out["losses"][loss] = rows
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mx", type=int, default=256)
    ap.add_argument("--my", type=int, default=128)
    ap.add_argument("--ppc", type=int, default=64)
    ap.add_argument("--steps", default="10,20,50,100,200,400", help="horizons, comma separated")
    ap.add_argument("--every", type=int, default=20)
    ap.add_argument("--fd", default="1e-3,1e-5,1e-7", help="relative finite-difference steps")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--loss", default="jdote,magnetic")
    a = ap.parse_args()
    res = check(a.mx, a.my, a.ppc, [int(x) for x in a.steps.split(",")], a.every,
                [float(x) for x in a.fd.split(",")], a.seed, a.loss.split(","))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
