"""The benchmark's y-slab path (bench.run_slabs: warm-up, timed steps between
barriers, slowest rank's time, own particles summed over the ranks, energies
and Gauss residual all-reduced) as two gloo ranks on CPU, each rank stepping
its slab with the CPU oracle: every rank reports the same line, the own
particles add up to the whole plasma, and the all-reduced energies equal the
single-domain oracle run's."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np

STEPS, WARMUP = 3, 1


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def case():
    from pbpic_b200 import configs
    return configs.harris(12, 20, 3, seed=41)


def worker(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from oracle import oracle as O
    from pbpic_b200.replicas import Ranks
    from pbpic_b200.slab import Layout, TorchDist, scatter_plasma
    from slab_oracle import OracleEngine
    ranks = Ranks("gloo", timeout_s=60)
    cfg, ld = case()
    p, yee = O.load_plasma(cfg, ld)
    lay = Layout(cfg["my"], world, rank, cfg["ybc"])
    e = OracleEngine(O, cfg, lay)
    lp, lf = scatter_plasma(p, yee, lay)
    e.load(lp, lf)
    r = bench.run_slabs(ranks, TorchDist(ranks.dist, "cpu"), e, STEPS, WARMUP, bench.HostClock())
    ranks.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as fh:
        json.dump({k: r[k] for k in ("ms", "own", "value", "energies", "gauss")}, fh)


def test_bench_slab_path_over_gloo(oracle_mod, tmp_path):
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(180)
        assert pr.exitcode == 0
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    assert res[0] == res[1]  # the slowest rank's time and the all-reduced figures on every rank
    cfg, ld = case()
    p, yee = oracle_mod.load_plasma(cfg, ld)
    assert res[0]["own"] == len(p)
    assert res[0]["value"] > 0
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p, capacity=4 * len(p))
    o.set_fields(yee)
    o.countingsort()
    for _ in range(WARMUP + STEPS):
        o.pusher()
        o.fieldsolver()
        o.countingsort()
    es = o.energies()
    assert np.allclose(res[0]["energies"], es, rtol=1e-10, atol=1e-14 * np.abs(es).max())
    assert res[0]["gauss"] < 1e-12
