"""The N > 1 path of the benchmark on CPU: two ranks over gloo run
independent replicas (each its own seed; here the CPU oracle stands in for
the GPU step), meet only at a barrier and in the max-reduction of their
times, and the job throughput is world x units x steps / max time."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from oracle import oracle as O
    from pbpic_b200 import configs
    from pbpic_b200.replicas import Ranks
    r = Ranks("gloo", timeout_s=60)
    cfg, ld = configs.uniform_c1(mx=16, my=8, ppc=2, seed=r.replica_seed(0))
    p, yee = O.load_plasma(cfg, ld)
    o = O.Oracle(**cfg)
    o.load_particles(p)
    o.set_fields(yee)
    r.barrier()
    for _ in range(3):
        o.pusher()
        o.fieldsolver()
    my_ms = 10.0 * (rank + 1)  # a stand-in for the rank's device time
    mx = r.max(my_ms)
    thr = r.throughput(len(p), 3, mx)
    res = dict(rank=rank, seed=ld["seed"], max=mx, thr=thr, n=len(p), energy=o.energies().tolist())
    r.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_replicas_over_gloo(tmp_path):
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert res[0]["seed"] != res[1]["seed"]
    assert res[0]["max"] == res[1]["max"] == 20.0
    assert res[0]["thr"] == 2 * res[0]["n"] * 3 / 20e-3
    assert not np.allclose(res[0]["energy"], res[1]["energy"])  # independent plasmas
