"""The y-slab decomposition as two gloo ranks on CPU (torch.distributed
point-to-point exchanges of the ghost bands, sizes then payloads), each rank
stepping its slab with the CPU oracle: the own particles and field rows of
the two ranks reproduce the single-domain oracle run within 1e-12 relative
(FP64; the order of the current sums differs), periodic and conducting y, and
every rank's all-reduced energies are the single domain's."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def case(kind):
    from pbpic_b200 import configs
    if kind == "uniform":
        cfg, ld = configs.uniform_c1(seed=31, mx=12, my=20, ppc=3)
        return cfg, dict(ld, vthe=0.3, vthi=0.1)
    return configs.harris(12, 20, 3, seed=32)


def worker(rank, world, port, kind, steps, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    from oracle import oracle as O
    from pbpic_b200.slab import Layout, SlabRun, TorchDist, scatter_plasma
    from slab_oracle import OracleEngine
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    cfg, ld = case(kind)
    p, yee = O.load_plasma(cfg, ld)
    p["pid"] = np.arange(len(p), dtype=np.int32)
    lay = Layout(cfg["my"], world, rank, cfg["ybc"])
    e = OracleEngine(O, cfg, lay)
    lp, lf = scatter_plasma(p, yee, lay)
    e.load(lp, lf)
    run = SlabRun({rank: e}, TorchDist(dist, "cpu"))
    run.start()
    run.step(steps)
    q = e.own_particles()
    f, top = e.own_fields()
    en = run.energies()  # every rank: an all-reduce of the slabs' own-row energies
    dist.destroy_process_group()
    np.save(os.path.join(out_dir, f"e{rank}.npy"), en)
    np.save(os.path.join(out_dir, f"p{rank}.npy"), q)
    np.save(os.path.join(out_dir, f"f{rank}.npy"), f)
    if top is not None:
        np.save(os.path.join(out_dir, f"top{rank}.npy"), top)
    with open(os.path.join(out_dir, f"lay{rank}.json"), "w") as fh:
        json.dump(dict(y0=lay.y0, y1=lay.y1), fh)


@pytest.mark.parametrize("kind", ["uniform", "harris"])
def test_two_slabs_over_gloo_match_single_oracle(oracle_mod, tmp_path, kind):
    world, steps = 2, 4
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=worker, args=(r, world, port, kind, steps, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(180)
        assert pr.exitcode == 0
    cfg, ld = case(kind)
    p, yee = oracle_mod.load_plasma(cfg, ld)
    p["pid"] = np.arange(len(p), dtype=np.int32)
    o = oracle_mod.Oracle(**cfg)
    o.load_particles(p, capacity=4 * len(p))
    o.set_fields(yee)
    o.countingsort()
    for _ in range(steps):
        o.pusher()
        o.fieldsolver()
        o.countingsort()
    ps, fs = o.particles(), o.fields()
    pg = np.concatenate([np.load(tmp_path / f"p{r}.npy") for r in range(world)])
    assert len(pg) == len(ps)
    pg, ps = pg[np.argsort(pg["pid"])], ps[np.argsort(ps["pid"])]
    assert np.array_equal(pg["pid"], ps["pid"]) and np.array_equal(pg["grid"], ps["grid"])
    for c in ("dx", "dy", "ux", "uy", "uz"):
        assert np.abs(pg[c] - ps[c]).max() <= 1e-12 * max(1.0, np.abs(ps[c]).max()), c
    fg = np.zeros_like(fs)
    for r in range(world):
        lay = json.load(open(tmp_path / f"lay{r}.json"))
        fg[:, :, lay["y0"]:lay["y1"]] = np.load(tmp_path / f"f{r}.npy")
        if (tmp_path / f"top{r}.npy").exists():
            fg[:, :, cfg["my"]] = np.load(tmp_path / f"top{r}.npy")
    rows = cfg["my"] + (1 if cfg["ybc"] == 1 else 0)
    assert np.abs(fg[:, :, :rows] - fs[:, :, :rows]).max() <= 1e-12 * np.abs(fs).max()
    es = o.energies()  # the single domain's totene row of its last step
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"e{r}.npy"), es, rtol=1e-10, atol=1e-14 * np.abs(es).max())


class _FixedSlab:
    """A slab whose own-row energies and Gauss residual are fixed numbers."""

    def __init__(self, rank):
        self.e = np.array([1.0, 2.0, 3.0, 4.0]) * (rank + 1)
        self.g = 0.5 - 0.25 * rank

    def energies(self):
        return self.e

    def gauss_residual(self):
        return self.g


def reduce_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    from pbpic_b200.slab import SlabRun, TorchDist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    run = SlabRun({rank: _FixedSlab(rank)}, TorchDist(dist, "cpu"))
    e = run.energies()
    g = run.gauss_residual()
    dist.destroy_process_group()
    np.save(os.path.join(out_dir, f"red{rank}.npy"), np.concatenate([e, [g]]))


def test_slab_energies_and_gauss_reduce_over_ranks(tmp_path):
    """Every rank gets the sum of the slabs' energies and the largest of their
    Gauss residuals (an all-reduce over gloo)."""
    world = 3
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=reduce_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(120)
        assert pr.exitcode == 0
    want = np.concatenate([np.array([1.0, 2.0, 3.0, 4.0]) * 6.0, [0.5]])
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"red{r}.npy"), want)
