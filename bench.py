#!/usr/bin/env python
"""Benchmark of the pbpic B200 step: particle-steps/s on one B200, FP32 mixed
vs FP64 plain, at a stated energy error.

Workload: the GEM Harris sheet on 1024x512 cells with 100 particles per cell
per species (104,857,600 particles), conducting walls in y, seeded synthetic
loading. A step is push + field solve + counting sort (sort every step).
Timing: device time with CUDA events on the library's stream, warm-up steps
untimed, max over ranks. The particle state (2.5 GB mixed, 4.6 GB plain) is
far larger than L2, so no flush is needed between steps.

--impl reference times the CPU restatement of the reference (oracle/, OpenMP
over all host threads, FP64) on the whole workload with the same warm-up and
timed steps; the GPU arm's cpu_baseline times it on a bounded sample.
Multi-GPU (N > 1, one process per GPU): the reference's y-slab decomposition,
weak-scaled -- the Harris sheet on 1024 x (512 N) cells, 512 own rows per
rank, ghost bands and ghost field rows exchanged with the neighbours over
NCCL point-to-point every step (pbpic_b200/slab.py); --replicas runs N
independent replicas instead. --slabs runs the slab path at one GPU too.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200: FP32 mixed vs FP64 plain at stated energy error"
# DRAM bytes per particle of one launch of the mixed-form push as benchmarked (read + write: the
# state read through the sort's permutation, the permutation itself, the state written in cell
# order), from the ncu capture of the 512x256 sheet summarised in
# profiles/k_push_fp32_harris_512x256_ppc100.txt; traffic grows in proportion to the particles.
PUSH_DRAM_BYTES_PER_PARTICLE = 61.2
PUSH_KERNEL = "k_push<float,true,true,false,true>"
UNIT = "particle-steps/s"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="harris_1024x512_ppc100")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="time the FP64 plain form only (profiling)")
    ap.add_argument("--sort-every", type=int, default=1)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-steps", type=int, default=20)
    ap.add_argument("--no-c5", action="store_true", help="skip the 4096x2048 Harris sheet (1.68 G particles)")
    ap.add_argument("--c5-steps", type=int, default=10)
    ap.add_argument("--c5-sub-steps", type=int, default=200,
                    help="steps of the FP32-vs-FP64 comparison on the 1024x512 subsample of that sheet")
    ap.add_argument("--slabs", action="store_true",
                    help="run the y-slab decomposition also at one GPU (it is the default for N > 1)")
    ap.add_argument("--replicas", action="store_true", help="N > 1: independent replicas instead of y slabs")
    ap.add_argument("--slab-rows", type=int, default=512, help="own cell rows per rank of the y-slab run")
    return ap.parse_args(argv)


def workload(name, seed_offset=0):
    from pbpic_b200 import configs
    cfg, ld = configs.WORKLOADS[name]()
    ld = dict(ld, seed=ld["seed"] + seed_offset)
    return cfg, ld


def workload_kind(name):
    """What the workload's plasma is, in words."""
    if name.startswith("double_harris"):
        return "double Harris sheet (the reference's own run)"
    if name.startswith("harris"):
        return "GEM Harris sheet"
    return "uniform periodic plasma"


L2_BYTES = 126e6  # B200 L2


def workload_config(name, n):
    """The `config` object of a workload: its grid, particles, boundaries and
    whether its particle state exceeds L2 (no flush needed between steps)."""
    cfg, ld = workload(name)
    s32, s64 = 24.0 * n, 44.0 * n
    if s32 > L2_BYTES:
        l2 = f"inputs larger than L2 (particle state {s32 / 1e9:.2f} GB FP32, {s64 / 1e9:.2f} GB FP64; L2 126 MB)"
    else:
        l2 = f"particle state {s32 / 1e6:.0f} MB FP32 fits in L2 (126 MB); no flush between steps"
    return {"workload": name, "grid": f"{cfg['mx']}x{cfg['my']}", "particles": n,
            "ppc_per_species": ld["ppc"], "ybc": "conducting" if cfg["ybc"] == 1 else "periodic",
            "xbc": "periodic", "seed": ld["seed"], "l2": l2}


# HBM3e of an HGX B200 as specified (the roofline's denominator is the measured copy bandwidth)
NOMINAL_HBM_GBS = 7700.0


def host_cpu():
    """Host threads and CPU model of the machine the CPU baseline runs on."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.lines = []
        self.active = False
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            if self.active:
                self.lines.append(line.strip())

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------- GPU
def run_gpu(args, ranks):
    import torch

    import pbpic_b200

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    cfg, ld = workload(args.workload, seed_offset=ranks.replica_seed(0))
    barrier, max_over_ranks = ranks.barrier, ranks.max
    world = ranks.world

    results = {}
    sampler = ClockSampler(dev)
    for prec in [p for p in ("fp32", "fp64") if not (p == "fp32" and args.no_fp32) and not (p == "fp64" and args.no_fp64)]:
        n = pbpic_b200.Simulation(**cfg, precision=prec, capacity=1).loader_count(**ld)
        # sort every step: the push and the counting sort are timed as separate
        # calls; another cadence: the library's default, the push sorts anyway
        opts = pbpic_b200.OPT_NO_AUTOSORT if args.sort_every == 1 else 0
        with pbpic_b200.Simulation(**cfg, precision=prec, capacity=n, options=opts) as s:
            s.set_stream(stream.cuda_stream)
            s.init_plasma(**ld)
            s.step(args.warmup, sort_every=args.sort_every)
            s.synchronize()
            barrier()
            torch.cuda.synchronize()
            K = args.steps
            launches0 = pbpic_b200.kernel_launches()
            if prec == "fp32":
                sampler.active = True
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for k in range(K):  # the library's step (pbpic_step): the push, then the field solve beside the sort
                s.step(1, sort_every=args.sort_every)
            end.record(stream)
            torch.cuda.synchronize()
            sampler.active = False
            launches = pbpic_b200.kernel_launches() - launches0
            barrier()
            total_ms = max_over_ranks(start.elapsed_time(end))
            # the phases: K more steps as the three calls in order, with events between them
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
            start.record(stream)
            for k in range(K):
                ev[k][0].record(stream)
                s.pusher()
                ev[k][1].record(stream)
                s.fieldsolver()
                ev[k][2].record(stream)
                if args.sort_every > 0 and s.itime() % args.sort_every == 0:
                    s.countingsort()
                ev[k][3].record(stream)
            end.record(stream)
            torch.cuda.synchronize()
            separate_ms = max_over_ranks(start.elapsed_time(end))
            t_push = np.mean([e[0].elapsed_time(e[1]) for e in ev])
            t_field = np.mean([e[1].elapsed_time(e[2]) for e in ev])
            t_sort = np.mean([e[2].elapsed_time(e[3]) for e in ev])
            hist = s.energy_history()
            tot = hist.sum(axis=1)
            results[prec] = dict(n=n, total_ms=total_ms, ms_per_step=total_ms / K, separate_ms_per_step=separate_ms / K,
                                 t_push=t_push, t_field=t_field,
                                 t_sort=t_sort, launches=launches, hist=hist,
                                 energy_drift=float(abs(tot[-1] / tot[0] - 1.0)),
                                 gauss=s.gauss_residual(), flux=s.reconnected_flux(), status=s.status())
    clocks = sampler.stop()

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, cfg, ld, stream, barrier, max_over_ranks)
    ens = None
    if not args.no_ensemble and world == 1:
        try:
            ens = run_ensemble(args)
        except Exception as exc:  # reported in the line; the headline stands on its own
            ens = dict(error=f"{type(exc).__name__}: {exc}")
    c5 = None
    if not args.no_c5 and world == 1:
        try:
            c5 = run_c5(args, stream)
        except Exception as exc:  # reported in the line; the headline stands on its own
            c5 = dict(error=f"{type(exc).__name__}: {exc}")
    return cfg, results, clocks, e2e, dict(ensemble=ens, c5=c5)


def run_e2e(args, cfg, ld, stream, barrier, max_over_ranks):
    """The same step through the C ABI with host-resident reference records:
    H2D of the initial particles (pinned), K steps each followed by a D2H read
    of the energies (totene row), and a D2H store of the final particles."""
    import torch

    import pbpic_b200
    prec = "fp32"
    n = pbpic_b200.Simulation(**cfg, precision=prec, capacity=1).loader_count(**ld)
    host = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True).numpy().view(pbpic_b200.PARTICLE_F32)
    out = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True).numpy().view(pbpic_b200.PARTICLE_F32)
    K = args.steps
    with pbpic_b200.Simulation(**cfg, precision=prec, capacity=n) as s:
        s.set_stream(stream.cuda_stream)
        s.init_plasma(**ld)
        import ctypes
        from pbpic_b200 import _lib as L
        got = ctypes.c_int64()
        L.check(L.lib().pbpic_store_particles_f32(s.handle, L.ptr(host), n, ctypes.byref(got)))
        en = torch.empty(4, dtype=torch.float64, pin_memory=True).numpy()
        s.step(args.warmup, sort_every=1)
        s.synchronize()
        barrier()
        t0 = time.perf_counter()
        L.check(L.lib().pbpic_load_particles_f32(s.handle, L.ptr(host), n))
        s.countingsort()
        for _ in range(K):
            s.step(1, sort_every=args.sort_every)
            L.check(L.lib().pbpic_energies(s.handle, L.ptr(en)))
        L.check(L.lib().pbpic_store_particles_f32(s.handle, L.ptr(out), n, ctypes.byref(got)))
        dt = time.perf_counter() - t0
    dt = max_over_ranks(dt)
    return dict(seconds=dt, n=n, K=K, h2d=n * 32 / K, d2h=32 + n * 32 / K)


def timed_steps(s, stream, K):
    """K steps (push, field solve, sort as separate calls) timed with CUDA
    events on the handle's stream: total ms and the mean ms of each phase."""
    import torch
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for k in range(K):
        ev[k][0].record(stream)
        s.pusher()
        ev[k][1].record(stream)
        s.fieldsolver()
        ev[k][2].record(stream)
        s.countingsort()
        ev[k][3].record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    return (start.elapsed_time(end), float(np.mean([e[0].elapsed_time(e[1]) for e in ev])),
            float(np.mean([e[1].elapsed_time(e[2]) for e in ev])), float(np.mean([e[2].elapsed_time(e[3]) for e in ev])))


def run_c5(args, stream):
    """The large Harris sheet: 4096 x 2048 cells of 0.05 d_i, 100 particles per
    cell per species (1,677,721,600 particles, 40 GB of FP32 state, 114 GB
    with the sort's second buffer and tables), mi/me = 100, nb = 0.1, guide
    field 0.2, seed 4, FP32 mixed, sort every step: device-timed steps with
    per-phase times. Its energy error: the FP32 mixed and FP64 plain forms
    stepped side by side on a 1024 x 512 subsample of the same sheet (the same
    cell size and physics), their largest relative total-energy difference."""
    import pbpic_b200
    from pbpic_b200 import configs
    cfg, ld = configs.harris_c5()
    n = pbpic_b200.Simulation(**cfg, precision="fp32", capacity=1).loader_count(**ld)
    with pbpic_b200.Simulation(**cfg, precision="fp32", capacity=n, options=pbpic_b200.OPT_NO_AUTOSORT) as s:
        s.set_stream(stream.cuda_stream)
        s.init_plasma(**ld)
        s.step(max(args.warmup, 3), sort_every=1)
        s.synchronize()
        import torch
        l0 = pbpic_b200.kernel_launches()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.c5_steps):  # the library's step; then the phases as separate calls
            s.step(1, sort_every=1)
        b.record(stream)
        torch.cuda.synchronize()
        total = a.elapsed_time(b)
        launches = pbpic_b200.kernel_launches() - l0
        _, tp, tf, ts = timed_steps(s, stream, args.c5_steps)
        status = s.status()
        gauss = s.gauss_residual()
    K = args.c5_steps
    sub_cfg, sub_ld = configs.harris(1024, 512, 100, seed=4, mime=100.0, nb=0.1, bguide=0.2, dx=0.05)
    hist = {}
    for prec in ("fp32", "fp64"):
        m = pbpic_b200.Simulation(**sub_cfg, precision=prec, capacity=1).loader_count(**sub_ld)
        with pbpic_b200.Simulation(**sub_cfg, precision=prec, capacity=m) as s:
            s.set_stream(stream.cuda_stream)
            s.init_plasma(**sub_ld)
            s.step(args.c5_sub_steps, sort_every=1)
            hist[prec] = s.energy_history().sum(axis=1)
    rel = np.abs(hist["fp32"] - hist["fp64"]) / np.abs(hist["fp64"])
    return {"workload": "harris_4096x2048_ppc100 (mi/me 100, nb 0.1, guide field 0.2, dx 0.05, seed 4)",
            "particles": n, "steps": K, "ms_per_step": total / K, "value": n * K / (total * 1e-3), "unit": UNIT,
            "phase_ms": {"push": tp, "fieldsolve": tf, "sort": ts},
            "push_gbs": 48.0 * n / (tp * 1e-3) / 1e9, "sort_gbs_8B": 8.0 * n / (ts * 1e-3) / 1e9,
            "gpu_launches": launches, "gauss_residual": gauss, "status": status,
            "energy_error_subsample": {"grid": "1024x512", "steps": args.c5_sub_steps,
                                       "mixed_vs_fp64_total_energy_rel_err_max": float(rel.max()),
                                       "fp32_drift": float(abs(hist["fp32"][-1] / hist["fp32"][0] - 1.0)),
                                       "fp64_drift": float(abs(hist["fp64"][-1] / hist["fp64"][0] - 1.0))}}


def run_ensemble(args):
    """The batched ensemble: 64 two-stream / Weibel instances of uneven size
    (194M particles in all), FP32. Tiles autotuned (its trial steps are steps
    of the run), then K batched steps timed with CUDA events on the batch's
    stream, against K steps of the same domains launched one instance at a
    time (pbpic_step per domain, the same tiles)."""
    import torch

    from pbpic_b200 import configs
    from pbpic_b200.batch import Batch
    from pbpic_b200.sim import kernel_launches
    doms = configs.ensemble_c3()
    n = configs.ensemble_particles(doms)
    K = args.ensemble_steps
    with Batch(doms) as b:
        st = torch.cuda.ExternalStream(b.stream)
        tiles, groups, tune_ms = b.autotune(8)
        b.step(max(2, args.warmup))
        b.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        l0 = kernel_launches()
        ev[0].record(st)
        b.step(K)
        ev[1].record(st)
        b.synchronize()
        l1 = kernel_launches()
        sims = [b.domain(d) for d in range(len(doms))]
        ev[2].record(st)
        for _ in range(K):
            for s in sims:
                s.step(1, sort_every=1)
        ev[3].record(st)
        b.synchronize()
        l2 = kernel_launches()
        t_batch = ev[0].elapsed_time(ev[1])
        t_single = ev[2].elapsed_time(ev[3])
        gauss = max(s.gauss_residual() for s in sims[1::2])  # Weibel: mobile ions, residual starts at 0
        status = 0
        for s in sims:
            status |= s.status()
        return dict(n=n, K=K, t_batch=t_batch, t_single=t_single, tiles=sorted(set(int(t) for t in tiles)),
                    groups=groups, tune_ms=tune_ms, launches_batch=l1 - l0, launches_single=l2 - l1,
                    gauss=gauss, status=status)


# ------------------------------------------------------------- y slabs (N > 1)
def slab_workload(world, rows=512, mx=1024, ppc=100, seed=1):
    """The benchmark's Harris sheet weak-scaled over y slabs: mx x (rows * world)
    cells of 0.1 d_i, 100 particles per cell per species, conducting walls in
    y, the sheet in the middle of the global domain; each rank owns `rows` rows."""
    from pbpic_b200 import configs
    return configs.harris(mx, rows * world, ppc, seed)


def gpu_slab_engine(cfg, ld, lay, precision="fp32"):
    """This rank's slab of the global plasma on its GPU: the loader draws the
    whole plasma on the device (by pair index, so every rank draws the same
    one), the slab's own rows and field rows are cut out with the band and
    row API, the global handle is freed, and the slab handle is filled from
    the cut. Returns the engine (ghost bands are filled by SlabRun.start)."""
    import ctypes

    import torch

    from pbpic_b200 import _lib as L
    from pbpic_b200.sim import Simulation
    from pbpic_b200.slab import GpuEngine
    lib = L.lib()
    rec = L.PARTICLE_F32 if precision == "fp32" else L.PARTICLE_F64
    ftype = torch.float32 if precision == "fp32" else torch.float64
    n = Simulation(**cfg, precision=precision, capacity=1).loader_count(**ld)
    rows = lay.own + (1 if lay.wall_hi >= 0 else 0)  # the top wall's node row on the last slab
    cnt = ctypes.c_int64()
    with Simulation(**cfg, precision=precision, capacity=n) as g:
        g.init_plasma(**ld)
        rc = lib.pbpic_band_extract(g.handle, lay.y0, lay.y1, lay.my, 0, None, 0, ctypes.byref(cnt))
        if rc not in (L.PBPIC_OK, L.ERR_CAPACITY):
            L.check(rc)
        own = cnt.value
        band = torch.empty(max(own, 1) * rec.itemsize, dtype=torch.uint8, device="cuda")
        L.check(lib.pbpic_band_extract(g.handle, lay.y0, lay.y1, lay.my, 0, ctypes.c_void_p(band.data_ptr()), own,
                                       ctypes.byref(cnt)))
        f = torch.empty(6 * cfg["mx"] * rows, dtype=ftype, device="cuda")
        L.check(lib.pbpic_field_rows_get(g.handle, lay.y0, rows, ctypes.c_void_p(f.data_ptr())))
    # own particles plus room for two sets of ghost bands (the bands a step receives are converted
    # after the particles it holds, which include the last bands): 8 rows on each side, a sheet
    # row holding up to 6x the mean
    cap = own + 2 * 8 * 6 * (own // max(lay.own, 1)) + (1 << 20)
    e = GpuEngine(cfg, lay, precision, capacity=cap)
    e.append(band[: own * rec.itemsize], lay.row_offset)
    del band
    e.set_field_rows(lay.lo, rows, f)
    return e


class CudaClock:
    """Device time of a region on the current stream (CUDA events)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)

    def sync(self):
        self.torch.cuda.synchronize()

    def start(self):
        self.a.record()

    def stop(self):
        self.b.record()
        self.b.synchronize()
        return self.a.elapsed_time(self.b)


class HostClock:
    """Wall time of a region (CPU engines)."""

    def sync(self):
        pass

    def start(self):
        self.t0 = time.perf_counter()

    def stop(self):
        return 1e3 * (time.perf_counter() - self.t0)


def run_slabs(ranks, transport, engine, steps, warmup, clock, counter=None):
    """The y-slab step on every rank: `warmup` untimed steps, then `steps`
    timed ones (push, field solve, ghost-band and ghost-row exchange with the
    neighbours, sort), a barrier and a synchronisation on both sides, the
    slowest rank's time. Work units are the own particles of every rank (the
    ghosts each rank also pushes are redundant work). Every rank returns the
    same dict."""
    from pbpic_b200.slab import SlabRun
    run = SlabRun({ranks.rank: engine}, transport)
    run.start()
    run.step(warmup)
    clock.sync()
    ranks.barrier()
    l0 = counter() if counter else 0
    clock.start()
    run.step(steps)
    ms = clock.stop()
    launches = (counter() - l0) if counter else None
    ranks.barrier()
    ms = ranks.max(ms)
    own = float(transport.allreduce([engine.own_count()], "sum")[0])
    en = run.energies()
    gauss = run.gauss_residual()
    return dict(ms=ms, own=own, value=own * steps / (ms * 1e-3), energies=en.tolist(), gauss=gauss,
                launches=launches)


def run_slabs_e2e(ranks, transport, cfg, lay, host_rec, fields, steps, make_engine):
    """The y-slab step end to end: each rank's own particle records go from
    pinned host memory to its GPU (H2D) and into a fresh slab, the ghost bands
    are exchanged, `steps` steps run with the all-reduced energies read back
    to the host after every step, and the own particles come back to pinned
    host memory (D2H). Wall time, the slowest rank's."""
    import torch

    from pbpic_b200.slab import SlabRun
    e = make_engine()
    dev = torch.empty(host_rec.numel(), dtype=torch.uint8, device="cuda")
    out = torch.empty_like(host_rec).pin_memory()
    torch.cuda.synchronize()
    ranks.barrier()
    t0 = time.perf_counter()
    dev.copy_(host_rec, non_blocking=True)
    e.append(dev, lay.row_offset)
    e.set_field_rows(lay.lo, fields.numel() // (6 * cfg["mx"]), fields)
    run = SlabRun({ranks.rank: e}, transport)
    run.start()
    for _ in range(steps):
        run.step(1)
        run.energies()
    back = e.extract(lay.lo, lay.hi, 2)
    out[: back.numel()].copy_(back)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    ranks.barrier()
    return ranks.max(dt), host_rec.numel(), back.numel()


def slab_line(args, ranks):
    """The JSON line of the y-slab run on N GPUs (one slab per rank, NCCL
    point-to-point exchanges between neighbours, FP32 mixed form)."""
    import torch

    from pbpic_b200.slab import Layout, TorchDist
    dev = ranks.local_rank
    torch.cuda.set_device(dev)
    cfg, ld = slab_workload(ranks.world, rows=args.slab_rows)
    lay = Layout(cfg["my"], ranks.world, ranks.rank, cfg["ybc"])
    transport = TorchDist(ranks.dist, f"cuda:{dev}") if ranks.dist is not None else SelfTransport()
    import pbpic_b200
    eng = gpu_slab_engine(cfg, ld, lay)
    sampler = ClockSampler(dev)
    sampler.active = True
    r = run_slabs(ranks, transport, eng, args.steps, args.warmup, CudaClock(), pbpic_b200.kernel_launches)
    sampler.active = False
    clocks = sampler.stop()
    e2e = None
    if not args.no_e2e:
        rows = lay.own + (1 if lay.wall_hi >= 0 else 0)
        band = eng.extract(lay.lo, lay.hi, 2)
        host = torch.empty(band.numel(), dtype=torch.uint8).pin_memory()
        host.copy_(band)
        fields = eng.field_rows(lay.lo, rows).clone()
        cap = eng.sim.cfg.capacity
        del band, eng
        torch.cuda.empty_cache()
        from pbpic_b200.slab import GpuEngine
        sec, h2d, d2h = run_slabs_e2e(ranks, transport, cfg, lay, host, fields, args.steps,
                                      lambda: GpuEngine(cfg, lay, "fp32", capacity=cap))
        tot = transport.allreduce([h2d, d2h], "sum")
        e2e = {"value": r["own"] * args.steps / sec, "unit": UNIT, "h2d_bytes_per_step": float(tot[0]) / args.steps,
               "d2h_bytes_per_step": float(tot[1]) / args.steps + 32.0, "K": args.steps,
               "what": "every rank: H2D of its own particle records (pinned) into a fresh slab, ghost-band exchange, "
                       "K steps each reading the all-reduced energies back, D2H of its own particles; the two "
                       "state copies are shared by the K steps"}
    peak, peak_kind = measured_peak_hbm()
    n = int(r["own"])
    cells = cfg["mx"] * cfg["my"]
    step_bytes = 96.0 * n + 60.0 * cells  # push 48 B + sort 48 B per particle, grid 60 B per cell
    return {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (int64 fixed-point current, f64 energies)",
        "data": "synthetic: seeded Philox GEM Harris sheet",
        "config": {"workload": f"harris_{cfg['mx']}x{cfg['my']}_ppc{ld['ppc']}_yslabs",
                   "grid": f"{cfg['mx']}x{cfg['my']}", "particles": n, "ppc_per_species": ld["ppc"],
                   "rows_per_rank": args.slab_rows, "ghost_rows": lay.g, "ybc": "conducting", "xbc": "periodic",
                   "seed": ld["seed"], "step": "push+fieldsolve+exchange+sort", "sort_every": 1,
                   "l2": "inputs larger than L2 (particle state per rank about 2.5 GB FP32)",
                   "parallelism": f"y-slabs x{ranks.world} (NCCL point-to-point ghost bands and rows)"},
        "roofline": {"bound": "hbm", "step_frac": step_bytes / (r["ms"] / args.steps * 1e-3) / 1e9 / ranks.world / peak,
                     "peak": peak, "unit": "GB/s", "peak_kind": peak_kind},
        "energy": {"total": float(sum(r["energies"])), "gauss_residual": r["gauss"]},
        "e2e": e2e,
        "gpu_launches": r["launches"],
        "clocks": clocks,
    }


class SelfTransport:
    """One slab in one process (a single GPU): every exchange is with itself."""

    def allreduce(self, values, op):
        import numpy as np
        return np.asarray(values, dtype=np.float64)

    def exchange(self, slabs, outgoing):
        from pbpic_b200.slab import InProcess
        return InProcess().exchange(slabs, outgoing)


# ---------------------------------------------------------------------- CPU
def run_cpu_sample(workload_name, steps, seed_offset=0):
    """The oracle (OpenMP over all host threads) on a bounded sample of the
    workload: the same grid and physics with 1/4 of the particles per cell."""
    from oracle import oracle as O
    from pbpic_b200 import configs
    base = configs.WORKLOADS[workload_name]
    cfg, ld = base()
    ppc = max(1, ld["ppc"] // 4)
    if workload_name.startswith("harris"):
        cfg, ld = configs.harris(cfg["mx"], cfg["my"], ppc, ld["seed"] + seed_offset,
                                 mime=cfg["mime"], nb=ld["nb"], bguide=ld["bguide"], dx=cfg["dx"])
    else:
        cfg, ld = base(mx=cfg["mx"], my=cfg["my"], ppc=ppc)
    p, yee = O.load_plasma(cfg, ld)
    o = O.Oracle(**cfg)
    o.load_particles(p)
    del p
    o.set_fields(yee)
    nth = O.max_threads()
    o.omp_countingsort(nth)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.omp_pusher(nth)
        o.fieldsolver()
        o.omp_countingsort(nth)
    dt = time.perf_counter() - t0
    n = o.L.orc_nptl(o.h)
    o.close()
    return dict(value=n * steps / dt, cores=nth, n=n, steps=steps, seconds=dt,
                sample=f"{cfg['mx']}x{cfg['my']} cells, {ppc} particles/cell/species ({n} particles), {steps} steps "
                       "of push+fieldsolve+sort, FP64, OpenMP over all host threads")


def run_cpu_full(workload_name, steps, warmup):
    """The oracle (OpenMP over all host threads, FP64) on the whole workload:
    `warmup` untimed steps, then `steps` timed steps of push + field solve +
    sort, as the GPU arm runs them."""
    from oracle import oracle as O
    cfg, ld = workload(workload_name)
    p, yee = O.load_plasma(cfg, ld)
    o = O.Oracle(**cfg)
    o.load_particles(p)
    n = len(p)
    del p
    o.set_fields(yee)
    nth = O.max_threads()
    o.omp_countingsort(nth)

    def one():
        o.omp_pusher(nth)
        o.fieldsolver()
        o.omp_countingsort(nth)

    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    dt = time.perf_counter() - t0
    o.close()
    return dict(value=n * steps / dt, cores=nth, n=n, steps=steps, warmup=warmup, seconds=dt,
                sample=f"the whole workload: {cfg['mx']}x{cfg['my']} cells, {n} particles, {warmup} untimed + "
                       f"{steps} timed steps of push+fieldsolve+sort, FP64, OpenMP over all host threads")


def run_cpu_single_f32(steps=3):
    """One host thread of the oracle in FP32 with every compat switch on (the
    reference's own precision and arithmetic) on the 128x128 uniform plasma,
    32 particles per cell per species."""
    from oracle import oracle as O
    from pbpic_b200 import configs
    cfg, ld = configs.uniform_c1()
    p, yee = O.load_plasma(cfg, ld)
    o = O.Oracle(**dict(cfg, compat=7), precision="f32")
    o.load_particles(p)
    del p
    o.set_fields(yee)
    o.countingsort()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.pusher()
        o.fieldsolver()
        o.countingsort()
    dt = time.perf_counter() - t0
    n = o.L.orc_nptl(o.h)
    o.close()
    return {"value": n * steps / dt, "unit": UNIT, "cores": 1,
            "sample": f"{cfg['mx']}x{cfg['my']} cells, {n} particles, {steps} steps of push+fieldsolve+sort, FP32 with "
                      "the compat switches (7), one thread"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        r = run_cpu_full(args.workload, args.steps, args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": r["steps"], "warmup": r["warmup"], "ms_per_step": 1e3 * r["seconds"] / r["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: seeded Philox " + workload_kind(args.workload),
                "config": dict(workload_config(args.workload, r["n"]), sample=r["sample"]),
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "port",
                                 "sample": r["sample"], "host": host_cpu()},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    from pbpic_b200.replicas import Ranks
    ranks = Ranks("nccl")
    if (world > 1 and not args.replicas) or args.slabs:
        line = slab_line(args, ranks)
        ranks.close()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    cfg, res, clocks, e2e, extra = run_gpu(args, ranks)
    ens, c5 = extra["ensemble"], extra["c5"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_sample(args.workload, 4)
        cpu["single_thread_fp32"] = run_cpu_single_f32()
    ranks.close()
    if rank != 0:
        return
    if "fp32" not in res:  # --no-fp32: a profiling run of the plain form
        d = res["fp64"]
        print(json.dumps({"metric": METRIC, "fp64_plain_only": True, "value": d["n"] * args.steps / (d["total_ms"] * 1e-3),
                          "unit": UNIT, "ms_per_step": d["ms_per_step"],
                          "phase_ms": {"push": d["t_push"], "fieldsolve": d["t_field"], "sort": d["t_sort"]}}))
        return
    m = res["fp32"]
    n = m["n"]
    K = args.steps
    value = ranks.throughput(n, K, m["total_ms"])
    peak, peak_kind = measured_peak_hbm()
    bytes_push = 48.0 * n  # read + write of cell (4 B), offsets (2x4 B), momenta (3x4 B)
    achieved_push = bytes_push / (m["t_push"] * 1e-3) / 1e9
    cells = cfg["mx"] * cfg["my"]
    step_bytes = 48.0 * n + (48.0 * n if args.sort_every == 1 else 48.0 * n / max(args.sort_every, 1)) + 60.0 * cells
    # the bytes the step moves: the push's 48 B, the ranking's cell word read and permutation entry
    # written (8 B) at each sort, the grid's 60 B per cell
    step_moved = 48.0 * n + 8.0 * n / max(args.sort_every, 1) + 60.0 * cells
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (int64 fixed-point current, f64 energies)",
        "data": "synthetic: seeded Philox " + workload_kind(args.workload),
        "config": dict(workload_config(args.workload, n),
                       step="push+fieldsolve+sort (pbpic_step: the field solve on a second stream beside the sort)",
                       sort_every=args.sort_every, parallelism=f"replicas x{world}"),
        "roofline": {"bound": "hbm", "achieved": achieved_push, "peak": peak, "unit": "GB/s",
                     "frac": achieved_push / peak,
                     "traffic": PUSH_DRAM_BYTES_PER_PARTICLE * n if PUSH_DRAM_BYTES_PER_PARTICLE else None,
                     "kernel": PUSH_KERNEL,
                     "bytes_per_launch": bytes_push, "peak_kind": peak_kind,
                     "peak_nominal": NOMINAL_HBM_GBS, "frac_nominal": achieved_push / NOMINAL_HBM_GBS,
                     "step_frac": step_bytes / (m["ms_per_step"] * 1e-3) / 1e9 / peak,
                     "step_frac_moved": step_moved / (m["ms_per_step"] * 1e-3) / 1e9 / peak},
        "phase_ms": {"push": m["t_push"], "fieldsolve": m["t_field"], "sort": m["t_sort"],
                     "what": "K further steps as separate calls in order, events between them",
                     "step_separate_calls": m["separate_ms_per_step"]},
        "energy": {"mixed_drift": m["energy_drift"], "gauss_residual": m["gauss"], "reconnected_flux": m["flux"]},
        "gpu_launches": m["launches"],
        "clocks": clocks,
    }
    if "fp64" in res:
        d = res["fp64"]
        vd = world * d["n"] * K / (d["total_ms"] * 1e-3)
        hm, hd = m["hist"], d["hist"]
        rows = min(len(hm), len(hd))
        rel = np.abs(hm[:rows].sum(1) - hd[:rows].sum(1)) / np.abs(hd[:rows].sum(1))
        line["fp64_plain"] = {"value": vd, "ms_per_step": d["ms_per_step"],
                              "phase_ms": {"push": d["t_push"], "fieldsolve": d["t_field"], "sort": d["t_sort"],
                                           "step_separate_calls": d["separate_ms_per_step"]},
                              "push_gbs": 88.0 * d["n"] / (d["t_push"] * 1e-3) / 1e9,
                              "energy_drift": d["energy_drift"], "gauss_residual": d["gauss"]}
        line["mixed_over_fp64"] = value / vd
        line["energy"]["mixed_vs_fp64_total_energy_rel_err_max"] = float(rel.max())
    if e2e:
        line["e2e"] = {"value": world * e2e["n"] * e2e["K"] / e2e["seconds"], "unit": UNIT,
                       "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"], "K": e2e["K"],
                       "what": "H2D of the initial reference particle records (pinned), K steps each with a D2H "
                               "of the energies, D2H of the final particles; the two state copies are shared "
                               "by the K steps, so the figure grows with K"}
    if ens and "error" in ens:
        line["ensemble"] = ens
    elif ens:
        vb = ens["n"] * ens["K"] / (ens["t_batch"] * 1e-3)
        vs = ens["n"] * ens["K"] / (ens["t_single"] * 1e-3)
        line["ensemble"] = {
            "workload": "64 two-stream/Weibel instances, grids 64x64..256x256, 16-128 ppc/species, FP32",
            "particles": ens["n"], "steps": ens["K"], "value": vb, "unit": UNIT,
            "ms_per_step": ens["t_batch"] / ens["K"], "per_instance_value": vs,
            "per_instance_ms_per_step": ens["t_single"] / ens["K"], "batched_over_per_instance": vb / vs,
            "autotuned": {"tile_rows": ens["tiles"], "particles_per_thread": 4 * ens["groups"],
                          "trial_ms_per_step": ens["tune_ms"]},
            "gpu_launches": {"batched": ens["launches_batch"], "per_instance": ens["launches_single"]},
            "step_frac_hbm": 96.0 * ens["n"] * ens["K"] / (ens["t_batch"] * 1e-3) / 1e9 / peak,
            "weibel_gauss_residual_max": ens["gauss"], "status": ens["status"]}
    if c5:
        if "push_gbs" in c5:
            c5["push_frac"] = c5["push_gbs"] / peak
        line["c5"] = c5
    if cpu:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                                "sample": cpu["sample"], "host": host_cpu(),
                                "single_thread_fp32": cpu["single_thread_fp32"]}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
