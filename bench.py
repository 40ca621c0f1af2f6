#!/usr/bin/env python
"""Benchmark: SPH + Barnes-Hut giant-impact particle-steps/s on one or more B200s.

Default workload (N=1): the 1,048,576-particle impact (953,250 target + 95,326 impactor; 30 % iron /
70 % basalt by mass; Tillotson; Wendland C2 with 64 neighbours and the smoothing-length solve; monopole +
quadrupole Barnes-Hut at θ = 0.6 with 16-particle leaves; adaptive CFL 0.3 dt; FP32 SoA fields with FP64
positions), seeded synthetic initial conditions. One step = one KDK leapfrog step (two force evaluations,
as the reference's encode_kdk). Inputs are resident in HBM and the per-step working set (particle state,
neighbour lists, tree) is larger than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload impact_1m|impact_4m|impact_10k|batch_256|...]
    python bench.py --impl reference ...    # the reference's CPU path (HydroBody::step) on the host cores
    python bench.py --path measure [--measure-workload post_impact_1m] [--variant 0|1]   # disk measurement

Multi-GPU: replicas (one independent impact per rank, no collective on the data path); value is the sum
over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SPH+gravity particle-steps/s"
UNIT = "particle-steps/s"

from botheadstudios_b200.workloads import WORKLOADS, n_particles  # noqa: E402

# Algorithmic bytes per particle per phase execution (state read/written once, SoA f32/f64 layout):
# sort = bbox/Morton 40 + radix (key,idx) 16 + permutation 132; tree = 20 + 304/L per particle;
# gravity 32; neighbours 36 (pos 16 + list write 4·k_avg counted separately); density 28 + EOS 20;
# forces 64; integrate: kick-drift 128 + kick 48 + CFL 36 per step (two phase executions). The gather phases
# also stream each particle's neighbour list from HBM (4 B per entry, once per gather pass): LIST_PASSES.
BYTES_PER_PARTICLE = dict(sort=188.0, tree=39.0, gravity=32.0, neighbours=16.0, hsolve=28.0, density=48.0,
                          forces=64.0, integrate=106.0)


def list_passes(wl: dict) -> dict:
    """Neighbour-list reads per particle per phase call: one per gather pass (the plain smoothing-length solve
    makes h_iters + 1 = 3; the learned form's first check is counted alone, a lower bound)."""
    return dict(forces=1, density=1, hsolve=3 if wl.get("h_solve") == 1 else 1)


def phase_bytes(k: str, wl: dict, lbar: float) -> float:
    return BYTES_PER_PARTICLE[k] + 4.0 * lbar * list_passes(wl).get(k, 0)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return dict(hbm=float(d["hbm_gbs"]), bf16=float(d["bf16_tflops"]), src="measured")
    return dict(hbm=6650.0, bf16=1590.0, src="fallback")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=smax, reasons=sorted(reasons), samples=len(sm))


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def _reduce(pg, v: float, local: int, op: str) -> float:
    """All-reduce one number over the ranks (NCCL on the rank's GPU; gloo on the host)."""
    if pg is None:
        return v
    import torch
    dev = "cpu" if pg.get_backend() == "gloo" else f"cuda:{local}"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=getattr(pg.ReduceOp, op))
    return float(t.item())


def max_over_ranks(pg, v: float, local: int) -> float:
    """The slowest rank's time: replicas are timed on the device, the job takes the maximum."""
    return _reduce(pg, v, local, "MAX")


def sum_over_ranks(pg, v: float, local: int) -> float:
    """Work summed over the replicas (each rank's workload is its own seeded draw, so sizes may differ)."""
    return _reduce(pg, v, local, "SUM")


def replica_value(pg, units_local: float, ms_local: float, local: int) -> float:
    """Whole-job throughput of independent replicas: the units all ranks processed ÷ the slowest rank's time."""
    return sum_over_ranks(pg, units_local, local) / (max_over_ranks(pg, ms_local, local) / 1000.0)


def conservation_drifts(start: list, end: list) -> dict:
    """Drifts over a run from the FP64 device sums of each context (`GpuSph.diag` at its start and end):
    total energy change ÷ |potential| at the start; |ΔP| ÷ sqrt(2·M·KE) at the start (momentum against the
    system's kinetic momentum scale); |ΔL| ÷ |L| at the start (L about the origin). Each context's impacts are
    isolated systems, so the sums over contexts are conserved too; None where the scale is zero."""
    def tot(ds, k):
        return sum(d[k] for d in ds)

    def vec(ds, k):
        return [sum(d[k][i] for d in ds) for i in range(3)]

    def norm(v):
        return math.sqrt(sum(x * x for x in v))

    e0 = tot(start, "kinetic") + tot(start, "internal") + tot(start, "potential")
    e1 = tot(end, "kinetic") + tot(end, "internal") + tot(end, "potential")
    pot0 = abs(tot(start, "potential"))
    p0, p1 = vec(start, "momentum"), vec(end, "momentum")
    l0, l1 = vec(start, "angular_momentum"), vec(end, "angular_momentum")
    pscale = math.sqrt(2.0 * tot(start, "mass") * tot(start, "kinetic"))
    dp = norm([b - a for a, b in zip(p0, p1)])
    dl = norm([b - a for a, b in zip(l0, l1)])
    return dict(energy_drift=(e1 - e0) / pot0 if pot0 else None,
                momentum_drift=dp / pscale if pscale else None,
                angular_momentum_drift=dl / norm(l0) if norm(l0) else None)


def build_workload(wl: dict, seed: int):
    from botheadstudios_b200 import workloads
    return workloads.build(wl, seed)


class SingleRunner:
    """One impact in one context (the interface of batching.BucketedBatch)."""

    def __init__(self, wl: dict, I, device: int):
        from botheadstudios_b200 import workloads
        self.I = I
        self.s = workloads.solver(wl, I, device)
        self.ctxs = [self.s]
        self.n = len(I.particles)
        self.batch = I

    def upload(self, particles=None):
        p = self.I.particles if particles is None else particles
        if hasattr(self.I, "offsets"):
            self.s.upload_batch(p, self.I.offsets, self.I.eos, self.I.softening)
        else:
            self.s.upload(p, self.I.eos, self.I.softening)

    def encode_kdk(self, k):
        self.s.encode_kdk(k)

    def sync(self):
        self.s.sync()

    def readback_into(self, out):
        self.s.readback_into(out)


def make_runner(wl: dict, I, device: int):
    """The runner of a workload and, for a batch, the autotuner's choices and measurements."""
    if wl.get("kind") != "batch":
        return SingleRunner(wl, I, device), None
    from botheadstudios_b200 import batching, workloads
    base = workloads.config(wl, I)
    tuned = None
    choices = {}
    if wl.get("autotune"):
        choices, log = batching.tune_buckets(I, base, device=device)
        tuned = dict(choices={str(b): c for b, c in choices.items()},
                     measured=[dict(c["choice"], rate=round(c["rate"])) for c in log])
    return batching.BucketedBatch(I, base, choices, device=device), tuned


def timed(ctxs, encode, steps: int, local: int) -> float:
    """Device time (ms) of encode(steps) over the contexts `ctxs`: an event on the current stream that every
    context stream waits for, the steps, then an event after every context stream has finished."""
    import torch
    main = torch.cuda.current_stream(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    exts = [torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}") for s in ctxs]
    e0.record(main)
    for x in exts:
        x.wait_event(e0)
    encode(steps)
    for x in exts:
        ev = torch.cuda.Event()
        ev.record(x)
        main.wait_event(ev)
    e1.record(main)
    e1.synchronize()
    return e0.elapsed_time(e1)


def density_error(wl: dict, I, state, device: int) -> dict:
    """Densities of a state (48-byte particles) against a converged smoothing-length solve (8 Newton iterations)
    on the same positions: the accuracy the learned and the plain forms are compared at."""
    from botheadstudios_b200 import workloads
    with workloads.solver(wl, I, device, h_mode=1, h_iters=8) as s:
        s.upload(state, I.eos, I.softening)
        s.eval_forces()
        rho = s.inspect("RHO")
    e = np.abs(state["rho"].astype(np.float64) / rho - 1.0)
    return dict(rms=float(np.sqrt(np.mean(e * e))), max=float(e.max()))


def plain_same(wl: dict, I, device: int, steps: int, warmup: int, h_iters: int = 2) -> dict:
    """The plain GPU form (iterated h: SPH_H_SOLVE with h_iters Newton iterations) on the same initial
    conditions, timed the same way, with the density error of its final state: the comparison of the learned
    form."""
    from botheadstudios_b200 import workloads
    with workloads.solver(wl, I, device, h_mode=1, h_iters=h_iters) as s:
        workloads.upload(s, I)
        s.encode_kdk(warmup)
        s.sync()
        ms = timed([s], s.encode_kdk, steps, max(device, 0))
        d = s.diag()
        state = s.readback()
    return dict(value=len(I.particles) * steps / (ms / 1000.0), ms_per_step=ms / steps, h_iters=h_iters,
                h_residual=d["h_residual"], density_error=density_error(wl, I, state, device))


def plain_batched(wl: dict, B, choices: dict, device: int, steps: int, warmup: int) -> dict:
    """The plain form (iterated h) of a batch with the learned run's tuned choices, contexts and graphs, timed the
    same way: what the learned smoothing length changes with everything else equal."""
    from botheadstudios_b200 import batching, workloads
    base = workloads.config(wl, B, h_mode=1)
    with batching.BucketedBatch(B, base, choices, device=device) as r:
        r.upload()
        r.encode_kdk(warmup)
        r.sync()
        ms = timed(r.ctxs, r.encode_kdk, steps, max(device, 0))
        res = max(d["h_residual"] for d in r.diag())
    return dict(value=r.n * steps / (ms / 1000.0), ms_per_step=ms / steps, h_residual=res, contexts=len(r.ctxs))


def plain_sequential(wl: dict, B, device: int, impacts: int = 16, steps: int = 2) -> dict:
    """The plain GPU form on a batch's impacts: one impact at a time, each in its own context with the
    workload's untuned configuration, no graph (the reference's offline driver runs impacts sequentially)."""
    from botheadstudios_b200 import workloads
    from botheadstudios_b200.gpusph import GpuSph
    tot_ps, tot_ms, res = 0, 0.0, 0.0
    for k in range(min(impacts, B.n_impacts)):
        p = B.impact(k)
        # the plain form is the iterated smoothing-length solve, whatever the workload's own form
        with GpuSph(len(p), device=device, **workloads.config(wl, B, graph=0, h_mode=1)) as s:
            s.upload(p, B.eos, float(B.softening[k]))
            s.encode_kdk(1)
            s.sync()
            tot_ms += timed([s], s.encode_kdk, steps, max(device, 0))
            tot_ps += len(p) * steps
            res = max(res, s.diag()["h_residual"])
    return dict(value=tot_ps / (tot_ms / 1000.0), impacts=min(impacts, B.n_impacts), steps=steps,
                h_residual_max=res)


# ---------------------------------------------------------------------------------------------------------
# CPU baseline: the reference's CPU path of record (HydroBody::step, hydrostatic.rs:345: f64, octree
# Barnes-Hut θ = 0.5, hash-grid neighbours, two force evaluations per KDK step) restated in C++, in the
# reference's own SI units, on the benchmark's own initial conditions (the same seeded workload the GPU arm
# runs). All host cores: OpenMP over the per-particle loops, full KDK steps. One core (the reference's own
# path is single-threaded: no rayon in its Cargo.lock): one force evaluation at full size whose builds run in
# full and whose per-particle loops run on every 64th block of 512 particles, scaled up.
# ---------------------------------------------------------------------------------------------------------
CPU_STRIDE = 64


def host_info() -> dict:
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return dict(nproc=usable, cpus=os.cpu_count(), model=model)


def cpu_bodies(wl: dict, seed: int = 1, sample_impacts: int = 8):
    """HydroBody handles on the workload's own initial conditions in SI units: the impact itself, or for a
    batch its first `sample_impacts` impacts (a seeded sample, labelled as such). Returns (bodies, counts)."""
    import oracle
    from botheadstudios_b200.materials import eos_table64, SI
    I = build_workload(wl, seed)
    U = I.units
    kernel = 1 if wl["kernel"] == "wendland" else 0
    p_all = I.particles
    if hasattr(I, "offsets"):
        spans = [(int(I.offsets[k]), int(I.offsets[k + 1]), float(I.softening[k]))
                 for k in range(min(sample_impacts, I.n_impacts))]
        pos_all = p_all["pos"].astype(np.float64)
    else:
        spans = [(0, len(p_all), float(I.softening))]
        pos_all = I.pos64
    out, counts = [], []
    for a, b, soft in spans:
        p = p_all[a:b]
        hb = oracle.HydroBody(pos_all[a:b] * U.L, p["vel"].astype(np.float64) * U.speed,
                              p["mass"].astype(np.float64) * U.M, p["u"].astype(np.float64) * U.energy,
                              p["h"].astype(np.float64) * U.L, p["mat"].astype(np.int32), eos_table64(SI),
                              soft * U.L, G=6.674e-11, theta=0.5, kernel=kernel)
        out.append(hb)
        counts.append(b - a)
    return out, counts


def cpu_full_steps(bodies, counts, nthreads: int, max_steps: int, budget_s: float):
    """Full KDK steps (HydroBody::step) at the Courant dt, all bodies per step, until max_steps or the budget
    (at least one step). Returns particle-steps/s and the steps run."""
    dts = []
    for hb in bodies:
        hb.compute_density(nthreads)
        dts.append(hb.courant_dt(0.3))
    done, t0 = 0, time.perf_counter()
    while done < max(max_steps, 1):
        for hb, dt in zip(bodies, dts):
            hb.step(dt, nthreads)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return dict(value=sum(counts) * done / el, steps_run=done, seconds=el)


def cpu_single_thread(bodies, counts, stride: int = CPU_STRIDE):
    """One core: a step is two force evaluations, each estimated from one sampled evaluation at full size."""
    t_step = 0.0
    for hb in bodies:
        full, sampled = hb.eval_sampled(stride)
        t_step += 2.0 * (full + stride * sampled)
    return dict(value=sum(counts) / t_step, seconds_per_step=t_step)


def cpu_sample_text(wl, counts, r, nthreads):
    what = (f"the first {len(counts)} impacts ({sum(counts):,} particles) of the workload's seeded draw"
            if wl.get("kind") == "batch" else f"the workload's own {sum(counts):,}-particle initial conditions")
    return (f"HydroBody::step restated in C++ (f64, octree Barnes-Hut theta=0.5, hash-grid neighbours, 2 force "
            f"evaluations per KDK step, SI units) on {what}: {r['steps_run']} full KDK step(s) in "
            f"{r['seconds']:.1f} s on {nthreads} OpenMP threads")


def cpu_baseline_leg(wl: dict, budget_s: float = 30.0, max_steps: int = 2) -> dict:
    import oracle
    bodies, counts = cpu_bodies(wl)
    nthreads = oracle.max_threads()
    r = cpu_full_steps(bodies, counts, nthreads, max_steps, budget_s)
    one = cpu_single_thread(bodies, counts)
    return dict(value=r["value"], unit=UNIT, cores=nthreads, kind="port",
                sample=cpu_sample_text(wl, counts, r, nthreads),
                single_thread=dict(value=one["value"], unit=UNIT, cores=1, kind="port",
                                   sample=f"the reference's single-threaded loops (symmetric pair loops, per-particle "
                                          f"octree walk) on the same state: grid/octree builds and the EOS at full "
                                          f"size, per-particle loops on every {CPU_STRIDE}th block of 512 particles, "
                                          f"scaled by {CPU_STRIDE}; {one['seconds_per_step']:.1f} s per step"),
                host=host_info())


def run_reference(args, wl, world, rank, local, pg):
    """The reference arm: the CPU path of record on this configuration, full KDK steps on all host cores,
    until --steps steps or 150 s (its warm-up is none: a CPU step needs no compilation or cache warm-up, and
    one more 1M-particle step would cost tens of seconds). Rank 0 alone runs it."""
    if rank != 0:
        return
    import oracle
    bodies, counts = cpu_bodies(wl)
    nthreads = oracle.max_threads()
    r = cpu_full_steps(bodies, counts, nthreads, args.steps, budget_s=150.0)
    n = n_particles(wl)
    line = dict(metric=METRIC, value=r["value"], unit=UNIT, impl="reference", n_gpus=args.gpus, steps=args.steps,
                steps_run=r["steps_run"], warmup=args.warmup, warmup_run=0,
                ms_per_step=1000.0 * r["seconds"] / max(r["steps_run"], 1),
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                config=bench_config(args, wl, n, world),
                cpu_baseline=dict(value=r["value"], unit=UNIT, cores=nthreads, kind="port",
                                  sample=cpu_sample_text(wl, counts, r, nthreads), host=host_info()),
                e2e=dict(value=r["value"], unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def bench_config(args, wl: dict, n: int, world: int) -> dict:
    """The workload as both arms name it (the same dict in the GPU line and the reference line)."""
    return dict(workload=args.workload, particles=n, impacts=wl.get("n_impacts", 1), kernel=wl["kernel"],
                neighbours=wl["n_ngb"], theta=wl["theta"], quadrupole=bool(wl["quad"]), leaf=wl["leaf"],
                h_mode=["fixed", "solve", "learned"][wl["h_solve"]], dt="adaptive CFL 0.3",
                parallelism=f"replicas{world}", l2="working set > L2 (no flush needed)")


def run_ours(args, wl, world, rank, local, pg):
    import torch

    I = build_workload(wl, seed=1 + rank)
    runner, tuned = make_runner(wl, I, local)
    n = runner.n
    runner.upload()
    # warm-up (includes the first full force evaluation, and the graph captures when graphs are on)
    runner.encode_kdk(args.warmup)
    runner.sync()
    dstart = [s.diag() for s in runner.ctxs]
    for s in runner.ctxs:
        s.profile_enable(False)  # launch count only: phase events off, so captured graphs replay
    barrier(pg)
    torch.cuda.synchronize(local)
    with ClockSampler(local) as clk:
        ms = timed(runner.ctxs, runner.encode_kdk, args.steps, local)
    torch.cuda.synchronize(local)
    barrier(pg)
    launches = sum(s.profile_read()["kernel_launches"] for s in runner.ctxs)
    ms_max = max_over_ranks(pg, ms, local)
    value = replica_value(pg, n * args.steps, ms, local)
    # per-phase breakdown and walk counters: a few more steps with phase events (eager launches), one
    # context at a time so that every kernel duration is its own
    prof = dict(ms={}, calls={})
    d0, d1 = [], []
    for s in runner.ctxs:
        d0.append(s.diag())
        s.profile_enable(True)
        s.encode_kdk(min(args.steps, 4))
        pr = s.profile_read()
        s.profile_enable(False)
        d1.append(s.diag(check=False))
        cnt = s.count()
        for k, t in pr["ms"].items():
            prof["ms"][k] = prof["ms"].get(k, 0.0) + t
            prof["calls"][k] = prof["calls"].get(k, 0) + pr["calls"][k]
            prof.setdefault("pcalls", {})[k] = prof.setdefault("pcalls", {}).get(k, 0) + pr["calls"][k] * cnt

    def dsum(ds, key):
        return sum(d[key] for d in ds)

    learned_state = None
    if wl.get("h_solve") == 2 and wl.get("kind") != "batch" and rank == 0 and not args.no_plain:
        learned_state = runner.s.readback()  # the learned form's state after its timed and profiled steps

    # mean neighbour-list length (the lists the gather phases stream)
    lsum, lcnt = 0.0, 0
    for s in runner.ctxs:
        c = s.inspect("NBR_COUNT").astype(np.float64)
        lsum += float(c.sum())
        lcnt += len(c)
    lbar = lsum / max(lcnt, 1)

    # ---- end to end through the public API: per step, upload the state from pinned host memory, one KDK
    # step, read the state back into host memory ----
    pin = torch.empty(n * 48, dtype=torch.uint8, pin_memory=True).numpy().view(runner.batch.particles.dtype)
    runner.readback_into(pin)
    e2e_steps = max(2, min(args.steps, 10))

    def e2e_run(k):
        for _ in range(k):
            runner.upload(pin)          # H2D of the step's input state from pinned memory
            runner.encode_kdk(1)
            runner.readback_into(pin)   # D2H of the step's result into the same pinned buffer

    barrier(pg)
    e2e_ms = timed(runner.ctxs, e2e_run, e2e_steps, local)  # device events around the whole sequence
    e2e_value = replica_value(pg, n * e2e_steps, e2e_ms, local)
    plain = None
    if wl.get("kind") == "batch" and rank == 0 and not args.no_plain:
        plain = plain_sequential(wl, I, local)
        if wl.get("h_solve") == 2:
            plain = dict(sequential=plain, batched_same_tuning=plain_batched(
                wl, I, {int(b): c for b, c in (tuned or {}).get("choices", {}).items()}, local, args.steps,
                args.warmup))
    elif wl.get("h_solve") == 2 and rank == 0 and not args.no_plain:
        plain = dict(newton_2=plain_same(wl, I, local, args.steps, args.warmup, h_iters=2),
                     newton_1=plain_same(wl, I, local, args.steps, args.warmup, h_iters=1),
                     learned_density_error=density_error(wl, I, learned_state, local))

    if rank != 0:
        return
    # ---- roofline of the dominant phase (device-timed with CUDA events on the library's stream) ----
    pk = peaks()
    phases = {}
    for k, t in prof["ms"].items():
        calls = prof["calls"][k]
        if calls == 0 or t <= 0:
            continue
        b = phase_bytes(k, wl, lbar) * prof["pcalls"][k]  # particles processed over all calls
        phases[k] = dict(ms=round(t, 4), share=round(t / sum(prof["ms"].values()), 4), calls=calls,
                         gbs=round(b / (t / 1000.0) / 1e9, 1))
    dom = max(phases, key=lambda k: phases[k]["ms"])
    dom_ms = phases[dom]["ms"] / phases[dom]["calls"]
    n_per_call = prof["pcalls"][dom] / phases[dom]["calls"]  # particles per launch of the dominant phase
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(args.workload, {}).get(dom)
    if dom == "gravity" and wl.get("quad") is not None:
        # The walk (group-MAC gravity fused with the neighbour lists) is FP32-pipe bound: algorithmic FLOPs
        # from the device counters — 65 per quadrupole (20 per monopole) multipole evaluation at a particle,
        # 20 per particle × source-particle pair (real sources only: the padding slots of partial leaves are
        # reported beside it, not counted), 12 per node acceptance test, 180 (80 monopole) per node expanded
        # about a group's centre and 60 per particle evaluating that expansion — over its CUDA-event time.
        # Peak: FP32 FMA throughput of 148 SMs × 128 lanes × 2 FLOP × the max SM clock (nominal; no measured
        # FP32 peak exists here).
        walks = max(phases["gravity"]["calls"], 1)

        def per_walk(key):
            return (dsum(d1, key) - dsum(d0, key)) / walks
        m2p, p2p, vis = per_walk("m2p_interactions"), per_walk("p2p_interactions"), per_walk("walk_nodes")
        m2l, slots = per_walk("local_expansions"), per_walk("p2p_slots")
        quad = bool(wl["quad"])
        flops = ((65.0 if quad else 20.0) * m2p + 20.0 * p2p + 12.0 * vis + (180.0 if quad else 80.0) * m2l +
                 (60.0 * n_per_call if m2l > 0 else 0.0))
        clk_max = (clk.summary() or {}).get("sm_max_mhz") or 1965.0
        peak_tf = 148 * 128 * 2 * clk_max * 1e6 / 1e12
        achieved = flops / (dom_ms / 1000.0) / 1e12
        roof = dict(bound="fp32", kernel="k_tree_walk", achieved=round(achieved, 2), peak=round(peak_tf, 1),
                    unit="TFLOP/s", frac=round(achieved / peak_tf, 4), traffic=traffic,
                    peak_source="nominal FP32 FMA peak (148 SM x 128 lanes x 2 x max SM clock)",
                    flops_per_launch=flops, ms_per_launch=round(dom_ms, 4),
                    interactions_per_particle=dict(multipole=m2p / n_per_call, pairwise=p2p / n_per_call,
                                                   pairwise_slots=slots / n_per_call, nodes=vis / n_per_call,
                                                   local_expansions_per_group=m2l / max(n_per_call / 32.0, 1.0)))
    else:
        dom_bytes = phase_bytes(dom, wl, lbar) * n_per_call
        achieved = dom_bytes / (dom_ms / 1000.0) / 1e9
        roof = dict(bound="hbm", kernel_phase=dom, achieved=round(achieved, 1), peak=pk["hbm"], unit="GB/s",
                    frac=round(achieved / pk["hbm"], 4), traffic=traffic, peak_source=pk["src"],
                    bytes_per_launch=dom_bytes, ms_per_launch=round(dom_ms, 4))
    # memory-bound phases against the measured HBM copy bandwidth
    mem = [k for k in ("sort", "tree", "density", "forces", "integrate", "hsolve") if k in phases]
    mem_bytes = sum(phase_bytes(k, wl, lbar) * prof["pcalls"][k] for k in mem)
    mem_ms = sum(phases[k]["ms"] for k in mem)
    roof_hbm = dict(bound="hbm", phases=mem, achieved=round(mem_bytes / (mem_ms / 1000.0) / 1e9, 1),
                    peak=pk["hbm"], unit="GB/s", frac=round(mem_bytes / (mem_ms / 1000.0) / 1e9 / pk["hbm"], 4),
                    peak_source=pk["src"], mean_list_entries=round(lbar, 1),
                    per_phase={k: round(phases[k]["gbs"] / pk["hbm"], 4) for k in mem})
    # ---- CPU baseline on the host cores (rank 0, N=1 only) ----
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_baseline_leg(wl)
    dd = d1[0]
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=ms_max / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic (seeded lattice impact)",
                config=bench_config(args, wl, n, world),
                runner=dict(contexts=len(runner.ctxs), graph=bool(wl.get("graph", 0))),
                e2e=dict(value=e2e_value, unit=UNIT, h2d_bytes_per_step=48 * n, d2h_bytes_per_step=48 * n,
                         steps=e2e_steps),
                gpu_launches=launches, roofline=roof, roofline_hbm=roof_hbm, phases=phases, cpu_baseline=cpu,
                clocks=clk.summary(),
                autotune=tuned, **({} if not plain else
                                   {"plain_sequential": plain} if wl.get("h_solve") != 2 else {"plain_form": plain}),
                physics=dict(**conservation_drifts(dstart, d1),
                             sim_time=dd["time"], dt=dd["dt"],
                             max_neighbours=max(d["max_neighbours_seen"] for d in d1),
                             overflow_flags=max(d["overflow_flags"] for d in d1),
                             h_accepted_fraction=(sum(d["h_accepted"] for d in d1) / n
                                                  if wl.get("h_solve") == 2 else None),
                             h_residual=max(d["h_residual"] for d in d1)))
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------------
# The disk measurement of a finished impact (sph_measure_disk; impact-run main.rs:732-878): one "step" is one
# measurement of a post-impact field held on the device; e2e adds the upload of the field from host memory.
# ---------------------------------------------------------------------------------------------------------
MEASURE_METRIC = "disk-measurement particles/s"


def _measure_field(args, rank):
    from botheadstudios_b200 import ic, workloads
    return ic.post_impact_scene(seed=1 + rank, **workloads.MEASURE_WORKLOADS[args.measure_workload])


def run_measure(args, world, rank, local, pg):
    import torch
    from botheadstudios_b200 import ic
    from botheadstudios_b200.gpusph import GpuSph
    from botheadstudios_b200.materials import SI, eos_table

    p = _measure_field(args, rank)
    n, eos = len(p), eos_table()
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2
    with GpuSph(n, device=local, **ic.config_kwargs(SI)) as s:
        ext = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}")
        s.upload(p, eos, 1.0e4)
        for _ in range(args.warmup):
            res = s.measure_disk(0, variant=args.variant)
        launches0 = s.profile_read()["kernel_launches"]

        def one(e2e: bool) -> float:
            with torch.cuda.stream(ext):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            if e2e:
                s.upload(p, eos, 1.0e4)
            s.measure_disk(0, variant=args.variant)
            e1.record(ext)
            e1.synchronize()
            return e0.elapsed_time(e1)

        barrier(pg)
        torch.cuda.synchronize(local)
        dev = [one(False) for _ in range(args.steps)]
        launches = (s.profile_read()["kernel_launches"] - launches0) // max(args.steps, 1)
        e2e = [one(True) for _ in range(args.steps)]
        barrier(pg)
        res = s.measure_disk(0, variant=args.variant)
    value = replica_value(pg, n, sum(dev) / len(dev), local)
    value_e2e = replica_value(pg, n, sum(e2e) / len(e2e), local)
    ms = max_over_ranks(pg, sum(dev) / len(dev), local)
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = measure_reference_run(p, args.variant)
    line = dict(metric=MEASURE_METRIC, value=value, unit="particles/s", n_gpus=world,
                steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic",
                config=dict(workload=args.measure_workload, particles=n, disk_particles=res["n_disk"],
                            variant=args.variant, l2="flushed (256 MB write) before every measurement"),
                e2e=dict(value=value_e2e, unit="particles/s", h2d_bytes_per_step=48 * n,
                         d2h_bytes_per_step=112),
                gpu_launches=int(launches), result=res)
    if cpu is not None:
        line["cpu_baseline"] = dict(value=n / cpu["seconds"], unit="particles/s", cores=cpu["cores"], kind="port",
                                    sample=cpu["sample"])
    print(json.dumps(line), flush=True)


def measure_reference_run(p, variant: int) -> dict:
    import oracle
    from botheadstudios_b200.materials import G_SI
    t0 = time.perf_counter()
    oracle.measure_disk(p, G_SI, variant=variant)
    el = time.perf_counter() - t0
    cores = oracle.max_threads()
    form = "impact-run measure + moon_candidate" if variant == 0 else "disk_stats_json + find_clumps"
    return dict(seconds=el, cores=cores,
                sample=f"{form} restated in C++ (O(k^2) friends-of-friends pairs on {cores} OpenMP threads) on "
                       f"the whole {len(p):,}-particle field, one measurement in {el:.2f} s")


def run_measure_reference(args, world, rank, local, pg):
    if rank != 0:
        return
    p = _measure_field(args, 0)
    runs = [measure_reference_run(p, args.variant) for _ in range(max(1, min(args.steps, 3)))]
    sec = sum(r["seconds"] for r in runs) / len(runs)
    v = len(p) / sec
    line = dict(metric=MEASURE_METRIC, value=v, unit="particles/s", impl="reference", n_gpus=args.gpus,
                steps=len(runs), warmup=0, ms_per_step=1000.0 * sec, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic",
                config=dict(workload=args.measure_workload, particles=len(p), variant=args.variant),
                cpu_baseline=dict(value=v, unit="particles/s", cores=runs[0]["cores"], kind="port",
                                  sample=runs[0]["sample"]),
                e2e=dict(value=v, unit="particles/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="impact_1m", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="batch workloads: skip the sequential plain-form leg")
    ap.add_argument("--path", default="step", choices=["step", "measure"],
                    help="measure: the disk measurement of a finished impact instead of the KDK step")
    ap.add_argument("--measure-workload", default="post_impact_1m",
                    choices=["post_impact_200k", "post_impact_1m", "post_impact_4m"])
    ap.add_argument("--variant", type=int, default=0, choices=[0, 1],
                    help="measure: 0 = the impact-run tool, 1 = the engine's disk statistics")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    world, rank, local, pg = dist_setup(args)
    try:
        if args.path == "measure":
            (run_measure_reference if args.impl == "reference" else run_measure)(args, world, rank, local, pg)
        elif args.impl == "reference":
            run_reference(args, wl, world, rank, local, pg)
        else:
            run_ours(args, wl, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
