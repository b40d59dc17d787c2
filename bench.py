#!/usr/bin/env python
"""Benchmark of the Aperture3 particle update on B200.

Workload (one step = the reference lab's loop body, labs/box/src/main.cpp:
81-91): ptc_updater::update_particles (Vay push + Esirkepov deposit + move,
tile counting sort, current fold) and field_solver::update_fields (Yee
FDTD), plus sort_particles every sort_interval (20) steps, on the 2D
Cartesian box: 1024 x 1024 cells, 64 particles per cell (67,108,864), seeded
synthetic initial state (aperture3_b200.ic.box2d). The particle SoA
(3.2 GB) is far larger than L2 (126 MB), so no L2 flush is needed between
steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched with torch.distributed.run): every rank runs its own box
(replicas: the single-GPU path has no cross-GPU exchange); value is the
particle-steps of all ranks over the slowest rank's device time.
--impl reference times the CPU path (the reference's own kernels compiled
for the host when available, else the C restatement) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s (push+deposit)"
UNIT = "particle-steps/s"
ALG_BYTES_PER_PARTICLE = 68  # 36 B read + 32 B written per particle-step
ALG_BYTES_PER_CELL = 36      # 6 field reads + 3 current writes, 4 B each


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=1024)
    ap.add_argument("--ppc", type=int, default=64)
    ap.add_argument("--tile", type=int, nargs=2, default=(16, 16))
    ap.add_argument("--sort-interval", type=int, default=20)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--compact", type=int, default=2,
                    help="rewrite the particle store in tile order every n steps (0: never); "
                         "particles keep their values, only their slots change")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batched workload: keep every run's tile shape")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of CPU work for the cpu_baseline sample")
    ap.add_argument("--workload", default="box",
                    choices=["box", "batched", "served", "logsph"],
                    help="box: the 2D box (headline line); batched: many uneven boxes "
                         "through ap_batch_* against the same runs one at a time; served: "
                         "a Poisson stream of 1D gap runs, continuous batching against "
                         "first-come-first-served one at a time; logsph: the log-spherical "
                         "1024x1024 grid (ptc_updater_logsph + field_solver_logsph)")
    ap.add_argument("--steps-scale", type=float, default=1.0,
                    help="served: run lengths are 200-5000 steps times this factor")
    ap.add_argument("--hbm-budget", type=float, default=60.0,
                    help="served: GB of device memory the resident runs may occupy")
    ap.add_argument("--runs", type=int, default=24, help="batched: number of runs")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds for the whole --impl reference run")
    return ap.parse_args()


def workload_config(args, tile):
    n = args.N * args.N * args.ppc
    return {
        "workload": (f"2D Cartesian periodic box {args.N}x{args.N}, {args.ppc} ppc "
                     f"({n} particles, e-/e+ pairs, gamma log-uniform in [1,1e3]), "
                     "B3=1 + 8 Fourier modes in E and B; per step Vay push + Esirkepov "
                     "deposit + tile counting sort + Yee FDTD, sort_by_cell every "
                     f"{args.sort_interval} steps"),
        "grid": [args.N, args.N], "ppc": args.ppc, "particles": n,
        "capacity": 2 * n if args.compact else n,
        "tile": list(tile), "sort_interval": args.sort_interval,
        "compaction_interval": args.compact,
        "l2": "inputs larger than L2 (particle SoA 48 B x N_p)",
    }


# --------------------------------------------------------------------------
# clocks

class ClockSampler:
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            sel = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", sel, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, t0, t1):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        ts = time.mktime(time.strptime(parts[0].split(".")[0],
                                                       "%Y/%m/%d %H:%M:%S"))
                        frac = float("0." + parts[0].split(".")[1]) if "." in parts[0] else 0.0
                        rows.append((ts + frac, float(parts[1]), float(parts[2]), parts[5:9]))
                    except Exception:
                        continue
        except Exception:
            return None
        if not rows:
            return None
        inside = [r for r in rows if t0 - 0.15 <= r[0] <= t1 + 0.15]
        if not inside:
            inside = sorted(rows, key=lambda r: abs(r[0] - 0.5 * (t0 + t1)))[:3]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i, v in enumerate(r[3])
                          if v.lower() in ("active", "1")})
        return {"sm_mhz": statistics.median(r[1] for r in inside),
                "sm_max_mhz": max(r[2] for r in inside), "reasons": reasons,
                "samples": len(inside)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per particle of the fused kernel from the committed ncu
    summary (line 'dram_bytes_per_particle: X'), or None."""
    path = os.path.join(ROOT, "profiles", "k_push_deposit_2d_box.md")
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("dram_bytes_per_particle:"):
                    return float(line.split(":")[1])
    except Exception:
        pass
    return None


# --------------------------------------------------------------------------
# CPU path (baseline leg and reference arm)

def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class CpuBox:
    """The same step on the host, on all host threads: the reference's own
    push and deposit kernels compiled for the host (oracle/_ref/
    libapref_mt.so, kind "reference") when that library was built, else
    the C restatement (oracle/liboracle.so, kind "port"); the guard fold,
    wrap, FDTD and sort are the restatement's in both cases."""

    def __init__(self, params, fields_np, ptc_np, threads):
        import numpy as np
        import oracle
        self.o = oracle
        self.np = np
        self.m = oracle.make_mesh(params.N, params.guard, params.lower, params.size)
        self.f = oracle.new_fields(self.m, params.num_species)
        for c in range(3):
            self.f["E"][c][:] = fields_np["E"][c]
            self.f["B"][c][:] = fields_np["B"][c]
        self.p = ptc_np
        self.n = len(ptc_np["x1"])
        self.params = params
        self.threads = threads
        q = 1.0
        self.charges = [-q] + [q] * 7
        self.masses = [q] * 8
        self.periodic = [1, 1, 0]
        self.ref = oracle.load_ref_mt(build=False) is not None
        self.kind = "reference" if self.ref else "port"

    def describe(self):
        if self.ref:
            return ("the reference's push and deposit kernels compiled for the host "
                    "(oracle/_ref), restated guard fold, wrap, FDTD and sort")
        return "C restatement of the reference (oracle/liboracle.so)"

    def step(self, step):
        if self.ref:
            self.o.ref_update_particles_mt(self.m, self.p, self.n, self.f, self.params.delta_t,
                                           step, self.params.data_interval, 2, self.charges,
                                           self.masses, self.periodic, self.threads)
        else:
            self.o.update_particles(self.m, self.p, self.n, self.f, self.params.delta_t, step,
                                    self.params.data_interval, 2, 0, self.charges, self.masses,
                                    self.periodic, self.threads)
        self.o.update_fields(self.m, self.f, self.params.delta_t, step, self.periodic)
        if step % 20 == 0 and step != 0:
            self.n = self.o.sort_by_cell(self.m, self.p, self.n)


def cpu_sample(args, ppc_sample, seed=1):
    from aperture3_b200 import ic
    params, fields, ptc = ic.box2d(seed=seed, N=args.N, ppc=ppc_sample, device="cpu")
    fields_np = {"E": [f.numpy() for f in fields["E"]], "B": [f.numpy() for f in fields["B"]]}
    return params, fields_np, ic.to_numpy_ptc(ptc)


def time_cpu(args, budget_s, min_steps=1, max_steps=None):
    """Runs the CPU step on a sample of the workload sized to budget_s.
    Returns (particle-steps/s, threads, sample description, steps)."""
    threads = cpu_threads()
    # calibrate on 1 ppc
    params, f, p = cpu_sample(args, 2)
    box = CpuBox(params, f, p, threads)
    t = time.perf_counter()
    box.step(1)
    dt1 = time.perf_counter() - t
    per_particle = dt1 / box.n
    steps = max(min_steps, 1)
    ppc = 2
    while ppc * 2 <= args.ppc and per_particle * args.N * args.N * ppc * 2 * steps <= budget_s:
        ppc *= 2
    params, f, p = cpu_sample(args, ppc)
    box = CpuBox(params, f, p, threads)
    nsteps = steps if max_steps is None else max_steps
    box.step(0)  # warm-up (includes the half step of E)
    t = time.perf_counter()
    for s in range(1, nsteps + 1):
        box.step(s)
    el = time.perf_counter() - t
    rate = box.n * nsteps / el
    desc = (f"{args.N}x{args.N} grid, {ppc} ppc ({box.n} particles), {nsteps} step(s) after "
            f"1 warm-up, {threads} threads, {box.describe()}")
    return rate, threads, desc, box.kind


def run_reference(args, rank):
    if rank != 0:
        return
    threads = cpu_threads()
    params, f, p = cpu_sample(args, 2)
    box = CpuBox(params, f, p, threads)
    t = time.perf_counter()
    box.step(1)
    per_particle = (time.perf_counter() - t) / box.n
    total_steps = args.steps + args.warmup
    ppc = 2
    while ppc * 2 <= args.ppc and per_particle * args.N * args.N * ppc * 2 * total_steps <= args.ref_budget:
        ppc *= 2
    params, f, p = cpu_sample(args, ppc)
    box = CpuBox(params, f, p, threads)
    for s in range(args.warmup):
        box.step(s)
    t = time.perf_counter()
    for s in range(args.warmup, args.warmup + args.steps):
        box.step(s)
    el = time.perf_counter() - t
    value = box.n * args.steps / el
    sample = (f"{args.N}x{args.N} grid, {ppc} ppc ({box.n} particles) of the {args.ppc}-ppc "
              f"workload, {args.steps} timed steps, {box.describe()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)", "config": workload_config(args, (0, 0)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": box.kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU path

def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    from aperture3_b200 import SimData, SimEnvironment, field_solver, ic, ptc_updater
    from aperture3_b200._lib import ApPhaseTimes, check

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    params, fields, ptc = ic.box2d(seed=1000 + rank, N=args.N, ppc=args.ppc, device=dev,
                                   tile=tuple(args.tile))
    params.chunk = args.chunk
    n = ptc["x1"].numel()
    env = SimEnvironment(params)
    # twice the particles: compactions write the tile-ordered store into the
    # free half instead of copying it back
    data = SimData(env, capacity=2 * n if args.compact else n)
    data.set_fields_device(fields)
    data.set_particles_device(ptc)
    del ptc
    torch.cuda.empty_cache()
    stream = torch.cuda.Stream()
    env.set_stream(stream)
    env.set_sync(False)
    env.set_compaction(args.compact)
    pusher, solver = ptc_updater(env), field_solver(env)
    dt = params.delta_t
    lib = env._lib

    def one_step(s):
        pusher.update_particles(data, dt, s)
        solver.update_fields(data, dt, s)
        if s % args.sort_interval == 0 and s != 0:
            data.sort_particles()

    def barrier():
        if world > 1:
            dist.barrier()

    sampler = ClockSampler(local_rank)
    with torch.cuda.stream(stream):
        for s in range(args.warmup):
            one_step(s)
        env.sync()
        check(lib.ap_set_profiling(env.ctx, 1), "profiling")
        check(lib.ap_get_phase_times(env.ctx, ApPhaseTimes(), 1), "reset")
        launches0 = env.launch_count()
        barrier()
        torch.cuda.synchronize()
        t_wall0 = time.time()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(args.warmup, args.warmup + args.steps):
            one_step(s)
        e1.record(stream)
        torch.cuda.synchronize()
        t_wall1 = time.time()
        barrier()
        env.sync()  # raises on a device-reported error
    ms = e0.elapsed_time(e1)
    launches = env.launch_count() - launches0
    pt = ApPhaseTimes()
    check(lib.ap_get_phase_times(env.ctx, pt, 1), "phase times")
    check(lib.ap_set_profiling(env.ctx, 0), "profiling off")
    sampler.stop()
    clocks = sampler.summary(t_wall0, t_wall1)

    ms_max = ms
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = n * args.steps * world / (ms_max / 1e3)

    # roofline of the fused push/deposit kernel
    G = (args.N + 4) * (args.N + 4)
    alg_bytes = ALG_BYTES_PER_PARTICLE * n + ALG_BYTES_PER_CELL * G
    k_ms = pt.push_deposit_ms / max(pt.push_deposit_launches, 1)
    achieved = alg_bytes / (k_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    tpp = profiled_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tpp * n if tpp is not None else None),
                "kernel": "k_push_deposit_2d", "kernel_ms": k_ms,
                "phases_ms_per_step": {
                    "push_deposit": pt.push_deposit_ms / args.steps,
                    "tile_sort": pt.order_ms / args.steps,
                    "rebuild": pt.rebuild_ms / args.steps,
                    "finalize": pt.finalize_ms / args.steps,
                    "fields": pt.fields_ms / args.steps,
                    "sort_by_cell": pt.sort_ms / args.steps}}

    env.sync()
    check_live(data, n, "box")  # the periodic box keeps every particle

    # e2e through the C ABI with host buffers: upload the run's initial state
    # from pinned host memory, run the steps, read the FP64 diagnostics back
    # every step, download the final particles and fields.
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, env, data, pusher, solver, dt, stream, n)
    if world > 1 and e2e is not None:
        t = torch.tensor([e2e["ms"]], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e["value"] = n * args.steps * world / (float(t.item()) / 1e3)
    if e2e is not None:
        e2e.pop("ms")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, threads, desc, kind = time_cpu(args, args.cpu_budget)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded initial state, aperture3_b200.ic.box2d)",
        "config": dict(workload_config(args, (env.ap_params.tile[0] or 16,
                                              env.ap_params.tile[1] or 16)),
                       parallelism=("replicas" if world > 1 else "single")),
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": launches, "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    env.close()


AUTOTUNE_STEPS = 8  # 2 candidate tile shapes x 4 steps (ap_batch_autotune)


def check_live(data, n, what):
    """Every particle of a periodic box is still in the store."""
    first, end = data.slot_range()
    live = int((data.particles["cell"][first:end] != -1).sum())  # int32 view of MAX_CELL
    if live != n:
        raise RuntimeError(f"{what}: {live} particles in the store, expected {n}")


def run_batched(args):
    """Batched uneven boxes: `runs` independent periodic boxes, side uniform
    in {128, 192, 256, 384, 512}, 16-128 particles per cell (even), the
    box2d field setup, each with its own dt. Two legs from the same seeded
    initial states, timing the same steps: one at a time through the plain
    path (each run created, advanced with the lab loop -- synchronous
    update_particles, update_fields, sort every sort_interval steps -- and
    freed before the next), then all runs together through one batch, whose
    first AUTOTUNE_STEPS steps are the autotuner's (the single runs take
    the same steps untimed). Wall clock between device synchronisations;
    aggregate particle-steps/s."""
    import numpy as np
    import torch
    from aperture3_b200 import Batch, SimData, SimEnvironment, field_solver, ic, ptc_updater

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(4)
    specs = [(int(rng.choice([128, 192, 256, 384, 512])), 2 * int(rng.integers(8, 65)))
             for _ in range(args.runs)]

    def make(r):
        side, ppc = specs[r]
        params, fields, ptc = ic.box2d(seed=5000 + r, N=side, ppc=ppc, device=dev)
        n = ptc["x1"].numel()
        env = SimEnvironment(params)
        data = SimData(env, capacity=2 * n if args.compact else n)
        data.set_fields_device(fields)
        data.set_particles_device(ptc)
        env.set_compaction(args.compact)
        return env, data, n

    s_first = AUTOTUNE_STEPS + args.warmup
    steps = range(s_first, s_first + args.steps)

    # one at a time through the plain path
    t_alone, total = 0.0, 0
    for r in range(len(specs)):
        env, data, n = make(r)
        total += n
        pusher, solver = ptc_updater(env), field_solver(env)
        dt = env.params.delta_t

        def step(s):
            pusher.update_particles(data, dt, s)
            solver.update_fields(data, dt, s)
            if s % args.sort_interval == 0 and s != 0:
                data.sort_particles()
        for s in range(s_first):
            step(s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in steps:
            step(s)
        torch.cuda.synchronize()
        t_alone += time.perf_counter() - t0
        check_live(data, n, f"run {r} alone")
        env.close()
        del data
        torch.cuda.empty_cache()
    alone = total * args.steps / t_alone

    # the same runs in one batch
    runs = [make(r) for r in range(len(specs))]
    torch.cuda.synchronize()
    batch = Batch([d for _, d, _ in runs])

    def bstep(s):
        batch.update_particles(s)
        batch.update_fields(s)
        if s % args.sort_interval == 0 and s != 0:
            batch.sort_particles()
    if args.no_autotune:
        used = 0
    else:
        used = batch.autotune(0)
        assert used == AUTOTUNE_STEPS, used
    for s in range(used, s_first):
        bstep(s)
    batch.sync()
    t0 = time.perf_counter()
    for s in steps:
        bstep(s)
    batch.sync()
    t_batch = time.perf_counter() - t0
    batched = total * args.steps / t_batch
    for r, (_, d, n) in enumerate(runs):
        check_live(d, n, f"run {r} in the batch")
    shapes = {}
    for (side, ppc), shape in zip(specs, batch.tile_shapes()):
        shapes[str(side)] = f"{shape[0]}x{shape[1]}"
    batch.close()
    line = {
        "metric": "aggregate particle-steps/s (batched uneven boxes)", "value": batched,
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded, aperture3_b200.ic.box2d per run)",
        "config": {"workload": f"{args.runs} periodic boxes, side in {{128,192,256,384,512}}, "
                               "16-128 ppc, random-mode fields, own dt each",
                   "runs": args.runs, "particles": total, "timed_steps": [steps[0], steps[-1]],
                   "compaction_interval": args.compact,
                   "sides": [sp[0] for sp in specs], "ppc": [sp[1] for sp in specs]},
        "one_at_a_time": alone, "speedup_vs_one_at_a_time": batched / alone,
        "autotune_steps": used, "tile_shapes": shapes,
    }
    print(json.dumps(line), flush=True)
    for env, _, _ in runs:
        env.close()


def run_logsph(args):
    """Log-spherical grid 1024 x 1024, r in [1, 50], dipole B with corotation
    E, 32 particles per cell scaled by exp(-(r - 1) / 0.5), gamma up to 1e6
    along B (aperture3_b200.ic.logsph). A step is the pulsar lab's loop body:
    ptc_updater_logsph::update_particles, field_solver_logsph::update_fields
    and apply_boundary, sort every sort_interval steps. Device time (CUDA
    events) over `steps` steps after `warmup`."""
    import torch
    from aperture3_b200 import (SimData, SimEnvironment, field_solver_logsph, ic,
                                ptc_updater_logsph)
    from aperture3_b200._lib import ApPhaseTimes, check

    dev = torch.device("cuda", 0)
    params, fields, ptc = ic.logsph(seed=11, N=args.N, ppc=32, device=dev)
    n = ptc["x1"].numel()
    env = SimEnvironment(params)
    data = SimData(env, capacity=n)
    data.set_fields_device(fields)
    data.set_particles_device(ptc)
    del ptc
    stream = torch.cuda.Stream()
    env.set_stream(stream)
    env.set_sync(False)
    pusher, solver = ptc_updater_logsph(env), field_solver_logsph(env)
    dt = params.delta_t
    lib = env._lib

    def one_step(s):
        pusher.update_particles(data, dt, s)
        solver.update_fields(data, dt, s * dt)
        solver.apply_boundary(data, params.omega, s * dt)
        if s % args.sort_interval == 0 and s != 0:
            data.sort_particles()

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for s in range(args.warmup):
            one_step(s)
        env.sync()
        check(lib.ap_set_profiling(env.ctx, 1), "profiling")
        check(lib.ap_get_phase_times(env.ctx, ApPhaseTimes(), 1), "reset")
        n0 = data.number
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(args.warmup, args.warmup + args.steps):
            one_step(s)
        e1.record(stream)
        torch.cuda.synchronize()
        env.sync()
    ms = e0.elapsed_time(e1)
    pt = ApPhaseTimes()
    check(lib.ap_get_phase_times(env.ctx, pt, 1), "phase times")
    data.refresh_number()
    live = (n0 + data.number) / 2
    line = {
        "metric": "particle-steps/s (log-spherical push+move+deposit)",
        "value": live * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded, aperture3_b200.ic.logsph)",
        "config": {"workload": f"log-spherical {args.N}x{args.N}, r in [1,50], dipole B, "
                               "32 ppc x exp(-(r-1)/0.5), gamma up to 1e6 along B",
                   "particles_start": n0, "particles_end": data.number},
        "phases_ms_per_step": {"push_deposit": pt.push_deposit_ms / args.steps,
                               "tile_sort": pt.order_ms / args.steps,
                               "rebuild": pt.rebuild_ms / args.steps,
                               "finalize": pt.finalize_ms / args.steps,
                               "fields": pt.fields_ms / args.steps,
                               "sort_by_cell": pt.sort_ms / args.steps},
    }
    print(json.dumps(line), flush=True)
    env.close()


def run_served(args):
    """Served stream of 1D gap runs: `runs` requests with Poisson arrivals
    (50/s), 512-16384 cells, 32-256 particles per cell, 200-5000 steps
    scaled by --steps-scale, E_parallel ramp amplitude in [0.1, 10], pair
    injection above gamma 1e6 (exponential free path, mean 0.05, Philox).
    Leg 1: continuous batching under the HBM budget; leg 2: the same
    requests first come, first served, one at a time through the plain
    path. Wall clock; aggregate particle-steps/s and completion latency
    (finish - arrival) percentiles."""
    import torch
    from aperture3_b200 import serve

    lo, hi = max(1, int(200 * args.steps_scale)), max(2, int(5000 * args.steps_scale))
    reqs = serve.request_stream(args.runs, seed=5, rate=50.0, steps=(lo, hi))
    dev = torch.device("cuda", 0)
    # warm the code paths (module loads, kernel first launches)
    serve.run_alone(serve.GapRequest(rid=-1, cells=512, ppc=32, steps=3, ramp=1.0, seed=9),
                    dev, keep_result=False)
    server = serve.GapServer(dev, hbm_budget=args.hbm_budget * 1e9, round_steps=16)
    st_b = server.serve(reqs, realtime=True)
    st_a = serve.serve_one_at_a_time(reqs, dev, realtime=True)
    line = {
        "metric": "aggregate particle-steps/s (served 1D gap runs)", "value": st_b["throughput"],
        "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded request stream, aperture3_b200.serve)",
        "config": {"workload": f"{args.runs} requests, Poisson 50/s, 512-16384 cells, "
                               f"32-256 ppc, {lo}-{hi} steps, pair injection",
                   "hbm_budget_gb": args.hbm_budget},
        "served": st_b, "one_at_a_time": st_a,
        "speedup_vs_one_at_a_time": st_b["throughput"] / st_a["throughput"],
    }
    print(json.dumps(line), flush=True)


def run_e2e(args, env, data, pusher, solver, dt, stream, n):
    import ctypes as C

    import numpy as np
    import torch
    from aperture3_b200._lib import check
    from aperture3_b200.sim import PTC_FIELDS

    names = [k for k, _ in PTC_FIELDS]
    # the initial state of the end-to-end run: the current particles, sorted
    # by cell into one contiguous slot range (the lower or the upper half of
    # the doubled capacity; the periodic box loses none)
    data.sort_particles()
    s0, s1 = data.slot_range()
    if s1 - s0 != n:
        raise RuntimeError(f"expected {n} particles after the sort, found {s1 - s0}")
    host = {k: torch.empty_like(data.particles[k][:n], device="cpu").pin_memory() for k in names}
    fhost = {k: [torch.empty(a.shape, dtype=a.dtype).pin_memory() for a in getattr(data, k)]
             for k in ("E", "B", "J")}
    with torch.cuda.stream(stream):
        for k in names:
            host[k].copy_(data.particles[k][s0:s1], non_blocking=True)
        for k in fhost:
            for h, a in zip(fhost[k], getattr(data, k)):
                h.copy_(a, non_blocking=True)
    torch.cuda.synchronize()
    h2d = sum(t.numel() * t.element_size() for t in host.values()) + \
        sum(t.numel() * t.element_size() for k in ("E", "B") for t in fhost[k])
    d2h = sum(t.numel() * t.element_size() for t in host.values()) + \
        sum(t.numel() * t.element_size() for v in fhost.values() for t in v)
    # per-step FP64 diagnostics copied into pinned host memory without a
    # host synchronisation per step (ap_diagnostics_async)
    diag_host = torch.zeros((args.steps, 6), dtype=torch.float64).pin_memory()
    d2h_diag = 48
    lib = env._lib
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k in names:
            data.particles[k][:n].copy_(host[k], non_blocking=True)
        for k in ("E", "B"):
            for h, a in zip(fhost[k], getattr(data, k)):
                a.copy_(h, non_blocking=True)
        data.particles_modified(n)
        for s in range(args.steps):
            pusher.update_particles(data, dt, s)
            solver.update_fields(data, dt, s)
            if s % args.sort_interval == 0 and s != 0:
                data.sort_particles()
            check(lib.ap_diagnostics_async(env.ctx, C.c_void_p(diag_host[s].data_ptr())),
                  "ap_diagnostics_async")
        first, end = data.slot_range()  # host-side bounds, no synchronisation
        for k in names:
            host[k][:end - first].copy_(data.particles[k][first:end], non_blocking=True)
        for k in fhost:
            for h, a in zip(fhost[k], getattr(data, k)):
                h.copy_(a, non_blocking=True)
        e1.record(stream)
    torch.cuda.synchronize()
    env.sync()
    ms = e0.elapsed_time(e1)
    live = int((host["cell"][:end - first] != -1).sum())  # int32 view of MAX_CELL
    if live != n:
        raise RuntimeError(f"end-to-end run returned {live} particles, expected {n}")
    kin = diag_host[:, 0].numpy()
    if not (np.all(np.isfinite(kin)) and np.all(kin > 0)):
        raise RuntimeError("end-to-end run: per-step kinetic energy not finite and positive")
    return {"value": n * args.steps / (ms / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps,
            "d2h_bytes_per_step": d2h / args.steps + d2h_diag, "ms": ms,
            "includes": "initial-state upload, all steps with a per-step FP64 diagnostics "
                        "readback, final particle and field download"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.workload in ("batched", "served", "logsph"):
            if rank == 0:
                {"batched": run_batched, "served": run_served,
                 "logsph": run_logsph}[args.workload](args)
            return
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
