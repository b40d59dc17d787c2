"""Served stream of 1D gap runs with continuous batching.

Requests arrive over time (Poisson); each is an independent 1D run: a gap of
`cells` cells with `ppc` particles per cell, a linear E_parallel ramp of
amplitude `ramp`, and pair injection for particles above gamma 1e6
(ap_pair_params). The server keeps every admitted run's particles and
fields resident on the device, admits queued requests in arrival order while
their HBM footprint fits the budget, and advances all resident runs
together through one batch (ap_batch_*), a round of steps per call
(ap_batch_advance): per step one batched push / deposit launch, batched
field updates and one pair-injection pass, each run at its own step. A run leaves the batch when it
has done its steps; the batch is rebuilt when its membership changes.

Each run computes exactly what it computes alone through the plain path
(`run_alone`): the batch changes scheduling, not arithmetic.
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Dict, List, Optional

import numpy as np
import torch

from .sim import (ELECTRON, POSITRON, Batch, SimData, SimEnvironment, SimParams, field_solver,
                  ptc_updater, species_flag)

SORT_INTERVAL = 20
GAMMA_THR = 1e6
FREE_PATH = 0.05
PAIR_ENERGY = 50.0
HOT_FRACTION = 0.01


@dataclasses.dataclass
class GapRequest:
    rid: int
    cells: int
    ppc: int
    steps: int
    ramp: float
    arrival: float = 0.0  # seconds after the start of serving
    seed: int = 0
    hot_fraction: float = HOT_FRACTION


def request_stream(n: int, seed: int = 0, rate: float = 50.0, cells=(512, 16384),
                   ppc=(32, 256), steps=(200, 5000), ramp=(0.1, 10.0)) -> List[GapRequest]:
    """Poisson arrivals at `rate` per second; cells, ppc (even) and steps
    uniform integers, ramp amplitude uniform, all from one seeded stream."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        out.append(GapRequest(rid=i, cells=int(rng.integers(cells[0], cells[1] + 1)),
                              ppc=2 * int(rng.integers(ppc[0] // 2, ppc[1] // 2 + 1)),
                              steps=int(rng.integers(steps[0], steps[1] + 1)),
                              ramp=float(rng.uniform(ramp[0], ramp[1])), arrival=t,
                              seed=int(seed) * 100003 + i + 1))
    return out


def gap_params(req: GapRequest) -> SimParams:
    N = req.cells
    dx = 1.0 / N
    n = N * req.ppc
    return SimParams(N=(N, 1, 1), guard=(2, 0, 0), size=(1.0, 1.0, 1.0),
                     delta_t=float(np.float32(0.5 * dx)), q_e=1.0, num_species=2,
                     periodic_boundary=(False, False, False), data_interval=1 << 30,
                     max_ptc_number=int(n + n // 4 + 1024), B0=1.0)


def gap_state(req: GapRequest, device):
    """Fields and particles of one gap run: E1 = Ebg1 = ramp * x on the E1
    stagger, B1 = Bbg1 = 1; ppc/2 e-/e+ pairs per cell at one uniform
    position each, momenta N(0, 0.1) per component, and a fraction of hot
    pairs with gamma log-uniform in [1e5, 1e7] along +-x."""
    params = gap_params(req)
    N, g = req.cells, 2
    dims0 = N + 2 * g
    gen = torch.Generator(device=device)
    gen.manual_seed(req.seed)
    x = (torch.arange(dims0, device=device, dtype=torch.float64) - g + 0.5) / N
    E1 = (req.ramp * x).float()
    one = torch.ones(dims0, device=device)
    zero = torch.zeros(dims0, device=device)
    fields = {"E": [E1, zero, zero], "B": [one, zero, zero], "Ebg": [E1.clone(), zero, zero],
              "Bbg": [one.clone(), zero, zero]}
    npair = N * req.ppc // 2
    cells = (torch.arange(N, device=device) + g).repeat_interleave(req.ppc // 2)
    rel = torch.rand(npair, generator=gen, device=device)
    p = 0.1 * torch.randn((3, npair), generator=gen, device=device, dtype=torch.float64)
    hot = torch.rand(npair, generator=gen, device=device) < req.hot_fraction
    lg = 5.0 + 2.0 * torch.rand(npair, generator=gen, device=device, dtype=torch.float64)
    gam = torch.pow(10.0, lg)
    sgn = torch.where(torch.rand(npair, generator=gen, device=device) < 0.5, -1.0, 1.0)
    p[0] = torch.where(hot, sgn * torch.sqrt(gam * gam - 1.0), p[0])
    p[1] = torch.where(hot, torch.zeros_like(p[1]), p[1])
    p[2] = torch.where(hot, torch.zeros_like(p[2]), p[2])
    n = 2 * npair
    rep = lambda a: a.repeat_interleave(2)  # noqa: E731
    pf = [rep(p[k]).float() for k in range(3)]
    E = torch.sqrt(1.0 + pf[0].double() ** 2 + pf[1].double() ** 2 + pf[2].double() ** 2)
    sp = torch.tensor([species_flag(ELECTRON), species_flag(POSITRON)], dtype=torch.int64,
                      device=device)
    ptc = {"x1": rep(rel), "x2": torch.zeros(n, device=device),
           "x3": torch.zeros(n, device=device), "p1": pf[0], "p2": pf[1], "p3": pf[2],
           "E": E.float(), "weight": torch.ones(n, device=device),
           "cell": rep(cells).to(torch.int64), "id": torch.arange(n, device=device),
           "flag": sp.repeat(npair)}
    return params, fields, ptc


def footprint_bytes(req: GapRequest) -> int:
    """Device memory of one resident run: the particle SoA (48 B) plus the
    library's per-particle state (tile order and directions, 9 B; sort
    scratch, 24 B) over the capacity, and the field, accumulator and filter
    arrays (18 float arrays, 5 64-bit accumulators) over the cells."""
    p = gap_params(req)
    cap = p.max_ptc_number
    cells = req.cells + 4
    return int(cap * (48 + 9 + 24) + cells * (18 * 4 + 5 * 8) + (1 << 20))


class GapRun:
    def __init__(self, req: GapRequest, device):
        self.req = req
        params, fields, ptc = gap_state(req, device)
        self.env = SimEnvironment(params)
        self.data = SimData(self.env, capacity=params.max_ptc_number)
        self.data.set_fields_device(fields)
        self.data.set_particles_device(ptc)
        self.env.set_pair_params(GAMMA_THR, FREE_PATH, PAIR_ENERGY, seed=req.seed,
                                 first_id=1 << 40)
        torch.cuda.current_stream().synchronize()  # the copies above ran on torch's stream
        self.dt = params.delta_t
        self.step = 0
        self.fp = footprint_bytes(req)

    def particle_steps(self) -> int:
        """Live particle slots summed over the steps done (device counter)."""
        return self.data.pair_stats()[0]

    def result(self) -> Dict[str, object]:
        return {"particles": self.data.particles_host(), "fields": self.data.fields_host(),
                "number": self.data.number}

    def close(self):
        self.env.close()


def run_alone(req: GapRequest, device, keep_result: bool = True, retired=None):
    """The plain path: the lab loop of one run, synchronous calls. With a
    `retired` list the finished run is appended to it instead of being
    released (the caller releases it later, as the server does)."""
    run = GapRun(req, device)
    pusher, solver = ptc_updater(run.env), field_solver(run.env)
    for s in range(req.steps):
        pusher.update_particles(run.data, run.dt, s)
        solver.update_fields(run.data, run.dt, s)
        run.data.inject_pairs(run.dt, s)
        if s % SORT_INTERVAL == 0 and s != 0:
            run.data.sort_particles()
    torch.cuda.synchronize()
    out = run.result() if keep_result else None
    ps = run.particle_steps()
    if retired is None:
        run.close()
    else:
        retired.append(run)
    return out, ps


class GapServer:
    """Continuous batching of gap runs under an HBM budget. Finished runs
    leave the batch at once; their device memory is released when a later
    admission needs the room, or after the last request."""

    def __init__(self, device=None, hbm_budget: float = 40e9, round_steps: int = 16,
                 keep_results: bool = False):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = float(hbm_budget)
        self.round_steps = int(round_steps)
        self.keep = keep_results
        self.results: Dict[int, Dict[str, object]] = {}
        # per round: (start s, resident runs, resident particles, steps, wall s);
        # per admission ("admit", rid, start s, s) and retirement ("retire",
        # rid, start s, s waiting for the batch, s reading the run's counters,
        # s releasing the run)
        self.trace: List[tuple] = []
        self.events: List[tuple] = []
        self.retired: List["GapRun"] = []  # finished runs whose memory is not yet released
        self.retired_bytes = 0

    def serve(self, requests: List[GapRequest], realtime: bool = True) -> Dict[str, object]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in pending:
            if footprint_bytes(r) > self.budget:
                raise ValueError(f"request {r.rid} does not fit the HBM budget")
        active: List[GapRun] = []
        batch = Batch()
        used = 0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0 if realtime else math.inf  # noqa: E731
        admitted, finished, particle_steps = {}, {}, 0
        while pending or active:
            # admission: arrived requests, in order, while the budget allows
            while pending and pending[0].arrival <= now() and used + footprint_bytes(
                    pending[0]) <= self.budget:
                req = pending.pop(0)
                t_adm = time.perf_counter()
                self._release_if_needed(footprint_bytes(req))
                run = GapRun(req, self.device)
                batch.add(run.data)
                self.events.append(("admit", req.rid, t_adm - t0, time.perf_counter() - t_adm))
                active.append(run)
                used += run.fp
                admitted[req.rid] = now() if realtime else 0.0
            if not active:
                wait = pending[0].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 0.05))
                continue
            # a round of steps over the resident runs, each at its own step
            rounds = min(self.round_steps, min(r.req.steps - r.step for r in active))
            # the lab loop of every resident run for `rounds` steps in one
            # call: update_particles, update_fields, inject_pairs, sort every
            # SORT_INTERVAL steps (ap_batch_advance)
            t_round = time.perf_counter()
            batch.advance([r.step for r in active], rounds, SORT_INTERVAL, inject=True)
            for r in active:
                r.step += rounds
            self.trace.append((t_round - t0, len(active),
                               sum(r.req.cells * r.req.ppc for r in active), rounds,
                               time.perf_counter() - t_round))
            for r in [r for r in active if r.step >= r.req.steps]:
                t_ret = time.perf_counter()
                batch.remove(r.data)  # waits for the batch's stream
                t_rem = time.perf_counter() - t_ret
                t_ps = time.perf_counter()
                finished[r.req.rid] = time.perf_counter() - t0
                particle_steps += r.particle_steps()
                if self.keep:
                    self.results[r.req.rid] = r.result()
                active.remove(r)
                used -= r.fp
                t_cl = time.perf_counter()
                # the run's device memory is released off the critical path:
                # when a later admission needs the room, else after the last
                # request (cudaFree waits for the whole device and can take
                # tens of milliseconds per run)
                self.retired.append(r)
                self.retired_bytes += r.fp
                if self.retired_bytes > self.budget:
                    self._release()
                t_end = time.perf_counter()
                self.events.append(("retire", r.req.rid, t_ret - t0, t_rem, t_cl - t_ps,
                                    t_end - t_cl))
        batch.close()
        torch.cuda.synchronize()
        makespan = time.perf_counter() - t0
        self._release()
        return _stats(requests, admitted, finished, particle_steps, makespan)

    def _release(self):
        for r in self.retired:
            r.close()
        self.retired.clear()
        self.retired_bytes = 0

    def _release_if_needed(self, need: int):
        """Frees the retired runs when the device lacks room for `need` bytes
        and a 2 GB reserve."""
        if self.retired and torch.cuda.mem_get_info(self.device)[0] < need + (2 << 30):
            self._release()


def serve_one_at_a_time(requests: List[GapRequest], device=None, realtime: bool = True):
    """The same requests served first come, first served, one at a time
    through the plain path. Finished runs are released off the critical
    path, as by the server: when the next request needs the room, else at
    the end."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    admitted, finished, total = {}, {}, 0
    retired: List[GapRun] = []
    for req in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        if realtime:
            wait = req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        admitted[req.rid] = time.perf_counter() - t0
        if retired and torch.cuda.mem_get_info(device)[0] < footprint_bytes(req) + (2 << 30):
            for r in retired:
                r.close()
            retired.clear()
        _, ps = run_alone(req, device, keep_result=False, retired=retired)
        total += ps
        finished[req.rid] = time.perf_counter() - t0
    makespan = time.perf_counter() - t0
    for r in retired:
        r.close()
    return _stats(requests, admitted, finished, total, makespan)


def _stats(requests, admitted, finished, particle_steps, makespan):
    lat = np.array([finished[r.rid] - r.arrival for r in requests])
    return {"requests": len(requests), "particle_steps": int(particle_steps),
            "makespan_s": makespan, "throughput": particle_steps / makespan,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_mean_s": float(lat.mean())}


def resident_steps(nsteps: int, requests: int = 24, seed: int = 5, warmup: int = 5,
                   device=None) -> Dict[str, float]:
    """Every request of the stream resident in one batch, `nsteps` batched
    steps timed after `warmup` (the full phase of a served run, without
    arrivals or departures): for profiling the batched serving step."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    reqs = request_stream(requests, seed=seed, rate=50.0, steps=(200, 5000))
    runs = [GapRun(r, device) for r in reqs]
    batch = Batch()
    for r in runs:
        batch.add(r.data)

    def step():
        batch.advance([r.step for r in runs], 1, SORT_INTERVAL, inject=True)
        for r in runs:
            r.step += 1

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        step()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    n = sum(r.req.cells * r.req.ppc for r in runs)
    for r in runs:
        batch.remove(r.data)
        r.close()
    batch.close()
    return {"particles": n, "ms_per_step": 1e3 * dt / max(nsteps, 1),
            "particle_steps_per_s": n * nsteps / dt if dt > 0 else 0.0}


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="batched serving step with every request resident")
    ap.add_argument("--resident-steps", type=int, default=200)
    ap.add_argument("--requests", type=int, default=24)
    a = ap.parse_args()
    print(json.dumps(resident_steps(a.resident_steps, a.requests)))
