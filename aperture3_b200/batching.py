"""Many independent 2D periodic boxes advanced in batches under an HBM budget.

A batch of runs of uneven sizes (ap_batch_*: one persistent push / deposit
launch per tile shape over all runs' tiles) does not fit the device when
the runs' particles exceed the memory: `BoxBatcher` admits runs in order
while their device footprint fits the budget, tunes the tile shape once
per box size with the project autotuner, advances the resident runs in
rounds of lab-loop steps (ap_batch_advance), retires the runs that are
done and admits the next ones. Each run computes exactly what it computes
alone (the batch changes scheduling, not arithmetic; a tile shape changed
by the autotuner can move the current's last bits, as alone).
"""
from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import ic
from .sim import Batch, SimData, SimEnvironment


@dataclasses.dataclass
class BoxRequest:
    rid: int
    side: int
    ppc: int
    steps: int
    seed: int


def box_requests(n: int, seed: int = 4, sides=(128, 192, 256, 384, 512), ppc=(16, 128),
                 steps: int = 500) -> List[BoxRequest]:
    """n periodic boxes: side uniform in `sides`, an even ppc uniform in
    [ppc[0], ppc[1]], the same number of steps each; seeded."""
    rng = np.random.default_rng(seed)
    return [BoxRequest(rid=r, side=int(rng.choice(sides)),
                       ppc=2 * int(rng.integers(ppc[0] // 2, ppc[1] // 2 + 1)), steps=steps,
                       seed=5000 + r) for r in range(n)]


def footprint_bytes(req: BoxRequest, compact: int) -> int:
    """Device memory of one resident run: the particle SoA (48 B per slot,
    twice the particles with compaction), the library's per-particle state
    (tile order and directions 9 B, sort scratch 24 B, per slot), and the
    fields, accumulators and tile bookkeeping per cell."""
    n = req.side * req.side * req.ppc
    cap = 2 * n if compact else n
    cells = (req.side + 4) ** 2
    return int(cap * 48 + n * (9 + 24) + cells * (18 * 4 + 5 * 8 + 16) + (1 << 20))


class BoxRun:
    def __init__(self, req: BoxRequest, device, compact: int, sort_interval: int):
        self.req = req
        params, fields, ptc = ic.box2d(seed=req.seed, N=req.side, ppc=req.ppc, device=device)
        self.n = ptc["x1"].numel()
        self.env = SimEnvironment(params)
        self.data = SimData(self.env, capacity=2 * self.n if compact else self.n)
        self.data.set_fields_device(fields)
        self.data.set_particles_device(ptc)
        self.env.set_compaction(compact)
        torch.cuda.current_stream().synchronize()
        self.step = 0
        self.fp = footprint_bytes(req, compact)

    def close(self):
        self.env.close()


class BoxBatcher:
    """Admission by HBM footprint, autotuned tile shapes per box size,
    rounds of `round_steps` batched steps."""

    def __init__(self, device=None, hbm_budget: float = 120e9, round_steps: int = 50,
                 compact: int = 2, sort_interval: int = 20, autotune: bool = True):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.budget = float(hbm_budget)
        self.round_steps = int(round_steps)
        self.compact = int(compact)
        self.sort_interval = int(sort_interval)
        self.autotune = autotune
        self.shapes: Dict[int, Tuple[int, int]] = {}  # side -> tuned (tx, ty)
        self.schedule: List[Dict[str, object]] = []

    def run(self, requests: List[BoxRequest]) -> Dict[str, object]:
        pending = list(requests)
        for r in pending:
            if footprint_bytes(r, self.compact) > self.budget:
                raise ValueError(f"run {r.rid} does not fit the HBM budget")
        batch = Batch()
        active: List[BoxRun] = []
        used = 0
        done: Dict[int, float] = {}
        particle_steps = 0
        tune_steps = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while pending or active:
            admitted = []
            while pending and used + footprint_bytes(pending[0], self.compact) <= self.budget:
                req = pending.pop(0)
                run = BoxRun(req, self.device, self.compact, self.sort_interval)
                if req.side in self.shapes:
                    run.env.set_tile_shape(*self.shapes[req.side])
                batch.add(run.data)
                active.append(run)
                admitted.append(run)
                used += run.fp
            if admitted:
                self.schedule.append({"t_s": time.perf_counter() - t0,
                                      "admitted": [r.req.rid for r in admitted],
                                      "resident": len(active), "resident_gb": used / 1e9})
                untuned = sorted({r.req.side for r in admitted if r.req.side not in self.shapes})
                if self.autotune and untuned:
                    # the project autotuner over the whole batch (runs of sizes
                    # already tuned keep their shape class timing too)
                    n = batch.autotune([r.step for r in active])
                    tune_steps += n
                    for r in active:
                        r.step += n
                    for r, shape in zip(active, batch.tile_shapes()):
                        self.shapes.setdefault(r.req.side, shape)
            rounds = min(self.round_steps, min(r.req.steps - r.step for r in active))
            if rounds > 0:
                batch.advance([r.step for r in active], rounds, self.sort_interval)
                for r in active:
                    r.step += rounds
            for r in [r for r in active if r.step >= r.req.steps]:
                batch.remove(r.data)  # waits for the batch's stream
                done[r.req.rid] = time.perf_counter() - t0
                particle_steps += r.n * r.req.steps
                active.remove(r)
                used -= r.fp
                r.close()
                del r
            if not active:
                torch.cuda.empty_cache()
        batch.close()
        torch.cuda.synchronize()
        makespan = time.perf_counter() - t0
        return {"runs": len(requests), "particle_steps": int(particle_steps),
                "makespan_s": makespan, "throughput": particle_steps / makespan,
                "autotune_steps": tune_steps, "waves": len(self.schedule),
                "schedule": self.schedule,
                "tile_shapes": {str(k): f"{v[0]}x{v[1]}" for k, v in sorted(self.shapes.items())}}


def run_alone(req: BoxRequest, device, compact: int = 2, sort_interval: int = 20) -> int:
    """The plain path: the lab loop of one run with synchronous calls;
    returns its particle-steps."""
    from .sim import field_solver, ptc_updater
    run = BoxRun(req, device, compact, sort_interval)
    pusher, solver = ptc_updater(run.env), field_solver(run.env)
    dt = run.env.params.delta_t
    for s in range(req.steps):
        pusher.update_particles(run.data, dt, s)
        solver.update_fields(run.data, dt, s)
        if s % sort_interval == 0 and s != 0:
            run.data.sort_particles()
    torch.cuda.synchronize()
    ps = run.n * req.steps
    run.close()
    return ps
