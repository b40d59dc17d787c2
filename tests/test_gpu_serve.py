"""Served 1D gap runs: pair injection on the GPU against the CPU oracle (bit
for bit), and continuous batching: every request's final state is the same
served in a mix, admitted as memory frees up, as run alone through the
plain path."""
import numpy as np
import pytest
import torch

import oracle
from aperture3_b200 import serve
from aperture3_b200.serve import GapRequest, GapRun, GapServer, run_alone
from _gpu_helpers import assert_bits

pytestmark = pytest.mark.gpu


def _small_requests(n=5, seed=3):
    rng = np.random.default_rng(seed)
    return [GapRequest(rid=i, cells=int(rng.integers(200, 700)), ppc=2 * int(rng.integers(3, 9)),
                       steps=int(rng.integers(30, 70)), ramp=float(rng.uniform(0.1, 10)),
                       arrival=0.0, seed=1000 + i, hot_fraction=0.2) for i in range(n)]


def test_inject_pairs_matches_oracle():
    dev = torch.device("cuda", 0)
    req = GapRequest(rid=0, cells=512, ppc=16, steps=1, ramp=1.0, seed=77, hot_fraction=0.5)
    run = GapRun(req, dev)
    cap = run.data.capacity
    host = run.data.particles_host()
    n = run.data.number
    em, dr = run.data.inject_pairs(run.dt, 5)
    got = run.data.particles_host()
    # the oracle appends past the live slots: give it arrays of the capacity
    p = {k: np.concatenate([v, np.zeros(cap - n, v.dtype)]) for k, v in host.items()}
    n2, em2, dr2 = oracle.inject_pairs(p, n, cap, np.float32(run.dt), 5, serve.GAMMA_THR,
                                       serve.FREE_PATH, serve.PAIR_ENERGY, req.seed, 1 << 40)
    assert (em, dr) == (em2, dr2) and em > 10
    assert run.data.number == n2 == n + 2 * em
    for k in got:
        assert_bits(got[k][:n2], p[k][:n2], f"particles.{k}")
    run.close()


def test_served_mix_equals_alone():
    dev = torch.device("cuda", 0)
    reqs = _small_requests()
    fps = sorted(serve.footprint_bytes(r) for r in reqs)
    budget = sum(fps[-3:]) + 1  # about three resident runs at a time
    server = GapServer(dev, hbm_budget=budget, round_steps=8, keep_results=True)
    stats = server.serve(reqs, realtime=False)
    assert stats["requests"] == len(reqs) and stats["throughput"] > 0
    assert stats["latency_p50_s"] <= stats["latency_p99_s"]
    emitted_any = False
    for r in reqs:
        alone, _ = run_alone(r, dev)
        mixed = server.results[r.rid]
        assert alone["number"] == mixed["number"], r.rid
        n = alone["number"]
        emitted_any |= bool(np.any(alone["particles"]["id"][:n] >= (1 << 40)))
        for k, v in alone["particles"].items():
            assert_bits(mixed["particles"][k][:n], v[:n], f"run {r.rid}: particles.{k}")
        for key in ("E", "B", "J"):
            for c in range(3):
                assert_bits(mixed["fields"][key][c], alone["fields"][key][c],
                            f"run {r.rid}: {key}{c + 1}")
    assert emitted_any
