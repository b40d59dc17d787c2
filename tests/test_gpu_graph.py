"""The update is CUDA-graph capturable: with pipelined calls (ap_set_sync
0) on a caller's stream, four steps of update_particles + update_fields
(compaction every 2 updates into a doubled capacity) are captured into one
CUDA graph and replayed; the state after the replays equals, bit for bit
(particles compared by id), the state of the same steps run call by call."""
import numpy as np
import pytest
import torch

import oracle
from _gpu_helpers import assert_bits
from aperture3_b200 import SimData, SimEnvironment, field_solver, ic, ptc_updater

pytestmark = pytest.mark.gpu


def _run(graph, steps_after_warmup=12):
    dev = torch.device("cuda", 0)
    params, fields, ptc = ic.box2d(seed=3, N=128, ppc=16, device=dev)
    n = ptc["x1"].numel()
    env = SimEnvironment(params)
    data = SimData(env, capacity=2 * n)
    data.set_fields_device(fields)
    data.set_particles_device(ptc)
    stream = torch.cuda.Stream()
    env.set_stream(stream)
    env.set_sync(False)
    env.set_compaction(2)
    pu, fs = ptc_updater(env), field_solver(env)
    dt = params.delta_t
    torch.cuda.synchronize()

    def step(s):
        pu.update_particles(data, dt, s)
        fs.update_fields(data, dt, s)

    for s in range(2):  # warm-up: order rebuild, scratch allocation
        step(s)
    env.sync()
    if graph:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            for s in range(2, 6):
                step(s)
        # the capture recorded the work without running it
        for _ in range(steps_after_warmup // 4):
            g.replay()
        torch.cuda.synchronize()
    else:
        for s in range(2, 2 + steps_after_warmup):
            step(s if s < 6 else 2 + (s - 2) % 4)
        env.sync()
    out = data.particles_host(), data.fields_host()
    env.close()
    return out


def test_captured_steps_equal_call_by_call():
    (pa, fa), (pb, fb) = _run(False), _run(True)
    la, lb = pa["cell"] != oracle.MAX_CELL, pb["cell"] != oracle.MAX_CELL
    assert la.sum() == lb.sum() > 0
    ia = np.argsort(pa["id"][la], kind="stable")
    ib = np.argsort(pb["id"][lb], kind="stable")
    for k in ("x1", "x2", "x3", "p1", "p2", "p3", "E", "cell", "flag", "weight", "id"):
        assert_bits(pb[k][lb][ib], pa[k][la][ia], f"particles.{k}")
    for key in ("E", "B", "J"):
        for c in range(3):
            assert_bits(fb[key][c], fa[key][c], f"{key}{c + 1}")


def test_captured_batch_steps_equal_call_by_call():
    """A batch of uneven 2D boxes (compaction every 2 updates), four batched
    steps captured into one CUDA graph in the batch's capture mode and
    replayed three times: every run ends bit for bit where the same steps
    run call by call leave it."""
    from aperture3_b200 import Batch

    def make_runs():
        dev = torch.device("cuda", 0)
        out = []
        for r, (N, ppc) in enumerate([(64, 8), (96, 4), (128, 6)]):
            params, fields, ptc = ic.box2d(seed=40 + r, N=N, ppc=ppc, device=dev)
            n = ptc["x1"].numel()
            env = SimEnvironment(params)
            data = SimData(env, capacity=2 * n)
            data.set_fields_device(fields)
            data.set_particles_device(ptc)
            env.set_compaction(2)
            out.append((env, data))
        torch.cuda.synchronize()
        return out

    def run(graph):
        runs = make_runs()
        batch = Batch([d for _, d in runs])
        stream = torch.cuda.Stream()
        batch.set_stream(stream)
        for s in range(2):
            batch.update_particles(s)
            batch.update_fields(s)
        batch.sync()
        if graph:
            batch.set_capture(True)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
                for s in range(2, 6):
                    batch.update_particles(s)
                    batch.update_fields(s)
            for _ in range(3):
                g.replay()
            torch.cuda.synchronize()
            del g
            batch.set_capture(False)
        else:
            for k in range(12):
                s = 2 + k % 4
                batch.update_particles(s)
                batch.update_fields(s)
        batch.sync()
        out = [(d.particles_host(), d.fields_host()) for _, d in runs]
        batch.close()
        for env, _ in runs:
            env.close()
        return out

    for r, ((pa, fa), (pb, fb)) in enumerate(zip(run(False), run(True))):
        la, lb = pa["cell"] != oracle.MAX_CELL, pb["cell"] != oracle.MAX_CELL
        assert la.sum() == lb.sum() > 0
        ia = np.argsort(pa["id"][la], kind="stable")
        ib = np.argsort(pb["id"][lb], kind="stable")
        for k in ("x1", "x2", "p1", "p2", "p3", "E", "cell", "id"):
            assert_bits(pb[k][lb][ib], pa[k][la][ia], f"run {r}: particles.{k}")
        for key in ("E", "B", "J"):
            for c in range(3):
                assert_bits(fb[key][c], fa[key][c], f"run {r}: {key}{c + 1}")
