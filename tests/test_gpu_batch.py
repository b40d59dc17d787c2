"""Batched mode: many uneven periodic boxes, each with its own time step,
advanced by one persistent push / deposit launch per tile shape
(ap_batch_*). Each run in the batch must give the same particles, bit for
bit, as the same run advanced alone through the plain path, and the same
fields (bit for bit with the same tile shape; within 1e-6 of the maximum
after the autotuner changed the shape, which moves the fixed-point scale of
the current)."""
import numpy as np
import pytest

import oracle
from _cases import mesh_2d, random_fields, random_particles
from _gpu_helpers import assert_bits, make_params
from aperture3_b200 import Batch, SimData, SimEnvironment, field_solver, ptc_updater

pytestmark = pytest.mark.gpu


def _specs(seed, nruns):
    rng = np.random.default_rng(seed)
    return [(int(rng.choice([32, 48, 64, 96])), int(rng.choice([32, 48, 64])),
             int(rng.integers(2, 9)), seed * 1000 + r) for r in range(nruns)]


def _make(spec, data_interval=2, spare=1, compact=0, tile=(0, 0)):
    N0, N1, ppc, s = spec
    n = N0 * N1 * ppc
    params = make_params((N0, N1), periodic=(True, True), capacity=spare * n,
                         data_interval=data_interval, tile=tile)
    params.delta_t = float(np.float32(0.45 / max(N0, N1)))
    rng = np.random.default_rng(s)
    m = mesh_2d(N0, N1)
    f = random_fields(m, rng, amp=0.3)
    for key in ("E", "B", "Ebg", "Bbg"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 1, 0))
    p = random_particles(m, n, rng, gamma_max=100.0)
    env = SimEnvironment(params)
    data = SimData(env, capacity=spare * n)
    data.set_fields(f)
    data.set_particles(p)
    env.set_compaction(compact)
    return env, data


def _step_alone(runs, step):
    for env, data in runs:
        ptc_updater(env).update_particles(data, env.params.delta_t, step)
        field_solver(env).update_fields(data, env.params.delta_t, step)


def _compare(alone, batched, tol=0.0):
    for r, ((_, da), (_, db)) in enumerate(zip(alone, batched)):
        pa, pb = da.particles_host(), db.particles_host()
        for k in ("x1", "x2", "x3", "p1", "p2", "p3", "E", "cell", "flag", "weight", "id"):
            assert_bits(pb[k], pa[k], f"run {r}: particles.{k}")
        fa, fb = da.fields_host(), db.fields_host()
        for key in ("J", "E", "B"):
            for c in range(3):
                if tol == 0.0:
                    assert_bits(fb[key][c], fa[key][c], f"run {r}: {key}{c + 1}")
                else:
                    scale = max(np.abs(fa[key][c]).max(), 1e-30)
                    err = np.abs(fb[key][c].astype(np.float64) - fa[key][c]).max() / scale
                    assert err <= tol, f"run {r}: {key}{c + 1} {err:.3g}"


def _close(batch, *groups):
    batch.close()
    for g in groups:
        for env, _ in g:
            env.close()


def test_batch_equals_alone():
    specs = _specs(1, 12)
    alone = [_make(s) for s in specs]
    batched = [_make(s) for s in specs]
    batch = Batch([d for _, d in batched])
    assert len(set(batch.dt)) > 1  # uneven boxes, each with its own dt
    for step in range(7):
        _step_alone(alone, step)
        batch.update_particles(step)
        batch.update_fields(step)
        if step == 3:
            for _, data in alone:
                data.sort_particles()
            batch.sort_particles()
    batch.sync()
    _compare(alone, batched)
    _close(batch, alone, batched)


def test_batch_autotune_then_steps():
    specs = _specs(2, 8)
    alone = [_make(s) for s in specs]
    batched = [_make(s) for s in specs]
    batch = Batch([d for _, d in batched])
    used = batch.autotune(0)
    assert used >= 2
    for step in range(used):
        _step_alone(alone, step)
    for step in range(used, used + 4):
        _step_alone(alone, step)
        batch.update_particles(step)
        batch.update_fields(step)
    batch.sync()
    shapes = batch.tile_shapes()
    assert all(s in ((16, 16), (32, 16), (16, 8), (8, 8), (4, 4)) for s in shapes)
    _compare(alone, batched, tol=1e-6)
    _close(batch, alone, batched)


def test_batch_mixed_steps_and_data_interval():
    """Runs at different step numbers, with different charge-deposition
    schedules, in one batch."""
    specs = _specs(3, 5)
    dis = [1, 2, 3, 2, 1]
    alone = [_make(s, data_interval=d) for s, d in zip(specs, dis)]
    batched = [_make(s, data_interval=d) for s, d in zip(specs, dis)]
    offs = [0, 3, 1, 7, 2]
    batch = Batch([d for _, d in batched])
    for k in range(5):
        for (env, data), o in zip(alone, offs):
            ptc_updater(env).update_particles(data, env.params.delta_t, o + k)
            field_solver(env).update_fields(data, env.params.delta_t, o + k)
        batch.update_particles([o + k for o in offs])
        batch.update_fields([o + k for o in offs])
    batch.sync()
    _compare(alone, batched)
    for r, ((_, da), (_, db)) in enumerate(zip(alone, batched)):
        fa, fb = da.fields_host(), db.fields_host()
        for s_ in range(len(fa["Rho"])):
            assert_bits(fb["Rho"][s_], fa["Rho"][s_], f"run {r}: Rho{s_}")
    _close(batch, alone, batched)


@pytest.mark.parametrize("tile,spare", [((16, 16), 2), ((32, 16), 2), ((32, 16), 1)])
def test_batch_compaction_equals_alone(tile, spare):
    """Runs that rewrite their store in tile order every 3 updates (into the
    free half of a doubled capacity, or through scratch) give, in a batch,
    the particles of the same runs advanced alone, compared by id, and the
    same fields bit for bit; no particle is lost."""
    specs = _specs(5, 6)
    alone = [_make(s_, spare=spare, compact=3, tile=tile) for s_ in specs]
    batched = [_make(s_, spare=spare, compact=3, tile=tile) for s_ in specs]
    batch = Batch([d for _, d in batched])
    for step in range(8):
        _step_alone(alone, step)
        batch.update_particles(step)
        batch.update_fields(step)
        if step == 5:
            for _, data in alone:
                data.sort_particles()
            batch.sort_particles()
    batch.sync()
    for r, ((_, da), (_, db), spec) in enumerate(zip(alone, batched, specs)):
        pa, pb = da.particles_host(), db.particles_host()
        la, lb = pa["cell"] != oracle.MAX_CELL, pb["cell"] != oracle.MAX_CELL
        n = spec[0] * spec[1] * spec[2]
        assert la.sum() == n and lb.sum() == n, (r, la.sum(), lb.sum(), n)
        ia = np.argsort(pa["id"][la], kind="stable")
        ib = np.argsort(pb["id"][lb], kind="stable")
        for k in ("x1", "x2", "x3", "p1", "p2", "p3", "E", "cell", "flag", "weight", "id"):
            assert_bits(pb[k][lb][ib], pa[k][la][ia], f"run {r}: particles.{k}")
        fa, fb = da.fields_host(), db.fields_host()
        for key in ("J", "E", "B"):
            for c in range(3):
                assert_bits(fb[key][c], fa[key][c], f"run {r}: {key}{c + 1}")
    _close(batch, alone, batched)


def test_batch_advance_equals_alone_with_sorts():
    """ap_batch_advance (a whole round of lab-loop steps in one call, with
    sort_by_cell every 3 steps and compaction on) leaves every run as the
    same steps taken alone through the plain path."""
    specs = _specs(5, 6)
    alone = [_make(s, spare=2, compact=2) for s in specs]
    batched = [_make(s, spare=2, compact=2) for s in specs]
    batch = Batch([d for _, d in batched])
    for step in range(7):
        _step_alone(alone, step)
        if step % 3 == 0 and step != 0:
            for _, d in alone:
                d.sort_particles()
    batch.advance([0] * len(specs), 4, sort_interval=3)
    batch.advance([4] * len(specs), 3, sort_interval=3)
    batch.sync()
    _compare(alone, batched)
    _close(batch, alone, batched)
