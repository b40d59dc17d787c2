"""GPU parity of the C ABI against the CPU oracle (run on a B200).

Bar: particle momenta, gamma, positions and cell indices bit-exact; the
tile order and sort_by_cell bit-exact; J and Rho within 1e-6 of their
maximum magnitude against the oracle's FP64-accumulated deposit; the field
solver and guard exchange bit-exact on identical inputs.
"""
import numpy as np
import pytest

import oracle
from _cases import mesh_1d, random_fields, random_particles
from _gpu_helpers import Pair, assert_bits, make_params

pytestmark = pytest.mark.gpu

J_TOL = 1e-6  # of max |J| (and max |rho|)


def _fields(m, rng, amp=0.3):
    f = random_fields(m, rng, amp=amp)
    for key in ("E", "B", "Ebg", "Bbg"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 1, 0))
    return f


def _setup(N, nptc, seed, tile=(0, 0), periodic=(True, True), data_interval=1, row_align=4,
           gamma_max=50.0, chunk=0, capacity=None):
    params = make_params(N, periodic=periodic, data_interval=data_interval, tile=tile,
                         capacity=capacity or nptc)
    params.chunk = chunk
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(seed)
    f = _fields(m, rng)
    p = random_particles(m, nptc, rng, gamma_max=gamma_max)
    return Pair(params, f, p, capacity=capacity, row_align=row_align)


@pytest.mark.parametrize("tile", [(4, 4), (8, 8), (16, 16), (16, 8)])
def test_2d_push_deposit_bitexact(tile):
    pr = _setup((64, 48), 6000, seed=1, tile=tile)
    for step in range(4):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL, rho=True)


@pytest.mark.parametrize("chunk", [256, 512, 1024, 2048])
def test_2d_push_deposit_bitexact_chunks(chunk):
    """Every staged-chunk variant (256 and 512 double-buffered, 1024 and 2048
    single-buffered) gives the same bits; tiles of 16 x 16 with 64 particles
    per cell need several chunks."""
    pr = _setup((64, 48), 64 * 48 * 64, seed=7, tile=(16, 16), chunk=chunk)
    for step in range(3):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL, rho=True)


PTC_KEYS = ("x1", "x2", "x3", "p1", "p2", "p3", "E", "cell", "flag", "weight", "id")


def _same_by_id(got, ref, what):
    live_g = got["cell"] != oracle.MAX_CELL
    live_o = ref["cell"] != oracle.MAX_CELL
    ig = np.argsort(got["id"][live_g], kind="stable")
    io = np.argsort(ref["id"][live_o], kind="stable")
    for k in PTC_KEYS:
        assert_bits(got[k][live_g][ig], ref[k][live_o][io], f"{what}: {k}")


def test_2d_upper_half_store_with_rebuilt_order():
    """A grid of 2 x 2 tiles has no incremental tile order (rebuilt from the
    slots every step); with compaction on, a sort moves the store into the
    upper half of a doubled capacity and the rebuilt order must follow it."""
    n = 4096
    pr = _setup((32, 32), n, seed=12, tile=(16, 16), capacity=2 * n)
    pr.env.set_compaction(3)
    for step in range(2):
        pr.both_update_particles(step)
    pr.data.sort_particles()
    n_ref = oracle.sort_by_cell(pr.m, pr.p, len(pr.p["x1"]))
    assert pr.data.slot_range() == (n, n + n_ref)
    for step in range(2, 5):
        pr.both_update_particles(step)
        got = pr.data.particles_host()
        _same_by_id(got, pr.p, f"step {step}")
        pr.check_current(J_TOL, rho=True)


@pytest.mark.parametrize("interval,spare", [(1, 1), (3, 1), (1, 2), (3, 2)])
def test_2d_compaction_keeps_every_particle(interval, spare):
    """With the store rewritten in tile order every `interval` updates (into
    scratch and copied back when the capacity equals the particle count,
    into the free half of a capacity of twice the count) the particles
    change slots but not values: compared by id they equal the oracle bit
    for bit, the current is unchanged, and a sort_by_cell afterwards gives
    the oracle's cells and, per cell, the same particles."""
    n = 20000
    pr = _setup((64, 48), n, seed=8, tile=(8, 8), capacity=spare * n)
    pr.env.set_compaction(interval)
    for step in range(5):
        pr.both_update_particles(step)
        got = pr.data.particles_host()
        first, end = pr.data.slot_range()
        assert end - first <= n and (spare == 2 or first == 0)
        assert np.all(got["cell"][:first] == oracle.MAX_CELL)
        _same_by_id(got, pr.p, f"step {step}")
        pr.check_current(J_TOL, rho=True)
    # slots did move (into the upper half, or within the lower one)
    assert first > 0 or not np.array_equal(got["id"][:len(pr.p["id"])], pr.p["id"])
    pr.data.sort_particles()
    n_ref = oracle.sort_by_cell(pr.m, pr.p, len(pr.p["x1"]))
    first, end = pr.data.slot_range()
    # sorted into slots [0, live), or into the free half with compaction on
    assert end - first == n_ref and first in (0, spare * n // 2)
    got = {k: v[first:end] for k, v in pr.data.particles_host().items()}
    og = np.lexsort((got["id"], got["cell"]))
    oo = np.lexsort((pr.p["id"][:n_ref], pr.p["cell"][:n_ref]))
    assert_bits(got["cell"], pr.p["cell"][:n_ref], "cells after sort_by_cell")
    for k in PTC_KEYS:
        assert_bits(got[k][og], pr.p[k][:n_ref][oo], f"after sort_by_cell: {k}")
    # and the update continues from the sorted store
    pr.both_update_particles(5)
    _same_by_id(pr.data.particles_host(), pr.p, "step 5")


def test_2d_tile_order_is_stable_counting_sort():
    pr = _setup((64, 64), 8000, seed=2, tile=(8, 8))
    tile = (8, 8)
    cells0 = pr.data.particles_host()["cell"]
    keys = np.array([oracle.tile_key(pr.m, tile, int(c)) for c in cells0], np.uint32)
    nt = oracle.tile_key(pr.m, tile, oracle.MAX_CELL)
    order = oracle.stable_counting_sort(keys, nt + 1)
    order = order[keys[order] < nt]
    for step in range(5):
        pr.both_update_particles(step)
        cells = pr.p["cell"]
        order_ref, start_ref = oracle.tile_order(pr.m, tile, cells, order)
        order_gpu, start_gpu = pr.data.tile_order()
        assert_bits(start_gpu, start_ref, f"tile_start step {step}")
        assert_bits(order_gpu, order_ref, f"tile order step {step}")
        order = order_ref


@pytest.mark.parametrize("chunk", [0, 256])
def test_2d_tile_order_with_crowded_tiles(chunk):
    """The one-pass order update (chunk counts from the push / deposit) and
    its two-pass fallback for tiles of more than 128 staged chunks give the
    stable counting sort: one of the 3 x 3 tiles holds 70,000 particles."""
    tile = (16, 16)
    n_bg, n_crowd = 9 * 4000, 70000
    pr = _setup((48, 48), n_bg + n_crowd, seed=13, tile=tile, chunk=chunk)
    m = pr.m
    rng = np.random.default_rng(14)
    g0, g1 = m.guard[0], m.guard[1]
    c1 = rng.integers(g0 + 16, g0 + 32, n_crowd)
    c2 = rng.integers(g1 + 16, g1 + 32, n_crowd)
    pr.p["cell"][n_bg:] = (c1 + c2 * m.dims[0]).astype(np.uint32)
    pr.data.set_particles(pr.p)
    cells0 = pr.p["cell"]
    keys = np.array([oracle.tile_key(m, tile, int(c)) for c in cells0], np.uint32)
    nt = oracle.tile_key(m, tile, oracle.MAX_CELL)
    order = oracle.stable_counting_sort(keys, nt + 1)
    order = order[keys[order] < nt]
    for step in range(3):
        pr.both_update_particles(step)
        order_ref, start_ref = oracle.tile_order(m, tile, pr.p["cell"], order)
        order_gpu, start_gpu = pr.data.tile_order()
        assert_bits(start_gpu, start_ref, f"tile_start step {step}")
        assert_bits(order_gpu, order_ref, f"tile order step {step}")
        order = order_ref
        pr.check_particles()


def test_1d_push_deposit_bitexact():
    params = make_params((512,), periodic=(True,), capacity=4096)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(3)
    f = random_fields(m, rng, amp=0.3)
    for key in ("E", "B"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 0, 0))
    p = random_particles(m, 4096, rng, gamma_max=50.0)
    pr = Pair(params, f, p)
    for step in range(4):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL, rho=True)


@pytest.mark.parametrize("order", ["cell_sorted", "pairs_sorted"])
def test_1d_push_deposit_bitexact_cell_sorted(order):
    """A cell-sorted 1D run with many particles per cell puts the lanes of a
    warp on one or two cells, which is where the deposit sums the lanes'
    fixed-point words before one lane adds them; e-/e+ pairs at the same
    position (as the served runs start) make those lanes add equal values.
    Particles bit-exact, J and Rho within the tolerance, over four steps."""
    params = make_params((256,), periodic=(True,), capacity=256 * 128)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(11)
    f = random_fields(m, rng, amp=0.3)
    for key in ("E", "B"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 0, 0))
    n = 256 * 128
    p = random_particles(m, n if order == "cell_sorted" else n // 2, rng, gamma_max=50.0)
    if order == "pairs_sorted":
        # each particle twice, the copy with the other species bit
        q = {}
        for k, v in p.items():
            q[k] = np.repeat(v, 2)
        q["flag"][1::2] ^= np.uint32(1 << 29)
        q["id"] = np.arange(n, dtype=q["id"].dtype)
        p = q
    perm = np.argsort(p["cell"], kind="stable")
    p = {k: np.ascontiguousarray(v[perm]) for k, v in p.items()}
    pr = Pair(params, f, p)
    for step in range(4):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL, rho=True)


@pytest.mark.parametrize("N", [(64, 48), (512,)])
def test_update_fields_bitexact(N):
    params = make_params(N, capacity=1)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(4)
    per = (1, 1 if m.dimension > 1 else 0, 0)
    f = random_fields(m, rng)
    for c in range(3):
        f["J"][c][:] = (0.1 * rng.standard_normal(f["J"][c].shape)).astype(np.float32)
    for key in ("E", "B", "Ebg", "Bbg"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], per)
    pr = Pair(params, f, random_particles(m, 0, rng))
    for step in range(3):
        pr.both_update_fields(step)
        g = pr.data.fields_host()
        for key in ("E", "B"):
            for c in range(3):
                assert_bits(g[key][c], pr.f[key][c], f"{key}{c + 1} step {step}")
        g0, g1 = m.guard[0], m.guard[1]
        sl = ((slice(g1, m.dims[1] - g1) if m.dimension > 1 else slice(0, 1)),
              slice(g0, m.dims[0] - g0))
        assert_bits(g["divE"][sl], pr.f["divE"][sl], "divE")
        assert_bits(g["divB"][sl], pr.f["divB"][sl], "divB")


@pytest.mark.parametrize("N", [(40, 24), (64,)])
def test_guard_exchange_bitexact(N):
    params = make_params(N, capacity=1)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(5)
    pr = Pair(params, {}, random_particles(m, 0, rng))
    per = (1, 1 if m.dimension > 1 else 0, 0)
    a = rng.standard_normal(pr.f["J"][0].shape).astype(np.float32)
    pr.data.set_fields({"J": [a, a, a]})
    pr.env.send_guard_cells(pr.data.J[0])
    pr.env.send_add_guard_cells(pr.data.J[1])
    ref_copy, ref_add = a.copy(), a.copy()
    oracle.send_guard_cells(m, ref_copy, per)
    oracle.send_add_guard_cells(m, ref_add, per)
    g = pr.data.fields_host()
    assert_bits(g["J"][0], ref_copy, "send_guard_cells")
    assert_bits(g["J"][1], ref_add, "send_add_guard_cells")


def test_sort_by_cell_bitexact():
    params = make_params((32, 32), capacity=5000)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(6)
    p = random_particles(m, 5000, rng)
    holes = rng.random(5000) < 0.1
    p["cell"][holes] = oracle.MAX_CELL
    pr = Pair(params, {}, p)
    pr.data.sort_particles()
    n_ref = oracle.sort_by_cell(m, pr.p, 5000)
    assert pr.data.number == n_ref
    got = pr.data.particles_host()
    for k, _ in oracle.PTC_FIELDS:
        assert_bits(got[k], pr.p[k][:n_ref], f"sorted {k}")


@pytest.mark.parametrize("tile,crowd", [((8, 8), 0), ((16, 16), 0), ((16, 8), 5000)])
def test_sort_by_cell_after_updates_bitexact(tile, crowd):
    """sort_by_cell right after updates (stable radix sort of the cell keys,
    one gather per member) gives the oracle's stable sort slot for slot,
    also with one cell holding `crowd` more particles than the rest."""
    pr = _setup((64, 48), 12000, seed=21, tile=tile, capacity=12000 + crowd)
    if crowd:
        # `crowd` more particles at rest in one cell
        rng = np.random.default_rng(3)
        n0 = len(pr.p["x1"])
        extra = random_particles(pr.m, crowd, rng, gamma_max=1.0)
        c0 = pr.p["cell"][0]
        extra["cell"][:] = c0
        for k in ("p1", "p2", "p3"):
            extra[k][:] = 0
        extra["E"][:] = 1
        extra["id"][:] = np.arange(n0, n0 + crowd, dtype=np.uint64)
        pr.p = {k: np.concatenate([pr.p[k], extra[k]]) for k in pr.p}
        pr.data.set_particles(pr.p)
    for step in range(3):
        pr.both_update_particles(step)
    pr.data.sort_particles()
    n_ref = oracle.sort_by_cell(pr.m, pr.p, len(pr.p["x1"]))
    assert pr.data.number == n_ref and pr.data.slot_range() == (0, n_ref)
    got = pr.data.particles_host()
    for k, _ in oracle.PTC_FIELDS:
        assert_bits(got[k], pr.p[k][:n_ref], f"sorted {k}")
    pr.p = {k: v[:n_ref].copy() for k, v in pr.p.items()}
    pr.both_update_particles(3)
    pr.check_particles()


@pytest.mark.parametrize("N,tile,crowd,spare", [
    ((64, 48), (8, 8), 0, 2), ((64, 48), (16, 8), 0, 2), ((64, 64), (16, 16), 3000, 2),
    ((128, 64), (32, 16), 0, 2), ((64, 48), (8, 8), 0, 1)])
def test_sort_by_cell_is_stable_sort_of_the_store(N, tile, crowd, spare):
    """After compacting updates, sort_by_cell gives, slot for slot and for
    every member, the stable sort by cell of the slots it started from (into
    the free half with spare 2, back into slots [0, live) with spare 1),
    also with one cell holding `crowd` more particles."""
    n = N[0] * N[1] * 6
    pr = _setup(N, n, seed=31, tile=tile, capacity=spare * (n + crowd))
    if crowd:
        rng = np.random.default_rng(4)
        extra = random_particles(pr.m, crowd, rng, gamma_max=1.0)
        extra["cell"][:] = pr.p["cell"][0]
        for k in ("p1", "p2", "p3"):
            extra[k][:] = 0
        extra["id"][:] = np.arange(n, n + crowd, dtype=np.uint64)
        pr.p = {k: np.concatenate([pr.p[k], extra[k]]) for k in pr.p}
        pr.data.set_particles(pr.p)
    pr.env.set_compaction(2)
    for step in range(3):
        pr.pusher.update_particles(pr.data, pr.dt, step)
    first, end = pr.data.slot_range()
    seg = {k: v[first:end].copy() for k, v in pr.data.particles_host().items()}
    live = np.flatnonzero(seg["cell"] != oracle.MAX_CELL)
    order = live[np.argsort(seg["cell"][live], kind="stable")]
    pr.data.sort_particles()
    f2, e2 = pr.data.slot_range()
    assert e2 - f2 == len(order) and (spare == 1 or f2 != first)
    got = {k: v[f2:e2] for k, v in pr.data.particles_host().items()}
    for k in PTC_KEYS:
        assert_bits(got[k], seg[k][order], f"sorted {k}")
    # the tile order after the sort covers exactly the sorted slots
    o, _ = pr.data.tile_order()
    assert np.array_equal(np.sort(o), np.arange(f2, e2, dtype=np.uint32))


def test_tile_order_after_sort_by_cell():
    """sort_by_cell leaves the tile order equal to a stable counting sort by
    tile of the cell-sorted slots, and the next steps stay bit-exact."""
    pr = _setup((64, 48), 6000, seed=17, tile=(8, 8))
    pr.both_update_particles(0)
    pr.data.sort_particles()
    n_ref = oracle.sort_by_cell(pr.m, pr.p, len(pr.p["x1"]))
    pr.p = {k: v[:n_ref].copy() for k, v in pr.p.items()}
    assert pr.data.number == n_ref
    keys = np.array([oracle.tile_key(pr.m, (8, 8), int(c)) for c in pr.p["cell"]], np.uint32)
    nt = oracle.tile_key(pr.m, (8, 8), oracle.MAX_CELL)
    order_ref = oracle.stable_counting_sort(keys, nt + 1)
    order_ref = order_ref[keys[order_ref] < nt]
    order_gpu, start_gpu = pr.data.tile_order()
    assert_bits(order_gpu, order_ref, "tile order after sort_by_cell")
    for step in range(1, 3):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL)


def test_no_tensor_map_path_bitexact():
    """Rows packed to an odd length make the field tiles load without TMA."""
    pr = _setup((61, 45), 4000, seed=7, row_align=1)
    for step in range(3):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL)


def test_empty_and_single_particle():
    pr = _setup((32, 32), 0, seed=8)
    pr.both_update_particles(0)
    assert all(np.abs(j).max() == 0 for j in pr.data.fields_host()["J"])
    pr = _setup((32, 32), 1, seed=9)
    for step in range(3):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL)


def test_lost_through_non_periodic_sides():
    pr = _setup((32, 32), 6000, seed=10, periodic=(False, False), gamma_max=200.0)
    lost = 0
    for step in range(4):
        lost += pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL)
    assert lost > 0
    assert int(pr.data.stats().live) == int(np.sum(pr.p["cell"] != oracle.MAX_CELL))


def test_ignore_flags_bitexact():
    pr = _setup((32, 32), 3000, seed=11)
    rng = np.random.default_rng(12)
    fl = pr.p["flag"]
    fl[rng.random(3000) < 0.2] |= np.uint32(1 << 4)   # ignore_EM
    fl[rng.random(3000) < 0.2] |= np.uint32(1 << 3)   # ignore_current
    pr.data.set_particles(pr.p)
    for step in range(3):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL)


def test_nan_momentum_is_reported_not_trapped():
    from aperture3_b200._lib import ApError
    pr = _setup((32, 32), 500, seed=13)
    pr.p["p1"][7] = np.float32("nan")
    pr.data.set_particles(pr.p)
    with pytest.raises(ApError) as e:
        pr.pusher.update_particles(pr.data, pr.dt, 0)
    assert e.value.status == 3
    assert pr.data.stats().nan_momenta == 1


def test_moved_far_is_reported():
    from aperture3_b200._lib import ApError
    pr = _setup((32, 32), 500, seed=14, gamma_max=1000.0)
    with pytest.raises(ApError) as e:
        pr.pusher.update_particles(pr.data, pr.dt * 8, 0)
    assert e.value.status == 4


def test_bounded_wait_timeout_is_reported_and_context_survives():
    """A device-side wait that nothing completes gives up after its limit and
    comes back as AP_ERR_TIMEOUT; the same context then steps bit-exactly."""
    pr = _setup((32, 32), 800, seed=15, tile=(8, 8))
    st = pr.env._lib.ap_selftest_wait_timeout(pr.env.ctx)
    assert st == 6
    assert pr.env._lib.ap_last_error(pr.env.ctx) == 6
    for step in range(2):
        pr.both_update_particles(step)
        pr.check_particles()
        pr.check_current(J_TOL, rho=True)


def test_continuity_residual():
    """Esirkepov charge conservation through the ABI: rho(t+1) - rho(t) +
    div J = 0 on the bulk, within 1e-6 of max|rho|."""
    pr = _setup((48, 48), 8000, seed=15, tile=(8, 8))
    pr.env.set_continuity_check(True)
    pr.pusher.update_particles(pr.data, pr.dt, 0)
    assert np.isnan(pr.data.diagnostics().continuity_residual)  # no rho(t) yet
    rho0 = sum(r.cpu().double() for r in pr.data.Rho).numpy()
    pr.pusher.update_particles(pr.data, pr.dt, 1)
    g = pr.data.fields_host()
    rho1 = sum(r.astype(np.float64) for r in g["Rho"])
    J1, J2 = g["J"][0].astype(np.float64), g["J"][1].astype(np.float64)
    m = pr.m
    ys = slice(m.guard[1], m.dims[1] - m.guard[1])
    xs = slice(m.guard[0], m.dims[0] - m.guard[0])
    # the upper face of the last bulk cell is the periodic image of the first
    # (the guard cells keep the raw deposit, as the reference leaves them)
    j1, j2 = J1[ys, xs], J2[ys, xs]
    div = (np.roll(j1, -1, axis=1) - j1) + (np.roll(j2, -1, axis=0) - j2)
    res = np.abs(rho1[ys, xs] - rho0[ys, xs] + div).max()
    assert res <= 1e-6 * np.abs(rho1).max(), res
    # the same reduction on the device, in FP64 (ap_set_continuity_check)
    dev = pr.data.diagnostics().continuity_residual
    assert np.isclose(dev, res, rtol=1e-12, atol=1e-300), (dev, res)


def test_coupled_steps_within_tolerance():
    """Particles + fields for several steps: the GPU's J is not summed in the
    oracle's order, so coupled runs are compared within the stated
    tolerances (momenta 1e-5 relative)."""
    pr = _setup((48, 48), 6000, seed=16, tile=(8, 8))
    for step in range(5):
        pr.pusher.update_particles(pr.data, pr.dt, step)
        pr.solver.update_fields(pr.data, pr.dt, step)
        pr.step = step
        oracle.update_particles(pr.m, pr.p, len(pr.p["x1"]), pr.f, pr.dt, step, 1, 2, 0,
                                pr.env.charges, pr.env.masses, pr.periodic)
        oracle.update_fields(pr.m, pr.f, pr.dt, step, pr.periodic)
    got = pr.data.particles_host()
    same_cell = got["cell"] == pr.p["cell"]
    assert same_cell.mean() > 0.999
    for k in ("p1", "p2", "p3"):
        a, b = got[k].astype(np.float64), pr.p[k].astype(np.float64)
        scale = np.maximum(np.abs(b), 1e-3)
        assert (np.abs(a - b) / scale).max() <= 1e-5, k


def test_fp64_diagnostics_sync_and_async():
    """ap_diagnostics (and ap_diagnostics_async into pinned memory) against
    the same reductions in numpy FP64 on the copied state: kinetic energy
    sum w m (gamma - 1), total charge, field energy 1/2 sum(E^2 + B^2) dV
    over the bulk, max |rho|, max |divE - rho|, max |J|."""
    import ctypes as C

    import torch
    pr = _setup((64, 48), 20000, seed=31, tile=(8, 8), capacity=40000)
    pr.env.set_compaction(2)
    for step in range(3):
        pr.both_update_particles(step)
        pr.both_update_fields(step)
    d = pr.data.diagnostics()
    host = torch.zeros(7, dtype=torch.float64).pin_memory()
    check_status = pr.env._lib.ap_diagnostics_async(pr.env.ctx, C.c_void_p(host.data_ptr()))
    assert check_status == 0
    pr.env.sync()
    got = pr.data.particles_host()
    live = got["cell"] != oracle.MAX_CELL
    sp = (got["flag"][live] >> 29).astype(np.int64)
    p2 = sum(got[k][live].astype(np.float64) ** 2 for k in ("p1", "p2", "p3"))
    w = got["weight"][live].astype(np.float64)
    charges = np.array(pr.env.charges, np.float64)
    masses = np.array(pr.env.masses, np.float64)
    kin = np.sum(w * masses[sp] * (p2 / (np.sqrt(1.0 + p2) + 1.0)))
    q = np.sum(w * charges[sp])
    g = pr.data.fields_host()
    m = pr.m
    sl = (slice(m.guard[1], m.dims[1] - m.guard[1]), slice(m.guard[0], m.dims[0] - m.guard[0]))
    en = 0.5 * sum(np.sum(g[k][c][sl].astype(np.float64) ** 2)
                   for k in ("E", "B") for c in range(3)) * float(m.delta[0]) * float(m.delta[1])
    rho = sum(g["Rho"][s][sl].astype(np.float64) for s in range(len(g["Rho"])))
    ref = [kin, q, en, np.abs(rho).max(), np.abs(g["divE"][sl].astype(np.float64) - rho).max(),
           max(np.abs(g["J"][c][sl]).max() for c in range(3))]
    vals = [d.kinetic, d.charge, d.field_energy, d.max_abs_rho, d.gauss_residual, d.max_abs_j]
    for name, a, b, c in zip(("kinetic", "charge", "field", "rho", "gauss", "J"), vals,
                             host.numpy(), ref):
        assert np.isclose(a, c, rtol=1e-10, atol=1e-12), (name, a, c)
        assert np.isclose(b, c, rtol=1e-10, atol=1e-12), (name, b, c)


@pytest.mark.parametrize("N,periodic", [((64, 48), (True, True)), ((64, 48), (False, True)),
                                        ((96,), (True, True)), ((96,), (False, False))])
def test_smooth_array_bitexact(N, periodic):
    """smooth_current(multi_array&) (filter_current_cart_{1,2}d,
    ptc_updater.cu:501-560) on one array: the bulk equals the oracle's
    binomial filter bit for bit, with and without boundary sides."""
    pr = _setup(N, 10, seed=41, periodic=periodic)
    rng = np.random.default_rng(42)
    a = rng.standard_normal(pr.f["J"][0].shape).astype(np.float32)
    import torch
    dev = pr.data.J[0]
    dev.copy_(torch.from_numpy(a).reshape(dev.shape))
    pr.pusher.smooth_current(dev)
    got = dev.cpu().numpy().reshape(a.shape)
    ref = a.copy()
    bnd = (int(not pr.periodic[0]), int(not pr.periodic[0]), int(not pr.periodic[1]),
           int(not pr.periodic[1]))
    oracle.filter_current(pr.m, ref, np.zeros_like(ref), bnd)
    m = pr.m
    sl = (slice(m.guard[1], m.dims[1] - m.guard[1]) if m.dimension > 1 else slice(0, 1),
          slice(m.guard[0], m.dims[0] - m.guard[0]))
    assert_bits(got[sl], ref[sl], "filtered bulk")


@pytest.mark.parametrize("N", [(64, 48), (512,)])
@pytest.mark.parametrize("smoothing", [1, 2, 3])
def test_update_with_current_smoothing(N, smoothing):
    """update_particles with current_smoothing passes (smooth_current,
    ptc_updater.cu:852-873): J and Rho equal the oracle's filter passes
    (each followed by the periodic guard copy) applied to the same
    update's unsmoothed current, bit for bit; the particles are unchanged
    by the smoothing."""
    n = 8000
    raw = _setup(N, n, seed=43)
    params = make_params(N, smoothing=smoothing, capacity=n)
    sm = Pair(params, raw.f, raw.p)
    for step in range(2):
        raw.pusher.update_particles(raw.data, raw.dt, step)
        sm.pusher.update_particles(sm.data, sm.dt, step)
        assert_bits(sm.data.particles_host()["p1"], raw.data.particles_host()["p1"], "p1")
        g_raw, g_sm = raw.data.fields_host(), sm.data.fields_host()
        m = raw.m
        bnd = (int(not raw.periodic[0]),) * 2 + (int(not raw.periodic[1]),) * 2
        J = [g_raw["J"][c].copy() for c in range(3)]
        R = [r.copy() for r in g_raw["Rho"]]
        tmp = np.zeros_like(J[0])
        for _ in range(smoothing):
            for c in range(3):
                oracle.filter_current(m, J[c], tmp, bnd)
                oracle.send_guard_cells(m, J[c], raw.periodic)
            for r in R:  # data_interval 1: every step has charge output
                oracle.filter_current(m, r, tmp, bnd)
                oracle.send_guard_cells(m, r, raw.periodic)
        for c in range(3):
            assert_bits(g_sm["J"][c], J[c], f"step {step}: J{c + 1}")
        for s, r in enumerate(R):
            assert_bits(g_sm["Rho"][s], r, f"step {step}: Rho{s}")
