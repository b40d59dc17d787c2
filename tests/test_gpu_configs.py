"""Parity at the sizes of the benchmark workloads (run on a B200).

The other parity tests use small grids; these run the seeded initial
states of the benchmarked configurations (aperture3_b200.ic) at their own
sizes, or at a labelled reduction where the CPU oracle would take minutes:

* 1D periodic plain PIC: 4096 cells, 2^20 particles, seed 0, 100 coupled
  steps of update_particles + update_fields, at full size;
* 2D box: 256 x 256 cells at 64 particles per cell with 16 x 16 tiles, so
  every tile holds the 16,384 particles the 1024^2 x 64 ppc box has per
  tile (the population that sets the fixed-point current format), with
  compaction into a doubled capacity as in the benchmark, then a
  sort_by_cell.

Coupled runs are compared in lock step: each step the oracle's field solver
is given the current the GPU deposited (after that current has been checked
against the oracle's FP64-accumulated deposit), so that E and B stay
identical and the particles can be compared bit for bit after every step.
Bars: particles bit-exact; J and Rho within 1e-6 of their maximum; the
continuity residual rho(t+1) - rho(t) + div J within 1e-6 of the largest
charge density the species deposit, max over cells of sum_s |rho_s|. (The
1D state is a pair plasma whose e- and e+ start at the same positions, so
the net density is a small difference of two densities of about 128 each;
each is stored in FP32, and their rounding, not the deposit, sets the
floor of the residual. Normalised by the net density the same residual
reads about 3e-6.)
"""
import numpy as np
import pytest

import oracle
from _gpu_helpers import Pair, assert_bits
from aperture3_b200 import ic

pytestmark = pytest.mark.gpu

TOL = 1e-6
PTC_KEYS = ("x1", "x2", "x3", "p1", "p2", "p3", "E", "cell", "flag", "weight", "id")


def _pair(params, fields, ptc, capacity=None):
    host_f = {k: [c.cpu().numpy() for c in v] for k, v in fields.items()}
    return Pair(params, host_f, ic.to_numpy_ptc(ptc), capacity=capacity)


def _lock_step_fields(pr, step):
    """Field update on both sides from the GPU's current."""
    g = pr.data.fields_host()
    for c in range(3):
        pr.f["J"][c][:] = g["J"][c]
    pr.both_update_fields(step)


def _continuity_1d(rho0, rho1, J1, g):
    """max |rho1 - rho0 + div J| over the bulk (the face past the last bulk
    cell is the first one's periodic image) and max |rho1| there."""
    sl = slice(g, rho1.shape[-1] - g)
    r0, r1, j = rho0[..., sl], rho1[..., sl], J1[..., sl]
    div = np.roll(j, -1, axis=-1) - j
    return np.abs(r1 - r0 + div).max(), np.abs(r1).max()


def _species_scale(rhos, g):
    """max over bulk cells of sum_s |rho_s|."""
    sl = slice(g, rhos[0].shape[-1] - g)
    return sum(np.abs(r[..., sl].astype(np.float64)) for r in rhos).max()


def test_config1_full_size_100_coupled_steps():
    params, fields, ptc = ic.box1d(seed=0)
    assert params.N[0] == 4096 and ptc["x1"].numel() == 1 << 20
    pr = _pair(params, fields, ptc)
    pr.env.set_continuity_check(True)
    g0 = params.guard[0]
    rho_prev = None
    worst = {"J": 0.0, "Rho": 0.0, "continuity": 0.0}
    for step in range(100):
        lost = pr.both_update_particles(step)
        assert lost == 0
        errs = pr.check_current(TOL, rho=True)
        worst["J"] = max(worst["J"], *(errs[f"J{c}"] for c in (1, 2, 3)))
        worst["Rho"] = max(worst["Rho"], errs["Rho0"], errs["Rho1"])
        g = pr.data.fields_host()
        rho = sum(r.astype(np.float64) for r in g["Rho"])
        if rho_prev is not None:
            raw, scale = _continuity_1d(rho_prev, rho, g["J"][0].astype(np.float64), g0)
            res = raw / _species_scale(g["Rho"], g0)
            assert res <= TOL, f"step {step}: continuity residual {res:.3g}"
            # the same reduction on the device (ap_set_continuity_check)
            dev = pr.data.diagnostics()
            assert np.isclose(dev.continuity_residual, raw, rtol=1e-9, atol=1e-300), \
                (step, dev.continuity_residual, raw)
            assert np.isclose(dev.max_abs_rho, scale, rtol=1e-12)
            worst["continuity"] = max(worst["continuity"], res)
        rho_prev = rho
        _lock_step_fields(pr, step)
        if step % 10 == 9:
            pr.check_particles(PTC_KEYS)
            got = pr.data.fields_host()
            for key in ("E", "B"):
                for c in range(3):
                    assert_bits(got[key][c], pr.f[key][c], f"step {step}: {key}{c + 1}")
    print("config 1 worst errors over 100 steps:", worst)


def _same_by_id(got, ref, what):
    live_g = got["cell"] != oracle.MAX_CELL
    live_o = ref["cell"] != oracle.MAX_CELL
    assert live_g.sum() == live_o.sum(), what
    ig = np.argsort(got["id"][live_g], kind="stable")
    io = np.argsort(ref["id"][live_o], kind="stable")
    for k in PTC_KEYS:
        assert_bits(got[k][live_g][ig], ref[k][live_o][io], f"{what}: {k}")


def test_config2_tile_population_with_compaction_and_sort():
    params, fields, ptc = ic.box2d(seed=3, N=256, ppc=64, tile=(16, 16), data_interval=1)
    n = ptc["x1"].numel()
    assert n == 256 * 256 * 64
    pr = _pair(params, fields, ptc, capacity=2 * n)
    pr.env.set_compaction(2)
    for step in range(4):
        pr.both_update_particles(step)
        _same_by_id(pr.data.particles_host(), pr.p, f"step {step}")
        pr.check_current(TOL, rho=True)
        _lock_step_fields(pr, step)
    # the tile population that set the fixed-point format
    o, starts = pr.data.tile_order()
    assert int(np.diff(starts).max()) >= 16 * 16 * 64 - 1024
    # sort_by_cell of the compacted store: the stable sort by cell of the
    # slots it started from
    first, end = pr.data.slot_range()
    seg = {k: v[first:end].copy() for k, v in pr.data.particles_host().items()}
    live = np.flatnonzero(seg["cell"] != oracle.MAX_CELL)
    order = live[np.argsort(seg["cell"][live], kind="stable")]
    pr.data.sort_particles()
    f2, e2 = pr.data.slot_range()
    assert e2 - f2 == n
    got = {k: v[f2:e2] for k, v in pr.data.particles_host().items()}
    for k in PTC_KEYS:
        assert_bits(got[k], seg[k][order], f"sorted {k}")
    # and the next update continues bit-exactly from the sorted store
    pr.both_update_particles(4)
    _same_by_id(pr.data.particles_host(), pr.p, "step 4")
    pr.check_current(TOL, rho=True)
