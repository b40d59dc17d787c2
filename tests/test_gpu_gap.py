"""1D gap lab on the GPU (ptc_updater_1dgap / field_solver_1dgap through
ap_ctx_create_1dgap) against the oracle, itself pinned to the lab's own
kernels: particles bit for bit, the smoothed E3 (and its scratch E2) bit for
bit, J1 and Rho within 1e-6 of their maximum of the FP64-accumulated
deposit (the library sums exactly in fixed point, the reference in float
atomics), the E1 update bit for bit."""
import numpy as np
import pytest

import oracle
from _cases import GAP_CHARGES, GAP_MASSES, gap_state, mesh_gap
from _gpu_helpers import assert_bits
from aperture3_b200 import (SimData, SimEnvironment, SimParams, field_solver_1dgap,
                            ptc_updater_1dgap)

pytestmark = pytest.mark.gpu

REL = 1e-6


def _setup(N, lower, n, seed, smoothing, B0=0.7):
    rng = np.random.default_rng(seed)
    m = mesh_gap(N, lower)
    E1, p = gap_state(m, n, rng)
    params = SimParams(N=(N, 1, 1), guard=(2, 0, 0), lower=(lower, 0.0, 0.0),
                       size=(1.0, 1.0, 1.0), delta_t=float(np.float32(0.5 * m.delta[0])),
                       q_e=1.0, num_species=2, periodic_boundary=(False, False, False),
                       current_smoothing=smoothing, max_ptc_number=n, B0=B0,
                       coord_system="1dgap")
    env = SimEnvironment(params)
    data = SimData(env, capacity=n)
    f = oracle.new_fields(m, 2)
    f["E"][0][:] = E1
    f["E"][1][:] = np.float32(0.25)  # scratch of the smoothing: overwritten when smoothing > 0
    f["E"][2][:] = np.float32(-3.0)
    data.set_fields(f)
    data.set_particles(p)
    return m, env, data, f, oracle.copy_ptc(p)


def _flat(a, n):
    return np.ascontiguousarray(a).reshape(-1)[:n]


def _smooth64(m, a, times, bnd):
    """The gap filter in FP64 (same stencil, ends and zero padding)."""
    n, g = m.dims[0], m.guard[0]
    for _ in range(times):
        out = np.empty_like(a)
        for i in range(n):
            dp = 0 if (bnd[1] and i == n - g - 1) else 1
            dm = 0 if (bnd[0] and i == g) else 1
            jp = a[i + dp] if i + dp < n else 0.0
            jm = a[i - dm] if i - dm >= 0 else 0.0
            out[i] = 0.5 * a[i] + 0.25 * jp + 0.25 * jm
        a = out
    return a


@pytest.mark.parametrize("N,lower,smoothing", [(256, 0.0, 0), (300, -0.6, 1), (512, 0.2, 3)])
def test_gap_update_particles(N, lower, smoothing):
    m, env, data, f, p = _setup(N, lower, 6000, 7 + N, smoothing)
    n = m.dims[0]
    dt = env.params.delta_t
    ptc_updater_1dgap(env).update_particles(data, dt, 0)
    # oracle: the full update (float J) and the FP64 deposit for the current
    bnd = (1, 1)
    fo = oracle.copy_fields(f)
    po = oracle.copy_ptc(p)
    oracle.update_particles_1dgap(m, po, len(p["x1"]), fo, dt, smoothing, 2, GAP_CHARGES,
                                  GAP_MASSES, bnd)
    p64 = oracle.copy_ptc(p)
    J64 = np.zeros(n)
    R64 = [np.zeros(n) for _ in range(2)]
    oracle.update_ptc_1dgap(m, p64, len(p["x1"]), dt, fo["E"][2], J64, R64, GAP_CHARGES,
                            GAP_MASSES, f64=True)
    got = data.particles_host()
    for k in po:
        assert_bits(got[k], po[k], f"particles.{k}")
    g = data.fields_host()
    assert_bits(_flat(g["E"][2], n), _flat(fo["E"][2], n), "E3 (smoothed E1)")
    assert_bits(_flat(g["E"][1], n), _flat(fo["E"][1], n), "E2 (smoothing scratch)")
    for name, got_a, ref in [("J1", g["J"][0], _smooth64(m, J64, smoothing, bnd))] + [
            (f"Rho{s}", g["Rho"][s], _smooth64(m, R64[s], smoothing, bnd)) for s in range(2)]:
        scale = max(np.abs(ref).max(), 1e-30)
        err = np.abs(_flat(got_a, n).astype(np.float64) - ref).max() / scale
        assert err <= REL, f"{name}: {err:.3g} of max"
    assert np.abs(_flat(g["J"][1], n)).max() == 0 and np.abs(_flat(g["J"][2], n)).max() == 0
    env.close()


def test_gap_update_fields():
    m, env, data, f, p = _setup(300, 0.0, 2000, 3, 0, B0=1.3)
    n = m.dims[0]
    dt = env.params.delta_t
    ptc_updater_1dgap(env).update_particles(data, dt, 0)
    g0 = data.fields_host()
    field_solver_1dgap(env).update_fields(data, dt, 0.0)
    g1 = data.fields_host()
    E1 = _flat(g0["E"][0], n).copy()
    oracle.update_fields_1dgap(m, E1, _flat(g0["J"][0], n).copy(), 1.3, dt)
    assert_bits(_flat(g1["E"][0], n), E1, "E1")
    env.close()


def test_gap_multi_step_run():
    """Five particle + field steps: the coupled run stays within 1e-5 of the
    oracle's (the current differs from the reference's float sums in the
    last bits, and that feeds back through E1); nothing is lost."""
    m, env, data, f, p = _setup(256, -0.3, 4000, 11, 1)
    n = m.dims[0]
    dt = env.params.delta_t
    pu, fs = ptc_updater_1dgap(env), field_solver_1dgap(env)
    fo, po = oracle.copy_fields(f), oracle.copy_ptc(p)
    for step in range(5):
        pu.update_particles(data, dt, step)
        fs.update_fields(data, dt, 0.0)
        oracle.update_particles_1dgap(m, po, len(p["x1"]), fo, dt, 1, 2, GAP_CHARGES,
                                      GAP_MASSES, (1, 1))
        oracle.update_fields_1dgap(m, fo["E"][0], fo["J"][0], 0.7, dt)
    got = data.particles_host()
    live_g, live_o = got["cell"] != oracle.MAX_CELL, po["cell"] != oracle.MAX_CELL
    assert np.array_equal(live_g, live_o)
    for k in ("p1", "E", "x1"):
        a, b = got[k][live_g].astype(np.float64), po[k][live_o].astype(np.float64)
        assert np.allclose(a, b, rtol=1e-5, atol=1e-5), k
    g = data.fields_host()
    assert np.allclose(_flat(g["E"][0], n), _flat(fo["E"][0], n), rtol=1e-5, atol=1e-6)
    env.close()
