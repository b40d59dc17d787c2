"""Log-spherical (ln r, theta) path on the GPU against the CPU oracle.

The GPU evaluates the reference's expressions in FP32 with CUDA's float
transcendentals (expf, sinf, cosf, acosf, logf, atan2f), as the reference's
device code does; the FP32 oracle uses the C library's. Both round
differently in the last bits, so the particle move is compared by its error
against the FP64 oracle: the GPU's FP32 error must not exceed the
FP32 oracle's by more than a small factor. Everything without a
transcendental (the coefficients, the divergences, the field update away
from the axis rows when compactness is 0) is compared bit for bit.
"""
import numpy as np
import pytest

import oracle
from oracle import logsph as ls
from _cases import (LS_CHARGES, LS_MASSES, logsph_dt, logsph_fields, logsph_particles,
                    mesh_logsph)
from _gpu_helpers import assert_bits
from aperture3_b200 import (SimData, SimEnvironment, SimParams, field_solver_logsph,
                            ptc_updater_logsph)

pytestmark = pytest.mark.gpu

NSP = 3
# GPU error / FP32-oracle error against FP64, and the floor below which an
# error counts as FP32 rounding (relative)
ERR_FACTOR = 4.0
ERR_FLOOR = 2e-6


def _params(m, smoothing=0, data_interval=1, **lsp):
    kw = dict(compactness=0.0, omega=0.1, gravity=0.0, rad_cooling_on=False,
              rad_cooling_coef=1.0, damping_length=16, damping_coef=0.002, B0=1.0)
    kw.update(lsp)
    N = (m.dims[0] - 2 * m.guard[0], m.dims[1] - 2 * m.guard[1], 1)
    return SimParams(N=N, guard=(m.guard[0], m.guard[1], 0), lower=(0.0, 0.0, 0.0),
                     size=(m.sizes[0], m.sizes[1], 1.0), delta_t=float(logsph_dt(m)),
                     q_e=1.0, ion_mass=10.0, num_species=NSP,
                     periodic_boundary=(False, False, False), data_interval=data_interval,
                     current_smoothing=smoothing, coord_system="LogSpherical", **kw), kw


class LsCase:
    """One log-spherical state on the GPU, in the FP32 oracle and in the FP64
    oracle."""

    def __init__(self, N, n, seed, gamma_max=1e6, smoothing=0, data_interval=1, **lsp):
        rng = np.random.default_rng(seed)
        self.m = m = mesh_logsph(*N)
        self.params, kw = _params(m, smoothing, data_interval, **lsp)
        self.lp = ls.ls_params(**{k: kw[k] for k in ("compactness", "omega", "gravity",
                                                     "rad_cooling_coef", "B0", "damping_coef",
                                                     "rad_cooling_on", "damping_length")})
        self.f = logsph_fields(m, rng, num_species=NSP)
        self.p = logsph_particles(m, n, rng, gamma_max=gamma_max)
        self.n = n
        self.dt = np.float32(self.params.delta_t)
        self.env = SimEnvironment(self.params)
        self.data = SimData(self.env, capacity=n)
        self.data.set_fields(self.f)
        self.data.set_particles(self.p)
        self.pusher = ptc_updater_logsph(self.env)
        self.solver = field_solver_logsph(self.env)
        self.c32 = ls.coef(m)
        self.c64 = ls.coef(m, f64=True)
        self.p64 = ls.to_f64(self.p)
        self.f64 = ls.fields_to_f64(self.f)
        self.smoothing = smoothing
        self.di = data_interval

    def step_particles(self, step):
        self.pusher.update_particles(self.data, float(self.dt), step)
        r32 = ls.update_particles(self.m, self.lp, self.p, self.n, self.f, self.c32, self.dt,
                                  step, self.di, NSP, self.smoothing, LS_CHARGES, LS_MASSES)
        r64 = ls.update_particles(self.m, self.lp, self.p64, self.n, self.f64, self.c64,
                                  self.dt, step, self.di, NSP, self.smoothing, LS_CHARGES,
                                  LS_MASSES)
        return r32, r64

    def step_fields(self, omega=None):
        self.solver.update_fields(self.data, float(self.dt))
        ls.update_fields(self.m, self.lp, self.f, self.c32, self.dt)
        ls.update_fields(self.m, self.lp, self.f64, self.c64, self.dt)
        if omega is not None:
            self.solver.apply_boundary(self.data, omega)
            ls.field_boundary(self.m, self.lp, self.f, np.float32(omega))
            ls.field_boundary(self.m, self.lp, self.f64, np.float32(omega))

    def close(self):
        self.env.close()


def _phys(m, p):
    """Physical (ln r, theta) position in cells of every live particle."""
    c = p["cell"].astype(np.int64)
    live = p["cell"] != oracle.MAX_CELL
    c1 = c % m.dims[0]
    c2 = c // m.dims[0]
    return live, c1 + p["x1"].astype(np.float64), c2 + p["x2"].astype(np.float64)


def _p(p):
    return np.stack([p["p1"], p["p2"], p["p3"]]).astype(np.float64)


def _errors(m, a, ref):
    """Position error (cells) and relative momentum error of a against ref
    over particles live in both; and the fraction live in only one."""
    la, xa, ya = _phys(m, a)
    lr, xr, yr = _phys(m, ref)
    both = la & lr
    pos = np.hypot(xa - xr, ya - yr)[both]
    pa, pr = _p(a)[:, both], _p(ref)[:, both]
    mom = np.linalg.norm(pa - pr, axis=0) / np.maximum(np.linalg.norm(pr, axis=0), 1e-30)
    return pos, mom, float(np.mean(la != lr))


def _check_against_f64(case, what):
    pos_g, mom_g, dead_g = _errors(case.m, case.data.particles_host(), case.p64)
    pos_o, mom_o, dead_o = _errors(case.m, case.p, case.p64)
    for name, g, o in (("position", pos_g, pos_o), ("momentum", mom_g, mom_o)):
        for q in (50, 99):
            eg, eo = np.percentile(g, q), np.percentile(o, q)
            assert eg <= ERR_FACTOR * eo + ERR_FLOOR, \
                f"{what}: {name} p{q} error {eg:.3g} vs FP32 oracle {eo:.3g}"
    assert dead_g <= 2 * dead_o + 1e-3, (what, dead_g, dead_o)
    return {"pos_p99": float(np.percentile(pos_g, 99)), "mom_p99": float(np.percentile(mom_g, 99))}


def _current_errors(case):
    g = case.data.fields_host()
    out = {}
    for key, arrs, arrs64 in (("J", case.f["J"], case.f64["J"]),
                              ("Rho", case.f["Rho"], case.f64["Rho"])):
        for k, (a32, a64) in enumerate(zip(arrs, arrs64)):
            gk = g[key][k].astype(np.float64)
            scale = max(np.abs(a64).max(), 1e-30)
            eg = np.abs(gk - a64).max() / scale
            eo = np.abs(a32.astype(np.float64) - a64).max() / scale
            dg = np.percentile(np.abs(gk - a64) / scale, 99.9)
            do = np.percentile(np.abs(a32.astype(np.float64) - a64) / scale, 99.9)
            out[f"{key}{k}"] = (eg, eo, float(dg), float(do))
    return out


def test_coefficients_bit_exact():
    """Grid_LogSph::compute_coef on the library's host side, uploaded, equals
    the oracle (and so the reference) bit for bit."""
    case = LsCase((64, 32), 1000, 0)
    for k, name in enumerate(ls.COEF_NAMES):
        assert_bits(case.env.logsph_coef(k), case.c32[k], name)
    case.close()


@pytest.mark.parametrize("opts", [
    {},
    {"compactness": 0.5, "omega": 0.2},
    {"gravity": 0.3, "rad_cooling_on": True, "rad_cooling_coef": 0.05, "compactness": 0.4},
])
def test_one_step_against_fp64(opts):
    """One ptc_updater_logsph step: particles and J / Rho against the FP64
    oracle, no worse than the FP32 oracle, in the maximum and at the 99.9th
    percentile of the cells (errors relative to max|J|)."""
    case = LsCase((128, 64), 40000, 3, **opts)
    case.step_particles(0)
    _check_against_f64(case, f"step 0 {opts}")
    for name, (eg, eo, dg, do) in _current_errors(case).items():
        print(f"{name}: max error {eg:.3g} (FP32 oracle {eo:.3g}), "
              f"p99.9 {dg:.3g} (FP32 oracle {do:.3g})")
        assert eg <= ERR_FACTOR * eo + 1e-5, f"{name}: {eg:.3g} vs FP32 oracle {eo:.3g}"
        assert dg <= ERR_FACTOR * do + 1e-6, f"{name}: p99.9 {dg:.3g} vs FP32 oracle {do:.3g}"
    got = case.data.particles_host()
    same = got["cell"] == case.p["cell"]
    assert same.mean() > 0.999
    # ptc_outflow flags and the untouched members
    assert_bits(got["flag"][same], case.p["flag"][same], "flag")
    assert_bits(got["weight"], case.p["weight"], "weight")
    assert_bits(got["id"], case.p["id"], "id")
    case.close()


def test_axis_reflection_and_outflow_ran():
    """Particles crossing theta = 0 / pi are reflected (same cell rows as the
    oracle) and particles deep in the damping layer get ignore_EM."""
    case = LsCase((64, 64), 30000, 5, damping_length=40)
    case.step_particles(0)
    got = case.data.particles_host()
    row = (got["cell"].astype(np.int64) // case.m.dims[0])
    live = got["cell"] != oracle.MAX_CELL
    g = case.m.guard[1]
    assert np.any(live & (row == g)) and np.any(live & (row == case.m.dims[1] - g - 1))
    flagged = (got["flag"] & (1 << 4)) != 0
    assert flagged.sum() > 0
    assert np.array_equal(flagged, (case.p["flag"] & (1 << 4)) != 0) or \
        np.mean(flagged != ((case.p["flag"] & (1 << 4)) != 0)) < 1e-3
    case.close()


@pytest.mark.parametrize("compactness", [0.0, 0.5])
def test_field_update(compactness):
    """field_solver_logsph::update_fields: bit-exact except the two E1 rows
    whose update uses expf (theta = pi row and the axis guard row), which
    with compactness 0 is the only transcendental; with compactness > 0
    beta_phi (sinf, expf) enters B3 and the check is relative."""
    case = LsCase((128, 64), 10, 7, compactness=compactness)
    rng = np.random.default_rng(7)
    J = [(0.01 * rng.standard_normal(case.f["J"][0].shape)).astype(np.float32) for _ in range(3)]
    for k in range(3):
        case.f["J"][k][:] = J[k]
    case.data.set_fields(case.f)
    case.f64 = ls.fields_to_f64(case.f)
    case.step_fields()
    g = case.data.fields_host()
    m = case.m
    rows_exp = [m.guard[1] - 1, m.dims[1] - m.guard[1] - 1]
    for key in ("E", "B"):
        for k in range(3):
            a, b = g[key][k], case.f[key][k]
            if compactness == 0.0:
                mask = np.ones(a.shape, bool)
                if key == "E" and k == 0:
                    mask[rows_exp, :] = False
                assert_bits(a[mask], b[mask], f"{key}{k + 1}")
            scale = max(np.abs(b).max(), 1e-30)
            assert np.abs(a.astype(np.float64) - b).max() / scale < 1e-6, f"{key}{k + 1}"
    assert_bits(g["divB"], case.f["divB"], "divB")
    scale = np.abs(case.f["divE"]).max()
    assert np.abs(g["divE"].astype(np.float64) - case.f["divE"]).max() / scale < 1e-5
    case.close()


@pytest.mark.parametrize("damping_length", [12, 67])
def test_field_boundary(damping_length):
    """Stellar surface, outflow damping and axis boundaries. 12: the bands
    of the stellar and the damped columns are apart (one thread per cell);
    67 of the 68 columns: the damped band reaches into the stellar one and
    each row is processed in the reference's order (stellar first)."""
    case = LsCase((64, 32), 10, 8, compactness=0.3, damping_length=damping_length,
                  damping_coef=0.3)
    case.step_fields(omega=0.07)
    g = case.data.fields_host()
    for key in ("E", "B"):
        for k in range(3):
            a, b = g[key][k].astype(np.float64), case.f[key][k]
            scale = max(np.abs(b).max(), 1e-30)
            assert np.abs(a - b).max() / scale < 1e-6, f"{key}{k + 1}"
    case.close()


def _live_by_id(p):
    live = p["cell"] != oracle.MAX_CELL
    order = np.argsort(p["id"][live], kind="stable")
    return {k: v[live][order] for k, v in p.items()}


def _errors_by_id(m, a, ref):
    """_errors over the particles live in both, matched by id (the GPU run
    sorts its store, the oracles do not)."""
    a, ref = _live_by_id(a), _live_by_id(ref)
    _, ia, ir = np.intersect1d(a["id"], ref["id"], assume_unique=True, return_indices=True)
    a = {k: v[ia] for k, v in a.items()}
    ref = {k: v[ir] for k, v in ref.items()}
    _, xa, ya = _phys(m, a)
    _, xr, yr = _phys(m, ref)
    pos = np.hypot(xa - xr, ya - yr)
    pa, pr = _p(a), _p(ref)
    mom = np.linalg.norm(pa - pr, axis=0) / np.maximum(np.linalg.norm(pr, axis=0), 1e-30)
    return pos, mom


@pytest.mark.parametrize("smoothing,data_interval", [(0, 2), (2, 1)])
def test_multi_step_run(smoothing, data_interval):
    """Ten coupled steps (particles, fields, boundaries, a sort on the GPU):
    against the FP64 oracle run alongside, the GPU's particle errors (p50,
    p99, matched by id) and current errors (maximum and 99.9th percentile of
    the cells, relative to max|J|) stay within ERR_FACTOR of the FP32
    oracle's own; the live count and the total weight agree with the FP32
    oracle."""
    case = LsCase((96, 64), 30000, 9, gamma_max=1e4, smoothing=smoothing,
                  data_interval=data_interval, compactness=0.2)
    for step in range(10):
        case.step_particles(step)
        case.step_fields(omega=0.05)
        if step == 4:
            case.data.sort_particles()
    got = case.data.particles_host()
    live_g = int((got["cell"] != oracle.MAX_CELL).sum())
    live_o = int((case.p["cell"] != oracle.MAX_CELL).sum())
    assert abs(live_g - live_o) <= max(3, live_o // 1000), (live_g, live_o)
    w = lambda p: float((p["weight"].astype(np.float64) * (p["cell"] != oracle.MAX_CELL)).sum())
    assert abs(w(got) - w(case.p)) <= 1e-3 * w(case.p)
    pos_g, mom_g = _errors_by_id(case.m, got, case.p64)
    pos_o, mom_o = _errors_by_id(case.m, case.p, case.p64)
    for name, g, o in (("position", pos_g, pos_o), ("momentum", mom_g, mom_o)):
        for q in (50, 99):
            eg, eo = np.percentile(g, q), np.percentile(o, q)
            print(f"{name} p{q}: GPU {eg:.3g}, FP32 oracle {eo:.3g}")
            assert eg <= ERR_FACTOR * eo + ERR_FLOOR, f"{name} p{q}: {eg:.3g} vs {eo:.3g}"
    for name, (eg, eo, dg, do) in _current_errors(case).items():
        print(f"{name}: max {eg:.3g} (FP32 oracle {eo:.3g}), p99.9 {dg:.3g} ({do:.3g})")
        assert eg <= ERR_FACTOR * eo + 1e-5, f"{name}: {eg:.3g} vs FP32 oracle {eo:.3g}"
        assert dg <= ERR_FACTOR * do + 1e-6, f"{name}: p99.9 {dg:.3g} vs FP32 oracle {do:.3g}"
    case.close()


def test_inject_ptc_matches_oracle():
    """ptc_updater_logsph::inject_ptc (build semantics, ap_logsph_inject)
    against the oracle with the same Philox draws: slots, cells, positions,
    flags, ids and E bit for bit; p1, p2 and the weights, which go through
    CUDA's sinf / cosf instead of glibc's, within 1e-6; the same rows skip
    a dense surface."""
    import test_inject_oracle as tio
    m = mesh_logsph(64, 48)
    n, inj = 3000, 2
    red = m.dims[1] - 2 * m.guard[1]
    cap = n + 2 * inj * red
    p = tio._surface_ptc(m, n, np.random.default_rng(4), cap)
    params, _ = _params(m, 0, 1)
    params.q_e = 60.0
    params.max_ptc_number = cap
    env = SimEnvironment(params)
    data = SimData(env, capacity=cap)
    data.set_fields(oracle.new_fields(m, NSP))
    data.set_particles({k: v[:n] for k, v in p.items()})
    seed = 0x1234ABCD
    ptc_updater_logsph(env).inject_ptc(data, inj, 3.0, 0.0, 0.0, 0.5, 0.1, seed=seed)
    assert data.number == cap
    new_n = oracle.ls_inject(m, p, n, cap, inj, 3.0, 0.5, 60.0, seed, 0, 1 << 62)
    assert new_n == cap
    got = data.particles_host()
    for k in ("cell", "x1", "x2", "x3", "p3", "E", "flag", "id"):
        live = p["cell"] != oracle.MAX_CELL
        a, b = got[k], p[k]
        if k != "cell" and k != "id":
            a, b = a[live], b[live]
        assert_bits(a, b, k)
    live = p["cell"][n:] != oracle.MAX_CELL
    assert 0 < live.sum() < live.size
    for k in ("p1", "p2", "weight"):
        a = got[k][n:][live].astype(np.float64)
        b = p[k][n:][live].astype(np.float64)
        assert np.allclose(a, b, rtol=1e-6, atol=1e-7), k
    # the injected particles take part in the next update
    ptc_updater_logsph(env).update_particles(data, float(params.delta_t), 0)
    env.close()


@pytest.mark.parametrize("passes,data_interval", [(1, 1), (3, 1), (2, 2)])
def test_smoothing_bit_exact(passes, data_interval):
    """smooth_current of the log-spherical updater (filter_current_logsph,
    ptc_updater_logsph.cu:616-666, weighted by the face areas and the cell
    volume, then axis_rho, :414-438) on the same J and Rho equals the
    oracle's passes bit for bit: the filter has no transcendental, so the
    loose bound of the coupled run is not needed here."""
    case = LsCase((96, 64), 10, 12, smoothing=passes, data_interval=data_interval)
    rng = np.random.default_rng(13)
    for key, n in (("J", 3), ("Rho", NSP)):
        for k in range(n):
            case.f[key][k][:] = rng.standard_normal(case.f[key][k].shape).astype(np.float32)
    case.data.set_fields(case.f)
    case.pusher.smooth_current(case.data, 0)
    m = case.m
    tmp = np.zeros_like(case.f["J"][0])
    for _ in range(passes):
        for k in range(3):
            ls.filter_current(m, case.f["J"][k], tmp, case.c32[ls.A1E + k])
        if data_interval == 1:
            for k in range(NSP):
                ls.filter_current(m, case.f["Rho"][k], tmp, case.c32[ls.DV])
    ls.axis_rho(m, case.f["J"][2])
    g = case.data.fields_host()
    sl = (slice(m.guard[1], m.dims[1] - m.guard[1]), slice(m.guard[0], m.dims[0] - m.guard[0]))
    for k in range(3):
        assert_bits(g["J"][k][sl], case.f["J"][k][sl], f"J{k + 1}")
    for k in range(NSP):
        assert_bits(g["Rho"][k][sl], case.f["Rho"][k][sl], f"Rho{k}")
    case.close()
