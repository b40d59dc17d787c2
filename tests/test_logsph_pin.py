"""Pins the log-spherical CPU oracle (oracle/ap_logsph.c, FP32 build) to the
reference's own log-spherical code run on the host (oracle/ref_build,
libapref_ls.so): Grid_LogSph::compute_coef, user_push_2d_logsph,
deposit_and_move_2d_log_sph, process_j, axis_rho_*, ptc_outflow,
filter_current_logsph, compute_{b,e}_update_logsph, compute_divs_logsph and
the four field boundaries. Every comparison is bit-exact; both sides call
the same C library float functions. The FP64 build is checked for
agreement with the FP32 one at FP32 resolution. Cases that need the
reference tree skip where it is absent; the committed fixtures in
tests/golden/logsph_*.npz cover those machines.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from oracle import logsph as ls
from _cases import (LS_CHARGES, LS_MASSES, logsph_dt, logsph_fields, logsph_particles,
                    mesh_logsph)
from test_oracle_pin import _same

REF = ls.load_ref(build=True)
needs_ref = pytest.mark.skipif(REF is None, reason="reference pin library not built")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

# bulk sizes are multiples of the reference's 32 x 16 launch blocks
MESHES = [(64, 32), (96, 64)]


def _case(N, seed, n=4000, gamma_max=1e3, **kw):
    rng = np.random.default_rng(seed)
    m = mesh_logsph(*N)
    f = logsph_fields(m, rng)
    p = logsph_particles(m, n, rng, gamma_max=gamma_max)
    lp = ls.ls_params(**kw)
    return m, f, p, lp


@needs_ref
@pytest.mark.parametrize("N", MESHES + [(50, 30)])
def test_coefficients_match_reference(N):
    m = mesh_logsph(*N)
    a, b = ls.coef(m), ls.ref_coef(m)
    for k, name in enumerate(ls.COEF_NAMES):
        _same(a[k], b[k], name)


def test_coefficients_f64_agree():
    m = mesh_logsph(64, 32)
    a, b = ls.coef(m), ls.coef(m, f64=True)
    for k, name in enumerate(ls.COEF_NAMES):
        err = np.abs(a[k] - b[k]) / np.maximum(np.abs(b[k]), 1e-30)
        assert err.max() < 1e-5, (name, err.max())
    # no zero cell volume or face area anywhere (the updater divides by them)
    for k in (ls.A1E, ls.A2E, ls.DV):
        assert np.all(a[k] != 0)


@needs_ref
@pytest.mark.parametrize("N,seed", [(MESHES[0], 0), (MESHES[1], 1)])
@pytest.mark.parametrize("opts", [{}, {"gravity": 0.3, "rad_cooling_on": True,
                                       "rad_cooling_coef": 0.05, "compactness": 0.4}])
def test_push_matches_reference(N, seed, opts):
    m, f, p, lp = _case(N, seed, **opts)
    dt = logsph_dt(m)
    F = f["E"] + f["B"]
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    ls.push(m, lp, po, len(p["x1"]), dt, F, LS_CHARGES, LS_MASSES)
    ls.ref_push(m, lp, pr, len(p["x1"]), dt, F, LS_CHARGES, LS_MASSES)
    for k in po:
        _same(po[k], pr[k], k)
    assert not np.array_equal(po["p1"], p["p1"])


@needs_ref
@pytest.mark.parametrize("N,seed", [(MESHES[0], 2), (MESHES[1], 3)])
@pytest.mark.parametrize("step", [0, 4])
@pytest.mark.parametrize("compactness", [0.0, 0.5])
def test_deposit_matches_reference(N, seed, step, compactness):
    m, f, p, lp = _case(N, seed, compactness=compactness, gamma_max=1e6)
    dt = logsph_dt(m)
    c = ls.coef(m)
    F = f["E"] + f["B"]
    ls.push(m, lp, p, len(p["x1"]), dt, F, LS_CHARGES, LS_MASSES)
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    shape = f["E"][0].shape
    Jo = [np.zeros(shape, np.float32) for _ in range(3)]
    Jr = [np.zeros(shape, np.float32) for _ in range(3)]
    Ro = [np.zeros(shape, np.float32) for _ in range(3)]
    Rr = [np.zeros(shape, np.float32) for _ in range(3)]
    far = ls.deposit(m, lp, po, len(p["x1"]), dt, step, 5, Jo, Ro, c[ls.DV], LS_CHARGES)
    ls.ref_deposit(m, lp, pr, len(p["x1"]), dt, step, 5, Jr, Rr, c, LS_CHARGES)
    assert far == 0
    for k in po:
        _same(po[k], pr[k], k)
    for k in range(3):
        _same(Jo[k], Jr[k], f"J{k + 1}")
        _same(Ro[k], Rr[k], f"Rho{k}")
    assert np.abs(Jo[0]).max() > 0
    if step == 4:
        assert np.abs(Ro[0]).max() > 0
    # the axis reflection path ran
    th = (np.asarray(pr["cell"]) // m.dims[0]).astype(int)
    assert np.any(th == m.guard[1]) and np.any(th == m.dims[1] - m.guard[1] - 1)


@needs_ref
def test_process_j_axis_outflow_filter_match_reference():
    m, f, p, lp = _case(MESHES[0], 5, damping_length=20)
    rng = np.random.default_rng(5)
    c = ls.coef(m)
    shape = f["E"][0].shape
    J = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    R = [rng.standard_normal(shape).astype(np.float32) for _ in range(3)]
    Jo, Ro = [a.copy() for a in J], [a.copy() for a in R]
    Jr, Rr = [a.copy() for a in J], [a.copy() for a in R]
    dt = logsph_dt(m)
    ls.process_j(m, Jo, Ro, c, dt)
    ls.ref_process_j(m, Jr, Rr, c, dt)
    for k in range(3):
        _same(Jo[k], Jr[k], f"J{k + 1}")
        _same(Ro[k], Rr[k], f"Rho{k}")
    ls.axis_rho(m, Jo[2])
    ls.ref_axis_rho(m, Jr[2], c)
    _same(Jo[2], Jr[2], "J3 axis")
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    ls.ptc_outflow(m, lp, po, len(p["x1"]))
    ls.ref_ptc_outflow(m, lp, pr, len(p["x1"]))
    _same(po["flag"], pr["flag"], "flag")
    assert not np.array_equal(po["flag"], p["flag"])
    for k, A in ((0, c[ls.A1E]), (1, c[ls.A2E]), (2, c[ls.A3E])):
        jo, to = J[k].copy(), np.zeros(shape, np.float32)
        jr, tr = J[k].copy(), np.zeros(shape, np.float32)
        ls.filter_current(m, jo, to, A)
        ls.ref_filter(m, jr, tr, A)
        g0, g1 = m.guard[0], m.guard[1]
        _same(to[g1:-g1, g0:-g0], tr[g1:-g1, g0:-g0], f"filter J{k + 1}")


@needs_ref
@pytest.mark.parametrize("N,seed", [(MESHES[0], 6), (MESHES[1], 7)])
@pytest.mark.parametrize("compactness", [0.0, 0.5])
def test_field_update_matches_reference(N, seed, compactness):
    m, f, p, lp = _case(N, seed, compactness=compactness)
    rng = np.random.default_rng(seed)
    for k in range(3):
        f["J"][k][:] = (0.01 * rng.standard_normal(f["J"][k].shape)).astype(np.float32)
    c = ls.coef(m)
    dt = logsph_dt(m)
    fo, fr = oracle.copy_fields(f), oracle.copy_fields(f)
    ls.update_fields(m, lp, fo, c, dt)
    ls.ref_update_fields(m, lp, fr, c, dt)
    for key in ("E", "B"):
        for k in range(3):
            _same(fo[key][k], fr[key][k], f"{key}{k + 1}")
    _same(fo["divE"], fr["divE"], "divE")
    _same(fo["divB"], fr["divB"], "divB")
    assert not np.array_equal(fo["E"][0], f["E"][0])
    ls.field_boundary(m, lp, fo, np.float32(0.07))
    ls.ref_field_boundary(m, lp, fr, np.float32(0.07))
    for key in ("E", "B"):
        for k in range(3):
            _same(fo[key][k], fr[key][k], f"boundary {key}{k + 1}")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "logsph_*.npz"))))
def test_golden_logsph(path):
    """Committed outputs of the reference's log-spherical code (made by
    tests/golden/make_golden.py) against the FP32 oracle."""
    z = np.load(path)
    m = oracle.mesh_from_dict({k: list(z["mesh_" + k]) for k in
                               ("dims", "guard", "delta", "inv_delta", "lower", "sizes")} |
                              {"dimension": int(z["mesh_dimension"])})
    lp = ls.ls_params(*[float(v) for v in z["lp"][:6]], rad_cooling_on=bool(z["lp"][6]),
                      damping_length=int(z["lp"][7]))
    c = ls.coef(m)
    for k, name in enumerate(ls.COEF_NAMES):
        _same(c[k], z["coef_" + name], name)
    p = {k[5:]: z[k].copy() for k in z.files if k.startswith("in_p_")}
    f = {}
    for key in ("E", "B", "Ebg", "Bbg"):
        f[key] = [z[f"in_{key}{k}"].copy() for k in range(3)]
    shape = f["E"][0].shape
    f["J"] = [np.zeros(shape, np.float32) for _ in range(3)]
    f["Rho"] = [np.zeros(shape, np.float32) for _ in range(3)]
    f["divE"] = np.zeros(shape, np.float32)
    f["divB"] = np.zeros(shape, np.float32)
    dt = np.float32(z["dt"])
    n = len(p["x1"])
    ls.push(m, lp, p, n, dt, f["E"] + f["B"], LS_CHARGES, LS_MASSES)
    ls.deposit(m, lp, p, n, dt, 0, 1, f["J"], f["Rho"], c[ls.DV], LS_CHARGES)
    for k in p:
        _same(p[k], z["out_p_" + k], k)
    for k in range(3):
        _same(f["J"][k], z[f"out_J{k}"], f"J{k + 1}")
        _same(f["Rho"][k], z[f"out_Rho{k}"], f"Rho{k}")
    ls.update_fields(m, lp, f, c, dt)
    for key in ("E", "B"):
        for k in range(3):
            _same(f[key][k], z[f"out_{key}{k}"], f"{key}{k + 1}")
