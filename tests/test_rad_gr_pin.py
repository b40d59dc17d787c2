"""The oracle's 1D GR radiative transfer (oracle/ap_rad.c, model GR1D) pinned
bit for bit to the 1D GR lab's own user radiative functions
(labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh), compiled for
the host by oracle/ref_build (libapref_rad_gr.so) together with the
reference's own inverse-Compton lookups (find_ic_rate, find_gg_rate,
gen_photon_e of rt_ic.cu) on the oracle's tables (pinned to the reference's
init by tests/test_ic_oracle.py): this pins the oracle's lookups, metric
interpolation, energy loss, photon and pair momenta, flags and draw order. The oracle's GR photon mover is pinned
to the reference's update_photon_1dgr (ptc_updater_1dgr.cu:301-400), which
the 1D GR pin library (libapref_gr.so) compiles for the host."""
import numpy as np
import pytest

import oracle
from oracle import rad
from _cases import GR_A, GR_OMEGA, empty_ptc, gap_rad_case, gr_dt, gr_mesh, gr_particles, gr_table

pytestmark = pytest.mark.skipif(rad.load_ref_gr() is None,
                                reason="reference tree not present and no prebuilt pin library")

NG, NE = 64, 56


def _case(n=6000, n_ph=6000, ic_path=0.004, seed=11):
    rng = np.random.default_rng(seed)
    m = gr_mesh(512)
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, 1.0, gr_table())
    p0 = gr_particles(m, co, n, rng, p_sigma=3000.0)
    dt = gr_dt(m, co, p0)
    cap, ph_cap = 4 * n + 1024, 3 * n_ph + 1024
    p = empty_ptc(cap)
    for k in p0:
        p[k][:n] = p0[k]
    p["id"][:n] = np.arange(n, dtype=np.uint64) + 77
    p["cell"][n:] = oracle.MAX_CELL
    ph = rad.new_photons(ph_cap)
    g = m.guard[0]
    ph["cell"][:n_ph] = rng.integers(g + 2, m.dims[0] - g - 2, n_ph).astype(np.uint32)
    ph["cell"][:n_ph][rng.random(n_ph) < 0.1] = oracle.MAX_CELL
    ph["x1"][:n_ph] = rng.random(n_ph, dtype=np.float32)
    E = np.exp(np.log(10.0) + rng.random(n_ph) * np.log(1e6))
    ph["p1"][:n_ph] = (np.where(rng.random(n_ph) < 0.5, -1, 1) * E * rng.random(n_ph)).astype(
        np.float32)
    ph["p3"][:n_ph] = (0.1 * E * rng.standard_normal(n_ph)).astype(np.float32)
    ph["E"][:n_ph] = E.astype(np.float32)
    ph["weight"][:n_ph] = (0.5 + rng.random(n_ph)).astype(np.float32)
    ph["id"][:n_ph] = np.arange(n_ph, dtype=np.uint64) + 900_000
    tables = rad.IcTables(rad.gr1d_spectrum(1e-3), 1e-10, 0.1, 1.5e24 / ic_path, NG, NE)
    gr = rad.GrRad(co, GR_A, GR_OMEGA, tables)
    rp = rad.gr_rad_params(gr, float(dt), track_percent=0.3, seed=5)
    return m, rp, gr, p, ph, n, n_ph, cap, ph_cap


def _same(a, b, what):
    for k in a:
        x, y = a[k], b[k]
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (what, k)


@pytest.mark.parametrize("call", [0, 3])
def test_gr_emission_bit_exact(call):
    m, rp, gr, p, ph, n, n_ph, cap, ph_cap = _case()
    po, pho = oracle.copy_ptc(p), rad.copy_photons(ph)
    pr, phr = oracle.copy_ptc(p), rad.copy_photons(ph)
    f = oracle.new_fields(m, 2)
    n1, c1 = rad.emit_photons(m, rp, po, n, pho, n_ph, ph_cap, f, None, call, 1 << 40)
    n2, c2 = rad.ref_gr_emit_photons(m, rp, pr, n, phr, n_ph, ph_cap, call, 1 << 40)
    assert (n1, c1.marked, c1.written) == (n2, c2.marked, c2.written)
    assert c1.marked > 200
    _same(po, pr, "particles")
    _same(pho, phr, "photons")


@pytest.mark.parametrize("call", [0, 2])
def test_gr_conversion_bit_exact(call):
    m, rp, gr, p, ph, n, n_ph, cap, ph_cap = _case(ic_path=0.002)
    po, pho = oracle.copy_ptc(p), rad.copy_photons(ph)
    pr, phr = oracle.copy_ptc(p), rad.copy_photons(ph)
    f = oracle.new_fields(m, 2)
    n1, c1 = rad.produce_pairs(m, rp, pho, n_ph, po, n, cap, f, None, call, 1 << 41)
    n2, c2 = rad.ref_gr_produce_pairs(m, rp, phr, n_ph, pr, n, cap, call, 1 << 41)
    assert (n1, c1.marked, c1.written) == (n2, c2.marked, c2.written)
    assert c1.marked > 100
    _same(po, pr, "particles")
    _same(pho, phr, "photons")


def test_gr_capacity_rules_bit_exact():
    """Emissions past the photon capacity and pairs past the particle
    capacity, with the build's rules on both sides."""
    m, rp, gr, p, ph, n, n_ph, cap, ph_cap = _case()
    f = oracle.new_fields(m, 2)
    small = n_ph + 50
    po, pho = oracle.copy_ptc(p), rad.copy_photons(ph)
    pr, phr = oracle.copy_ptc(p), rad.copy_photons(ph)
    n1, c1 = rad.emit_photons(m, rp, po, n, pho, n_ph, small, f, None, 1, 7)
    n2, c2 = rad.ref_gr_emit_photons(m, rp, pr, n, phr, n_ph, small, 1, 7)
    assert (n1, c1.marked, c1.written, c1.dropped) == (n2, c2.marked, c2.written, c2.dropped)
    assert c1.dropped > 0
    _same(po, pr, "particles")
    _same(pho, phr, "photons")


@pytest.mark.skipif(oracle.load_ref_gr() is None, reason="no 1D GR pin library")
def test_gr_photon_mover_bit_exact():
    """Three moves with tracked photons on an output step and photons
    starting outside the bulk."""
    import ctypes as C
    m, rp, gr, p, ph, n, n_ph, cap, ph_cap = _case()
    ph["cell"][:20] = np.uint32(1)  # in the guard: removed first
    ph["flag"][:n_ph] = (np.arange(n_ph) % 3 == 0).astype(np.uint32) << np.uint32(1)
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, 1.0, gr_table())
    cos = [np.ascontiguousarray(c, np.float32) for c in co]
    ptrs = (C.c_void_p * 15)(*[c.ctypes.data for c in cos])
    a, b = rad.copy_photons(ph), rad.copy_photons(ph)
    for step in range(3):
        rad.move_photons_gr(m, gr, a, n_ph, rp.delta_t, step, 2)
        oracle.load_ref_gr().ref_gr_move_photons(C.byref(m), C.byref(rad.photons_struct(b)), n_ph,
                                                 rp.delta_t, step, 2, ptrs)
    _same(a, b, "photons")
    assert (a["cell"][:n_ph] == oracle.MAX_CELL).sum() >= 20


# ---- the 1D gap lab (labs/1dgap/src/cuda/radiation/user_radiative_functions.cuh)

gap_pin = pytest.mark.skipif(rad.load_ref_gap_rad() is None, reason="no 1D gap radiation pin")


@gap_pin
@pytest.mark.parametrize("call", [0, 4])
def test_gap_emission_bit_exact(call):
    m, rp, gap, p, ph, n, n_ph, cap, ph_cap = gap_rad_case(NG, NE)
    po, pho = oracle.copy_ptc(p), rad.copy_photons(ph)
    pr, phr = oracle.copy_ptc(p), rad.copy_photons(ph)
    f = oracle.new_fields(m, 2)
    n1, c1 = rad.emit_photons(m, rp, po, n, pho, n_ph, ph_cap, f, None, call, 1 << 40)
    n2, c2 = rad.ref_gr_emit_photons(m, rp, pr, n, phr, n_ph, ph_cap, call, 1 << 40)
    assert (n1, c1.marked, c1.written) == (n2, c2.marked, c2.written)
    assert c1.marked > 200
    _same(po, pr, "particles")
    _same(pho, phr, "photons")


@gap_pin
def test_gap_conversion_bit_exact():
    m, rp, gap, p, ph, n, n_ph, cap, ph_cap = gap_rad_case(NG, NE, ic_path=0.0005)
    po, pho = oracle.copy_ptc(p), rad.copy_photons(ph)
    pr, phr = oracle.copy_ptc(p), rad.copy_photons(ph)
    f = oracle.new_fields(m, 2)
    n1, c1 = rad.produce_pairs(m, rp, pho, n_ph, po, n, cap, f, None, 1, 1 << 41)
    n2, c2 = rad.ref_gr_produce_pairs(m, rp, phr, n_ph, pr, n, cap, 1, 1 << 41)
    assert (n1, c1.marked, c1.written) == (n2, c2.marked, c2.written)
    assert c1.marked > 100
    _same(po, pr, "particles")
    _same(pho, phr, "photons")


@pytest.mark.skipif(oracle.load_ref_gap() is None, reason="no 1D gap pin library")
def test_gap_photon_mover_bit_exact():
    import ctypes as C
    m, rp, gap, p, ph, n, n_ph, cap, ph_cap = gap_rad_case(NG, NE)
    ph["cell"][:10] = np.uint32(0)  # in the guard: removed first
    a, b = rad.copy_photons(ph), rad.copy_photons(ph)
    for step in range(4):
        rad.move_photons_gap(m, a, n_ph, 2e-3)
        oracle.load_ref_gap().ref_gap_move_photons(C.byref(m), C.byref(rad.photons_struct(b)),
                                                   n_ph, 2e-3, step)
    _same(a, b, "photons")
