"""Inverse-Compton tables and the 1D GR lab's radiative transfer on the GPU
against the CPU oracle (oracle/ap_ic.c, the GR model and mover of
oracle/ap_rad.c).

The tables are integrals of the reference's integrands in double; the GPU
evaluates exp / log / pow with CUDA's functions and sums each rate over a
CTA in a fixed tree order, the oracle with the C library's functions in the
reference's sequential order, so the stored floats agree to a few units in
the last place (relative 1e-5 below, 1e-6 on the cumulative distributions).
The Lorentz-factor grid and the steps are host arithmetic on both sides and
agree bit for bit. The emission and conversion tests then see the same
uniform draws on both sides; a decision can only differ where a draw falls
within the rates' last-bit difference of its threshold, and the sampled
photon energies inherit the tables' relative difference, amplified where a
cumulative distribution is flat (relative 1e-3 below).
"""
import numpy as np
import pytest

import oracle
from oracle import rad
from _cases import GR_A, GR_OMEGA, empty_ptc, gr_dt, gr_mesh, gr_particles, gr_table
from _gpu_helpers import assert_bits
from aperture3_b200 import (SimData, SimEnvironment, SimParams, inverse_compton,
                            ptc_updater_1dgr, radiative_transfer)

pytestmark = pytest.mark.gpu

NG, NE = 96, 80
FIRST_PH, FIRST_PTC = 1 << 40, 1 << 41


def _env(N=1024, n_cap=40000, ph_cap=60000, ic_path=1.0, dt=None, seed=7, di=4):
    m = gr_mesh(N)
    tab = gr_table()
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, 1.0, tab)
    params = SimParams(N=(N, 1, 1), guard=(3, 0, 0), lower=(-6.273, 0.0, 0.0),
                       size=(6.138, 1.0, 1.0), delta_t=dt or 0.01, q_e=1.2, num_species=2,
                       periodic_boundary=(False, False, False), data_interval=di,
                       coord_system="1DGR", a=GR_A, omega=GR_OMEGA, B0=1.0,
                       max_ptc_number=n_cap, create_pairs=True, max_photon_number=ph_cap,
                       rad_model="gr1d", rad_seed=seed, e_min=1e-3, ic_path=ic_path,
                       n_gamma=NG, n_ep=NE, track_percent=0.3)
    env = SimEnvironment(params, gr_table=tab)
    return m, co, params, env


def _oracle_tables(ic_path):
    return rad.IcTables(rad.gr1d_spectrum(1e-3), 1e-10, 0.1, 1.5e24 / ic_path, NG, NE)


@pytest.mark.parametrize("spectrum,emin,emax,n0", [
    (("broken_power_law", 1.25, 1.1, 1e-3, 1e-10, 0.1), 1e-10, 0.1, 1.5e24),
    (("black_body", 3e-6), 3e-16, 3e-3, 1.0e-6),
    (("power_law_soft", 2.0, 1e-6, 1e-2), 1e-6, 1e-2, 1.0e20),
])
def test_ic_tables_match_oracle(spectrum, emin, emax, n0):
    """inverse_compton::init on the GPU against the oracle's sequential sums."""
    m, co, params, env = _env()
    ic = inverse_compton(env)
    ic.init(spectrum, emin, emax, n0)
    got = ic.tables()
    kind = {"broken_power_law": rad.SPEC_BROKEN_POWER_LAW, "black_body": rad.SPEC_BLACK_BODY,
            "power_law_soft": rad.SPEC_POWER_LAW_SOFT}[spectrum[0]]
    ref = rad.IcTables(rad.spectrum(kind, *spectrum[1:]), emin, emax, n0, NG, NE)
    assert_bits(got["gammas"], ref.gammas, "gammas")
    for k in ("dep", "dg", "dlep"):
        assert np.float32(got[k]) == np.float32(getattr(ref, k)), k
    for k in ("ic_rate", "gg_rate"):
        a, b = got[k].astype(np.float64), getattr(ref, k).astype(np.float64)
        scale = np.maximum(np.abs(b), 1e-30)
        assert np.all((np.abs(a - b) / scale <= 1e-5) | (a == b)), (k, np.max(np.abs(a - b) / scale))
    for k in ("dNde", "dNde_thomson"):
        a, b = got[k], getattr(ref, k)
        assert np.array_equal(np.isnan(a), np.isnan(b)), k
        ok = ~np.isnan(b)
        assert np.abs(a[ok].astype(np.float64) - b[ok]).max() <= 1e-6, k
    env.close()


def _photons_gr(m, n, cap, rng, E_range=(10.0, 1e7)):
    ph = rad.new_photons(cap)
    g = m.guard[0]
    ph["cell"][:n] = rng.integers(g + 2, m.dims[0] - g - 2, n).astype(np.uint32)
    ph["x1"][:n] = rng.random(n, dtype=np.float32)
    E = np.exp(np.log(E_range[0]) + rng.random(n) * np.log(E_range[1] / E_range[0]))
    sgn = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    ph["p1"][:n] = (sgn * E * rng.random(n)).astype(np.float32)
    ph["p3"][:n] = (0.1 * E * rng.standard_normal(n)).astype(np.float32)
    ph["E"][:n] = E.astype(np.float32)
    ph["weight"][:n] = (0.5 + rng.random(n)).astype(np.float32)
    ph["id"][:n] = np.arange(n, dtype=np.uint64) + 5_000_000
    ph["flag"][:n] = (rng.random(n) < 0.3).astype(np.uint32) << np.uint32(1)
    return ph


class GrRadCase:
    def __init__(self, n=20000, n_ph=20000, ic_path=0.004, seed=3, p_sigma=3000.0):
        rng = np.random.default_rng(seed)
        self.cap, self.ph_cap = 4 * n + 4096, 3 * n_ph + 4096
        m = gr_mesh(1024)
        co = oracle.gr_coef(m, GR_A, GR_OMEGA, 1.0, gr_table())
        p = gr_particles(m, co, n, rng, p_sigma=p_sigma)
        dt = gr_dt(m, co, p)
        self.m, self.co, params, self.env = _env(n_cap=self.cap, ph_cap=self.ph_cap,
                                                 ic_path=ic_path, dt=dt)
        self.dt = np.float32(params.delta_t)
        self.n, self.n_ph = n, n_ph
        self.p = empty_ptc(self.cap)
        for k in p:
            self.p[k][:n] = p[k]
        self.p["id"][:n] = np.arange(n, dtype=np.uint64) + 1000
        self.p["cell"][n:] = oracle.MAX_CELL  # empty slots, as the store has them
        self.ph = _photons_gr(m, n_ph, self.ph_cap, rng)
        self.data = SimData(self.env, capacity=self.cap, photon_capacity=self.ph_cap)
        self.data.set_particles({k: v[:n] for k, v in self.p.items()})
        self.data.set_photons({k: v[:n_ph] for k, v in self.ph.items()})
        self.rt = radiative_transfer(self.env, first_photon_id=FIRST_PH,
                                     first_particle_id=FIRST_PTC)
        self.tables = _oracle_tables(ic_path)
        self.gr = rad.GrRad(self.co, GR_A, GR_OMEGA, self.tables)
        self.rp = rad.gr_rad_params(self.gr, float(self.dt), track_percent=0.3, seed=7)
        self.f = oracle.new_fields(m, 2)  # not read by the GR functions

    def close(self):
        self.env.close()


def _mismatch(a, b):
    return int(np.count_nonzero(a != b))


def test_gr_emission_matches_oracle():
    """emit_photons with the 1D GR lab's functions: the same emitters, the
    same parents' energy loss and the same photons (within the tables'
    difference), photons below 50 not kept but their energy taken."""
    case = GrRadCase()
    got = case.rt.emit_photons(case.data)
    po, pho = oracle.copy_ptc(case.p), rad.copy_photons(case.ph)
    n_ph, c = rad.emit_photons(case.m, case.rp, po, case.n, pho, case.n_ph, case.ph_cap, case.f,
                               None, 0, FIRST_PH)
    assert c.marked > 1000 and c.marked < case.n - 1000, c.marked
    assert abs(got["marked"] - c.marked) <= 2, (got, c.marked)
    g, gph = case.data.particles_host(), case.data.photons_host()
    if got["marked"] == c.marked:
        assert case.data.photon_number == n_ph
        live = pho["cell"][:n_ph] != oracle.MAX_CELL
        assert _mismatch(gph["cell"][:n_ph] != oracle.MAX_CELL, live) <= 2
        both = live & (gph["cell"][:n_ph] != oracle.MAX_CELL)
        assert both.sum() > 100
        for k in ("cell", "x1", "weight", "flag", "id"):
            assert_bits(gph[k][:n_ph][both], pho[k][:n_ph][both], f"photon {k}")
        for k in ("E", "p1", "p3"):
            a, b = gph[k][:n_ph][both].astype(np.float64), pho[k][:n_ph][both]
            err = np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * np.abs(pho["E"][:n_ph][both]))
            assert np.quantile(err, 0.999) <= 1e-3 and err.max() <= 1e-2, (k, err.max())
    # the parents: E and p1 changed only where an emission happened
    a, b = g["E"][:case.n].astype(np.float64), po["E"][:case.n]
    err = np.abs(a - b) / np.abs(b)
    assert np.quantile(err, 0.999) <= 1e-3, np.quantile(err, 0.999)
    for k in ("cell", "x1", "weight", "flag", "id"):
        assert_bits(g[k][:case.n], po[k][:case.n], f"particle {k}")
    case.close()


def test_gr_pair_production_matches_oracle():
    """produce_pairs with the 1D GR lab's functions: conversion by the
    gamma-gamma rate, pairs of half the photon's energy along its p1."""
    case = GrRadCase(ic_path=0.002)
    got = case.rt.produce_pairs(case.data)
    po, pho = oracle.copy_ptc(case.p), rad.copy_photons(case.ph)
    n_p, c = rad.produce_pairs(case.m, case.rp, pho, case.n_ph, po, case.n, case.cap, case.f,
                               None, 0, FIRST_PTC)
    assert c.marked > 500 and c.marked < case.n_ph - 500, c.marked
    assert abs(got["marked"] - c.marked) <= 2, (got, c.marked)
    g, gph = case.data.particles_host(), case.data.photons_host()
    assert _mismatch(gph["cell"][:case.n_ph], pho["cell"][:case.n_ph]) <= 2
    if got["marked"] == c.marked:
        assert case.data.number == n_p
        sl = slice(case.n, n_p)
        for k in ("cell", "x1", "weight", "flag", "id", "E"):
            assert_bits(g[k][sl], po[k][sl], f"pair {k}")
        a, b = g["p1"][sl].astype(np.float64), po["p1"][sl]
        err = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
        assert err.max() <= 1e-5, err.max()
    case.close()


def test_gr_photon_mover_matches_oracle():
    """update_photon_1dgr in ptc_updater_1dgr::update_particles: the photons
    move (and leave the bulk) as the oracle moves them; tracked photons
    record the lower u_0 on output steps."""
    case = GrRadCase(n=2000, n_ph=20000)
    pusher = ptc_updater_1dgr(case.env)
    pho = rad.copy_photons(case.ph)
    for step in range(3):
        pusher.update_particles(case.data, float(case.dt), step)
        rad.move_photons_gr(case.m, case.gr, pho, case.n_ph, case.dt, step, 4)
    gph = case.data.photons_host()
    n = case.n_ph
    assert_bits(gph["cell"][:n], pho["cell"][:n], "photon cell")
    live = pho["cell"][:n] != oracle.MAX_CELL
    assert live.sum() > 1000
    for k in ("x1", "p1", "E", "p2"):
        a, b = gph[k][:n][live].astype(np.float64), pho[k][:n][live]
        scale = np.maximum(np.abs(b), 1e-3 * np.abs(pho["E"][:n][live]))
        err = np.abs(a - b) / np.maximum(scale, 1e-6)
        assert err.max() <= 1e-4, (k, err.max())
    case.close()
