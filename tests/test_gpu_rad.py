"""Photons and pair production on the GPU against the CPU oracle (pinned to
the reference's own user radiative functions and photon movers by
tests/test_rad_pin.py).

Bit for bit where the arithmetic has no transcendental: the Cartesian
photon movers, the default model's emission (photon energy, parent update)
and every pair production (the pulsar model's conversion test uses only
+, -, *, /, sqrt). The default model's free path goes through sinf, the
pulsar model's emission through expf, sinf, cosf and a double pow, and the
log-spherical mover through the reference's float transcendentals: those
values are compared within 1e-5 relative (CUDA's functions against the C
library's), their decisions exactly.
"""
import numpy as np
import pytest

import oracle
from oracle import rad
from _cases import (logsph_fields, logsph_particles, mesh_1d, mesh_2d, mesh_logsph, rad_photons,
                    rad_rho, random_fields, random_particles)
from _gpu_helpers import assert_bits
from aperture3_b200 import (SimData, SimEnvironment, SimParams, ptc_updater, ptc_updater_logsph,
                            radiative_transfer)

pytestmark = pytest.mark.gpu

REL = 1e-5
FIRST_PH, FIRST_PTC = 1 << 40, 1 << 41


def _rel(a, b):
    a, b = a.astype(np.float64), b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


def _close(a, b, what, rel=REL):
    err = _rel(a, b)
    assert err.size == 0 or err.max() <= rel, (what, float(err.max()))


class RadCase:
    def __init__(self, kind, seed, n=20000, ph_n=6000, ph_cap=40000, ptc_extra=60000):
        rng = np.random.default_rng(seed)
        self.kind = kind
        if kind == "logsph":
            m = mesh_logsph(96, 96, rmax=8.0)
            f = logsph_fields(m, rng, omega=0.1, noise=0.0, num_species=2)
            p = logsph_particles(m, n, rng, gamma_max=3e4)
            coord, periodic = "LogSpherical", (False, False, False)
            rp = rad.rad_params(rad.RAD_PULSAR, delta_t=0.01, e_curv=2e-8, l_curv=2.0, BQ=0.05,
                                omega=0.1, r_cutoff=6.0, track_percent=0.3, seed=77)
        else:
            m = mesh_1d(256) if kind == "cart1d" else mesh_2d(64, 48, size=(1.0, 3.0))
            f = random_fields(m, rng)
            p = random_particles(m, n, rng, gamma_max=200.0, species=(0, 1, 2))
            coord, periodic = "Cartesian", (True, kind == "cart2d", False)
            rp = rad.rad_params(rad.RAD_DEFAULT, gamma_thr=20.0, E_secondary=4.0,
                                photon_path=0.5, r_cutoff=3.0, track_percent=0.25, seed=5)
        rad_rho(f, rng)
        self.m, self.f, self.p, self.rp, self.n = m, f, p, rp, n
        self.ph = rad_photons(m, ph_n, ph_cap, rng)
        self.ph_n, self.ph_cap = ph_n, ph_cap
        self.cap = n + ptc_extra
        N = (m.dims[0] - 2 * m.guard[0], max(1, m.dims[1] - 2 * m.guard[1]), 1)
        model = "pulsar" if kind == "logsph" else "default"
        params = SimParams(N=N, guard=(m.guard[0], m.guard[1], 0), lower=tuple(m.lower),
                           size=tuple(m.sizes), delta_t=rp.delta_t, q_e=1.0, ion_mass=10.0,
                           num_species=2, periodic_boundary=periodic, data_interval=1,
                           coord_system=coord, omega=rp.omega, compactness=0.0,
                           max_ptc_number=self.cap, create_pairs=True, max_photon_number=ph_cap,
                           gamma_thr=rp.gamma_thr, track_percent=rp.track_percent, BQ=rp.BQ,
                           photon_path=rp.photon_path, E_secondary=rp.E_secondary,
                           r_cutoff=rp.r_cutoff, l_curv=rp.l_curv, e_curv=rp.e_curv,
                           rad_model=model, rad_seed=rp.seed)
        self.env = SimEnvironment(params)
        self.data = SimData(self.env)
        self.data.set_fields(f)
        self.data.set_particles(p)
        self.data.set_photons({k: v[:ph_n] for k, v in self.ph.items()})
        self.rt = radiative_transfer(self.env, first_photon_id=FIRST_PH,
                                     first_particle_id=FIRST_PTC)
        # the oracle's particle store at the GPU's capacity
        self.po = {k: np.concatenate([v, np.zeros(self.cap - n, v.dtype)])
                   for k, v in p.items()}
        self.po["cell"][n:] = oracle.MAX_CELL
        self.pho = rad.copy_photons(self.ph)
        self.number, self.ph_number = n, ph_n
        self.emit_calls = self.pair_calls = 0
        self.next_ph, self.next_ptc = FIRST_PH, FIRST_PTC

    def emit(self):
        got = self.rt.emit_photons(self.data)
        cnt_o = np.zeros_like(self.f["Rho"][0])
        n_ph, c = rad.emit_photons(self.m, self.rp, self.po, self.number, self.pho, self.ph_number,
                                   self.ph_cap, self.f, cnt_o, self.emit_calls, self.next_ph)
        assert (got["marked"], got["written"], got["dropped"]) == (c.marked, c.written, c.dropped)
        assert self.data.photon_number == n_ph
        self.emit_calls += 1
        self.next_ph += c.marked
        self.ph_number = n_ph
        return c, cnt_o

    def pairs(self):
        got = self.rt.produce_pairs(self.data)
        cnt_o = np.zeros_like(self.f["Rho"][0])
        n_p, c = rad.produce_pairs(self.m, self.rp, self.pho, self.ph_number, self.po, self.number,
                                   self.cap, self.f, cnt_o, self.pair_calls, self.next_ptc)
        assert (got["marked"], got["written"], got["dropped"]) == (c.marked, c.written, c.dropped)
        assert self.data.number == n_p
        self.pair_calls += 1
        self.next_ptc += 2 * c.marked
        self.number = n_p
        return c, cnt_o

    def gpu_particles(self):
        return self.data.particles_host()

    def close(self):
        self.env.close()


def _field(data_arr, m):
    """A device field tensor (padded rows) as the oracle's (dims[1], dims[0])."""
    a = data_arr.cpu().numpy()
    return a[:, :m.dims[0]].reshape(m.dims[1] * m.dims[2], m.dims[0])


def _check_photons(g, o, n, exact_keys, tol_keys, what):
    assert_bits(g["cell"][:n], o["cell"][:n], f"{what}: photon cell")
    live = o["cell"][:n] != oracle.MAX_CELL
    for k in exact_keys:
        assert_bits(g[k][:n][live], o[k][:n][live], f"{what}: photon {k}")
    for k in tol_keys:
        _close(g[k][:n][live], o[k][:n][live], f"{what}: photon {k}")


@pytest.mark.parametrize("kind", ["cart1d", "cart2d"])
def test_default_model(kind):
    """emit_photons bit for bit but the free path (sinf); produce_pairs bit
    for bit; the per-cell counters within 1e-5 (float atomics in any order)."""
    case = RadCase(kind, 3 if kind == "cart1d" else 4)
    c, cnt_o = case.emit()
    assert c.marked > 1000
    g = case.gpu_particles()
    for k in ("p1", "p2", "p3", "E", "cell", "flag", "id"):
        assert_bits(g[k][:case.n], case.po[k][:case.n], f"emit: particle {k}")
    gph = case.data.photons_host()
    _check_photons(gph, case.pho, case.ph_number,
                   ("x1", "x2", "x3", "p1", "p2", "p3", "E", "weight", "id", "flag"), (), "emit")
    # path = min(10, (1 / sinf(theta) - 1) photon_path) (0.5 + 0.5 u): the
    # subtraction cancels near theta = pi / 2, so sinf's last bit is measured
    # against the terms before it, photon_path / |sin theta|
    live = case.pho["cell"][:case.ph_number] != oracle.MAX_CELL
    c2 = (case.pho["cell"][:case.ph_number][live] // case.m.dims[0]).astype(np.int64)
    if case.m.dimension > 1:
        theta = case.m.lower[1] + case.m.delta[1] * (c2 - case.m.guard[1] +
                                                     case.pho["x2"][:case.ph_number][live])
    else:
        theta = case.pho["x2"][:case.ph_number][live].astype(np.float64) * case.m.delta[1]
    scale = case.rp.photon_path / np.abs(np.sin(theta))
    dpath = np.abs(gph["path_left"][live].astype(np.float64) -
                   case.pho["path_left"][:case.ph_number][live])
    assert (dpath <= REL * scale).all(), float((dpath / scale).max())
    _close(_field(case.data.photon_produced, case.m), cnt_o, "photon_produced")
    c2, cnt2 = case.pairs()
    assert c2.written > 500
    g = case.gpu_particles()
    lo, hi = case.n, case.number
    assert_bits(g["cell"][lo:hi], case.po["cell"][lo:hi], "pairs: cell")
    live = case.po["cell"][lo:hi] != oracle.MAX_CELL
    for k in ("x1", "x2", "x3", "p1", "p2", "p3", "E", "weight", "flag", "id"):
        assert_bits(g[k][lo:hi][live], case.po[k][lo:hi][live], f"pairs: {k}")
    gph = case.data.photons_host()
    assert_bits(gph["cell"], case.pho["cell"][:case.ph_number], "photons after conversion")
    _close(_field(case.data.pair_produced, case.m), cnt2, "pair_produced")
    case.close()


def test_pulsar_model():
    """The pulsar lab's emission within 1e-5 (expf, sinf, cosf, pow) with
    the same emitters; its conversion bit for bit on the same photons."""
    case = RadCase("logsph", 11)
    c, _ = case.emit()
    assert c.marked > 500
    g = case.gpu_particles()
    changed_g = g["E"][:case.n] != case.p["E"]
    changed_o = case.po["E"][:case.n] != case.p["E"]
    assert np.array_equal(changed_g, changed_o)
    # The parent keeps pf = sqrt((gamma - Eph)^2 - 1) along its direction.
    # Eph carries the last bits of expf / sinf / cosf / pow (relative
    # DELTA); where Eph is close to gamma - 1, pf^2 cancels and moves by up
    # to 2 (gamma - Eph) Eph DELTA + (Eph DELTA)^2, so pf moves by at most
    # the square root of that.
    DELTA = 1e-6
    ch = changed_o
    gam = case.p["E"][ch].astype(np.float64)
    d = case.po["E"][:case.n][ch].astype(np.float64)  # gamma - Eph
    eph = gam - d
    pf_tol = np.sqrt(2 * d * eph * DELTA + (eph * DELTA) ** 2)
    pi = np.sqrt(sum(case.p[k][ch].astype(np.float64) ** 2 for k in ("p1", "p2", "p3")))
    for k in ("p1", "p2", "p3"):
        diff = np.abs(g[k][:case.n][ch].astype(np.float64) - case.po[k][:case.n][ch])
        tol = np.abs(case.p[k][ch]) / pi * pf_tol * 1.01 + 1e-6 * np.abs(case.po[k][:case.n][ch])
        assert (diff <= tol).all(), (k, float((diff / tol).max()))
    diffE = np.abs(g["E"][:case.n][ch].astype(np.float64) - d)
    assert (diffE <= eph * DELTA + 1e-6 * d).all(), "emit: particle E"
    for k in ("p1", "p2", "p3", "E"):
        assert_bits(g[k][:case.n][~ch], case.po[k][:case.n][~ch], f"emit: unchanged {k}")
    gph = case.data.photons_host()
    _check_photons(gph, case.pho, case.ph_number, ("x1", "x2", "x3", "weight", "id", "flag",
                                                   "path_left"), ("p1", "p2", "p3", "E"), "emit")
    # the same photons on both sides, then the conversion
    case.data.set_photons({k: v[:case.ph_number] for k, v in case.pho.items()})
    c2, _ = case.pairs()
    assert c2.written > 500
    g = case.gpu_particles()
    lo, hi = case.n, case.number
    assert_bits(g["cell"][lo:hi], case.po["cell"][lo:hi], "pairs: cell")
    live = case.po["cell"][lo:hi] != oracle.MAX_CELL
    for k in ("x1", "x2", "x3", "p1", "p2", "p3", "E", "weight", "flag", "id"):
        assert_bits(g[k][lo:hi][live], case.po[k][lo:hi][live], f"pairs: {k}")
    gph = case.data.photons_host()
    assert_bits(gph["cell"], case.pho["cell"][:case.ph_number], "photons after conversion")
    case.close()


@pytest.mark.parametrize("kind", ["cart1d", "cart2d", "logsph"])
def test_photon_move_in_update(kind):
    """update_particles moves the bound photons after the particles, then
    wraps (periodic) or removes (other sides) those that left the bulk."""
    case = RadCase(kind, 20 + len(kind), n=2000, ph_n=20000, ph_cap=20000)
    dt = np.float32(0.7 * min(case.m.delta[0], case.m.delta[1] if case.m.dimension > 1 else 1.0))
    if kind == "logsph":
        ptc_updater_logsph(case.env).update_particles(case.data, float(dt), 0)
        rad.move_photons_logsph(case.m, case.rp, case.pho, case.ph_number, dt)
    else:
        ptc_updater(case.env).update_particles(case.data, float(dt), 0)
        rad.move_photons_cart(case.m, case.pho, case.ph_number, dt,
                              case.env.params.periodic_boundary)
    gph = case.data.photons_host()
    if kind == "logsph":
        o = {k: v[:case.ph_number] for k, v in case.pho.items()}
        same = gph["cell"] == o["cell"]
        assert same.mean() > 0.999
        live = same & (gph["cell"] != oracle.MAX_CELL)
        # acosf and atan2f are ill-conditioned at the axis: photons with
        # sin(theta) < 0.1 are held to 1e-2, the rest to 1e-4 (positions in
        # cells, momenta relative to the photon energy)
        c2 = (o["cell"][live] // case.m.dims[0]).astype(np.int64)
        theta = case.m.delta[1] * (c2 - case.m.guard[1] + o["x2"][live])
        tol = np.where(np.abs(np.sin(theta)) < 0.1, 1e-2, 1e-4)
        for k in ("x1", "x2"):
            err = np.abs(gph[k][live].astype(np.float64) - o[k][live])
            assert (err <= tol).all(), (k, float((err / tol).max()))
        E = np.abs(o["E"][live]).astype(np.float64)
        for k in ("p1", "p2", "p3"):
            err = np.abs(gph[k][live].astype(np.float64) - o[k][live]) / E
            assert (err <= tol).all(), (k, float((err / tol).max()))
        dphi = np.abs(gph["x3"][live].astype(np.float64) - o["x3"][live])
        dphi = np.minimum(dphi, 2 * np.pi - dphi)
        assert (dphi <= 100 * tol).all(), float((dphi / tol).max())
        assert_bits(gph["path_left"][live], o["path_left"][live], "path")
    else:
        _check_photons(gph, case.pho, case.ph_number,
                       ("x1", "x2", "x3", "p1", "p2", "p3", "E", "path_left"), (), kind)
    case.close()


def test_sort_particles_sorts_photons():
    """sim_data::sort_particles sorts the photons too: a stable sort by cell
    with the empty slots trimmed (numpy's stable argsort on the host)."""
    case = RadCase("cart2d", 31)
    case.emit()
    before = case.data.photons_host()
    case.data.sort_particles()
    after = case.data.photons_host()
    ncells = case.m.dims[0] * case.m.dims[1]
    keys = np.where(before["cell"] == oracle.MAX_CELL, ncells, before["cell"]).astype(np.int64)
    perm = np.argsort(keys, kind="stable")
    live = int((before["cell"] != oracle.MAX_CELL).sum())
    assert len(after["cell"]) == live
    for k in before:
        assert_bits(after[k], before[k][perm][:live], f"sorted photon {k}")
    case.close()


def test_empty_passes_keep_the_reference_padding():
    """A conversion pass over no photons and an emission pass with no
    emitter still grow the counts by the reference's padding (50 particle
    slots, one photon slot), on both sides."""
    case = RadCase("cart2d", 41, n=3000, ph_n=0, ph_cap=1000)
    c2, _ = case.pairs()
    assert c2.marked == 0 and case.data.number == 3000 + 50
    case.rp.gamma_thr = 1e9  # no particle is above it: the oracle's copy, the library's below
    import ctypes as C
    from aperture3_b200._lib import ApRadParams, check
    rp = ApRadParams()
    for name, _ in ApRadParams._fields_:
        setattr(rp, name, getattr(case.rp, name) if hasattr(case.rp, name) else 0)
    rp.first_photon_id, rp.first_particle_id = FIRST_PH, FIRST_PTC
    check(case.env._lib.ap_set_rad_params(case.env.ctx, C.byref(rp)), "ap_set_rad_params")
    case.emit_calls = case.pair_calls = 0
    case.next_ph, case.next_ptc = FIRST_PH, FIRST_PTC
    c, _ = case.emit()
    assert c.marked == 0 and case.data.photon_number == 1
    case.close()
