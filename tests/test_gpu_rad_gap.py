"""The 1D gap lab's radiative transfer on the GPU against the CPU oracle
(the gap model and mover of oracle/ap_rad.c, pinned to the lab's own code
by tests/test_rad_gr_pin.py): emission by the inverse-Compton rate with the
photon energy drawn from the tables, conversion by the gamma-gamma rate,
the photon mover of ptc_updater_1dgap. The tables differ from the oracle's
in the last bits of CUDA's exp / log / pow (tests/test_gpu_rad_gr.py), so a
decision can differ only where a draw meets a rate's last bit and the
sampled photon energies agree to 1e-3 relative at p99.9."""
import numpy as np
import pytest

import oracle
from oracle import rad
from _gpu_helpers import assert_bits
from aperture3_b200 import SimData, SimEnvironment, SimParams, ptc_updater_1dgap, radiative_transfer
from _cases import gap_rad_case

NG, NE = 64, 56

pytestmark = pytest.mark.gpu

FIRST_PH, FIRST_PTC = 1 << 40, 1 << 41


class GapRadCase:
    def __init__(self, ic_path=0.004, n=20000, n_ph=20000):
        (self.m, self.rp, self.gap, self.p, self.ph, self.n, self.n_ph, self.cap,
         self.ph_cap) = gap_rad_case(NG, NE, n=n, n_ph=n_ph, ic_path=ic_path)
        m = self.m
        params = SimParams(N=(m.dims[0] - 4, 1, 1), guard=(2, 0, 0), lower=(0.0, 0.0, 0.0),
                           size=(1.0, 1.0, 1.0), delta_t=2e-3, q_e=1.0, num_species=2,
                           periodic_boundary=(False, False, False), max_ptc_number=self.cap,
                           B0=0.7, coord_system="1dgap", create_pairs=True,
                           max_photon_number=self.ph_cap, rad_model="gap1d", rad_seed=9,
                           e_min=1e-3, ic_path=ic_path, n_gamma=NG, n_ep=NE,
                           track_percent=0.3)
        self.env = SimEnvironment(params)
        self.data = SimData(self.env, capacity=self.cap, photon_capacity=self.ph_cap)
        self.data.set_particles({k: v[:self.n] for k, v in self.p.items()})
        self.data.set_photons({k: v[:self.n_ph] for k, v in self.ph.items()})
        self.rt = radiative_transfer(self.env, first_photon_id=FIRST_PH,
                                     first_particle_id=FIRST_PTC)
        self.f = oracle.new_fields(m, 2)

    def close(self):
        self.env.close()


def _rel(a, b, floor):
    return np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), floor)


def test_gap_emission_matches_oracle():
    case = GapRadCase()
    got = case.rt.emit_photons(case.data)
    po, pho = oracle.copy_ptc(case.p), rad.copy_photons(case.ph)
    n_ph, c = rad.emit_photons(case.m, case.rp, po, case.n, pho, case.n_ph, case.ph_cap, case.f,
                               None, 0, FIRST_PH)
    assert c.marked > 1000, c.marked
    assert abs(got["marked"] - c.marked) <= 2, (got, c.marked)
    g, gph = case.data.particles_host(), case.data.photons_host()
    for k in ("cell", "x1", "weight", "flag", "id"):
        assert_bits(g[k][:case.n], po[k][:case.n], f"particle {k}")
    for k in ("E", "p1"):
        err = _rel(g[k][:case.n], po[k][:case.n], 1e-6)
        assert np.quantile(err, 0.999) <= 1e-3, (k, np.quantile(err, 0.999))
    if got["marked"] == c.marked:
        assert case.data.photon_number == n_ph
        live = (pho["cell"][:n_ph] != oracle.MAX_CELL) & (gph["cell"][:n_ph] != oracle.MAX_CELL)
        assert live.sum() > 100
        for k in ("cell", "x1", "weight", "flag", "id"):
            assert_bits(gph[k][:n_ph][live], pho[k][:n_ph][live], f"photon {k}")
        for k in ("E", "p1"):
            err = _rel(gph[k][:n_ph][live], pho[k][:n_ph][live], 1e-6)
            assert np.quantile(err, 0.999) <= 1e-3 and err.max() <= 1e-2, (k, err.max())
    case.close()


def test_gap_pair_production_matches_oracle():
    case = GapRadCase(ic_path=0.0005)
    got = case.rt.produce_pairs(case.data)
    po, pho = oracle.copy_ptc(case.p), rad.copy_photons(case.ph)
    n_p, c = rad.produce_pairs(case.m, case.rp, pho, case.n_ph, po, case.n, case.cap, case.f,
                               None, 0, FIRST_PTC)
    assert c.marked > 500, c.marked
    assert abs(got["marked"] - c.marked) <= 2, (got, c.marked)
    g, gph = case.data.particles_host(), case.data.photons_host()
    assert np.count_nonzero(gph["cell"][:case.n_ph] != pho["cell"][:case.n_ph]) <= 2
    if got["marked"] == c.marked:
        assert case.data.number == n_p
        sl = slice(case.n, n_p)
        for k in ("cell", "x1", "weight", "flag", "id", "p1", "E"):
            assert_bits(g[k][sl], po[k][sl], f"pair {k}")
    case.close()


def test_gap_photon_mover_in_update():
    """update_particles of the gap lab moves the photons after the
    particles (and removes those outside the bulk), bit for bit."""
    case = GapRadCase(n=2000)
    pusher = ptc_updater_1dgap(case.env)
    pho = rad.copy_photons(case.ph)
    for step in range(3):
        pusher.update_particles(case.data, 2e-3, step)
        rad.move_photons_gap(case.m, pho, case.n_ph, np.float32(2e-3))
    gph = case.data.photons_host()
    for k in ("cell", "x1", "p1", "E"):
        assert_bits(gph[k][:case.n_ph], pho[k][:case.n_ph], f"photon {k}")
    case.close()
