"""Pin of the photon and pair-production oracle (oracle/ap_rad.c) to the
reference's own code compiled for the host (oracle/_ref/libapref_rad.so:
the user radiative functions of src/ and of the pulsar lab, unmodified;
the photon movers of ptc_updater.cu and ptc_updater_logsph.cu), bit for
bit, and to the committed fixture tests/golden/rad_a.npz. The passes around
the user functions follow the build's rules (slot order, Philox draws, ids,
capacity), which the pin drivers restate.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import rad
from _cases import (LS_CHARGES, mesh_1d, mesh_2d, mesh_logsph, logsph_fields, logsph_particles,
                    rad_photons, rad_rho, random_fields, random_particles)
from _gpu_helpers import assert_bits

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rad_a.npz")

needs_ref = pytest.mark.skipif(not rad.ref_available(), reason="reference tree not present")


def _live_equal(a, b, n, what, keys=None):
    """Cells of all n slots equal; every member equal on live slots."""
    assert_bits(a["cell"][:n], b["cell"][:n], f"{what}: cell")
    live = a["cell"][:n] != oracle.MAX_CELL
    for k in keys or a.keys():
        if k == "cell":
            continue
        assert_bits(a[k][:n][live], b[k][:n][live], f"{what}: {k}")


def _wrap_cells(m, cell, periodic):
    """send_particles for one rank: cells outside the bulk wrapped through
    periodic sides, else emptied."""
    out = cell.copy()
    live = cell != oracle.MAX_CELL
    c = cell[live].astype(np.int64)
    c1, c2 = c % m.dims[0], c // m.dims[0]
    keep = np.ones(c.size, bool)
    for d, cc in ((0, c1), (1, c2)):
        if d >= m.dimension:
            continue
        g, n = m.guard[d], m.dims[d]
        lo, hi = cc < g, cc >= n - g
        if periodic[d]:
            cc[lo] += n - 2 * g
            cc[hi] -= n - 2 * g
        else:
            keep &= ~(lo | hi)
    nc = (c1 + c2 * m.dims[0]).astype(np.uint32)
    nc[~keep] = oracle.MAX_CELL
    out[live] = nc
    return out


def _emit_case(model, m, f, p, n, ph, ph_num, ph_cap, rp, call, first_id):
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    pho, phr = rad.copy_photons(ph), rad.copy_photons(ph)
    cnt_o = np.zeros_like(f["Rho"][0])
    cnt_r = np.zeros_like(f["Rho"][0])
    no, co = rad.emit_photons(m, rp, po, n, pho, ph_num, ph_cap, f, cnt_o, call, first_id)
    nr, cr = rad.ref_emit_photons(m, rp, pr, n, phr, ph_num, ph_cap, f, cnt_r, call, first_id)
    assert no == nr and (co.marked, co.written) == (cr.marked, cr.written)
    for k in po:
        assert_bits(po[k][:n], pr[k][:n], f"emit {model}: particle {k}")
    _live_equal(pho, phr, ph_cap, f"emit {model}: photons")
    assert_bits(pho["id"][ph_num:no], phr["id"][ph_num:no], "photon ids")
    assert_bits(pho["flag"][ph_num:no], phr["flag"][ph_num:no], "photon flags")
    assert_bits(cnt_o, cnt_r, "photon_produced")
    return po, pho, no, co


def _pair_case(model, m, f, ph, ph_num, p, n, cap, rp, call, first_id):
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    pho, phr = rad.copy_photons(ph), rad.copy_photons(ph)
    cnt_o = np.zeros_like(f["Rho"][0])
    cnt_r = np.zeros_like(f["Rho"][0])
    no, co = rad.produce_pairs(m, rp, pho, ph_num, po, n, cap, f, cnt_o, call, first_id)
    nr, cr = rad.ref_produce_pairs(m, rp, phr, ph_num, pr, n, cap, f, cnt_r, call, first_id)
    assert no == nr and (co.marked, co.written) == (cr.marked, cr.written)
    _live_equal(po, pr, cap, f"pairs {model}: particles")
    assert_bits(po["id"][n:no], pr["id"][n:no], "pair ids")
    assert_bits(po["flag"][n:no], pr["flag"][n:no], "pair flags")
    assert_bits(pho["cell"][:ph_num], phr["cell"][:ph_num], "photon cells after conversion")
    assert_bits(cnt_o, cnt_r, "pair_produced")
    return po, pho, no, co


def pulsar_state(seed, N=96, n=6000, ph_n=3000):
    m = mesh_logsph(N, N, rmax=8.0)
    rng = np.random.default_rng(seed)
    f = logsph_fields(m, rng, omega=0.1, noise=0.0)
    rad_rho(f, rng)
    p = logsph_particles(m, n, rng, gamma_max=3e4)
    ph = rad_photons(m, ph_n, 4 * ph_n, rng, E_range=(2.5, 500.0))
    rp = rad.rad_params(rad.RAD_PULSAR, delta_t=0.01, e_curv=2e-8, l_curv=2.0, BQ=0.05, omega=0.1,
                        r_cutoff=6.0, track_percent=0.3, seed=77)
    return m, f, p, ph, rp


def default_state(seed, dim, n=6000, ph_n=3000):
    rng = np.random.default_rng(seed)
    if dim == 1:
        m = mesh_1d(256)
    else:
        m = mesh_logsph(64, 64, rmax=8.0)
    f = random_fields(m, rng)
    rad_rho(f, rng)
    p = random_particles(m, n, rng, gamma_max=200.0, species=(0, 1, 2))
    ph = rad_photons(m, ph_n, 4 * ph_n, rng)
    rp = rad.rad_params(rad.RAD_DEFAULT, gamma_thr=20.0, E_secondary=4.0, photon_path=0.5,
                        r_cutoff=3.0, track_percent=0.25, seed=5)
    return m, f, p, ph, rp


@needs_ref
@pytest.mark.parametrize("dim", [1, 2])
def test_default_model_bit_exact(dim):
    m, f, p, ph, rp = default_state(3 + dim, dim)
    n, ph_num = p["x1"].size, 3000
    po, pho, no, co = _emit_case("default", m, f, p, n, ph, ph_num, ph["x1"].size, rp, 1, 500)
    assert co.marked > 100 and co.written == co.marked
    # photons whose path is over: the default check_produce_pair
    cap = n + 2 * 3000 + 200
    big = oracle.copy_ptc(po)
    for k in big:
        big[k] = np.concatenate([big[k], np.zeros(cap - n, big[k].dtype)])
    big["cell"][n:] = oracle.MAX_CELL
    _pair_case("default", m, f, pho, no, big, n, cap, rp, 1, 90_000)


@needs_ref
def test_pulsar_model_bit_exact():
    m, f, p, ph, rp = pulsar_state(11)
    n, ph_num = p["x1"].size, 3000
    po, pho, no, co = _emit_case("pulsar", m, f, p, n, ph, ph_num, ph["x1"].size, rp, 4, 700)
    assert co.marked > 50
    live_new = pho["cell"][ph_num:no] != oracle.MAX_CELL
    assert 0 < live_new.sum() < co.marked or co.marked > 0
    cap = n + 2 * 8000 + 200
    big = oracle.copy_ptc(po)
    for k in big:
        big[k] = np.concatenate([big[k], np.zeros(cap - n, big[k].dtype)])
    big["cell"][n:] = oracle.MAX_CELL
    pb, phb, nb, cb = _pair_case("pulsar", m, f, pho, no, big, n, cap, rp, 4, 123_456)
    assert cb.marked > 50
    # the guards removed some photons without pairs
    removed = (pho["cell"][:no] != oracle.MAX_CELL) & (phb["cell"][:no] == oracle.MAX_CELL)
    assert removed.sum() > cb.written


@needs_ref
def test_capacity_limits_bit_exact():
    """Emissions past the photon capacity leave their parents unchanged;
    pairs whose second slot is past the particle capacity remove their
    photon: the same on both sides."""
    m, f, p, ph, rp = default_state(21, 2)
    n = p["x1"].size
    _, _, no, co = _emit_case("default", m, f, p, n, ph, 3000, 3100, rp, 2, 0)
    assert co.dropped > 0 and no == 3100
    cap = n + 2 * 50 + 21
    big = oracle.copy_ptc(p)
    for k in big:
        big[k] = np.concatenate([big[k], np.zeros(cap - n, big[k].dtype)])
    big["cell"][n:] = oracle.MAX_CELL
    ph2 = rad.copy_photons(ph)
    ph2["path_left"][:3000] = -1.0
    _, _, nb, cb = _pair_case("default", m, f, ph2, 3000, big, n, cap, rp, 2, 0)
    assert cb.dropped > 0 and nb == cap


@needs_ref
@pytest.mark.parametrize("dim,periodic", [(1, (1, 0, 0)), (1, (0, 0, 0)), (2, (1, 1, 0)),
                                          (2, (0, 1, 0))])
def test_cartesian_mover_bit_exact(dim, periodic):
    rng = np.random.default_rng(30 + dim)
    m = mesh_1d(64) if dim == 1 else mesh_2d(32, 24)
    ph = rad_photons(m, 4000, 4000, rng)
    # put photons at the edges of the bulk moving outwards
    ph["x1"][:200] = np.float32(0.999)
    ph["x1"][200:400] = np.float32(0.0)
    dt = np.float32(0.7 * min(m.delta[0], m.delta[1] if dim > 1 else 1.0))
    po, pr = rad.copy_photons(ph), rad.copy_photons(ph)
    rad.move_photons_cart(m, po, 4000, dt, periodic)
    rad.ref_move_photons_cart(m, pr, 4000, dt)
    pr["cell"][:] = _wrap_cells(m, pr["cell"], periodic)
    _live_equal(po, pr, 4000, f"cart {dim}D mover")
    assert (po["cell"] == oracle.MAX_CELL).sum() > (ph["cell"] == oracle.MAX_CELL).sum() or \
        periodic[0]


@needs_ref
def test_logsph_mover_bit_exact():
    m = mesh_logsph(64, 64, rmax=8.0)
    rng = np.random.default_rng(41)
    ph = rad_photons(m, 5000, 5000, rng)
    # photons by the axis heading across it, and by the outer radius
    g1 = m.guard[1]
    ph["cell"][:300] = (rng.integers(m.guard[0], m.dims[0] - m.guard[0], 300) + g1 * m.dims[0]
                        ).astype(np.uint32)
    ph["x2"][:300] = np.float32(0.05)
    ph["p2"][:300] = -np.abs(ph["p2"][:300]) - 1.0
    dt = np.float32(0.9 * min(m.delta[0], m.delta[1]))
    rp = rad.rad_params(rad.RAD_PULSAR, r_cutoff=6.0)
    po, pr = rad.copy_photons(ph), rad.copy_photons(ph)
    rad.move_photons_logsph(m, rp, po, 5000, dt)
    rad.ref_move_photons_logsph(m, rp.r_cutoff, pr, 5000, dt)
    pr["cell"][:] = _wrap_cells(m, pr["cell"], (0, 0, 0))
    _live_equal(po, pr, 5000, "log-spherical mover")
    assert (po["cell"][:300] == oracle.MAX_CELL).sum() > 0  # some crossed the axis


def test_oracle_matches_golden():
    """The oracle against the committed fixture made from the pin library
    (tests/golden/make_golden.py rad): the pulsar lab's functions through
    emit_photons and produce_pairs."""
    g = dict(np.load(GOLDEN))
    N = int(g["N"])
    m = mesh_logsph(N, N, rmax=8.0)
    f = oracle.new_fields(m, 2)
    for c in range(3):
        f["B"][c][:] = g["B"][c]
    for s in range(2):
        f["Rho"][s][:] = g["Rho"][s]
    p = {k[7:]: g[k].copy() for k in g if k.startswith("in_ptc_")}
    ph_num, ph_cap = int(g["ph_num"]), int(g["ph_cap"])
    ph = rad.new_photons(ph_cap)
    for k in ph:
        ph[k][:ph_num] = g["in_ph_" + k]
    rp = rad.rad_params(rad.RAD_PULSAR, delta_t=0.01, e_curv=2e-8, l_curv=2.0, BQ=0.05,
                        omega=0.1, r_cutoff=6.0, track_percent=0.3, seed=77)
    n = p["x1"].size
    no, _ = rad.emit_photons(m, rp, p, n, ph, ph_num, ph_cap, f, None, 4, 700)
    for k in ("p1", "p2", "p3", "E"):
        assert_bits(p[k], g["emit_ptc_" + k], "emit: particle " + k)
    live = g["emit_ph_cell"] != oracle.MAX_CELL
    assert_bits(ph["cell"][:no], g["emit_ph_cell"], "emit: photon cell")
    for k in ph:
        assert_bits(ph[k][:no][live], g["emit_ph_" + k][live], "emit: photon " + k)
    cap = n + 2 * no + 60
    big = {k: np.concatenate([v, np.zeros(cap - n, v.dtype)]) for k, v in p.items()}
    big["cell"][n:] = oracle.MAX_CELL
    nb, cnt = rad.produce_pairs(m, rp, ph, no, big, n, cap, f, None, 4, 123_456)
    assert cnt.written > 0
    assert_bits(ph["cell"][:no], g["pairs_ph_cell"], "pairs: photon cell")
    live = g["pairs_ptc_cell"] != oracle.MAX_CELL
    assert_bits(big["cell"][n:nb], g["pairs_ptc_cell"], "pairs: cell")
    for k in big:
        assert_bits(big[k][n:nb][live], g["pairs_ptc_" + k][live], "pairs: " + k)
