"""Log-spherical surface injection in the oracle (or_ls_inject, the build
semantics of ptc_updater_logsph::inject_ptc): the surface densities against
the reference's own measure_surface_density (run on the host by
oracle/ref_build; float sums there, double here), and the injection rules
(rows with a dense surface skipped, slots, momenta, weights, ids, counter-
based draws, capacity)."""
import numpy as np
import pytest

import oracle
from oracle import logsph as ls
from _cases import empty_ptc, mesh_logsph

REF = ls.load_ref(build=True)


def _surface_ptc(m, n, rng, cap):
    """n particles in the cells next to the stellar surface (c1 from guard
    to guard + 5), species e-, e+, ion, weights in [0.5, 2]."""
    p = empty_ptc(cap)
    p["cell"][:] = oracle.MAX_CELL
    g0, g1 = m.guard[0], m.guard[1]
    c1 = rng.integers(g0, g0 + 6, n)
    c2 = rng.integers(g1, m.dims[1] - g1, n)
    p["cell"][:n] = (c1 + c2 * m.dims[0]).astype(np.uint32)
    p["x1"][:n] = rng.random(n, dtype=np.float32)
    p["x2"][:n] = rng.random(n, dtype=np.float32)
    p["weight"][:n] = rng.uniform(0.5, 2.0, n).astype(np.float32)
    p["flag"][:n] = rng.integers(0, 3, n).astype(np.uint32) << 29
    p["E"][:n] = 1.0
    p["id"][:n] = np.arange(n, dtype=np.uint64)
    return p


@pytest.mark.skipif(REF is None, reason="reference pin library not built")
def test_surface_density_matches_reference():
    m = mesh_logsph(64, 48)
    rng = np.random.default_rng(3)
    p = _surface_ptc(m, 5000, rng, 5000)
    se, sp = oracle.ls_surface_density(m, p, 5000)
    red = m.dims[1] - 2 * m.guard[1]
    re, rp = np.zeros(red, np.float32), np.zeros(red, np.float32)
    s = oracle.ptc_struct(p)
    REF.ref_ls_surface_density(oracle.C.byref(m), oracle.C.byref(s), 5000, oracle._p(re),
                               oracle._p(rp))
    assert np.abs(se).max() > 0 and np.abs(sp).max() > 0
    assert np.allclose(se, re, rtol=1e-5, atol=0)
    assert np.allclose(sp, rp, rtol=1e-5, atol=0)


def test_injection_rules():
    m = mesh_logsph(64, 48)
    rng = np.random.default_rng(4)
    n, inj = 3000, 2
    red = m.dims[1] - 2 * m.guard[1]
    cap = n + 2 * inj * red
    p = _surface_ptc(m, n, rng, cap)
    se, sp = oracle.ls_surface_density(m, p, n)
    q_e = 60.0
    new_n = oracle.ls_inject(m, p, n, cap, inj, 3.0, 0.5, q_e, 77, 5, 10 ** 6)
    assert new_n == cap
    g0, g1 = m.guard[0], m.guard[1]
    inv_d = np.float32(1) / np.float32(m.delta[1])
    injected = 0
    for r in range(red):
        i = r + g1
        th_c = np.float32(m.lower[1] + m.delta[1] * np.float32(r + 0.5))
        dense = np.float32(q_e) * np.float32(max(se[r], sp[r])) > \
            np.float32(1.5) * inv_d * inv_d * np.float32(np.sin(th_c))
        on = (g1 + 1 <= i < m.dims[1] - g1 - 1) and not dense
        sl = slice(n + 2 * r * inj, n + 2 * (r + 1) * inj)
        if not on:
            assert np.all(p["cell"][sl] == oracle.MAX_CELL)
            continue
        injected += 1
        assert np.all(p["cell"][sl] == g0 + 2 + i * m.dims[0])
        assert np.all(p["x1"][sl] == 0.5) and np.all((p["x2"][sl] > 0) & (p["x2"][sl] < 1))
        th = m.lower[1] + m.delta[1] * (r + p["x2"][sl].astype(np.float64))
        assert np.allclose(p["p1"][sl], 3.0 * 2 * np.abs(np.cos(th)), rtol=1e-5, atol=1e-6)
        assert np.allclose(p["p2"][sl], 3.0 * np.sin(th) * np.sign(np.cos(th)), rtol=1e-5,
                           atol=1e-6)
        assert np.allclose(p["weight"][sl], 0.5 * np.sin(th), rtol=1e-5)
        assert np.all(p["E"][sl] == np.float32(np.sqrt(10.0)))
        assert np.array_equal(p["flag"][sl] >> 29, np.tile([0, 1], inj).astype(np.uint32))
        assert np.all((p["flag"][sl] & (1 << 6)) != 0)
    assert 0 < injected < red - 2  # some rows were dense enough to skip
    assert np.array_equal(p["id"][n:cap], 10 ** 6 + np.arange(cap - n, dtype=np.uint64))
    # counter-based: the same call draws the same positions, another call not
    p2 = _surface_ptc(m, n, np.random.default_rng(4), cap)
    oracle.ls_inject(m, p2, n, cap, inj, 3.0, 0.5, q_e, 77, 5, 10 ** 6)
    assert np.array_equal(p2["x2"], p["x2"])
    p3 = _surface_ptc(m, n, np.random.default_rng(4), cap)
    oracle.ls_inject(m, p3, n, cap, inj, 3.0, 0.5, q_e, 77, 6, 10 ** 6)
    live = p["cell"][n:] != oracle.MAX_CELL
    assert not np.array_equal(p3["x2"][n:][live], p["x2"][n:][live])
    # no room: nothing changes
    p4 = _surface_ptc(m, n, np.random.default_rng(4), cap - 1)
    assert oracle.ls_inject(m, p4, n, cap - 1, inj, 3.0, 0.5, q_e, 77, 5, 10 ** 6) == n
