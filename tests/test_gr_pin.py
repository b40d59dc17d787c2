"""Pins the 1D GR restatement in the oracle (or_gr_coef, or_update_ptc_1dgr,
or_filter_gr, or_update_e_1dgr) to the 1D GR lab's own code run on the host
by oracle/ref_build: Grid_1dGR::compute_coef (src/grids/grid_1dgr.cpp) fed
the same tables its HDF5 file would hold, update_ptc_1dgr and
filter_current1d (src/cuda/algorithms/ptc_updater_1dgr.cu) and update_e_1dgr
(field_solver_1dgr.cu); and to the committed fixture made from them.
Bit-exact throughout: both visit the particles in slot order with plain
float adds and the same C library transcendentals."""
import os

import numpy as np
import pytest

import oracle
from _cases import GR_A, GR_OMEGA, gr_dt, gr_mesh, gr_particles, gr_table

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "gr_a.npz")
REF = oracle.load_ref_gr(build=True)
needs_ref = pytest.mark.skipif(REF is None, reason="reference pin library not built")
CHARGES = [-1.2, 1.2] + [1.2] * 6
MASSES = [1.2] * 8


def _bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    if a.dtype.kind == "f":
        bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
    else:
        bad = np.flatnonzero(a != b)
    assert bad.size == 0, f"{what}: {bad.size} differ, first {bad[:5]}"


def _ref_coef(m, tab, B0=1.0):
    out = [np.zeros(m.dims[0], np.float32) for _ in range(oracle.GR_NCOEF)]
    cols = [np.ascontiguousarray(tab[k], np.float32) for k in oracle.GR_TABLE_KEYS]
    REF.ref_gr_coef(oracle.C.byref(m), np.float32(GR_A), np.float32(GR_OMEGA), np.float32(B0),
                    *[oracle._p(c) for c in cols], len(cols[0]), oracle._arr(out, 15))
    return out


def _case(N, n, seed):
    m = gr_mesh(N)
    tab = gr_table()
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, 1.0, tab)
    rng = np.random.default_rng(seed)
    p = gr_particles(m, co, n, rng)
    E3 = (0.05 * np.sin(0.013 * np.arange(m.dims[0]))).astype(np.float32)
    return m, tab, co, p, E3, np.float32(gr_dt(m, co, p))


@needs_ref
@pytest.mark.parametrize("N,B0", [(512, 1.0), (2048, 3.0)])
def test_coef_matches_reference(N, B0):
    m = gr_mesh(N)
    tab = gr_table()
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, B0, tab)
    ref = _ref_coef(m, tab, B0)
    for name, a, b in zip(oracle.GR_COEF_NAMES, co, ref):
        _bits(a, b, name)
    assert np.all(np.isfinite(co[oracle.GR_COEF_NAMES.index("K1")]))


@needs_ref
@pytest.mark.parametrize("N,n,seed,step", [(512, 3000, 1, 0), (2048, 20000, 2, 3), (1024, 8000, 3, 4)])
def test_push_deposit_matches_reference(N, n, seed, step):
    m, tab, co, p, E3, dt = _case(N, n, seed)
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    nc = m.dims[0]
    Jo, Jr = np.zeros(nc, np.float32), np.zeros(nc, np.float32)
    Ro = [np.zeros(nc, np.float32) for _ in range(2)]
    Rr = [np.zeros(nc, np.float32) for _ in range(2)]
    far = oracle.update_ptc_1dgr(m, po, n, dt, step, 4, GR_A, GR_OMEGA, E3, co, Jo, Ro, CHARGES,
                                 MASSES)
    REF.ref_gr_push(oracle.C.byref(m), oracle.C.byref(oracle.ptc_struct(pr)), n, dt, step, 4,
                    np.float32(GR_A), np.float32(GR_OMEGA), oracle._p(E3),
                    oracle._arr(co, 15), oracle._p(Jr), oracle._arr(Rr, 8), 2,
                    oracle._fa(CHARGES), oracle._fa(MASSES))
    assert far == 0
    for k in po:
        _bits(po[k], pr[k], f"particles.{k}")
    _bits(Jo, Jr, "J1")
    for s in range(2):
        _bits(Ro[s], Rr[s], f"Rho{s}")
    tracked = (p["flag"] & 2) != 0
    assert np.abs(Jo).max() > 0 and np.any(po["p1"] != p["p1"])
    if step % 4 == 0:
        assert np.any(po["p2"][tracked] != 0)


@needs_ref
@pytest.mark.parametrize("bnd", [(1, 1), (0, 0), (1, 0)])
def test_filter_and_e_update_match_reference(bnd):
    m, tab, co, p, E3, dt = _case(700, 10, 4)
    rng = np.random.default_rng(5)
    j = rng.standard_normal(m.dims[0]).astype(np.float32)
    to, tr = np.zeros_like(j), np.zeros_like(j)
    for k1 in (co[oracle.GR_COEF_NAMES.index("K1")], co[oracle.GR_COEF_NAMES.index("K1_j")]):
        oracle.filter_gr(m, j, to, k1, bnd)
        REF.ref_gr_filter(oracle.C.byref(m), oracle._p(j), oracle._p(tr), oracle._p(k1), *bnd)
        _bits(to, tr, "filtered")
    Eo, Er = j.copy(), j.copy()
    J1 = rng.standard_normal(m.dims[0]).astype(np.float32)
    oracle.update_e_1dgr(m, Eo, J1, co[oracle.GR_COEF_NAMES.index("j0")], dt)
    REF.ref_gr_update_e(oracle.C.byref(m), oracle._p(Er), oracle._p(J1), oracle._arr(co, 15),
                        dt)
    _bits(Eo, Er, "E1")


def test_oracle_matches_committed_fixture():
    """The restatement against outputs of the lab's own code saved by
    tests/golden/make_golden.py (runs without the reference tree)."""
    g = np.load(GOLDEN)
    m = gr_mesh(int(g["N"]))
    tab = {k: g["tab_" + k] for k in oracle.GR_TABLE_KEYS}
    co = oracle.gr_coef(m, GR_A, GR_OMEGA, float(g["B0"]), tab)
    for k, name in enumerate(oracle.GR_COEF_NAMES):
        _bits(co[k], g["coef"][k], name)
    p = {k: g["in_" + k].copy() for k, _ in oracle.PTC_FIELDS}
    n = len(p["x1"])
    nc = m.dims[0]
    J1 = np.zeros(nc, np.float32)
    Rho = [np.zeros(nc, np.float32) for _ in range(2)]
    oracle.update_ptc_1dgr(m, p, n, g["dt"], int(g["step"]), 4, GR_A, GR_OMEGA, g["E3"], co, J1,
                           Rho, CHARGES, MASSES)
    for k, _ in oracle.PTC_FIELDS:
        _bits(p[k], g["out_" + k], f"particles.{k}")
    _bits(J1, g["J1"], "J1")
    for s in range(2):
        _bits(Rho[s], g["Rho"][s], f"Rho{s}")
