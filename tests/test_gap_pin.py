"""Pins the 1D gap restatement in the oracle (or_update_ptc_1dgap,
or_filter_gap, or_update_fields_1dgap) to the 1D gap lab's own kernels
(src/cuda/algorithms/ptc_updater_1dgap.cu update_ptc_1dgap and
filter_current1d, field_solver_1dgap.cu update_e_1dgap) run on the host by
oracle/ref_build, and to the committed fixtures made from them. Bit-exact
throughout: both visit the particles in slot order with plain float adds."""
import glob
import os

import numpy as np
import pytest

import oracle
from _cases import GAP_CHARGES, GAP_MASSES, gap_state, mesh_gap

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REF = oracle.load_ref_gap(build=True)
needs_ref = pytest.mark.skipif(REF is None, reason="reference pin library not built")


def _bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    if a.dtype.kind == "f":
        bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
    else:
        bad = np.flatnonzero(a != b)
    assert bad.size == 0, f"{what}: {bad.size} differ, first {bad[:5]}"


def _ref_push(m, p, E3, J1, Rho, dt):
    s = oracle.ptc_struct(p)
    REF.ref_gap_push_deposit(oracle.C.byref(m), oracle.C.byref(s), len(p["x1"]),
                             np.float32(dt), oracle._p(E3), oracle._p(J1),
                             oracle._arr(Rho, 8), len(Rho), oracle._fa(GAP_CHARGES),
                             oracle._fa(GAP_MASSES))


@needs_ref
@pytest.mark.parametrize("N,lower,seed", [(256, 0.0, 1), (300, -0.6, 2), (1024, 0.3, 3)])
def test_gap_push_deposit_matches_reference(N, lower, seed):
    rng = np.random.default_rng(seed)
    m = mesh_gap(N, lower)
    E3, p = gap_state(m, 4000, rng)
    dt = np.float32(0.5 * m.delta[0])
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    nc = m.dims[0]
    Jo, Jr = np.zeros(nc, np.float32), np.zeros(nc, np.float32)
    Ro = [np.zeros(nc, np.float32) for _ in range(2)]
    Rr = [np.zeros(nc, np.float32) for _ in range(2)]
    far = oracle.update_ptc_1dgap(m, po, len(p["x1"]), dt, E3, Jo, Ro, GAP_CHARGES, GAP_MASSES)
    _ref_push(m, pr, E3, Jr, Rr, dt)
    assert far == 0
    for k in po:
        _bits(po[k], pr[k], f"particles.{k}")
    _bits(Jo, Jr, "J1")
    for s in range(2):
        _bits(Ro[s], Rr[s], f"Rho{s}")
    assert np.abs(Jo).max() > 0 and np.any(po["p1"] != p["p1"])


@needs_ref
@pytest.mark.parametrize("bnd", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_gap_filter_matches_reference(bnd):
    rng = np.random.default_rng(5)
    m = mesh_gap(200)
    j = rng.standard_normal(m.dims[0]).astype(np.float32)
    to, tr = np.zeros_like(j), np.zeros_like(j)
    oracle.filter_gap(m, j, to, bnd)
    REF.ref_gap_filter(oracle.C.byref(m), oracle._p(j), oracle._p(tr), bnd[0], bnd[1])
    _bits(to, tr, f"filter {bnd}")


@needs_ref
def test_gap_update_e_matches_reference():
    rng = np.random.default_rng(6)
    m = mesh_gap(300)
    E1 = rng.standard_normal(m.dims[0]).astype(np.float32)
    J1 = rng.standard_normal(m.dims[0]).astype(np.float32)
    Eo, Er = E1.copy(), E1.copy()
    B0, dt = np.float32(1.7), np.float32(0.0013)
    oracle.update_fields_1dgap(m, Eo, J1, B0, dt)
    REF.ref_gap_update_e(oracle.C.byref(m), oracle._p(Er), oracle._p(J1.copy()),
                         np.float32(B0 * 1.6), dt)
    _bits(Eo, Er, "E1")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "gap_*.npz"))))
def test_golden_gap(path):
    """The restatement reproduces the fixtures made from the reference's
    kernels (tests/golden/make_golden.py)."""
    z = np.load(path)
    m = oracle.mesh_from_dict({k[5:]: z[k] for k in z.files if k.startswith("mesh_")})
    p = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
    nc = m.dims[0]
    J = np.zeros(nc, np.float32)
    R = [np.zeros(nc, np.float32) for _ in range(2)]
    oracle.update_ptc_1dgap(m, p, len(p["x1"]), z["dt"], z["E3"], J, R, GAP_CHARGES,
                            GAP_MASSES)
    for k in p:
        _bits(p[k], z["out_" + k], f"particles.{k}")
    _bits(J, z["out_J1"], "J1")
    for s in range(2):
        _bits(R[s], z[f"out_Rho{s}"], f"Rho{s}")
