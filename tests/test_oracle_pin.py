"""Pins the CPU oracle (oracle/ap_oracle.c) to the reference.

Two sources of truth, both CPU-only:
* tests/golden/*.npz -- outputs of the reference's own kernels (run on the
  host by oracle/ref_build) on seeded inputs, committed with the script
  that made them (tests/golden/make_golden.py);
* oracle/_ref/libapref.so itself, when it was built (needs the reference
  tree; absent on machines without it, where those cases skip).

Every comparison is bit-exact: the restatement evaluates the same FP32
expressions in the same order as the reference kernels run sequentially.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from _cases import CHARGES, MASSES, mesh_1d, mesh_2d, random_fields, random_particles

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REF = oracle.load_ref(build=True)
needs_ref = pytest.mark.skipif(REF is None, reason="reference pin library not built")


def _F(f):
    return f["E"] + f["B"]


def _same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, what
    if a.dtype.kind == "f":
        ok = (a.view(np.uint32 if a.dtype == np.float32 else np.uint64)
              == b.view(np.uint32 if b.dtype == np.float32 else np.uint64))
        bad = np.flatnonzero(~ok.ravel())
        assert bad.size == 0, f"{what}: {bad.size} differ, first {bad[:5]} {a.ravel()[bad[:3]]} vs {b.ravel()[bad[:3]]}"
    else:
        assert np.array_equal(a, b), what


CASES = [("1d", 512, 0), ("1d", 512, 1), ("2d", (32, 16), 2), ("2d", (64, 32), 3)]


def _case(kind, N, seed, n=3000):
    rng = np.random.default_rng(seed)
    m = mesh_1d(N) if kind == "1d" else mesh_2d(*N)
    f = random_fields(m, rng)
    p = random_particles(m, n, rng)
    return m, f, p


@needs_ref
@pytest.mark.parametrize("kind,N,seed", CASES)
def test_push_deposit_matches_reference_kernels(kind, N, seed):
    m, f, p = _case(kind, N, seed)
    dt = np.float32(0.5 * m.delta[0])
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    oracle.push(m, po, len(p["x1"]), dt, _F(f), CHARGES, MASSES)
    oracle.ref_push(m, pr, len(p["x1"]), dt, _F(f), CHARGES, MASSES)
    for k in po:
        _same(po[k], pr[k], f"push {k}")
    Jo = [np.zeros_like(f["J"][0]) for _ in range(3)]
    Jr = [np.zeros_like(f["J"][0]) for _ in range(3)]
    Ro = [np.zeros_like(f["J"][0]) for _ in range(2)]
    Rr = [np.zeros_like(f["J"][0]) for _ in range(2)]
    oracle.deposit(m, po, len(p["x1"]), dt, 0, 1, Jo, Ro, CHARGES)
    oracle.ref_deposit(m, pr, len(p["x1"]), dt, 0, 1, Jr, Rr, CHARGES)
    for k in po:
        _same(po[k], pr[k], f"deposit {k}")
    for c in range(3):
        _same(Jo[c], Jr[c], f"J{c + 1}")
    for s in range(2):
        _same(Ro[s], Rr[s], f"Rho{s}")


@needs_ref
@pytest.mark.parametrize("kind,N,seed", CASES)
def test_field_kernels_match_reference_kernels(kind, N, seed):
    m, f, _ = _case(kind, N, seed, n=1)
    rng = np.random.default_rng(seed + 100)
    for c in range(3):
        f["J"][c][:] = rng.standard_normal(f["J"][c].shape).astype(np.float32)
    dt = np.float32(0.5 * m.delta[0])
    fo, fr = oracle.copy_fields(f), oracle.copy_fields(f)
    oracle.update_e(m, fo, dt)
    oracle.ref_update_e(m, fr, dt)
    oracle.update_b(m, fo, dt)
    oracle.ref_update_b(m, fr, dt)
    oracle.compute_divs(m, fo)
    oracle.ref_compute_divs(m, fr)
    for key in ("E", "B"):
        for c in range(3):
            _same(fo[key][c], fr[key][c], f"{key}{c + 1}")
    _same(fo["divE"], fr["divE"], "divE")
    _same(fo["divB"], fr["divB"], "divB")


@needs_ref
@pytest.mark.parametrize("kind,N,seed", CASES)
@pytest.mark.parametrize("bnd", [(0, 0, 0, 0), (1, 1, 1, 1), (1, 0, 0, 1)])
def test_filter_matches_reference_kernel(kind, N, seed, bnd):
    m, f, _ = _case(kind, N, seed, n=1)
    rng = np.random.default_rng(seed + 200)
    j = rng.standard_normal(f["J"][0].shape).astype(np.float32)
    jo, jr = j.copy(), j.copy()
    oracle.filter_current(m, jo, np.zeros_like(j), bnd)
    oracle.ref_filter(m, jr, np.zeros_like(j), bnd)
    g0, g1 = m.guard[0], m.guard[1]
    sl = (slice(g1, m.dims[1] - g1) if m.dimension > 1 else slice(0, 1),
          slice(g0, m.dims[0] - g0))
    _same(jo[sl], jr[sl], "filtered bulk")


def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


def test_golden_fixtures_present():
    assert len(_golden_files()) >= 4, "tests/golden fixtures missing"


@pytest.mark.parametrize("path", _golden_files(), ids=os.path.basename)
def test_oracle_matches_golden(path):
    """Replays a fixture made by the reference's own kernels (no reference
    tree needed)."""
    z = np.load(path, allow_pickle=False)
    m = oracle.mesh_from_dict({k[5:]: list(z[k]) if z[k].ndim else int(z[k])
                               for k in z.files if k.startswith("mesh_")})
    dt = np.float32(z["dt"])
    step = int(z["step"])
    data_interval = int(z["data_interval"])
    p = {name: z["in_" + name].copy() for name, _ in oracle.PTC_FIELDS}
    F = [z[f"in_F{k}"].copy() for k in range(6)]
    n = len(p["x1"])
    oracle.push(m, p, n, dt, F, CHARGES, MASSES)
    J = [np.zeros_like(F[0]) for _ in range(3)]
    R = [np.zeros_like(F[0]) for _ in range(2)]
    oracle.deposit(m, p, n, dt, step, data_interval, J, R, CHARGES)
    for name, _ in oracle.PTC_FIELDS:
        _same(p[name], z["out_" + name], f"particles {name}")
    for c in range(3):
        _same(J[c], z[f"out_J{c}"], f"J{c + 1}")
    for s in range(2):
        _same(R[s], z[f"out_Rho{s}"], f"Rho{s}")
    # field solver on the fixture's fields
    f = {"E": [z[f"in_F{k}"].copy() for k in range(3)],
         "B": [z[f"in_F{k}"].copy() for k in range(3, 6)],
         "Ebg": [z[f"in_Ebg{k}"].copy() for k in range(3)],
         "Bbg": [z[f"in_Bbg{k}"].copy() for k in range(3)],
         "J": [z[f"in_J{k}"].copy() for k in range(3)],
         "Rho": [], "divE": np.zeros_like(F[0]), "divB": np.zeros_like(F[0])}
    oracle.update_e(m, f, dt)
    oracle.update_b(m, f, dt)
    oracle.compute_divs(m, f)
    for k in range(3):
        _same(f["E"][k], z[f"fs_E{k}"], f"E{k + 1}")
        _same(f["B"][k], z[f"fs_B{k}"], f"B{k + 1}")
    _same(f["divE"], z["fs_divE"], "divE")
    _same(f["divB"], z["fs_divB"], "divB")


REF_MT = oracle.load_ref_mt(build=True)


@pytest.mark.skipif(REF_MT is None, reason="threaded reference library not built")
@pytest.mark.parametrize("nthreads", [1, 3])
def test_threaded_reference_update_matches_oracle(nthreads):
    """The CPU baseline (the reference's kernels on several host threads)
    computes what the oracle computes with the same particle split: the
    same particles bit for bit, and the same current (both sum per-thread
    buffers in thread order)."""
    m, f, p = _case("2d", (64, 32), 5, n=6000)
    f["Rho"] = [np.zeros_like(f["J"][0]) for _ in range(2)]
    fo, fr = oracle.copy_fields(f), oracle.copy_fields(f)
    po, pr = oracle.copy_ptc(p), oracle.copy_ptc(p)
    dt = np.float32(0.5 * m.delta[0])
    n = len(p["x1"])
    oracle.update_particles(m, po, n, fo, dt, 3, 1, 2, 0, CHARGES, MASSES, [1, 1, 0], nthreads)
    oracle.ref_update_particles_mt(m, pr, n, fr, dt, 3, 1, 2, CHARGES, MASSES, [1, 1, 0],
                                   nthreads)
    for k in po:
        _same(pr[k], po[k], f"particles.{k}")
    for c in range(3):
        _same(fr["J"][c], fo["J"][c], f"J{c + 1}")
    for s in range(2):
        _same(fr["Rho"][s], fo["Rho"][s], f"Rho{s}")
