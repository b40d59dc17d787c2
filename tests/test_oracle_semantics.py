"""Known-answer tests of the CPU oracle from the physics and from the
reference's data semantics. The reference's own push, deposit and solver
tests cannot build (they include headers that no longer exist), so these
properties are checked directly."""
import numpy as np
import pytest

import oracle
from _cases import CHARGES, MASSES, mesh_1d, mesh_2d, random_fields, random_particles


def _one(m, c1, c2, x1, x2, p, sp=1):
    q = {name: np.zeros(1, dt) for name, dt in oracle.PTC_FIELDS}
    q["cell"][0] = c1 + c2 * m.dims[0]
    q["x1"][0], q["x2"][0] = x1, x2
    q["p1"][0], q["p2"][0], q["p3"][0] = p
    q["E"][0] = np.sqrt(1 + sum(np.float64(v) ** 2 for v in p))
    q["weight"][0] = 1.0
    q["flag"][0] = np.uint32(sp) << np.uint32(29)
    return q


def _uniform(m, E=(0, 0, 0), B=(0, 0, 0)):
    f = oracle.new_fields(m)
    for c in range(3):
        f["E"][c][:] = E[c]
        f["B"][c][:] = B[c]
    return f


def test_vay_gyration_conserves_gamma():
    """E = 0, uniform B: the Vay rotation keeps |p| (vay_push.cuh:8-30)."""
    m = mesh_2d(16, 16)
    f = _uniform(m, B=(0.0, 0.0, 1.0))
    p = _one(m, 8, 8, 0.5, 0.5, (3.0, 1.0, 0.5))
    g0 = np.sqrt(1 + 9 + 1 + 0.25)
    dt = np.float32(0.05)
    for _ in range(200):
        oracle.push(m, p, 1, dt, f["E"] + f["B"], CHARGES, MASSES)
    g = np.sqrt(1 + p["p1"][0] ** 2 + p["p2"][0] ** 2 + p["p3"][0] ** 2)
    assert abs(g - g0) / g0 < 1e-5
    assert abs(p["p3"][0] - 0.5) < 1e-5  # no force along B


def test_exb_drift_velocity():
    """E x B drift: a positron released at rest in E = (0, 0.1, 0),
    B = (0, 0, 1) drifts along +x at |E|/|B| on average."""
    m = mesh_2d(16, 16)
    f = _uniform(m, E=(0.0, 0.1, 0.0), B=(0.0, 0.0, 1.0))
    p = _one(m, 8, 8, 0.5, 0.5, (0.0, 0.0, 0.0))
    dt = np.float32(0.01)
    v = []
    for _ in range(4000):
        oracle.push(m, p, 1, dt, f["E"] + f["B"], CHARGES, MASSES)
        g = np.sqrt(1 + p["p1"][0] ** 2 + p["p2"][0] ** 2 + p["p3"][0] ** 2)
        v.append(p["p1"][0] / g)
    assert abs(np.mean(v) - 0.1) < 5e-3


@pytest.mark.parametrize("seed", range(4))
def test_single_particle_charge_conservation_2d(seed):
    """Esirkepov: rho_new - rho_old + div J = 0 for one particle
    (ptc_updater.cu:295-386), including cell crossings."""
    rng = np.random.default_rng(seed)
    m = mesh_2d(16, 16)
    f = _uniform(m)
    p = _one(m, 8, 8, rng.random(), rng.random(), tuple(4 * rng.standard_normal(3)))
    dt = np.float32(0.5 * m.delta[0])
    sh = f["J"][0].shape
    J = [np.zeros(sh) for _ in range(3)]
    R0 = [np.zeros(sh) for _ in range(2)]
    R1 = [np.zeros(sh) for _ in range(2)]
    q = oracle.copy_ptc(p)
    # rho at the start: deposit a zero-length move
    q2 = oracle.copy_ptc(p)
    q2["p1"][0] = q2["p2"][0] = q2["p3"][0] = 0.0
    q2["E"][0] = 1.0
    oracle.deposit(m, q2, 1, dt, 0, 1, [np.zeros(sh)] * 3, R0, CHARGES, f64=True)
    oracle.deposit(m, q, 1, dt, 0, 1, J, R1, CHARGES, f64=True)
    d = (R1[0] + R1[1]) - (R0[0] + R0[1])
    div = np.zeros(sh)
    div[:, :-1] += J[0][:, 1:] - J[0][:, :-1]
    div[:-1, :] += J[1][1:, :] - J[1][:-1, :]
    assert np.abs(d + div).max() < 1e-6


def test_stable_counting_sort_matches_numpy():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 37, 5000).astype(np.uint32)
    perm = oracle.stable_counting_sort(keys, 37)
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))


def test_wrap_in_place_equals_hole_and_append():
    """send_particles (hole + append, sim_environment_impl.hpp:319-412) and
    the in-place wrap leave the same set of particles, compared by id."""
    rng = np.random.default_rng(4)
    m = mesh_2d(24, 20)
    p = random_particles(m, 2000, rng)
    g0, g1 = m.guard[0], m.guard[1]
    c1 = rng.integers(g0 - 1, m.dims[0] - g0 + 1, 2000)
    c2 = rng.integers(g1 - 1, m.dims[1] - g1 + 1, 2000)
    p["cell"][:] = (c1 + c2 * m.dims[0]).astype(np.uint32)
    for per in [(1, 1, 0), (1, 0, 0), (0, 0, 0)]:
        a = oracle.copy_ptc(p)
        big = {k: np.concatenate([v, np.zeros(4000, v.dtype)]) for k, v in p.items()}
        n_out = oracle.send_particles(m, big, 2000, 6000, per)
        oracle.wrap_particles(m, a, 2000, per)
        keep_a = a["cell"] != oracle.MAX_CELL
        keep_b = big["cell"][:n_out] != oracle.MAX_CELL
        ia = dict(zip(a["id"][keep_a], a["cell"][keep_a]))
        ib = dict(zip(big["id"][:n_out][keep_b], big["cell"][:n_out][keep_b]))
        assert ia == ib


def test_guard_exchange_on_tiny_grid():
    """send_guard_cells copies interior strips; send_add_guard_cells adds the
    guard strips into the opposite interior and leaves the guards."""
    m = mesh_2d(6, 5, guard=2)
    a = np.arange(m.dims[0] * m.dims[1], dtype=np.float32).reshape(m.dims[1], m.dims[0])
    b = a.copy()
    oracle.send_guard_cells(m, b, (1, 1, 0))
    r0, r1 = m.dims[0] - 4, m.dims[1] - 4
    for y in range(m.dims[1]):
        for x in range(m.dims[0]):
            xi = x if 2 <= x < 2 + r0 else (x + r0 if x < 2 else x - r0)
            yi = y if 2 <= y < 2 + r1 else (y + r1 if y < 2 else y - r1)
            assert b[y, x] == a[yi, xi]
    c = a.copy()
    oracle.send_add_guard_cells(m, c, (1, 1, 0))
    assert c[0, 0] == a[0, 0]  # guards untouched
    assert c[2, 2] == a[2, 2] + a[2, 2 + r0] + a[2 + r1, 2] + a[2 + r1, 2 + r0]


def test_oracle_multithread_deposit_matches_single_thread_fp64_within_rounding():
    rng = np.random.default_rng(5)
    m = mesh_2d(32, 32)
    f = random_fields(m, rng, amp=0.3)
    p = random_particles(m, 20000, rng)
    a, b = oracle.copy_ptc(p), oracle.copy_ptc(p)
    fa, fb = oracle.copy_fields(f), oracle.copy_fields(f)
    oracle.update_particles(m, a, 20000, fa, 0.5 * m.delta[0], 0, 1, 2, 0, CHARGES, MASSES, (1, 1, 0), 1)
    oracle.update_particles(m, b, 20000, fb, 0.5 * m.delta[0], 0, 1, 2, 0, CHARGES, MASSES, (1, 1, 0), 4)
    for k in ("p1", "x1", "cell"):
        assert np.array_equal(a[k], b[k])
    for c in range(3):
        s = np.abs(fa["J"][c]).max()
        assert np.abs(fa["J"][c] - fb["J"][c]).max() <= 2e-6 * s
