"""Pair injection in the CPU oracle: the Philox4x32-10 generator against the
known-answer vectors published with the algorithm (Random123 kat_vectors,
philox4x32 with 10 rounds), and the injection semantics (energy
bookkeeping, ids, slot order, capacity limit)."""
import numpy as np

import oracle
from _cases import empty_ptc

KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


def test_philox_known_answers():
    for ctr, key, want in KAT:
        assert oracle.philox4x32_10(ctr, key) == want


def _beam(n, cap, rng, hot_frac=0.5):
    p = empty_ptc(cap)
    p["cell"][:] = oracle.MAX_CELL
    p["cell"][:n] = rng.integers(2, 514, n).astype(np.uint32)
    p["x1"][:n] = rng.random(n, dtype=np.float32)
    hot = rng.random(n) < hot_frac
    g = np.where(hot, 10 ** rng.uniform(6.2, 7.0, n), 1 + rng.random(n))
    p["p1"][:n] = (np.sign(rng.standard_normal(n)) * np.sqrt(g * g - 1)).astype(np.float32)
    p["E"][:n] = np.sqrt(1 + p["p1"][:n].astype(np.float64) ** 2).astype(np.float32)
    p["weight"][:n] = 1.0
    p["flag"][:n] = (rng.integers(0, 2, n).astype(np.uint32) << 29)
    p["id"][:n] = np.arange(n, dtype=np.uint64) * 7 + 3
    return p


def test_injection_semantics():
    rng = np.random.default_rng(0)
    n, cap = 4000, 40000
    p = _beam(n, cap, rng)
    before = oracle.copy_ptc(p)
    dt, thr, lam, eph = np.float32(0.01), 1e6, 0.05, np.float32(50.0)
    new_n, em, dr = oracle.inject_pairs(p, n, cap, dt, 7, thr, lam, eph, 1234, 10 ** 9)
    assert dr == 0 and new_n == n + 2 * em
    # about P = 1 - exp(-dt / lambda) of the hot particles emit
    hot = before["E"][:n] > thr
    expect = hot.sum() * (1 - np.exp(-dt / lam))
    assert abs(em - expect) < 5 * np.sqrt(expect) + 5
    emitters = np.flatnonzero(p["E"][:n] != before["E"][:n])
    assert len(emitters) == em and np.all(hot[emitters])
    # parents lose exactly the photon energy (in FP32), keep direction
    assert np.allclose(before["E"][emitters] - p["E"][emitters], eph, rtol=0, atol=1.0)
    assert np.all(np.sign(p["p1"][emitters]) == np.sign(before["p1"][emitters]))
    # pairs: slot order of the parents, ids consecutive, e- then e+
    kids = slice(n, new_n)
    assert np.array_equal(p["id"][kids], 10 ** 9 + np.arange(2 * em, dtype=np.uint64))
    assert np.array_equal(p["flag"][kids] >> 29, np.tile([0, 1], em).astype(np.uint32))
    assert np.all((p["flag"][kids] & (1 << 7)) != 0)
    assert np.array_equal(p["cell"][n:new_n:2], before["cell"][emitters])
    q = np.sqrt(0.25 * 50.0 ** 2 - 1)
    assert np.allclose(np.abs(p["p1"][kids]), q, rtol=1e-6)
    # the same call again draws the same numbers (counter-based)
    p2 = oracle.copy_ptc(before)
    assert oracle.inject_pairs(p2, n, cap, dt, 7, thr, lam, eph, 1234, 10 ** 9) == (new_n, em, 0)
    for k in p:
        assert np.array_equal(p[k], p2[k])
    # another step or seed draws differently
    p3 = oracle.copy_ptc(before)
    _, em3, _ = oracle.inject_pairs(p3, n, cap, dt, 8, thr, lam, eph, 1234, 10 ** 9)
    assert not np.array_equal(p3["E"][:n], p["E"][:n]) or em3 != em


def test_injection_capacity_limit():
    rng = np.random.default_rng(1)
    n = 3000
    p = _beam(n, n + 11, rng, hot_frac=1.0)
    new_n, em, dr = oracle.inject_pairs(p, n, n + 11, np.float32(1.0), 0, 1e6, 0.05, 50.0, 9, 0)
    assert em == 5 and new_n == n + 10 and dr > 0
