"""The inverse-Compton oracle (oracle/ap_ic.c) pinned bit for bit to the
reference's own inverse_compton::init (src/cuda/radiation/rt_ic.cu,
compiled for the host by oracle/ref_build as libapref_ic.so), and checked
against properties of the tables and of the lookups that sample them."""
import math

import numpy as np
import pytest

from oracle import rad

NG, NE = 48, 40


@pytest.fixture(scope="module")
def tables():
    return rad.IcTables(rad.gr1d_spectrum(1e-3), 1e-10, 0.1, 1.5e24, NG, NE)


def test_grid(tables):
    """Lorentz factors log-spaced from MIN_GAMMA = 1.01 to MAX_GAMMA = 1e15;
    the energy steps span [0, 1] and [1e-10, 1]."""
    t = tables
    assert t.gammas[0] == np.float32(1.01)
    assert abs(math.log(t.gammas[-1] / 1e15)) < 1e-5
    assert np.all(np.diff(t.gammas) > 0)
    assert t.dep == np.float32(1.0 / (NE - 1))
    assert abs(t.dlep * (NE - 1) - math.log(1e10)) < 1e-4


def test_rates(tables):
    """Scattering rates positive; the pair rate zero below a photon energy
    of 2 (the threshold of gamma-gamma pair creation) and positive above
    where the background reaches the threshold."""
    t = tables
    assert np.all(t.ic_rate > 0)
    assert np.all(t.gg_rate[t.gammas < 2.0] == 0)
    assert np.all(t.gg_rate[t.gammas > 100.0] > 0)


def test_cumulative_spectra(tables):
    """Every row with emission is a distribution: non-decreasing from >= 0
    to exactly 1 (the reference divides by the last entry); rows without
    any contribution are 0 / 0."""
    for d in (tables.dNde, tables.dNde_thomson):
        for row in d:
            if np.isnan(row[-1]):
                assert np.all(np.isnan(row))
                continue
            assert row[-1] == np.float32(1.0)
            assert row[0] >= 0
            assert np.all(np.diff(row) >= -1e-7)


def test_lookups(tables):
    """find_ic_rate interpolates the table (exact at the grid points up to
    the float log), find_gg_rate is zero below 2, gen_photon_e stays in
    [0, gamma - 1.01] (it is not monotonic in the uniform: below the third
    entry of the linear table it switches to the logarithmic one)."""
    t = tables
    for n in (3, 10, 30):
        g = float(t.gammas[n])
        assert abs(t.rate(g) - t.ic_rate[n]) <= 1e-5 * abs(t.ic_rate[n]) + 1e-30
    assert t.gg(1.5) == 0.0
    for g in (1.5, 30.0, 1e4, 1e9):
        es = [t.photon_e(g, u) for u in np.linspace(0.01, 1.0, 25)]
        assert all(0.0 <= e <= max(0.0, g - 1.01) * (1 + 1e-6) for e in es), (g, es)


def test_spectra():
    """The spectra's densities as the reference's functors: zero outside
    their range, the broken power law continuous at its peak."""
    b = rad.gr1d_spectrum(1e-3)
    lib = rad.lib
    import ctypes as C
    lib.or_spectrum_ne.restype = C.c_double
    lib.or_spectrum_ne.argtypes = [C.c_void_p, C.c_double]
    ne = lambda s, e: lib.or_spectrum_ne(C.byref(s), e)  # noqa: E731
    assert ne(b, 1e-11) == 0.0 and ne(b, 0.2) == 0.0
    lo, hi = ne(b, 0.999e-3), ne(b, 1.001e-3)
    assert abs(lo - hi) / hi < 0.01
    bb = rad.spectrum(rad.SPEC_BLACK_BODY, 1e-4)
    e = 2e-4
    kT = float(np.float32(1e-4))
    assert abs(ne(bb, e) - 1.75464e30 * e * e / math.expm1(e / kT)) < 1e-12 * ne(bb, e)


SPECTRA = [
    (rad.SPEC_BROKEN_POWER_LAW, (1.25, 1.1, 1e-3, 1e-10, 0.1), 1e-10, 0.1, 1.5e24),
    (rad.SPEC_BLACK_BODY, (3e-6,), 3e-16, 3e-3, 1e-6),
    (rad.SPEC_POWER_LAW_HARD, (0.5, 1e-6, 1e-2), 1e-6, 1e-2, 1e20),
    (rad.SPEC_POWER_LAW_SOFT, (2.0, 1e-6, 1e-2), 1e-6, 1e-2, 1e20),
    (rad.SPEC_MONO_ENERGETIC, (1e-3, 1e-4), 1e-5, 1e-1, 1e18),
]


@pytest.mark.skipif(rad.load_ref_ic() is None, reason="reference tree not present")
@pytest.mark.parametrize("kind,p,emin,emax,n0", SPECTRA)
def test_tables_bit_exact_against_reference(kind, p, emin, emax, n0):
    """Every table entry and step of the oracle equals the reference's own
    init on the same grid, for each of its spectra."""
    ng, ne = 24, 20
    spec = rad.spectrum(kind, *p)
    ref = rad.ref_ic_tables(spec, emin, emax, n0, ng, ne)
    got = rad.IcTables(spec, emin, emax, n0, ng, ne)
    for k in ("dep", "dg", "dlep"):
        assert np.float32(getattr(got, k)) == np.float32(ref[k]), k
    for k in ("ic_rate", "gg_rate", "gammas", "dNde", "dNde_thomson"):
        a, b = getattr(got, k), ref[k]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, np.flatnonzero(
            a.view(np.uint32).ravel() != b.view(np.uint32).ravel())[:5])
