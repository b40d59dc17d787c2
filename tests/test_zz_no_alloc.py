"""The allocation-free 1D update against the oracle and the context path.

ap_update_particles_1d_noalloc serves callers that cannot let a library
allocate device memory while they update particles -- for example a process
whose HBM is fully reserved by another allocator. It uses only the arrays
the caller passes plus a fixed file-scope device array. This file is
collected last on purpose; it must pass on its own in a fresh process and
after the rest of the suite.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest
import torch

import oracle
from _cases import random_fields, random_particles
from _gpu_helpers import Pair, assert_bits, make_params
from aperture3_b200 import SimData, SimEnvironment, _lib, ptc_updater
from aperture3_b200._lib import ApFields, ApParticles
from aperture3_b200.sim import PTC_FIELDS, array_view

pytestmark = pytest.mark.gpu

TOL = 1e-6  # of max |J| and max |rho|, as the other parity tests
MAX_CELLS = 16392  # AP_NOALLOC_MAX_CELLS, guard cells included
MAX_SPECIES = 3    # AP_NOALLOC_MAX_SPECIES


def _fields(data):
    f = ApFields()
    for key in ("E", "B", "Ebg", "Bbg", "J"):
        arr = getattr(f, key)
        for c in range(3):
            arr[c] = array_view(getattr(data, key)[c])
    for s, r in enumerate(data.Rho):
        f.Rho[s] = array_view(r)
    f.divE = array_view(data.divE)
    f.divB = array_view(data.divB)
    return f


def _particles(data):
    p = ApParticles()
    for name, _ in PTC_FIELDS:
        setattr(p, name, data.particles[name].data_ptr())
    return p


def _noalloc(env, data, dt, step):
    st = _lib.lib().ap_update_particles_1d_noalloc(
        C.byref(env.mesh), C.byref(env.ap_params), C.byref(_particles(data)), data.number,
        C.byref(_fields(data)), dt, step, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, _lib.STATUS.get(st, st)
    torch.cuda.synchronize()


def _setup(N, n, seed, data_interval, num_species):
    params = dataclasses.replace(
        make_params((N,), periodic=(True,), capacity=n, data_interval=data_interval),
        num_species=num_species)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(seed)
    f = random_fields(m, rng, amp=0.3, num_species=num_species)
    for key in ("E", "B"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 0, 0))
    p = random_particles(m, n, rng, gamma_max=50.0, species=tuple(range(num_species)))
    return params, f, p


def _compare_with_context(params, f, p, steps):
    n = len(p["x1"])
    env_a = SimEnvironment(params)  # existing, context-based entry point
    da = SimData(env_a, capacity=n)
    da.set_fields(f)
    da.set_particles(p)
    env_b = SimEnvironment(params)  # only for its mesh/params structs and arrays
    db = SimData(env_b, capacity=n)
    db.set_fields(f)
    db.set_particles(p)
    pusher = ptc_updater(env_a)
    for step in steps:
        pusher.update_particles(da, params.delta_t, step)
        _noalloc(env_b, db, params.delta_t, step)
        ga, gb = da.particles_host(), db.particles_host()
        for k, _ in PTC_FIELDS:
            assert_bits(gb[k], ga[k], f"call {step}: particles.{k}")
        fa, fb = da.fields_host(), db.fields_host()
        for key in ("J", "Rho"):
            for c, (a, b) in enumerate(zip(fa[key], fb[key])):
                scale = max(np.abs(a).max(), 1e-30)
                err = np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / scale
                assert err <= TOL, f"call {step}: {key}{c}: {err:.3g}"
                if key == "Rho" and (step + 1) % params.data_interval != 0:
                    assert not np.any(b), f"call {step}: Rho{c} not cleared"
    env_a.close()
    env_b.close()


def test_noalloc_matches_context_path_on_two_calls():
    params, f, p = _setup(512, 4096, 21, data_interval=1, num_species=2)
    _compare_with_context(params, f, p, (0, 1))


def test_noalloc_both_charge_branches_at_species_limit():
    """data_interval 2 over steps 0 and 1: the first call clears Rho (no
    charge output), the second deposits it, with AP_NOALLOC_MAX_SPECIES
    species."""
    params, f, p = _setup(700, 6000, 22, data_interval=2, num_species=MAX_SPECIES)
    _compare_with_context(params, f, p, (0, 1))


def test_noalloc_matches_oracle_at_its_cell_limit():
    """Exactly AP_NOALLOC_MAX_CELLS cells (guards included) and
    AP_NOALLOC_MAX_SPECIES species with charge output on every call, so
    the last accumulator words of the fixed array and the state words
    behind them are in use; two calls in a row against the CPU oracle."""
    N = MAX_CELLS - 4  # two guard cells on each side
    params, f, p = _setup(N, 1 << 16, 23, data_interval=1, num_species=MAX_SPECIES)
    pair = Pair(params, f, p)
    assert pair.data.J[0].shape[-1] == MAX_CELLS
    for step in (0, 1):
        pair.step = step
        _noalloc(pair.env, pair.data, pair.dt, step)
        lost = pair.oracle_update_particles()
        assert lost == 0
        pair.check_particles()
        errs = pair.check_current(rel=TOL, rho=True)
        assert set(errs) == {"J1", "J2", "J3", "Rho0", "Rho1", "Rho2"}
    pair.env.close()


def test_noalloc_allocates_no_device_memory():
    """After a first call (which looks up the fixed array's address), further
    calls leave the free device memory unchanged."""
    params, f, p = _setup(512, 4096, 24, data_interval=1, num_species=2)
    env = SimEnvironment(params)
    data = SimData(env, capacity=len(p["x1"]))
    data.set_fields(f)
    data.set_particles(p)
    _noalloc(env, data, params.delta_t, 0)
    free0 = torch.cuda.mem_get_info()[0]
    for step in (1, 2, 3):
        _noalloc(env, data, params.delta_t, step)
    assert torch.cuda.mem_get_info()[0] == free0
    env.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    """A grid whose row (guards included) exceeds AP_NOALLOC_MAX_CELLS = 16392
    is refused with AP_ERR_CAPACITY before any device work."""
    lib = _lib.lib()
    params = make_params((16392,), periodic=(True,), capacity=1)  # 16396 cells with guards
    env = SimEnvironment(params)
    data = SimData(env, capacity=1)
    st = lib.ap_update_particles_1d_noalloc(
        C.byref(env.mesh), C.byref(env.ap_params), C.byref(_particles(data)), 0,
        C.byref(_fields(data)), params.delta_t, 0, None)
    assert st == 5  # AP_ERR_CAPACITY
    env.close()
