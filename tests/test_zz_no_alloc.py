"""The allocation-free 1D update against the context-based one.

ap_update_particles_1d_noalloc serves callers that cannot let a library
allocate device memory while they update particles -- for example a process
whose HBM is fully reserved by another allocator. It uses only the arrays
the caller passes plus a fixed file-scope device array. This file is
collected last on purpose; it must pass on its own in a fresh process and
after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from _cases import random_fields, random_particles
from _gpu_helpers import assert_bits, make_params
from aperture3_b200 import SimData, SimEnvironment, _lib, ptc_updater
from aperture3_b200._lib import ApFields, ApParticles
from aperture3_b200.sim import PTC_FIELDS, array_view

pytestmark = pytest.mark.gpu

TOL = 1e-6  # of max |J| and max |rho|, as the other parity tests


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


def test_noalloc_matches_context_path_on_two_calls():
    n = 4096
    params = make_params((512,), periodic=(True,), capacity=n, data_interval=1)
    m = oracle.make_mesh(params.N, params.guard, size=params.size)
    rng = np.random.default_rng(21)
    f = random_fields(m, rng, amp=0.3)
    for key in ("E", "B"):
        for c in range(3):
            oracle.send_guard_cells(m, f[key][c], (1, 0, 0))
    p = random_particles(m, n, rng, gamma_max=50.0)

    env_a = SimEnvironment(params)  # existing, context-based entry point
    da = SimData(env_a, capacity=n)
    da.set_fields(f)
    da.set_particles(p)
    env_b = SimEnvironment(params)  # only for its mesh/params structs and arrays
    db = SimData(env_b, capacity=n)
    db.set_fields(f)
    db.set_particles(p)
    lib = _lib.lib()
    pusher = ptc_updater(env_a)
    for step in (0, 1):
        pusher.update_particles(da, params.delta_t, step)
        st = lib.ap_update_particles_1d_noalloc(
            C.byref(env_b.mesh), C.byref(env_b.ap_params), C.byref(_particles(db)), db.number,
            C.byref(_fields(db)), params.delta_t, step,
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0, _lib.STATUS.get(st, st)
        torch.cuda.synchronize()
        ga, gb = da.particles_host(), db.particles_host()
        for k, _ in PTC_FIELDS:
            assert_bits(gb[k], ga[k], f"call {step}: particles.{k}")
        fa, fb = da.fields_host(), db.fields_host()
        for key in ("J", "Rho"):
            for c, (a, b) in enumerate(zip(fa[key], fb[key])):
                scale = max(np.abs(a).max(), 1e-30)
                err = np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / scale
                assert err <= TOL, f"call {step}: {key}{c}: {err:.3g}"
    env_a.close()
    env_b.close()


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
