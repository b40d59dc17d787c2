"""Log-spherical oracle wrappers -- TEST INFRASTRUCTURE ONLY.

Wraps the ``*_f32`` (FP32-literal) and ``*_f64`` (full FP64) restatements
in ``ap_logsph.c`` and the optional pin library ``_ref/libapref_ls.so``,
which runs the reference's own log-spherical kernels
(``src/cuda/algorithms/ptc_updater_logsph.cu``, ``field_solver_logsph.cu``,
``src/grids/grid_log_sph.cpp``) on the host.

Coefficient arrays come as a list of 13 ``(dims[1], dims[0])`` arrays in
the order of ``COEF_NAMES`` (the ``Grid_LogSph`` members).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import (PTC_FIELDS, _HERE, _arr, _build, _fa, _p, fields_struct, lib, ref_tree_present,
               ptc_struct)

COEF_NAMES = ("l1_e", "l2_e", "l3_e", "l1_b", "l2_b", "l3_b",
              "A1_e", "A2_e", "A3_e", "A1_b", "A2_b", "A3_b", "dV")
A1E, A2E, A3E, DV = 6, 7, 8, 12


class LsParams(C.Structure):
    """or_ls_params: the dev_params members the log-spherical kernels read."""
    _fields_ = [
        ("compactness", C.c_float), ("omega", C.c_float), ("gravity", C.c_float),
        ("rad_cooling_coef", C.c_float), ("B0", C.c_float), ("damping_coef", C.c_float),
        ("rad_cooling_on", C.c_int), ("damping_length", C.c_int),
    ]


def ls_params(compactness=0.0, omega=0.1, gravity=0.0, rad_cooling_coef=1.0, B0=1.0,
              damping_coef=0.002, rad_cooling_on=False, damping_length=30):
    return LsParams(compactness, omega, gravity, rad_cooling_coef, B0, damping_coef,
                    1 if rad_cooling_on else 0, damping_length)


class PtcD(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _ in PTC_FIELDS]


PTC_FIELDS_F64 = tuple((n, (np.float64 if dt == np.float32 else dt)) for n, dt in PTC_FIELDS)

_vp, _sz, _u64, _f, _d, _u32, _i = (C.c_void_p, C.c_size_t, C.c_uint64, C.c_float,
                                    C.c_double, C.c_uint32, C.c_int)
for _name, _res, _args in [
    ("or_ls_coef_f32", None, [_vp, _vp]),
    ("or_ls_coef_f64", None, [_vp, _vp]),
    ("or_ls_push_f32", _u64, [_vp, _vp, _vp, _sz, _f, _vp, _vp, _vp]),
    ("or_ls_deposit_f32", _u64, [_vp, _vp, _vp, _sz, _f, _u32, _i, _vp, _vp, _i, _vp, _vp]),
    ("or_ls_process_j_f32", None, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _f]),
    ("or_ls_axis_rho_f32", None, [_vp, _vp]),
    ("or_ls_ptc_outflow_f32", None, [_vp, _vp, _vp, _sz]),
    ("or_ls_filter_f32", None, [_vp, _vp, _vp, _vp, _vp]),
    ("or_ls_update_b_f32", None, [_vp, _vp, _vp, _vp, _f]),
    ("or_ls_update_e_f32", None, [_vp, _vp, _vp, _vp, _f]),
    ("or_ls_divs_f32", None, [_vp, _vp, _vp]),
    ("or_ls_field_boundary_f32", None, [_vp, _vp, _vp, _f]),
    ("or_ls_field_boundary_f64", None, [_vp, _vp, _vp, _f]),
    ("or_ls_update_particles_f32", _u64, [_vp, _vp, _vp, _sz, _vp, _vp, _d, _u32, _i, _i, _i,
                                          _vp, _vp, _i]),
    ("or_ls_update_particles_f64", _u64, [_vp, _vp, _vp, _sz, _vp, _vp, _d, _u32, _i, _i, _i,
                                          _vp, _vp, _i]),
    ("or_ls_update_fields_f32", None, [_vp, _vp, _vp, _vp, _d]),
    ("or_ls_update_fields_f64", None, [_vp, _vp, _vp, _vp, _d]),
]:
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def new_coef(m, dtype=np.float32):
    return [np.zeros((m.dims[1], m.dims[0]), dtype) for _ in COEF_NAMES]


def coef(m, f64=False):
    """Grid_LogSph::compute_coef (grid_log_sph.cpp:11-126)."""
    c = new_coef(m, np.float64 if f64 else np.float32)
    (lib.or_ls_coef_f64 if f64 else lib.or_ls_coef_f32)(C.byref(m), _arr(c, 13))
    return c


def ptc_struct_f64(p):
    s = PtcD()
    for name, dt in PTC_FIELDS_F64:
        a = p[name]
        assert a.dtype == dt and a.flags.c_contiguous, name
        setattr(s, name, a.ctypes.data)
    return s


def to_f64(p):
    return {k: (v.astype(np.float64) if v.dtype == np.float32 else v.copy())
            for k, v in p.items()}


def fields_to_f64(f):
    return {k: ([a.astype(np.float64) for a in v] if isinstance(v, list)
                else v.astype(np.float64)) for k, v in f.items()}


def push(m, lp, p, num, dt, F, charges, masses):
    s = ptc_struct(p)
    return lib.or_ls_push_f32(C.byref(m), C.byref(lp), C.byref(s), num, dt, _arr(F, 6),
                              _fa(charges), _fa(masses))


def deposit(m, lp, p, num, dt, step, data_interval, J, Rho, dV, charges):
    """FP32 contributions into J / Rho (float32 or float64 accumulators)."""
    acc64 = 1 if J[0].dtype == np.float64 else 0
    s = ptc_struct(p)
    return lib.or_ls_deposit_f32(C.byref(m), C.byref(lp), C.byref(s), num, dt, step,
                                 data_interval, _arr(J, 3), _arr(Rho, 8), acc64, _p(dV),
                                 _fa(charges))


def process_j(m, J, Rho, c, dt):
    lib.or_ls_process_j_f32(C.byref(m), _arr(J, 3), _arr(Rho, 8), len(Rho), _p(c[A1E]),
                            _p(c[A2E]), _p(c[DV]), dt)


def axis_rho(m, J3):
    lib.or_ls_axis_rho_f32(C.byref(m), _p(J3))


def ptc_outflow(m, lp, p, num):
    s = ptc_struct(p)
    lib.or_ls_ptc_outflow_f32(C.byref(m), C.byref(lp), C.byref(s), num)


def filter_current(m, j, tmp, A, bnd=(1, 1, 1, 1)):
    lib.or_ls_filter_f32(C.byref(m), _p(j), _p(tmp), _p(A), _fa(bnd, C.c_int, 4))


def update_b(m, lp, f, c, dt):
    fs = fields_struct(f)
    lib.or_ls_update_b_f32(C.byref(m), C.byref(lp), C.byref(fs), _arr(c, 13), dt)


def update_e(m, lp, f, c, dt):
    fs = fields_struct(f)
    lib.or_ls_update_e_f32(C.byref(m), C.byref(lp), C.byref(fs), _arr(c, 13), dt)


def compute_divs(m, f, c):
    fs = fields_struct(f)
    lib.or_ls_divs_f32(C.byref(m), C.byref(fs), _arr(c, 13))


def field_boundary(m, lp, f, omega):
    fs = fields_struct(f)
    fn = lib.or_ls_field_boundary_f64 if f["E"][0].dtype == np.float64 else \
        lib.or_ls_field_boundary_f32
    fn(C.byref(m), C.byref(lp), C.byref(fs), omega)


def update_fields(m, lp, f, c, dt):
    fs = fields_struct(f)
    fn = lib.or_ls_update_fields_f64 if f["E"][0].dtype == np.float64 else \
        lib.or_ls_update_fields_f32
    fn(C.byref(m), C.byref(lp), C.byref(fs), _arr(c, 13), dt)


def update_particles(m, lp, p, num, f, c, dt, step, data_interval, num_species,
                     current_smoothing, charges, masses, acc64=True):
    """ptc_updater_logsph::update_particles + apply_boundary. FP32 when the
    particle arrays are float32, FP64 when they are float64. Returns
    (nan_count, lost)."""
    f64 = p["p1"].dtype == np.float64
    s = ptc_struct_f64(p) if f64 else ptc_struct(p)
    fs = fields_struct(f)
    fn = lib.or_ls_update_particles_f64 if f64 else lib.or_ls_update_particles_f32
    r = fn(C.byref(m), C.byref(lp), C.byref(s), num, C.byref(fs), _arr(c, 13), dt, step,
           data_interval, num_species, current_smoothing, _fa(charges), _fa(masses),
           1 if acc64 else 0)
    return r >> 32, r & 0xFFFFFFFF


# ---------------------------------------------------------------------------
# The reference's own log-spherical code on the host (optional pin library).

_REF_PATH = os.path.join(_HERE, "_ref", "libapref_ls.so")
ref = None


def load_ref(build=True):
    global ref
    if ref is not None:
        return ref
    if not os.path.exists(_REF_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_ls.so")
        except Exception:
            return None
    if not os.path.exists(_REF_PATH):
        return None
    r = C.CDLL(_REF_PATH)
    for name, args in [
        ("ref_ls_coef", [_vp, _vp]),
        ("ref_ls_push", [_vp, _vp, _vp, _sz, _f, _vp, _vp, _vp]),
        ("ref_ls_deposit", [_vp, _vp, _vp, _sz, _f, _u32, _i, _vp, _vp, _i, _vp, _vp]),
        ("ref_ls_process_j", [_vp, _vp, _vp, _i, _vp, _f]),
        ("ref_ls_axis_rho", [_vp, _vp, _vp]),
        ("ref_ls_ptc_outflow", [_vp, _vp, _vp, _sz]),
        ("ref_ls_filter", [_vp, _vp, _vp, _vp]),
        ("ref_ls_update_fields", [_vp, _vp, _vp, _vp, _f]),
        ("ref_ls_field_boundary", [_vp, _vp, _vp, _f]),
        ("ref_ls_surface_density", [_vp, _vp, _sz, _vp, _vp]),
    ]:
        fn = getattr(r, name)
        fn.restype = None
        fn.argtypes = args
    ref = r
    return ref


def ref_coef(m):
    c = new_coef(m)
    load_ref().ref_ls_coef(C.byref(m), _arr(c, 13))
    return c


def ref_push(m, lp, p, num, dt, F, charges, masses):
    s = ptc_struct(p)
    load_ref().ref_ls_push(C.byref(m), C.byref(lp), C.byref(s), num, dt, _arr(F, 6),
                           _fa(charges), _fa(masses))


def ref_deposit(m, lp, p, num, dt, step, data_interval, J, Rho, c, charges):
    s = ptc_struct(p)
    load_ref().ref_ls_deposit(C.byref(m), C.byref(lp), C.byref(s), num, dt, step,
                              data_interval, _arr(J, 3), _arr(Rho, 8), len(Rho), _arr(c, 13),
                              _fa(charges))


def ref_process_j(m, J, Rho, c, dt):
    load_ref().ref_ls_process_j(C.byref(m), _arr(J, 3), _arr(Rho, 8), len(Rho), _arr(c, 13), dt)


def ref_axis_rho(m, J3, c):
    load_ref().ref_ls_axis_rho(C.byref(m), _p(J3), _arr(c, 13))


def ref_ptc_outflow(m, lp, p, num):
    s = ptc_struct(p)
    load_ref().ref_ls_ptc_outflow(C.byref(m), C.byref(lp), C.byref(s), num)


def ref_filter(m, j, tmp, A):
    load_ref().ref_ls_filter(C.byref(m), _p(j), _p(tmp), _p(A))


def ref_update_fields(m, lp, f, c, dt):
    fs = fields_struct(f)
    load_ref().ref_ls_update_fields(C.byref(m), C.byref(lp), C.byref(fs), _arr(c, 13), dt)


def ref_field_boundary(m, lp, f, omega):
    fs = fields_struct(f)
    load_ref().ref_ls_field_boundary(C.byref(m), C.byref(lp), C.byref(fs), omega)
