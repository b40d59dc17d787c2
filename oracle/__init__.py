"""CPU oracle for the Aperture3 particle update -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker. The product
(``aperture3_b200``) never imports, loads or calls anything here.

Two libraries are wrapped:

* ``liboracle.so`` (``ap_oracle.c``, ``ap_logsph.c``): a plain-C
  restatement of the reference algorithm (``src/cuda/algorithms/
  ptc_updater.cu``, ``field_solver.cu``, ``sim_environment_impl.hpp``,
  ``core/particle_base_impl.hpp``; the log-spherical files are wrapped in
  ``oracle.logsph``), FP32 literal, built with ``-ffp-contract=off``.
* ``_ref/libapref.so`` (built by ``ref_build/Makefile`` when the reference
  tree is present): the reference's own kernel bodies compiled as host code.
  It pins the restatement; it is optional at run time.

Particles are dicts of numpy arrays with the reference's SoA members
(``particle_data.h:50-61``); fields are ``(dims[1], dims[0])`` float32
arrays (row-major, no padding).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))



def _ref_tree() -> str:
    """The reference tree the pin libraries are built from: REF of
    ref_build/Makefile (APERTURE_REF in the environment overrides it)."""
    try:
        out = subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref_build"), "print-ref"],
                             check=True, capture_output=True, text=True).stdout.strip()
    except Exception:
        out = ""
    return out


REF_TREE = _ref_tree()


def ref_tree_present() -> bool:
    return bool(REF_TREE) and os.path.isdir(os.path.join(REF_TREE, "src"))
MAX_CELL = 0xFFFFFFFF

PTC_FIELDS = (
    ("x1", np.float32), ("x2", np.float32), ("x3", np.float32),
    ("p1", np.float32), ("p2", np.float32), ("p3", np.float32),
    ("E", np.float32), ("weight", np.float32),
    ("cell", np.uint32), ("id", np.uint64), ("flag", np.uint32),
)


class Mesh(C.Structure):
    """Mirror of Quadmesh (src/core/quadmesh.h:16-29)."""
    _fields_ = [
        ("dims", C.c_int * 3), ("guard", C.c_int * 3),
        ("delta", C.c_float * 3), ("inv_delta", C.c_float * 3),
        ("lower", C.c_float * 3), ("sizes", C.c_float * 3),
        ("dimension", C.c_int),
    ]


class Ptc(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _ in PTC_FIELDS]


class Fields(C.Structure):
    _fields_ = [
        ("E", C.c_void_p * 3), ("B", C.c_void_p * 3), ("Ebg", C.c_void_p * 3),
        ("Bbg", C.c_void_p * 3), ("J", C.c_void_p * 3), ("Rho", C.c_void_p * 8),
        ("divE", C.c_void_p), ("divB", C.c_void_p),
    ]


def make_mesh(N, guard, lower=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    """Grid::init (src/core/grid.cpp:31-48): delta = size / N in float,
    inv_delta = 1.0 / delta in double then stored as float."""
    N = list(N) + [1] * (3 - len(N))
    guard = list(guard) + [0] * (3 - len(guard))
    m = Mesh()
    for i in range(3):
        m.guard[i] = guard[i]
        m.dims[i] = N[i] + 2 * guard[i]
        m.lower[i] = float(np.float32(lower[i]))
        m.sizes[i] = float(np.float32(size[i]))
        d = np.float32(np.float32(size[i]) / np.float32(N[i]))
        m.delta[i] = float(d)
        m.inv_delta[i] = float(np.float32(1.0 / np.float64(d)))
    if m.dims[1] <= 1 and m.dims[2] <= 1:
        m.dimension = 1
    elif m.dims[2] <= 1:
        m.dimension = 2
    else:
        m.dimension = 3
    return m


def mesh_dict(m):
    return {
        "dims": list(m.dims), "guard": list(m.guard), "delta": list(m.delta),
        "inv_delta": list(m.inv_delta), "lower": list(m.lower),
        "sizes": list(m.sizes), "dimension": m.dimension,
    }


def mesh_from_dict(d):
    m = Mesh()
    for k in ("dims", "guard", "delta", "inv_delta", "lower", "sizes"):
        arr = getattr(m, k)
        for i in range(3):
            arr[i] = d[k][i]
    m.dimension = d["dimension"]
    return m


def _build(target_dir, target):
    subprocess.run(["make", "-s", "-C", target_dir], check=True)
    return os.path.join(target_dir, target)


def _load_oracle():
    path = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, n) for n in ("ap_oracle.c", "ap_oracle.h", "ap_logsph.c",
                                              "ap_logsph.h", "ap_gr.c", "ap_gr.h", "ap_rad.c",
                                              "ap_rad.h", "ap_ic.c", "ap_ic.h")]
    if not os.path.exists(path) or any(os.path.getmtime(path) < os.path.getmtime(s)
                                       for s in srcs):
        _build(_HERE, "liboracle.so")
    return C.CDLL(path)


lib = _load_oracle()
_u64 = C.c_uint64
_vp = C.c_void_p
_sz = C.c_size_t
for _name, _res, _args in [
    ("or_push_cart_1d", _u64, [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp]),
    ("or_push_cart_2d", _u64, [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp]),
    ("or_deposit_cart_1d", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp, _vp]),
    ("or_deposit_cart_2d", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp, _vp]),
    ("or_deposit_cart_1d_f64", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp, _vp]),
    ("or_deposit_cart_2d_f64", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp, _vp]),
    ("or_send_guard_cells", None, [_vp, _vp, _vp]),
    ("or_send_add_guard_cells", None, [_vp, _vp, _vp]),
    ("or_send_add_guard_cells_f64", None, [_vp, _vp, _vp]),
    ("or_send_particles", _sz, [_vp, _vp, _sz, _sz, _vp]),
    ("or_wrap_particles", _u64, [_vp, _vp, _sz, _vp]),
    ("or_update_e_1d", None, [_vp, _vp, C.c_float]),
    ("or_update_b_1d", None, [_vp, _vp, C.c_float]),
    ("or_compute_divs_1d", None, [_vp, _vp]),
    ("or_update_e_2d", None, [_vp, _vp, C.c_float]),
    ("or_update_b_2d", None, [_vp, _vp, C.c_float]),
    ("or_compute_divs_2d", None, [_vp, _vp]),
    ("or_update_fields", None, [_vp, _vp, C.c_double, C.c_uint32, _vp]),
    ("or_filter_1d", None, [_vp, _vp, _vp, _vp]),
    ("or_filter_2d", None, [_vp, _vp, _vp, _vp]),
    ("or_update_particles", _u64, [_vp, _vp, _sz, _vp, C.c_double, C.c_uint32, C.c_int,
                                   C.c_int, C.c_int, _vp, _vp, _vp, C.c_int]),
    ("or_stable_counting_sort", None, [_vp, _sz, C.c_uint32, _vp]),
    ("or_sort_by_cell", _sz, [_vp, _vp, _sz]),
    ("or_tile_key", C.c_uint32, [_vp, _vp, C.c_uint32]),
    ("or_tile_order", _sz, [_vp, _vp, _vp, _vp, _sz, _vp, _vp]),
    ("or_philox4x32_10", None, [_vp, _vp, _vp]),
    ("or_inject_pairs", _sz, [_vp, _sz, _sz, C.c_float, C.c_uint32, C.c_float, C.c_float,
                              C.c_float, C.c_uint64, C.c_uint64, _vp, _vp]),
    ("or_gr_coef", None, [_vp, C.c_float, C.c_float, C.c_float, _vp, _vp, _vp, _vp, _vp, _vp,
                          _vp, _sz, _vp]),
    ("or_update_ptc_1dgr", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, C.c_float,
                                  C.c_float, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("or_update_ptc_1dgr_f64", _u64, [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, C.c_float,
                                      C.c_float, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("or_filter_gr", None, [_vp, _vp, _vp, _vp, _vp]),
    ("or_update_particles_1dgr", _u64, [_vp, _vp, _sz, _vp, C.c_float, C.c_uint32, C.c_int,
                                        C.c_int, C.c_int, C.c_float, C.c_float, _vp, _vp, _vp,
                                        _vp]),
    ("or_update_e_1dgr", None, [_vp, _vp, _vp, _vp, C.c_float]),
    ("or_update_ptc_1dgap", _u64, [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp, _vp, _vp]),
    ("or_update_ptc_1dgap_f64", _u64, [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp, _vp, _vp]),
    ("or_filter_gap", None, [_vp, _vp, _vp, _vp]),
    ("or_update_particles_1dgap", _u64, [_vp, _vp, _sz, _vp, C.c_float, C.c_int, C.c_int,
                                         _vp, _vp, _vp]),
    ("or_update_fields_1dgap", None, [_vp, _vp, _vp, C.c_float, C.c_float]),
    ("or_ls_inject", _sz, [_vp, _vp, _sz, _sz, C.c_int, C.c_float, C.c_float, C.c_float,
                           C.c_uint64, C.c_uint32, C.c_uint64]),
    ("or_ls_surface_density", None, [_vp, _vp, _sz, _vp, _vp]),
]:
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _arr(ptrs, n):
    out = (C.c_void_p * n)()
    for i, a in enumerate(ptrs):
        out[i] = a.ctypes.data if a is not None else None
    return out


def _fa(vals, ctype=C.c_float, n=8):
    out = (ctype * n)()
    for i, v in enumerate(vals):
        out[i] = v
    return out


def ptc_struct(p):
    s = Ptc()
    for name, dt in PTC_FIELDS:
        a = p[name]
        assert a.dtype == dt and a.flags.c_contiguous, name
        setattr(s, name, a.ctypes.data)
    return s


def fields_struct(f):
    s = Fields()
    for key in ("E", "B", "Ebg", "Bbg", "J"):
        arr = getattr(s, key)
        for c in range(3):
            arr[c] = f[key][c].ctypes.data
    for sp, a in enumerate(f.get("Rho", [])):
        s.Rho[sp] = a.ctypes.data
    s.divE = f["divE"].ctypes.data
    s.divB = f["divB"].ctypes.data
    return s


def _ptc_view(p, lo=0):
    """Ptc struct pointing at element lo of every member."""
    s = Ptc()
    for name, dt in PTC_FIELDS:
        setattr(s, name, p[name].ctypes.data + lo * np.dtype(dt).itemsize)
    return s


def new_fields(m, num_species=2):
    shape = (m.dims[1] * m.dims[2], m.dims[0])
    z = lambda: np.zeros(shape, np.float32)  # noqa: E731
    return {
        "E": [z() for _ in range(3)], "B": [z() for _ in range(3)],
        "Ebg": [z() for _ in range(3)], "Bbg": [z() for _ in range(3)],
        "J": [z() for _ in range(3)], "Rho": [z() for _ in range(num_species)],
        "divE": z(), "divB": z(),
    }


def copy_fields(f):
    return {k: ([a.copy() for a in v] if isinstance(v, list) else v.copy())
            for k, v in f.items()}


def copy_ptc(p):
    return {k: v.copy() for k, v in p.items()}


def push(m, p, num, dt, F, charges, masses):
    fn = lib.or_push_cart_1d if m.dimension == 1 else lib.or_push_cart_2d
    s = ptc_struct(p)
    return fn(C.byref(m), C.byref(s), num, dt, _arr(F, 6), _fa(charges), _fa(masses))


def deposit(m, p, num, dt, step, data_interval, J, Rho, charges, f64=False):
    if m.dimension == 1:
        fn = lib.or_deposit_cart_1d_f64 if f64 else lib.or_deposit_cart_1d
    else:
        fn = lib.or_deposit_cart_2d_f64 if f64 else lib.or_deposit_cart_2d
    s = ptc_struct(p)
    return fn(C.byref(m), C.byref(s), num, dt, step, data_interval,
              _arr(J, 3), _arr(Rho, 8), _fa(charges))


def send_guard_cells(m, a, periodic):
    lib.or_send_guard_cells(C.byref(m), _p(a), _fa(periodic, C.c_int, 3))


def send_add_guard_cells(m, a, periodic):
    fn = lib.or_send_add_guard_cells_f64 if a.dtype == np.float64 else lib.or_send_add_guard_cells
    fn(C.byref(m), _p(a), _fa(periodic, C.c_int, 3))


def wrap_particles(m, p, num, periodic):
    s = ptc_struct(p)
    return lib.or_wrap_particles(C.byref(m), C.byref(s), num, _fa(periodic, C.c_int, 3))


def send_particles(m, p, num, cap, periodic):
    s = ptc_struct(p)
    return lib.or_send_particles(C.byref(m), C.byref(s), num, cap, _fa(periodic, C.c_int, 3))


def update_e(m, f, dt):
    fs = fields_struct(f)
    (lib.or_update_e_1d if m.dimension == 1 else lib.or_update_e_2d)(C.byref(m), C.byref(fs), dt)


def update_b(m, f, dt):
    fs = fields_struct(f)
    (lib.or_update_b_1d if m.dimension == 1 else lib.or_update_b_2d)(C.byref(m), C.byref(fs), dt)


def compute_divs(m, f):
    fs = fields_struct(f)
    (lib.or_compute_divs_1d if m.dimension == 1 else lib.or_compute_divs_2d)(C.byref(m), C.byref(fs))


def update_fields(m, f, dt, step, periodic):
    fs = fields_struct(f)
    lib.or_update_fields(C.byref(m), C.byref(fs), dt, step, _fa(periodic, C.c_int, 3))


def filter_current(m, j, tmp, bnd):
    fn = lib.or_filter_1d if m.dimension == 1 else lib.or_filter_2d
    fn(C.byref(m), _p(j), _p(tmp), _fa(bnd, C.c_int, 4))


def update_particles(m, p, num, f, dt, step, data_interval, num_species,
                     current_smoothing, charges, masses, periodic, nthreads=1):
    """ptc_updater::update_particles with the in-place wrap. Returns
    (nan_count, lost)."""
    s = ptc_struct(p)
    fs = fields_struct(f)
    r = lib.or_update_particles(C.byref(m), C.byref(s), num, C.byref(fs), dt, step,
                                data_interval, num_species, current_smoothing,
                                _fa(charges), _fa(masses), _fa(periodic, C.c_int, 3),
                                nthreads)
    return r >> 32, r & 0xFFFFFFFF


def stable_counting_sort(keys, nkeys):
    keys = np.ascontiguousarray(keys, np.uint32)
    perm = np.empty(len(keys), np.uint32)
    lib.or_stable_counting_sort(_p(keys), len(keys), nkeys, _p(perm))
    return perm


def sort_by_cell(m, p, num):
    s = ptc_struct(p)
    return lib.or_sort_by_cell(C.byref(m), C.byref(s), num)


def tile_key(m, tile, cell):
    return lib.or_tile_key(C.byref(m), _fa(tile, C.c_int, 2), cell)


def tile_order(m, tile, cell, order_in):
    order_in = np.ascontiguousarray(order_in, np.uint32)
    nt = tile_key(m, tile, MAX_CELL)
    out = np.empty(len(order_in), np.uint32)
    ts = np.empty(nt + 1, np.uint32)
    n = lib.or_tile_order(C.byref(m), _fa(tile, C.c_int, 2), _p(cell), _p(order_in),
                          len(order_in), _p(out), _p(ts))
    return out[:n], ts


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    lib.or_philox4x32_10(c, k, out)
    return list(out)


def inject_pairs(p, num, cap, dt, step, gamma_thr, free_path, pair_energy, seed, first_id):
    """Pair injection in slot order. Returns (new_num, emitted, dropped)."""
    s = ptc_struct(p)
    em, dr = C.c_uint64(), C.c_uint64()
    n = lib.or_inject_pairs(C.byref(s), num, cap, dt, step, gamma_thr, free_path, pair_energy,
                            seed, first_id, C.byref(em), C.byref(dr))
    return int(n), int(em.value), int(dr.value)


# ---------------------------------------------------------------------------
# The reference's own kernels on the host (optional pin library).

_REF_PATH = os.path.join(_HERE, "_ref", "libapref.so")
ref = None


def load_ref(build=True):
    """Load (building if the reference tree is present) the pin library."""
    global ref
    if ref is not None:
        return ref
    if not os.path.exists(_REF_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref.so")
        except Exception:
            return None
    if not os.path.exists(_REF_PATH):
        return None
    r = C.CDLL(_REF_PATH)
    for name, args in [
        ("ref_push", [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp]),
        ("ref_deposit", [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp, C.c_int, _vp]),
        ("ref_update_e", [_vp, _vp, _vp, _vp, _vp, C.c_float]),
        ("ref_update_b", [_vp, _vp, _vp, _vp, C.c_float]),
        ("ref_compute_divs", [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
        ("ref_filter", [_vp, _vp, _vp, _vp]),
    ]:
        fn = getattr(r, name)
        fn.restype = None
        fn.argtypes = args
    ref = r
    return ref


def ref_push(m, p, num, dt, F, charges, masses):
    s = ptc_struct(p)
    load_ref().ref_push(C.byref(m), C.byref(s), num, dt, _arr(F, 6), _fa(charges), _fa(masses))


def ref_deposit(m, p, num, dt, step, data_interval, J, Rho, charges):
    s = ptc_struct(p)
    load_ref().ref_deposit(C.byref(m), C.byref(s), num, dt, step, data_interval,
                           _arr(J, 3), _arr(Rho, 8), len(Rho), _fa(charges))


def ref_update_e(m, f, dt):
    load_ref().ref_update_e(C.byref(m), _arr(f["E"], 3), _arr(f["B"], 3), _arr(f["Bbg"], 3),
                            _arr(f["J"], 3), dt)


def ref_update_b(m, f, dt):
    load_ref().ref_update_b(C.byref(m), _arr(f["E"], 3), _arr(f["Ebg"], 3), _arr(f["B"], 3), dt)


def ref_compute_divs(m, f):
    load_ref().ref_compute_divs(C.byref(m), _arr(f["E"], 3), _arr(f["B"], 3), _arr(f["Ebg"], 3),
                                _arr(f["Bbg"], 3), _p(f["divE"]), _p(f["divB"]))


def ref_filter(m, j, tmp, bnd):
    load_ref().ref_filter(C.byref(m), _p(j), _p(tmp), _fa(bnd, C.c_int, 4))


# ---------------------------------------------------------------------------
# The reference's own push / deposit kernels on all host threads (timing
# build, oracle/_ref/libapref_mt.so): the CPU baseline of the benchmark.

_REF_MT_PATH = os.path.join(_HERE, "_ref", "libapref_mt.so")
ref_mt = None


def load_ref_mt(build=True):
    """Load (building if the reference tree is present) the threaded
    reference library, or None when it is not available."""
    global ref_mt
    if ref_mt is not None:
        return ref_mt
    if not os.path.exists(_REF_MT_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_mt.so")
        except Exception:
            return None
    if not os.path.exists(_REF_MT_PATH):
        return None
    r = C.CDLL(_REF_MT_PATH)
    r.ref_push_mt.restype = None
    r.ref_push_mt.argtypes = [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp, C.c_int]
    r.ref_deposit_mt.restype = None
    r.ref_deposit_mt.argtypes = [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp, _vp,
                                 C.c_int, _vp, C.c_int]
    ref_mt = r
    return ref_mt


def ref_update_particles_mt(m, p, num, f, dt, step, data_interval, num_species, charges,
                            masses, periodic, nthreads):
    """ptc_updater::update_particles (ptc_updater.cu:748-841) with the
    reference's push and deposit kernels (ptc_updater.cu:78-141, 295-386)
    on nthreads host threads, then the guard fold and in-place wrap of this
    module (sim_environment_impl.hpp:274-448)."""
    r = load_ref_mt()
    for c in range(3):
        f["J"][c][:] = 0
    for s in range(num_species):
        f["Rho"][s][:] = 0
    if num:
        s = ptc_struct(p)
        F = [f["E"][0], f["E"][1], f["E"][2], f["B"][0], f["B"][1], f["B"][2]]
        r.ref_push_mt(C.byref(m), C.byref(s), num, np.float32(dt), _arr(F, 6), _fa(charges),
                      _fa(masses), nthreads)
        r.ref_deposit_mt(C.byref(m), C.byref(s), num, np.float32(dt), step, data_interval,
                         _arr(f["J"], 3), _arr(f["Rho"][:num_species], 8), num_species,
                         _fa(charges), nthreads)
    for c in range(3):
        send_add_guard_cells(m, f["J"][c], periodic)
    if (step + 1) % data_interval == 0:
        for s in range(num_species):
            send_add_guard_cells(m, f["Rho"][s], periodic)
    return wrap_particles(m, p, num, periodic)



# ---------------------------------------------------------------------------
# 1D GR lab (ap_gr.c: grid_1dgr.cpp, ptc_updater_1dgr.cu, field_solver_1dgr.cu).

GR_NCOEF = 15
GR_COEF_NAMES = ("D1", "D2", "D3", "alpha", "theta", "K1", "K1_j", "j0", "agrr", "agrf", "rho0",
                 "gamma_rr", "gamma_ff", "beta_phi", "B3B1")
GR_TABLE_KEYS = ("r", "B1", "B3", "jr", "rho", "theta", "dpsidth")


def gr_coef(m, a, omega, B0, table):
    """Grid_1dGR::compute_coef from the tabulated arrays; returns the 15
    coefficient arrays (float32, dims[0] each) in mesh_ptrs order."""
    cols = [np.ascontiguousarray(table[k], dtype=np.float32) for k in GR_TABLE_KEYS]
    out = [np.zeros(m.dims[0], np.float32) for _ in range(GR_NCOEF)]
    lib.or_gr_coef(C.byref(m), np.float32(a), np.float32(omega), np.float32(B0),
                   *[_p(c) for c in cols], len(cols[0]), _arr(out, GR_NCOEF))
    return out


def update_ptc_1dgr(m, p, num, dt, step, data_interval, a, omega, E3, co, J1, Rho, charges,
                    masses, f64=False):
    s = ptc_struct(p)
    fn = lib.or_update_ptc_1dgr_f64 if f64 else lib.or_update_ptc_1dgr
    return fn(C.byref(m), C.byref(s), num, np.float32(dt), int(step), int(data_interval),
              np.float32(a), np.float32(omega), _p(E3), _arr(co, GR_NCOEF), _p(J1),
              _arr(Rho, 8), _fa(charges), _fa(masses))


def filter_gr(m, j, tmp, k1, bnd):
    lib.or_filter_gr(C.byref(m), _p(j), _p(tmp), _p(k1), _fa(bnd, C.c_int, 2))


def update_particles_1dgr(m, p, num, f, dt, step, data_interval, smoothing, num_species, a,
                          omega, co, charges, masses, bnd):
    s = ptc_struct(p)
    fs = fields_struct(f)
    return lib.or_update_particles_1dgr(C.byref(m), C.byref(s), num, C.byref(fs),
                                        np.float32(dt), int(step), int(data_interval),
                                        int(smoothing), int(num_species), np.float32(a),
                                        np.float32(omega), _arr(co, GR_NCOEF), _fa(charges),
                                        _fa(masses), _fa(bnd, C.c_int, 2))


def update_e_1dgr(m, E1, J1, j0, dt):
    lib.or_update_e_1dgr(C.byref(m), _p(E1), _p(J1), _p(j0), np.float32(dt))


# ---------------------------------------------------------------------------
# 1D gap lab (ptc_updater_1dgap.cu, field_solver_1dgap.cu).

def update_ptc_1dgap(m, p, num, dt, E3, J1, Rho, charges, masses, f64=False):
    """update_ptc_1dgap on slots [0, num): float adds into J1 / Rho, or
    double adds of the same float contributions (f64). Returns the count of
    moves of more than one cell."""
    s = ptc_struct(p)
    fn = lib.or_update_ptc_1dgap_f64 if f64 else lib.or_update_ptc_1dgap
    return fn(C.byref(m), C.byref(s), num, np.float32(dt), _p(E3), _p(J1), _arr(Rho, 8),
              _fa(charges), _fa(masses))


def filter_gap(m, j, tmp, bnd):
    lib.or_filter_gap(C.byref(m), _p(j), _p(tmp), _fa(bnd, C.c_int, 2))


def update_particles_1dgap(m, p, num, f, dt, smoothing, num_species, charges, masses, bnd):
    s = ptc_struct(p)
    fs = fields_struct(f)
    return lib.or_update_particles_1dgap(C.byref(m), C.byref(s), num, C.byref(fs),
                                         np.float32(dt), smoothing, num_species, _fa(charges),
                                         _fa(masses), _fa(bnd, C.c_int, 2))


def update_fields_1dgap(m, E1, J1, B0, dt):
    lib.or_update_fields_1dgap(C.byref(m), _p(E1), _p(J1), np.float32(B0), np.float32(dt))


_REF_GAP_PATH = os.path.join(_HERE, "_ref", "libapref_gap.so")
ref_gap = None


def load_ref_gap(build=True):
    """The 1D gap lab's own kernels on the host (pin library), or None."""
    global ref_gap
    if ref_gap is not None:
        return ref_gap
    if not os.path.exists(_REF_GAP_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_gap.so")
        except Exception:
            return None
    if not os.path.exists(_REF_GAP_PATH):
        return None
    r = C.CDLL(_REF_GAP_PATH)
    r.ref_gap_push_deposit.restype = None
    r.ref_gap_push_deposit.argtypes = [_vp, _vp, _sz, C.c_float, _vp, _vp, _vp, C.c_int, _vp,
                                       _vp]
    r.ref_gap_filter.restype = None
    r.ref_gap_filter.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int]
    r.ref_gap_update_e.restype = None
    r.ref_gap_update_e.argtypes = [_vp, _vp, _vp, C.c_float, C.c_float]
    r.ref_gap_move_photons.restype = None
    r.ref_gap_move_photons.argtypes = [_vp, _vp, _sz, C.c_float, C.c_uint32]
    ref_gap = r
    return ref_gap



_REF_GR_PATH = os.path.join(_HERE, "_ref", "libapref_gr.so")
ref_gr = None


def load_ref_gr(build=True):
    """The 1D GR lab's own kernels and Grid_1dGR::compute_coef on the host
    (pin library), or None."""
    global ref_gr
    if ref_gr is not None:
        return ref_gr
    if not os.path.exists(_REF_GR_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_gr.so")
        except Exception:
            return None
    if not os.path.exists(_REF_GR_PATH):
        return None
    r = C.CDLL(_REF_GR_PATH)
    r.ref_gr_coef.restype = None
    r.ref_gr_coef.argtypes = [_vp, C.c_float, C.c_float, C.c_float, _vp, _vp, _vp, _vp, _vp, _vp,
                              _vp, _sz, _vp]
    r.ref_gr_push.restype = None
    r.ref_gr_push.argtypes = [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, C.c_float,
                              C.c_float, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp]
    r.ref_gr_filter.restype = None
    r.ref_gr_filter.argtypes = [_vp, _vp, _vp, _vp, C.c_int, C.c_int]
    r.ref_gr_update_e.restype = None
    r.ref_gr_update_e.argtypes = [_vp, _vp, _vp, _vp, C.c_float]
    r.ref_gr_move_photons.restype = None
    r.ref_gr_move_photons.argtypes = [_vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int, _vp]
    ref_gr = r
    return ref_gr


def ls_inject(m, p, num, cap, inj, p1, w, q_e, seed, call, first_id):
    """Log-spherical surface injection (build semantics, ap_oracle.h);
    returns the new number."""
    s = ptc_struct(p)
    return lib.or_ls_inject(C.byref(m), C.byref(s), num, cap, inj, np.float32(p1),
                            np.float32(w), np.float32(q_e), seed, call, first_id)


def ls_surface_density(m, p, num):
    red = m.dims[1] - 2 * m.guard[1]
    se, sp = np.zeros(red), np.zeros(red)
    s = ptc_struct(p)
    lib.or_ls_surface_density(C.byref(m), C.byref(s), num, _p(se), _p(sp))
    return se, sp
