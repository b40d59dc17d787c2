"""CPU oracle for photons and pair production -- TEST INFRASTRUCTURE ONLY.

Wraps ``ap_rad.c`` of ``liboracle.so`` (the restatement of the photon movers
and of ``radiative_transfer`` with the default, the pulsar lab's and the 1D
GR lab's user radiative functions), ``ap_ic.c`` (the inverse-Compton tables
of ``src/cuda/radiation/rt_ic.cu``), the pin library ``_ref/libapref_rad_gr.so``
that runs the 1D GR lab's own user radiative functions on the host and the pin library ``_ref/libapref_rad.so`` that runs
the reference's own user functions on the host (built by
``ref_build/Makefile`` when the reference tree is present), plus the photon
movers of ``_ref/libapref.so`` and ``_ref/libapref_ls.so``.

Photons are dicts of numpy arrays with the members of ``photon_data``
(``particle_data.h:68-80``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import (_HERE, _arr, _build, _p, _vp, _sz, fields_struct, lib, load_ref as _load_ref_cart,
               ptc_struct, ref_tree_present)
from . import logsph as _ls

PH_FIELDS = (
    ("x1", np.float32), ("x2", np.float32), ("x3", np.float32),
    ("p1", np.float32), ("p2", np.float32), ("p3", np.float32),
    ("E", np.float32), ("weight", np.float32), ("path_left", np.float32),
    ("cell", np.uint32), ("id", np.uint64), ("flag", np.uint32),
)

RAD_DEFAULT, RAD_PULSAR, RAD_GR1D, RAD_GAP1D = 0, 1, 2, 3
SPEC_POWER_LAW_HARD, SPEC_POWER_LAW_SOFT, SPEC_BROKEN_POWER_LAW = 0, 1, 2
SPEC_BLACK_BODY, SPEC_MONO_ENERGETIC = 3, 4


class Photons(C.Structure):
    _fields_ = [(n, C.c_void_p) for n, _ in PH_FIELDS]


class RadParams(C.Structure):
    """or_rad_params (ap_rad.h)."""
    _fields_ = [
        ("model", C.c_int), ("delta_t", C.c_float), ("gamma_thr", C.c_float),
        ("E_secondary", C.c_float), ("photon_path", C.c_float), ("r_cutoff", C.c_float),
        ("track_percent", C.c_float), ("e_curv", C.c_float), ("l_curv", C.c_float),
        ("BQ", C.c_float), ("omega", C.c_float), ("seed", C.c_uint64), ("gr", C.c_void_p),
        ("e_min", C.c_float),
    ]


class Spectrum(C.Structure):
    """or_spectrum (ap_ic.h)."""
    _fields_ = [("kind", C.c_int), ("p", C.c_float * 5)]


class IcTablesS(C.Structure):
    """or_ic_tables (ap_ic.h)."""
    _fields_ = [("n_gamma", C.c_int), ("n_ep", C.c_int), ("dep", C.c_float), ("dg", C.c_float),
                ("dlep", C.c_float), ("ic_rate", C.c_void_p), ("gg_rate", C.c_void_p),
                ("gammas", C.c_void_p), ("dNde", C.c_void_p), ("dNde_thomson", C.c_void_p)]


class RadGr(C.Structure):
    """or_rad_gr (ap_rad.h)."""
    _fields_ = [(n, C.c_void_p) for n in ("alpha", "D1", "D2", "D3", "B3B1", "gamma_rr",
                                          "gamma_ff", "beta_phi", "theta")] + [
        ("a", C.c_float), ("omega", C.c_float), ("ic", C.c_void_p)]


class RadCounts(C.Structure):
    _fields_ = [("marked", C.c_uint64), ("written", C.c_uint64), ("dropped", C.c_uint64)]


def rad_params(model=RAD_DEFAULT, delta_t=0.01, gamma_thr=20.0, E_secondary=4.0,
               photon_path=1.0, r_cutoff=4.0, track_percent=0.2, e_curv=6.4e-9, l_curv=6.0,
               BQ=1.0, omega=0.2, seed=1):
    """RadParams with the reference's SimParams defaults (sim_params.h:50-83)."""
    return RadParams(model, delta_t, gamma_thr, E_secondary, photon_path, r_cutoff,
                     track_percent, e_curv, l_curv, BQ, omega, seed, None, 1e-3)


def spectrum(kind, *p):
    s = Spectrum()
    s.kind = kind
    for k, v in enumerate(p):
        s.p[k] = v
    return s


class IcTables:
    """inverse_compton's tables for one spectrum (or_ic_init): numpy arrays
    ic_rate, gg_rate, gammas (n_gamma) and dNde, dNde_thomson (n_gamma x
    n_ep), and the steps dep, dg, dlep."""

    def __init__(self, spec, emin, emax, n0, n_gamma=600, n_ep=600):
        self.ic_rate = np.zeros(n_gamma, np.float32)
        self.gg_rate = np.zeros(n_gamma, np.float32)
        self.gammas = np.zeros(n_gamma, np.float32)
        self.dNde = np.zeros((n_gamma, n_ep), np.float32)
        self.dNde_thomson = np.zeros((n_gamma, n_ep), np.float32)
        self.s = IcTablesS(n_gamma, n_ep, 0.0, 0.0, 0.0, self.ic_rate.ctypes.data,
                           self.gg_rate.ctypes.data, self.gammas.ctypes.data,
                           self.dNde.ctypes.data, self.dNde_thomson.ctypes.data)
        lib.or_ic_init(C.byref(spec), float(emin), float(emax), float(n0), C.byref(self.s))
        self.dep, self.dg, self.dlep = self.s.dep, self.s.dg, self.s.dlep

    def rate(self, gamma):
        return lib.or_ic_rate(C.byref(self.s), float(gamma))

    def gg(self, eph):
        return lib.or_gg_rate(C.byref(self.s), float(eph))

    def photon_e(self, gamma, u):
        return lib.or_ic_photon_e(C.byref(self.s), float(gamma), float(u))


def gr1d_spectrum(e_min):
    """The 1D GR lab's background (user_rt_init, labs/1dgr/src/cuda/
    radiation/user_radiative_functions.cuh:191-203): broken_power_law(1.25,
    1.1, e_min, 1e-10, 0.1); tables over [1e-10, 0.1] with n0 = 1.5e24 /
    ic_path."""
    return spectrum(SPEC_BROKEN_POWER_LAW, 1.25, 1.1, e_min, 1e-10, 0.1)


class GrRad:
    """or_rad_gr over the 15 Grid_1dGR arrays of oracle.gr_coef and an
    IcTables (kept alive with it)."""

    NAMES = ("alpha", "D1", "D2", "D3", "B3B1", "gamma_rr", "gamma_ff", "beta_phi", "theta")

    def __init__(self, co, a, omega, ic):
        from . import GR_COEF_NAMES
        self.arrs = [np.ascontiguousarray(co[GR_COEF_NAMES.index(n)], np.float32)
                     for n in self.NAMES]
        self.ic = ic
        self.s = RadGr(*[x.ctypes.data for x in self.arrs], float(a), float(omega),
                       C.addressof(ic.s))


class GapRad:
    """or_rad_gr carrying only the tables, for the 1D gap lab's model."""

    def __init__(self, ic):
        self.ic = ic
        self.s = RadGr(*([None] * 9), 0.0, 0.0, C.addressof(ic.s))


def gap_rad_params(gap, delta_t, e_min=1e-3, track_percent=0.2, seed=1):
    rp = rad_params(model=RAD_GAP1D, delta_t=delta_t, track_percent=track_percent, seed=seed)
    rp.gr = C.addressof(gap.s)
    rp.e_min = e_min
    return rp


def move_photons_gap(m, ph, num, dt):
    s = photons_struct(ph)
    lib.or_move_photons_gap(C.byref(m), C.byref(s), num, dt)


def gr_rad_params(gr, delta_t, track_percent=0.2, seed=1):
    rp = rad_params(model=RAD_GR1D, delta_t=delta_t, track_percent=track_percent, seed=seed)
    rp.gr = C.addressof(gr.s)
    return rp


for _name, _res, _args in [
    ("or_rad_uniforms", None, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _vp]),
    ("or_move_photons_cart", None, [_vp, _vp, _sz, C.c_float, _vp]),
    ("or_move_photons_logsph", None, [_vp, _vp, _vp, _sz, C.c_float]),
    ("or_emit_photons", None, [_vp, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _vp, C.c_uint32,
                               C.c_uint64, _vp]),
    ("or_produce_pairs", None, [_vp, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _vp, C.c_uint32,
                                C.c_uint64, _vp]),
    ("or_move_photons_gr", None, [_vp, _vp, _vp, _sz, C.c_float, C.c_uint32, C.c_int]),
    ("or_move_photons_gap", None, [_vp, _vp, _sz, C.c_float]),
    ("or_ic_init", None, [_vp, C.c_double, C.c_double, C.c_double, _vp]),
    ("or_ic_rate", C.c_float, [_vp, C.c_float]),
    ("or_gg_rate", C.c_float, [_vp, C.c_float]),
    ("or_ic_photon_e", C.c_float, [_vp, C.c_float, C.c_float]),
]:
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def new_photons(cap):
    ph = {n: np.zeros(cap, dt) for n, dt in PH_FIELDS}
    ph["cell"][:] = 0xFFFFFFFF
    return ph


def copy_photons(ph):
    return {k: v.copy() for k, v in ph.items()}


def photons_struct(ph):
    s = Photons()
    for name, dt in PH_FIELDS:
        a = ph[name]
        assert a.dtype == dt and a.flags.c_contiguous, name
        setattr(s, name, a.ctypes.data)
    return s


def uniforms(seed, tag, call, ids):
    """The four build uniforms of each id (or_rad_uniforms), shape (n, 4)."""
    out = np.zeros((len(ids), 4), np.float32)
    u = (C.c_float * 4)()
    for k, i in enumerate(ids):
        lib.or_rad_uniforms(seed, tag, call, int(i), u)
        out[k] = np.frombuffer(u, np.float32)
    return out


def move_photons_cart(m, ph, num, dt, periodic):
    s = photons_struct(ph)
    lib.or_move_photons_cart(C.byref(m), C.byref(s), num, dt,
                             (C.c_int * 3)(*[int(bool(x)) for x in periodic]))


def move_photons_logsph(m, rp, ph, num, dt):
    s = photons_struct(ph)
    lib.or_move_photons_logsph(C.byref(m), C.byref(rp), C.byref(s), num, dt)


def move_photons_gr(m, gr, ph, num, dt, step, data_interval):
    s = photons_struct(ph)
    lib.or_move_photons_gr(C.byref(m), C.byref(gr.s), C.byref(s), num, dt, step, data_interval)


def emit_photons(m, rp, p, ptc_num, ph, ph_num, ph_cap, f, photon_produced, call, first_id):
    """Returns (new photon number, RadCounts)."""
    sp, sph, sf = ptc_struct(p), photons_struct(ph), fields_struct(f)
    n = C.c_size_t(ph_num)
    cnt = RadCounts()
    lib.or_emit_photons(C.byref(m), C.byref(rp), C.byref(sp), ptc_num, C.byref(sph), C.byref(n),
                        ph_cap, C.byref(sf), _p(photon_produced), call, first_id, C.byref(cnt))
    return n.value, cnt


def produce_pairs(m, rp, ph, ph_num, p, ptc_num, ptc_cap, f, pair_produced, call, first_id):
    """Returns (new particle number, RadCounts)."""
    sp, sph, sf = ptc_struct(p), photons_struct(ph), fields_struct(f)
    n = C.c_size_t(ptc_num)
    cnt = RadCounts()
    lib.or_produce_pairs(C.byref(m), C.byref(rp), C.byref(sph), ph_num, C.byref(sp), C.byref(n),
                         ptc_cap, C.byref(sf), _p(pair_produced), call, first_id, C.byref(cnt))
    return n.value, cnt


# ---------------------------------------------------------------------------
# The reference's own functions on the host (pin libraries).

_REF_PATH = os.path.join(_HERE, "_ref", "libapref_rad.so")
ref = None


def load_ref(build=True):
    """The reference's user radiative functions on the host, or None."""
    global ref
    if ref is not None:
        return ref
    if not os.path.exists(_REF_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_rad.so")
        except Exception:
            return None
    if not os.path.exists(_REF_PATH):
        return None
    r = C.CDLL(_REF_PATH)
    for name in ("ref_rad_emit_photons", "ref_rad_produce_pairs"):
        fn = getattr(r, name)
        fn.restype = C.c_int
        fn.argtypes = [_vp, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _vp, _vp, C.c_uint64, _vp]
    ref = r
    return ref


def ref_emit_photons(m, rp, p, ptc_num, ph, ph_num, ph_cap, f, photon_produced, call, first_id):
    u4 = uniforms(rp.seed, 1, call, p["id"][:ptc_num])
    sp, sph, sf = ptc_struct(p), photons_struct(ph), fields_struct(f)
    n = C.c_size_t(ph_num)
    cnt = RadCounts()
    rc = load_ref().ref_rad_emit_photons(C.byref(m), C.byref(rp), C.byref(sp), ptc_num,
                                         C.byref(sph), C.byref(n), ph_cap, C.byref(sf),
                                         _p(photon_produced), _p(u4), first_id, C.byref(cnt))
    assert rc == 0, "a user function drew more uniforms than the build gives it"
    return n.value, cnt


def ref_produce_pairs(m, rp, ph, ph_num, p, ptc_num, ptc_cap, f, pair_produced, call, first_id):
    u4 = uniforms(rp.seed, 2, call, ph["id"][:ph_num])
    sp, sph, sf = ptc_struct(p), photons_struct(ph), fields_struct(f)
    n = C.c_size_t(ptc_num)
    cnt = RadCounts()
    rc = load_ref().ref_rad_produce_pairs(C.byref(m), C.byref(rp), C.byref(sph), ph_num,
                                          C.byref(sp), C.byref(n), ptc_cap, C.byref(sf),
                                          _p(pair_produced), _p(u4), first_id, C.byref(cnt))
    assert rc == 0, "a user function drew more uniforms than the build gives it"
    return n.value, cnt


def ref_move_photons_cart(m, ph, num, dt):
    """The reference's move_photons_cart_1d / _2d (no wrap)."""
    r = _load_ref_cart()
    fn = r.ref_move_photons_cart
    fn.restype = None
    fn.argtypes = [_vp, _vp, _sz, C.c_float]
    s = photons_struct(ph)
    fn(C.byref(m), C.byref(s), num, dt)


def ref_move_photons_logsph(m, r_cutoff, ph, num, dt):
    """The reference's log-spherical move_photons (no guard clearing)."""
    r = _ls.load_ref()
    fn = r.ref_ls_move_photons
    fn.restype = None
    fn.argtypes = [_vp, C.c_float, _vp, _sz, C.c_float]
    s = photons_struct(ph)
    fn(C.byref(m), r_cutoff, C.byref(s), num, dt)


def ref_available():
    return (ref_tree_present() or os.path.exists(_REF_PATH)) and load_ref() is not None


_REF_GR_PATH = os.path.join(_HERE, "_ref", "libapref_rad_gr.so")
ref_gr = None


def load_ref_gr(build=True):
    """The 1D GR lab's own user radiative functions on the host (with the
    oracle's inverse-Compton lookups), or None."""
    global ref_gr
    if ref_gr is not None:
        return ref_gr
    if not os.path.exists(_REF_GR_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_rad_gr.so")
        except Exception:
            return None
    if not os.path.exists(_REF_GR_PATH):
        return None
    ref_gr = _rgr_lib(_REF_GR_PATH)
    return ref_gr


def _rgr_lib(path):
    r = C.CDLL(path)
    r.ref_rgr_set_e_min.restype = None
    r.ref_rgr_set_e_min.argtypes = [C.c_float]
    r.ref_gr_emit_photons.restype = C.c_int
    r.ref_gr_emit_photons.argtypes = [_vp, _vp, C.c_float, C.c_float, _vp, _sz, _vp, _vp, _sz,
                                      _vp, C.c_uint64, _vp]
    r.ref_gr_produce_pairs.restype = C.c_int
    r.ref_gr_produce_pairs.argtypes = [_vp, _vp, C.c_float, C.c_float, _vp, _sz, _vp, _vp, _sz,
                                       _vp, C.c_uint64, _vp]
    return r


_REF_GAP_RAD_PATH = os.path.join(_HERE, "_ref", "libapref_rad_gap.so")
ref_gap_rad = None


def load_ref_gap_rad(build=True):
    """The 1D gap lab's own user radiative functions on the host (the same
    driver as load_ref_gr), or None."""
    global ref_gap_rad
    if ref_gap_rad is not None:
        return ref_gap_rad
    if not os.path.exists(_REF_GAP_RAD_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_rad_gap.so")
        except Exception:
            return None
    if not os.path.exists(_REF_GAP_RAD_PATH):
        return None
    ref_gap_rad = _rgr_lib(_REF_GAP_RAD_PATH)
    return ref_gap_rad


def _ref_lib_of(rp):
    if rp.model == RAD_GAP1D:
        r = load_ref_gap_rad()
        r.ref_rgr_set_e_min(rp.e_min)
        return r
    return load_ref_gr()


def ref_gr_emit_photons(m, rp, p, ptc_num, ph, ph_num, ph_cap, call, first_id):
    """The lab's check_emit_photon / emit_photon in the build's pass, of the
    1D GR lab (rp from gr_rad_params) or of the 1D gap lab (gap_rad_params).
    Returns (new photon number, RadCounts)."""
    u4 = uniforms(rp.seed, 1, call, p["id"][:ptc_num])
    sp, sph = ptc_struct(p), photons_struct(ph)
    n = C.c_size_t(ph_num)
    cnt = RadCounts()
    rc = _ref_lib_of(rp).ref_gr_emit_photons(C.byref(m), rp.gr, rp.delta_t, rp.track_percent,
                                           C.byref(sp), ptc_num, C.byref(sph), C.byref(n),
                                           ph_cap, _p(u4), first_id, C.byref(cnt))
    assert rc == 0, "a user function drew more uniforms than the build gives it"
    return n.value, cnt


def ref_gr_produce_pairs(m, rp, ph, ph_num, p, ptc_num, ptc_cap, call, first_id):
    u4 = uniforms(rp.seed, 2, call, ph["id"][:ph_num])
    sp, sph = ptc_struct(p), photons_struct(ph)
    n = C.c_size_t(ptc_num)
    cnt = RadCounts()
    rc = _ref_lib_of(rp).ref_gr_produce_pairs(C.byref(m), rp.gr, rp.delta_t, rp.track_percent,
                                            C.byref(sph), ph_num, C.byref(sp), C.byref(n),
                                            ptc_cap, _p(u4), first_id, C.byref(cnt))
    assert rc == 0, "a user function drew more uniforms than the build gives it"
    return n.value, cnt


_REF_IC_PATH = os.path.join(_HERE, "_ref", "libapref_ic.so")
ref_ic = None


def load_ref_ic(build=True):
    """The reference's own inverse_compton::init on the host, or None."""
    global ref_ic
    if ref_ic is not None:
        return ref_ic
    if not os.path.exists(_REF_IC_PATH) and build and ref_tree_present():
        try:
            _build(os.path.join(_HERE, "ref_build"), "../_ref/libapref_ic.so")
        except Exception:
            return None
    if not os.path.exists(_REF_IC_PATH):
        return None
    r = C.CDLL(_REF_IC_PATH)
    r.ref_ic_init.restype = C.c_int
    r.ref_ic_init.argtypes = [C.c_int, _vp, C.c_float, C.c_float, C.c_double, C.c_int, C.c_int,
                              _vp, _vp, _vp, _vp, _vp, _vp]
    ref_ic = r
    return ref_ic


def ref_ic_tables(spec, emin, emax, n0, n_gamma, n_ep):
    """The tables of the reference's inverse_compton::init, as a dict."""
    out = {k: np.zeros(n_gamma, np.float32) for k in ("ic_rate", "gg_rate", "gammas")}
    out.update({k: np.zeros((n_gamma, n_ep), np.float32) for k in ("dNde", "dNde_thomson")})
    steps = np.zeros(3, np.float32)
    p = np.array(list(spec.p), np.float32)
    rc = load_ref_ic().ref_ic_init(spec.kind, p.ctypes.data, float(emin), float(emax), float(n0),
                                   n_gamma, n_ep, *[out[k].ctypes.data for k in (
                                       "ic_rate", "gg_rate", "gammas", "dNde", "dNde_thomson")],
                                   steps.ctypes.data)
    assert rc == 0
    out["dep"], out["dg"], out["dlep"] = steps
    return out
