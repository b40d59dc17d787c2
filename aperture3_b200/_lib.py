"""ctypes binding of libaperture_b200.so (the C ABI in include/aperture_b200.h).

The library is the only compute path: importing this module fails loudly if
the shared object is missing or does not export the declared symbols.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaperture_b200.so")

AP_MAX_SPECIES = 8
AP_MAX_CELL = 0xFFFFFFFF

STATUS = {
    0: "AP_OK", 1: "AP_ERR_INVALID", 2: "AP_ERR_CUDA", 3: "AP_ERR_NAN",
    4: "AP_ERR_MOVED_FAR", 5: "AP_ERR_CAPACITY", 6: "AP_ERR_TIMEOUT",
    7: "AP_ERR_UNSUPPORTED", 8: "AP_ERR_NOMEM", 9: "AP_ERR_TILE",
}


class ApError(RuntimeError):
    """A nonzero ap_status. The reference reports these conditions by
    throwing from CudaSafeCall or trapping in the kernel
    (src/cuda/cudaUtility.h:34-74, ptc_updater.cu:102-109)."""

    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")


class ApMesh(C.Structure):
    _fields_ = [
        ("dims", C.c_int * 3), ("guard", C.c_int * 3),
        ("delta", C.c_float * 3), ("inv_delta", C.c_float * 3),
        ("lower", C.c_float * 3), ("sizes", C.c_float * 3),
        ("dimension", C.c_int),
    ]


class ApParams(C.Structure):
    _fields_ = [
        ("num_species", C.c_int), ("data_interval", C.c_int),
        ("current_smoothing", C.c_int), ("periodic", C.c_int * 3),
        ("charges", C.c_float * AP_MAX_SPECIES), ("masses", C.c_float * AP_MAX_SPECIES),
        ("tile", C.c_int * 2), ("chunk", C.c_int),
    ]


class ApArray(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("pitch", C.c_size_t)]


class ApFields(C.Structure):
    _fields_ = [
        ("E", ApArray * 3), ("B", ApArray * 3), ("Ebg", ApArray * 3), ("Bbg", ApArray * 3),
        ("J", ApArray * 3), ("Rho", ApArray * AP_MAX_SPECIES), ("divE", ApArray),
        ("divB", ApArray),
    ]


class ApParticles(C.Structure):
    _fields_ = [
        ("x1", C.c_void_p), ("x2", C.c_void_p), ("x3", C.c_void_p),
        ("p1", C.c_void_p), ("p2", C.c_void_p), ("p3", C.c_void_p),
        ("E", C.c_void_p), ("weight", C.c_void_p), ("cell", C.c_void_p),
        ("id", C.c_void_p), ("flag", C.c_void_p),
    ]


class ApStepStats(C.Structure):
    _fields_ = [("nan_momenta", C.c_uint64), ("moved_far", C.c_uint64),
                ("lost", C.c_uint64), ("tile_faults", C.c_uint64), ("live", C.c_uint64)]


class ApDiag(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("charge", C.c_double),
                ("field_energy", C.c_double), ("max_abs_rho", C.c_double),
                ("gauss_residual", C.c_double), ("max_abs_j", C.c_double),
                ("continuity_residual", C.c_double)]


class ApPhaseTimes(C.Structure):
    _fields_ = [("push_deposit_ms", C.c_double), ("order_ms", C.c_double),
                ("rebuild_ms", C.c_double), ("finalize_ms", C.c_double),
                ("fields_ms", C.c_double), ("sort_ms", C.c_double),
                ("push_deposit_launches", C.c_uint64)]


class ApGapParams(C.Structure):
    """ap_gap_params: SimParams::B0 for the 1D gap lab."""
    _fields_ = [("B0", C.c_float)]


class ApGrParams(C.Structure):
    """ap_gr_params: SimParams::a, omega, B0 for the 1D GR lab."""
    _fields_ = [("a", C.c_float), ("omega", C.c_float), ("B0", C.c_float)]


class ApGrTable(C.Structure):
    """ap_gr_table: the tabulated field-line data of the 1D GR lab."""
    _fields_ = [("r", C.c_void_p), ("B1", C.c_void_p), ("B3", C.c_void_p), ("jr", C.c_void_p),
                ("rho", C.c_void_p), ("theta", C.c_void_p), ("dpsidth", C.c_void_p),
                ("n", C.c_size_t)]


GR_TABLE_KEYS = ("r", "B1", "B3", "jr", "rho", "theta", "dpsidth")
GR_COEF_NAMES = ("D1", "D2", "D3", "alpha", "theta", "K1", "K1_j", "j0", "agrr", "agrf", "rho0",
                 "gamma_rr", "gamma_ff", "beta_phi", "B3B1")


class ApLogsphParams(C.Structure):
    """ap_logsph_params: the dev_params members of the log-spherical kernels."""
    _fields_ = [("compactness", C.c_float), ("omega", C.c_float), ("gravity", C.c_float),
                ("rad_cooling_coef", C.c_float), ("B0", C.c_float),
                ("damping_coef", C.c_float), ("rad_cooling_on", C.c_int),
                ("damping_length", C.c_int)]


class ApPairParams(C.Structure):
    """ap_pair_params: pair injection of the served 1D gap runs."""
    _fields_ = [("gamma_thr", C.c_float), ("free_path", C.c_float),
                ("pair_energy", C.c_float), ("enabled", C.c_int), ("seed", C.c_uint64),
                ("first_id", C.c_uint64)]


class ApPhotons(C.Structure):
    """ap_photons: photon_data (particle_data.h:68-80)."""
    _fields_ = [
        ("x1", C.c_void_p), ("x2", C.c_void_p), ("x3", C.c_void_p),
        ("p1", C.c_void_p), ("p2", C.c_void_p), ("p3", C.c_void_p),
        ("E", C.c_void_p), ("weight", C.c_void_p), ("path_left", C.c_void_p),
        ("cell", C.c_void_p), ("id", C.c_void_p), ("flag", C.c_void_p),
    ]


class ApRadParams(C.Structure):
    """ap_rad_params: radiative transfer model and parameters."""
    _fields_ = [("model", C.c_int), ("delta_t", C.c_float), ("gamma_thr", C.c_float),
                ("E_secondary", C.c_float), ("photon_path", C.c_float),
                ("r_cutoff", C.c_float), ("track_percent", C.c_float), ("e_curv", C.c_float),
                ("l_curv", C.c_float), ("BQ", C.c_float), ("omega", C.c_float),
                ("seed", C.c_uint64), ("first_photon_id", C.c_uint64),
                ("first_particle_id", C.c_uint64), ("e_min", C.c_float),
                ("ic_path", C.c_float), ("n_gamma", C.c_int), ("n_ep", C.c_int)]


class ApSpectrum(C.Structure):
    """ap_spectrum: a background photon spectrum (AP_SPEC_*)."""
    _fields_ = [("kind", C.c_int), ("p", C.c_float * 5)]


class ApRadCounts(C.Structure):
    _fields_ = [("marked", C.c_uint64), ("written", C.c_uint64), ("dropped", C.c_uint64)]


RAD_DEFAULT, RAD_PULSAR, RAD_GR1D, RAD_GAP1D = 0, 1, 2, 3
SPEC_POWER_LAW_HARD, SPEC_POWER_LAW_SOFT, SPEC_BROKEN_POWER_LAW = 0, 1, 2
SPEC_BLACK_BODY, SPEC_MONO_ENERGETIC = 3, 4

COEF_NAMES = ("l1_e", "l2_e", "l3_e", "l1_b", "l2_b", "l3_b",
              "A1_e", "A2_e", "A3_e", "A1_b", "A2_b", "A3_b", "dV")

_vp = C.c_void_p
_i = C.c_int
# name -> (restype, argtypes); every function declared in aperture_b200.h
SIGNATURES = {
    "ap_version": (C.c_char_p, []),
    "ap_status_string": (C.c_char_p, [_i]),
    "ap_ctx_create": (_i, [C.POINTER(ApMesh), C.POINTER(ApParams), C.POINTER(_vp)]),
    "ap_ctx_destroy": (_i, [_vp]),
    "ap_set_stream": (_i, [_vp, _vp]),
    "ap_set_sync": (_i, [_vp, _i]),
    "ap_sync": (_i, [_vp]),
    "ap_bind_fields": (_i, [_vp, C.POINTER(ApFields)]),
    "ap_bind_particles": (_i, [_vp, C.POINTER(ApParticles), C.c_size_t, C.c_size_t]),
    "ap_particles_modified": (_i, [_vp, C.c_size_t]),
    "ap_get_number": (_i, [_vp, C.POINTER(C.c_size_t)]),
    "ap_get_slot_range": (_i, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "ap_diagnostics_async": (_i, [_vp, _vp]),
    "ap_selftest_wait_timeout": (_i, [_vp]),
    "ap_update_particles": (_i, [_vp, C.c_double, C.c_uint32]),
    "ap_smooth_current": (_i, [_vp, C.c_uint32]),
    "ap_smooth_array": (_i, [_vp, ApArray]),
    "ap_update_fields": (_i, [_vp, C.c_double, C.c_uint32]),
    "ap_update_e_field": (_i, [_vp, C.c_double]),
    "ap_update_b_field": (_i, [_vp, C.c_double]),
    "ap_compute_divs": (_i, [_vp]),
    "ap_send_guard_cells": (_i, [_vp, ApArray]),
    "ap_send_add_guard_cells": (_i, [_vp, ApArray]),
    "ap_sort_by_cell": (_i, [_vp]),
    "ap_get_tile_order": (_i, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_uint32),
                               C.POINTER(C.c_size_t)]),
    "ap_get_stats": (_i, [_vp, C.POINTER(ApStepStats)]),
    "ap_diagnostics": (_i, [_vp, C.POINTER(ApDiag)]),
    "ap_set_profiling": (_i, [_vp, _i]),
    "ap_get_phase_times": (_i, [_vp, C.POINTER(ApPhaseTimes), _i]),
    "ap_last_error": (_i, [_vp]),
    "ap_launch_count": (C.c_uint64, [_vp]),
    "ap_ctx_create_logsph": (_i, [C.POINTER(ApMesh), C.POINTER(ApParams),
                                  C.POINTER(ApLogsphParams), C.POINTER(_vp)]),
    "ap_logsph_coef": (_i, [_vp, _i, C.POINTER(ApArray)]),
    "ap_gr_coef": (_i, [_vp, _i, C.POINTER(ApArray)]),
    "ap_ctx_create_1dgr": (_i, [C.POINTER(ApMesh), C.POINTER(ApParams), C.POINTER(ApGrParams),
                                C.POINTER(ApGrTable), C.POINTER(_vp)]),
    "ap_ctx_create_1dgap": (_i, [C.POINTER(ApMesh), C.POINTER(ApParams), C.POINTER(ApGapParams),
                                 C.POINTER(_vp)]),
    "ap_logsph_field_boundary": (_i, [_vp, C.c_double]),
    "ap_logsph_inject": (_i, [_vp, _i, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                              C.c_uint64]),
    "ap_batch_create": (_i, [C.POINTER(_vp), _i, C.POINTER(_vp)]),
    "ap_batch_set_capture": (_i, [_vp, _i]),
    "ap_batch_destroy": (_i, [_vp]),
    "ap_batch_add": (_i, [_vp, _vp]),
    "ap_batch_remove": (_i, [_vp, _vp]),
    "ap_batch_size": (_i, [_vp, C.POINTER(_i)]),
    "ap_batch_set_stream": (_i, [_vp, _vp]),
    "ap_batch_update_particles": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    "ap_batch_update_fields": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    "ap_batch_sort_by_cell": (_i, [_vp]),
    "ap_batch_sync": (_i, [_vp, C.POINTER(_i)]),
    "ap_batch_advance": (_i, [_vp, _vp, _vp, _i, _i, _i]),
    "ap_batch_autotune": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                               C.POINTER(_i)]),
    "ap_set_tile_shape": (_i, [_vp, _i, _i]),
    "ap_set_compaction": (_i, [_vp, _i]),
    "ap_set_continuity_check": (_i, [_vp, _i]),
    "ap_get_tile_shape": (_i, [_vp, C.POINTER(_i), C.POINTER(_i)]),
    "ap_set_pair_params": (_i, [_vp, C.POINTER(ApPairParams)]),
    "ap_get_pair_stats": (_i, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                               C.POINTER(C.c_uint64)]),
    "ap_inject_pairs": (_i, [_vp, C.c_double, C.c_uint32, C.POINTER(C.c_uint64),
                             C.POINTER(C.c_uint64)]),
    "ap_batch_inject_pairs": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_uint32)]),
    "ap_bind_photons": (_i, [_vp, C.POINTER(ApPhotons), C.c_size_t, C.c_size_t]),
    "ap_get_photon_number": (_i, [_vp, C.POINTER(C.c_size_t)]),
    "ap_set_rad_params": (_i, [_vp, C.POINTER(ApRadParams)]),
    "ap_emit_photons": (_i, [_vp, ApArray, C.POINTER(ApRadCounts)]),
    "ap_produce_pairs": (_i, [_vp, ApArray, C.POINTER(ApRadCounts)]),
    "ap_move_photons": (_i, [_vp, C.c_double]),
    "ap_ic_init": (_i, [_vp, C.POINTER(ApSpectrum), C.c_double, C.c_double, C.c_double, _i, _i]),
    "ap_ic_tables": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ap_update_particles_1d_noalloc": (_i, [C.POINTER(ApMesh), C.POINTER(ApParams),
                                            C.POINTER(ApParticles), C.c_size_t,
                                            C.POINTER(ApFields), C.c_double, C.c_uint32, _vp]),
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python aperture3_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is not exported
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(status, what):
    if status != 0:
        raise ApError(status, what)
    return status
