"""The C-ABI library loads and exports every function include/aperture_b200.h
declares; the ctypes binding covers them all. No device calls."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aperture_b200.h")


def declared():
    text = open(HEADER).read()
    return set(re.findall(r"AP_API\s+[\w\s\*]+?\b(ap_\w+)\s*\(", text))


def test_header_declares_entry_points():
    names = declared()
    for n in ("ap_ctx_create", "ap_update_particles", "ap_update_fields", "ap_sort_by_cell",
              "ap_send_guard_cells", "ap_send_add_guard_cells", "ap_diagnostics"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from aperture3_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert declared() == set(_lib.SIGNATURES), declared() ^ set(_lib.SIGNATURES)


def test_status_strings_and_version():
    from aperture3_b200 import _lib
    lib = _lib.lib()
    assert b"sm_100a" in lib.ap_version()
    for s in range(10):
        assert lib.ap_status_string(s)
    assert lib.ap_status_string(0) == b"ok"


def test_struct_layouts_match_header():
    """ap_mesh has the Quadmesh layout; ap_params/ap_fields sizes as the header."""
    from aperture3_b200._lib import ApFields, ApMesh, ApParams, ApParticles
    assert C.sizeof(ApMesh) == 4 * (3 + 3 + 3 + 3 + 3 + 3 + 1)
    assert C.sizeof(ApParams) == 4 * (1 + 1 + 1 + 3 + 8 + 8 + 2 + 1)
    assert C.sizeof(ApParticles) == 8 * 11
    assert C.sizeof(ApFields) == 16 * (3 * 5 + 8 + 2)
    from aperture3_b200._lib import ApRadParams, ApSpectrum
    # model, 10 floats, padding, 3 x uint64, e_min, ic_path, n_gamma, n_ep
    assert C.sizeof(ApRadParams) == 4 + 40 + 4 + 24 + 16
    assert C.sizeof(ApSpectrum) == 4 + 20


def test_invalid_arguments_are_rejected_without_a_device():
    from aperture3_b200 import _lib
    lib = _lib.lib()
    assert lib.ap_ctx_create(None, None, None) == 1
    assert lib.ap_update_particles(None, 0.1, 0) == 1
    assert lib.ap_ctx_destroy(None) == 1
