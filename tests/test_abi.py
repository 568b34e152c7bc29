"""The C-ABI library loads and exports every entry point include/pscuda.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "pscuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "ps_synthesis" in names and "ps_adjoint" in names and "ps_plan_create" in names


def test_library_exports_every_symbol():
    from polyspec_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from polyspec_b200 import build
        build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers every declared entry point
    assert not [n for n in declared() if n not in _lib.SIGNATURES], "binding incomplete"


def test_error_strings_without_gpu():
    from polyspec_b200 import _lib
    L = _lib.lib()
    assert L.ps_error_string(0) == b"ok"
    assert L.ps_error_string(-5) == b"workspace too small"
    assert L.ps_version() >= 100


def test_invalid_arguments_are_rejected_without_touching_the_gpu():
    from polyspec_b200 import _lib
    L = _lib.lib()
    assert L.ps_plan_create(0, 10, 10, 1, 0, ctypes.byref(ctypes.c_void_p())) == -1
    assert L.ps_plan_create(16, 10, 9, 1, 0, ctypes.byref(ctypes.c_void_p())) == -1
    assert L.ps_synthesis(None, None, None, 1, 0, None, 0, None) == -1
    assert L.ps_adjoint(None, None, None, 1, 0, 1.0, None, 0, None) == -1


def test_collider_entry_points_reject_invalid_arguments_without_the_gpu():
    """The collider entry points validate pointers and sizes on the host before any launch."""
    from polyspec_b200 import _lib
    L = _lib.lib()
    nb = ctypes.c_size_t()
    assert L.ps_tau_collider_workspace_bytes(0, ctypes.byref(nb)) == -1
    assert L.ps_kint_collider_jlK(None, None, 10, 1, None, 1, None, 1, None, None) == -1
    assert L.ps_kint_collider_F(None, 1, 0, None, 1, None, 1, 2, 10, 0, 11, None, None) == -1
    assert L.ps_tau_sum_collider_diag(None, None, 1, None, None, 1, 2, 10, None, 11, None, 1, 1.0, 0.0, None, None,
                                      0, None) == -1
    assert L.ps_tau_sum_collider_general(None, None, None, None, None, None, 1, 0, 10, 2, 10, None, 11, 2, None, 1,
                                         1, 1, None, None, None, 0, None) == -1
    assert L.ps_convolve_F_collider(None, None, None, None, None, 1, 0, 10, 2, 10, None, 11, 1, 2, None, None, 1, 1,
                                    0, None, None, None, None) == -1
    assert L.ps_pF_map_complex(None, None, 10, 1, None, 3, 11, 1, 1, None, None, None, None, 1, 1, 0, 1, None,
                               None) == -1
