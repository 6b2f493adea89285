"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

HEADERS = glob.glob(os.path.join(ROOT, "include", "*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(ht_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "ht_version" in names and "ht_prop_D" in names
    assert len(names) >= 6


def test_library_exports_all_declared_symbols():
    from holotomocupy_b200 import _lib
    L = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"library does not export {missing}"


def test_binding_table_matches_header():
    from holotomocupy_b200 import _lib
    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_version_and_error_calls_need_no_gpu():
    from holotomocupy_b200 import _lib
    L = _lib.lib()
    assert L.ht_version() >= 100
    assert isinstance(L.ht_last_error(), bytes)


def test_bad_arguments_are_rejected_without_gpu():
    from holotomocupy_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.ht_prop_create(0, 8, 1, None, ctypes.byref(h)) == 1
    assert L.ht_prop_D(None, None, None, 1, 0, None) == 1
    assert b"null" in L.ht_last_error()


def test_new_entry_points_reject_bad_arguments_without_gpu():
    """The padded-grid, slab, chunk, shared-coefficient and probe-fit entry
    points check their arguments before touching a device."""
    from holotomocupy_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.ht_conv2d_create(100, 64, ctypes.byref(h)) == 3          # 100 is not 2^a 3^b
    assert L.ht_conv2d_run(None, None, None, None, 1, None) == 1
    assert L.ht_pad_mirror(None, None, 1, 8, 8, None) == 1
    x = ctypes.c_void_p(16)                                           # never dereferenced: the check fails first
    assert L.ht_pad_mirror(x, x, 1, 8, 7, None) == 1                  # odd width
    assert L.ht_pad_fold(x, x, 1, 7, 8, None) == 1                    # odd height
    assert L.ht_tomo_R_slab(None, None, None, 1, 1, 0, None) == 1
    assert L.ht_tomo_RT_slab(None, None, None, 1, 1, 0, 1.0, None) == 1
    assert L.ht_rec_set_data_size(None, 1.0) == 1
    assert L.ht_rec_set_shared_coefficients(None, 1) == 1
    assert L.ht_prbfit_grad(None, None, None, None, None, 1.0, None) == 1
    assert L.ht_prbfit_forms(None, None, None, None, None, None, None, 1.0, 0, None) == 1
    assert b"null" in L.ht_last_error()
