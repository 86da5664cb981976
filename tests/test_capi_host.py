"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and rejects bad arguments on the host (before any CUDA call) with
the codes include/sfemans_nl.h documents."""
import ctypes
import os
import re

import numpy as np
import pytest

import sfemans_b200 as sf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sfnl_\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = sf.lib()
    declared = _declared()
    assert len(declared) >= 23
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert L.sfnl_version().startswith(b"sfemans_nl")


def test_bindings_cover_the_header():
    # every declared entry point has a ctypes signature in the Python layer
    declared = _declared() - {"sfnl_last_error", "sfnl_version"}
    assert declared <= set(sf._SIGS), declared - set(sf._SIGS)


NULL = ctypes.c_void_p(0)


@pytest.mark.parametrize("args,code", [
    ((0, NULL, NULL, NULL, 10, 0, 6, 0, 0, NULL), -1),        # m_max = 0 (m_max_c==0 in the reference)
    ((0, NULL, NULL, NULL, -1, 4, 6, 0, 0, NULL), -1),        # np < 0
    ((0, NULL, NULL, NULL, 10, 4, 3, 0, 0, NULL), -3),        # m_max_pad < m_max
    ((0, NULL, NULL, NULL, 10, 4, 6, 5, 0, NULL), -3),        # explicit grid shorter than 2m-1
    ((7, NULL, NULL, NULL, 10, 4, 6, 0, 0, NULL), -1),        # unknown op
    ((0, NULL, NULL, NULL, 10, 4, 6, 0, 0, NULL), -1),        # null arrays with np > 0
])
def test_product_argument_errors(args, code):
    assert sf.lib().sfnl_product_f64(*args) == code
    assert sf.last_error()


def test_zero_points_is_a_no_op():
    assert sf.lib().sfnl_product_f64(0, NULL, NULL, NULL, 0, 4, 6, 0, 0, NULL) == 0


def test_fortran_signature_checks():
    L = sf.lib()
    a = np.zeros((4, 6, 2), order="F")
    p = ctypes.c_void_p(a.ctypes.data)
    # odd nb_field (fft_parallel.F90:188)
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 5, 2, 1, 5, 3, NULL) == -1
    # m_max_c == 0
    assert L.sfnl_fft_par_dot_prod_dcl(p, p, p, 4, 6, 0, 1, 5, 3, NULL) == -1
    # nb_field 4 cannot form a cross product
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 4, 2, 1, 5, 3, NULL) == -2
    # more than one Fourier rank on one GPU
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 6, 2, 2, 5, 3, NULL) == -4
    # np > nb_procs*bloc_size (the reference's buffer bound)
    assert L.sfnl_fft_par_prod_dcl(p, p, p, 4, 2, 1, 3, 3, NULL) == -2


def test_split_argument_errors():
    L = sf.lib()
    assert L.sfnl_product_split(0, NULL, NULL, NULL, 10, 4, 6, 5, NULL) == -1     # split not 2/3
    assert L.sfnl_product_split(0, NULL, NULL, NULL, 10, 4, 4, 3, NULL) == -1     # null arrays first
    a = ctypes.c_void_p(16)
    assert L.sfnl_product_split(0, a, a, a, 10, 8, 8, 3, NULL) == -3             # aliasing pad


def test_batch_argument_errors():
    L = sf.lib()
    a = ctypes.c_void_p(16)
    assert L.sfnl_cross_jvp_f64(a, a, a, a, 10, 4, 6, 0, NULL) == -1
    assert L.sfnl_mhd_vjp_f64(a, a, a, a, a, 10, 4, 6, 70000, NULL) == -1
    assert L.sfnl_mhd_jvp_f64(a, a, NULL, a, a, 10, 4, 6, 2, NULL) == -1
