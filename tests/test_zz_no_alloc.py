"""sfnl_cross_f64_noalloc: the cross product for callers that cannot allocate
device memory (their GPU memory belongs to their own pool or to another
framework, or cudaMalloc's implicit synchronisation is not acceptable in
their time loop).

Its result must equal the allocating entry point's (sfnl_cross_f64) and the
long-double oracle's within the FP64 tolerance of the other parity tests, on
two calls in a row (the first call sets up the library's static table, the
second reuses it), also when consecutive calls on one stream change m_max
(each change rewrites the table the previous kernel read), and sizes beyond
the static table must be refused.  The file is collected last so that a run
stopping at its first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _run(fn, V1, V2, npts, m, pad):
    import torch

    a, b = sf.to_device(V1), sf.to_device(V2)
    out = sf.fortran_empty(npts, 6, m)
    out.fill_(np.nan)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(out.data_ptr()), npts, m, pad, st)
    assert rc == 0, sf.last_error()
    torch.cuda.synchronize()
    return sf.to_host(out)


@pytest.mark.parametrize("npts,m", [(1000, 16), (257, 64), (33, 5)])
def test_noalloc_matches_the_allocating_entry_point_on_two_calls(npts, m):
    pad = 3 * m // 2
    L = sf.lib()
    V1 = R.synthetic_field(npts, 6, m, 0.2, 71)
    V2 = R.synthetic_field(npts, 6, m, 0.2, 72)
    ref = _run(L.sfnl_cross_f64, V1, V2, npts, m, pad)
    orc = R.c_oracle("cross", V1, V2, pad)
    first = _run(L.sfnl_cross_f64_noalloc, V1, V2, npts, m, pad)
    second = _run(L.sfnl_cross_f64_noalloc, V1, V2, npts, m, pad)
    assert R.rel_l2(first, ref) <= FP64_TOL
    assert R.rel_l2(second, ref) <= FP64_TOL
    assert R.rel_l2(first, orc) <= FP64_TOL
    assert R.rel_l2(second, orc) <= FP64_TOL


def test_noalloc_alternating_m_on_one_stream():
    # m = 16, 64, 16, 7, 64: every change of m rewrites the static table after the previous call's
    # kernel was queued on the same stream; each result is checked against the oracle.
    L = sf.lib()
    npts = 301
    cases = {}
    for m in (16, 64, 7):
        V1 = R.synthetic_field(npts, 6, m, 0.15, 90 + m)
        V2 = R.synthetic_field(npts, 6, m, 0.15, 190 + m)
        cases[m] = (V1, V2, R.c_oracle("cross", V1, V2, 3 * m // 2))
    import torch

    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    runs = []
    for m in (16, 64, 16, 7, 64):  # queued back to back, one synchronisation at the end
        V1, V2, orc = cases[m]
        a, b = sf.to_device(V1), sf.to_device(V2)
        out = sf.fortran_empty(npts, 6, m)
        out.fill_(np.nan)
        rc = L.sfnl_cross_f64_noalloc(P(a), P(b), P(out), npts, m, 3 * m // 2, st)
        assert rc == 0, sf.last_error()
        runs.append((m, a, b, out, orc))
    torch.cuda.synchronize()
    for m, _, _, out, orc in runs:
        assert R.rel_l2(sf.to_host(out), orc) <= FP64_TOL, m


def test_noalloc_refuses_sizes_beyond_its_table():
    L = sf.lib()
    a = ctypes.c_void_p(16)
    rc = L.sfnl_cross_f64_noalloc(a, a, a, 10, 65, 97, None)
    assert rc == -4 and "64" in sf.last_error()
    assert L.sfnl_cross_f64_noalloc(a, a, a, 10, 8, 8, None) == -3  # aliasing pad
