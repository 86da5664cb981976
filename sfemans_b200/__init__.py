"""sfemans_b200 -- B200 pseudo-spectral nonlinear terms of SFEMaNS.

Python host layer over the C-ABI library ``_lib/libsfemans_nl.so``
(include/sfemans_nl.h).  It mirrors the reference's MODULE fft_parallele
(SOURCES/POST_PROCESSING/fft_parallel.F90, PUBLIC list :8-17) for the three
dealiased products, with the same names, argument order and meaning:

    FFT_PAR_CROSS_PROD_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_PAR_DOT_PROD_DCL  (communicator, V1_in, V2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_PAR_PROD_DCL      (communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None)

Arrays are Fortran-ordered (np, nslot, m): numpy arrays in host memory
(copied through the library's host entry points) or CUDA tensors with
Fortran strides (1, np, np*nslot) (see :func:`fortran_empty`).  A non-zero
status of the library raises :class:`SfnlError` -- the reference prints
``BUG in FFT_PAR_...`` and STOPs (fft_parallel.F90:188-191).

There is no CPU fallback: every call goes through the CUDA library, and
importing the bindings fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsfemans_nl.so")

OP_CROSS, OP_DOT, OP_PROD = 0, 1, 2
ALGO_AUTO, ALGO_GRID, ALGO_FAST = 0, 1, 2
SPLIT_BF16X2, SPLIT_BF16X3 = 2, 3

ERRORS = {
    0: "OK", -1: "SFNL_ERR_ARG", -2: "SFNL_ERR_SHAPE", -3: "SFNL_ERR_ALIAS", -4: "SFNL_ERR_UNSUPPORTED",
    -5: "SFNL_ERR_CUDA", -6: "SFNL_ERR_NONFINITE", -7: "SFNL_ERR_ALLOC",
}


class SfnlError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_SIGS = {
    "sfnl_cross_f64": [_P, _P, _P, _L, _I, _I, _P],
    "sfnl_dot_f64": [_P, _P, _P, _L, _I, _I, _P],
    "sfnl_prod_f64": [_P, _P, _P, _L, _I, _I, _P],
    "sfnl_product_f64": [_I, _P, _P, _P, _L, _I, _I, _I, _I, _P],
    "sfnl_cross_f64_noalloc": [_P, _P, _P, _L, _I, _I, _P],
    "sfnl_bundle_mhd_f64": [_P] * 9 + [_L, _I, _I, _I, _P],
    "sfnl_cross_jvp_f64": [_P, _P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_cross_vjp_f64": [_P, _P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_mhd_jvp_f64": [_P, _P, _P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_mhd_vjp_f64": [_P, _P, _P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_product_split": [_I, _P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_bundle_mhd_split": [_P] * 9 + [_L, _I, _I, _I, _P],
    "sfnl_mhd_jvp_split": [_P, _P, _P, _P, _P, _L, _I, _I, _I, _I, _P],
    "sfnl_mhd_vjp_split": [_P, _P, _P, _P, _P, _L, _I, _I, _I, _I, _P],
    "sfnl_fft_par_cross_prod_dcl": [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P],
    "sfnl_fft_par_dot_prod_dcl": [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P],
    "sfnl_fft_par_prod_dcl": [_P, _P, _P, _I, _I, _I, _I, _I, _P],
    "sfnl_product_f64_host": [_I, _P, _P, _P, _L, _I, _I, _I],
    "sfnl_bundle_mhd_host": [_P] * 9 + [_L, _I, _I, _I],
    "sfnl_set_check_finite": [_I],
    "sfnl_finalize": [],
    "sfnl_last_host_timing": [_P],
}


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"CUDA library missing: {LIB_PATH} (run `python -m sfemans_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.sfnl_last_error.restype = ctypes.c_char_p
        L.sfnl_last_error.argtypes = []
        L.sfnl_version.restype = ctypes.c_char_p
        L.sfnl_version.argtypes = []
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise SfnlError(rc, lib().sfnl_last_error().decode())


def last_error() -> str:
    return lib().sfnl_last_error().decode()


# ----------------------------------------------------------------------------
# tensor helpers
# ----------------------------------------------------------------------------
def fortran_empty(npts: int, nslot: int, m: int, k: int | None = None, device="cuda", dtype=None):
    """Uninitialised CUDA tensor of shape (np, nslot, m[, k]) in Fortran order."""
    import torch

    dtype = dtype or torch.float64
    if k is None:
        return torch.empty((m, nslot, npts), device=device, dtype=dtype).permute(2, 1, 0)
    return torch.empty((k, m, nslot, npts), device=device, dtype=dtype).permute(3, 2, 1, 0)


def to_device(a, device="cuda"):
    """numpy Fortran array (np, nslot, m[, k]) -> CUDA tensor with the same Fortran layout."""
    import numpy as np
    import torch

    a = np.asfortranarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(device)
    return t.permute(*reversed(range(t.dim())))


def to_host(t):
    """CUDA tensor in Fortran layout -> numpy Fortran array."""
    import numpy as np

    return np.asfortranarray(t.permute(*reversed(range(t.dim()))).contiguous().cpu().numpy().T)


def _is_fortran(t) -> bool:
    expect, s = [], 1
    for d in t.shape:
        expect.append(s)
        s *= d
    return t.is_cuda and t.dtype.itemsize == 8 and (t.numel() == 0 or list(t.stride()) == expect
                                                   or all(st == e for st, e, d in zip(t.stride(), expect, t.shape) if d > 1))


def _dptr(t, what):
    if t is None:
        return None
    if not _is_fortran(t):
        raise ValueError(f"{what}: expected a float64 CUDA tensor in Fortran order (np, nslot, m[, k])")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


# ----------------------------------------------------------------------------
# device-tensor API
# ----------------------------------------------------------------------------
def product(op: int, a, b, out=None, m_max_pad: int | None = None, n_theta: int = 0, algo: int = ALGO_AUTO,
            split: int | None = None, stream=None):
    """Dealiased product of two Fortran-layout CUDA tensors (op: 0 cross, 1 dot, 2 prod)."""
    npts, nsl, m = a.shape
    if m_max_pad is None:
        m_max_pad = 3 * m // 2
    if out is None:
        out = fortran_empty(npts, 6 if op == OP_CROSS else 2, m, device=a.device)
    if split is None:
        _check(lib().sfnl_product_f64(op, _dptr(a, "a"), _dptr(b, "b"), _dptr(out, "out"), npts, m, m_max_pad,
                                      n_theta, algo, _stream(stream)))
    else:
        if n_theta:
            raise ValueError("split forms pick their own grid")
        _check(lib().sfnl_product_split(op, _dptr(a, "a"), _dptr(b, "b"), _dptr(out, "out"), npts, m, m_max_pad,
                                        split, _stream(stream)))
    return out


def bundle_mhd(u, w, b, j, gradt, m_max_pad: int | None = None, outs=None, algo: int = ALGO_AUTO,
               split: int | None = None, stream=None):
    """(u x w, u x b, j x b, u . gradT) in one launch."""
    npts, _, m = u.shape
    if m_max_pad is None:
        m_max_pad = 3 * m // 2
    if outs is None:
        outs = tuple(fortran_empty(npts, 6, m, device=u.device) for _ in range(3)) + (
            fortran_empty(npts, 2, m, device=u.device),)
    ptrs = [_dptr(x, n) for x, n in zip((u, w, b, j, gradt) + tuple(outs),
                                          ("u", "w", "b", "j", "gradt", "uxw", "uxb", "jxb", "ugradt"))]
    if split is None:
        _check(lib().sfnl_bundle_mhd_f64(*ptrs, npts, m, m_max_pad, algo, _stream(stream)))
    else:
        _check(lib().sfnl_bundle_mhd_split(*ptrs, npts, m, m_max_pad, split, _stream(stream)))
    return outs


def _linear(fn, base, x, nout_slots, m_max_pad, out, stream, split=None):
    npts, _, m = base[0].shape
    k = x.shape[3] if x.dim() == 4 else 1
    if m_max_pad is None:
        m_max_pad = 3 * m // 2
    if out is None:
        out = fortran_empty(npts, nout_slots, m, k, device=x.device)
    args = [_dptr(t, "base") for t in base] + [_dptr(x, "x"), _dptr(out, "out"), npts, m, m_max_pad, k]
    if split is not None:
        args.append(split)
    _check(fn(*args, _stream(stream)))
    return out


def cross_jvp(u, w, tan, m_max_pad=None, out=None, stream=None):
    """du x w + u x dw for tangents tan = (du, dw): (np, 12, m[, k]) -> (np, 6, m[, k])."""
    return _linear(lib().sfnl_cross_jvp_f64, (u, w), tan, 6, m_max_pad, out, stream)


def cross_vjp(u, w, cot, m_max_pad=None, out=None, stream=None):
    """Transpose of :func:`cross_jvp`: (np, 6, m[, k]) -> (np, 12, m[, k])."""
    return _linear(lib().sfnl_cross_vjp_f64, (u, w), cot, 12, m_max_pad, out, stream)


def mhd_jvp(u, w, b, tan, m_max_pad=None, out=None, split=None, stream=None):
    """(du x w + u x dw, du x b + u x db): (np, 18, m[, k]) -> (np, 12, m[, k])."""
    fn = lib().sfnl_mhd_jvp_f64 if split is None else lib().sfnl_mhd_jvp_split
    return _linear(fn, (u, w, b), tan, 12, m_max_pad, out, stream, split)


def mhd_vjp(u, w, b, cot, m_max_pad=None, out=None, split=None, stream=None):
    """Transpose of :func:`mhd_jvp`: (np, 12, m[, k]) -> (np, 18, m[, k])."""
    fn = lib().sfnl_mhd_vjp_f64 if split is None else lib().sfnl_mhd_vjp_split
    return _linear(fn, (u, w, b), cot, 18, m_max_pad, out, stream, split)


def set_check_finite(on: bool):
    _check(lib().sfnl_set_check_finite(1 if on else 0))


def finalize():
    _check(lib().sfnl_finalize())


# ----------------------------------------------------------------------------
# reference-named mirror of MODULE fft_parallele
# ----------------------------------------------------------------------------
def _host_ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def _fortran_call(kind, communicator, x, y, out, nb_procs, bloc_size, m_max_pad, temps):
    import numpy as np

    if communicator is not None:
        from .parallel import fft_par_distributed

        return fft_par_distributed(kind, communicator, x, y, out, nb_procs, bloc_size, m_max_pad, temps)
    if hasattr(x, "is_cuda"):
        op = {"cross": OP_CROSS, "dot": OP_DOT, "prod": OP_PROD}[kind]
        if nb_procs != 1:
            raise SfnlError(-4, "one GPU holds all modes: nb_procs must be 1")
        if x.shape[0] > nb_procs * bloc_size:
            raise SfnlError(-2, "np > nb_procs*bloc_size")
        product(op, x, y, out=out, m_max_pad=m_max_pad)
        if temps is not None:
            temps[:] = 0.0
        return out
    for arr in (x, y, out):
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.flags.f_contiguous):
            raise ValueError("host arrays must be float64 and Fortran-contiguous")
    t3 = np.zeros(3) if temps is None else temps
    npts, nf, mc = x.shape
    L = lib()
    if kind == "cross":
        rc = L.sfnl_fft_par_cross_prod_dcl(_host_ptr(x), _host_ptr(y), _host_ptr(out), npts, nf, mc, nb_procs,
                                           bloc_size, m_max_pad, _host_ptr(t3))
    elif kind == "dot":
        rc = L.sfnl_fft_par_dot_prod_dcl(_host_ptr(x), _host_ptr(y), _host_ptr(out), npts, nf, mc, nb_procs,
                                         bloc_size, m_max_pad, _host_ptr(t3))
    else:
        rc = L.sfnl_fft_par_prod_dcl(_host_ptr(x), _host_ptr(y), _host_ptr(out), npts, mc, nb_procs, bloc_size,
                                     m_max_pad, _host_ptr(t3))
    _check(rc)
    return out


def FFT_PAR_CROSS_PROD_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps=None):
    """V_out = V1_in x V2_in, dealiased (fft_parallel.F90:147-328)."""
    return _fortran_call("cross", communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps)


def FFT_PAR_DOT_PROD_DCL(communicator, V1_in, V2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None):
    """c_out = V1_in . V2_in, dealiased (fft_parallel.F90:330-500)."""
    return _fortran_call("dot", communicator, V1_in, V2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)


def FFT_PAR_PROD_DCL(communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None):
    """c_out = c1_in * c2_in, dealiased (fft_parallel.F90:502-665)."""
    return _fortran_call("prod", communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)
