"""sfemans_b200 -- B200 pseudo-spectral nonlinear terms of SFEMaNS.

Python host layer over the C-ABI library ``_lib/libsfemans_nl.so``
(include/sfemans_nl.h).  It mirrors the reference's MODULE fft_parallele
(SOURCES/POST_PROCESSING/fft_parallel.F90, PUBLIC list :8-17) for the
dealiased products, with the same names, argument order and meaning:

    FFT_PAR_CROSS_PROD_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_PAR_DOT_PROD_DCL  (communicator, V1_in, V2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_PAR_PROD_DCL      (communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_PAR_DIV_DCL       (communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_SCALAR_VECT_DCL   (communicator, V1_in, V2_in, V_out, pb, nb_procs, bloc_size, m_max_pad, temps=None)
    FFT_TENSOR_DCL        (communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps=None,
                           opt_tension=None)
    FFT_PAR_REAL          (communicator, V1_in, V_out=None, opt_nb_plane=None) -> V_out
    FFT_MAX_VEL_DCL       (communicator, V1_in, nb_procs, bloc_size, m_max_pad) -> V_out (a float)

(FFT_PAR_REAL's V_out is ALLOCATABLE in the reference and FFT_MAX_VEL_DCL's a scalar INTENT(OUT):
here both are returned.)

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

OP_CROSS, OP_DOT, OP_PROD, OP_DIV, OP_SCALAR_VECT, OP_VECT_SCALAR, OP_TENSOR, OP_TENSION = range(8)
ALGO_AUTO, ALGO_GRID, ALGO_FAST = 0, 1, 2
# routine name -> (op code, slots of the first input, of the second, of the output); the tensor
# routines return V_out(3, np, 6, m) (fft_parallel.F90:1552)
KINDS = {
    "cross": (OP_CROSS, 6, 6, 6), "dot": (OP_DOT, 6, 6, 2), "prod": (OP_PROD, 2, 2, 2), "div": (OP_DIV, 2, 2, 2),
    "svect": (OP_SCALAR_VECT, 6, 2, 6), "svdiv": (OP_VECT_SCALAR, 6, 2, 6), "tensor": (OP_TENSOR, 6, 6, 6),
    "tension": (OP_TENSION, 6, 6, 6),
}
OP_KIND = {v[0]: k for k, v in KINDS.items()}
TENSOR_OPS = (OP_TENSOR, OP_TENSION)
SPLIT_BF16X2, SPLIT_BF16X3 = 2, 3

ERRORS = {
    0: "OK", -1: "SFNL_ERR_ARG", -2: "SFNL_ERR_SHAPE", -3: "SFNL_ERR_ALIAS", -4: "SFNL_ERR_UNSUPPORTED",
    -5: "SFNL_ERR_CUDA", -6: "SFNL_ERR_NONFINITE", -7: "SFNL_ERR_ALLOC", -8: "SFNL_ERR_TIMEOUT",
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
    "sfnl_div_f64": [_P, _P, _P, _L, _I, _I, _P],
    "sfnl_scalar_vect_f64": [_P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_tensor_f64": [_P, _P, _P, _L, _I, _I, _I, _P],
    "sfnl_fft_par_div_dcl": [_P, _P, _P, _I, _I, _I, _I, _I, _P],
    "sfnl_fft_scalar_vect_dcl": [_P, _P, _P] + [_I] * 8 + [_P],
    "sfnl_fft_tensor_dcl": [_P, _P, _P] + [_I] * 7 + [_P],
    "sfnl_real_f64": [_P, _P, _L, _I, _I, _I, _P],
    "sfnl_cross_gauss_f64": [_P] * 8 + [_I] * 6 + [_P, _P],
    "sfnl_smb_cross_prod_gauss": [_P] * 5 + [_I] + [_P] * 3 + [_I] * 6,
    "sfnl_curlh_cross_b_gauss_f64": [_P] * 8 + [_I] * 6 + [_P, _P],
    "sfnl_smb_curlh_cross_b_gauss": [_P] * 6 + [_I] + [_P] * 2 + [_I] * 6,
    "sfnl_ugradc_gauss_f64": [_P] * 3 + [_I] + [_P] * 6 + [_I] * 6 + [_P, _P],
    "sfnl_smb_ugradc_gauss": [_P] * 3 + [_I] + [_P] * 4 + [_I] + [_P] * 2 + [_I] * 6,
    "sfnl_gauss_operands_f64": [_I] + [_P] * 4 + [_I] + [_P] * 9 + [_I] * 5 + [_P],
    "sfnl_max_vel_f64": [_P, _P, _L, _I, _I, _I, _P],
    "sfnl_fft_par_real_planes": [_I, _I],
    "sfnl_fft_par_real": [_P, _P] + [_I] * 5,
    "sfnl_fft_max_vel_dcl": [_P, _P] + [_I] * 6,
    "sfnl_bundle_mhd_host": [_P] * 9 + [_L, _I, _I, _I],
    "sfnl_set_check_finite": [_I],
    "sfnl_finalize": [],
    "sfnl_last_host_timing": [_P],
    "sfnl_test_inject_timeout": [],
    "sfnl_set_bundle_kernel": [_I],
    "sfnl_test_large_workspace_cap": [_L],
    "sfnl_test_large_residues": [_I],
    "sfnl_probe_fp64_tflops": [_P, _P],
    "sfnl_fft_par_pack_modes": [_P, _P] + [_I] * 6,
    "sfnl_fft_par_block": [_I, _P, _P, _P] + [_I] * 4 + [_P],
    "sfnl_fft_par_unpack_modes": [_P, _P] + [_I] * 6,
    "sfnl_cross_jvp_host": [_P] * 4 + [_L, _I, _I, _I],
    "sfnl_cross_vjp_host": [_P] * 4 + [_L, _I, _I, _I],
    "sfnl_mhd_jvp_host": [_P] * 5 + [_L, _I, _I, _I],
    "sfnl_mhd_vjp_host": [_P] * 5 + [_L, _I, _I, _I],
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


def tensor_empty(npts: int, m: int, device="cuda", dtype=None):
    """Uninitialised CUDA tensor of shape (3, np, 6, m) in Fortran order (FFT_TENSOR_DCL's V_out)."""
    import torch

    dtype = dtype or torch.float64
    return torch.empty((m, 6, npts, 3), device=device, dtype=dtype).permute(3, 2, 1, 0)


def out_empty(op: int, npts: int, m: int, device="cuda"):
    """Output tensor of product ``op`` for np points and m modes."""
    if op in TENSOR_OPS:
        return tensor_empty(npts, m, device=device)
    return fortran_empty(npts, KINDS[OP_KIND[op]][3], m, device=device)


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
    """Product ``op`` (OP_*) of two Fortran-layout CUDA tensors: cross, dot, prod, div, scalar x vector,
    vector / scalar, tensor, tension tensor.  Shapes follow ``KINDS``."""
    if op not in OP_KIND:
        raise SfnlError(-1, f"op must be one of OP_* (0..7), got {op}")
    _, nsl_a, nsl_b, nsl_o = KINDS[OP_KIND[op]]
    npts, nsl, m = a.shape
    if nsl != nsl_a or tuple(b.shape) != (npts, nsl_b, m):
        raise SfnlError(-2, f"{OP_KIND[op]}: inputs must be (np, {nsl_a}, m) and (np, {nsl_b}, m)")
    if m_max_pad is None:
        m_max_pad = 3 * m // 2
    if out is None:
        out = out_empty(op, npts, m, device=a.device)
    want = (3, npts, 6, m) if op in TENSOR_OPS else (npts, nsl_o, m)
    if tuple(out.shape) != want:
        raise SfnlError(-2, f"{OP_KIND[op]}: output must be {want}")
    if split is None:
        _check(lib().sfnl_product_f64(op, _dptr(a, "a"), _dptr(b, "b"), _dptr(out, "out"), npts, m, m_max_pad,
                                      n_theta, algo, _stream(stream)))
    else:
        if n_theta:
            raise ValueError("split forms pick their own grid")
        _check(lib().sfnl_product_split(op, _dptr(a, "a"), _dptr(b, "b"), _dptr(out, "out"), npts, m, m_max_pad,
                                        split, _stream(stream)))
    return out


def div(c1, c2, out=None, m_max_pad=None, stream=None):
    """c1 / c2 on the caller's grid (FFT_PAR_DIV_DCL, fft_parallel.F90:667-830): (np, 2, m) -> (np, 2, m)."""
    return product(OP_DIV, c1, c2, out=out, m_max_pad=m_max_pad, stream=stream)


def scalar_vect(v, s, pb: int = 1, out=None, m_max_pad=None, split=None, stream=None):
    """FFT_SCALAR_VECT_DCL (fft_parallel.F90:1021-1220): pb = 1 -> s v, pb = 2 -> v / s."""
    if pb not in (1, 2):
        raise SfnlError(-1, "error in problem type while calling FFT_SCALAR_VECT_DCL")
    return product(OP_SCALAR_VECT if pb == 1 else OP_VECT_SCALAR, v, s, out=out, m_max_pad=m_max_pad, split=split,
                   stream=stream)


def tensor(v1, v2, tension: bool = False, out=None, m_max_pad=None, split=None, stream=None):
    """FFT_TENSOR_DCL (fft_parallel.F90:1543-1796): (np, 6, m) x (np, 6, m) -> (3, np, 6, m)."""
    return product(OP_TENSION if tension else OP_TENSOR, v1, v2, out=out, m_max_pad=m_max_pad, split=split,
                   stream=stream)


def real_planes(m_max: int, opt_nb_plane: int | None = None) -> int:
    """Grid length of FFT_PAR_REAL (fft_parallel.F90:71-80)."""
    n = lib().sfnl_fft_par_real_planes(m_max, opt_nb_plane or 0)
    _check(min(n, 0))
    return n


def synthesis(v, n_theta: int | None = None, out=None, stream=None):
    """Values of every field of v (np, nslot, m) at theta_j = 2 pi j / N: a CUDA tensor (N, nslot/2, np)
    in Fortran order (FFT_PAR_REAL, fft_parallel.F90:28-145; N = 2*m_max-1 by default)."""
    import torch

    npts, nsl, m = v.shape
    N = n_theta or real_planes(m)
    if out is None:
        out = torch.empty((npts, nsl // 2, N), device=v.device, dtype=torch.float64).permute(2, 1, 0)
    if tuple(out.shape) != (N, nsl // 2, npts):
        raise SfnlError(-2, f"out must be {(N, nsl // 2, npts)}")
    _check(lib().sfnl_real_f64(_dptr(v, "v"), _dptr(out, "out"), npts, nsl, m, N, _stream(stream)))
    return out


def max_vel(v, m_max_pad: int | None = None, stream=None) -> float:
    """FFT_MAX_VEL_DCL (fft_parallel.F90:1426-1541): max over points and the 2*m_max_pad-1 angles of |v|."""
    import torch

    npts, nsl, m = v.shape
    res = torch.empty(1, device=v.device, dtype=torch.float64)
    _check(lib().sfnl_max_vel_f64(_dptr(v, "v"), ctypes.c_void_p(res.data_ptr()), npts, nsl, m, m_max_pad or m,
                                  _stream(stream)))
    return float(res.item())


def cross_gauss(v, mesh, list_mode, omega=None, m_max_pad=None, out=None, work=None, stream=None):
    """(curl v + 2 omega) x v at the Gauss points from the nodal v (np_nodes, 6, nmod): the operands and
    product of smb_cross_prod_gauss_sft_par (subroutine_ns_with_velocity.F90:512-629).  ``mesh``: CUDA
    tensors jj (n_w, me) int32 1-based, ww (n_w, l_G), dw (2, n_w, l_G, me), rr (2, np_nodes), all in
    Fortran order; list_mode: int32 CUDA tensor of the nmod mode numbers.  Returns (l_G*me, 6, nmod)."""
    npn, _, nmod = v.shape
    n_w, me = mesh["jj"].shape
    l_G = mesh["ww"].shape[1]
    if out is None:
        out = fortran_empty(l_G * me, 6, nmod, device=v.device)
    ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _check(lib().sfnl_cross_gauss_f64(_dptr(v, "v"), ptr(mesh["jj"]), ptr(mesh["ww"]), ptr(mesh["dw"]),
                                      ptr(mesh["rr"]), ptr(list_mode), None if omega is None else _dptr(omega, "omega"),
                                      _dptr(out, "out"), npn, me, n_w, l_G, nmod, m_max_pad or 0, ptr(work),
                                      _stream(stream)))
    return out


def _gauss_dims(v, mesh):
    npn, _, nmod = v.shape
    n_w, me = mesh["jj"].shape
    return npn, nmod, n_w, me, mesh["ww"].shape[1]


def curlh_cross_b_gauss(h, b, mesh, list_mode, m_max_pad=None, out=None, work=None, stream=None):
    """(curl h) x b at the Gauss points from the nodal h, b (np_nodes, 6, nmod): the Lorentz-force term
    of smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883).  ``mesh`` and ``list_mode`` as
    in :func:`cross_gauss`.  Returns (l_G*me, 6, nmod)."""
    npn, nmod, n_w, me, l_G = _gauss_dims(h, mesh)
    if out is None:
        out = fortran_empty(l_G * me, 6, nmod, device=h.device)
    ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _check(lib().sfnl_curlh_cross_b_gauss_f64(_dptr(h, "h"), _dptr(b, "b"), ptr(mesh["jj"]), ptr(mesh["ww"]),
                                              ptr(mesh["dw"]), ptr(mesh["rr"]), ptr(list_mode), _dptr(out, "out"),
                                              npn, me, n_w, l_G, nmod, m_max_pad or 0, ptr(work), _stream(stream)))
    return out


def ugradc_gauss(v, c, mesh, list_mode, heat=None, conservative=False, m_max_pad=None, out=None, work=None,
                 stream=None):
    """(heat grad c) . v [+ div v (heat c) when conservative] at the Gauss points from the nodal velocity
    v (np_nodes, 6, nmod) and scalar c (np_nodes, 2, nmod): the advection term of smb_ugradc_gauss_fft_par
    (level set: conservative False; temperature: conservative, heat = the heat capacity of each element;
    concentration: conservative).  Returns (l_G*me, 2, nmod)."""
    npn, nmod, n_w, me, l_G = _gauss_dims(v, mesh)
    if out is None:
        out = fortran_empty(l_G * me, 2, nmod, device=v.device)
    ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _check(lib().sfnl_ugradc_gauss_f64(_dptr(v, "v"), _dptr(c, "c"), ptr(heat), 1 if conservative else 0,
                                       ptr(mesh["jj"]), ptr(mesh["ww"]), ptr(mesh["dw"]), ptr(mesh["rr"]),
                                       ptr(list_mode), _dptr(out, "out"), npn, me, n_w, l_G, nmod, m_max_pad or 0,
                                       ptr(work), _stream(stream)))
    return out


GAUSS_NS, GAUSS_LORENTZ, GAUSS_ADVECT = 0, 1, 2


def gauss_operands(kind, v, mesh, list_mode, v2=None, omega=None, heat=None, conservative=False, stream=None):
    """The Gauss-point operands of one caller without the product (CUDA tensors, ``mesh`` and
    ``list_mode`` as in :func:`cross_gauss`): GAUSS_NS -> (RotV + 2 omega, W); GAUSS_LORENTZ (v = H,
    v2 = B) -> (curl H, B); GAUSS_ADVECT (v = u, v2 = c) -> (heat grad c, W[, div u, heat c] when
    conservative).  Each (l_G*me, nslot, nmod)."""
    npn, nmod, n_w, me, l_G = _gauss_dims(v, mesh)
    ng = l_G * me
    outs = [fortran_empty(ng, 6, nmod, device=v.device), fortran_empty(ng, 6, nmod, device=v.device)]
    cons = kind == GAUSS_ADVECT and conservative
    if cons:
        outs += [fortran_empty(ng, 2, nmod, device=v.device), fortran_empty(ng, 2, nmod, device=v.device)]
    ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    o = outs + [None] * (4 - len(outs))
    _check(lib().sfnl_gauss_operands_f64(kind, _dptr(v, "v"), None if v2 is None else _dptr(v2, "v2"),
                                         None if omega is None else _dptr(omega, "omega"), ptr(heat),
                                         1 if cons else 0, ptr(mesh["jj"]), ptr(mesh["ww"]), ptr(mesh["dw"]),
                                         ptr(mesh["rr"]), ptr(list_mode), *[ptr(t) for t in o], npn, me, n_w, l_G,
                                         nmod, _stream(stream)))
    return tuple(outs)


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


BUNDLE_RESIDUE, BUNDLE_THIRD_FOLD = 0, 1


def set_bundle_kernel(kind: int) -> int:
    """Kernel of the FAST MHD bundle at m = 64 (process-wide): BUNDLE_RESIDUE (default, the grid split into
    its three residue classes) or BUNDLE_THIRD_FOLD (one 192-angle transform).  Returns the previous kind."""
    rc = lib().sfnl_set_bundle_kernel(int(kind))
    _check(min(rc, 0))
    return rc


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
        op = KINDS[kind][0]
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
    if out.shape != (out_shape := ((3, npts, 6, mc) if KINDS[kind][0] in TENSOR_OPS else (npts, KINDS[kind][3], mc))):
        raise SfnlError(-2, f"V_out must be {out_shape}")
    X, Y, O, T = _host_ptr(x), _host_ptr(y), _host_ptr(out), _host_ptr(t3)
    if kind == "cross":
        rc = L.sfnl_fft_par_cross_prod_dcl(X, Y, O, npts, nf, mc, nb_procs, bloc_size, m_max_pad, T)
    elif kind == "dot":
        rc = L.sfnl_fft_par_dot_prod_dcl(X, Y, O, npts, nf, mc, nb_procs, bloc_size, m_max_pad, T)
    elif kind == "prod":
        rc = L.sfnl_fft_par_prod_dcl(X, Y, O, npts, mc, nb_procs, bloc_size, m_max_pad, T)
    elif kind == "div":
        rc = L.sfnl_fft_par_div_dcl(X, Y, O, npts, mc, nb_procs, bloc_size, m_max_pad, T)
    elif kind in ("svect", "svdiv"):
        rc = L.sfnl_fft_scalar_vect_dcl(X, Y, O, 1 if kind == "svect" else 2, npts, nf, y.shape[1], mc, nb_procs,
                                        bloc_size, m_max_pad, T)
    else:
        rc = L.sfnl_fft_tensor_dcl(X, Y, O, npts, nf, mc, nb_procs, bloc_size, m_max_pad,
                                   1 if kind == "tension" else -1, T)
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


def FFT_PAR_DIV_DCL(communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps=None):
    """c_out = c1_in / c2_in on the grid of 2*m_max_pad-1 angles (fft_parallel.F90:667-830)."""
    return _fortran_call("div", communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)


def FFT_SCALAR_VECT_DCL(communicator, V1_in, V2_in, V_out, pb, nb_procs, bloc_size, m_max_pad, temps=None):
    """V_out = V2_in * V1_in (pb = 1) or V1_in / V2_in (pb = 2); V1_in a vector (np, 6, m), V2_in a
    scalar (np, 2, m) (fft_parallel.F90:1021-1220)."""
    if V1_in.shape[1] != 6 or V2_in.shape[1] != 2:
        raise SfnlError(-2, "error in dimension of INPUT variables while calling FFT_SCALAR_VECT_DCL")
    if pb not in (1, 2):
        raise SfnlError(-1, "error in problem type while calling FFT_SCALAR_VECT_DCL")
    return _fortran_call("svect" if pb == 1 else "svdiv", communicator, V1_in, V2_in, V_out, nb_procs, bloc_size,
                         m_max_pad, temps)


def FFT_TENSOR_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps=None, opt_tension=None):
    """V_out(k, :, 2l-1:2l, :) = coefficients of V1_k V2_l, V_out of shape (3, np, 6, m); with
    opt_tension=True the tension form (fft_parallel.F90:1543-1796).  opt_tension=False is rejected,
    as the reference does (:1705)."""
    if opt_tension is not None and not opt_tension:
        raise SfnlError(-1, "BUG in FFT_TENSOR_DCL : opt_tension should be true if used")
    return _fortran_call("tension" if opt_tension else "tensor", communicator, V1_in, V2_in, V_out, nb_procs,
                         bloc_size, m_max_pad, temps)


def FFT_PAR_REAL(communicator, V1_in, V_out=None, opt_nb_plane=None):
    """Values of the fields of V1_in (np, nb_field, m) on the N = 2*m_max_pad-1 angles 2*pi*j/N
    (fft_parallel.F90:28-145): V_out (N, nb_field/2, np), returned (and filled in when given)."""
    import numpy as np

    npts, nf, mc = V1_in.shape
    if communicator is not None:
        from .parallel import fft_par_real_distributed

        return fft_par_real_distributed(communicator, V1_in, opt_nb_plane)
    N = real_planes(mc, opt_nb_plane)
    if hasattr(V1_in, "is_cuda"):
        return synthesis(V1_in, n_theta=N, out=V_out)
    V1_in = np.asfortranarray(V1_in, dtype=np.float64)
    if V_out is None:
        V_out = np.zeros((N, nf // 2, npts), order="F")
    if V_out.shape != (N, nf // 2, npts) or not V_out.flags.f_contiguous or V_out.dtype != np.float64:
        raise SfnlError(-2, f"V_out must be a float64 Fortran array of shape {(N, nf // 2, npts)}")
    _check(lib().sfnl_fft_par_real(_host_ptr(V1_in), _host_ptr(V_out), npts, nf, mc, 1, opt_nb_plane or 0))
    return V_out


def FFT_MAX_VEL_DCL(communicator, V1_in, nb_procs, bloc_size, m_max_pad):
    """Maximum over the points and the 2*m_max_pad-1 angles of |V1_in| (its first 3-vector for
    nb_field == 6, |first field| otherwise) (fft_parallel.F90:1426-1541)."""
    import numpy as np

    npts, nf, mc = V1_in.shape
    if communicator is not None:
        from .parallel import fft_max_vel_distributed

        return fft_max_vel_distributed(communicator, V1_in, nb_procs, bloc_size, m_max_pad)
    if hasattr(V1_in, "is_cuda"):
        if nb_procs != 1:
            raise SfnlError(-4, "one GPU holds all modes: nb_procs must be 1")
        if npts > nb_procs * bloc_size:
            raise SfnlError(-2, "np > nb_procs*bloc_size")
        return max_vel(V1_in, m_max_pad)
    V1_in = np.asfortranarray(V1_in, dtype=np.float64)
    res = np.zeros(1)
    _check(lib().sfnl_fft_max_vel_dcl(_host_ptr(V1_in), _host_ptr(res), npts, nf, mc, nb_procs, bloc_size, m_max_pad))
    return float(res[0])


def smb_cross_prod_gauss_sft_par(communicator, mesh, list_mode, V_in, V_out=None, precession_in=False,
                                 taux_precession=0.0, angle_s_pi=0.0):
    """The Navier-Stokes nonlinear term at the Gauss points (subroutine_ns_with_velocity.F90:512-629) on
    host arrays: ``mesh`` holds the numpy arrays jj (n_w, me, 1-based), ww, dw, rr of mesh%... ; the
    precession parameters stand for the reference's inputs%taux_precession and inputs%angle_s_pi.
    Returns V_out (l_G*me, 6, nmod)."""
    import numpy as np

    if communicator is not None:
        raise SfnlError(-4, "one GPU holds all modes: the Gauss-point entry runs on one Fourier rank")
    V_in = np.asfortranarray(V_in, dtype=np.float64)
    npn, _, nmod = V_in.shape
    jj = np.asfortranarray(mesh["jj"], dtype=np.int32)
    n_w, me = jj.shape
    ww = np.asfortranarray(mesh["ww"], dtype=np.float64)
    dw = np.asfortranarray(mesh["dw"], dtype=np.float64)
    rr = np.asfortranarray(mesh["rr"], dtype=np.float64)
    l_G = ww.shape[1]
    lm = np.ascontiguousarray(list_mode, dtype=np.int32)
    om = None
    if precession_in:  # the nodal rotation field of :540-554
        om = np.zeros_like(V_in)
        for i, mode in enumerate(lm):
            if mode == 1:
                om[:, 0, i] = taux_precession * np.sin(angle_s_pi * np.pi)
                om[:, 3, i] = -taux_precession * np.sin(angle_s_pi * np.pi)
            elif mode == 0:
                om[:, 4, i] = taux_precession * np.cos(angle_s_pi * np.pi)
    if V_out is None:
        V_out = np.zeros((l_G * me, 6, nmod), order="F")
    _check(lib().sfnl_smb_cross_prod_gauss(_host_ptr(V_in), _host_ptr(jj), _host_ptr(ww), _host_ptr(dw), _host_ptr(rr),
                                           rr.shape[0], _host_ptr(lm), None if om is None else _host_ptr(om),
                                           _host_ptr(V_out), npn, me, n_w, l_G, nmod, 1))
    return V_out


def _host_mesh(mesh, list_mode):
    import numpy as np

    jj = np.asfortranarray(mesh["jj"], dtype=np.int32)
    ww = np.asfortranarray(mesh["ww"], dtype=np.float64)
    dw = np.asfortranarray(mesh["dw"], dtype=np.float64)
    rr = np.asfortranarray(mesh["rr"], dtype=np.float64)
    return jj, ww, dw, rr, np.ascontiguousarray(list_mode, dtype=np.int32)


def smb_CurlH_cross_B_gauss_sft_par(communicator, mesh, list_mode, V_in, W_in, V_out=None):
    """The Lorentz force (curl H) x B at the Gauss points (subroutine_ns_with_m.F90:788-883) on host
    arrays: V_in = H, W_in = B (np_nodes, 6, nmod).  Returns V_out (l_G*me, 6, nmod)."""
    import numpy as np

    if communicator is not None:
        raise SfnlError(-4, "one GPU holds all modes: the Gauss-point entry runs on one Fourier rank")
    V_in = np.asfortranarray(V_in, dtype=np.float64)
    W_in = np.asfortranarray(W_in, dtype=np.float64)
    npn, _, nmod = V_in.shape
    jj, ww, dw, rr, lm = _host_mesh(mesh, list_mode)
    n_w, me = jj.shape
    l_G = ww.shape[1]
    if V_out is None:
        V_out = np.zeros((l_G * me, 6, nmod), order="F")
    _check(lib().sfnl_smb_curlh_cross_b_gauss(_host_ptr(V_in), _host_ptr(W_in), _host_ptr(jj), _host_ptr(ww),
                                              _host_ptr(dw), _host_ptr(rr), rr.shape[0], _host_ptr(lm),
                                              _host_ptr(V_out), npn, me, n_w, l_G, nmod, 1))
    return V_out


def _host_ugradc(communicator, mesh, list_mode, V_in, c_in, c_out, heat, conservative):
    import numpy as np

    if communicator is not None:
        raise SfnlError(-4, "one GPU holds all modes: the Gauss-point entry runs on one Fourier rank")
    V_in = np.asfortranarray(V_in, dtype=np.float64)
    c_in = np.asfortranarray(c_in, dtype=np.float64)
    npn, _, nmod = V_in.shape
    jj, ww, dw, rr, lm = _host_mesh(mesh, list_mode)
    n_w, me = jj.shape
    l_G = ww.shape[1]
    hc = None if heat is None else np.ascontiguousarray(heat, dtype=np.float64)
    if hc is not None and hc.shape[0] < me:
        raise SfnlError(-1, "heat_capa_in holds fewer values than elements")
    if c_out is None:
        c_out = np.zeros((l_G * me, 2, nmod), order="F")
    _check(lib().sfnl_smb_ugradc_gauss(_host_ptr(V_in), _host_ptr(c_in), None if hc is None else _host_ptr(hc),
                                       1 if conservative else 0, _host_ptr(jj), _host_ptr(ww), _host_ptr(dw),
                                       _host_ptr(rr), rr.shape[0], _host_ptr(lm), _host_ptr(c_out), npn, me, n_w,
                                       l_G, nmod, 1))
    return c_out


def smb_ugradc_gauss_fft_par(communicator, mesh, list_mode, V_in, c_in, nb_procs=1, c_out=None):
    """The level-set advection term grad c . u at the Gauss points (subroutine_level_set.F90:434-534)
    on host arrays: V_in (np_nodes, 6, nmod), c_in (np_nodes, 2, nmod).  Returns c_out (l_G*me, 2, nmod)."""
    if nb_procs != 1:
        raise SfnlError(-4, "one GPU holds all modes: nb_procs must be 1")
    return _host_ugradc(communicator, mesh, list_mode, V_in, c_in, c_out, None, False)


def smb_ugradc_gauss_fft_par_temperature(communicator, mesh, list_mode, heat_capa_in, V_in, c_in, c_out=None):
    """The temperature equation's smb_ugradc_gauss_fft_par (subroutine_temperature_with_T.F90:247-350):
    (C grad T) . u + div u (C T), C = heat_capa_in(m) of each element."""
    return _host_ugradc(communicator, mesh, list_mode, V_in, c_in, c_out, heat_capa_in, True)


def smb_ugradc_gauss_fft_par_conc(communicator, mesh, list_mode, V_in, c_in, c_out=None):
    """The concentration equation's advection term grad c . u + c div u
    (subroutine_concentration.F90:243-341)."""
    return _host_ugradc(communicator, mesh, list_mode, V_in, c_in, c_out, None, True)
