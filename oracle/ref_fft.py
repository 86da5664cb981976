"""CPU oracle, Python side.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module: it is the checker for the CUDA path, never part of it.

Three independent CPU formulations of the dealiased products of
SOURCES/POST_PROCESSING/fft_parallel.F90 (FFT_PAR_CROSS_PROD_DCL :147-328,
FFT_PAR_DOT_PROD_DCL :330-500, FFT_PAR_PROD_DCL :502-665, FFT_PAR_DIV_DCL
:667-830, FFT_SCALAR_VECT_DCL :1021-1220, FFT_TENSOR_DCL :1543-1796), and
of the synthesis-only FFT_PAR_REAL (:28-145) and FFT_MAX_VEL_DCL
(:1426-1541) (``c_real``, ``c_max_vel``, ``synth_grid``):

* ``c_oracle``   -- ctypes binding of oracle/sfnl_oracle.c, the step-by-step
  long-double restatement of the reference (pack, emulated MPI_ALLTOALL,
  c2r, product, r2c, 1/N, 2*CONJG, truncation, unpack).
* ``fft_par``    -- the same algorithm with a library FFT (scipy.fft, i.e.
  pocketfft, multithreaded) in place of FFTW: the FFTW-class CPU path that
  bench.py times as the CPU baseline.
* ``spectral_product`` -- the exact truncated product computed directly in
  coefficient space (discrete convolution of the two Fourier series in long
  double): no grid, no aliasing, no transform.

Arrays follow the reference's Fortran layout: numpy arrays of shape
(np, nslot, m) in Fortran (column-major) order, slot 2k holds the cosine and
slot 2k+1 the sine coefficient of component k (0-based), mode n along the
last axis.  The sine of mode 0 is ignored on input and 0 on output.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OP_CROSS, OP_DOT, OP_PROD, OP_DIV, OP_SVECT, OP_SVDIV, OP_TENSOR, OP_TENSION = range(8)
_OPS = {"cross": OP_CROSS, "dot": OP_DOT, "prod": OP_PROD, "div": OP_DIV, "svect": OP_SVECT, "svdiv": OP_SVDIV,
        "tensor": OP_TENSOR, "tension": OP_TENSION}
# input slots (V1, V2) and output slots each routine takes and returns
_IN_SLOTS = {OP_CROSS: (6, 6), OP_DOT: (6, 6), OP_PROD: (2, 2), OP_DIV: (2, 2), OP_SVECT: (6, 2), OP_SVDIV: (6, 2),
             OP_TENSOR: (6, 6), OP_TENSION: (6, 6)}
_NOUT = {OP_CROSS: 3, OP_DOT: 1, OP_PROD: 1, OP_DIV: 1, OP_SVECT: 3, OP_SVDIV: 3, OP_TENSOR: 9, OP_TENSION: 9}


def out_shape(op: str, npts: int, m: int):
    """Shape of V_out: (np, 2*ncomp, m), or (3, np, 6, m) for the tensor routine (fft_parallel.F90:1552)."""
    opc = _OPS[op]
    if opc in (OP_TENSOR, OP_TENSION):
        return (3, npts, 6, m)
    return (npts, 2 * _NOUT[opc], m)


# ----------------------------------------------------------------------------
# synthetic inputs (SplitMix64 -> Box-Muller), shared by tests and bench
# ----------------------------------------------------------------------------
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(seed: int, count: int) -> np.ndarray:
    """``count`` consecutive SplitMix64 outputs for state ``seed``."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def synthetic_field(npts: int, nslot: int, m: int, alpha: float, seed: int) -> np.ndarray:
    """Fortran-ordered (npts, nslot, m) array: x[p,s,n] = z*exp(-alpha*n).

    z ~ N(0,1) from SplitMix64 + Box-Muller in Fortran memory order; the sine
    slot of mode 0 is set to 0 (the reference ignores it, fft_parallel.F90:241).
    """
    total = npts * nslot * m
    pairs = (total + 1) // 2
    bits = _splitmix64(seed, 2 * pairs)
    u = ((bits >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    rad = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * pairs)
    z[0::2] = rad * np.cos(2.0 * np.pi * u2)
    z[1::2] = rad * np.sin(2.0 * np.pi * u2)
    x = z[:total].reshape((npts, nslot, m), order="F")
    x = x * np.exp(-alpha * np.arange(m))[None, None, :]
    x[:, 1::2, 0] = 0.0
    return np.asfortranarray(x)


# ----------------------------------------------------------------------------
# C oracle (long double restatement of the reference)
# ----------------------------------------------------------------------------
def _lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(HERE, "_build", "libsfnl_oracle.so")
        if not os.path.exists(so):
            subprocess.check_call(["make", "-s", "-C", HERE])
        lib = ctypes.CDLL(so)
        P = ctypes.POINTER(ctypes.c_double)
        for name in ("orc_fft_par_dcl",):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, P, P, P] + [ctypes.c_int] * 6
        f = lib.orc_fft_par_dcl_n
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_double)] + [ctypes.c_int] * 7
        f = lib.orc_apply_n
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int, P] + [ctypes.c_int] * 6
        lib.orc_fft_par_real_planes.restype = ctypes.c_int
        lib.orc_fft_par_real_planes.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.orc_fft_par_real.restype = ctypes.c_int
        lib.orc_fft_par_real.argtypes = [P] + [ctypes.c_int] * 5 + [P]
        lib.orc_fft_max_vel.restype = ctypes.c_int
        lib.orc_fft_max_vel.argtypes = [P] + [ctypes.c_int] * 6 + [P]
        IP = ctypes.POINTER(ctypes.c_int)
        lib.orc_cross_gauss.restype = ctypes.c_int
        lib.orc_cross_gauss.argtypes = [P, IP, P, P, P, IP, P] + [ctypes.c_int] * 5 + [P, P, P]
        lib.orc_curlh_cross_b_gauss.restype = ctypes.c_int
        lib.orc_curlh_cross_b_gauss.argtypes = [P, P, IP, P, P, P, IP] + [ctypes.c_int] * 5 + [P, P, P]
        lib.orc_ugradc_gauss.restype = ctypes.c_int
        lib.orc_ugradc_gauss.argtypes = [P, P, P, ctypes.c_int, IP, P, P, P, IP] + [ctypes.c_int] * 5 + [P] * 5
        _LIB = lib
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ----------------------------------------------------------------------------
# O(N log N) C restatement on host threads (the timed CPU baseline)
# ----------------------------------------------------------------------------
_CPU = None


def _cpu_lib():
    global _CPU
    if _CPU is None:
        so = os.path.join(HERE, "_build", "libsfnl_cpu.so")
        if not os.path.exists(so):
            subprocess.check_call(["make", "-s", "-C", HERE])
        lib = ctypes.CDLL(so)
        P = ctypes.POINTER(ctypes.c_double)
        lib.sfnl_cpu_product.restype = ctypes.c_int
        lib.sfnl_cpu_product.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int64] + [ctypes.c_int] * 3
        lib.sfnl_cpu_mhd_bundle.restype = ctypes.c_int
        lib.sfnl_cpu_mhd_bundle.argtypes = [P] * 9 + [ctypes.c_int64] + [ctypes.c_int] * 3
        lib.sfnl_cpu_threads.restype = ctypes.c_int
        lib.sfnl_cpu_threads.argtypes = []
        _CPU = lib
    return _CPU


def cpu_threads() -> int:
    return int(_cpu_lib().sfnl_cpu_threads())


def cpu_product(op: str, V1, V2, m_max_pad: int, n_theta: int | None = None, threads: int = 0):
    """FFT_PAR_{CROSS,DOT,}_PROD_DCL by the C restatement with O(N log N) real FFTs on ``threads``
    host threads (0: all), grid N = n_theta or the reference's 2*m_max_pad - 1."""
    V1 = np.asfortranarray(V1, dtype=np.float64)
    V2 = np.asfortranarray(V2, dtype=np.float64)
    npts, _, m = V1.shape
    N = n_theta or 2 * m_max_pad - 1
    out = np.zeros(out_shape(op, npts, m), order="F")
    rc = _cpu_lib().sfnl_cpu_product({"cross": 0, "dot": 1, "prod": 2}[op], _ptr(V1), _ptr(V2), _ptr(out), npts, m, N,
                                     threads)
    if rc:
        raise RuntimeError(f"sfnl_cpu_product failed ({rc})")
    return out


def cpu_mhd_bundle(u, w, b, j, gradT, m_max_pad: int, n_theta: int | None = None, threads: int = 0):
    """(u x w, u x b, j x b, u . gradT) by the C restatement, point block by point block."""
    ins = [np.asfortranarray(x, dtype=np.float64) for x in (u, w, b, j, gradT)]
    npts, _, m = ins[0].shape
    N = n_theta or 2 * m_max_pad - 1
    outs = [np.zeros((npts, 6, m), order="F") for _ in range(3)] + [np.zeros((npts, 2, m), order="F")]
    rc = _cpu_lib().sfnl_cpu_mhd_bundle(*[_ptr(x) for x in ins + outs], npts, m, N, threads)
    if rc:
        raise RuntimeError(f"sfnl_cpu_mhd_bundle failed ({rc})")
    return tuple(outs)


def c_oracle(op: str, V1, V2, m_max_pad: int, nb_procs: int = 1, bloc_size: int | None = None,
             n_theta: int | None = None):
    """Long-double restatement of FFT_PAR_*_DCL on global arrays.

    ``V1``/``V2`` hold all m_max = m_max_c*nb_procs modes; rank r of the
    emulated Fourier communicator owns modes [r*m_max_c, (r+1)*m_max_c).
    ``bloc_size`` defaults to the callers' choice np/nb_procs+1
    (subroutine_ns_with_velocity.F90:625).  Returns V_out (np, 2*ncomp, m_max),
    or (3, np, 6, m_max) for "tensor" / "tension".
    Raises ValueError with the oracle's status for inputs the reference rejects.
    """
    opc = _OPS[op]
    V1 = np.asfortranarray(V1, dtype=np.float64)
    V2 = np.asfortranarray(V2, dtype=np.float64)
    npts, nf1, m = V1.shape
    nf2 = V2.shape[1]
    if m % nb_procs:
        raise ValueError("m_max must be a multiple of nb_procs")
    if bloc_size is None:
        bloc_size = npts // nb_procs + 1
    out = np.zeros(out_shape(op, npts, m), order="F")
    N = 2 * m_max_pad - 1 if n_theta is None else n_theta
    rc = _lib().orc_apply_n(opc, _ptr(V1), nf1, _ptr(V2), nf2, _ptr(out), npts, m // nb_procs, nb_procs,
                            bloc_size, m_max_pad, N)
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return out


def real_planes(m_max: int, opt_nb_plane: int | None = None) -> int:
    """Grid length of FFT_PAR_REAL: 2*m_max_pad-1, m_max_pad = (opt_nb_plane+1)/2 when opt_nb_plane > 2m-1."""
    return _lib().orc_fft_par_real_planes(m_max, opt_nb_plane or 0)


def c_real(V, nb_procs: int = 1, opt_nb_plane: int | None = None):
    """Long-double restatement of FFT_PAR_REAL: (N, nslot/2, np) Fortran array of the values of every
    field at the angles 2*pi*j/N (the ranks' V_out one after the other)."""
    V = np.asfortranarray(V, dtype=np.float64)
    npts, nsl, m = V.shape
    if m % nb_procs:
        raise ValueError("m_max must be a multiple of nb_procs")
    N = real_planes(m, opt_nb_plane)
    out = np.zeros((N, nsl // 2, npts), order="F")
    rc = _lib().orc_fft_par_real(_ptr(V), nsl, npts, m // nb_procs, nb_procs, opt_nb_plane or 0, _ptr(out))
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return out


def c_max_vel(V, m_max_pad: int, nb_procs: int = 1, bloc_size: int | None = None) -> float:
    """Long-double restatement of FFT_MAX_VEL_DCL: max over points and the 2*m_max_pad-1 angles of |v|."""
    V = np.asfortranarray(V, dtype=np.float64)
    npts, nsl, m = V.shape
    if bloc_size is None:
        bloc_size = npts // nb_procs + 1
    res = np.zeros(1)
    rc = _lib().orc_fft_max_vel(_ptr(V), nsl, npts, m // nb_procs, nb_procs, bloc_size, m_max_pad, _ptr(res))
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return float(res[0])


def synth_grid(V, N: int, workers: int = 1):
    """pocketfft synthesis of every field on N angles 2*pi*j/N: (N, nslot/2, np) Fortran array."""
    import scipy.fft as sfft

    npts, nsl, m = V.shape
    cu = np.zeros((npts, nsl // 2, N // 2 + 1), dtype=np.complex128)
    cu[:, :, :m] = _to_complex(V, nsl // 2)
    ru = sfft.irfft(cu, n=N, axis=2, norm="forward", workers=workers)  # (np, nf, N)
    return np.asfortranarray(np.transpose(ru, (2, 1, 0)))


def synthetic_p2_mesh(nr: int, nz: int, seed: int = 0):
    """A P2 triangle mesh of the meridian rectangle r in [0.1, 1.1], z in [0, 1] (nr x nz squares, two
    triangles each, vertices jittered by a seeded generator), in the arrays the Gauss-point callers
    read: jj (6, me) 1-based nodes (3 vertices, then the midpoints of edges 2-3, 3-1, 1-2), rr (2, np)
    coordinates (r, z), and at 7 interior quadrature points ww (6, 7) = the P2 basis and
    dw (2, 6, 7, me) = its (d/dr, d/dz) on each element.  Geometry only matters for realistic sizes."""
    rng = np.random.default_rng(seed)
    hr, hz = 1.0 / nr, 1.0 / nz
    vr = np.array([[0.1 + i * hr for j in range(nz + 1)] for i in range(nr + 1)])
    vz = np.array([[j * hz for j in range(nz + 1)] for i in range(nr + 1)])
    jit = 0.15 * rng.uniform(-1, 1, size=(2, nr + 1, nz + 1))
    vr[1:-1, :] += jit[0, 1:-1, :] * hr
    vz[:, 1:-1] += jit[1, :, 1:-1] * hz
    coords = [(vr[i, j], vz[i, j]) for i in range(nr + 1) for j in range(nz + 1)]
    vid = lambda i, j: i * (nz + 1) + j  # noqa: E731
    mid = {}
    tris = []
    for i in range(nr):
        for j in range(nz):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            tris += [(a, b, c), (a, c, d)]
    jj = []
    for (a, b, c) in tris:
        e = []
        for (x, y) in ((b, c), (c, a), (a, b)):
            key = (min(x, y), max(x, y))
            if key not in mid:
                mid[key] = len(coords)
                coords.append(((coords[x][0] + coords[y][0]) / 2, (coords[x][1] + coords[y][1]) / 2))
            e.append(mid[key])
        jj.append([a, b, c] + e)
    jj = np.asfortranarray(np.array(jj, dtype=np.int32).T + 1)
    rr = np.asfortranarray(np.array(coords).T)
    # 7 interior points (barycentric): the centroid and two orbits of 3
    bary = np.array([[1 / 3, 1 / 3, 1 / 3], [2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3],
                     [0.1, 0.45, 0.45], [0.45, 0.1, 0.45], [0.45, 0.45, 0.1]])
    L = bary.T  # (3, 7)
    ww = np.asfortranarray(np.vstack([L[0] * (2 * L[0] - 1), L[1] * (2 * L[1] - 1), L[2] * (2 * L[2] - 1),
                                      4 * L[1] * L[2], 4 * L[2] * L[0], 4 * L[0] * L[1]]))
    # d(basis)/d(lambda_k) at the points: (6, 3, 7)
    dl = np.zeros((6, 3, 7))
    for k in range(3):
        dl[k, k] = 4 * L[k] - 1
    for e, (x, y) in enumerate(((1, 2), (2, 0), (0, 1))):
        dl[3 + e, x] = 4 * L[y]
        dl[3 + e, y] = 4 * L[x]
    me = len(tris)
    dw = np.zeros((2, 6, 7, me), order="F")
    for m, (a, b, c) in enumerate(tris):
        P = np.array([coords[a], coords[b], coords[c]])  # (3, 2)
        T = np.array([[P[0, 0] - P[2, 0], P[1, 0] - P[2, 0]], [P[0, 1] - P[2, 1], P[1, 1] - P[2, 1]]])
        G = np.linalg.inv(T)  # rows: d(lambda_1, lambda_2)/d(r, z)
        dlam = np.array([G[0], G[1], -G[0] - G[1]])  # (3 lambdas, 2 coords)
        dw[:, :, :, m] = np.einsum("nkl,kd->dnl", dl, dlam)
    return {"jj": jj, "rr": rr, "ww": ww, "dw": dw, "np": rr.shape[1], "me": me, "n_w": 6, "l_G": 7}


def c_cross_gauss(V, mesh, list_mode, omega=None, product=True):
    """Long-double / FP64 restatement of smb_cross_prod_gauss_sft_par (subroutine_ns_with_velocity.F90:
    512-629): returns (V_out, RotV, W), each (l_G*me, 6, nmod) Fortran (V_out zero when product=False:
    the operands only, for sizes where the O(N^2) oracle product is too slow)."""
    V = np.asfortranarray(V, dtype=np.float64)
    npn, _, nmod = V.shape
    ng = mesh["l_G"] * mesh["me"]
    outs = [np.zeros((ng, 6, nmod), order="F") for _ in range(3)]
    lm = np.ascontiguousarray(list_mode, dtype=np.int32)
    om = None if omega is None else np.asfortranarray(omega, dtype=np.float64)
    IP = ctypes.POINTER(ctypes.c_int)
    rc = _lib().orc_cross_gauss(_ptr(V), mesh["jj"].ctypes.data_as(IP), _ptr(mesh["ww"]), _ptr(mesh["dw"]),
                                _ptr(mesh["rr"]), lm.ctypes.data_as(IP), None if om is None else _ptr(om), npn,
                                mesh["me"], mesh["n_w"], mesh["l_G"], nmod, _ptr(outs[0]) if product else None,
                                _ptr(outs[1]), _ptr(outs[2]))
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return tuple(outs)


def c_curlh_cross_b_gauss(H, B, mesh, list_mode, product=True):
    """FP64 restatement of smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883): returns
    (V_out, RotV, W), each (l_G*me, 6, nmod) Fortran, V_out = (curl H) x B (zero when product=False)."""
    H = np.asfortranarray(H, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    npn, _, nmod = H.shape
    ng = mesh["l_G"] * mesh["me"]
    outs = [np.zeros((ng, 6, nmod), order="F") for _ in range(3)]
    lm = np.ascontiguousarray(list_mode, dtype=np.int32)
    IP = ctypes.POINTER(ctypes.c_int)
    rc = _lib().orc_curlh_cross_b_gauss(_ptr(H), _ptr(B), mesh["jj"].ctypes.data_as(IP), _ptr(mesh["ww"]),
                                        _ptr(mesh["dw"]), _ptr(mesh["rr"]), lm.ctypes.data_as(IP), npn, mesh["me"],
                                        mesh["n_w"], mesh["l_G"], nmod, _ptr(outs[0]) if product else None,
                                        _ptr(outs[1]), _ptr(outs[2]))
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return tuple(outs)


def c_ugradc_gauss(V, C, mesh, list_mode, heat=None, conservative=False, product=True):
    """FP64 restatement of smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534: conservative
    False, heat None; subroutine_temperature_with_T.F90:247-350: conservative, heat per element) and
    smb_ugradc_gauss_fft_par_conc (subroutine_concentration.F90:243-341: conservative, no heat).
    Returns (c_out (l_G*me, 2, nmod), Gradc, W, Div, Cgauss); c_out is zero when product=False."""
    V = np.asfortranarray(V, dtype=np.float64)
    C = np.asfortranarray(C, dtype=np.float64)
    npn, _, nmod = V.shape
    ng = mesh["l_G"] * mesh["me"]
    outs = [np.zeros((ng, n, nmod), order="F") for n in (2, 6, 6, 2, 2)]
    lm = np.ascontiguousarray(list_mode, dtype=np.int32)
    hc = None if heat is None else np.ascontiguousarray(heat, dtype=np.float64)
    IP = ctypes.POINTER(ctypes.c_int)
    rc = _lib().orc_ugradc_gauss(_ptr(V), _ptr(C), None if hc is None else _ptr(hc), 1 if conservative else 0,
                                 mesh["jj"].ctypes.data_as(IP), _ptr(mesh["ww"]), _ptr(mesh["dw"]), _ptr(mesh["rr"]),
                                 lm.ctypes.data_as(IP), npn, mesh["me"], mesh["n_w"], mesh["l_G"], nmod,
                                 _ptr(outs[0]) if product else None, *[_ptr(o) for o in outs[1:]])
    if rc != 0:
        raise ValueError(f"oracle rejected arguments (status {rc})")
    return tuple(outs)


def precession_omega(npn: int, list_mode, taux: float, angle_s_pi: float):
    """The nodal rotation field of the precession case (subroutine_ns_with_velocity.F90:540-554)."""
    om = np.zeros((npn, 6, len(list_mode)), order="F")
    for i, mode in enumerate(list_mode):
        if mode == 1:
            om[:, 0, i] = taux * np.sin(angle_s_pi * np.pi)
            om[:, 3, i] = -taux * np.sin(angle_s_pi * np.pi)
        elif mode == 0:
            om[:, 4, i] = taux * np.cos(angle_s_pi * np.pi)
    return om


# ----------------------------------------------------------------------------
# pocketfft restatement (FFTW-class CPU path; the timed CPU baseline)
# ----------------------------------------------------------------------------
def _to_complex(V, nfield):
    """cu = 0.5*(a - i b), cu_0 = a_0 (fft_parallel.F90:234-241); V (np, 2*nfield, m)."""
    a = V[:, 0::2, :]
    b = V[:, 1::2, :]
    cu = 0.5 * (a - 1j * b)
    cu[:, :, 0] = a[:, :, 0]
    return cu


def _pointwise(op, ru):
    """Grid products, fft_parallel.F90:270-274, :449-451, :617, :786, :1150-1157, :1676-1706."""
    if op == OP_CROSS:
        r1, r2, r3, r4, r5, r6 = (ru[:, k, :] for k in range(6))
        return np.stack([r2 * r6 - r3 * r5, r3 * r4 - r1 * r6, r1 * r5 - r2 * r4], axis=1)
    if op == OP_DOT:
        return (ru[:, 0] * ru[:, 3] + ru[:, 1] * ru[:, 4] + ru[:, 2] * ru[:, 5])[:, None, :]
    if op == OP_PROD:
        return (ru[:, 0] * ru[:, 1])[:, None, :]
    if op == OP_DIV:
        return (ru[:, 0] / ru[:, 1])[:, None, :]
    if op == OP_SVECT:
        return ru[:, 3:4] * ru[:, 0:3]
    if op == OP_SVDIV:
        return ru[:, 0:3] / ru[:, 3:4]
    t = ru[:, 0:3, None, :] * ru[:, None, 3:6, :]  # t[:, k, l] = u_k v_l
    if op == OP_TENSION:
        nrm = np.sqrt(ru[:, 3] ** 2 + ru[:, 4] ** 2 + ru[:, 5] ** 2)[:, None, None, :]
        t = t / (nrm + 1.0e-14) - np.eye(3)[None, :, :, None] * nrm
    return t.reshape(ru.shape[0], 9, ru.shape[2])


def fft_par(op: str, V1, V2, m_max_pad: int, n_theta: int | None = None, workers: int = 1):
    """pocketfft version of FFT_PAR_*_DCL for one rank holding all modes.

    Same steps as the reference: half-complex pack with zero padding to
    m_max_pad, c2r of length N = 2*m_max_pad-1 (unnormalised: N*irfft),
    pointwise product, r2c, 1/N, 2*CONJG, truncation to m_max.
    """
    import scipy.fft as sfft

    opc = _OPS[op]
    npts, nf1, m = V1.shape
    nf2 = V2.shape[1]
    N = 2 * m_max_pad - 1 if n_theta is None else n_theta
    nh = N // 2 + 1
    n1, n2 = nf1 // 2, nf2 // 2
    cu = np.zeros((npts, n1 + n2, nh), dtype=np.complex128)
    cu[:, :n1, :m] = _to_complex(V1, n1)
    cu[:, n1:, :m] = _to_complex(V2, n2)
    ru = sfft.irfft(cu, n=N, axis=2, norm="forward", workers=workers)  # unnormalised c2r
    prod_ru = _pointwise(opc, ru)
    pc = sfft.rfft(prod_ru, n=N, axis=2, norm="forward", workers=workers)  # includes 1/N
    pc = pc[:, :, :m]
    out = np.empty((npts, 2 * pc.shape[1], m), order="F")
    out[:, 0::2, :] = 2.0 * pc.real
    out[:, 1::2, :] = -2.0 * pc.imag
    out[:, 0::2, 0] = pc[:, :, 0].real
    out[:, 1::2, 0] = pc[:, :, 0].imag
    if opc in (OP_TENSOR, OP_TENSION):
        return tensor_layout(out)
    return out


def tensor_layout(flat):
    """(np, 18, m) with component o = 3k+l in slots 2o, 2o+1  ->  V_out(3, np, 6, m): V_out[k, :, 2l(+1), :]."""
    npts, _, m = flat.shape
    t = np.empty((3, npts, 6, m), order="F")
    for k in range(3):
        t[k] = flat[:, 6 * k:6 * k + 6, :]
    return t


# ----------------------------------------------------------------------------
# exact spectral convolution (no grid)
# ----------------------------------------------------------------------------
def _full_spectrum(a, b):
    """Complex coefficients F_n, n = -(m-1)..m-1, of f = sum a_n cos + b_n sin."""
    m = a.shape[-1]
    F = np.zeros(a.shape[:-1] + (2 * m - 1,), dtype=np.clongdouble)
    c = 0.5 * (a.astype(np.longdouble) - 1j * b.astype(np.longdouble))
    F[..., m - 1] = a[..., 0].astype(np.longdouble)
    F[..., m:] = c[..., 1:]
    F[..., : m - 1] = np.conj(c[..., 1:][..., ::-1])
    return F


def _scalar_product_coeffs(a1, b1, a2, b2):
    """cos/sin coefficients (modes < m) of (f1*f2), exact convolution in long double."""
    m = a1.shape[-1]
    F1 = _full_spectrum(a1, b1)
    F2 = _full_spectrum(a2, b2)
    H = np.zeros(a1.shape[:-1] + (m,), dtype=np.clongdouble)
    # H_k = sum_n F1_n F2_{k-n}, k = 0..m-1, n over -(m-1)..m-1
    for k in range(m):
        for n in range(-(m - 1), m):
            q = k - n
            if -(m - 1) <= q <= m - 1:
                H[..., k] += F1[..., n + m - 1] * F2[..., q + m - 1]
    a = 2.0 * H.real
    b = -2.0 * H.imag
    a[..., 0] = H[..., 0].real
    b[..., 0] = 0.0
    return a, b


def spectral_product(op: str, V1, V2):
    """Exact dealiased truncated product, no transform: (np, 6|2, m) float64."""
    opc = _OPS[op]
    npts, nf, m = V1.shape

    def sp(f1, k1, f2, k2):
        return _scalar_product_coeffs(f1[:, 2 * k1, :], f1[:, 2 * k1 + 1, :], f2[:, 2 * k2, :], f2[:, 2 * k2 + 1, :])

    if opc == OP_CROSS:
        comps = []
        for (i, j) in ((1, 2), (2, 0), (0, 1)):  # out_r = v1_t v2_z - v1_z v2_t, ...
            a1, b1 = sp(V1, i, V2, j)
            a2, b2 = sp(V1, j, V2, i)
            comps.append((a1 - a2, b1 - b2))
    elif opc == OP_DOT:
        a = b = 0
        for k in range(3):
            ak, bk = sp(V1, k, V2, k)
            a, b = a + ak, b + bk
        comps = [(a, b)]
    elif opc == OP_PROD:
        comps = [sp(V1, 0, V2, 0)]
    elif opc == OP_SVECT:
        comps = [sp(V1, k, V2, 0) for k in range(3)]
    elif opc == OP_TENSOR:
        comps = [sp(V1, k, V2, l) for k in range(3) for l in range(3)]
    else:
        raise ValueError(f"{op}: not a bilinear product (depends on the grid)")
    out = np.empty((npts, 2 * len(comps), m), order="F")
    for c, (a, b) in enumerate(comps):
        out[:, 2 * c, :] = a.astype(np.float64)
        out[:, 2 * c + 1, :] = b.astype(np.float64)
    if opc == OP_TENSOR:
        return tensor_layout(out)
    return out


# ----------------------------------------------------------------------------
# compositions used by the bundle / linearised forms
# ----------------------------------------------------------------------------
def mhd_bundle(u, w, b, j, gradT, m_max_pad, engine=None):
    """(u x w, u x b, j x b, u . gradT) through the reference routines."""
    f = engine or (lambda op, x, y: c_oracle(op, x, y, m_max_pad))
    return f("cross", u, w), f("cross", u, b), f("cross", j, b), f("dot", u, gradT)


def cross_jvp(u, w, du, dw, m_max_pad, engine=None):
    """d(u x w) = du x w + u x dw (the cross product is bilinear, so exact)."""
    f = engine or (lambda op, x, y: c_oracle(op, x, y, m_max_pad))
    return f("cross", du, w) + f("cross", u, dw)


def _grid(m, N):
    th = 2.0 * np.pi * np.arange(N) / N
    n = np.arange(m)
    return np.cos(np.outer(n, th)), np.sin(np.outer(n, th))


def cross_vjp(u, w, cot, N=None):
    """Transpose of v=(du,dw) -> du x w + u x dw on the coefficient arrays.

    J^T c = ( S^T[W x (S D c)],  S^T[(S D c) x U] ) with S the synthesis on an
    alias-free grid, D = diag(1/N, 2/N, ...) the analysis scaling and
    U = S u, W = S w.  Returns (np, 12, m).
    """
    npts, _, m = u.shape
    if N is None:
        N = 3 * m
    C, S = _grid(m, N)

    def synth(V, scale):
        a = V[:, 0::2, :] * scale[None, None, :]
        b = V[:, 1::2, :] * scale[None, None, :]
        b = b.copy()
        b[:, :, 0] = 0.0
        return np.einsum("pkn,nj->pkj", a, C) + np.einsum("pkn,nj->pkj", b, S)

    def synthT(G):
        out = np.empty((npts, 2 * G.shape[1], m), order="F")
        out[:, 0::2, :] = np.einsum("pkj,nj->pkn", G, C)
        out[:, 1::2, :] = np.einsum("pkj,nj->pkn", G, S)
        out[:, 1::2, 0] = 0.0
        return out

    one = np.ones(m)
    dsc = np.full(m, 2.0 / N)
    dsc[0] = 1.0 / N
    U, W = synth(u, one), synth(w, one)
    Cg = synth(cot, dsc)
    gu = np.cross(W, Cg, axis=1)      # W x (S D c)
    gw = np.cross(Cg, U, axis=1)      # (S D c) x U
    return np.concatenate([synthT(gu), synthT(gw)], axis=1)


def rel_l2(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(x - ref) / (den if den > 0 else 1.0))
