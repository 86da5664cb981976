"""GPU parity of the same-pattern siblings of the dealiased products:
FFT_PAR_DIV_DCL (fft_parallel.F90:667-830), FFT_SCALAR_VECT_DCL (:1021-1220)
and FFT_TENSOR_DCL (:1543-1796, with and without opt_tension).

Bars: FP64 forms rel-L2 <= 1e-12 per output component against the
long-double oracle (FP64_TOL); split forms of the bilinear ones (scalar x
vector, tensor) <= 1e-7 with 3 slices (SPLIT_TOL), <= 1e-4 with 2 (HILO_TOL).
The quotients and the tension tensor depend on the grid and run on the
caller's grid N = 2*m_max_pad-1 only (the FAST and split forms refuse them).
"""
import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
SPLIT_TOL = 1e-7
HILO_TOL = 1e-4
DIVISOR_OFFSET = 4.0  # added to the mode-0 cosine of every divisor so that it stays away from 0


def dev(a):
    return sf.to_device(a)


def host(t):
    return sf.to_host(t)


def _sync():
    import torch

    torch.cuda.synchronize()


def _inputs(kind, npts, m, alpha, seed):
    _, n1, n2, _ = sf.KINDS[kind]
    V1 = R.synthetic_field(npts, n1, m, alpha, seed)
    V2 = R.synthetic_field(npts, n2, m, alpha, seed + 1)
    if kind in ("div", "svdiv"):
        V2[:, 0, 0] += DIVISOR_OFFSET
    return V1, V2


def _components(kind, a):
    """Output components (cos, sin slot pairs) of an output array, for per-component errors."""
    if kind in ("tensor", "tension"):
        return [a[k, :, 2 * l:2 * l + 2, :] for k in range(3) for l in range(3)]
    return [a[:, 2 * c:2 * c + 2, :] for c in range(a.shape[1] // 2)]


def _worst(kind, got, ref):
    return max(R.rel_l2(g, r) for g, r in zip(_components(kind, got), _components(kind, ref)))


KIND_NAMES = ["div", "svect", "svdiv", "tensor", "tension"]
CASES = [(1, 1, 1), (5, 2, 3), (33, 5, 7), (257, 16, 24), (130, 13, 19), (1000, 32, 48), (77, 64, 96)]


@pytest.mark.parametrize("kind", KIND_NAMES)
@pytest.mark.parametrize("npts,m,pad", CASES)
@pytest.mark.parametrize("algo", [sf.ALGO_GRID, sf.ALGO_AUTO])
def test_siblings_match_oracle(kind, npts, m, pad, algo):
    V1, V2 = _inputs(kind, npts, m, 0.2, 300 + m)
    ref = R.c_oracle(kind, V1, V2, pad)
    out = sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=pad, algo=algo)
    _sync()
    assert _worst(kind, host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("kind", ["svect", "tensor"])
@pytest.mark.parametrize("npts,m,pad", [(33, 5, 7), (257, 16, 24), (1000, 32, 48), (77, 64, 96), (50, 72, 108)])
def test_fast_form_of_the_bilinear_siblings(kind, npts, m, pad):
    V1, V2 = _inputs(kind, npts, m, 0.2, 400 + m)
    ref = R.c_oracle(kind, V1, V2, pad)
    out = sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=pad, algo=sf.ALGO_FAST)
    _sync()
    assert _worst(kind, host(out), ref) <= FP64_TOL


def test_tensor_beyond_the_fused_kernel():
    # m = 96: the tensor's nine outputs do not fit the fused kernel's shared memory; FAST (and AUTO)
    # take the two-kernel form, whose program kernel analyses the outputs in three groups.
    V1, V2 = _inputs("tensor", 20, 96, 0.1, 7)
    ref = R.c_oracle("tensor", V1, V2, 144)
    for algo in (sf.ALGO_FAST, sf.ALGO_AUTO):
        out = sf.product(sf.OP_TENSOR, dev(V1), dev(V2), m_max_pad=144, algo=algo)
        _sync()
        assert _worst("tensor", host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("kind", ["div", "svdiv", "tension"])
def test_grid_dependent_siblings_follow_the_grid(kind):
    # An explicit grid length changes these results (no dealiasing identity); GRID reproduces it.
    V1, V2 = _inputs(kind, 40, 8, 0.3, 11)
    for n_theta in (0, 30, 41):
        ref = R.c_oracle(kind, V1, V2, 12, n_theta=n_theta or None)
        out = sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=12, n_theta=n_theta, algo=sf.ALGO_GRID)
        _sync()
        assert _worst(kind, host(out), ref) <= FP64_TOL
    with pytest.raises(sf.SfnlError) as e:
        sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=12, algo=sf.ALGO_FAST)
    assert e.value.code == -4
    with pytest.raises(sf.SfnlError) as e:
        sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=12, split=sf.SPLIT_BF16X3)
    assert e.value.code == -4


@pytest.mark.parametrize("kind", ["svect", "tensor"])
@pytest.mark.parametrize("npts,m", [(28000, 16), (333, 5), (700, 32), (129, 33), (300, 64)])
def test_split_forms_of_the_bilinear_siblings(kind, npts, m):
    pad = 3 * m // 2
    V1, V2 = _inputs(kind, npts, m, 0.3, 500 + m)
    ref = R.fft_par(kind, V1, V2, pad) if npts > 2000 else R.c_oracle(kind, V1, V2, pad)
    op = sf.KINDS[kind][0]
    e3 = _worst(kind, host(sf.product(op, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X3)), ref)
    e2 = _worst(kind, host(sf.product(op, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X2)), ref)
    print(f"{kind} np={npts} m={m}: bf16x3 {e3:.2e}  bf16x2 {e2:.2e}")
    assert e3 <= SPLIT_TOL
    assert e2 <= HILO_TOL


@pytest.mark.parametrize("kind", KIND_NAMES)
def test_reference_signature_on_host_arrays(kind):
    npts, m, pad = 61, 8, 12
    V1, V2 = _inputs(kind, npts, m, 0.2, 21)
    ref = R.c_oracle(kind, V1, V2, pad)
    out = np.zeros(ref.shape, order="F")
    temps = np.full(3, -1.0)
    bloc = npts + 3
    if kind == "div":
        sf.FFT_PAR_DIV_DCL(None, V1, V2, out, 1, bloc, pad, temps)
    elif kind in ("svect", "svdiv"):
        sf.FFT_SCALAR_VECT_DCL(None, V1, V2, out, 1 if kind == "svect" else 2, 1, bloc, pad, temps)
    else:
        sf.FFT_TENSOR_DCL(None, V1, V2, out, 1, bloc, pad, temps, opt_tension=True if kind == "tension" else None)
    assert _worst(kind, out, ref) <= FP64_TOL
    # temps(1) = host<->device copy seconds, temps(2) = kernel seconds, temps(3) = 0 (nothing repacked)
    assert temps[0] > 0.0 and temps[1] > 0.0 and temps[2] == 0.0


@pytest.mark.parametrize("kind", ["svect", "tensor", "tension"])
def test_reference_signature_on_device_tensors(kind):
    npts, m, pad = 45, 16, 24
    V1, V2 = _inputs(kind, npts, m, 0.2, 31)
    ref = R.c_oracle(kind, V1, V2, pad)
    out = sf.out_empty(sf.KINDS[kind][0], npts, m)
    if kind == "svect":
        sf.FFT_SCALAR_VECT_DCL(None, dev(V1), dev(V2), out, 1, 1, npts, pad)
    else:
        sf.FFT_TENSOR_DCL(None, dev(V1), dev(V2), out, 1, npts, pad, opt_tension=True if kind == "tension" else None)
    _sync()
    assert _worst(kind, host(out), ref) <= FP64_TOL


def test_host_tensor_entry_point_in_chunks():
    # More points than one chunk of the host pipeline holds: the (3, np, 6, m) layout is cut by points.
    npts, m, pad = 150_000, 32, 48
    V1, V2 = _inputs("tensor", npts, m, 0.2, 41)
    out = np.zeros((3, npts, 6, m), order="F")
    sf.FFT_TENSOR_DCL(None, V1, V2, out, 1, npts, pad)
    ref = R.fft_par("tensor", V1, V2, pad, workers=8)
    assert _worst("tensor", out, ref) <= FP64_TOL


def test_full_size_identities():
    # Size-independent properties at the 100k-point, m=64 size: trace(u (x) v) = u . v, the tensor's
    # rows are the scalar x vector products u_k v, and a constant scalar scales every mode.
    import torch

    npts, m, pad = 100_000, 64, 96
    U = R.synthetic_field(npts, 6, m, 0.1, 51)
    V = R.synthetic_field(npts, 6, m, 0.1, 52)
    u, v = dev(U), dev(V)
    t = sf.tensor(u, v, m_max_pad=pad)
    d = sf.product(sf.OP_DOT, u, v, m_max_pad=pad)
    trace = t[0, :, 0:2, :] + t[1, :, 2:4, :] + t[2, :, 4:6, :]
    assert float((trace - d).norm() / d.norm()) <= 1e-13
    for k in range(3):
        s = sf.to_device(np.asfortranarray(U[:, 2 * k:2 * k + 2, :]))
        sv = sf.scalar_vect(v, s, pb=1, m_max_pad=pad)
        assert float((sv - t[k]).norm() / t[k].norm()) <= 1e-13
    c = np.zeros((npts, 2, m), order="F")
    c[:, 0, 0] = 2.5
    sc = sf.scalar_vect(v, dev(c), pb=1, m_max_pad=pad)
    q = sf.scalar_vect(v, dev(c), pb=2, m_max_pad=pad)
    torch.cuda.synchronize()
    assert float((sc - 2.5 * v).norm() / v.norm()) <= 1e-13
    assert float((q - v / 2.5).norm() / v.norm()) <= 1e-13
