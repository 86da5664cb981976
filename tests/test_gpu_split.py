"""Split-precision (tcgen05, bf16-sliced) forms against the FP64 oracle.

Bar: rel-L2 <= 1e-7 per output array for the 3-slice form
(SPLIT_TOL).  The 2-slice "bf16 hi/lo" form is reported and held to 1e-4.
"""
import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-7
HILO_TOL = 1e-4


def dev(a):
    return sf.to_device(a)


def host(t):
    return sf.to_host(t)


@pytest.mark.parametrize("op", [0, 1, 2])
@pytest.mark.parametrize("npts,m", [(28000, 16), (1000, 1), (333, 5), (517, 17), (700, 32), (129, 33), (300, 64)])
def test_split3_products(op, npts, m):
    name = ("cross", "dot", "prod")[op]
    nsl = 2 if op == 2 else 6
    pad = 3 * m // 2 if m > 1 else 1
    V1 = R.synthetic_field(npts, nsl, m, 0.3, 500 + m)
    V2 = R.synthetic_field(npts, nsl, m, 0.3, 600 + m)
    ref = R.fft_par(name, V1, V2, pad) if npts > 2000 else R.c_oracle(name, V1, V2, pad)
    out = host(sf.product(op, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X3))
    assert R.rel_l2(out, ref) <= SPLIT_TOL


@pytest.mark.parametrize("alpha", [0.02, 0.05, 0.1, 0.2, 0.3, 0.5])
def test_split_decay_sweep_28k_points(alpha):
    # the split-precision form of the 28k-point, m=16 cross product, decay swept 0.02..0.5
    npts, m, pad = 28000, 16, 24
    V1 = R.synthetic_field(npts, 6, m, alpha, 700)
    V2 = R.synthetic_field(npts, 6, m, alpha, 701)
    ref = R.fft_par("cross", V1, V2, pad)
    e3 = R.rel_l2(host(sf.product(0, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X3)), ref)
    e2 = R.rel_l2(host(sf.product(0, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X2)), ref)
    print(f"alpha={alpha}: bf16x3 {e3:.2e}  bf16x2 {e2:.2e}")
    assert e3 <= SPLIT_TOL
    assert e2 <= HILO_TOL


def test_split_bundle_m64():
    npts, m, pad = 1000, 64, 96
    f = [R.synthetic_field(npts, 6, m, 0.1, 800 + i) for i in range(5)]
    refs = R.mhd_bundle(*f, pad, engine=lambda op, x, y: R.fft_par(op, x, y, pad))
    outs = sf.bundle_mhd(*[dev(x) for x in f], m_max_pad=pad, split=sf.SPLIT_BF16X3)
    for o, r in zip(outs, refs):
        assert R.rel_l2(host(o), r) <= SPLIT_TOL


def test_split_mhd_linearised_against_the_oracle():
    # linearised u x w and u x b about (u, w, b): the JVP against the oracle's cross products
    # (du x w + u x dw, du x b + u x db), the VJP against the oracle's transposes of both
    npts, m, k, pad = 400, 32, 3, 48
    u, w, b = (R.synthetic_field(npts, 6, m, 0.2, 900 + i) for i in range(3))
    v = np.empty((npts, 18, m, k), order="F")
    c = np.empty((npts, 12, m, k), order="F")
    for t in range(k):
        v[..., t] = R.synthetic_field(npts, 18, m, 0.2, 910 + t)
        c[..., t] = R.synthetic_field(npts, 12, m, 0.2, 920 + t)
    U, W, B = dev(u), dev(w), dev(b)
    jvs = host(sf.mhd_jvp(U, W, B, dev(v), m_max_pad=pad, split=sf.SPLIT_BF16X3))
    jts = host(sf.mhd_vjp(U, W, B, dev(c), m_max_pad=pad, split=sf.SPLIT_BF16X3))
    for t in range(k):
        du, dw, db = v[:, 0:6, :, t], v[:, 6:12, :, t], v[:, 12:18, :, t]
        jv = np.concatenate([R.cross_jvp(u, w, du, dw, pad), R.cross_jvp(u, b, du, db, pad)], axis=1)
        g1 = R.cross_vjp(u, w, np.asfortranarray(c[:, 0:6, :, t]))
        g2 = R.cross_vjp(u, b, np.asfortranarray(c[:, 6:12, :, t]))
        jt = np.concatenate([g1[:, :6] + g2[:, :6], g1[:, 6:], g2[:, 6:]], axis=1)
        assert R.rel_l2(jvs[..., t], jv) <= SPLIT_TOL
        assert R.rel_l2(jts[..., t], jt) <= SPLIT_TOL


def test_split_refuses_aliasing_pad_and_large_m():
    V = dev(R.synthetic_field(10, 6, 8, 0.1, 1))
    with pytest.raises(sf.SfnlError) as e:
        sf.product(0, V, V, m_max_pad=8, split=sf.SPLIT_BF16X3)
    assert e.value.code == -3
    W = dev(R.synthetic_field(4, 6, 80, 0.1, 1))
    with pytest.raises(sf.SfnlError) as e:
        sf.product(0, W, W, m_max_pad=120, split=sf.SPLIT_BF16X3)
    assert e.value.code == -4


def test_split_timeout_status_is_reported_once_and_cleared():
    # Host-side injection: the status word is marked as a split kernel marks it when a bounded wait on
    # its tensor-core operations gives up; no device wait is made to run out.
    L = sf.lib()
    npts, m, pad = 200, 16, 24
    V1 = R.synthetic_field(npts, 6, m, 0.3, 901)
    V2 = R.synthetic_field(npts, 6, m, 0.3, 902)
    ref = R.c_oracle("cross", V1, V2, pad)
    assert L.sfnl_test_inject_timeout() == 0
    with pytest.raises(sf.SfnlError) as e:
        sf.product(0, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X3)
    assert e.value.code == -8 and "tensor-core" in str(e.value)
    out = host(sf.product(0, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X3))  # cleared
    assert R.rel_l2(out, ref) <= SPLIT_TOL
    # the FP64 forms do not use the word: an injected status waits for the next split call
    assert L.sfnl_test_inject_timeout() == 0
    fp = host(sf.product(0, dev(V1), dev(V2), m_max_pad=pad))
    assert R.rel_l2(fp, ref) <= 1e-12
    with pytest.raises(sf.SfnlError) as e:
        sf.product(0, dev(V1), dev(V2), m_max_pad=pad, split=sf.SPLIT_BF16X2)
    assert e.value.code == -8
