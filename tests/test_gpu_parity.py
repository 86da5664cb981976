"""GPU parity of the all-FP64 forms against the CPU oracle.

Bar: rel-L2 <= 1e-12 per output array against the long-double
restatement of fft_parallel.F90 (FP64_TOL below).  Every call goes through
the C-ABI library (ctypes), on device tensors or on host arrays.
"""
import glob
import os

import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ALGOS = [sf.ALGO_GRID, sf.ALGO_AUTO]


def dev(a):
    return sf.to_device(a)


def host(t):
    return sf.to_host(t)


def _sync():
    import torch

    torch.cuda.synchronize()


PRODUCT_FIXTURES = sorted(p for p in glob.glob(os.path.join(GOLD, "*.npz"))
                          if not os.path.basename(p).startswith(("real_", "maxvel_")))  # synthesis: test_gpu_synthesis


@pytest.mark.parametrize("path", PRODUCT_FIXTURES)
@pytest.mark.parametrize("algo", ALGOS)
def test_golden_fixtures(path, algo):
    z = np.load(path)
    npts, m, pad, procs = (int(v) for v in z["meta"])
    op = sf.KINDS[str(z["op"])][0]
    out = sf.product(op, dev(z["V1"]), dev(z["V2"]), m_max_pad=pad, algo=algo)
    _sync()
    assert R.rel_l2(host(out), z["out"]) <= FP64_TOL


CASES = [  # np, m, m_max_pad
    (1, 1, 1), (5, 2, 3), (33, 5, 7), (257, 16, 24), (130, 13, 19), (1000, 32, 48), (77, 64, 96),
]


@pytest.mark.parametrize("op", [0, 1, 2])
@pytest.mark.parametrize("npts,m,pad", CASES)
@pytest.mark.parametrize("algo", ALGOS)
def test_products_match_oracle(op, npts, m, pad, algo):
    name = ("cross", "dot", "prod")[op]
    nsl = 2 if op == 2 else 6
    V1 = R.synthetic_field(npts, nsl, m, 0.2, 100 + m)
    V2 = R.synthetic_field(npts, nsl, m, 0.2, 200 + m)
    ref = R.c_oracle(name, V1, V2, pad)
    out = sf.product(op, dev(V1), dev(V2), m_max_pad=pad, algo=algo)
    _sync()
    assert R.rel_l2(host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("npts,m,pad,n_theta", [(64, 16, 24, 48), (50, 7, 10, 22), (40, 8, 8, 0)])
def test_grid_form_follows_the_grid(npts, m, pad, n_theta):
    # GRID on an explicit grid, including the aliasing pad m_max_pad = m_max.
    V1 = R.synthetic_field(npts, 6, m, 0.0, 1)
    V2 = R.synthetic_field(npts, 6, m, 0.0, 2)
    ref = R.c_oracle("cross", V1, V2, pad, n_theta=n_theta or None)
    out = sf.product(0, dev(V1), dev(V2), m_max_pad=pad, n_theta=n_theta, algo=sf.ALGO_GRID)
    _sync()
    assert R.rel_l2(host(out), ref) <= FP64_TOL


def test_fast_form_refuses_aliasing_pad():
    V = dev(R.synthetic_field(10, 6, 8, 0.1, 1))
    with pytest.raises(sf.SfnlError) as e:
        sf.product(0, V, V, m_max_pad=8, algo=sf.ALGO_FAST)
    assert e.value.code == -3


@pytest.mark.parametrize("kind", ["cross", "dot", "prod"])
def test_reference_signature_on_host_arrays(kind):
    m, npts = 12, 301
    nsl = 2 if kind == "prod" else 6
    V1 = R.synthetic_field(npts, nsl, m, 0.3, 11)
    V2 = R.synthetic_field(npts, nsl, m, 0.3, 12)
    out = np.zeros((npts, 6 if kind == "cross" else 2, m), order="F")
    temps = np.full(3, 7.0)
    fn = {"cross": sf.FFT_PAR_CROSS_PROD_DCL, "dot": sf.FFT_PAR_DOT_PROD_DCL, "prod": sf.FFT_PAR_PROD_DCL}[kind]
    bloc = npts + 1  # the callers' bloc_size = np/nb_procs+1
    fn(None, V1, V2, out, 1, bloc, 3 * m // 2, temps)
    assert R.rel_l2(out, R.c_oracle(kind, V1, V2, 3 * m // 2)) <= FP64_TOL
    # zeroed on entry, then device seconds: copies (where the reference has its all-to-alls), kernels, 0
    assert temps[0] > 0 and temps[0] < 7.0 and temps[1] > 0 and temps[1] < 7.0 and temps[2] == 0.0


def test_reference_signature_on_device_tensors():
    m, npts = 8, 100
    V1 = R.synthetic_field(npts, 6, m, 0.3, 13)
    V2 = R.synthetic_field(npts, 6, m, 0.3, 14)
    out = sf.fortran_empty(npts, 6, m)
    sf.FFT_PAR_CROSS_PROD_DCL(None, dev(V1), dev(V2), out, 1, npts + 1, 12)
    _sync()
    assert R.rel_l2(host(out), R.c_oracle("cross", V1, V2, 12)) <= FP64_TOL


@pytest.mark.parametrize("npts,m", [(200, 8), (65, 21), (61, 64), (200, 64)])
@pytest.mark.parametrize("algo", ALGOS)
def test_mhd_bundle(npts, m, algo):
    pad = 3 * m // 2
    f = [R.synthetic_field(npts, 6, m, 0.1, 300 + i) for i in range(5)]
    refs = R.mhd_bundle(*f, pad)
    outs = sf.bundle_mhd(*[dev(x) for x in f], m_max_pad=pad, algo=algo)
    _sync()
    for o, r in zip(outs, refs):
        assert R.rel_l2(host(o), r) <= FP64_TOL


@pytest.mark.parametrize("npts", [1, 7, 61, 3001, 100_003, 2, 64, 3002, 100_002])
def test_bundle_kernels_agree(npts):
    # the two kernels of the m = 64 bundle (grid split into its residue classes; one 192-angle transform)
    # against each other, and against the oracle where it is cheap; odd counts take the 8-byte copies,
    # even ones the residue kernel's bulk tensor copies (2 and 3002: a last tile past np, filled with zeros)
    m, pad = 64, 96
    f = [R.synthetic_field(npts, 6, m, 0.1, 700 + i) for i in range(5)]
    d = [dev(x) for x in f]
    prev = sf.set_bundle_kernel(sf.BUNDLE_THIRD_FOLD)
    try:
        tf = [host(o) for o in sf.bundle_mhd(*d, m_max_pad=pad)]
        assert sf.set_bundle_kernel(sf.BUNDLE_RESIDUE) == sf.BUNDLE_THIRD_FOLD
        r3 = [host(o) for o in sf.bundle_mhd(*d, m_max_pad=pad)]
    finally:
        sf.set_bundle_kernel(prev)
    refs = R.mhd_bundle(*f, pad) if npts <= 3002 else None
    for i in range(4):
        assert R.rel_l2(r3[i], tf[i]) <= 1e-13
        if refs is not None:
            assert R.rel_l2(r3[i], refs[i]) <= FP64_TOL


def test_bundle_unaligned_inputs_take_the_copy_path():
    # inputs 8 bytes off a 16-byte boundary cannot feed the bulk tensor copies: with an even point count the
    # residue kernel stages them with 8-byte cp.async copies instead, to the same results
    import torch

    npts, m, pad = 64, 64, 96
    f = [R.synthetic_field(npts, 6, m, 0.1, 720 + i) for i in range(5)]
    d = []
    for x in f:
        t = dev(x)
        buf = torch.empty(t.numel() + 1, dtype=torch.float64, device="cuda")
        v = buf[1:].view(m, 6, npts).permute(2, 1, 0)  # Fortran strides, base 8 bytes past the allocation
        v.copy_(t)
        assert v.data_ptr() % 16 == 8
        d.append(v)
    outs = [host(o) for o in sf.bundle_mhd(*d, m_max_pad=pad)]
    for o, r in zip(outs, R.mhd_bundle(*f, pad)):
        assert R.rel_l2(o, r) <= FP64_TOL


def test_bundle_reports_a_wait_that_gave_up():
    # Host-side injection: the wait-status word is marked as the m = 64 bundle kernel marks it when a bounded
    # wait on its bulk copies gives up; no device wait is made to run out.  The next bundle call reports
    # it and clears it.
    npts, m, pad = 64, 64, 96
    f = [R.synthetic_field(npts, 6, m, 0.1, 710 + i) for i in range(5)]
    d = [dev(x) for x in f]
    assert sf.lib().sfnl_test_inject_timeout() == 0
    with pytest.raises(sf.SfnlError) as e:
        sf.bundle_mhd(*d, m_max_pad=pad)
    assert e.value.code == -8 and "bulk copies" in str(e.value)
    outs = [host(o) for o in sf.bundle_mhd(*d, m_max_pad=pad)]  # cleared
    for o, r in zip(outs, R.mhd_bundle(*f, pad)):
        assert R.rel_l2(o, r) <= FP64_TOL


@pytest.mark.parametrize("npts,m", [(90, 10), (3001, 64)])
def test_host_bundle_entry_point(npts, m):
    import ctypes

    pad = 3 * m // 2
    f = [R.synthetic_field(npts, 6, m, 0.1, 400 + i) for i in range(5)]
    outs = [np.zeros((npts, 6, m), order="F") for _ in range(3)] + [np.zeros((npts, 2, m), order="F")]
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    rc = sf.lib().sfnl_bundle_mhd_host(*[P(a) for a in f + outs], npts, m, pad, 0)
    assert rc == 0, sf.last_error()
    for o, r in zip(outs, R.mhd_bundle(*f, pad)):
        assert R.rel_l2(o, r) <= FP64_TOL


def _batched(npts, nslot, m, k, alpha, seed):
    x = np.empty((npts, nslot, m, k), order="F")
    for t in range(k):
        x[:, :, :, t] = R.synthetic_field(npts, nslot, m, alpha, seed + t)
    return x


@pytest.mark.parametrize("npts,m,k", [(120, 8, 3), (33, 17, 1), (41, 64, 2), (29, 90, 2), (25, 96, 1)])
def test_cross_jvp_matches_linearisation(npts, m, k):
    pad = 3 * m // 2
    u = R.synthetic_field(npts, 6, m, 0.2, 1)
    w = R.synthetic_field(npts, 6, m, 0.2, 2)
    tan = _batched(npts, 12, m, k, 0.2, 10)
    out = host(sf.cross_jvp(dev(u), dev(w), dev(tan), m_max_pad=pad))
    for t in range(k):
        du = np.asfortranarray(tan[:, :6, :, t])
        dw = np.asfortranarray(tan[:, 6:, :, t])
        assert R.rel_l2(out[:, :, :, t], R.cross_jvp(u, w, du, dw, pad)) <= FP64_TOL


def test_cross_jvp_central_finite_differences():
    # N(u + h du, w + h dw) - N(u - h du, w - h dw) = 2h J(du, dw) exactly for a
    # bilinear N; the check bounds rounding at ~eps/h (h = 1e-6).
    npts, m, h = 700, 32, 1e-6
    pad = 48
    u = R.synthetic_field(npts, 6, m, 0.2, 21)
    w = R.synthetic_field(npts, 6, m, 0.2, 22)
    du = R.synthetic_field(npts, 6, m, 0.2, 23)
    dw = R.synthetic_field(npts, 6, m, 0.2, 24)
    tan = np.asfortranarray(np.concatenate([du, dw], axis=1))
    jv = host(sf.cross_jvp(dev(u), dev(w), dev(tan), m_max_pad=pad))[..., 0]
    plus = host(sf.product(0, dev(u + h * du), dev(w + h * dw), m_max_pad=pad))
    minus = host(sf.product(0, dev(u - h * du), dev(w - h * dw), m_max_pad=pad))
    fd = (plus - minus) / (2 * h)
    assert R.rel_l2(jv, fd) < 1e-8


@pytest.mark.parametrize("npts,m,k", [(150, 8, 2), (40, 32, 1), (37, 64, 2)])
def test_cross_vjp_dot_product_identity(npts, m, k):
    pad = 3 * m // 2
    u = R.synthetic_field(npts, 6, m, 0.2, 31)
    w = R.synthetic_field(npts, 6, m, 0.2, 32)
    v = _batched(npts, 12, m, k, 0.2, 40)
    c = _batched(npts, 6, m, k, 0.2, 50)
    jv = host(sf.cross_jvp(dev(u), dev(w), dev(v), m_max_pad=pad))
    jtc = host(sf.cross_vjp(dev(u), dev(w), dev(c), m_max_pad=pad))
    for t in range(k):
        lhs = np.dot(jv[..., t].ravel(), c[..., t].ravel())
        rhs = np.dot(v[..., t].ravel(), jtc[..., t].ravel())
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.linalg.norm(jv[..., t]) * np.linalg.norm(c[..., t]))
        assert R.rel_l2(jtc[..., t], R.cross_vjp(u, w, np.asfortranarray(c[..., t]))) <= FP64_TOL


@pytest.mark.parametrize("npts,m,k", [(90, 12, 2), (43, 64, 2), (27, 90, 2)])
def test_mhd_jvp_vjp(npts, m, k):
    pad = 3 * m // 2
    u, w, b = (R.synthetic_field(npts, 6, m, 0.2, 60 + i) for i in range(3))
    v = _batched(npts, 18, m, k, 0.2, 70)
    c = _batched(npts, 12, m, k, 0.2, 80)
    jv = host(sf.mhd_jvp(dev(u), dev(w), dev(b), dev(v), m_max_pad=pad))
    jtc = host(sf.mhd_vjp(dev(u), dev(w), dev(b), dev(c), m_max_pad=pad))
    for t in range(k):
        du, dw, db = (np.asfortranarray(v[:, 6 * i:6 * i + 6, :, t]) for i in range(3))
        assert R.rel_l2(jv[:, :6, :, t], R.cross_jvp(u, w, du, dw, pad)) <= FP64_TOL
        assert R.rel_l2(jv[:, 6:, :, t], R.cross_jvp(u, b, du, db, pad)) <= FP64_TOL
        lhs = np.dot(jv[..., t].ravel(), c[..., t].ravel())
        rhs = np.dot(v[..., t].ravel(), jtc[..., t].ravel())
        assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(jv[..., t]) * np.linalg.norm(c[..., t])


def test_finite_check_mode():
    V1 = R.synthetic_field(64, 6, 4, 0.1, 1)
    V1[3, 2, 1] = np.nan
    V2 = R.synthetic_field(64, 6, 4, 0.1, 2)
    sf.set_check_finite(True)
    try:
        with pytest.raises(sf.SfnlError) as e:
            sf.product(0, dev(V1), dev(V2), m_max_pad=6)
        assert e.value.code == -6
    finally:
        sf.set_check_finite(False)


# m = 100: the whole grid, odd tile count; 128: the whole grid with the third fold; 256 and 512: the grid's
# three residue classes
LARGE = [(37, 100, 150), (20, 128, 192), (9, 256, 384), (5, 512, 768)]


@pytest.mark.parametrize("op", [0, 1, 2])
@pytest.mark.parametrize("npts,m,pad", LARGE)
@pytest.mark.parametrize("algo", [sf.ALGO_AUTO, sf.ALGO_FAST])
def test_large_m_products(op, npts, m, pad, algo):
    # m beyond what one CTA holds: the two-kernel FAST form (synthesis to grid values, then program + analysis)
    name = ("cross", "dot", "prod")[op]
    nsl = 2 if op == 2 else 6
    V1 = R.synthetic_field(npts, nsl, m, 0.05, 900 + m)
    V2 = R.synthetic_field(npts, nsl, m, 0.05, 950 + m)
    out = sf.product(op, dev(V1), dev(V2), m_max_pad=pad, algo=algo)
    _sync()
    assert R.rel_l2(host(out), R.c_oracle(name, V1, V2, pad)) <= FP64_TOL


@pytest.mark.parametrize("kind", ["svect", "tensor"])
def test_large_m_siblings(kind):
    npts, m, pad = 11, 200, 300
    _, n1, n2, _ = sf.KINDS[kind]
    V1 = R.synthetic_field(npts, n1, m, 0.05, 31)
    V2 = R.synthetic_field(npts, n2, m, 0.05, 32)
    out = sf.product(sf.KINDS[kind][0], dev(V1), dev(V2), m_max_pad=pad, algo=sf.ALGO_FAST)
    _sync()
    assert R.rel_l2(host(out), R.c_oracle(kind, V1, V2, pad)) <= FP64_TOL


def test_large_m_linearised_batched():
    # the 16-tangent linearised configuration's shape (m = 256), on few points and 3 tangents
    npts, m, k, pad = 13, 256, 3, 384
    u, w, b = (R.synthetic_field(npts, 6, m, 0.05, 70 + i) for i in range(3))
    v = _batched(npts, 18, m, k, 0.05, 80)
    c = _batched(npts, 12, m, k, 0.05, 90)
    jv = host(sf.mhd_jvp(dev(u), dev(w), dev(b), dev(v), m_max_pad=pad))
    jtc = host(sf.mhd_vjp(dev(u), dev(w), dev(b), dev(c), m_max_pad=pad))
    for t in range(k):
        du, dw, db = (np.asfortranarray(v[:, 6 * i:6 * i + 6, :, t]) for i in range(3))
        assert R.rel_l2(jv[:, :6, :, t], R.cross_jvp(u, w, du, dw, pad)) <= FP64_TOL
        assert R.rel_l2(jv[:, 6:, :, t], R.cross_jvp(u, b, du, db, pad)) <= FP64_TOL
        lhs = np.dot(jv[..., t].ravel(), c[..., t].ravel())
        rhs = np.dot(v[..., t].ravel(), jtc[..., t].ravel())
        assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(jv[..., t]) * np.linalg.norm(c[..., t])


@pytest.mark.parametrize("npts,m", [(21, 128), (6, 300)])
def test_large_m_bundle(npts, m):
    # ten outputs: four output groups of the program kernel over one set of grid values
    pad = 3 * m // 2
    f = [R.synthetic_field(npts, 6, m, 0.05, 500 + i) for i in range(5)]
    outs = sf.bundle_mhd(*[dev(x) for x in f], m_max_pad=pad, algo=sf.ALGO_FAST)
    _sync()
    for o, r in zip(outs, R.mhd_bundle(*f, pad)):
        assert R.rel_l2(host(o), r) <= FP64_TOL


@pytest.mark.parametrize("npts,m,k", [(17, 112, 2), (10, 160, 1)])
def test_large_m_cross_jvp_vjp(npts, m, k):
    pad = 3 * m // 2
    u = R.synthetic_field(npts, 6, m, 0.05, 531)
    w = R.synthetic_field(npts, 6, m, 0.05, 532)
    v = _batched(npts, 12, m, k, 0.05, 540)
    c = _batched(npts, 6, m, k, 0.05, 550)
    jv = host(sf.cross_jvp(dev(u), dev(w), dev(v), m_max_pad=pad))
    jtc = host(sf.cross_vjp(dev(u), dev(w), dev(c), m_max_pad=pad))
    for t in range(k):
        du, dw = (np.asfortranarray(v[:, 6 * i:6 * i + 6, :, t]) for i in range(2))
        assert R.rel_l2(jv[..., t], R.cross_jvp(u, w, du, dw, pad)) <= FP64_TOL
        assert R.rel_l2(jtc[..., t], R.cross_vjp(u, w, np.asfortranarray(c[..., t]))) <= FP64_TOL


def test_large_m_linearised_point_chunks():
    # the base state is synthesised once per point chunk and the tangents per batch entry: more points
    # than one chunk of grid values (about 9.7k points at m = 256 for the 18 fields of the MHD JVP)
    npts, m, k, pad = 12_001, 256, 2, 384
    u, w, b = (R.synthetic_field(npts, 6, m, 0.05, 570 + i) for i in range(3))
    v = _batched(npts, 18, m, k, 0.05, 580)
    jv = host(sf.mhd_jvp(dev(u), dev(w), dev(b), dev(v), m_max_pad=pad))
    eng = lambda op, x, y: R.fft_par(op, x, y, pad, workers=8)  # noqa: E731
    for t in range(k):
        du, dw, db = (np.asfortranarray(v[:, 6 * i:6 * i + 6, :, t]) for i in range(3))
        assert R.rel_l2(jv[:, :6, :, t], R.cross_jvp(u, w, du, dw, pad, engine=eng)) <= FP64_TOL
        assert R.rel_l2(jv[:, 6:, :, t], R.cross_jvp(u, b, du, db, pad, engine=eng)) <= FP64_TOL


@pytest.mark.parametrize("m,pad", [(128, 192), (256, 384)])
def test_large_m_small_workspace_bound(m, pad):
    # a test-only workspace bound (2 MB) makes the large-m form run many point chunks (and, for the tangents,
    # batch groups of one entry): at m = 256 the residues' coefficients and sums, at m = 128 the grid values
    npts, k = 1201, 3
    u, w = (R.synthetic_field(npts, 6, m, 0.05, 600 + i) for i in range(2))
    tan = _batched(npts, 12, m, k, 0.05, 610)
    ref_cross = R.fft_par("cross", u, w, pad, workers=8)
    ref_jvp = host(sf.cross_jvp(dev(u), dev(w), dev(tan), m_max_pad=pad))  # production bounds: one chunk
    assert sf.lib().sfnl_test_large_workspace_cap(2 << 20) == 0
    try:
        out = host(sf.product(0, dev(u), dev(w), m_max_pad=pad, algo=sf.ALGO_FAST))
        jvp = host(sf.cross_jvp(dev(u), dev(w), dev(tan), m_max_pad=pad))
    finally:
        assert sf.lib().sfnl_test_large_workspace_cap(0) == 0
    assert R.rel_l2(out, ref_cross) <= FP64_TOL
    assert R.rel_l2(jvp, ref_jvp) <= 1e-13


@pytest.mark.parametrize("m,pad,splits", [(256, 384, (3, 6, 12)), (512, 768, (3, 6, 12)), (128, 192, (0, 3, 6))])
def test_large_m_residue_classes(m, pad, splits):
    # the large-m form on the grid split into R residue classes (a test hook forces R; 0: the whole grid):
    # every split against the oracle, and the cross JVP of every split against the first one
    npts, k = 203, 2
    u, w = (R.synthetic_field(npts, 6, m, 0.05, 620 + i) for i in range(2))
    tan = _batched(npts, 12, m, k, 0.05, 630)
    ref = R.fft_par("cross", u, w, pad, workers=8)
    jvps = []
    try:
        for split in splits:
            assert sf.lib().sfnl_test_large_residues(split) == 0
            out = host(sf.product(0, dev(u), dev(w), m_max_pad=pad, algo=sf.ALGO_FAST))
            assert R.rel_l2(out, ref) <= FP64_TOL, split
            jvps.append(host(sf.cross_jvp(dev(u), dev(w), dev(tan), m_max_pad=pad)))
    finally:
        assert sf.lib().sfnl_test_large_residues(0) == 0
    for jv in jvps[1:]:
        assert R.rel_l2(jv, jvps[0]) <= 1e-13


def test_large_m_point_chunks():
    # more points than one workspace chunk of grid values holds (about 29k points at m = 256)
    npts, m, pad = 70_001, 256, 384
    V1 = R.synthetic_field(npts, 6, m, 0.05, 41)
    V2 = R.synthetic_field(npts, 6, m, 0.05, 42)
    out = host(sf.product(0, dev(V1), dev(V2), m_max_pad=pad, algo=sf.ALGO_FAST))
    assert R.rel_l2(out, R.fft_par("cross", V1, V2, pad, workers=8)) <= FP64_TOL


def _ranks_run(kind, V1, V2, P, pad):
    """The mode-distributed path of the reference-signature routines with P emulated Fourier ranks: pack
    on every rank, the all-to-all as a buffer transpose, the block's product on the GPU, back, unpack."""
    import ctypes

    L = sf.lib()
    op, nsl1, nsl2, nout = sf.KINDS[kind]
    tensor = kind in ("tensor", "tension")
    ew = 3 if tensor else 1
    npts, _, m = V1.shape
    mc, bloc = m // P, npts // P + 1
    ptr = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731

    def pack(V, nsl, r):
        loc = np.asfortranarray(V[:, :, r * mc:(r + 1) * mc])
        buf = np.zeros(P * mc * nsl * bloc)
        assert L.sfnl_fft_par_pack_modes(ptr(loc), ptr(buf), npts, nsl, mc, P, bloc, 1) == 0
        return buf.reshape(P, -1)

    s1 = [pack(V1, nsl1, r) for r in range(P)]
    s2 = [pack(V2, nsl2, r) for r in range(P)]
    backs = []
    for q in range(P):
        r1 = np.ascontiguousarray(np.stack([s1[r][q] for r in range(P)]))
        r2 = np.ascontiguousarray(np.stack([s2[r][q] for r in range(P)]))
        back = np.zeros(P * mc * nout * bloc * ew)
        temps = np.zeros(3)
        rc = L.sfnl_fft_par_block(op, ptr(r1), ptr(r2), ptr(back), bloc, mc, P, pad, ptr(temps))
        assert rc == 0, sf.last_error()
        assert temps[1] > 0.0
        backs.append(back.reshape(P, -1))
    outs = []
    for r in range(P):
        got = np.ascontiguousarray(np.stack([backs[q][r] for q in range(P)]))
        shape = (3, npts, 6, mc) if tensor else (npts, nout, mc)
        out = np.zeros(shape, order="F")
        assert L.sfnl_fft_par_unpack_modes(ptr(got), ptr(out), npts, nout, mc, P, bloc, ew) == 0
        outs.append(out)
    return outs


@pytest.mark.parametrize("kind,P,npts,m", [("cross", 2, 61, 8), ("cross", 3, 100, 12), ("dot", 3, 47, 9),
                                           ("prod", 2, 33, 16), ("svect", 2, 29, 6), ("div", 3, 20, 6),
                                           ("tensor", 2, 25, 4), ("tension", 3, 17, 6)])
def test_mode_distributed_block_path(kind, P, npts, m):
    # the body of FFT_PAR_*_DCL between and around its two MPI_ALLTOALLs (fft_parallel.F90:205-217, :306-324),
    # each emulated rank's block on the GPU, against the oracle on the global arrays
    _, nsl1, nsl2, _ = sf.KINDS[kind]
    V1 = R.synthetic_field(npts, nsl1, m, 0.2, 301)
    V2 = R.synthetic_field(npts, nsl2, m, 0.2, 302)
    if kind == "div":
        V2[:, 0, 0] += 4.0
    pad = 3 * m // 2
    ref = R.c_oracle(kind, V1, V2, pad)
    mc = m // P
    for r, out in enumerate(_ranks_run(kind, V1, V2, P, pad)):
        assert R.rel_l2(out, ref[..., r * mc:(r + 1) * mc]) <= FP64_TOL, r


def test_cross_jacobian_operator_drives_a_krylov_svd():
    # the linearised term as a Krylov operator (matvec = JVP, rmatvec = VJP): the leading singular values
    # that scipy's svds finds through it match those of the dense Jacobian built column by column from
    # the oracle's bilinear products
    from scipy.sparse.linalg import svds

    from sfemans_b200.linop import CrossJacobian

    npts, m = 3, 5
    pad = 3 * m // 2
    u = R.synthetic_field(npts, 6, m, 0.2, 71)
    w = R.synthetic_field(npts, 6, m, 0.2, 72)
    n_in, n_out = npts * 12 * m, npts * 6 * m
    J = np.zeros((n_out, n_in))
    for i in range(n_in):
        e = np.zeros(n_in)
        e[i] = 1.0
        v = e.reshape((npts, 12, m), order="F")
        col = R.cross_jvp(u, w, np.asfortranarray(v[:, :6]), np.asfortranarray(v[:, 6:]), pad)
        J[:, i] = col.ravel(order="F")
    ref = np.sort(np.linalg.svd(J, compute_uv=False))[::-1][:6]
    op = CrossJacobian(dev(u), dev(w), m_max_pad=pad).as_linear_operator()
    x = np.random.default_rng(3).standard_normal(n_in)
    c = np.random.default_rng(4).standard_normal(n_out)
    assert np.linalg.norm(op.matvec(x) - J @ x) <= 1e-12 * np.linalg.norm(J @ x)
    assert np.linalg.norm(op.rmatvec(c) - J.T @ c) <= 1e-12 * np.linalg.norm(J.T @ c)
    sv = np.sort(svds(op, k=6, tol=1e-12, random_state=0, return_singular_vectors=False))[::-1]
    assert np.allclose(sv, ref, rtol=1e-9, atol=0.0)


@pytest.mark.parametrize("kind,k", [("cross_jvp", 3), ("cross_vjp", 2), ("mhd_jvp", 2), ("mhd_vjp", 1)])
def test_linearised_host_entries(kind, k):
    # the host-array forms of the linearised programs equal the device forms
    import ctypes

    npts, m, pad = 517, 12, 18
    nin, nout = {"cross_jvp": (12, 6), "cross_vjp": (6, 12), "mhd_jvp": (18, 12), "mhd_vjp": (12, 18)}[kind]
    nb = 3 if kind.startswith("mhd") else 2
    base = [R.synthetic_field(npts, 6, m, 0.2, 80 + i) for i in range(nb)]
    x = np.asfortranarray(np.stack([R.synthetic_field(npts, nin, m, 0.2, 90 + t) for t in range(k)], axis=-1))
    out = np.zeros((npts, nout, m, k), order="F")
    P = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    rc = getattr(sf.lib(), f"sfnl_{kind}_host")(*[P(b) for b in base], P(x), P(out), npts, m, pad, k)
    assert rc == 0, sf.last_error()
    ref = host(getattr(sf, kind)(*[dev(b) for b in base], dev(x), m_max_pad=pad))
    assert R.rel_l2(out, ref) <= FP64_TOL


def test_mhd_linearised_k16_m256_against_the_port():
    # the 16-tangent linearised pair (u x w, u x b) at m = 256 (two-kernel large-m form), every tangent
    # against the C restatement (itself pinned to the long-double oracle), and the adjoint identity
    npts, m, k = 96, 256, 16
    pad = 3 * m // 2
    u, w, b = (R.synthetic_field(npts, 6, m, 0.2, 400 + i) for i in range(3))
    tan = np.asfortranarray(np.stack([R.synthetic_field(npts, 18, m, 0.2, 410 + t) for t in range(k)], axis=-1))
    cot = np.asfortranarray(np.stack([R.synthetic_field(npts, 12, m, 0.2, 430 + t) for t in range(k)], axis=-1))
    U, W, B = dev(u), dev(w), dev(b)
    jv = host(sf.mhd_jvp(U, W, B, dev(tan), m_max_pad=pad))
    jt = host(sf.mhd_vjp(U, W, B, dev(cot), m_max_pad=pad))
    c = lambda x, y: R.cpu_product("cross", np.asfortranarray(x), np.asfortranarray(y), pad, n_theta=2 * pad)  # noqa: E731
    for t in range(k):
        du, dw, db = tan[:, 0:6, :, t], tan[:, 6:12, :, t], tan[:, 12:18, :, t]
        ref = np.concatenate([c(du, w) + c(u, dw), c(du, b) + c(u, db)], axis=1)
        assert R.rel_l2(jv[..., t], ref) <= FP64_TOL, t
    lhs, rhs = float(np.sum(jv * cot)), float(np.sum(tan * jt))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_linearised_700k_points_full_size():
    # the linearised cross product at its configuration's size (700k points, m = 32): central differences
    # of the FP64 product at h = 1e-6 and the adjoint identity, both on the device over every point
    import torch

    npts, m, pad, h = 700_000, 32, 48, 1e-6

    def field(nslot, seed):
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        t = torch.randn((m, nslot, npts), generator=g, device="cuda", dtype=torch.float64)
        t *= torch.exp(-0.2 * torch.arange(m, device="cuda", dtype=torch.float64))[:, None, None]
        t[0, 1::2, :] = 0.0
        return t.permute(2, 1, 0)

    u, w, tan, cot = field(6, 1), field(6, 2), field(12, 3), field(6, 4)
    jv = sf.cross_jvp(u, w, tan, m_max_pad=pad)[..., 0]
    jt = sf.cross_vjp(u, w, cot, m_max_pad=pad)[..., 0]

    def fortran(t):
        o = sf.fortran_empty(*t.shape)
        o.copy_(t)
        return o

    du, dw = tan[:, 0:6, :], tan[:, 6:12, :]
    plus = sf.product(sf.OP_CROSS, fortran(u + h * du), fortran(w + h * dw), m_max_pad=pad)
    minus = sf.product(sf.OP_CROSS, fortran(u - h * du), fortran(w - h * dw), m_max_pad=pad)
    fd = (plus - minus) / (2 * h)
    assert float(torch.linalg.vector_norm(fd - jv) / torch.linalg.vector_norm(jv)) <= 1e-8
    lhs, rhs = float(torch.sum(jv * cot)), float(torch.sum(tan * jt))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_mhd_linearised_k16_m256_at_call_size():
    # the 16-tangent linearised pair (u x w, u x b) at m = 256 with the point count of one call of its
    # configuration (350k points in ten calls of 35k; production workspace bounds): central differences of
    # the FP64 cross products at h = 1e-6 for every tangent and the adjoint identity, over every point
    import torch

    npts, m, k, h = 35_000, 256, 16, 1e-6
    pad = 3 * m // 2
    decay = None

    def field(nslot, seed, kk=None):
        nonlocal decay
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        shape = (m, nslot, npts) if kk is None else (kk, m, nslot, npts)
        t = torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
        if decay is None:
            decay = torch.exp(-0.2 * torch.arange(m, device="cuda", dtype=torch.float64))
        t *= decay[:, None, None]
        return t.permute(*reversed(range(t.dim())))

    u, w, b = field(6, 11), field(6, 12), field(6, 13)
    tan, cot = field(18, 14, k), field(12, 15, k)
    jv = sf.mhd_jvp(u, w, b, tan, m_max_pad=pad)
    jt = sf.mhd_vjp(u, w, b, cot, m_max_pad=pad)

    def fortran(t):
        o = sf.fortran_empty(*t.shape)
        o.copy_(t)
        return o

    def cross(x, y):
        return sf.product(sf.OP_CROSS, fortran(x), fortran(y), m_max_pad=pad)

    for t in range(k):
        du, dw, db = tan[:, 0:6, :, t], tan[:, 6:12, :, t], tan[:, 12:18, :, t]
        for c, (base, dbase, out) in enumerate(((w, dw, jv[:, 0:6, :, t]), (b, db, jv[:, 6:12, :, t]))):
            fd = (cross(u + h * du, base + h * dbase) - cross(u - h * du, base - h * dbase)) / (2 * h)
            assert float(torch.linalg.vector_norm(fd - out) / torch.linalg.vector_norm(out)) <= 1e-8, (t, c)
            del fd
    lhs, rhs = float(torch.sum(jv * cot)), float(torch.sum(tan * jt))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    del u, w, b, tan, cot, jv, jt
    torch.cuda.empty_cache()


def test_bundle_full_size_matches_the_elementary_products():
    # the MHD bundle at its configuration's size (1.4 M points, m = 64): the one-launch kernel against the
    # elementary cross and dot products (other kernels, each pinned to the oracle above) over every point
    import torch

    npts, m, pad = 1_400_000, 64, 96

    def field(seed):
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        t = torch.randn((m, 6, npts), generator=g, device="cuda", dtype=torch.float64)
        t *= torch.exp(-0.1 * torch.arange(m, device="cuda", dtype=torch.float64))[:, None, None]
        t[0, 1::2, :] = 0.0
        return t.permute(2, 1, 0)

    u, w, b, j, gt = (field(500 + i) for i in range(5))
    outs = sf.bundle_mhd(u, w, b, j, gt, m_max_pad=pad)
    refs = (sf.product(sf.OP_CROSS, u, w, m_max_pad=pad, algo=sf.ALGO_FAST),
            sf.product(sf.OP_CROSS, u, b, m_max_pad=pad, algo=sf.ALGO_FAST),
            sf.product(sf.OP_CROSS, j, b, m_max_pad=pad, algo=sf.ALGO_FAST),
            sf.product(sf.OP_DOT, u, gt, m_max_pad=pad, algo=sf.ALGO_FAST))
    for o, r in zip(outs, refs):
        assert float(torch.linalg.vector_norm(o - r) / torch.linalg.vector_norm(r)) <= FP64_TOL
