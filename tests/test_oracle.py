"""The CPU oracle, pinned before it is trusted.

The reference ships no array-level golden vectors for FFT_PAR_*_DCL; its
only known answers that isolate the product arithmetic are the manufactured
nonlinear sources of the regression tests (REGRESSION_SUITE/TEST1/
LOCAL_SOURCES/condlim.F90:140-210: mode-1 fields whose product lands on
modes 0 and 2 by the rule (a cos + b sin)(c cos + d sin) = (ac+bd)/2 +
(ac-bd)/2 cos 2t + (ad+bc)/2 sin 2t).  The oracle is pinned by that
identity, by two independent formulations (pocketfft and an exact spectral
convolution with no grid), and by the committed fixtures.
"""
import glob
import os

import numpy as np
import pytest

from oracle import ref_fft as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _mode1_fields(npts, m, seed):
    rng = np.random.default_rng(seed)
    V = np.zeros((npts, 6, m), order="F")
    V[:, :, 1] = rng.standard_normal((npts, 6))
    return V


@pytest.mark.parametrize("nb_procs", [1, 3])
def test_mode1_product_identity(nb_procs):
    # TEST1 runs m_max = 3 on 3 Fourier ranks (REGRESSION_TESTS/data); u and
    # curl u are pure mode-1 fields.
    m = 3
    U = _mode1_fields(17, m, 1)
    W = _mode1_fields(17, m, 2)
    out = R.c_oracle("cross", U, W, 3 * m // 2, nb_procs=nb_procs)
    c = lambda V, k: V[:, 2 * k, 1]  # noqa: E731
    s = lambda V, k: V[:, 2 * k + 1, 1]  # noqa: E731

    def prod_rule(f, k1, g, k2):
        a, b, cc, d = c(f, k1), s(f, k1), c(g, k2), s(g, k2)
        return (a * cc + b * d) / 2, (a * cc - b * d) / 2, (a * d + b * cc) / 2

    for comp, (i, j) in enumerate(((1, 2), (2, 0), (0, 1))):
        p = prod_rule(U, i, W, j)
        q = prod_rule(W, i, U, j)  # the second term of the cross product, u_j w_i
        mean, c2, s2 = (p[t] - q[t] for t in range(3))
        np.testing.assert_allclose(out[:, 2 * comp, 0], mean, rtol=0, atol=1e-14)
        np.testing.assert_allclose(out[:, 2 * comp, 2], c2, rtol=0, atol=1e-14)
        np.testing.assert_allclose(out[:, 2 * comp + 1, 2], s2, rtol=0, atol=1e-14)
        np.testing.assert_allclose(out[:, 2 * comp + 1, 0], 0.0, atol=0)
        np.testing.assert_allclose(out[:, 2 * comp:2 * comp + 2, 1], 0.0, atol=1e-14)


@pytest.mark.parametrize("op", ["cross", "dot", "prod"])
@pytest.mark.parametrize("npts,m,pad", [(23, 4, 6), (9, 9, 13), (31, 16, 24)])
def test_three_formulations_agree(op, npts, m, pad):
    nsl = 2 if op == "prod" else 6
    V1 = R.synthetic_field(npts, nsl, m, 0.2, 5)
    V2 = R.synthetic_field(npts, nsl, m, 0.2, 6)
    ref = R.c_oracle(op, V1, V2, pad)
    assert R.rel_l2(R.spectral_product(op, V1, V2), ref) < 1e-15
    assert R.rel_l2(R.fft_par(op, V1, V2, pad), ref) < 1e-14
    # The even grid N = 2*m_max_pad also dealiases: same truncated product.
    assert R.rel_l2(R.c_oracle(op, V1, V2, pad, n_theta=2 * pad), ref) < 1e-15


def test_nb_procs_emulation_is_layout_only():
    V1 = R.synthetic_field(29, 6, 6, 0.3, 7)
    V2 = R.synthetic_field(29, 6, 6, 0.3, 8)
    ref = R.c_oracle("cross", V1, V2, 9)
    for P in (2, 3, 6):
        np.testing.assert_array_equal(R.c_oracle("cross", V1, V2, 9, nb_procs=P), ref)
    # bloc_size larger than needed only adds dummy points
    np.testing.assert_array_equal(R.c_oracle("cross", V1, V2, 9, nb_procs=3, bloc_size=15), ref)


def test_short_pad_aliases():
    # m_max_pad = m_max: the grid is too short and the reference's result is aliased.
    V1 = R.synthetic_field(13, 6, 8, 0.0, 9)
    V2 = R.synthetic_field(13, 6, 8, 0.0, 10)
    ali = R.c_oracle("cross", V1, V2, 8)
    exact = R.spectral_product("cross", V1, V2)
    assert R.rel_l2(ali, exact) > 1e-3
    assert R.rel_l2(R.fft_par("cross", V1, V2, 8), ali) < 1e-14


def test_oracle_rejects_what_the_reference_cannot_do():
    V = R.synthetic_field(10, 6, 4, 0.1, 1)
    with pytest.raises(ValueError):
        R.c_oracle("cross", V, V, 3)                   # m_max_pad < m_max
    with pytest.raises(ValueError):
        R.c_oracle("cross", V, V, 6, nb_procs=2, bloc_size=4)  # np > nb_procs*bloc_size
    W = R.synthetic_field(10, 4, 4, 0.1, 1)
    with pytest.raises(ValueError):
        R.c_oracle("cross", W, W, 6)                   # nb_field != 6


def test_sine_of_mode_zero_is_ignored():
    V1 = R.synthetic_field(11, 6, 5, 0.2, 3)
    V2 = R.synthetic_field(11, 6, 5, 0.2, 4)
    ref = R.c_oracle("cross", V1, V2, 7)
    V1b = V1.copy(order="F")
    V1b[:, 1::2, 0] = 123.0
    np.testing.assert_array_equal(R.c_oracle("cross", V1b, V2, 7), ref)
    assert np.all(ref[:, 1::2, 0] == 0.0) or np.abs(ref[:, 1::2, 0]).max() < 1e-15


PRODUCT_FIXTURES = sorted(p for p in glob.glob(os.path.join(GOLD, "*.npz"))
                          if not os.path.basename(p).startswith(("real_", "maxvel_")))
SYNTH_FIXTURES = sorted(p for p in glob.glob(os.path.join(GOLD, "*.npz"))
                        if os.path.basename(p).startswith(("real_", "maxvel_")))


@pytest.mark.parametrize("path", PRODUCT_FIXTURES)
def test_golden_fixtures_reproduce(path):
    z = np.load(path)
    npts, m, pad, procs = (int(v) for v in z["meta"])
    op = str(z["op"])
    out = R.c_oracle(op, z["V1"], z["V2"], pad, nb_procs=procs)
    np.testing.assert_array_equal(out, z["out"])
    if op in ("div", "svdiv", "tension"):  # grid-dependent: same grid, library FFT
        assert R.rel_l2(R.fft_par(op, z["V1"], z["V2"], pad), z["out"]) < 1e-13
    else:
        assert R.rel_l2(R.spectral_product(op, z["V1"], z["V2"]), z["out"]) < 1e-15


def _mode0_scalar(npts, m, value):
    S = np.zeros((npts, 2, m), order="F")
    S[:, 0, 0] = value
    return S


def test_scalar_vect_known_answers():
    # FFT_SCALAR_VECT_DCL (fft_parallel.F90:1150-1157) with a constant scalar:
    # pb = 1 scales the vector, pb = 2 divides it, on every mode.
    V = R.synthetic_field(19, 6, 6, 0.3, 31)
    S = _mode0_scalar(19, 6, 2.5)
    np.testing.assert_allclose(R.c_oracle("svect", V, S, 9), 2.5 * V, rtol=0, atol=1e-14)
    np.testing.assert_allclose(R.c_oracle("svdiv", V, S, 9), V / 2.5, rtol=0, atol=1e-15)
    # mode-1 scalar times mode-1 vector: the product rule lands on modes 0 and 2
    U = _mode1_fields(13, 3, 3)
    S1 = np.zeros((13, 2, 3), order="F")
    S1[:, :, 1] = np.random.default_rng(4).standard_normal((13, 2))
    out = R.c_oracle("svect", U, S1, 4)
    for k in range(3):
        a, b, c, d = U[:, 2 * k, 1], U[:, 2 * k + 1, 1], S1[:, 0, 1], S1[:, 1, 1]
        np.testing.assert_allclose(out[:, 2 * k, 0], (a * c + b * d) / 2, atol=1e-14)
        np.testing.assert_allclose(out[:, 2 * k, 2], (a * c - b * d) / 2, atol=1e-14)
        np.testing.assert_allclose(out[:, 2 * k + 1, 2], (a * d + b * c) / 2, atol=1e-14)


def test_tensor_known_answers():
    # FFT_TENSOR_DCL (fft_parallel.F90:1676-1706, output layout :1786-1787):
    # V_out(k, :, 2l-1:2l, :) holds the coefficients of u_k v_l.
    U = _mode1_fields(11, 3, 5)
    W = _mode1_fields(11, 3, 6)
    out = R.c_oracle("tensor", U, W, 4)
    assert out.shape == (3, 11, 6, 3)
    for k in range(3):
        for l in range(3):
            a, b, c, d = U[:, 2 * k, 1], U[:, 2 * k + 1, 1], W[:, 2 * l, 1], W[:, 2 * l + 1, 1]
            np.testing.assert_allclose(out[k, :, 2 * l, 0], (a * c + b * d) / 2, atol=1e-14)
            np.testing.assert_allclose(out[k, :, 2 * l, 2], (a * c - b * d) / 2, atol=1e-14)
            np.testing.assert_allclose(out[k, :, 2 * l + 1, 2], (a * d + b * c) / 2, atol=1e-14)
    # opt_tension with a constant gradient (3, 4, 0): |g| = 5, out = u_k g_l / (5 + 1e-14) - 5 delta_kl
    G = np.zeros((11, 6, 3), order="F")
    G[:, 0, 0], G[:, 2, 0] = 3.0, 4.0
    V = R.synthetic_field(11, 6, 3, 0.3, 7)
    t = R.c_oracle("tension", V, G, 4)
    g = (3.0, 4.0, 0.0)
    for k in range(3):
        for l in range(3):
            want = V[:, 2 * k:2 * k + 2, :] * g[l] / (5.0 + 1e-14)
            want = want.copy()
            if k == l:
                want[:, 0, 0] -= 5.0
            np.testing.assert_allclose(t[k, :, 2 * l:2 * l + 2, :], want, rtol=0, atol=1e-14)


def test_div_known_answer():
    # FFT_PAR_DIV_DCL (fft_parallel.F90:786): a constant divisor divides every mode.
    C = R.synthetic_field(17, 2, 5, 0.3, 8)
    np.testing.assert_allclose(R.c_oracle("div", C, _mode0_scalar(17, 5, -4.0), 7), C / -4.0, rtol=0, atol=1e-15)


def test_sibling_routines_reject_wrong_shapes():
    V = R.synthetic_field(10, 6, 4, 0.1, 1)
    S = R.synthetic_field(10, 2, 4, 0.1, 2)
    with pytest.raises(ValueError):
        R.c_oracle("svect", V, V, 6)   # scalar must have 2 slots (:1158-1160)
    with pytest.raises(ValueError):
        R.c_oracle("svect", S, S, 6)
    with pytest.raises(ValueError):
        R.c_oracle("tensor", V, S, 6)
    with pytest.raises(ValueError):
        R.c_oracle("div", V, V, 6)


def test_synthetic_generator_shape_and_decay():
    x = R.synthetic_field(1000, 6, 8, 0.3, 42)
    assert x.flags.f_contiguous and x.shape == (1000, 6, 8)
    assert np.all(x[:, 1::2, 0] == 0.0)
    s = np.sqrt((x[:, 0::2, :] ** 2).mean(axis=(0, 1)))
    np.testing.assert_allclose(s / s[0], np.exp(-0.3 * np.arange(8)), rtol=0.1)
    np.testing.assert_array_equal(x, R.synthetic_field(1000, 6, 8, 0.3, 42))


def test_vjp_restatement_is_the_transpose():
    # Build J explicitly on a tiny case and compare J^T c with cross_vjp.
    npts, m = 2, 3
    u = R.synthetic_field(npts, 6, m, 0.0, 1)
    w = R.synthetic_field(npts, 6, m, 0.0, 2)
    cot = R.synthetic_field(npts, 6, m, 0.0, 3)
    pad = 3 * m // 2
    nin = npts * 12 * m
    J = np.zeros((npts * 6 * m, nin))
    for i in range(nin):
        e = np.zeros(nin)
        e[i] = 1.0
        v = e.reshape((npts, 12, m), order="F")
        J[:, i] = R.cross_jvp(u, w, np.asfortranarray(v[:, :6]), np.asfortranarray(v[:, 6:]), pad).reshape(-1, order="F")
    jt = (J.T @ cot.reshape(-1, order="F")).reshape((npts, 12, m), order="F")
    np.testing.assert_allclose(R.cross_vjp(u, w, cot), jt, rtol=0, atol=1e-13)


@pytest.mark.parametrize("path", SYNTH_FIXTURES)
def test_synthesis_fixtures_reproduce(path):
    z = np.load(path)
    npts, m, extra, procs = (int(v) for v in z["meta"])
    if str(z["kind"]) == "real":
        np.testing.assert_array_equal(R.c_real(z["V1"], nb_procs=procs, opt_nb_plane=extra or None), z["out"])
    else:
        assert R.c_max_vel(z["V1"], extra, nb_procs=procs) == z["out"][0]


def test_fft_par_real_known_answers():
    # FFT_PAR_REAL (fft_parallel.F90:28-145): a mode-1 field a cos t + b sin t at t_j = 2 pi j / N,
    # N = 2 m_max - 1, or 2 m_max_pad - 1 with m_max_pad = (opt_nb_plane + 1) / 2 when that is larger.
    m, npts = 4, 6
    V = np.zeros((npts, 4, m), order="F")
    rng = np.random.default_rng(9)
    V[:, 0, 0] = rng.standard_normal(npts)          # mean of field 1
    V[:, 0:2, 1] = rng.standard_normal((npts, 2))   # a, b of field 1
    V[:, 3, 3] = rng.standard_normal(npts)          # sin 3t of field 2
    for opt, N in ((None, 7), (5, 7), (12, 11), (13, 13)):
        out = R.c_real(V, nb_procs=2, opt_nb_plane=opt)
        assert out.shape == (N, 2, npts)
        t = 2 * np.pi * np.arange(N) / N
        want1 = V[None, :, 0, 0] + V[None, :, 0, 1] * np.cos(t)[:, None] + V[None, :, 1, 1] * np.sin(t)[:, None]
        np.testing.assert_allclose(out[:, 0, :], want1, atol=1e-14)
        np.testing.assert_allclose(out[:, 1, :], V[None, :, 3, 3] * np.sin(3 * t)[:, None], atol=1e-14)
    with pytest.raises(ValueError):
        R.c_real(np.zeros((5, 3, 4), order="F"))            # odd nb_field (:59)
    with pytest.raises(ValueError):
        R.c_real(np.zeros((5, 2, 4), order="F"), nb_procs=2)  # np not a multiple of nb_procs (:66-70)


def test_fft_max_vel_known_answers():
    # FFT_MAX_VEL_DCL (fft_parallel.F90:1426-1541): u = (cos t, sin t, 0) has |u| = 1 everywhere; a
    # scalar a0 + a1 cos t peaks at t = 0, which is on every grid.
    npts, m = 7, 3
    U = np.zeros((npts, 6, m), order="F")
    U[:, 0, 1] = 1.0   # u_r = cos t
    U[:, 3, 1] = 1.0   # u_theta = sin t
    assert abs(R.c_max_vel(U, 3) - 1.0) < 1e-15
    assert abs(R.c_max_vel(U, 3, nb_procs=3, bloc_size=3) - 1.0) < 1e-15
    S = np.zeros((npts, 2, m), order="F")
    S[:, 0, 0] = np.arange(npts)
    S[:, 0, 2] = 0.5
    assert abs(R.c_max_vel(S, 4) - (npts - 1 + 0.5)) < 1e-13


def test_gauss_point_curl_known_answer():
    # smb_cross_prod_gauss_sft_par (subroutine_ns_with_velocity.F90:512-629) on solid-body rotation
    # u = (0, r, 0), mode 0: curl u = (0, 0, 2) (u_theta/r + d u_theta/dr), which P2 elements reproduce
    # exactly, and (curl u) x u = (-2 r, 0, 0).
    mesh = R.synthetic_p2_mesh(4, 3, 2)
    V = np.zeros((mesh["np"], 6, 1), order="F")
    V[:, 2, 0] = mesh["rr"][0]
    out, rot, w = R.c_cross_gauss(V, mesh, [0])
    ray = np.einsum("nl,nm->lm", mesh["ww"], mesh["rr"][0][mesh["jj"] - 1]).T.ravel()  # Gauss radii
    np.testing.assert_allclose(rot[:, 4, 0], 2.0, atol=1e-12)
    np.testing.assert_allclose(np.delete(rot[:, :, 0], 4, axis=1), 0.0, atol=1e-12)
    np.testing.assert_allclose(w[:, 2, 0], ray, atol=1e-14)
    np.testing.assert_allclose(out[:, 0, 0], -2.0 * ray, atol=1e-12)
    # precession adds 2 Om to the curl: mode 0 carries Om_z = taux cos(angle pi)
    om = R.precession_omega(mesh["np"], [0], 0.5, 0.25)
    _, rot2, _ = R.c_cross_gauss(V, mesh, [0], om)
    np.testing.assert_allclose(rot2[:, 4, 0], 2.0 + 2 * 0.5 * np.cos(0.25 * np.pi), atol=1e-12)


def test_lorentz_caller_on_equal_fields_is_the_navier_stokes_caller():
    # smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883) with H = B builds the same
    # curl and values as smb_cross_prod_gauss_sft_par without precession: (curl u) x u
    mesh = R.synthetic_p2_mesh(4, 3, 6)
    lm = [0, 1, 2, 3]
    V = R.synthetic_field(mesh["np"], 6, 4, 0.3, 61)
    out_l, rot_l, w_l = R.c_curlh_cross_b_gauss(V, V, mesh, lm)
    out_n, rot_n, w_n = R.c_cross_gauss(V, mesh, lm)
    np.testing.assert_array_equal(rot_l, rot_n)
    np.testing.assert_array_equal(w_l, w_n)
    np.testing.assert_array_equal(out_l, out_n)
    # and W comes from the second field
    B = R.synthetic_field(mesh["np"], 6, 4, 0.3, 62)
    _, rot_b, w_b = R.c_curlh_cross_b_gauss(V, B, mesh, lm, product=False)
    np.testing.assert_array_equal(rot_b, rot_n)
    _, _, w_ref = R.c_cross_gauss(B, mesh, lm, product=False)
    np.testing.assert_array_equal(w_b, w_ref)


def test_advection_caller_known_answers():
    # smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534 and the temperature / concentration
    # versions): P2 elements reproduce linear fields exactly.
    mesh = R.synthetic_p2_mesh(4, 3, 7)
    npn, ng = mesh["np"], mesh["l_G"] * mesh["me"]
    r, z = mesh["rr"]
    # u = (0, 0, 1), c = z: grad c . u = 1; div u = 0
    V = np.zeros((npn, 6, 1), order="F")
    V[:, 4, 0] = 1.0
    C = np.zeros((npn, 2, 1), order="F")
    C[:, 0, 0] = z
    for cons in (False, True):
        out = R.c_ugradc_gauss(V, C, mesh, [0], conservative=cons)[0]
        np.testing.assert_allclose(out[:, 0, 0], 1.0, atol=1e-12)
        np.testing.assert_allclose(out[:, 1, 0], 0.0, atol=1e-15)
    # u = (r, 0, 0), c = 1: grad c = 0, div u = (1/r) d(r u_r)/dr = 2; the conservative form gives 2 c,
    # times the element's heat capacity in the temperature version
    V = np.zeros((npn, 6, 1), order="F")
    V[:, 0, 0] = r
    C = np.zeros((npn, 2, 1), order="F")
    C[:, 0, 0] = 1.0
    heat = np.linspace(1.0, 3.0, mesh["me"])
    out, gradc, w, div, cg = R.c_ugradc_gauss(V, C, mesh, [0], heat=heat, conservative=True)
    np.testing.assert_allclose(div[:, 0, 0], 2.0, atol=1e-12)
    np.testing.assert_allclose(cg[:, 0, 0], np.repeat(heat, mesh["l_G"]), atol=1e-14)
    np.testing.assert_allclose(out[:, 0, 0], 2.0 * np.repeat(heat, mesh["l_G"]), atol=1e-12)
    assert np.abs(R.c_ugradc_gauss(V, C, mesh, [0], conservative=False)[0]).max() < 1e-14
    # c = r cos(theta) (mode 1), u_theta = sin(theta): the theta gradient -sin(theta) gives
    # u . grad c = -sin^2 = -1/2 + cos(2 theta)/2
    V = np.zeros((npn, 6, 3), order="F")
    V[:, 3, 1] = 1.0
    C = np.zeros((npn, 2, 3), order="F")
    C[:, 0, 1] = r
    out, gradc, _, _, _ = R.c_ugradc_gauss(V, C, mesh, [0, 1, 2])
    np.testing.assert_allclose(gradc[:, 3, 1], -1.0, atol=1e-12)
    np.testing.assert_allclose(out[:, 0, 0], -0.5, atol=1e-12)
    np.testing.assert_allclose(out[:, 0, 2], 0.5, atol=1e-12)
    np.testing.assert_allclose(out[:, 0, 1], 0.0, atol=1e-12)
    assert out.shape == (ng, 2, 3)


@pytest.mark.parametrize("npts,m,pad,n_theta", [(37, 16, 24, None), (37, 16, 24, 48), (50, 64, 96, 192),
                                                  (21, 5, 7, None), (9, 1, 1, None), (17, 40, 60, 130)])
def test_cpu_baseline_port_matches_the_oracle(npts, m, pad, n_theta):
    # the O(N log N) C restatement timed as the CPU baseline: odd (reference) and even grids, partial
    # point blocks, every product and the bundle
    V1 = R.synthetic_field(npts, 6, m, 0.2, 11)
    V2 = R.synthetic_field(npts, 6, m, 0.2, 12)
    for op in ("cross", "dot"):
        ref = R.c_oracle(op, V1, V2, pad, n_theta=n_theta)
        assert R.rel_l2(R.cpu_product(op, V1, V2, pad, n_theta=n_theta, threads=3), ref) <= 1e-14
    S1, S2 = V1[:, :2].copy(order="F"), V2[:, :2].copy(order="F")
    ref = R.c_oracle("prod", S1, S2, pad, n_theta=n_theta)
    assert R.rel_l2(R.cpu_product("prod", S1, S2, pad, n_theta=n_theta), ref) <= 1e-14
    f = [R.synthetic_field(npts, 6, m, 0.1, 20 + i) for i in range(5)]
    for o, r in zip(R.cpu_mhd_bundle(*f, pad, n_theta=n_theta, threads=2), R.mhd_bundle(*f, pad)):
        assert R.rel_l2(o, r) <= 1e-14
