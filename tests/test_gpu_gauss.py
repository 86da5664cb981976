"""GPU parity of the Navier-Stokes caller of the cross product,
smb_cross_prod_gauss_sft_par (SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629):
Gauss-point velocity, curl (and precession rotation) built on the GPU from the
nodal coefficients and the mesh arrays, then (RotV + 2 Om) x W.

Bar: rel-L2 <= 1e-12 per output component against the CPU restatement
(FP64_TOL), on synthetic P2 meshes of the meridian plane.
"""
import numpy as np
import pytest
import torch

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _worst(got, ref):
    return max(R.rel_l2(got[:, 2 * c:2 * c + 2, :], ref[:, 2 * c:2 * c + 2, :]) for c in range(3))


def _dev_mesh(mesh):
    t = lambda a: sf.to_device(a) if a.dtype == np.float64 else torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T  # noqa: E731
    return {k: t(mesh[k]) for k in ("jj", "ww", "dw", "rr")}


@pytest.mark.parametrize("nr,nz,m,modes,prec", [(2, 1, 1, None, False), (6, 4, 8, None, True), (9, 5, 16, "sparse", False),
                                               (5, 3, 64, None, True)])
@pytest.mark.parametrize("own_work", [False, True])
def test_device_entry_matches_oracle(nr, nz, m, modes, prec, own_work):
    mesh = R.synthetic_p2_mesh(nr, nz, 3)
    lm = list(range(m)) if modes is None else [3 * i + (i % 2) for i in range(m)]  # select_mode-like list
    V = R.synthetic_field(mesh["np"], 6, m, 0.2, 11 + m)
    om = R.precession_omega(mesh["np"], lm, 0.3, 0.2) if prec else None
    ref, _, _ = R.c_cross_gauss(V, mesh, lm, om)
    work = torch.empty(12 * 7 * mesh["me"] * m, device="cuda", dtype=torch.float64) if own_work else None
    out = sf.cross_gauss(sf.to_device(V), _dev_mesh(mesh), torch.tensor(lm, dtype=torch.int32, device="cuda"),
                         omega=None if om is None else sf.to_device(om), work=work)
    torch.cuda.synchronize()
    assert _worst(sf.to_host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("prec", [False, True])
def test_reference_signature_on_host_arrays(prec):
    mesh = R.synthetic_p2_mesh(7, 6, 4)
    m = 12
    lm = list(range(m))
    V = R.synthetic_field(mesh["np"], 6, m, 0.3, 5)
    om = R.precession_omega(mesh["np"], lm, 0.7, 0.3) if prec else None
    ref, _, _ = R.c_cross_gauss(V, mesh, lm, om)
    out = sf.smb_cross_prod_gauss_sft_par(None, mesh, lm, V, precession_in=prec, taux_precession=0.7, angle_s_pi=0.3)
    assert _worst(out, ref) <= FP64_TOL


def test_medium_mesh_against_operands_and_library_product():
    # 20k Gauss points, m = 64: operands from the CPU restatement, product by the pocketfft restatement
    mesh = R.synthetic_p2_mesh(40, 36, 5)
    m = 64
    lm = list(range(m))
    V = R.synthetic_field(mesh["np"], 6, m, 0.1, 7)
    _, rot, w = R.c_cross_gauss(V, mesh, lm, product=False)
    ref = R.fft_par("cross", rot, w, 96, workers=8)
    out = sf.smb_cross_prod_gauss_sft_par(None, mesh, lm, V)
    assert _worst(out, ref) <= FP64_TOL


# ---- the Lorentz-force caller: smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883) ----
@pytest.mark.parametrize("nr,nz,m,modes", [(2, 1, 1, None), (6, 4, 8, None), (9, 5, 16, "sparse"), (5, 3, 64, None)])
@pytest.mark.parametrize("own_work", [False, True])
def test_lorentz_device_entry_matches_oracle(nr, nz, m, modes, own_work):
    mesh = R.synthetic_p2_mesh(nr, nz, 8)
    lm = list(range(m)) if modes is None else [3 * i + (i % 2) for i in range(m)]
    H = R.synthetic_field(mesh["np"], 6, m, 0.2, 21 + m)
    B = R.synthetic_field(mesh["np"], 6, m, 0.2, 31 + m)
    ref, _, _ = R.c_curlh_cross_b_gauss(H, B, mesh, lm)
    work = torch.empty(12 * 7 * mesh["me"] * m, device="cuda", dtype=torch.float64) if own_work else None
    out = sf.curlh_cross_b_gauss(sf.to_device(H), sf.to_device(B), _dev_mesh(mesh),
                                 torch.tensor(lm, dtype=torch.int32, device="cuda"), work=work)
    torch.cuda.synchronize()
    assert _worst(sf.to_host(out), ref) <= FP64_TOL


def test_lorentz_reference_signature_on_host_arrays():
    mesh = R.synthetic_p2_mesh(7, 6, 9)
    lm = list(range(12))
    H = R.synthetic_field(mesh["np"], 6, 12, 0.3, 41)
    B = R.synthetic_field(mesh["np"], 6, 12, 0.3, 42)
    ref, _, _ = R.c_curlh_cross_b_gauss(H, B, mesh, lm)
    assert _worst(sf.smb_CurlH_cross_B_gauss_sft_par(None, mesh, lm, H, B), ref) <= FP64_TOL


# ---- the advection callers: smb_ugradc_gauss_fft_par (level set, temperature) and _conc ----
VARIANTS = {"level_set": (False, False), "temperature": (True, True), "concentration": (True, False)}


def _heat(mesh, on):
    return np.linspace(0.5, 2.0, mesh["me"]) if on else None


@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("nr,nz,m,modes", [(2, 1, 1, None), (6, 4, 8, None), (9, 5, 16, "sparse"), (5, 3, 64, None)])
def test_advection_device_entry_matches_oracle(variant, nr, nz, m, modes):
    cons, heat_on = VARIANTS[variant]
    mesh = R.synthetic_p2_mesh(nr, nz, 10)
    lm = list(range(m)) if modes is None else [3 * i + (i % 2) for i in range(m)]
    V = R.synthetic_field(mesh["np"], 6, m, 0.2, 51 + m)
    C = R.synthetic_field(mesh["np"], 2, m, 0.2, 61 + m)
    heat = _heat(mesh, heat_on)
    ref = R.c_ugradc_gauss(V, C, mesh, lm, heat=heat, conservative=cons)[0]
    out = sf.ugradc_gauss(sf.to_device(V), sf.to_device(C), _dev_mesh(mesh),
                          torch.tensor(lm, dtype=torch.int32, device="cuda"),
                          heat=None if heat is None else torch.tensor(heat, device="cuda"), conservative=cons)
    torch.cuda.synchronize()
    assert R.rel_l2(sf.to_host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("modes,own_work", [(None, True), ("sparse", False), ("sparse", True)])
def test_advection_fused_m64(variant, modes, own_work):
    # m = 64 on P2 elements: the operands are built inside the product kernel (node-major copies of the
    # velocity and the scalar in the caller's work buffer or the library's), select_mode-like mode lists
    cons, heat_on = VARIANTS[variant]
    m = 64
    mesh = R.synthetic_p2_mesh(7, 4, 14)
    lm = list(range(m)) if modes is None else [3 * i + (i % 2) for i in range(m)]
    V = R.synthetic_field(mesh["np"], 6, m, 0.1, 151)
    C = R.synthetic_field(mesh["np"], 2, m, 0.1, 152)
    heat = _heat(mesh, heat_on)
    ref = R.c_ugradc_gauss(V, C, mesh, lm, heat=heat, conservative=cons)[0]
    nwork = (16 if cons else 12) * 7 * mesh["me"] * m
    work = torch.full((nwork,), float("nan"), device="cuda", dtype=torch.float64) if own_work else None
    out = sf.ugradc_gauss(sf.to_device(V), sf.to_device(C), _dev_mesh(mesh),
                          torch.tensor(lm, dtype=torch.int32, device="cuda"),
                          heat=None if heat is None else torch.tensor(heat, device="cuda"), conservative=cons,
                          work=work)
    torch.cuda.synchronize()
    assert R.rel_l2(sf.to_host(out), ref) <= FP64_TOL


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_advection_reference_signatures_on_host_arrays(variant):
    cons, heat_on = VARIANTS[variant]
    mesh = R.synthetic_p2_mesh(7, 6, 11)
    lm = list(range(12))
    V = R.synthetic_field(mesh["np"], 6, 12, 0.3, 71)
    C = R.synthetic_field(mesh["np"], 2, 12, 0.3, 72)
    heat = _heat(mesh, heat_on)
    ref = R.c_ugradc_gauss(V, C, mesh, lm, heat=heat, conservative=cons)[0]
    if variant == "level_set":
        out = sf.smb_ugradc_gauss_fft_par(None, mesh, lm, V, C, 1)
    elif variant == "temperature":
        out = sf.smb_ugradc_gauss_fft_par_temperature(None, mesh, lm, heat, V, C)
    else:
        out = sf.smb_ugradc_gauss_fft_par_conc(None, mesh, lm, V, C)
    assert R.rel_l2(out, ref) <= FP64_TOL


def test_medium_mesh_other_callers_against_operands_and_library_products():
    # 20k Gauss points, m = 64: operands from the CPU restatement, products by the pocketfft restatement
    mesh = R.synthetic_p2_mesh(40, 36, 12)
    m = 64
    lm = list(range(m))
    H = R.synthetic_field(mesh["np"], 6, m, 0.1, 81)
    B = R.synthetic_field(mesh["np"], 6, m, 0.1, 82)
    _, rot, w = R.c_curlh_cross_b_gauss(H, B, mesh, lm, product=False)
    assert _worst(sf.smb_CurlH_cross_B_gauss_sft_par(None, mesh, lm, H, B),
                  R.fft_par("cross", rot, w, 96, workers=8)) <= FP64_TOL
    C = R.synthetic_field(mesh["np"], 2, m, 0.1, 83)
    heat = _heat(mesh, True)
    _, g, w, d, cg = R.c_ugradc_gauss(H, C, mesh, lm, heat=heat, conservative=True, product=False)
    ref = R.fft_par("dot", g, w, 96, workers=8) + R.fft_par("prod", d, cg, 96, workers=8)
    assert R.rel_l2(sf.smb_ugradc_gauss_fft_par_temperature(None, mesh, lm, heat, H, C), ref) <= FP64_TOL


@pytest.mark.parametrize("kind,cons", [(sf.GAUSS_NS, False), (sf.GAUSS_LORENTZ, False), (sf.GAUSS_ADVECT, False),
                                       (sf.GAUSS_ADVECT, True)])
def test_operands_alone_match_the_restatement(kind, cons):
    # sfnl_gauss_operands_f64: the operand arrays the callers pass to the products (for callers that run
    # the product themselves, e.g. over a mode-distributed communicator)
    mesh = R.synthetic_p2_mesh(6, 4, 13)
    m = 8
    lm = [2 * i + 1 for i in range(m)]
    V = R.synthetic_field(mesh["np"], 6, m, 0.2, 91)
    V2 = R.synthetic_field(mesh["np"], 6 if kind == sf.GAUSS_LORENTZ else 2, m, 0.2, 92)
    om = R.precession_omega(mesh["np"], lm, 0.4, 0.3) if kind == sf.GAUSS_NS else None
    heat = np.linspace(0.5, 2.0, mesh["me"]) if cons else None
    if kind == sf.GAUSS_NS:
        ref = R.c_cross_gauss(V, mesh, lm, om, product=False)[1:]
    elif kind == sf.GAUSS_LORENTZ:
        ref = R.c_curlh_cross_b_gauss(V, V2, mesh, lm, product=False)[1:]
    else:
        ref = R.c_ugradc_gauss(V, V2, mesh, lm, heat=heat, conservative=cons, product=False)[1:]
        ref = ref if cons else ref[:2]
    got = sf.gauss_operands(kind, sf.to_device(V), _dev_mesh(mesh), torch.tensor(lm, dtype=torch.int32, device="cuda"),
                            v2=None if kind == sf.GAUSS_NS else sf.to_device(V2),
                            omega=None if om is None else sf.to_device(om),
                            heat=None if heat is None else torch.tensor(heat, device="cuda"), conservative=cons)
    torch.cuda.synchronize()
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert R.rel_l2(sf.to_host(g), r) <= 1e-13


def _p1_mesh(nr, nz, seed):
    # the vertices of a P2 mesh as a P1 mesh (3 nodes per element, linear basis at the same 7 points)
    m2 = R.synthetic_p2_mesh(nr, nz, seed)
    L = np.array([[1 / 3, 2 / 3, 1 / 6, 1 / 6, 0.1, 0.45, 0.45], [1 / 3, 1 / 6, 2 / 3, 1 / 6, 0.45, 0.1, 0.45],
                  [1 / 3, 1 / 6, 1 / 6, 2 / 3, 0.45, 0.45, 0.1]])
    jj = np.asfortranarray(m2["jj"][:3])
    me = jj.shape[1]
    dw = np.zeros((2, 3, 7, me), order="F")
    for e in range(me):
        P = m2["rr"][:, jj[:, e] - 1].T  # (3 vertices, (r, z))
        T = np.array([[P[0, 0] - P[2, 0], P[1, 0] - P[2, 0]], [P[0, 1] - P[2, 1], P[1, 1] - P[2, 1]]])
        G = np.linalg.inv(T)
        dlam = np.array([G[0], G[1], -G[0] - G[1]])  # (3 lambdas, 2 coords)
        dw[:, :, :, e] = dlam.T[:, :, None]
    return {"jj": jj, "rr": m2["rr"], "ww": np.asfortranarray(L), "dw": dw, "np": m2["np"], "me": me, "n_w": 3,
            "l_G": 7}


@pytest.mark.parametrize("m", [12, 64, 96])
def test_fused_general_kernel_p1_elements(m):
    # the general fused kernel (any element type; at m = 64 it serves the elements the third-fold kernels
    # do not): P1 elements, every caller, against the restatements
    mesh = _p1_mesh(5, 4, 21)
    lm = list(range(m))
    dm, lmd = _dev_mesh(mesh), torch.tensor(lm, dtype=torch.int32, device="cuda")
    V = R.synthetic_field(mesh["np"], 6, m, 0.2, 161)
    W2 = R.synthetic_field(mesh["np"], 6, m, 0.2, 162)
    C = R.synthetic_field(mesh["np"], 2, m, 0.2, 163)
    om = R.precession_omega(mesh["np"], lm, 0.3, 0.2)
    heat = _heat(mesh, True)
    ref = R.c_cross_gauss(V, mesh, lm, om)[0]
    out = sf.cross_gauss(sf.to_device(V), dm, lmd, omega=sf.to_device(om))
    assert _worst(sf.to_host(out), ref) <= FP64_TOL
    ref = R.c_curlh_cross_b_gauss(V, W2, mesh, lm)[0]
    out = sf.curlh_cross_b_gauss(sf.to_device(V), sf.to_device(W2), dm, lmd)
    assert _worst(sf.to_host(out), ref) <= FP64_TOL
    for cons, ht in ((False, None), (True, heat)):
        ref = R.c_ugradc_gauss(V, C, mesh, lm, heat=ht, conservative=cons)[0]
        out = sf.ugradc_gauss(sf.to_device(V), sf.to_device(C), dm, lmd,
                              heat=None if ht is None else torch.tensor(ht, device="cuda"), conservative=cons)
        torch.cuda.synchronize()
        assert R.rel_l2(sf.to_host(out), ref) <= FP64_TOL
