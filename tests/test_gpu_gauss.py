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
