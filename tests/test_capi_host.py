"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and rejects bad arguments on the host (before any CUDA call) with
the codes include/sfemans_nl.h documents."""
import ctypes
import os
import re

import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sfnl_\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = sf.lib()
    declared = _declared()
    assert len(declared) >= 23
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert L.sfnl_version().startswith(b"sfemans_nl")


def test_bindings_cover_the_header():
    # every declared entry point has a ctypes signature in the Python layer
    declared = _declared() - {"sfnl_last_error", "sfnl_version"}
    assert declared <= set(sf._SIGS), declared - set(sf._SIGS)


NULL = ctypes.c_void_p(0)


@pytest.mark.parametrize("args,code", [
    ((0, NULL, NULL, NULL, 10, 0, 6, 0, 0, NULL), -1),        # m_max = 0 (m_max_c==0 in the reference)
    ((0, NULL, NULL, NULL, -1, 4, 6, 0, 0, NULL), -1),        # np < 0
    ((0, NULL, NULL, NULL, 10, 4, 3, 0, 0, NULL), -3),        # m_max_pad < m_max
    ((0, NULL, NULL, NULL, 10, 4, 6, 5, 0, NULL), -3),        # explicit grid shorter than 2m-1
    ((8, NULL, NULL, NULL, 10, 4, 6, 0, 0, NULL), -1),        # unknown op
    ((0, NULL, NULL, NULL, 10, 4, 6, 0, 0, NULL), -1),        # null arrays with np > 0
])
def test_product_argument_errors(args, code):
    assert sf.lib().sfnl_product_f64(*args) == code
    assert sf.last_error()


def test_bundle_kernel_switch():
    prev = sf.set_bundle_kernel(sf.BUNDLE_THIRD_FOLD)
    try:
        assert prev in (sf.BUNDLE_RESIDUE, sf.BUNDLE_THIRD_FOLD)
        assert sf.set_bundle_kernel(sf.BUNDLE_RESIDUE) == sf.BUNDLE_THIRD_FOLD
        assert sf.lib().sfnl_set_bundle_kernel(2) == -1 and sf.last_error()
        assert sf.set_bundle_kernel(sf.BUNDLE_RESIDUE) == sf.BUNDLE_RESIDUE  # unchanged by the refusal
    finally:
        sf.set_bundle_kernel(prev)


def test_large_m_test_hooks_check_their_arguments():
    assert sf.lib().sfnl_test_large_workspace_cap(-1) == -1 and sf.last_error()
    assert sf.lib().sfnl_test_large_workspace_cap(0) == 0
    for bad in (-1, 1, 4, 24):
        assert sf.lib().sfnl_test_large_residues(bad) == -1 and sf.last_error()
    assert sf.lib().sfnl_test_large_residues(6) == 0 and sf.lib().sfnl_test_large_residues(0) == 0


def test_zero_points_is_a_no_op():
    assert sf.lib().sfnl_product_f64(0, NULL, NULL, NULL, 0, 4, 6, 0, 0, NULL) == 0


def test_fortran_signature_checks():
    L = sf.lib()
    a = np.zeros((4, 6, 2), order="F")
    p = ctypes.c_void_p(a.ctypes.data)
    # odd nb_field (fft_parallel.F90:188)
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 5, 2, 1, 5, 3, NULL) == -1
    # m_max_c == 0
    assert L.sfnl_fft_par_dot_prod_dcl(p, p, p, 4, 6, 0, 1, 5, 3, NULL) == -1
    # nb_field 4 cannot form a cross product
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 4, 2, 1, 5, 3, NULL) == -2
    # more than one Fourier rank on one GPU
    assert L.sfnl_fft_par_cross_prod_dcl(p, p, p, 4, 6, 2, 2, 5, 3, NULL) == -4
    # np > nb_procs*bloc_size (the reference's buffer bound)
    assert L.sfnl_fft_par_prod_dcl(p, p, p, 4, 2, 1, 3, 3, NULL) == -2


def test_split_argument_errors():
    L = sf.lib()
    assert L.sfnl_product_split(0, NULL, NULL, NULL, 10, 4, 6, 5, NULL) == -1     # split not 2/3
    assert L.sfnl_product_split(0, NULL, NULL, NULL, 10, 4, 4, 3, NULL) == -1     # null arrays first
    a = ctypes.c_void_p(16)
    assert L.sfnl_product_split(0, a, a, a, 10, 8, 8, 3, NULL) == -3             # aliasing pad


def test_batch_argument_errors():
    L = sf.lib()
    a = ctypes.c_void_p(16)
    assert L.sfnl_cross_jvp_f64(a, a, a, a, 10, 4, 6, 0, NULL) == -1
    assert L.sfnl_mhd_vjp_f64(a, a, a, a, a, 10, 4, 6, 70000, NULL) == -1
    assert L.sfnl_mhd_jvp_f64(a, a, NULL, a, a, 10, 4, 6, 2, NULL) == -1


def test_sibling_fortran_signature_checks():
    L = sf.lib()
    a = np.zeros((4, 6, 2), order="F")
    p = ctypes.c_void_p(a.ctypes.data)
    # FFT_SCALAR_VECT_DCL: odd slot count (fft_parallel.F90:1068), scalar with 6 slots (:1163), bad pb (:1160)
    assert L.sfnl_fft_scalar_vect_dcl(p, p, p, 1, 4, 6, 3, 2, 1, 5, 3, NULL) == -1
    assert L.sfnl_fft_scalar_vect_dcl(p, p, p, 1, 4, 6, 6, 2, 1, 5, 3, NULL) == -2
    assert L.sfnl_fft_scalar_vect_dcl(p, p, p, 3, 4, 6, 2, 2, 1, 5, 3, NULL) == -1
    assert "problem type" in sf.last_error()
    # FFT_TENSOR_DCL: opt_tension present and .FALSE. (:1705), nb_field != 6, m_max_c == 0
    assert L.sfnl_fft_tensor_dcl(p, p, p, 4, 6, 2, 1, 5, 3, 0, NULL) == -1
    assert "opt_tension" in sf.last_error()
    assert L.sfnl_fft_tensor_dcl(p, p, p, 4, 4, 2, 1, 5, 3, -1, NULL) == -2
    assert L.sfnl_fft_tensor_dcl(p, p, p, 4, 6, 0, 1, 5, 3, 1, NULL) == -1
    # FFT_PAR_DIV_DCL: m_max_c == 0 (:710), np > nb_procs*bloc_size
    assert L.sfnl_fft_par_div_dcl(p, p, p, 4, 0, 1, 5, 3, NULL) == -1
    assert L.sfnl_fft_par_div_dcl(p, p, p, 4, 2, 1, 3, 3, NULL) == -2


def test_grid_dependent_products_refuse_the_fast_and_split_forms():
    L = sf.lib()
    a = ctypes.c_void_p(16)
    for op in (sf.OP_DIV, sf.OP_VECT_SCALAR, sf.OP_TENSION):
        assert L.sfnl_product_f64(op, a, a, a, 10, 4, 6, 0, sf.ALGO_FAST, NULL) == -4
        assert L.sfnl_product_split(op, a, a, a, 10, 4, 6, 3, NULL) == -4
    assert L.sfnl_scalar_vect_f64(a, a, a, 10, 4, 6, 0, NULL) == -1


def test_python_mirror_rejects_what_the_reference_rejects():
    V = np.zeros((4, 6, 2), order="F")
    S = np.zeros((4, 2, 2), order="F")
    with pytest.raises(sf.SfnlError) as e:
        sf.FFT_SCALAR_VECT_DCL(None, V, V, V, 1, 1, 5, 3)
    assert e.value.code == -2
    with pytest.raises(sf.SfnlError) as e:
        sf.FFT_SCALAR_VECT_DCL(None, V, S, V, 0, 1, 5, 3)
    assert e.value.code == -1
    with pytest.raises(sf.SfnlError) as e:
        sf.FFT_TENSOR_DCL(None, V, V, np.zeros((3, 4, 6, 2), order="F"), 1, 5, 3, opt_tension=False)
    assert e.value.code == -1
    with pytest.raises(sf.SfnlError) as e:  # V_out of the wrong shape
        sf.FFT_TENSOR_DCL(None, V, V, V, 1, 5, 3)
    assert e.value.code == -2


def test_synthesis_argument_checks():
    L = sf.lib()
    a = np.zeros((4, 6, 2), order="F")
    p = ctypes.c_void_p(a.ctypes.data)
    # FFT_PAR_REAL: grid length (fft_parallel.F90:71-80), odd nb_field, more than one Fourier rank
    assert L.sfnl_fft_par_real_planes(4, 0) == 7 and L.sfnl_fft_par_real_planes(4, 12) == 11
    assert L.sfnl_fft_par_real(p, p, 4, 5, 2, 1, 0) == -1
    assert L.sfnl_fft_par_real(p, p, 4, 6, 0, 1, 0) == -1
    assert L.sfnl_fft_par_real(p, p, 4, 6, 2, 2, 0) == -4
    # device entry: a grid shorter than 2m-1 cannot hold the modes
    d = ctypes.c_void_p(16)
    assert L.sfnl_real_f64(d, d, 10, 6, 8, 14, NULL) == -3
    # FFT_MAX_VEL_DCL: odd nb_field, np > nb_procs*bloc_size, short pad, null result
    assert L.sfnl_fft_max_vel_dcl(p, p, 4, 3, 2, 1, 5, 3) == -1
    assert L.sfnl_fft_max_vel_dcl(p, p, 4, 6, 2, 1, 3, 3) == -2
    assert L.sfnl_fft_max_vel_dcl(p, p, 4, 6, 2, 1, 5, 1) == -3
    assert L.sfnl_max_vel_f64(d, NULL, 10, 6, 4, 6, NULL) == -1


def test_gauss_point_entry_checks():
    L = sf.lib()
    mesh = {"jj": np.ones((6, 2), dtype=np.int32, order="F"), "ww": np.zeros((6, 7), order="F"),
            "dw": np.zeros((2, 6, 7, 2), order="F"), "rr": np.ones((2, 5), order="F")}
    V = np.zeros((5, 6, 2), order="F")
    mesh["jj"][3, 1] = 9  # node 9 of 5
    with pytest.raises(sf.SfnlError) as e:
        sf.smb_cross_prod_gauss_sft_par(None, mesh, [0, 1], V)
    assert e.value.code == -1 and "jj" in sf.last_error()
    mesh["jj"][3, 1] = 2
    mesh["rr"] = np.ones((3, 5), order="F")  # k_d = 3
    with pytest.raises(sf.SfnlError) as e:
        sf.smb_cross_prod_gauss_sft_par(None, mesh, [0, 1], V)
    assert e.value.code == -4
    d = ctypes.c_void_p(16)
    assert L.sfnl_cross_gauss_f64(d, d, d, d, d, d, None, d, 5, 2, 11, 7, 2, 0, None, NULL) == -4  # n_w > 10
    assert L.sfnl_cross_gauss_f64(d, d, d, d, d, d, None, d, 0, 2, 6, 7, 2, 0, None, NULL) == -1


def test_other_gauss_point_entry_checks():
    # the Lorentz-force and advection callers reject what the Navier-Stokes one rejects, before any copy
    L = sf.lib()
    mesh = {"jj": np.ones((6, 2), dtype=np.int32, order="F"), "ww": np.zeros((6, 7), order="F"),
            "dw": np.zeros((2, 6, 7, 2), order="F"), "rr": np.ones((2, 5), order="F")}
    V = np.zeros((5, 6, 2), order="F")
    C = np.zeros((5, 2, 2), order="F")
    mesh["jj"][0, 0] = 0  # node numbers are 1-based
    for call in (lambda: sf.smb_CurlH_cross_B_gauss_sft_par(None, mesh, [0, 1], V, V),
                 lambda: sf.smb_ugradc_gauss_fft_par(None, mesh, [0, 1], V, C),
                 lambda: sf.smb_ugradc_gauss_fft_par_conc(None, mesh, [0, 1], V, C)):
        with pytest.raises(sf.SfnlError) as e:
            call()
        assert e.value.code == -1 and "jj" in sf.last_error()
    mesh["jj"][0, 0] = 1
    with pytest.raises(sf.SfnlError) as e:
        sf.smb_ugradc_gauss_fft_par(None, mesh, [0, 1], V, C, nb_procs=2)
    assert e.value.code == -4
    with pytest.raises(sf.SfnlError) as e:
        sf.smb_ugradc_gauss_fft_par_temperature(None, mesh, [0, 1], np.ones(1), V, C)  # 1 value, 2 elements
    assert e.value.code == -1
    d = ctypes.c_void_p(16)
    assert L.sfnl_ugradc_gauss_f64(d, d, None, 2, d, d, d, d, d, d, 5, 2, 6, 7, 2, 0, None, NULL) == -1
    assert L.sfnl_ugradc_gauss_f64(d, None, None, 0, d, d, d, d, d, d, 5, 2, 6, 7, 2, 0, None, NULL) == -1
    assert L.sfnl_curlh_cross_b_gauss_f64(d, None, d, d, d, d, d, d, 5, 2, 6, 7, 2, 0, None, NULL) == -1
    assert L.sfnl_curlh_cross_b_gauss_f64(d, d, d, d, d, d, d, d, 5, 2, 11, 7, 2, 0, None, NULL) == -4
    assert L.sfnl_smb_ugradc_gauss(d, d, None, 3, d, d, d, d, 2, d, d, 5, 2, 6, 7, 2, 1) == -1


def test_gauss_point_entries_with_no_elements_do_nothing():
    # me = 0: no Gauss points, nothing to launch (and no device needed)
    L = sf.lib()
    d = ctypes.c_void_p(16)
    assert L.sfnl_cross_gauss_f64(d, d, d, d, d, d, None, d, 5, 0, 6, 7, 4, 0, None, NULL) == 0
    assert L.sfnl_curlh_cross_b_gauss_f64(d, d, d, d, d, d, d, d, 5, 0, 6, 7, 4, 0, None, NULL) == 0
    for cons in (0, 1):
        assert L.sfnl_ugradc_gauss_f64(d, d, None, cons, d, d, d, d, d, d, 5, 0, 6, 7, 4, 0, None, NULL) == 0


def test_profiling_mesh_is_a_consistent_p2_mesh():
    # the structured P2 mesh of the profiling driver: partition of unity, exact derivatives of linear
    # fields, and the solid-body-rotation curl of the Navier-Stokes caller's restatement
    from sfemans_b200.profile_case import p2_rectangle
    from oracle import ref_fft as R

    m = p2_rectangle(5, 4)
    assert m["jj"].shape == (6, 40) and m["jj"].min() == 1 and m["jj"].max() == m["np"]
    assert np.abs(m["ww"].sum(axis=0) - 1.0).max() < 1e-14
    assert np.abs(m["dw"].sum(axis=1)).max() < 1e-12
    for c in range(2):
        d = np.einsum("dnle,ne->dle", m["dw"], m["rr"][c][m["jj"] - 1])
        assert np.abs(d[c] - 1.0).max() < 1e-12 and np.abs(d[1 - c]).max() < 1e-12
    V = np.zeros((m["np"], 6, 1), order="F")
    V[:, 2, 0] = m["rr"][0]
    _, rot, _ = R.c_cross_gauss(V, dict(m, n_w=6, l_G=7), [0], product=False)
    assert np.abs(rot[:, 4, 0] - 2.0).max() < 1e-12


def test_gauss_operands_entry_checks():
    L = sf.lib()
    d = ctypes.c_void_p(16)
    ops = [d, d, None, None]
    assert L.sfnl_gauss_operands_f64(3, d, d, None, None, 0, d, d, d, d, d, *ops, 5, 2, 6, 7, 2, NULL) == -1  # kind
    assert L.sfnl_gauss_operands_f64(2, d, d, None, None, 2, d, d, d, d, d, *ops, 5, 2, 6, 7, 2, NULL) == -1  # flag
    assert L.sfnl_gauss_operands_f64(1, d, None, None, None, 0, d, d, d, d, d, *ops, 5, 2, 6, 7, 2, NULL) == -1  # no B
    assert L.sfnl_gauss_operands_f64(2, d, d, None, None, 1, d, d, d, d, d, *ops, 5, 2, 6, 7, 2, NULL) == -1  # no o2/o3
    assert L.sfnl_gauss_operands_f64(0, d, None, None, None, 0, d, d, d, d, d, *ops, 5, 2, 11, 7, 2, NULL) == -4  # n_w
    assert L.sfnl_gauss_operands_f64(0, d, None, None, None, 0, d, d, d, d, d, *ops, 5, 0, 6, 7, 2, NULL) == 0  # me = 0


def _pack(L, V, nslot, mc, P, bloc, ew=1):
    npts = V.shape[-3] if ew == 3 else V.shape[0]
    send = np.zeros(P * bloc * nslot * mc * ew)
    assert L.sfnl_fft_par_pack_modes(ctypes.c_void_p(V.ctypes.data), ctypes.c_void_p(send.ctypes.data), npts, nslot,
                                     mc, P, bloc, ew) == 0
    return send.reshape(P, mc, nslot, bloc * ew)


@pytest.mark.parametrize("npts,nslot,m,P", [(23, 6, 6, 2), (31, 2, 9, 3), (7, 6, 4, 4), (1, 6, 2, 2)])
def test_mode_exchange_layout(npts, nslot, m, P):
    # rank r holds modes [r*mc, (r+1)*mc); after pack + all-to-all, rank q's received buffers hold block q of
    # every mode (global mode r*mc + i from peer r); sending the block's modes back and unpacking returns each
    # rank its own modes of every point (fft_parallel.F90:205-217, :306-324)
    L = sf.lib()
    mc, bloc = m // P, npts // P + 1
    V = R.synthetic_field(npts, nslot, m, 0.1, 5)
    local = [np.asfortranarray(V[:, :, r * mc:(r + 1) * mc]) for r in range(P)]
    sends = [_pack(L, local[r], nslot, mc, P, bloc) for r in range(P)]
    for q in range(P):
        recv = np.stack([sends[r][q] for r in range(P)])  # (P, mc, nslot, bloc)
        block = np.zeros((bloc, nslot, m))
        for r in range(P):
            block[:, :, r * mc:(r + 1) * mc] = recv[r].transpose(2, 1, 0)
        want = np.zeros((bloc, nslot, m))
        hi = min(npts, (q + 1) * bloc)
        if hi > q * bloc:
            want[:hi - q * bloc] = V[q * bloc:hi]
        assert np.array_equal(block, want)
    # identity "product": back[q'] = modes of q' of my block; then unpack
    backs = []
    for q in range(P):
        recv = np.stack([sends[r][q] for r in range(P)])
        backs.append(recv)  # modes of peer r are exactly what r sent: back[r] = recv[r]
    for r in range(P):
        got = np.ascontiguousarray(np.stack([backs[q][r] for q in range(P)]))
        out = np.zeros((npts, nslot, mc), order="F")
        assert L.sfnl_fft_par_unpack_modes(ctypes.c_void_p(got.ctypes.data), ctypes.c_void_p(out.ctypes.data), npts,
                                           nslot, mc, P, bloc, 1) == 0
        assert np.array_equal(out, local[r])


def test_mode_exchange_argument_checks():
    L = sf.lib()
    a = ctypes.c_void_p(16)
    assert L.sfnl_fft_par_pack_modes(a, a, 10, 6, 2, 2, 4, 1) == -2  # np > nb_procs*bloc_size
    assert L.sfnl_fft_par_pack_modes(a, a, 10, 6, 2, 2, 5, 2) == -1  # ew must be 1 or 3
    assert L.sfnl_fft_par_unpack_modes(a, a, 10, 6, 0, 2, 5, 1) == -1
    assert L.sfnl_fft_par_block(9, a, a, a, 5, 2, 2, 3, None) == -1  # unknown op
