"""GPU parity of the synthesis-only routines of MODULE fft_parallele:
FFT_PAR_REAL (fft_parallel.F90:28-145, the field values on the grid, used
for visualisation output) and FFT_MAX_VEL_DCL (:1426-1541, the maximum of
|v| on the grid, used for the CFL number).

Bars: grid values rel-L2 <= 1e-12 per field against the long-double oracle
(FP64_TOL); the maximum within 1e-13 relative (MAX_TOL: one FP64 synthesis
and square root against a long-double one).
"""
import glob
import os

import numpy as np
import pytest

import sfemans_b200 as sf
from oracle import ref_fft as R

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MAX_TOL = 1e-13
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def dev(a):
    return sf.to_device(a)


def host(t):
    return sf.to_host(t)


def _worst_field(got, ref):
    return max(R.rel_l2(got[:, f, :], ref[:, f, :]) for f in range(ref.shape[1]))


@pytest.mark.parametrize("npts,nsl,m,opt", [(1, 2, 1, None), (5, 6, 2, None), (33, 6, 5, 20), (257, 2, 16, None),
                                            (130, 4, 13, 40), (1000, 6, 32, None), (77, 6, 64, 191)])
def test_grid_values_match_oracle(npts, nsl, m, opt):
    V = R.synthetic_field(npts, nsl, m, 0.2, 700 + m)
    ref = R.c_real(V, opt_nb_plane=opt)
    out = host(sf.synthesis(dev(V), n_theta=sf.real_planes(m, opt)))
    assert out.shape == ref.shape
    assert _worst_field(out, ref) <= FP64_TOL
    # the reference signature on host arrays
    assert _worst_field(sf.FFT_PAR_REAL(None, V, opt_nb_plane=opt), ref) <= FP64_TOL


@pytest.mark.parametrize("npts,nsl,m,pad", [(1, 6, 1, 1), (5, 2, 2, 3), (33, 6, 5, 7), (257, 6, 16, 24),
                                            (130, 2, 13, 19), (1000, 6, 32, 48), (77, 6, 64, 96), (64, 4, 8, 12)])
def test_max_velocity_matches_oracle(npts, nsl, m, pad):
    V = R.synthetic_field(npts, nsl, m, 0.2, 800 + m)
    ref = R.c_max_vel(V, pad)
    assert abs(sf.max_vel(dev(V), pad) - ref) <= MAX_TOL * ref
    assert abs(sf.FFT_MAX_VEL_DCL(None, V, 1, npts + 1, pad) - ref) <= MAX_TOL * ref


def test_max_velocity_of_a_unit_field():
    # u = (cos t, sin t, 0) has |u| = 1 at every angle
    U = np.zeros((50, 6, 4), order="F")
    U[:, 0, 1] = 1.0
    U[:, 3, 1] = 1.0
    assert abs(sf.max_vel(dev(U), 6) - 1.0) <= 1e-15
    assert sf.max_vel(dev(np.zeros((50, 6, 4), order="F")), 6) == 0.0


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "real_*.npz")) +
                                        glob.glob(os.path.join(GOLD, "maxvel_*.npz"))))
def test_synthesis_fixtures(path):
    # fixtures made with several emulated Fourier ranks: the global result does not depend on them
    z = np.load(path)
    npts, m, extra, procs = (int(v) for v in z["meta"])
    if str(z["kind"]) == "real":
        out = host(sf.synthesis(dev(z["V1"]), n_theta=sf.real_planes(m, extra or None)))
        assert _worst_field(out, z["out"]) <= FP64_TOL
    else:
        assert abs(sf.max_vel(dev(z["V1"]), extra) - z["out"][0]) <= MAX_TOL * z["out"][0]


def test_host_entry_points_in_chunks():
    # more points than one chunk of the host pipeline: the (N, nf, np) output is cut by points
    npts, m = 150_000, 32
    V = R.synthetic_field(npts, 6, m, 0.2, 901)
    out = sf.FFT_PAR_REAL(None, V)
    assert _worst_field(out, R.synth_grid(V, 2 * m - 1, workers=8)) <= FP64_TOL
    g = R.synth_grid(V, 95, workers=8)
    ref = float(np.sqrt((g ** 2).sum(axis=1)).max())
    assert abs(sf.FFT_MAX_VEL_DCL(None, V, 1, npts, 48) - ref) <= MAX_TOL * ref
