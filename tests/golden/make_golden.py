"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

Each case stores the seeded inputs and the long-double oracle's output
(oracle/sfnl_oracle.c, the step-by-step restatement of
SOURCES/POST_PROCESSING/fft_parallel.F90:147-830, :1021-1220, :1543-1796).
Cases are small so that the fixtures stay a few hundred KB in total.  The
exact spectral convolution (oracle/ref_fft.py) is checked against every
bilinear case before it is written, so a fixture is only produced when two
independent formulations agree to 1e-15.  The quotients and the tension
tensor depend on the grid; their cases are checked against the pocketfft
restatement on the same grid (1e-13) instead.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_fft as R  # noqa: E402

# name, op, np, m, m_max_pad, nb_procs, alpha, seed
CASES = [
    ("cross_np37_m5", "cross", 37, 5, 7, 1, 0.3, 11),
    ("dot_np37_m5", "dot", 37, 5, 7, 1, 0.3, 12),
    ("prod_np37_m5", "prod", 37, 5, 7, 1, 0.3, 13),
    ("cross_np64_m16", "cross", 64, 16, 24, 1, 0.3, 14),   # the 3/2-rule pad of the 28k-point case
    ("cross_np29_m6_p3", "cross", 29, 6, 9, 3, 0.2, 15),   # 3 Fourier ranks, dummy points
    ("dot_np29_m6_p2", "dot", 29, 6, 9, 2, 0.2, 16),
    ("prod_np33_m7", "prod", 33, 7, 10, 1, 0.1, 17),       # m odd: N = 3m-2, the alias-free limit
    ("cross_np1_m3", "cross", 1, 3, 4, 1, 0.5, 18),        # single point
    ("cross_np40_m1", "cross", 40, 1, 1, 1, 0.0, 19),      # mode 0 only, N = 1
    ("dot_np70_m32", "dot", 70, 32, 48, 1, 0.05, 20),      # slow decay
    ("svect_np37_m5", "svect", 37, 5, 7, 1, 0.3, 21),      # FFT_SCALAR_VECT_DCL pb = 1
    ("svect_np31_m8_p2", "svect", 31, 8, 12, 2, 0.2, 22),
    ("svdiv_np37_m5", "svdiv", 37, 5, 7, 1, 0.3, 23),      # FFT_SCALAR_VECT_DCL pb = 2
    ("tensor_np37_m5", "tensor", 37, 5, 7, 1, 0.3, 24),    # FFT_TENSOR_DCL
    ("tensor_np29_m6_p3", "tensor", 29, 6, 9, 3, 0.2, 25),
    ("tension_np37_m5", "tension", 37, 5, 7, 1, 0.3, 26),  # FFT_TENSOR_DCL, opt_tension
    ("div_np37_m5", "div", 37, 5, 7, 1, 0.3, 27),          # FFT_PAR_DIV_DCL
    ("div_np33_m8_p2", "div", 33, 8, 12, 2, 0.2, 28),
]

# (slots of V1, slots of V2) per routine
SLOTS = {"cross": (6, 6), "dot": (6, 6), "prod": (2, 2), "div": (2, 2), "svect": (6, 2), "svdiv": (6, 2),
         "tensor": (6, 6), "tension": (6, 6)}
DENOMINATOR_OFFSET = 4.0  # added to the mode-0 cosine of a divisor so that it stays away from 0


def inputs(op, npts, m, alpha, seed):
    n1, n2 = SLOTS[op]
    V1 = R.synthetic_field(npts, n1, m, alpha, 1000 + seed)
    V2 = R.synthetic_field(npts, n2, m, alpha, 2000 + seed)
    if op in ("div", "svdiv"):
        V2[:, 0, 0] += DENOMINATOR_OFFSET
    return V1, V2


def make(case):
    name, op, npts, m, pad, procs, alpha, seed = case
    V1, V2 = inputs(op, npts, m, alpha, seed)
    out = R.c_oracle(op, V1, V2, pad, nb_procs=procs)
    if op in ("div", "svdiv", "tension"):
        err = R.rel_l2(out, R.fft_par(op, V1, V2, pad))
        assert err < 1e-13, (name, err)
    else:
        err = R.rel_l2(out, R.spectral_product(op, V1, V2))
        assert err < 1e-15, (name, err)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), V1=V1, V2=V2, out=out,
                        meta=np.array([npts, m, pad, procs], dtype=np.int64), op=np.array(op))
    return name, err


# synthesis-only routines: name, kind, np, nslot, m, nb_procs, opt_nb_plane (real) or m_max_pad (maxvel), alpha, seed
SYNTH_CASES = [
    ("real_np11_m6", "real", 11, 6, 6, 1, 0, 0.3, 31),          # FFT_PAR_REAL, N = 2m-1
    ("real_np12_m6_p3_opt20", "real", 12, 2, 6, 3, 20, 0.2, 32),  # 3 ranks, opt_nb_plane: N = 19
    ("maxvel_np13_m5", "maxvel", 13, 6, 5, 1, 7, 0.3, 33),       # FFT_MAX_VEL_DCL, |3-vector|
    ("maxvel_np13_m6_p2", "maxvel", 13, 2, 6, 2, 9, 0.2, 34),    # |scalar|, 2 ranks, dummy points
]


def make_synth(case):
    name, kind, npts, nsl, m, procs, extra, alpha, seed = case
    V = R.synthetic_field(npts, nsl, m, alpha, 3000 + seed)
    if kind == "real":
        out = R.c_real(V, nb_procs=procs, opt_nb_plane=extra or None)
        err = R.rel_l2(out, R.synth_grid(V, out.shape[0]))
    else:
        out = np.array([R.c_max_vel(V, extra, nb_procs=procs)])
        g = R.synth_grid(V, 2 * extra - 1)
        ex = np.sqrt((g[:, :3] ** 2).sum(axis=1)).max() if nsl == 6 else np.abs(g[:, 0]).max()
        err = abs(out[0] - ex) / ex
    assert err < 1e-14, (name, err)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), V1=V, out=out,
                        meta=np.array([npts, m, extra, procs], dtype=np.int64), kind=np.array(kind))
    return name, err


if __name__ == "__main__":
    for c in CASES:
        print(*make(c))
    for c in SYNTH_CASES:
        print(*make_synth(c))
