"""Time one program of the library on synthetic data (the command the ncu captures use).

    python -m sfemans_b200.profile_case --program bundle --form fast --np 100000 --m 64 --reps 1

Programs: cross, dot, prod, div, svect, svdiv, tensor, tension (the reference routines, by the op names of
sfemans_b200.KINDS), bundle (u x w, u x b, j x b, u . gradT), and the synthesis-only real (grid values of a
3-vector, FFT_PAR_REAL) and maxvel (FFT_MAX_VEL_DCL), fp64peak (the FP64 pipe's DMMA and DFMA throughput), and the linearised programs cross_jvp, cross_vjp,
mhd_jvp, mhd_vjp on --k tangents (or cotangents) at one base state, and the Gauss-point callers gauss_ns,
gauss_lorentz and gauss_advect on a P2 mesh of about --np Gauss points (nodal fields as inputs).
Forms: fast (FP64, folded transforms), grid (FP64, caller's grid), split3 / split2 (bf16 slices on tcgen05).
Inputs are N(0,1)*exp(-alpha*n) coefficients generated on the device; the padding is m_max_pad = 3*m/2.
Prints the average milliseconds per call, timed with CUDA events after one untimed call.
"""
from __future__ import annotations

import argparse


def p2_rectangle(nr: int, nz: int):
    """A P2 triangle mesh of the meridian rectangle r in [0.1, 1.1], z in [0, 1] (nr x nz squares, two
    triangles each) in the arrays the Gauss-point callers read (numpy, Fortran order): jj (6, me) 1-based
    nodes (3 vertices, then the midpoints of edges 2-3, 3-1, 1-2), rr (2, np_nodes), and at 7 interior
    quadrature points ww (6, 7) = the P2 basis and dw (2, 6, 7, me) = its (d/dr, d/dz) on each element."""
    import numpy as np

    nv = (nr + 1) * (nz + 1)
    nh, nvt, nd = nr * (nz + 1), (nr + 1) * nz, nr * nz
    i, j = np.meshgrid(np.arange(nr), np.arange(nz), indexing="ij")
    i, j = i.ravel(), j.ravel()
    v = lambda a, b: a * (nz + 1) + b  # noqa: E731
    H = lambda a, b: nv + a * (nz + 1) + b  # noqa: E731  edge (a, b)-(a+1, b)
    V = lambda a, b: nv + nh + a * nz + b  # noqa: E731  edge (a, b)-(a, b+1)
    D = lambda a, b: nv + nh + nvt + a * nz + b  # noqa: E731  edge (a, b)-(a+1, b+1)
    a, b, c, d = v(i, j), v(i + 1, j), v(i + 1, j + 1), v(i, j + 1)
    t1 = np.stack([a, b, c, V(i + 1, j), D(i, j), H(i, j)])
    t2 = np.stack([a, c, d, H(i, j + 1), V(i, j), D(i, j)])
    jj = np.empty((6, 2 * nd), dtype=np.int32)
    jj[:, 0::2], jj[:, 1::2] = t1, t2
    vr, vz = np.meshgrid(0.1 + np.arange(nr + 1) / nr, np.arange(nz + 1) / nz, indexing="ij")
    vr, vz = vr.ravel(), vz.ravel()
    pts = np.zeros((2, nv + nh + nvt + nd))
    pts[0, :nv], pts[1, :nv] = vr, vz
    ia, ja = np.meshgrid(np.arange(nr), np.arange(nz + 1), indexing="ij")
    pts[:, nv:nv + nh] = 0.5 * (pts[:, v(ia, ja).ravel()] + pts[:, v(ia + 1, ja).ravel()])
    ib, jb = np.meshgrid(np.arange(nr + 1), np.arange(nz), indexing="ij")
    pts[:, nv + nh:nv + nh + nvt] = 0.5 * (pts[:, v(ib, jb).ravel()] + pts[:, v(ib, jb + 1).ravel()])
    pts[:, nv + nh + nvt:] = 0.5 * (pts[:, v(i, j)] + pts[:, v(i + 1, j + 1)])
    L = np.array([[1 / 3, 2 / 3, 1 / 6, 1 / 6, 0.1, 0.45, 0.45], [1 / 3, 1 / 6, 2 / 3, 1 / 6, 0.45, 0.1, 0.45],
                  [1 / 3, 1 / 6, 1 / 6, 2 / 3, 0.45, 0.45, 0.1]])  # barycentric coordinates of the 7 points
    ww = np.vstack([L[0] * (2 * L[0] - 1), L[1] * (2 * L[1] - 1), L[2] * (2 * L[2] - 1),
                    4 * L[1] * L[2], 4 * L[2] * L[0], 4 * L[0] * L[1]])
    dl = np.zeros((6, 3, 7))  # d(basis)/d(lambda_k)
    for k in range(3):
        dl[k, k] = 4 * L[k] - 1
    for e, (x, y) in enumerate(((1, 2), (2, 0), (0, 1))):
        dl[3 + e, x] = 4 * L[y]
        dl[3 + e, y] = 4 * L[x]
    P = pts[:, jj[:3]]  # (2 coords, 3 vertices, me)
    T = np.stack([np.stack([P[0, 0] - P[0, 2], P[0, 1] - P[0, 2]]), np.stack([P[1, 0] - P[1, 2], P[1, 1] - P[1, 2]])])
    det = T[0, 0] * T[1, 1] - T[0, 1] * T[1, 0]
    G = np.stack([np.stack([T[1, 1], -T[0, 1]]), np.stack([-T[1, 0], T[0, 0]])]) / det  # rows: dlambda_1,2/d(r, z)
    dlam = np.stack([G[0], G[1], -G[0] - G[1]])  # (3 lambdas, 2 coords, me)
    dw = np.einsum("nkl,kde->dnle", dl, dlam)
    return {"jj": np.asfortranarray(jj + 1), "rr": np.asfortranarray(pts), "ww": np.asfortranarray(ww),
            "dw": np.asfortranarray(dw), "np": pts.shape[1], "me": 2 * nd}


# Gauss-point callers: nodal fields (slots) and the library call
GAUSS = ("gauss_ns", "gauss_lorentz", "gauss_advect")

# linearised programs: base fields, input slots per tangent, output slots per tangent
LINEAR = {"cross_jvp": (2, 12, 6), "cross_vjp": (2, 6, 12), "mhd_jvp": (3, 18, 12), "mhd_vjp": (3, 12, 18)}


def _field(torch, npts, nslot, m, alpha, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    t = torch.randn((m, nslot, npts), generator=g, device="cuda", dtype=torch.float64)
    t *= torch.exp(-alpha * torch.arange(m, device="cuda", dtype=torch.float64))[:, None, None]
    t[0, 1::2, :] = 0.0
    return t.permute(2, 1, 0)


def main(argv=None):
    import torch

    import sfemans_b200 as sf

    ap = argparse.ArgumentParser()
    ap.add_argument("--program", default="cross",
                    choices=list(sf.KINDS) + ["bundle", "real", "maxvel", "fp64peak"] + list(LINEAR) + list(GAUSS))
    ap.add_argument("--form", default="fast", choices=["fast", "grid", "split3", "split2"])
    ap.add_argument("--np", type=int, default=100_000)
    ap.add_argument("--m", type=int, default=64)
    ap.add_argument("--alpha", type=float, default=0.1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--k", type=int, default=1, help="tangents (cotangents) of a linearised program")
    ap.add_argument("--residues", type=int, default=0,
                    help="residue classes of the large-m FAST form (3, 6 or 12; 0: the library's choice)")
    a = ap.parse_args(argv)
    if a.residues:
        sf._check(sf.lib().sfnl_test_large_residues(a.residues))
    kw = {"fast": dict(algo=sf.ALGO_FAST), "grid": dict(algo=sf.ALGO_GRID), "split3": dict(split=sf.SPLIT_BF16X3),
          "split2": dict(split=sf.SPLIT_BF16X2)}[a.form]
    pad = 3 * a.m // 2 if a.m > 1 else 1
    if a.program == "fp64peak":  # FP64 pipe throughput (the FP64 forms' compute roofline)
        import ctypes

        dm, df = ctypes.c_double(), ctypes.c_double()
        sf._check(sf.lib().sfnl_probe_fp64_tflops(ctypes.byref(dm), ctypes.byref(df)))
        print(f"fp64peak: mma.sync.m8n8k4.f64 {dm.value:.2f} TFLOP/s, DFMA {df.value:.2f} TFLOP/s", flush=True)
        return
    if a.program in ("real", "maxvel"):
        x = _field(torch, a.np, 6, a.m, a.alpha, 1)
        if a.program == "real":
            out = sf.synthesis(x)
            call = lambda: sf.synthesis(x, out=out)  # noqa: E731
        else:
            call = lambda: sf.max_vel(x, pad)  # noqa: E731
    elif a.program in GAUSS:
        import math

        import numpy as np

        side = max(1, int(math.ceil(math.sqrt(a.np / 14.0))))  # about np Gauss points (7 per triangle)
        mesh = p2_rectangle(side, side)
        dmesh = {k: torch.from_numpy(np.ascontiguousarray(mesh[k].T)).cuda().permute(*range(mesh[k].ndim - 1, -1, -1))
                 for k in ("jj", "ww", "dw", "rr")}
        lm = torch.arange(a.m, dtype=torch.int32, device="cuda")
        v = _field(torch, mesh["np"], 6, a.m, a.alpha, 41)
        if a.program == "gauss_ns":
            call = lambda: sf.cross_gauss(v, dmesh, lm, m_max_pad=pad)  # noqa: E731
        elif a.program == "gauss_lorentz":
            b2 = _field(torch, mesh["np"], 6, a.m, a.alpha, 42)
            call = lambda: sf.curlh_cross_b_gauss(v, b2, dmesh, lm, m_max_pad=pad)  # noqa: E731
        else:
            c = _field(torch, mesh["np"], 2, a.m, a.alpha, 43)
            heat = torch.linspace(0.5, 2.0, mesh["me"], device="cuda", dtype=torch.float64)
            call = lambda: sf.ugradc_gauss(v, c, dmesh, lm, heat=heat, conservative=True, m_max_pad=pad)  # noqa: E731
        a.np = 7 * mesh["me"]
    elif a.program in LINEAR:
        nbase, nin, nout = LINEAR[a.program]
        fn = getattr(sf, a.program)
        base = [_field(torch, a.np, 6, a.m, a.alpha, 20 + i) for i in range(nbase)]
        x = sf.fortran_empty(a.np, nin, a.m, a.k)
        for t in range(a.k):
            x[..., t] = _field(torch, a.np, nin, a.m, a.alpha, 30 + t)
        out = sf.fortran_empty(a.np, nout, a.m, a.k)
        lk = {"split": kw["split"]} if "split" in kw else {}
        if lk and not a.program.startswith("mhd"):
            raise SystemExit("split forms of the linearised programs: mhd_jvp and mhd_vjp only")
        call = lambda: fn(*base, x, m_max_pad=pad, out=out, **lk)  # noqa: E731
    elif a.program == "bundle":
        ins = [_field(torch, a.np, 6, a.m, a.alpha, 10 + i) for i in range(5)]
        outs = tuple(sf.fortran_empty(a.np, 6, a.m) for _ in range(3)) + (sf.fortran_empty(a.np, 2, a.m),)
        call = lambda: sf.bundle_mhd(*ins, m_max_pad=pad, outs=outs, **kw)  # noqa: E731
    else:
        op, nsl1, nsl2, _ = sf.KINDS[a.program]
        x, y = _field(torch, a.np, nsl1, a.m, a.alpha, 1), _field(torch, a.np, nsl2, a.m, a.alpha, 2)
        if a.program in ("div", "svdiv"):
            y[:, 0, 0] += 4.0  # keep the divisor away from 0
        out = sf.out_empty(op, a.np, a.m)
        call = lambda: sf.product(op, x, y, out=out, m_max_pad=pad, **kw)  # noqa: E731
    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    ks = f" k={a.k}" if a.program in LINEAR else ""
    print(f"{a.program} {a.form} np={a.np} m={a.m}{ks}: {e0.elapsed_time(e1) / a.reps:.4f} ms/call", flush=True)


if __name__ == "__main__":
    main()
