"""Time one program of the library on synthetic data (the command the ncu captures use).

    python -m sfemans_b200.profile_case --program bundle --form fast --np 100000 --m 64 --reps 1

Programs: cross, dot, prod, div, svect, svdiv, tensor, tension (the reference routines, by the op names of
sfemans_b200.KINDS), bundle (u x w, u x b, j x b, u . gradT), and the synthesis-only real (grid values of a
3-vector, FFT_PAR_REAL) and maxvel (FFT_MAX_VEL_DCL), and the linearised programs cross_jvp, cross_vjp,
mhd_jvp, mhd_vjp on --k tangents (or cotangents) at one base state.
Forms: fast (FP64, folded transforms), grid (FP64, caller's grid), split3 / split2 (bf16 slices on tcgen05).
Inputs are N(0,1)*exp(-alpha*n) coefficients generated on the device; the padding is m_max_pad = 3*m/2.
Prints the average milliseconds per call, timed with CUDA events after one untimed call.
"""
from __future__ import annotations

import argparse


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
    ap.add_argument("--program", default="cross", choices=list(sf.KINDS) + ["bundle", "real", "maxvel"] + list(LINEAR))
    ap.add_argument("--form", default="fast", choices=["fast", "grid", "split3", "split2"])
    ap.add_argument("--np", type=int, default=100_000)
    ap.add_argument("--m", type=int, default=64)
    ap.add_argument("--alpha", type=float, default=0.1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--k", type=int, default=1, help="tangents (cotangents) of a linearised program")
    a = ap.parse_args(argv)
    kw = {"fast": dict(algo=sf.ALGO_FAST), "grid": dict(algo=sf.ALGO_GRID), "split3": dict(split=sf.SPLIT_BF16X3),
          "split2": dict(split=sf.SPLIT_BF16X2)}[a.form]
    pad = 3 * a.m // 2 if a.m > 1 else 1
    if a.program in ("real", "maxvel"):
        x = _field(torch, a.np, 6, a.m, a.alpha, 1)
        if a.program == "real":
            out = sf.synthesis(x)
            call = lambda: sf.synthesis(x, out=out)  # noqa: E731
        else:
            call = lambda: sf.max_vel(x, pad)  # noqa: E731
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
