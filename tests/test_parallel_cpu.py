"""Multi-rank host logic on CPU (gloo): point sharding and the reference's
mode-distributed layout with its two all-to-all exchanges
(fft_parallel.F90:217, :306).  The per-rank product on the gathered block
is the CPU oracle here (no GPU in this process); on GPUs it is the CUDA
kernel and the exchange runs over NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import ref_fft as R
import sfemans_b200 as sf
from sfemans_b200 import KINDS
from sfemans_b200.parallel import (fft_max_vel_distributed, fft_par_distributed, fft_par_real_distributed, shard_range,
                                   smb_gauss_distributed)


@pytest.mark.parametrize("npts,world", [(0, 1), (7, 3), (28000, 8), (1_400_000, 8), (5, 8)])
def test_shard_range_partitions_points(npts, world):
    spans = [shard_range(npts, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == npts
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_compute(kind, xb, yb, m_max_pad):
    to_np = lambda t: np.asfortranarray(t.permute(2, 1, 0).contiguous().numpy().T)  # noqa: E731
    out = R.c_oracle(kind, to_np(xb), to_np(yb), m_max_pad)
    return torch.from_numpy(np.ascontiguousarray(out.T)).permute(*reversed(range(out.ndim)))


def _worker(rank, world, port, kind, npts, m, pad, bloc, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, nsl1, nsl2, nout = KINDS[kind]
        V1 = R.synthetic_field(npts, nsl1, m, 0.2, 41)
        V2 = R.synthetic_field(npts, nsl2, m, 0.2, 42)
        if kind in ("div", "svdiv"):
            V2[:, 0, 0] += 4.0  # keep the divisor away from 0
        mc = m // world
        loc = lambda V: torch.from_numpy(np.ascontiguousarray(V[:, :, rank * mc:(rank + 1) * mc].T)).permute(2, 1, 0)  # noqa: E731
        if kind in ("tensor", "tension"):
            out = torch.zeros((mc, 6, npts, 3), dtype=torch.float64).permute(3, 2, 1, 0)
        else:
            out = torch.zeros((mc, nout, npts), dtype=torch.float64).permute(2, 1, 0)
        temps = np.full(3, 7.0)  # the reference zeroes temps on entry, then adds each stage's seconds
        fft_par_distributed(kind, None, loc(V1), loc(V2), out, world, bloc, pad, temps=temps, compute=_oracle_compute)
        ref = R.c_oracle(kind, V1, V2, pad)[..., rank * mc:(rank + 1) * mc]
        err = float(np.abs(out.numpy() - ref).max())
        if not (np.all(temps >= 0.0) and np.all(temps < 7.0) and temps[1] > 0.0):
            err = float("inf")  # temps not zeroed on entry, or the product's seconds missing
        q.put((rank, err))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world,npts,m", [("cross", 2, 23, 6), ("dot", 3, 31, 9), ("prod", 2, 40, 4),
                                                ("div", 2, 17, 4), ("svect", 2, 19, 6), ("svdiv", 3, 13, 6),
                                                ("tensor", 2, 21, 4), ("tension", 3, 11, 6)])
def test_mode_distributed_layout_matches_single_rank(kind, world, npts, m):
    pad = 3 * m // 2
    bloc = npts // world + 1  # the callers' bloc_size (subroutine_ns_with_velocity.F90:625)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, npts, m, pad, bloc, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = dict(q.get(timeout=5) for _ in range(world))
    assert all(p.exitcode == 0 for p in procs)
    for r in range(world):
        assert res[r] < 1e-14, res


def _synth_worker(rank, world, port, kind, npts, nsl, m, extra, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        V = R.synthetic_field(npts, nsl, m, 0.2, 61)
        mc = m // world
        loc = torch.from_numpy(np.ascontiguousarray(V[:, :, rank * mc:(rank + 1) * mc].T)).permute(2, 1, 0)
        to_np = lambda t: np.asfortranarray(t.permute(2, 1, 0).contiguous().numpy().T)  # noqa: E731
        if kind == "real":
            out = fft_par_real_distributed(None, loc, extra or None,
                                           compute=lambda xb, N: torch.from_numpy(
                                               np.ascontiguousarray(R.synth_grid(to_np(xb), N).T)).permute(2, 1, 0))
            bloc = npts // world
            ref = R.c_real(V, nb_procs=world, opt_nb_plane=extra or None)[:, :, rank * bloc:(rank + 1) * bloc]
            q.put((rank, float(np.abs(out.numpy() - ref).max())))
        else:
            bloc = npts // world + 1
            got = fft_max_vel_distributed(None, loc, world, bloc, extra,
                                          compute=lambda xb, pad: R.c_max_vel(to_np(xb), pad))
            q.put((rank, abs(got - R.c_max_vel(V, extra))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world,npts,nsl,m,extra", [("real", 2, 10, 6, 4, 0), ("real", 3, 9, 2, 6, 20),
                                                        ("maxvel", 2, 11, 6, 4, 6), ("maxvel", 3, 7, 2, 6, 9)])
def test_synthesis_routines_over_a_mode_distributed_communicator(kind, world, npts, nsl, m, extra):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_synth_worker, args=(r, world, port, kind, npts, nsl, m, extra, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = dict(q.get(timeout=5) for _ in range(world))
    assert all(p.exitcode == 0 for p in procs)
    for r in range(world):
        assert res[r] < 1e-14, res


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).permute(*reversed(range(a.ndim)))


def _oracle_operands(kind, V, mesh, lm, V2, omega, heat, conservative):
    to_np = lambda t: None if t is None else np.asfortranarray(t.permute(2, 1, 0).contiguous().numpy().T)  # noqa: E731
    if kind == sf.GAUSS_NS:
        _, rot, w = R.c_cross_gauss(to_np(V), mesh, lm, to_np(omega), product=False)
        return _t(rot), _t(w)
    if kind == sf.GAUSS_LORENTZ:
        _, rot, w = R.c_curlh_cross_b_gauss(to_np(V), to_np(V2), mesh, lm, product=False)
        return _t(rot), _t(w)
    _, g, w, d, cg = R.c_ugradc_gauss(to_np(V), to_np(V2), mesh, lm, heat=heat, conservative=conservative,
                                      product=False)
    return _t(g), _t(w), _t(d), _t(cg)


def _gauss_worker(rank, world, port, kind, cons, m, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh = R.synthetic_p2_mesh(4, 3, 9)
        lm = [2 * i + 1 for i in range(m)]  # a select_mode-like list of mode numbers
        V = R.synthetic_field(mesh["np"], 6, m, 0.2, 71)
        V2 = R.synthetic_field(mesh["np"], 6 if kind == sf.GAUSS_LORENTZ else 2, m, 0.2, 72)
        om = R.precession_omega(mesh["np"], lm, 0.4, 0.3) if kind == sf.GAUSS_NS else None
        heat = np.linspace(0.5, 2.0, mesh["me"]) if cons else None
        mc = m // world
        sl = slice(rank * mc, (rank + 1) * mc)
        loc = lambda A: None if A is None else _t(np.asfortranarray(A[:, :, sl]))  # noqa: E731
        out = smb_gauss_distributed(kind, None, mesh, lm[sl], loc(V), world, V2_in=loc(V2), omega=loc(om),
                                    heat=heat, conservative=cons, operands=_oracle_operands,
                                    compute=_oracle_compute)
        if kind == sf.GAUSS_NS:
            ref = R.c_cross_gauss(V, mesh, lm, om)[0]
        elif kind == sf.GAUSS_LORENTZ:
            ref = R.c_curlh_cross_b_gauss(V, V2, mesh, lm)[0]
        else:
            ref = R.c_ugradc_gauss(V, V2, mesh, lm, heat=heat, conservative=cons)[0]
        q.put((rank, float(np.abs(out.numpy() - ref[..., sl]).max() / np.abs(ref).max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,cons,world,m", [(0, False, 2, 4), (1, False, 3, 6), (2, False, 2, 4), (2, True, 2, 6)])
def test_gauss_point_callers_over_a_mode_distributed_communicator(kind, cons, world, m):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gauss_worker, args=(r, world, port, kind, cons, m, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = dict(q.get(timeout=5) for _ in range(world))
    assert all(p.exitcode == 0 for p in procs)
    for r in range(world):
        assert res[r] < 1e-13, res
