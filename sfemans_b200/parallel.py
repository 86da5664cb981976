"""Multi-rank plumbing around the single-GPU kernels.

Two decompositions, one process per GPU:

* Point sharding (the default, :func:`shard_range`): every point of the
  nonlinear term is independent (the transforms run along the azimuth of
  each point), so G GPUs each take a contiguous range of points and no data
  crosses NVLink.  bench.py runs this as weak scaling.

* The reference's mode-distributed layout (:func:`fft_par_distributed`):
  each rank owns m_max_c contiguous Fourier modes of every point
  (initialization.F90:823-835) and FFT_PAR_*_DCL transposes mode <-> point
  with two MPI_ALLTOALLs (fft_parallel.F90:217, :306).  Here the same two
  exchanges are ``torch.distributed.all_to_all_single`` calls (NCCL over
  NVLink on GPUs, gloo in the CPU tests), and the per-rank product on
  bloc_size points with all modes is the single-GPU kernel.  Dummy points
  beyond np are zero (the reference fills them with 1.d100, :211; they are
  dropped on output either way).
"""
from __future__ import annotations


def shard_range(npts: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) of the points rank ``rank`` of ``world`` owns."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, rem = divmod(npts, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def _default_compute(kind, x, y, m_max_pad):
    from . import KINDS, product

    return product(KINDS[kind][0], x, y, m_max_pad=m_max_pad)


def fft_par_distributed(kind, group, x, y, out, nb_procs, bloc_size, m_max_pad, temps=None, compute=None):
    """FFT_PAR_*_DCL, FFT_SCALAR_VECT_DCL or FFT_TENSOR_DCL over a mode-distributed communicator.

    kind: a key of ``sfemans_b200.KINDS``.  x, y: this rank's (np, nslot1, m_max_c) and
    (np, nslot2, m_max_c) tensors (Fortran layout); out: (np, nout, m_max_c), or (3, np, 6,
    m_max_c) for the tensor kinds.  ``compute(kind, xb, yb, m_max_pad)`` maps the gathered
    (bloc_size, nslot, m_max) blocks to the block's output; it defaults to the CUDA kernels.
    """
    import time

    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world != nb_procs:
        raise ValueError("nb_procs must equal the communicator size")
    if temps is not None:  # zeroed, then accumulated per stage as the reference does (:179, :203-290)
        temps[:] = 0.0
    sync = torch.cuda.synchronize if (temps is not None and x.is_cuda) else (lambda: None)
    clock = [time.perf_counter()]

    def lap(i):  # adds the time since the last lap to temps[i]: 0 exchange, 1 product, 2 repacking
        if temps is not None:
            sync()
            t = time.perf_counter()
            temps[i] += t - clock[0]
            clock[0] = t

    npts, nsl, mc = x.shape
    nsl2 = y.shape[1]
    np_tot = nb_procs * bloc_size
    if npts > np_tot:
        raise ValueError("np > nb_procs*bloc_size")
    compute = compute or _default_compute
    tensor_out = kind in ("tensor", "tension")

    def to_blocks(t, ns):
        # (np, ns, mc) -> send buffer [dest q][mode i][slot s][point n], points padded to np_tot.
        tp = torch.zeros((np_tot, ns, mc), dtype=t.dtype, device=t.device)
        tp[:npts] = t
        return tp.reshape(nb_procs, bloc_size, ns, mc).permute(0, 3, 2, 1).contiguous()

    send = torch.cat([to_blocks(x, nsl), to_blocks(y, nsl2)], dim=2)         # (P, mc, ns1+ns2, bloc)
    recv = torch.empty_like(send)
    lap(2)
    dist.all_to_all_single(recv.view(-1), send.view(-1), group=group)       # fft_parallel.F90:217
    lap(0)
    # recv[r] = source rank r's modes for my points -> (bloc, ns, m_max) Fortran layout with
    # global mode r*mc + i (the shiftl bookkeeping of :223-231).
    full = recv.permute(3, 2, 0, 1).reshape(bloc_size, nsl + nsl2, nb_procs * mc)
    xb = full[:, :nsl, :].contiguous().permute(2, 1, 0).contiguous().permute(2, 1, 0)
    yb = full[:, nsl:, :].contiguous().permute(2, 1, 0).contiguous().permute(2, 1, 0)
    lap(2)
    pb = compute(kind, xb, yb, m_max_pad)                                     # (bloc, nout, m_max)
    lap(1)
    if tensor_out:  # (3, bloc, 6, m_max) -> (bloc, 18, m_max), slot 3*s + k
        pb = pb.permute(1, 2, 0, 3).reshape(bloc_size, 18, nb_procs * mc)
    nout = pb.shape[1]
    # send back modes [q*mc, (q+1)*mc) of my points to rank q (:306)
    back = pb.reshape(bloc_size, nout, nb_procs, mc).permute(2, 3, 1, 0).contiguous()  # (P, mc, nout, bloc)
    got = torch.empty_like(back)
    lap(2)
    dist.all_to_all_single(got.view(-1), back.view(-1), group=group)
    lap(0)
    # got[q] = my modes for rank q's points -> (np_tot, nout, mc), drop dummies (:311-324)
    res = got.permute(0, 3, 2, 1).reshape(np_tot, nout, mc)[:npts]
    if tensor_out:
        res = res.reshape(npts, 6, 3, mc).permute(2, 0, 1, 3)
    out.copy_(res)
    lap(2)
    return out


def _gather_modes(group, x, nb_procs, bloc_size):
    """The first MPI_ALLTOALL of the reference (fft_parallel.F90:217, :93, :1482): this rank's m_max_c
    modes of all points -> all modes of its bloc_size points, (bloc_size, nslot, m_max) Fortran layout."""
    import torch
    import torch.distributed as dist

    npts, nsl, mc = x.shape
    np_tot = nb_procs * bloc_size
    tp = torch.zeros((np_tot, nsl, mc), dtype=x.dtype, device=x.device)
    tp[:npts] = x
    send = tp.reshape(nb_procs, bloc_size, nsl, mc).permute(0, 3, 2, 1).contiguous()  # (P, mc, nsl, bloc)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv.view(-1), send.view(-1), group=group)
    full = recv.permute(3, 2, 0, 1).reshape(bloc_size, nsl, nb_procs * mc)
    return full.contiguous().permute(2, 1, 0).contiguous().permute(2, 1, 0)


def _default_real(xb, N):
    from . import synthesis

    return synthesis(xb, n_theta=N)


def _default_max_vel(xb, m_max_pad):
    from . import max_vel

    return max_vel(xb, m_max_pad)


def fft_par_real_distributed(group, x, opt_nb_plane=None, compute=None):
    """FFT_PAR_REAL over a mode-distributed communicator: the rank's V_out (N, nslot/2, np/nb_procs)
    for its block of points (fft_parallel.F90:65-71: np must be a multiple of nb_procs).
    ``compute(xb, N)`` synthesises the gathered block; it defaults to the CUDA kernel."""
    import torch.distributed as dist

    nb_procs = dist.get_world_size(group)
    npts, nsl, mc = x.shape
    if npts % nb_procs:
        raise ValueError("Bug in FFT_PAR_REAL: np is not a multiple of nb_procs")
    m_max = mc * nb_procs
    m_max_pad = (opt_nb_plane + 1) // 2 if opt_nb_plane and opt_nb_plane > 2 * m_max - 1 else m_max
    xb = _gather_modes(group, x, nb_procs, npts // nb_procs)
    return (compute or _default_real)(xb, 2 * m_max_pad - 1)


def fft_max_vel_distributed(group, x, nb_procs, bloc_size, m_max_pad, compute=None):
    """FFT_MAX_VEL_DCL over a mode-distributed communicator: the gathered block's maximum, then the
    reference's MPI_ALLREDUCE(MAX) (fft_parallel.F90:1533-1535).  Dummy points are zero (:1478)."""
    import torch
    import torch.distributed as dist

    if dist.get_world_size(group) != nb_procs:
        raise ValueError("nb_procs must equal the communicator size")
    if x.shape[0] > nb_procs * bloc_size:
        raise ValueError("np > nb_procs*bloc_size")
    xb = _gather_modes(group, x, nb_procs, bloc_size)
    t = torch.tensor([float((compute or _default_max_vel)(xb, m_max_pad))], dtype=torch.float64, device=x.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def _default_gauss_operands(kind, V_in, mesh, list_mode, V2_in, omega, heat, conservative):
    from . import gauss_operands

    return gauss_operands(kind, V_in, mesh, list_mode, v2=V2_in, omega=omega, heat=heat, conservative=conservative)


def smb_gauss_distributed(kind, group, mesh, list_mode, V_in, nb_procs, V2_in=None, omega=None, heat=None,
                          conservative=False, temps=None, operands=None, compute=None):
    """The Gauss-point callers over the reference's mode-distributed communicator (comm_one_d(2)):
    smb_cross_prod_gauss_sft_par (kind GAUSS_NS, subroutine_ns_with_velocity.F90:512-629),
    smb_CurlH_cross_B_gauss_sft_par (GAUSS_LORENTZ, V_in = H, V2_in = B; subroutine_ns_with_m.F90:788-883)
    and smb_ugradc_gauss_fft_par (GAUSS_ADVECT, V_in = u, V2_in = c; subroutine_level_set.F90:434-534, and
    with ``conservative`` and ``heat`` subroutine_temperature_with_T.F90:247-350).

    Every rank holds its m_max_c modes of the nodal fields (``list_mode``: their mode numbers); the
    operands are built for those modes, and the product runs through :func:`fft_par_distributed` with the
    callers' bloc_size = l_G*me/nb_procs + 1 and m_max_pad = 3*m_max_c*nb_procs/2 (:625-626).  Returns
    this rank's modes of the result, (l_G*me, 6 | 2, m_max_c).  ``operands(kind, V_in, mesh, list_mode,
    V2_in, omega, heat, conservative)`` builds the Gauss-point arrays (default: the CUDA kernel, ``mesh``
    holding CUDA tensors as for :func:`sfemans_b200.cross_gauss`); ``compute`` is passed to
    :func:`fft_par_distributed`.
    """
    import torch

    from . import GAUSS_ADVECT, GAUSS_LORENTZ, GAUSS_NS

    if kind not in (GAUSS_NS, GAUSS_LORENTZ, GAUSS_ADVECT):
        raise ValueError("kind must be GAUSS_NS, GAUSS_LORENTZ or GAUSS_ADVECT")
    ops = (operands or _default_gauss_operands)(kind, V_in, mesh, list_mode, V2_in, omega, heat, conservative)
    ng, _, mc = ops[0].shape
    bloc = ng // nb_procs + 1
    pad = 3 * mc * nb_procs // 2
    empty = lambda nsl: torch.zeros((mc, nsl, ng), dtype=ops[0].dtype, device=ops[0].device).permute(2, 1, 0)  # noqa: E731
    if kind != GAUSS_ADVECT:
        return fft_par_distributed("cross", group, ops[0], ops[1], empty(6), nb_procs, bloc, pad, temps, compute)
    out = fft_par_distributed("dot", group, ops[0], ops[1], empty(2), nb_procs, bloc, pad, temps, compute)
    if conservative:  # + FFT_PAR_PROD_DCL(Div, Cgauss) (subroutine_temperature_with_T.F90:339-342)
        out += fft_par_distributed("prod", group, ops[2], ops[3], empty(2), nb_procs, bloc, pad, temps, compute)
    return out
