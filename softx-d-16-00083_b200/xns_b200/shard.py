"""One structure over several GPUs (one process per GPU, torch.distributed for the plumbing).

Debye double sum (int_debye): each rank sums its tile pairs (xns_calc_int_debye_shard, the self term
on rank 0 only) and an all-reduce of the nq FP64 values gives every rank the whole I(q).

Histogram path:
Each rank counts its shard of the pair-distance histogram (xns_hist_shard_device: the tile pairs w of
the whole structure's plan with w mod N = rank), an all-reduce sums the shards (NCCL over NVLink / NVSwitch on GPUs, gloo on
CPU), and every rank derives the PDF and I(q) from the sum (xns_pdf_and_debye_from_hist_device).  The
counts are integers, so the sum is the one-GPU histogram bit for bit, as the reference's MPI_Reduce of
its per-rank rij_hist is (CalcFunctions.cpp:804-807).  The exchange is P x nhist u64 (1.2 MB for the
rock-salt cube) after tens of milliseconds of counting: one NCCL call, no fused kernel.
"""
import ctypes as C

import numpy as np

from . import XnsError, lib

_p = C.c_void_p
lib.xns_hist_shard_device.argtypes = [_p, _p, _p, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, _p]
lib.xns_calc_hist_shard.argtypes = [_p, C.POINTER(_p), _p, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32,
                                    _p]
lib.xns_calc_int_debye_shard.argtypes = [_p, C.POINTER(_p), _p, C.c_uint32, C.c_uint32, _p, _p, C.c_uint32, C.c_int,
                                         C.POINTER(_p), _p, C.c_int, C.c_double, C.c_uint32, C.c_uint32, _p]
lib.xns_pdf_and_debye_from_hist_device.argtypes = [_p, _p, _p, C.c_uint32, C.c_uint32, C.c_double, C.c_int, C.c_int,
                                                   C.c_double, _p, C.c_uint32, C.c_int, C.POINTER(_p), _p, C.c_int,
                                                   C.c_double, _p, _p]


def _check(ctx, st):
    if st:
        raise XnsError(st, lib.xns_last_error(ctx.handle).decode())


def reduce_histogram(hist, group=None):
    """Sum an int64 histogram tensor over the ranks of the process group, in place."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(hist, op=dist.ReduceOp.SUM, group=group)
    return hist


def hist_shard(ctx, elements, nhist, bin, shard, nshard):
    """This shard's histogram of host coordinates (per-element (n, 3) arrays): P*nhist uint64."""
    arrs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for e in elements]
    n_el = np.array([len(a) for a in arrs], dtype=np.uint32)
    table = (_p * len(arrs))(*[a.ctypes.data_as(_p) if len(a) else None for a in arrs])
    out = np.zeros(len(arrs) * (len(arrs) + 1) // 2 * nhist, dtype=np.uint64)
    _check(ctx, lib.xns_calc_hist_shard(ctx.handle, table, n_el.ctypes.data_as(_p), len(arrs), nhist, bin, shard, nshard,
                                        out.ctypes.data_as(_p)))
    return out


def pdf_and_debye(ctx, xyz_dev, n_el, nhist, bin, scenario, pdftype, p0, q, source, sl, hist_dev, I_dev, pdf_dev,
                  rank=0, world=1, group=None, ff=None, polar=False, lam=0.0):
    """calcPDFandDebye for one structure split over the ranks of group: xyz_dev (element-major x y z
    doubles), hist_dev (P*nhist int64), I_dev (nq doubles) and pdf_dev ((1+P)*nhist doubles) are torch
    tensors on this rank's GPU; every rank ends with the whole histogram, I(q) and PDF."""
    n_el = np.ascontiguousarray(n_el, dtype=np.uint32)
    nel = len(n_el)
    q = np.ascontiguousarray(q, dtype=np.float64)
    sl = None if sl is None else np.ascontiguousarray(sl, dtype=np.float64)
    ffp = None
    if ff is not None:
        rows = [np.ascontiguousarray(r, dtype=np.float64) for r in ff]
        ffp = (_p * nel)(*[r.ctypes.data_as(_p) for r in rows])
    _check(ctx, lib.xns_hist_shard_device(ctx.handle, _p(xyz_dev.data_ptr()), n_el.ctypes.data_as(_p), nel, nhist, bin,
                                          rank, world, _p(hist_dev.data_ptr())))
    if world > 1:
        reduce_histogram(hist_dev, group)
        if hist_dev.device.type == "cuda":  # the library's stream may differ from torch's: let the sum land
            import torch
            torch.cuda.current_stream(hist_dev.device).synchronize()
    _check(ctx, lib.xns_pdf_and_debye_from_hist_device(
        ctx.handle, _p(hist_dev.data_ptr()), n_el.ctypes.data_as(_p), nel, nhist, bin, scenario, pdftype, p0,
        q.ctypes.data_as(_p), len(q), source, ffp, None if sl is None else sl.ctypes.data_as(_p), int(polar), lam,
        _p(I_dev.data_ptr()) if I_dev is not None else None, _p(pdf_dev.data_ptr()) if pdf_dev is not None else None))


def int_debye_shard(ctx, elements, q, source, sl=None, ff=None, polar=False, lam=0.0, shard=0, nshard=1,
                    n_el_block=None):
    """This shard's share of calcIntDebye (or of calcIntPartialDebye with n_el_block, element-major
    e * nblocks + b): nq doubles (or (1 + parts) x nq)."""
    arrs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 3) for e in elements]
    nel = len(arrs)
    n_el = np.array([len(a) for a in arrs], dtype=np.uint32)
    table = (_p * nel)(*[a.ctypes.data_as(_p) if len(a) else None for a in arrs])
    q = np.ascontiguousarray(q, dtype=np.float64)
    nb = 1 if n_el_block is None else len(n_el_block) // nel
    neb = None if n_el_block is None else np.ascontiguousarray(n_el_block, dtype=np.uint32)
    parts = nb * (nb + 1) // 2
    out = np.zeros((1 + parts if nb > 1 else 1) * len(q))
    slp = None if sl is None else np.ascontiguousarray(sl, dtype=np.float64)
    ffp, rows = None, None
    if ff is not None:
        rows = [np.ascontiguousarray(r, dtype=np.float64) for r in ff]
        ffp = (_p * nel)(*[r.ctypes.data_as(_p) for r in rows])
    _check(ctx, lib.xns_calc_int_debye_shard(ctx.handle, table, n_el.ctypes.data_as(_p), nel, nb,
                                             None if neb is None else neb.ctypes.data_as(_p), q.ctypes.data_as(_p),
                                             len(q), source, ffp, None if slp is None else slp.ctypes.data_as(_p),
                                             int(polar), lam, shard, nshard, out.ctypes.data_as(_p)))
    return out


def int_debye(ctx, elements, q, source, sl=None, ff=None, polar=False, lam=0.0, rank=0, world=1, group=None,
              n_el_block=None):
    """calcIntDebye for one structure split over the ranks of group; every rank returns the whole I(q)."""
    part = int_debye_shard(ctx, elements, q, source, sl, ff, polar, lam, rank, world, n_el_block)
    if world == 1:
        return part
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(part).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def q_rows(nq, rank, world):
    """The q rows [lo, hi) of rank in a balanced split of nq rows."""
    return nq * rank // world, nq * (rank + 1) // world


def int_2d(ctx, elements, q, nfi, euler_min, euler_max, euler_n, convention, lam, source, ff=None, sl=None,
           polar=False, rank=0, world=1, group=None):
    """calcInt2D (CalcFunctions.cpp:969-1091) for one structure split over the ranks by q rows (each row
    of the reference's polar mesh is independent of the others, as its OpenMP loop over q,
    :1023-1046, uses): every rank evaluates its rows and an all-gather assembles (I2D, I) on every
    rank."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    lo, hi = q_rows(len(q), rank, world)
    ffr = None if ff is None else [np.asarray(r)[lo:hi] for r in ff]
    I2D, I = (ctx.calc_int_2d(elements, q[lo:hi], nfi, euler_min, euler_max, euler_n, convention, lam, source, ff=ffr,
                              sl=sl, polar=polar) if hi > lo else (np.zeros((0, nfi)), np.zeros(0)))
    if world == 1:
        return I2D, I
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    rows = max(q_rows(len(q), r, world)[1] - q_rows(len(q), r, world)[0] for r in range(world))
    mine = torch.zeros((rows, nfi + 1), dtype=torch.float64, device=dev)  # padded to the largest share
    mine[:hi - lo, :nfi] = torch.from_numpy(I2D)
    mine[:hi - lo, nfi] = torch.from_numpy(I)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    full = torch.cat([parts[r][:q_rows(len(q), r, world)[1] - q_rows(len(q), r, world)[0]] for r in range(world)])
    full = full.cpu().numpy()
    return np.ascontiguousarray(full[:, :nfi]), np.ascontiguousarray(full[:, nfi])
