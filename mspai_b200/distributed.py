"""The setup sharded over the GPUs of one node (one process per GPU).

Columns are independent (the reference distributes them over MPI ranks,
src/Distribution.cpp:48-71, and fetches remote columns on demand); here every
rank holds the whole C (and B, P) and solves a contiguous range of problem
columns, chosen so that the ranks get about equal work: the ranges split the
prefix sum of a per-column estimate of the QR flops instead of the column
count.  The only exchange is at the end: the ranks' pieces of M are gathered,
and for the adjoint the per-rank gradients, which are zero outside each
rank's columns, are summed (all_reduce).

Two forms:
  * host matrices (scipy): sharded_setup / sharded_adjoint, M's pieces
    all-gathered as host objects;
  * device matrices (DeviceCSC in HBM): sharded_setup_device /
    sharded_adjoint_device.  The ranges are computed on the device, M stays in
    HBM and its pieces cross NVLink through NCCL: the column lengths by one
    all_reduce (zero outside each rank's range), the row indices and values
    by all_gather_into_tensor of segments padded to the longest (for a fixed
    scalar pattern M has P's structure, so only the values cross).

    import torch.distributed as dist
    dist.init_process_group("nccl")            # or "gloo" on CPU
    M = sharded_setup(handle, C, P, options=Options(ns=0))
    dC, dB, loss = sharded_adjoint(handle, C, B)
"""
from __future__ import annotations

from dataclasses import replace
from typing import List, Optional, Sequence, Tuple

import numpy as np
import scipy.sparse as sp

from .api import Handle, Options

Piece = Tuple[int, int, np.ndarray, np.ndarray, np.ndarray]  # lo, hi, colptr, rowidx, values


def column_work(C: sp.spmatrix, P: sp.spmatrix) -> np.ndarray:
    """Estimate of the work of each column's least-squares problem: with
    E_k entries of C(:, J_k) and n_k = |J_k|, the folded QR costs about
    2 (E_k / 2 + n_k) n_k^2 flops, plus the gather of the E_k entries."""
    C = sp.csc_matrix(C)
    P = sp.csc_matrix(P)
    colnnz = np.diff(C.indptr).astype(np.float64)
    nk = np.diff(P.indptr).astype(np.float64)
    per_entry = colnnz[P.indices] if P.nnz else np.zeros(0)
    Ek = np.zeros(P.shape[1])
    nonempty = nk > 0
    if P.nnz:
        Ek[nonempty] = np.add.reduceat(per_entry, P.indptr[:-1][nonempty])
    return 2.0 * (Ek / 2.0 + nk) * nk * nk + Ek


def balanced_ranges(work: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous column ranges, one per rank, splitting the prefix sum of
    `work` into `world` near-equal parts (every column in exactly one range)."""
    w = np.asarray(work, dtype=np.float64)
    n = len(w)
    pre = np.concatenate([[0.0], np.cumsum(w)])
    total = pre[-1]
    cuts = [0]
    for r in range(1, world):
        c = int(np.searchsorted(pre, total * r / world, side="left"))
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def local_piece(M: sp.csc_matrix, lo: int, hi: int) -> Piece:
    """Columns [lo, hi) of M as a piece (local column pointers from 0)."""
    M = sp.csc_matrix(M)
    a, b = M.indptr[lo], M.indptr[hi]
    return (lo, hi, (M.indptr[lo:hi + 1] - a).astype(np.int64),
            M.indices[a:b].astype(np.int32), M.data[a:b].astype(np.float64))


def assemble(pieces: Sequence[Piece], n: int) -> sp.csc_matrix:
    """The n x n CSC matrix made of the ranks' column pieces."""
    lens = np.zeros(n, dtype=np.int64)
    for lo, hi, cp, _, _ in pieces:
        lens[lo:hi] = np.diff(cp)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    indices = np.empty(indptr[-1], dtype=np.int32)
    data = np.empty(indptr[-1], dtype=np.float64)
    for lo, hi, cp, ri, vv in pieces:
        indices[indptr[lo]:indptr[hi]] = ri
        data[indptr[lo]:indptr[hi]] = vv
    return sp.csc_matrix((data, indices, indptr), shape=(n, n))


def gather_pieces(piece: Piece, n: int, group=None) -> sp.csc_matrix:
    """All-gathers every rank's piece and assembles M on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    pieces: List[Optional[Piece]] = [None] * world
    dist.all_gather_object(pieces, piece, group=group)
    return assemble(pieces, n)


def shard_range(C: sp.spmatrix, P: sp.spmatrix, rank: int, world: int) -> Tuple[int, int]:
    return balanced_ranges(column_work(C, P), world)[rank]


def sharded_setup(handle: Handle, C: sp.spmatrix, P: sp.spmatrix,
                  B: Optional[sp.spmatrix] = None, options: Optional[Options] = None,
                  group=None) -> sp.csc_matrix:
    """Each rank solves its balanced range of columns on its GPU; M is
    gathered on every rank.  Scalar setups (bs = 1)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = sp.csc_matrix(P).shape[1]
    lo, hi = shard_range(C, P, rank, world)
    # an empty range is written (n, n): (0, 0) would mean every column
    opts = replace(options or Options(), col_begin=lo if hi > lo else n,
                   col_end=hi if hi > lo else n)
    handle.setup(C, P, B=B, options=opts)
    piece = local_piece(handle.result(), lo, hi)
    return gather_pieces(piece, n, group)


def sharded_adjoint(handle: Handle, C: sp.spmatrix, B: Optional[sp.spmatrix] = None,
                    group=None):
    """Gradient of ||C M - B||_F^2 after sharded_setup: each rank's adjoint
    covers its own columns; the gradients and the loss are summed."""
    import torch
    import torch.distributed as dist
    dC, dB, loss = handle.adjoint(C, B)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.concatenate([dC, dB if dB is not None else np.zeros(0), [loss]]))
    t = t.to(dev)
    dist.all_reduce(t, group=group)
    t = t.cpu().numpy()
    nc = len(dC)
    nb = len(dB) if dB is not None else 0
    return t[:nc], (t[nc:nc + nb] if dB is not None else None), float(t[-1])


# ------------------------------------------------------------------ device form
def column_work_device(cptr, pptr, pidx):
    """column_work on the device: int64 CSC pointers of C and P, int32 rows
    of P (torch tensors); float64 work per problem column."""
    import torch
    colnnz = (cptr[1:] - cptr[:-1]).to(torch.float64)
    nk = (pptr[1:] - pptr[:-1]).to(torch.float64)
    per = colnnz[pidx.long()]
    cs = torch.zeros(per.numel() + 1, dtype=torch.float64, device=per.device)
    torch.cumsum(per, 0, out=cs[1:])
    Ek = cs[pptr[1:]] - cs[pptr[:-1]]
    return 2.0 * (Ek / 2.0 + nk) * nk * nk + Ek


def balanced_ranges_device(work, world: int) -> List[Tuple[int, int]]:
    """balanced_ranges on a device tensor of work (one small copy back)."""
    import torch
    n = work.numel()
    pre = torch.zeros(n + 1, dtype=torch.float64, device=work.device)
    torch.cumsum(work, 0, out=pre[1:])
    total = pre[-1]
    targets = total * torch.arange(1, world, dtype=torch.float64, device=work.device) / world
    cuts = torch.searchsorted(pre, targets, right=False).cpu().tolist() if world > 1 else []
    out, last = [0], 0
    for c in cuts:
        last = min(max(int(c), last), n)
        out.append(last)
    out.append(n)
    return [(out[r], out[r + 1]) for r in range(world)]


def gather_csc_device(colptr, rowidx, values, ranges: Sequence[Tuple[int, int]], rank: int,
                      group=None, known_structure=None):
    """Assembles M on every rank from the ranks' column ranges.

    colptr (int64, n + 1), rowidx (int32), values (float64): this rank's
    result, whose columns outside ranges[rank] are empty (or, with
    known_structure, the full structure shared by every rank: only the values
    of each range are exchanged).  Collectives: one all_reduce of the n column
    lengths (skipped with known_structure) and one all_gather_into_tensor each
    for the row indices and the values, of segments padded to the longest.
    Returns (colptr, rowidx, values) on the same device."""
    import torch
    import torch.distributed as dist
    world = len(ranges)
    dev = values.device
    if known_structure is not None:
        cp, ri = known_structure
    else:
        lens = colptr[1:] - colptr[:-1]
        dist.all_reduce(lens, group=group)
        cp = torch.zeros_like(colptr)
        torch.cumsum(lens, 0, out=cp[1:])
        ri = None
    bounds = torch.tensor([[cp[lo].item() if lo < len(cp) else 0, cp[hi].item()]
                           for lo, hi in ranges], dtype=torch.int64).tolist()
    segs = [b - a for a, b in bounds]
    seg_max = max(max(segs), 1)
    lo_r, hi_r = ranges[rank]
    a_loc, b_loc = int(colptr[lo_r]), int(colptr[hi_r])

    def gather(local, dtype):
        buf = torch.zeros(seg_max, dtype=dtype, device=dev)
        buf[:b_loc - a_loc] = local[a_loc:b_loc]
        allb = torch.empty(world * seg_max, dtype=dtype, device=dev)
        dist.all_gather_into_tensor(allb, buf, group=group)
        out = torch.empty(int(cp[-1]), dtype=dtype, device=dev)
        for r, (a, b) in enumerate(bounds):
            out[a:b] = allb[r * seg_max:r * seg_max + (b - a)]
        return out

    vals = gather(values, torch.float64)
    if ri is None:
        ri = gather(rowidx, torch.int32)
    return cp, ri, vals


def sharded_setup_device(handle: Handle, C, P, B=None, options: Optional[Options] = None,
                         group=None, ranges: Optional[Sequence[Tuple[int, int]]] = None):
    """sharded_setup with C, P (and B) as DeviceCSC on this rank's GPU: each
    rank solves its balanced range; M is assembled in HBM on every rank
    through NCCL.  Returns a DeviceCSC of M.  Scalar setups (bs = 1)."""
    import torch
    import torch.distributed as dist
    from .api import DeviceCSC
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = P.ncols
    if ranges is None:
        ranges = balanced_ranges_device(column_work_device(C.colptr, P.colptr, P.rowidx), world)
    lo, hi = ranges[rank]
    opts = replace(options or Options(), col_begin=lo if hi > lo else n,
                   col_end=hi if hi > lo else n)
    handle.setup(C, P, B=B, options=opts)
    nnz = handle.nnz()
    dev = P.colptr.device
    vv = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
    fixed = opts.ns == 0 or opts.mn == 0
    if fixed and opts.bs == 1:
        # M has P's structure (zeros outside the range): only the values of
        # each range cross, at P's offsets
        handle.result_into(None, None, vv, device=True)
        cp, ri, known = P.colptr, None, (P.colptr, P.rowidx)
    else:
        cp = torch.empty(n + 1, dtype=torch.int64, device=dev)
        ri = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        handle.result_into(cp, ri, vv, device=True)
        known = None
    mc, mr, mv = gather_csc_device(cp, ri, vv, ranges, rank, group, known_structure=known)
    return DeviceCSC(n, n, mc, mr, mv)


def sharded_adjoint_device(handle: Handle, C, dC, B=None, dB=None, group=None) -> float:
    """sharded_adjoint with device tensors: each rank's adjoint covers its own
    columns (dC, dB float64 CUDA tensors of C's / B's nonzeros); the
    gradients and the loss are summed by one NCCL all_reduce each."""
    import torch
    import torch.distributed as dist
    loss = handle.adjoint_device(C, dC, B, dB)
    dist.all_reduce(dC, group=group)
    if dB is not None:
        dist.all_reduce(dB, group=group)
    t = torch.tensor([loss], dtype=torch.float64, device=dC.device)
    dist.all_reduce(t, group=group)
    return float(t.item())
