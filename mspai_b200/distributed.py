"""The setup sharded over the GPUs of one node (one process per GPU).

Columns are independent (the reference distributes them over MPI ranks,
src/Distribution.cpp:48-71, and fetches remote columns on demand); here every
rank holds the whole C (and B, P) and solves a contiguous range of problem
columns, chosen so that the ranks get about equal work: the ranges split the
prefix sum of a per-column estimate of the QR flops instead of the column
count.  The only exchange is at the end: the ranks' pieces of M are gathered
(all_gather of the host pieces), and for the adjoint the per-rank gradients,
which are zero outside each rank's columns, are summed (all_reduce).

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
