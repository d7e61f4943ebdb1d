"""torch.autograd wrapper of the setup's adjoint.

`probing_loss(a, rho, ...)` is L(A, rho) = ||C M - B||_F^2 for the MSPAI
probing form C = [A; rho E^T A], B = [I; rho Be] and M the fixed-pattern
setup of C (every column's least-squares solution, computed on the GPU).  Its
backward pass is the hand-written adjoint kernel (mspai_adjoint): the
gradient with respect to the nonzeros of C and B, chained here through the
two places A enters C (its own block and the probing rows E^T A) and through
rho.  The setup runs in FP64 in the forward pass, and the adjoint kernel
recomputes each column's R for lambda = R^-1 R^-T gbar (Q is never stored).

Stationarity of M makes the chain exact: dL/dC is the envelope term plus the
correction of the adjoint system, so no gradient flows through the pattern
(which is fixed) and none is lost through M.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import scipy.sparse as sp
import torch

from .api import Handle, Options


def _assemble(A: sp.csc_matrix, E: Optional[np.ndarray], Be: Optional[sp.spmatrix], rho: float):
    """C = [A; rho E^T A] with every probing entry stored (also zeros, so that
    each has a gradient), B = [I; rho Be]; returns C, B and the positions of
    A's entries in C's nonzero order."""
    n = A.shape[1]
    if E is None:
        return A.copy(), None, np.arange(A.nnz)
    p = E.shape[1]
    CeT = np.asarray(A.T @ E)                      # n x p: column j of C's probing rows
    lens = np.diff(A.indptr) + p
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    indices = np.empty(indptr[-1], dtype=np.int32)
    data = np.empty(indptr[-1], dtype=np.float64)
    a_pos = np.empty(A.nnz, dtype=np.int64)
    for j in range(n):
        a0, a1 = A.indptr[j], A.indptr[j + 1]
        c0 = indptr[j]
        k = a1 - a0
        indices[c0:c0 + k] = A.indices[a0:a1]
        data[c0:c0 + k] = A.data[a0:a1]
        a_pos[a0:a1] = np.arange(c0, c0 + k)
        indices[c0 + k:c0 + k + p] = n + np.arange(p)
        data[c0 + k:c0 + k + p] = rho * CeT[j]
    C = sp.csc_matrix((data, indices, indptr), shape=(n + p, n))
    Bp = sp.csc_matrix(Be, dtype=np.float64) * rho
    B = sp.vstack([sp.identity(n, format="csc"), Bp], format="csc")
    B.sort_indices()
    return C, B, a_pos


class ProbingLoss(torch.autograd.Function):
    """L(a, rho) with a = A's nonzeros (CSC order of `structure`)."""

    @staticmethod
    def forward(ctx, a, rho, structure, E, Be, P, handle):
        A = sp.csc_matrix((a.detach().cpu().numpy().astype(np.float64), structure.indices,
                           structure.indptr), shape=structure.shape)
        r = float(rho.detach().cpu())
        C, B, a_pos = _assemble(A, E, Be, r)
        probing = E is not None
        handle.setup(C, P, B=B, options=Options(ns=0, prec="fp64", probing=int(probing), rho=r))
        dC, dB, L = handle.adjoint(C, B)
        n = A.shape[1]
        da = dC[a_pos].copy()
        drho = 0.0
        if probing:
            # probing entries C(n + q, j) = rho * sum_i E(i, q) A(i, j)
            p = E.shape[1]
            rows = C.indices
            probe = rows >= n
            g = np.zeros((n, p))
            cols = np.repeat(np.arange(n), np.diff(C.indptr))
            g[cols[probe], rows[probe] - n] = dC[probe]            # dL/dC(n+q, j)
            # dL/dA(i, j) += rho * sum_q E(i, q) g(j, q)
            Ai = A.indices
            Aj = np.repeat(np.arange(n), np.diff(A.indptr))
            da += r * np.einsum("kq,kq->k", E[Ai], g[Aj])
            bprobe = B.indices >= n
            drho = (np.dot(dC[probe], C.data[probe]) + np.dot(dB[bprobe], B.data[bprobe])) / r
        ctx.save_for_backward(torch.as_tensor(da, dtype=a.dtype, device=a.device),
                              torch.as_tensor(drho, dtype=rho.dtype, device=rho.device))
        return torch.as_tensor(L, dtype=a.dtype, device=a.device)

    @staticmethod
    def backward(ctx, gout):
        da, drho = ctx.saved_tensors
        return gout * da, gout * drho, None, None, None, None, None


def probing_loss(a: torch.Tensor, rho: torch.Tensor, structure: sp.csc_matrix,
                 E: Optional[np.ndarray], Be: Optional[sp.spmatrix], P: sp.spmatrix,
                 handle: Optional[Handle] = None) -> torch.Tensor:
    """||C M - B||_F^2 as a differentiable function of A's nonzeros `a` and of
    the weight `rho` (E: n x p probing vectors, Be: p x n probing targets;
    E = None for plain SPAI, C = A, B = I)."""
    h = handle if handle is not None else Handle(0)
    return ProbingLoss.apply(a, rho, sp.csc_matrix(structure), E, Be, P, h)
