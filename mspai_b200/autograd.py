"""torch.autograd wrappers of the setup's adjoint.

`probing_loss(a, rho, ...)` is L(A, rho) = ||C M - B||_F^2 for the MSPAI
probing form C = [A; rho E^T A], B = [I; rho Be] and M the setup of C
(every column's least-squares solution, computed on the GPU: fixed or
adaptive patterns, scalar or block columns, FP64 or mixed precision).
`setup_values(a, rho, ...)` is M itself (its nonzeros, in M's order).  Their
backward passes are the hand-written adjoint kernel (mspai_adjoint_weighted):
the gradient with respect to the nonzeros of C and B, chained here through
the two places A enters C (its own block and the probing rows E^T A) and
through rho.

At the pattern the setup chose the chain is exact: M is stationary, so the
residual term needs no solve, and the sensitivity of M itself needs
lambda_k = (C_k^T C_k)^-1 gbar_k, which the kernel takes from the R factors
the setup kept (keep_factors, fixed scalar patterns) or recomputes in FP64.
The pattern itself is a discrete choice: no gradient flows through it.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import scipy.sparse as sp
import torch

from .api import Handle, Options


@dataclass
class Assembled:
    C: sp.csc_matrix          # [A; rho E^T A] with every probing entry stored
    B: Optional[sp.csc_matrix]  # [I; rho Be] (None: B = I)
    a_pos: np.ndarray         # position of each of A's nonzeros in C's order
    probe: np.ndarray         # C's probing entries (bool over C's nonzeros)
    ce: np.ndarray            # (E^T A) at those entries (unscaled)
    bprobe: np.ndarray        # B's probing entries (bool over B's nonzeros)
    be: np.ndarray            # Be at those entries (unscaled)


def _assemble(A: sp.csc_matrix, E: Optional[np.ndarray], Be: Optional[sp.spmatrix],
              rho: float) -> Assembled:
    """C = [A; rho E^T A] with every probing entry stored (zeros too, so that
    each has a gradient), B = [I; rho Be]; column j of C holds A(:, j) and
    then the p probing entries."""
    n = A.shape[1]
    if E is None:
        return Assembled(A.copy(), None, np.arange(A.nnz), np.zeros(A.nnz, bool),
                         np.zeros(0), np.zeros(0, bool), np.zeros(0))
    p = E.shape[1]
    CeT = np.asarray(A.T @ E)                        # n x p: column j's probing entries
    alen = np.diff(A.indptr)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(alen + p, out=indptr[1:])
    nnz = int(indptr[-1])
    acol = np.repeat(np.arange(n), alen)
    a_pos = indptr[acol] + (np.arange(A.nnz) - A.indptr[acol])
    probe = np.ones(nnz, dtype=bool)
    probe[a_pos] = False
    indices = np.empty(nnz, dtype=np.int32)
    data = np.empty(nnz, dtype=np.float64)
    indices[a_pos] = A.indices
    data[a_pos] = A.data
    indices[probe] = np.tile(n + np.arange(p, dtype=np.int32), n)
    ce = CeT.ravel()                                   # column-major over (q, j)
    data[probe] = rho * ce
    C = sp.csc_matrix((data, indices, indptr), shape=(n + p, n))
    Bp = sp.csc_matrix(Be, dtype=np.float64)
    B = sp.vstack([sp.identity(n, format="csc"), Bp * rho], format="csc")
    B.sort_indices()
    bprobe = B.indices >= n
    Bu = sp.vstack([sp.csc_matrix((n, n)), Bp], format="csc")
    Bu.sort_indices()
    # Be's values in B's order (B's probing entries are exactly Bu's nonzeros)
    be = np.zeros(B.nnz)
    be[bprobe] = Bu.data
    return Assembled(C, B, a_pos, probe, ce, bprobe, be[bprobe])


def _chain(asm: Assembled, A: sp.csc_matrix, E: Optional[np.ndarray], dC: np.ndarray,
           dB: Optional[np.ndarray], rho: float):
    """dL/da (A's nonzeros) and dL/drho from dL/dC and dL/dB."""
    da = dC[asm.a_pos].copy()
    drho = 0.0
    if E is not None:
        n = A.shape[1]
        p = E.shape[1]
        g = dC[asm.probe].reshape(n, p)                # dL/dC(n + q, j)
        # C(n + q, j) = rho sum_i E(i, q) A(i, j): dL/dA(i, j) += rho E(i, :) . g(j, :)
        acol = np.repeat(np.arange(n), np.diff(A.indptr))
        da += rho * np.einsum("kq,kq->k", E[A.indices], g[acol])
        drho = float(np.dot(dC[asm.probe], asm.ce))
        if dB is not None:
            drho += float(np.dot(dB[asm.bprobe], asm.be))
    return da, drho


def _setup(handle: Handle, asm: Assembled, P, E, rho: float, options: dict, keep: bool):
    o = dict(options)
    o.setdefault("ns", 0)
    o.setdefault("prec", "fp64")
    adaptive = o.get("ns", 0) > 0 and o.get("mn", 5) > 0
    # the reference's option check allows probing only without pattern
    # updates; with updates the probing rows are passed with probing = 0
    probing = int(E is not None and not adaptive)
    handle.setup(asm.C, P, B=asm.B,
                 options=Options(probing=probing, rho=rho, keep_factors=keep, **o))


class ProbingLoss(torch.autograd.Function):
    """L(a, rho) with a = A's nonzeros (CSC order of `structure`)."""

    @staticmethod
    def forward(ctx, a, rho, structure, E, Be, P, handle, options):
        A = sp.csc_matrix((a.detach().cpu().numpy().astype(np.float64), structure.indices,
                           structure.indptr), shape=structure.shape)
        r = float(rho.detach().cpu())
        asm = _assemble(A, E, Be, r)
        _setup(handle, asm, P, E, r, options, keep=False)
        dC, dB, L = handle.adjoint(asm.C, asm.B)
        da, drho = _chain(asm, A, E, dC, dB, r)
        ctx.save_for_backward(torch.as_tensor(da, dtype=a.dtype, device=a.device),
                              torch.as_tensor(drho, dtype=rho.dtype, device=rho.device))
        return torch.as_tensor(L, dtype=a.dtype, device=a.device)

    @staticmethod
    def backward(ctx, gout):
        da, drho = ctx.saved_tensors
        return gout * da, gout * drho, None, None, None, None, None, None


class SetupValues(torch.autograd.Function):
    """M's nonzeros (M's order) as a function of a = A's nonzeros and rho."""

    @staticmethod
    def forward(ctx, a, rho, structure, E, Be, P, handle, options):
        A = sp.csc_matrix((a.detach().cpu().numpy().astype(np.float64), structure.indices,
                           structure.indptr), shape=structure.shape)
        r = float(rho.detach().cpu())
        asm = _assemble(A, E, Be, r)
        keep = options.get("ns", 0) == 0 and options.get("bs", 1) == 1
        _setup(handle, asm, P, E, r, options, keep=keep)
        M = handle.result()
        ctx.state = (handle, asm, A, E, r, M.nnz)
        ctx.a_meta = (a.dtype, a.device, rho.dtype, rho.device)
        return torch.as_tensor(M.data.copy(), dtype=a.dtype, device=a.device)

    @staticmethod
    def backward(ctx, gm):
        handle, asm, A, E, r, nnz = ctx.state
        adt, adev, rdt, rdev = ctx.a_meta
        g = gm.detach().cpu().numpy().astype(np.float64)
        # the handle still holds this setup (and its R factors) unless it was
        # reused in between; the adjoint checks C against it
        dC, dB, _ = handle.adjoint(asm.C, asm.B, gbar=g, residual_weight=0.0)
        da, drho = _chain(asm, A, E, dC, dB, r)
        return (torch.as_tensor(da, dtype=adt, device=adev),
                torch.as_tensor(drho, dtype=rdt, device=rdev), None, None, None, None, None, None)


def probing_loss(a: torch.Tensor, rho: torch.Tensor, structure: sp.csc_matrix,
                 E: Optional[np.ndarray], Be: Optional[sp.spmatrix], P: sp.spmatrix,
                 handle: Optional[Handle] = None, **options) -> torch.Tensor:
    """||C M - B||_F^2 as a differentiable function of A's nonzeros `a` and of
    the weight `rho` (E: n x p probing vectors, Be: p x n probing targets;
    E = None for plain SPAI, C = A, B = I).  `options` go to the setup
    (Options fields: prec, ns, mn, ep, bs, ...; default a fixed-pattern FP64
    setup)."""
    h = handle if handle is not None else Handle(0)
    return ProbingLoss.apply(a, rho, sp.csc_matrix(structure), E, Be, P, h, options)


def setup_values(a: torch.Tensor, rho: torch.Tensor, structure: sp.csc_matrix,
                 E: Optional[np.ndarray], Be: Optional[sp.spmatrix], P: sp.spmatrix,
                 handle: Optional[Handle] = None, **options) -> torch.Tensor:
    """The setup's M (nonzeros in M's CSC order) as a differentiable function
    of A's nonzeros and rho; the backward pass is the adjoint with gbar = the
    incoming gradient and residual weight 0.  Fixed scalar patterns keep their
    R factors for it; the handle must not run another setup before backward."""
    h = handle if handle is not None else Handle(0)
    return SetupValues.apply(a, rho, sp.csc_matrix(structure), E, Be, P, h, options)
