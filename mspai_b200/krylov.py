"""Preconditioned GMRES on the GPU: the application phase around the setup.

The reference applies its preconditioner inside PETSc's KSP (src/main.cpp,
Apply_MSPAI = MatMult with M, src/imspai.cpp:47-53).  Here restarted GMRES(m)
runs in FP64 torch tensors on the device with right preconditioning: it
solves A M y = b by Arnoldi on A M (modified Gram-Schmidt, Givens rotations)
and returns x = M y.  M is applied by mspai_apply (Handle.apply); A by any
device matvec (a torch sparse CSR matrix in the helpers below).
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np
import scipy.sparse as sp
import torch

Matvec = Callable[[torch.Tensor], torch.Tensor]


def csr_matvec(A: sp.spmatrix, device="cuda") -> Matvec:
    """x -> A x with A as a torch sparse CSR matrix on the device."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    At = torch.sparse_csr_tensor(torch.from_numpy(A.indptr.astype(np.int64)),
                                 torch.from_numpy(A.indices.astype(np.int64)),
                                 torch.from_numpy(A.data.astype(np.float64)),
                                 size=A.shape, device=device, check_invariants=True)
    return lambda x: torch.mv(At, x)


def gmres(A: Matvec, b: torch.Tensor, M: Optional[Matvec] = None, tol: float = 1e-8,
          restart: int = 50, maxiter: int = 2000) -> Tuple[torch.Tensor, int, float]:
    """Solves A x = b to ||b - A x|| <= tol ||b||; returns (x, matvecs with A,
    final relative residual)."""
    Mv = M if M is not None else (lambda v: v)
    n = b.numel()
    dt, dev = b.dtype, b.device
    x = torch.zeros_like(b)
    bnorm = float(torch.linalg.vector_norm(b))
    if bnorm == 0.0:
        return x, 0, 0.0
    its = 0
    r = b - A(x)
    beta = float(torch.linalg.vector_norm(r))
    while its < maxiter and beta > tol * bnorm:
        m = min(restart, maxiter - its)
        V = torch.zeros((m + 1, n), dtype=dt, device=dev)
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        V[0] = r / beta
        k_used = 0
        for k in range(m):
            w = A(Mv(V[k]))
            its += 1
            for i in range(k + 1):
                H[i, k] = float(torch.dot(w, V[i]))
                w = w - H[i, k] * V[i]
            H[k + 1, k] = float(torch.linalg.vector_norm(w))
            if H[k + 1, k] > 0:
                V[k + 1] = w / H[k + 1, k]
            for i in range(k):  # previous rotations
                t = cs[i] * H[i, k] + sn[i] * H[i + 1, k]
                H[i + 1, k] = -sn[i] * H[i, k] + cs[i] * H[i + 1, k]
                H[i, k] = t
            d = np.hypot(H[k, k], H[k + 1, k])
            cs[k], sn[k] = (H[k, k] / d, H[k + 1, k] / d) if d > 0 else (1.0, 0.0)
            H[k, k] = d
            H[k + 1, k] = 0.0
            g[k + 1] = -sn[k] * g[k]
            g[k] = cs[k] * g[k]
            k_used = k + 1
            if abs(g[k + 1]) <= tol * bnorm:
                break
        y = np.linalg.solve(np.triu(H[:k_used, :k_used]), g[:k_used])
        upd = torch.from_numpy(y).to(dev) @ V[:k_used]
        x = x + Mv(upd)
        r = b - A(x)
        beta = float(torch.linalg.vector_norm(r))
    return x, its, beta / bnorm
