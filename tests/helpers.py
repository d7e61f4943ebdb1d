"""Shared checks for the parity tests."""
import numpy as np
import scipy.sparse as sp


def same_pattern(A, B) -> bool:
    A = sp.csc_matrix(A); B = sp.csc_matrix(B)
    A.sort_indices(); B.sort_indices()
    return (A.shape == B.shape and np.array_equal(A.indptr, B.indptr)
            and np.array_equal(A.indices, B.indices))


COLUMN_FLOOR = 1e-3


def max_rel_diff(A, B, floor: float = COLUMN_FLOOR) -> float:
    """Largest per-entry relative difference of A from the reference B over the
    union of their patterns: |A_ij - B_ij| / max(|B_ij|, floor * max_i |B_ij|).

    Every entry is held to the tolerance relative to its own magnitude; only
    entries below `floor` times the largest entry of their column (where the
    least-squares error bound is normwise, not entrywise) are measured against
    that column floor instead.  A column of B that is entirely zero requires
    the same column of A to be exactly zero."""
    A = sp.csc_matrix(A)
    B = sp.csc_matrix(B)
    d = (A - B).tocoo()
    if d.nnz == 0:
        return 0.0
    Babs = abs(B).tocsc()
    colmax = np.asarray(Babs.max(axis=0).todense()).ravel()
    bval = np.asarray(Babs[d.row, d.col]).ravel()
    denom = np.maximum(bval, floor * colmax[d.col])
    diff = np.abs(d.data)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(denom > 0, diff / np.where(denom > 0, denom, 1.0),
                       np.where(diff > 0, np.inf, 0.0))
    return float(np.max(rel))


def column_residuals(C, M, B=None):
    """||C M(:,k) - B(:,k)||_2 per column (B = I when None)."""
    C = sp.csc_matrix(C); M = sp.csc_matrix(M)
    n = M.shape[1]
    if B is None:
        B = sp.vstack([sp.identity(n), sp.csc_matrix((C.shape[0] - n, n))]).tocsc()
    R = (C @ M - B).tocsc()
    return np.sqrt(np.asarray(R.multiply(R).sum(axis=0))).ravel()


def frob(C, M, B=None) -> float:
    return float(np.linalg.norm(column_residuals(C, M, B)))
