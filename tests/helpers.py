"""Shared checks for the parity tests."""
import numpy as np
import scipy.sparse as sp


def same_pattern(A, B) -> bool:
    A = sp.csc_matrix(A); B = sp.csc_matrix(B)
    A.sort_indices(); B.sort_indices()
    return (A.shape == B.shape and np.array_equal(A.indptr, B.indptr)
            and np.array_equal(A.indices, B.indices))


def max_rel_diff(A, B) -> float:
    """max |A - B| / max |B| over the union of the patterns."""
    d = sp.csc_matrix(A) - sp.csc_matrix(B)
    scale = max(np.max(np.abs(sp.csc_matrix(B).data)), 1e-300)
    return float(np.max(np.abs(d.data)) / scale) if d.nnz else 0.0


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
