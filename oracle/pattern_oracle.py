"""Restatement of the reference's power pattern (To_Pattern_Powers with its
count-based Sparsify) in numpy.  TEST INFRASTRUCTURE: the checker of
mspai_pattern_powers, never part of the product.

The reference reaches this code only through PETSc (Pattern_Switch cases 3/4,
src/Pattern_Switch.cpp:60-95), which the serial driver cannot run, so the
restatement is pinned by hand-worked cases in tests/test_pattern_powers.py,
not against the reference's output ("parity unpinned").

  Matrix::Sparsify            src/Matrix.imp:471-620
  Matrix::To_Pattern_Powers   src/Matrix.imp:359-470
  kLargest (qsort by magnitude, larger first)   src/Matrix.imp:3038-3050
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def sparsify(S: sp.csc_matrix, lfill: np.ndarray) -> sp.csc_matrix:
    """Per column k (src/Matrix.imp:514-590): the entries by magnitude, larger
    first (equal magnitudes in row order: a stable sort of the row-ordered
    column); keep max(lfill_k, 1) of them (at most the column); when the
    diagonal is not kept it replaces the smallest kept entry (value: the
    diagonal's magnitude, 0 when absent); then every further entry equal in
    magnitude to the originally smallest kept one.  Values are magnitudes."""
    S = sp.csc_matrix(S)
    S.sort_indices()
    n = S.shape[1]
    rows_out, cols_out, vals_out = [], [], []
    for k in range(n):
        a, b = S.indptr[k], S.indptr[k + 1]
        rows = S.indices[a:b]
        vals = np.abs(S.data[a:b])
        L = b - a
        order = sorted(range(L), key=lambda i: (-vals[i], i))
        nk = min(L, max(int(lfill[k]), 1)) if L else 0
        keep = set(order[:nk])
        diag = [i for i in range(L) if rows[i] == k]
        diag_in = any(rows[i] == k for i in keep)
        insert_zero = False
        if not diag_in:
            if nk > 0:
                keep.discard(order[nk - 1])
            if diag:
                keep.add(diag[0])
            else:
                insert_zero = True
        if nk > 0:
            vcut = vals[order[nk - 1]]
            t = nk
            while t < L and vals[order[t]] == vcut:
                keep.add(order[t])
                t += 1
        for i in sorted(keep):
            rows_out.append(rows[i]); cols_out.append(k); vals_out.append(vals[i])
        if insert_zero:
            rows_out.append(k); cols_out.append(k); vals_out.append(0.0)
    M = sp.csc_matrix((np.array(vals_out, dtype=np.float64),
                       (np.array(rows_out, dtype=np.int64), np.array(cols_out, dtype=np.int64))),
                      shape=S.shape)
    M.sort_indices()
    return M


def power_pattern(A: sp.spmatrix, nb_pw: int) -> sp.csc_matrix:
    """To_Pattern_Powers (src/Matrix.imp:359-401): S = Sparsify(|A|); nb_pw
    times { Sparsify from the second time on; S = S S }; S = Sparsify(S).
    The products keep every structural entry (magnitudes do not cancel)."""
    A = sp.csc_matrix(A)
    A.sort_indices()
    lfill = np.diff(A.indptr)
    S = sparsify(abs(A), lfill)
    for k in range(nb_pw):
        if k >= 1:
            S = sparsify(S, lfill)
        # structural product: keep explicit zeros (0 * x terms) as PETSc does
        S1 = S.copy()
        S1.data = np.ones_like(S1.data)
        pat = sp.csc_matrix(S1 @ S1)
        val = sp.csc_matrix(S @ S)
        P = pat.tocoo()
        V = np.asarray(val[P.row, P.col]).ravel()
        S = sp.csc_matrix((V, (P.row, P.col)), shape=A.shape)
        S.sort_indices()
    return sparsify(S, lfill)
