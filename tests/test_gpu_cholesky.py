"""The mixed mode's Cholesky of C^T C in the fixed-pattern solver
(fixed_solve.cuh, fix_cholesky: blocks of 16 columns, warp 0 factoring the
next diagonal block while the other warps finish the trailing update) at the
block boundaries, and its fallback to the Householder QR.

Every column of these patterns has |J_k| on or next to a multiple of 16 (the
last block full, one column into a new block, a single block) so that each
branch of the look-ahead runs; the values must match the oracle as every
fixed-pattern column does: identical patterns, 1e-8 per entry in mixed mode,
1e-10 in FP64 (helpers.max_rel_diff).  The fallback case puts two nearly
parallel columns of C into J_k: C^T C is then not numerically positive
definite in FP32 (kappa(C(I, J))^2 u_32 > 1), so the column leaves the
Cholesky (a pivot <= 0 or a refinement that does not contract) and the
Householder QR in FP32 with the FP64 refinement solves it to the same
tolerance."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import max_rel_diff, same_pattern
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}
SIZES = (16, 17, 31, 32, 33, 47, 48, 49, 64, 65)


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def random_matrix(n, per_col, seed):
    """n x n, per_col random off-diagonal entries a column, diagonally dominant."""
    rng = np.random.default_rng(seed)
    rows = np.concatenate([rng.choice(n, per_col, replace=False) for _ in range(n)])
    cols = np.repeat(np.arange(n), per_col)
    vals = rng.standard_normal(rows.size)
    A = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    A = A + sp.diags(2.0 * per_col + rng.random(n))
    A = sp.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return A


def boundary_pattern(n, seed, pairs=None):
    """Column k: k and |J_k| - 1 random other columns, |J_k| from SIZES in turn;
    pairs (a, b) are put together into the columns listed with them."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for k in range(n):
        s = SIZES[k % len(SIZES)]
        J = {k}
        if pairs is not None and k in pairs:
            J |= set(pairs[k])
        while len(J) < s:
            J.add(int(rng.integers(n)))
        rows.extend(sorted(J))
        cols.extend([k] * len(J))
    P = sp.csc_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    P.sort_indices()
    return P


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_block_boundaries_against_oracle(h, prec):
    A = random_matrix(400, 8, seed=5)
    P = boundary_pattern(400, seed=6)
    h.setup(A, P, options=mb.Options(ns=0, prec=prec))
    M = h.result()
    _, _, status = h.column_info()
    buckets = h.stats()["bucket_columns"]
    assert buckets[1] + buckets[2] > 0.9 * A.shape[1], buckets  # the fixed-pattern solver
    assert np.all(status == 0)
    o = O.spai_scalar(A, P, ns=0)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < TOL[prec]


def test_cholesky_fallback_on_nearly_parallel_columns(h):
    n = 400
    A = sp.lil_matrix(random_matrix(n, 8, seed=11))
    # column 1 = column 0 with one entry scaled by 1 + 1e-3: C^T C is
    # indefinite to FP32 for every J holding both (kappa ~ 1e4), while the
    # Householder R in FP32 still contracts the refinement (kappa u_32 ~ 1e-3)
    c0 = A[:, 0].toarray().ravel()
    nz = np.flatnonzero(c0)
    c1 = c0.copy()
    c1[nz[0]] *= 1.0 + 1e-3
    A[:, 1] = c1.reshape(-1, 1)
    A = sp.csc_matrix(A)
    A.sort_indices()
    hit = {k: (0, 1) for k in range(2, n, 9)}
    P = boundary_pattern(n, seed=12, pairs=hit)
    # the chosen columns do need the fallback: kappa^2 u_32 > 1
    k = 2
    J = P.indices[P.indptr[k]:P.indptr[k + 1]]
    I = np.unique(A[:, J].nonzero()[0])
    sv = np.linalg.svd(A[I][:, J].toarray(), compute_uv=False)
    assert (sv[0] / sv[-1]) ** 2 * 2.0 ** -24 > 1.0
    h.setup(A, P, options=mb.Options(ns=0, prec="mixed"))
    M = h.result()
    _, _, status = h.column_info()
    assert np.all(status == 0)
    o = O.spai_scalar(A, P, ns=0)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < TOL["mixed"]
