"""Edge cases of the setup on the GPU against the oracle: a 1 x 1 matrix, a
pattern column with no entries, a dense column of C (one large least-squares
problem among small ones), a single-entry pattern per column on a matrix
whose columns all have one entry, and columns with exactly the size limits
of the warp bucket (E = 64 entries, |J| = 16)."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import max_rel_diff, same_pattern
from mspai_b200 import workloads as W
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_one_by_one(h, prec):
    A = sp.csc_matrix(np.array([[2.0]]))
    h.setup(A, sp.identity(1, format="csc"), options=mb.Options(ns=0, prec=prec))
    M = h.result()
    assert M.shape == (1, 1) and M.nnz == 1 and abs(M.data[0] - 0.5) < 1e-14


def test_empty_pattern_column(h):
    A = W.poisson2d(8).A
    P = sp.lil_matrix(sp.csc_matrix(A != 0, dtype=float))
    P[:, 5] = 0
    P = sp.csc_matrix(P)
    P.eliminate_zeros()
    h.setup(A, P, options=mb.Options(ns=0, prec="fp64"))
    M = h.result()
    res, steps, status = h.column_info()
    assert M[:, 5].nnz == 0
    o = O.spai_scalar(A, P, ns=0)
    mask = np.ones(A.shape[1], dtype=bool)
    mask[5] = False
    assert max_rel_diff(M[:, mask], o.M[:, mask]) < 1e-10


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dense_column_among_sparse(h, prec):
    rng = np.random.default_rng(11)
    n = 1500
    A = sp.lil_matrix(sp.identity(n) * 4.0)
    A[:, 0] = rng.standard_normal((n, 1))
    A[0, 0] = 50.0
    for k in range(1, n):
        A[(k * 7) % n, k] += 0.3
    A = sp.csc_matrix(A)
    P = sp.csc_matrix(A != 0, dtype=float)
    h.setup(A, P, options=mb.Options(ns=0, prec=prec))
    M = h.result()
    o = O.spai_scalar(A, P, ns=0)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < (1e-10 if prec == "fp64" else 1e-8)


def test_diagonal_matrix_diagonal_pattern(h):
    d = np.linspace(1.0, 3.0, 257)
    A = sp.csc_matrix(sp.diags(d))
    h.setup(A, sp.identity(257, format="csc"), options=mb.Options(ns=0, prec="mixed"))
    M = h.result()
    assert np.allclose(M.diagonal(), 1.0 / d, rtol=1e-14)
    _, _, status = h.column_info()
    assert np.all(status == 0)


def test_warp_bucket_limits(h):
    """Columns with exactly 16 pattern entries and 64 entries of C(:,J): the
    largest problems of the warp bucket, next to ones just beyond it."""
    rng = np.random.default_rng(5)
    n = 400
    rows, cols, vals = [], [], []
    for j in range(n):
        k = 4 if j % 2 == 0 else 5  # 4 entries: 16 x 4 = 64; 5: 80 (CTA bucket)
        r = np.sort(rng.choice(np.delete(np.arange(n), j), size=k - 1, replace=False))
        rows += [j] + list(r); cols += [j] * k
        vals += [10.0] + list(rng.standard_normal(k - 1))
    A = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    P = sp.lil_matrix((n, n))
    for k in range(n):
        for q in range(16):
            P[(k + q * 2) % n, k] = 1.0
    P = sp.csc_matrix(P)
    for prec in ("fp64", "mixed"):
        h.setup(A, P, options=mb.Options(ns=0, prec=prec))
        M = h.result()
        st = h.stats()
        assert st["bucket_columns"][0] > 0 and sum(st["bucket_columns"]) == n
        o = O.spai_scalar(A, P, ns=0)
        assert same_pattern(M, o.M)
        assert max_rel_diff(M, o.M) < (1e-10 if prec == "fp64" else 1e-8)
