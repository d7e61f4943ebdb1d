"""The reference's power pattern with count-based sparsification
(mspai_pattern_powers; To_Pattern_Powers + Sparsify, src/Matrix.imp:359-620).

The reference reaches it only through PETSc, which the serial reference
driver cannot run: the numpy restatement (oracle/pattern_oracle.py) is pinned
by hand-worked cases here, and the GPU is checked against it: identical
patterns, values (magnitudes of the sparsified powers) within 1e-12."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import pattern_oracle as PO


def dense_cols(S):
    return {k: dict(zip(S.indices[S.indptr[k]:S.indptr[k + 1]], S.data[S.indptr[k]:S.indptr[k + 1]]))
            for k in range(S.shape[1])}


def test_sparsify_keeps_largest_and_the_diagonal():
    A = sp.csc_matrix(np.array([[1., 3., 0.], [0., 1., 0.], [0., 2., 1.]]))
    S = dense_cols(PO.sparsify(abs(A), np.array([1, 2, 1])))
    # column 1: 3 (row 0) and 2 (row 2) are the largest two; the diagonal
    # (1, row 1) takes the place of the smaller kept one
    assert S[1] == {0: 3.0, 1: 1.0}
    assert S[0] == {0: 1.0} and S[2] == {2: 1.0}


def test_sparsify_ties_and_missing_diagonal():
    # column 0: magnitudes 5 (row 1), 2, 2, 2 (rows 2, 3, 4), no diagonal entry
    A = sp.csc_matrix((np.array([5., -2., 2., -2.]), ([1, 2, 3, 4], [0, 0, 0, 0])), shape=(5, 5))
    S = dense_cols(PO.sparsify(A, np.array([3, 1, 1, 1, 1])))
    # kept: 5 and the first two 2s; no diagonal: the smallest kept (row 3)
    # gives way to a zero diagonal; the tie with the cut value (row 4) is kept
    assert S[0] == {0: 0.0, 1: 5.0, 2: 2.0, 4: 2.0}
    # empty columns get the zero diagonal
    assert S[3] == {3: 0.0}


def test_power_pattern_poisson_by_hand():
    # 1-D Laplacian 4 x 4 (2 on the diagonal, -1 off): |A|^2 has 5 / 4 / 1 patterns;
    # lfill = nnz of A's column (2 or 3): the column keeps its largest entries
    A = sp.diags([[-1.] * 3, [2.] * 4, [-1.] * 3], [-1, 0, 1], format="csc")
    S = dense_cols(PO.power_pattern(A, 1))
    # |A|^2 column 0: rows 0 (5), 1 (4), 2 (1); lfill 2 -> rows 0, 1
    assert S[0] == {0: 5.0, 1: 4.0}
    # column 1: rows 0 (4), 1 (6), 2 (4), 3 (1); lfill 3 -> 6, 4, 4
    assert S[1] == {0: 4.0, 1: 6.0, 2: 4.0}


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["poisson", "convdiff", "ragged", "nodiag"])
@pytest.mark.parametrize("nb_pw", [0, 1, 2])
def test_gpu_matches_restatement(case, nb_pw):
    import mspai_b200 as mb
    from mspai_b200 import workloads as W
    if case == "poisson":
        A = W.poisson2d(12).A
    elif case == "convdiff":
        A = W.convdiff3d(5).A
    elif case == "ragged":
        A = W.ragged_matrix(400, seed=3)
    else:
        rng = np.random.default_rng(4)
        A = sp.random(300, 300, density=0.02, format="csc", random_state=5)
        A.data = rng.standard_normal(A.nnz)
    A = sp.csc_matrix(A)
    A.sort_indices()
    got = mb.pattern_powers(A, nb_pw)
    ref = PO.power_pattern(A, nb_pw)
    got.sort_indices()
    assert np.array_equal(got.indptr, ref.indptr) and np.array_equal(got.indices, ref.indices)
    scale = np.maximum(np.abs(ref.data), 1e-300)
    assert np.all(np.abs(got.data - ref.data) <= 1e-12 * scale)
