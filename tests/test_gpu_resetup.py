"""Re-setups from the kept factors (reuse_factors): a setup with new values
of C on the structure of the previous keep_factors setup starts every column
of the fixed-pattern solver from its previous solution and R and refines in
FP64 against the new values; the columns that do not converge are factored
again.  The result equals a fresh setup of the new values: 1e-10 relative per
entry in FP64, 1e-8 in mixed mode (helpers.max_rel_diff).  A changed
structure or a setup that kept no factors makes the re-setup a full setup."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import max_rel_diff
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


@pytest.fixture(scope="module")
def case():
    A = W.ragged_matrix(20000, seed=31)
    P = mb.pattern_power2(A, 1e-3)
    return A, P


def perturbed(A, rel, seed):
    B = sp.csc_matrix(A, copy=True)
    B.data = B.data * (1.0 + rel * np.random.default_rng(seed).standard_normal(B.nnz))
    return B


def fresh(h, A, P, prec):
    h.setup(A, P, options=mb.Options(ns=0, prec=prec))
    return h.result()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_resetup_equals_fresh_setup(h, case, prec):
    A, P = case
    keep = mb.Options(ns=0, prec=prec, keep_factors=True)
    again = mb.Options(ns=0, prec=prec, keep_factors=True, reuse_factors=8)
    h.setup(A, P, options=keep)
    buckets = h.stats()["bucket_columns"]
    fixed_cols = sum(buckets[1:3])  # the fixed-pattern solver's two launches
    assert fixed_cols > 0.3 * A.shape[1], buckets
    prev = A
    for step, rel in enumerate((1e-4, 1e-3, 1e-4)):
        A2 = perturbed(prev, rel, seed=100 + step)
        h.setup(A2, P, options=again)
        M2 = h.result()
        res2, _, status2 = h.column_info()
        reused = h.stats()["factor_reuse_columns"]
        assert np.all(status2 == 0)
        ref = fresh(h, A2, P, prec)
        res_ref, _, _ = h.column_info()
        assert max_rel_diff(M2, ref) < TOL[prec], (step, rel)
        assert np.allclose(res2, res_ref, rtol=1e-8, atol=1e-14)
        # small changes: nearly every column of the fixed-pattern solver
        # converges from its kept factor
        assert reused >= 0.9 * fixed_cols, (step, reused, fixed_cols)
        # the fresh setup above kept no factors: set them again
        h.setup(A2, P, options=keep)
        prev = A2


def test_large_change_refactors(h, case):
    A, P = case
    h.setup(A, P, options=mb.Options(ns=0, prec="mixed", keep_factors=True))
    A2 = sp.csc_matrix(A, copy=True)
    A2.data = np.random.default_rng(9).standard_normal(A2.nnz)
    A2 = A2 + sp.diags(3.0 * np.asarray(abs(A2).sum(axis=0)).ravel())
    A2 = sp.csc_matrix(A2)
    A2.sort_indices()
    assert A2.nnz == A.nnz and np.array_equal(A2.indices, sp.csc_matrix(A).indices)
    h.setup(A2, P, options=mb.Options(ns=0, prec="mixed", keep_factors=True, reuse_factors=8))
    M2 = h.result()
    reused = h.stats()["factor_reuse_columns"]
    ref = fresh(h, A2, P, "mixed")
    assert max_rel_diff(M2, ref) < TOL["mixed"]
    assert reused < 0.5 * A.shape[1]  # new values: most columns factored again


def test_structure_change_is_a_full_setup(h, case):
    A, P = case
    h.setup(A, P, options=mb.Options(ns=0, prec="mixed", keep_factors=True))
    P2 = sp.csc_matrix(A != 0, dtype=np.float64)  # another pattern
    again = mb.Options(ns=0, prec="mixed", keep_factors=True, reuse_factors=8)
    h.setup(A, P2, options=again)
    assert h.stats()["factor_reuse_columns"] == 0
    M2 = h.result()
    assert max_rel_diff(M2, fresh(h, A, P2, "mixed")) < TOL["mixed"]
    # without kept factors (the fresh setup kept none) nothing is reused either
    h.setup(A, P2, options=again)
    assert h.stats()["factor_reuse_columns"] == 0
