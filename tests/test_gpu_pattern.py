"""Start pattern from A^2 on the GPU (mspai_pattern_power2) against the
seeded workloads' scipy definition: per column the rows of A^2 whose
magnitude reaches drop times the column's largest, the ragged benchmark
pattern.  Patterns are compared exactly (random values: no entry lies on the
threshold)."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import same_pattern
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,drop", [(3000, 1e-3), (20000, 1e-3), (3000, 0.0), (3000, 0.05)])
def test_ragged_square_pattern(n, drop):
    A = W.ragged_matrix(n)
    P = mb.pattern_power2(A, drop)
    ref = W.square_pattern_dropped(A, drop)
    assert same_pattern(P, ref)


def test_probing_rows_are_not_part_of_a():
    w = W.aniso2d_probing(16, kinds=("ones",), rho=10.0)
    C, _ = mb.assemble_probing(w.A, w.Ce, w.Be, 10.0)
    P = mb.pattern_power2(C, 0.0)
    ref = W.square_pattern_dropped(w.A, 0.0)
    assert P.shape == w.A.shape and same_pattern(P, ref)


def test_capacity_error():
    n = 200
    A = sp.csc_matrix(np.ones((n, n)))  # each column of A^2 gathers n^2 products
    with pytest.raises(mb.MspaiError, match="products"):
        mb.pattern_power2(A, 0.0)
