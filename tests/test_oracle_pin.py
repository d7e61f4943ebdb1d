"""The oracle (CPU restatement) against fixtures written by the reference itself.

The fixtures in tests/golden/ were produced by the reference sources compiled
here (tests/golden/make_golden.py); the reference prints 13 significant digits,
so values agree to that precision and patterns agree exactly.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden
from helpers import max_rel_diff, same_pattern, column_residuals
from mspai_b200 import workloads as W
from oracle import pyoracle as O

PRINT_TOL = 5e-12  # %.13e output of the reference


@pytest.mark.parametrize("nx", [16, 64])
def test_poisson_fixed_pattern(nx):
    w = W.poisson2d(nx)
    r = O.spai_scalar(w.A, w.P, ns=0)
    ref = load_golden(f"poisson2d_{nx}")
    assert same_pattern(r.M, ref)
    assert max_rel_diff(r.M, ref) < PRINT_TOL


@pytest.mark.parametrize("N,um,name", [(6, 1, "convdiff3d_6"), (10, 1, "convdiff3d_10"),
                                      (10, 0, "convdiff3d_10_um0")])
def test_convdiff_pattern_updates(N, um, name):
    w = W.convdiff3d(N)
    r = O.spai_scalar(w.A, w.P, ep=0.4, ns=5, mn=5, um=um)
    ref = load_golden(name)
    assert same_pattern(r.M, ref)
    assert max_rel_diff(r.M, ref) < PRINT_TOL


def test_probing_rows_in_C():
    """C = [A; rho Ce] with the reference's e_k right-hand side."""
    w = W.aniso2d_probing(16, kinds=("ones", "alt"), rho=10.0)
    C = O.stack_probing(w.A, w.Ce, 10.0)
    r = O.spai_scalar(C, w.P, ns=0)
    ref = load_golden("aniso16_probe")
    assert same_pattern(r.M, ref)
    assert max_rel_diff(r.M, ref) < PRINT_TOL


def test_ragged_fixed_pattern():
    w = W.ragged(3000)
    r = O.spai_scalar(w.A, w.P, ns=0)
    ref = load_golden("ragged_3000")
    assert same_pattern(r.M, ref)
    assert max_rel_diff(r.M, ref) < PRINT_TOL


def test_qr_update_reference_defect_documented():
    """-qr 2 must give the unrestrained result; the reference's QR-update path
    departs from it only on columns where its values are not least-squares
    solutions of its own pattern (a defect of the reference)."""
    w = W.convdiff3d(10)
    ref_qr = load_golden("convdiff3d_10_qr")
    ref_u = load_golden("convdiff3d_10")
    differ = np.where(np.diff(ref_qr.indptr) != np.diff(ref_u.indptr))[0]
    assert 0 < len(differ) < 20
    Pq = ref_qr.copy(); Pq.data[:] = 1.0
    ls = O.spai_scalar(w.A, Pq, ns=0).M
    for c in differ:
        # on every differing column the reference's QR-update values are not the
        # least-squares solution of its own pattern
        assert np.max(np.abs((ls[:, c] - ref_qr[:, c]).toarray())) > 1e-6
    same = np.setdiff1d(np.arange(w.n), differ)
    assert np.max(np.abs((ref_qr[:, same] - ref_u[:, same]).toarray())) < 1e-9


def test_oracle_b_aware_rhs_merges_target():
    """With B given, the right-hand side is B(I,k) (Create_bk_Hat merge)."""
    w = W.aniso2d_probing(8, kinds=("ones",), rho=10.0)
    C = O.stack_probing(w.A, w.Ce, 10.0)
    B = O.target(w.n, w.Be, 10.0)
    r = O.spai_scalar(C, w.P, B=B, ns=0)
    # dense check of a few columns with numpy least squares
    Cd = C.toarray(); Bd = B.toarray()
    for k in (0, 9, 63):
        J = w.P[:, k].indices
        I = np.nonzero(np.any(Cd[:, J] != 0, axis=1))[0]
        m, *_ = np.linalg.lstsq(Cd[np.ix_(I, J)], Bd[I, k], rcond=None)
        assert np.allclose(r.M[:, k].toarray().ravel()[J], m, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name,kind,kw", [
    ("block27_6", "A", dict(ns=0)),
    ("block27_6_upd", "diag", dict(ns=3, mn=3, ep=0.05)),
])
def test_block_spai(name, kind, kw):
    """Block SPAI (-bs 3) against the reference's block path."""
    w = W.block27(6, probing=False)
    Pb = O.block_pattern(w.A, 3) if kind == "A" else sp.identity(w.n // 3, format="csc")
    r = O.spai_block(w.A, Pb, 3, **kw)
    ref = load_golden(name)
    assert same_pattern(r.M, ref)
    assert max_rel_diff(r.M, ref) < PRINT_TOL
