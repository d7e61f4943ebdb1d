"""Adjoint of the fixed-pattern setup against central finite differences
(step 1e-6 relative to the parameter, agreement 1e-6 relative), a closed form,
and a dense FP64 QR reference loss.

Relative agreement is measured against max(|g|, 1e-3 * L / rho) for the
weight rho: near rho = 100 the probing rows are almost satisfied and dL/drho
falls to ~1e-7 while the loss is O(1), so the finite-difference quotient's own
rounding (~1e-16 L / step) is the floor, not the adjoint."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import column_residuals
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
FD_TOL = 1e-6


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def loss_and_grad(h, A, Ce, Be, rho, P, gbar=None):
    C, B = mb.assemble_probing(A, Ce, Be, rho)
    h.setup(C, P, B=B, options=mb.Options(ns=0, prec="fp64", probing=1, rho=rho))
    M = h.result()
    dC, dB, L = h.adjoint(C, B, gbar)
    return C, B, M, dC, dB, L


def drho(C, B, dC, dB, n, rho):
    """Chain rule for the weight: probing entries of C and B are rho * (Ce, Be)."""
    C = sp.csc_matrix(C); B = sp.csc_matrix(B)
    rows_c = C.indices >= n
    rows_b = B.indices >= n
    return (np.dot(dC[rows_c], C.data[rows_c]) + np.dot(dB[rows_b], B.data[rows_b])) / rho


def dense_loss(C, B, P):
    C = C.toarray(); B = B.toarray()
    n = P.shape[1]
    L = 0.0
    for k in range(n):
        J = P[:, k].indices
        I = np.nonzero(np.any(C[:, J] != 0, axis=1))[0]
        Q, R = np.linalg.qr(C[np.ix_(I, J)])
        m = np.linalg.solve(R, Q.T @ B[I, k])
        full = C[:, J] @ m - B[:, k]
        L += full @ full
    return L


@pytest.mark.parametrize("kinds,rho", [(("ones",), 1.0), (("ones", "alt"), 10.0),
                                       (("alt",), 100.0)])
def test_drho_finite_difference_and_closed_form(h, kinds, rho):
    w = W.aniso2d_probing(12, kinds=kinds, rho=rho)
    C, B, M, dC, dB, L = loss_and_grad(h, w.A, w.Ce, w.Be, rho, w.P)
    g = drho(C, B, dC, dB, w.n, rho)
    # closed form: dL/drho = 2 sum_k s_k^2 / rho, s_k the probing-row residuals
    R = (C @ M - B).tocsr()
    s2 = R[w.n:, :].multiply(R[w.n:, :]).sum()
    assert abs(g - 2.0 * s2 / rho) <= 1e-9 * max(abs(g), 1e-300)
    # loss reported by the adjoint
    assert abs(L - np.sum(column_residuals(C, M, B) ** 2)) <= 1e-10 * L
    # central differences
    hstep = FD_STEP * rho
    Lp = loss_and_grad(h, w.A, w.Ce, w.Be, rho + hstep, w.P)[5]
    Lm = loss_and_grad(h, w.A, w.Ce, w.Be, rho - hstep, w.P)[5]
    fd = (Lp - Lm) / (2 * hstep)
    assert abs(fd - g) <= FD_TOL * max(abs(g), 1e-3 * L / rho)


def test_dA_finite_difference(h):
    rho = 10.0
    w = W.aniso2d_probing(8, kinds=("ones", "alt"), rho=rho)
    A = sp.csc_matrix(w.A)
    E = W.probing_vectors(w.n, ("ones", "alt"))
    C, B, M, dC, dB, L = loss_and_grad(h, A, w.Ce, w.Be, rho, w.P)
    Cc = sp.csc_matrix(C)
    rng = np.random.default_rng(7)
    picks = rng.choice(A.nnz, size=12, replace=False)
    col_of = np.repeat(np.arange(w.n), np.diff(A.indptr))
    for q in picks:
        i, j = A.indices[q], col_of[q]
        # dL/dA(i,j): the A block of C plus the probing rows Ce = E A
        g = 0.0
        for p in range(Cc.indptr[j], Cc.indptr[j + 1]):
            r = Cc.indices[p]
            if r == i:
                g += dC[p]
            elif r >= w.n:
                g += dC[p] * rho * E[r - w.n, i]
        step = FD_STEP * max(1.0, abs(A.data[q]))
        vals = []
        for sgn in (+1, -1):
            Ap = A.copy()
            Ap.data[q] += sgn * step
            Cep = sp.csr_matrix(Ap.T.dot(E.T).T)
            vals.append(loss_and_grad(h, Ap, Cep, w.Be, rho, w.P)[5])
        fd = (vals[0] - vals[1]) / (2 * step)
        assert abs(fd - g) <= FD_TOL * max(abs(g), 1e-3), (q, fd, g)


def test_gbar_term_finite_difference(h):
    rho = 10.0
    w = W.aniso2d_probing(8, kinds=("ones",), rho=rho)
    rng = np.random.default_rng(3)
    C, B, M, dC0, dB0, L0 = loss_and_grad(h, w.A, w.Ce, w.Be, rho, w.P)
    gbar = rng.standard_normal(M.nnz)
    _, _, _, dC, dB, L = loss_and_grad(h, w.A, w.Ce, w.Be, rho, w.P, gbar=gbar)
    assert abs(L - (L0 + np.dot(gbar, M.data))) <= 1e-9 * abs(L)
    g = drho(C, B, dC, dB, w.n, rho)
    hstep = FD_STEP * rho
    vals = []
    for sgn in (+1, -1):
        Cp, Bp, Mp, *_ = loss_and_grad(h, w.A, w.Ce, w.Be, rho + sgn * hstep, w.P)
        vals.append(np.sum(column_residuals(Cp, Mp, Bp) ** 2) + np.dot(gbar, Mp.data))
    fd = (vals[0] - vals[1]) / (2 * hstep)
    assert abs(fd - g) <= FD_TOL * max(abs(g), 1e-3 * abs(L) / rho)


def test_loss_matches_dense_qr_reference(h):
    rho = 10.0
    w = W.aniso2d_probing(6, kinds=("ones", "alt"), rho=rho)
    C, B, M, dC, dB, L = loss_and_grad(h, w.A, w.Ce, w.Be, rho, w.P)
    assert abs(L - dense_loss(C, B, w.P)) <= 1e-10 * L
