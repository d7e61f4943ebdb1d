"""Adjoint beyond the fixed scalar FP64 setup: the R factors the setup keeps
(FP64, and FP32 refined in FP64) against R recomputed in FP64; the residual
weight; adaptive scalar and block setups at their final pattern against
central finite differences of fixed-pattern setups at that pattern; the
differentiable M of mspai_b200.autograd.setup_values (gradcheck).

Finite differences: step 1e-6 relative to the parameter, agreement 1e-6
relative (against max(|g|, 1e-3 L / rho) for the weight, where dL/drho can
fall to the quotient's own rounding floor)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import mspai_b200 as mb
from helpers import max_rel_diff
from mspai_b200 import workloads as W
from mspai_b200.autograd import probing_loss, setup_values

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
FD_TOL = 1e-6


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def structure(M):
    P = sp.csc_matrix(M, copy=True)
    P.data = np.ones_like(P.data)
    P.sort_indices()
    return P


def block_pattern(M, bs):
    """The block pattern of a block setup's scalar result."""
    S = structure(M)
    Pb = sp.csc_matrix(S[::bs, ::bs])
    Pb.data = np.ones_like(Pb.data)
    return Pb


def test_kept_factors_match_recomputed(h):
    """gbar term with R kept by the setup (FP64; FP32 + two FP64 refinement
    steps) equals the FP64 recomputation, on columns of every solver path
    (|J| from 1 to a few hundred)."""
    A = W.ragged_matrix(20000, seed=11)
    P = mb.pattern_power2(A, 1e-3)
    assert np.diff(P.indptr).max() > 150
    rng = np.random.default_rng(5)
    gbar = rng.standard_normal(P.nnz)
    out = {}
    for prec in ("fp64", "mixed"):
        for keep in (False, True):
            h.setup(A, P, options=mb.Options(ns=0, prec=prec, keep_factors=keep))
            dC, _, L = h.adjoint(A, None, gbar=gbar)
            out[prec, keep] = (dC, L)
    ref, Lref = out["fp64", False]
    scale = np.max(np.abs(ref))
    for key, tol in ((("fp64", True), 1e-11), (("mixed", True), 1e-8), (("mixed", False), 1e-8)):
        dC, L = out[key]
        assert np.max(np.abs(dC - ref)) <= tol * scale, key
        assert abs(L - Lref) <= tol * abs(Lref), key


def test_residual_weight(h):
    w = W.aniso2d_probing(16, kinds=("ones", "alt"), rho=10.0)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, 10.0)
    h.setup(C, w.P, B=B, options=mb.Options(ns=0, prec="fp64", probing=1, rho=10.0,
                                            keep_factors=True))
    M = h.result()
    gbar = np.random.default_rng(2).standard_normal(M.nnz)
    d1, b1, L1 = h.adjoint(C, B, gbar=gbar)
    d0, b0, L0 = h.adjoint(C, B)
    dg, bg, Lg = h.adjoint(C, B, gbar=gbar, residual_weight=0.0)
    d3, b3, L3 = h.adjoint(C, B, gbar=gbar, residual_weight=3.0)
    s = np.max(np.abs(d1))
    assert np.max(np.abs(d1 - d0 - dg)) <= 1e-12 * s
    assert np.max(np.abs(b1 - b0 - bg)) <= 1e-12 * s
    assert np.max(np.abs(d3 - 3 * d0 - dg)) <= 1e-12 * s
    assert Lg == pytest.approx(float(np.dot(gbar, M.data)), rel=1e-12)
    assert L3 == pytest.approx(3 * L0 + Lg, rel=1e-12)


def test_adaptive_scalar_at_final_pattern(h):
    w = W.convdiff3d(10)
    A = sp.csc_matrix(w.A)
    opts = dict(ep=0.4, ns=5, mn=5, um=1)
    h.setup(A, w.P, options=mb.Options(prec="fp64", **opts))
    M = h.result()
    _, steps, _ = h.column_info()
    assert steps.max() > 1
    dC, _, L = h.adjoint(A)
    Pf = structure(M)
    # the fixed-pattern setup at the final pattern reproduces M and the loss
    h.setup(A, Pf, options=mb.Options(ns=0, prec="fp64"))
    assert max_rel_diff(h.result(), M) < 1e-10
    dCf, _, Lf = h.adjoint(A)
    assert Lf == pytest.approx(L, rel=1e-11)
    assert np.max(np.abs(dCf - dC)) <= 1e-9 * np.max(np.abs(dC))
    # mixed forward: same final pattern, same gradient
    h.setup(A, w.P, options=mb.Options(prec="mixed", **opts))
    assert np.array_equal(structure(h.result()).indices, Pf.indices)
    dCm, _, Lm = h.adjoint(A)
    assert np.max(np.abs(dCm - dC)) <= 1e-8 * np.max(np.abs(dC))
    # central differences at the final pattern
    rng = np.random.default_rng(17)
    for q in rng.choice(A.nnz, size=10, replace=False):
        step = FD_STEP * max(1.0, abs(A.data[q]))
        vals = []
        for sgn in (+1, -1):
            Ap = A.copy()
            Ap.data[q] += sgn * step
            h.setup(Ap, Pf, options=mb.Options(ns=0, prec="fp64"))
            vals.append(h.adjoint(Ap)[2])
        fd = (vals[0] - vals[1]) / (2 * step)
        assert abs(fd - dC[q]) <= FD_TOL * max(abs(dC[q]), 1e-3), (q, fd, dC[q])


def _block_setup(h, A, Ce, Be, rho, P, bs, prec, **opts):
    C, B = mb.assemble_probing(A, Ce, Be, rho)
    h.setup(C, P, B=B, options=mb.Options(prec=prec, bs=bs, **opts))
    return C, B


def _drho(C, B, dC, dB, n, rho):
    C = sp.csc_matrix(C); B = sp.csc_matrix(B)
    rc = C.indices >= n
    rb = B.indices >= n
    return (np.dot(dC[rc], C.data[rc]) + np.dot(dB[rb], B.data[rb])) / rho


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_block_updates_drho_at_final_pattern(h, prec):
    rho, bs = 10.0, 3
    w = W.block27(6, rho=rho, probing=True)
    dpat = sp.identity(w.n // bs, format="csc")
    C, B = _block_setup(h, w.A, w.Ce, w.Be, rho, dpat, bs, prec, ep=0.05, ns=3, mn=3)
    M = h.result()
    _, steps, _ = h.column_info()
    assert steps.max() > 1
    dC, dB, L = h.adjoint(C, B)
    g = _drho(C, B, dC, dB, w.n, rho)
    Pb = block_pattern(M, bs)
    C0, B0 = _block_setup(h, w.A, w.Ce, w.Be, rho, Pb, bs, "fp64", ns=0)
    assert max_rel_diff(h.result(), M) < (1e-10 if prec == "fp64" else 1e-8)
    L0 = h.adjoint(C0, B0)[2]
    assert L0 == pytest.approx(L, rel=1e-10)
    step = FD_STEP * rho
    vals = []
    for sgn in (+1, -1):
        Cp, Bp = _block_setup(h, w.A, w.Ce, w.Be, rho + sgn * step, Pb, bs, "fp64", ns=0)
        vals.append(h.adjoint(Cp, Bp)[2])
    fd = (vals[0] - vals[1]) / (2 * step)
    assert abs(fd - g) <= FD_TOL * max(abs(g), 1e-3 * L / rho), (fd, g)


def test_block_dC_finite_difference(h):
    rho, bs = 10.0, 3
    w = W.block27(5, rho=rho, probing=True)
    dpat = sp.identity(w.n // bs, format="csc")
    C, B = _block_setup(h, w.A, w.Ce, w.Be, rho, dpat, bs, "fp64", ep=0.05, ns=3, mn=3)
    Pb = block_pattern(h.result(), bs)
    dC, dB, L = h.adjoint(C, B)
    C = sp.csc_matrix(C)
    rng = np.random.default_rng(23)
    for q in rng.choice(C.nnz, size=8, replace=False):
        step = FD_STEP * max(1.0, abs(C.data[q]))
        vals = []
        for sgn in (+1, -1):
            Cp = C.copy()
            Cp.data[q] += sgn * step
            h.setup(Cp, Pb, B=B, options=mb.Options(prec="fp64", bs=bs, ns=0))
            vals.append(h.adjoint(Cp, B)[2])
        fd = (vals[0] - vals[1]) / (2 * step)
        assert abs(fd - dC[q]) <= FD_TOL * max(abs(dC[q]), 1e-3), (q, fd, dC[q])
    # dL/dB at a few target entries
    B = sp.csc_matrix(B)
    for q in rng.choice(B.nnz, size=4, replace=False):
        vals = []
        for sgn in (+1, -1):
            Bp = B.copy()
            Bp.data[q] += sgn * FD_STEP
            h.setup(C, Pb, B=Bp, options=mb.Options(prec="fp64", bs=bs, ns=0))
            vals.append(h.adjoint(C, Bp)[2])
        fd = (vals[0] - vals[1]) / (2 * FD_STEP)
        assert abs(fd - dB[q]) <= FD_TOL * max(abs(dB[q]), 1e-3), (q, fd, dB[q])


def test_gbar_refused_for_blocks(h):
    w = W.block27(3, rho=10.0, probing=False)
    dpat = sp.identity(w.n // 3, format="csc")
    h.setup(w.A, dpat, options=mb.Options(prec="fp64", bs=3, ns=0))
    with pytest.raises(mb.MspaiError, match="gbar"):
        h.adjoint(w.A, None, gbar=np.zeros(h.nnz()))


def test_setup_values_gradcheck(h):
    A = W.aniso2d(5).tocsc()
    A.sort_indices()
    E = W.probing_vectors(A.shape[0], ("ones",)).T
    Be = sp.csr_matrix(E.T)
    P = sp.csc_matrix(A != 0, dtype=np.float64)
    a = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
    r = torch.tensor(4.0, dtype=torch.float64, requires_grad=True)
    f = lambda a_, r_: setup_values(a_, r_, A, E, Be, P, h)
    assert torch.autograd.gradcheck(f, (a, r), eps=1e-6, atol=1e-6, rtol=1e-5)


def test_mixed_and_adaptive_autograd(h):
    """probing_loss with a mixed forward equals the FP64 one; with pattern
    updates its gradient is the one at the final pattern."""
    A = W.aniso2d(12).tocsc()
    A.sort_indices()
    E = W.probing_vectors(A.shape[0], ("ones", "alt")).T
    Be = sp.csr_matrix(E.T)
    P = sp.csc_matrix(A != 0, dtype=np.float64)
    grads = {}
    for prec in ("fp64", "mixed"):
        a = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
        r = torch.tensor(10.0, dtype=torch.float64, requires_grad=True)
        L = probing_loss(a, r, A, E, Be, P, h, prec=prec)
        L.backward()
        grads[prec] = (float(L.detach()), a.grad.numpy().copy(), float(r.grad))
    (L64, ga, gr), (Lm, gam, grm) = grads["fp64"], grads["mixed"]
    assert Lm == pytest.approx(L64, rel=1e-10)
    assert np.max(np.abs(gam - ga)) <= 1e-8 * np.max(np.abs(ga))
    assert grm == pytest.approx(gr, rel=1e-7, abs=1e-9 * L64)
    # adaptive: the gradient at the final pattern (fixed-pattern gradcheck there)
    S = sp.identity(A.shape[0], format="csc")
    a = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
    r = torch.tensor(10.0, dtype=torch.float64, requires_grad=True)
    L = probing_loss(a, r, A, E, Be, S, h, ns=3, mn=2, ep=0.2)
    L.backward()
    Pf = structure(h.result())
    assert Pf.nnz > A.shape[0]  # the pattern grew
    a2 = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
    r2 = torch.tensor(10.0, dtype=torch.float64, requires_grad=True)
    L2 = probing_loss(a2, r2, A, E, Be, Pf, h)
    L2.backward()
    assert float(L2) == pytest.approx(float(L), rel=1e-10)
    assert np.max(np.abs(a2.grad.numpy() - a.grad.numpy())) <= 1e-9 * np.max(np.abs(a.grad.numpy()))
    assert float(r2.grad) == pytest.approx(float(r.grad), rel=1e-8, abs=1e-10 * float(L))
