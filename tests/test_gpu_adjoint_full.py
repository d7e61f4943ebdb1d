"""The adjoint at the benchmark sizes against central finite differences.

  anisotropic 1024^2   probing rows e = ones and alternating, rho 1, 10, 100:
                       dL/drho of the whole loss (FP64 and mixed forward);
                       dL/dA along a seeded random direction in each of 64
                       seeded columns of A (four corners among them), whose
                       column sets K_j = {k : j in J_k} are pairwise disjoint,
                       so that one pair of perturbed setups checks all 64:
                       the loss restricted to K_j moves only with column j
  27-point block 40^3  bs 3, pattern updates (-ns 3 -mn 3 -ep 0.05), probing
                       e = ones, rho 10: dL/drho at the final block pattern

Finite differences: step 1e-6 relative, agreement 1e-6 relative (dL/drho
against max(|g|, 1e-3 L / rho): near rho = 100 the probing rows are almost
satisfied and dL/drho falls towards the quotient's own rounding floor)."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import max_rel_diff
from mspai_b200 import workloads as W
from mspai_b200.autograd import _assemble, _chain

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
FD_TOL = 1e-6


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def _drho(C, B, dC, dB, n, rho):
    C = sp.csc_matrix(C); B = sp.csc_matrix(B)
    rc = C.indices >= n
    rb = B.indices >= n
    return (np.dot(dC[rc], C.data[rc]) + np.dot(dB[rb], B.data[rb])) / rho


def test_aniso_1024_drho(h):
    nx = 1024
    for rho in (1.0, 10.0, 100.0):
        w = W.aniso2d_probing(nx, kinds=("ones", "alt"), rho=rho)
        C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
        g = {}
        for prec in ("fp64", "mixed"):
            h.setup(C, w.P, B=B, options=mb.Options(ns=0, prec=prec, probing=1, rho=rho))
            dC, dB, L = h.adjoint(C, B)
            g[prec] = (_drho(C, B, dC, dB, w.n, rho), L)
        gd, L = g["fp64"]
        step = FD_STEP * rho
        vals = []
        for sgn in (+1, -1):
            Cp, Bp = mb.assemble_probing(w.A, w.Ce, w.Be, rho + sgn * step)
            h.setup(Cp, w.P, B=Bp, options=mb.Options(ns=0, prec="fp64", probing=1,
                                                      rho=rho + sgn * step))
            vals.append(h.adjoint(Cp, Bp)[2])
        fd = (vals[0] - vals[1]) / (2 * step)
        floor = max(abs(gd), 1e-3 * L / rho)
        assert abs(fd - gd) <= FD_TOL * floor, (rho, fd, gd)
        assert abs(g["mixed"][0] - gd) <= FD_TOL * floor, (rho, g["mixed"][0], gd)
        assert g["mixed"][1] == pytest.approx(L, rel=1e-10)


def _disjoint_columns(nx: int, count: int, seed: int) -> np.ndarray:
    """`count` grid nodes (the four corners first) at Manhattan distance >= 3
    from each other: their 5-point neighbourhoods do not meet."""
    rng = np.random.default_rng(seed)
    pts = [(0, 0), (0, nx - 1), (nx - 1, 0), (nx - 1, nx - 1)]
    while len(pts) < count:
        p = tuple(int(v) for v in rng.integers(0, nx, size=2))
        if all(abs(p[0] - q[0]) + abs(p[1] - q[1]) >= 3 for q in pts):
            pts.append(p)
    return np.array([iy * nx + ix for ix, iy in pts])


def test_aniso_1024_dA_64_columns(h):
    nx, rho = 1024, 10.0
    A = sp.csc_matrix(W.aniso2d(nx))
    A.sort_indices()
    n = A.shape[1]
    E = W.probing_vectors(n, ("ones", "alt")).T          # n x p
    Be = sp.csr_matrix(E.T)
    P = sp.csc_matrix(A != 0, dtype=np.float64)
    cols = _disjoint_columns(nx, 64, seed=0xADA)
    # K_j: the columns whose pattern holds j (P is symmetric: P's column j)
    K = [P.indices[P.indptr[j]:P.indptr[j + 1]] for j in cols]
    assert len(np.unique(np.concatenate(K))) == sum(len(k) for k in K)
    asm = _assemble(A, E, Be, rho)
    grads = {}
    for prec in ("fp64", "mixed"):
        h.setup(asm.C, P, B=asm.B, options=mb.Options(ns=0, prec=prec, probing=1, rho=rho))
        dC, dB, _ = h.adjoint(asm.C, asm.B)
        grads[prec], _ = _chain(asm, A, E, dC, dB, rho)
    da = grads["fp64"]
    # a seeded direction on A's nonzeros of each listed column
    rng = np.random.default_rng(0x5EED)
    d = np.zeros(A.nnz)
    for j in cols:
        d[A.indptr[j]:A.indptr[j + 1]] = rng.standard_normal(A.indptr[j + 1] - A.indptr[j])
    res = []
    for sgn in (+1, -1):
        Ap = A.copy()
        Ap.data = A.data + sgn * FD_STEP * d
        ap = _assemble(Ap, E, Be, rho)
        h.setup(ap.C, P, B=ap.B, options=mb.Options(ns=0, prec="fp64", probing=1, rho=rho))
        r, _, status = h.column_info()
        assert np.all(status == 0)
        res.append(r)
    for t, j in enumerate(cols):
        Lp = np.sum(res[0][K[t]] ** 2)
        Lm = np.sum(res[1][K[t]] ** 2)
        fd = (Lp - Lm) / (2 * FD_STEP)
        sl = slice(A.indptr[j], A.indptr[j + 1])
        g = float(np.dot(d[sl], da[sl]))
        gm = float(np.dot(d[sl], grads["mixed"][sl]))
        scale = max(abs(g), 1e-3 * np.linalg.norm(da[sl]) * np.linalg.norm(d[sl]))
        assert abs(fd - g) <= FD_TOL * scale, (j, fd, g)
        assert abs(gm - g) <= FD_TOL * scale, (j, gm, g)


def test_block27_40_drho_final_pattern(h):
    rho, bs = 10.0, 3
    w = W.block27(40, rho=rho, probing=True)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    dpat = sp.identity(w.n // bs, format="csc")
    opts = dict(ep=0.05, ns=3, mn=3, bs=bs)
    h.setup(C, dpat, B=B, options=mb.Options(prec="mixed", **opts))
    M = h.result()
    _, steps, _ = h.column_info()
    assert steps.max() > 1
    dC, dB, L = h.adjoint(C, B)
    g = _drho(C, B, dC, dB, w.n, rho)
    S = sp.csc_matrix(M, copy=True)
    S.data = np.ones_like(S.data)
    Pb = sp.csc_matrix(S[::bs, ::bs])
    Pb.data = np.ones_like(Pb.data)
    h.setup(C, Pb, B=B, options=mb.Options(prec="fp64", bs=bs, ns=0))
    assert max_rel_diff(h.result(), M) < 1e-8
    step = FD_STEP * rho
    vals = []
    for sgn in (+1, -1):
        Cp, Bp = mb.assemble_probing(w.A, w.Ce, w.Be, rho + sgn * step)
        h.setup(Cp, Pb, B=Bp, options=mb.Options(prec="fp64", bs=bs, ns=0))
        vals.append(h.adjoint(Cp, Bp)[2])
    fd = (vals[0] - vals[1]) / (2 * step)
    assert abs(fd - g) <= FD_TOL * max(abs(g), 1e-3 * L / rho), (fd, g)
