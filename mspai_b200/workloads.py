"""Seeded synthetic inputs for the five setup workloads.

No public matrix collection is named for the MSPAI setup benchmark, so every
workload is generated here from a documented recipe and a fixed seed
(numpy PCG64).  Each generator returns a ``Workload``: the system matrix A as
CSC (int64 column pointers, int32 sorted row indices, float64 values), the
start pattern P of M as CSC (pattern only), the probing rows Ce (p x n, CSR-like
row lists) and Be for probing workloads, and the reference options that
describe the run (-ep, -ns, -mn, -bs, -rho, ...).

Workloads (sizes are the full ones; every generator takes smaller grids for
tests):

* ``poisson2d``      -- 2-D 5-point Poisson, Dirichlet, diag 4, off -1.
                        P = pattern(A), no pattern updates.  (64 x 64, n=4096)
* ``convdiff3d``     -- 3-D 7-point convection-diffusion on an N^3 cell grid.
                        kappa per cell log-uniform in [1e-2, 1]; face
                        coefficient = harmonic mean of the two cells (the cell's
                        own kappa on a Dirichlet boundary face); first-order
                        upwind for v = Pe * (1, 0.5, 0.25) / max|v| with Pe = 20
                        (L = 1, kappa_ref = 1); rows scaled by h^2, h=1/(N+1).
                        P = diagonal, -ep 0.4 -ns 5 -mn 5 -um 1.  (48^3)
* ``ragged``         -- random nonsymmetric: per column k, U{4..32} distinct
                        off-diagonal rows drawn uniformly (!= k), values N(0,1),
                        diagonal 1.5 * sum |off|.  P = pattern(A^2) with
                        entries below 1e-3 of the column's max |A^2| dropped.
                        Fixed pattern.  (n = 1,000,000)
* ``aniso2d_probing``-- 2-D anisotropic 5-point on an N x N grid, coefficient 1
                        in x and 1e-3 in y (diag 2.002, off -1 / -0.001).
                        Probing vectors e = ones and e_i = (-1)^i; Ce = e^T A,
                        Be = e^T, weight rho.  P = pattern(A), -ns 0.
                        (1024 x 1024)
* ``block27``        -- 3-D 27-point stencil with 3 unknowns per node on an
                        N^3 node grid; diagonal blocks Q Q^T + 3 I, off-diagonal
                        blocks -(1/26) R, with Q drawn per node and R per
                        (node, neighbour) pair, entries N(0,1).  Block size 3,
                        P = block pattern of A, -ns 3 -mn 3; probing e = ones,
                        rho = 10.  (40^3 nodes, n = 192,000)
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np
import scipy.sparse as sp

SEEDS = {
    "poisson2d": 0x5EED0001,
    "convdiff3d": 0x5EED0002,
    "ragged": 0x5EED0003,
    "aniso2d_probing": 0x5EED0004,
    "block27": 0x5EED0005,
}


@dataclasses.dataclass
class Workload:
    name: str
    A: sp.csc_matrix                 # n x n system matrix
    P: sp.csc_matrix                 # n x n start pattern (values unused)
    Ce: Optional[sp.csr_matrix] = None   # p x n probing rows for C (e^T A)
    Be: Optional[sp.csr_matrix] = None   # p x n probing rows for B (e^T)
    options: dict = dataclasses.field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.A.shape[1]


def _canon_csc(M: sp.spmatrix) -> sp.csc_matrix:
    M = sp.csc_matrix(M, dtype=np.float64)
    M.sum_duplicates()
    M.sort_indices()
    return M


def csc_arrays(M: sp.spmatrix):
    """(colptr int64, rowidx int32, values float64) of a canonical CSC matrix."""
    M = _canon_csc(M)
    return (np.ascontiguousarray(M.indptr, dtype=np.int64),
            np.ascontiguousarray(M.indices, dtype=np.int32),
            np.ascontiguousarray(M.data, dtype=np.float64))


def _pattern(M: sp.spmatrix) -> sp.csc_matrix:
    P = _canon_csc(M).copy()
    P.data = np.ones_like(P.data)
    return P


def _lap1d(n: int, off: float) -> sp.csr_matrix:
    e = np.ones(n)
    return sp.diags([off * e[:-1], off * e[:-1]], [-1, 1], shape=(n, n), format="csr")


def poisson2d(nx: int = 64) -> Workload:
    """2-D 5-point Poisson on an nx x nx interior grid, Dirichlet boundaries."""
    n = nx * nx
    T = _lap1d(nx, -1.0)
    I = sp.identity(nx, format="csr")
    A = sp.kron(I, T) + sp.kron(T, I) + 4.0 * sp.identity(n)
    A = _canon_csc(A)
    return Workload("poisson2d", A, _pattern(A),
                    options=dict(ep=0.4, ns=0, mn=5, pattern="A", target="I"))


def aniso2d(nx: int = 1024, cy: float = 1e-3) -> sp.csc_matrix:
    n = nx * nx
    Tx = _lap1d(nx, -1.0)
    Ty = _lap1d(nx, -cy)
    I = sp.identity(nx, format="csr")
    # x varies fastest: index = y*nx + x
    A = sp.kron(I, Tx) + sp.kron(Ty, I) + (2.0 + 2.0 * cy) * sp.identity(n)
    return _canon_csc(A)


def probing_vectors(n: int, kinds=("ones", "alt")) -> np.ndarray:
    rows = []
    for k in kinds:
        if k == "ones":
            rows.append(np.ones(n))
        elif k == "alt":
            rows.append(np.where(np.arange(n) % 2 == 0, 1.0, -1.0))
        else:
            raise ValueError(k)
    return np.stack(rows)


def aniso2d_probing(nx: int = 1024, kinds=("ones",), rho: float = 1.0) -> Workload:
    """Anisotropic 2-D diffusion with probing rows Ce = e^T A, Be = e^T."""
    A = aniso2d(nx)
    E = probing_vectors(A.shape[0], kinds)
    Ce = sp.csr_matrix(A.T.dot(E.T).T)           # p x n: e^T A
    Ce.eliminate_zeros()
    Be = sp.csr_matrix(E)
    return Workload("aniso2d_probing", A, _pattern(A), Ce=Ce, Be=Be,
                    options=dict(ep=0.4, ns=0, mn=5, rho=rho, pattern="A", target="I"))


def convdiff3d(N: int = 48, pe: float = 20.0, seed: Optional[int] = None) -> Workload:
    """3-D 7-point convection-diffusion, upwind, random log-uniform kappa."""
    rng = np.random.Generator(np.random.PCG64(SEEDS["convdiff3d"] if seed is None else seed))
    n = N ** 3
    h = 1.0 / (N + 1)
    kappa = np.exp(rng.uniform(np.log(1e-2), np.log(1.0), size=n))
    v = np.array([1.0, 0.5, 0.25])
    v = v * (pe / np.max(np.abs(v)))
    idx = np.arange(n)
    x = idx % N
    y = (idx // N) % N
    z = idx // (N * N)
    coords = (x, y, z)
    strides = (1, N, N * N)
    diag = np.zeros(n)
    rows, cols, vals = [], [], []
    for d in range(3):
        c = coords[d]
        s = strides[d]
        for sgn in (-1, +1):
            has_nb = (c + sgn >= 0) & (c + sgn < N)
            nb = idx + sgn * s
            kf = np.where(has_nb,
                          2.0 * kappa * kappa[np.clip(nb, 0, n - 1)]
                          / (kappa + kappa[np.clip(nb, 0, n - 1)]),
                          kappa)
            diag += kf
            # upwind: the neighbour on the upstream side carries -h*|v_d|
            upstream = (sgn < 0) if v[d] > 0 else (sgn > 0)
            off = -kf - (h * abs(v[d]) if upstream else 0.0)
            sel = has_nb
            rows.append(idx[sel]); cols.append(nb[sel]); vals.append(off[sel])
        diag += h * abs(v[d])
    rows.append(idx); cols.append(idx); vals.append(diag)
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    A = _canon_csc(A)
    P = _canon_csc(sp.identity(n))
    return Workload("convdiff3d", A, P,
                    options=dict(ep=0.4, ns=5, mn=5, um=1, pattern="diag", target="I"))


def ragged_matrix(n: int, seed: Optional[int] = None) -> sp.csc_matrix:
    rng = np.random.Generator(np.random.PCG64(SEEDS["ragged"] if seed is None else seed))
    cnt = rng.integers(4, 33, size=n)             # U{4..32}
    total = int(cnt.sum())
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(cnt + 1, out=colptr[1:])
    # draw rows != k uniformly: r in [0, n-1), shift past k
    r = rng.integers(0, n - 1, size=total)
    colidx = np.repeat(np.arange(n), cnt)
    r = r + (r >= colidx)
    vals = rng.standard_normal(total)
    # make rows distinct within a column by redrawing duplicates
    order = np.lexsort((r, colidx))
    r = r[order]; vals = vals[order]
    for _ in range(64):
        dup = np.zeros(total, dtype=bool)
        dup[1:] = (r[1:] == r[:-1]) & (colidx[1:] == colidx[:-1])
        if not dup.any():
            break
        nd = int(dup.sum())
        rr = rng.integers(0, n - 1, size=nd)
        rr = rr + (rr >= colidx[dup])
        r[dup] = rr
        order = np.lexsort((r, colidx))
        r = r[order]; vals = vals[order]
    offsum = np.bincount(colidx, weights=np.abs(vals), minlength=n)
    rows = np.concatenate([r, np.arange(n)])
    cols = np.concatenate([colidx, np.arange(n)])
    data = np.concatenate([vals, 1.5 * offsum])
    A = sp.coo_matrix((data, (rows, cols)), shape=(n, n))
    return _canon_csc(A)


def square_pattern_dropped(A: sp.csc_matrix, drop: float = 1e-3, chunk: int = 65536) -> sp.csc_matrix:
    """Pattern of A^2, dropping |(A^2)_ij| < drop * max_i |(A^2)_ij| per column."""
    A = sp.csc_matrix(A)
    n = A.shape[1]
    pieces = []
    for c0 in range(0, n, chunk):
        S = (A @ A[:, c0:c0 + chunk]).tocsc()
        S.sum_duplicates()
        absd = np.abs(S.data)
        colmax = np.maximum.reduceat(absd, S.indptr[:-1]) if S.nnz else np.zeros(0)
        lens = np.diff(S.indptr)
        thr = np.repeat(drop * colmax[: len(lens)], lens)
        keep = absd >= thr
        S.data = np.where(keep, 1.0, 0.0)
        S.eliminate_zeros()
        pieces.append(S)
    P = sp.hstack(pieces, format="csc")
    return _pattern(P)


def ragged(n: int = 1_000_000, seed: Optional[int] = None) -> Workload:
    A = ragged_matrix(n, seed)
    P = square_pattern_dropped(A)
    return Workload("ragged", A, P,
                    options=dict(ep=0.4, ns=0, mn=5, pattern="file", target="I"))


def block27_matrix(N: int = 40, seed: Optional[int] = None) -> sp.csc_matrix:
    rng = np.random.Generator(np.random.PCG64(SEEDS["block27"] if seed is None else seed))
    nn = N ** 3
    idx = np.arange(nn)
    x = idx % N
    y = (idx // N) % N
    z = idx // (N * N)
    Q = rng.standard_normal((nn, 3, 3))
    D = np.einsum("nij,nkj->nik", Q, Q) + 3.0 * np.eye(3)[None]
    brow, bcol, blocks = [idx], [idx], [D]
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == 0 and dy == 0 and dz == 0:
                    continue
                ok = ((x + dx >= 0) & (x + dx < N) & (y + dy >= 0) & (y + dy < N)
                      & (z + dz >= 0) & (z + dz < N))
                src = idx[ok]
                nb = src + dx + dy * N + dz * N * N
                R = rng.standard_normal((nn, 3, 3))[ok]
                # block row = neighbour (row block), block column = node
                brow.append(nb); bcol.append(src); blocks.append(-(1.0 / 26.0) * R)
    brow = np.concatenate(brow); bcol = np.concatenate(bcol); blocks = np.concatenate(blocks)
    ii = (3 * brow[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
    jj = (3 * bcol[:, None, None] + np.arange(3)[None, None, :]).repeat(3, axis=1)
    A = sp.coo_matrix((blocks.ravel(), (ii.ravel(), jj.ravel())), shape=(3 * nn, 3 * nn))
    return _canon_csc(A)


def block27(N: int = 40, rho: float = 10.0, probing: bool = True) -> Workload:
    A = block27_matrix(N)
    Ce = Be = None
    if probing:
        E = probing_vectors(A.shape[0], ("ones",))
        Ce = sp.csr_matrix(A.T.dot(E.T).T)
        Be = sp.csr_matrix(E)
    return Workload("block27", A, _pattern(A), Ce=Ce, Be=Be,
                    options=dict(ep=0.4, ns=3, mn=3, bs=3, rho=rho, pattern="A", target="I"))


# ---------------------------------------------------------------- Matrix Market
def write_mm(path: str, M: sp.spmatrix, pattern: bool = False) -> None:
    """Matrix Market coordinate writer ('general'; 'pattern' drops values),
    entries in column order, values with 17 significant digits (exact)."""
    import pandas as pd
    C = sp.coo_matrix(M)
    order = np.lexsort((C.row, C.col))
    cols = {"r": C.row[order].astype(np.int64) + 1, "c": C.col[order].astype(np.int64) + 1}
    if not pattern:
        cols["v"] = C.data[order]
    with open(path, "w") as f:
        kind = "pattern" if pattern else "real"
        f.write(f"%%MatrixMarket matrix coordinate {kind} general\n")
        f.write(f"{C.shape[0]} {C.shape[1]} {C.nnz}\n")
        pd.DataFrame(cols).to_csv(f, sep=" ", header=False, index=False, float_format="%.17g")


def read_mm(path: str) -> sp.csc_matrix:
    """Matrix Market coordinate reader (real/pattern, general/symmetric)."""
    with open(path) as f:
        header = f.readline().split()
        kind = header[3].lower() if len(header) > 3 else "real"
        sym = header[4].lower() if len(header) > 4 else "general"
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(t) for t in line.split())
        data = np.loadtxt(f, ndmin=2) if nnz else np.zeros((0, 3))
    r = data[:, 0].astype(np.int64) - 1
    c = data[:, 1].astype(np.int64) - 1
    v = data[:, 2] if (kind != "pattern" and data.shape[1] > 2) else np.ones(len(r))
    if sym in ("symmetric", "hermitian"):
        off = r != c
        r, c, v = np.concatenate([r, c[off]]), np.concatenate([c, r[off]]), np.concatenate([v, v[off]])
    return _canon_csc(sp.coo_matrix((v, (r, c)), shape=(m, n)))


def write_workload(w: Workload, directory: str) -> dict:
    """Writes A, P and the probing files; returns the file paths."""
    os.makedirs(directory, exist_ok=True)
    paths = {"A": os.path.join(directory, "A.mtx"), "P": os.path.join(directory, "P.mtx")}
    write_mm(paths["A"], w.A)
    write_mm(paths["P"], w.P, pattern=True)
    if w.Ce is not None:
        paths["Ce"] = os.path.join(directory, "Ce.mtx")
        paths["Be"] = os.path.join(directory, "Be.mtx")
        write_mm(paths["Ce"], w.Ce)
        write_mm(paths["Be"], w.Be)
    return paths
