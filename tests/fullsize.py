"""Helpers of the full-size parity tests: run the reference's own column loop
(oracle/_ref/ref_driver, compiled from the reference sources) on a sample of
columns of a benchmark-size workload and compare with the GPU's columns.

Test infrastructure only.  The reference reads Matrix Market files, so the
helpers write them (pandas, 17 significant digits: the doubles round-trip
exactly) and read its output back."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pandas as pd
import scipy.sparse as sp

from helpers import max_rel_diff

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DRIVER = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_driver")


def write_mm(path: str, M: sp.spmatrix, pattern: bool = False) -> None:
    C = sp.coo_matrix(M)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {'pattern' if pattern else 'real'} general\n")
        f.write(f"{C.shape[0]} {C.shape[1]} {C.nnz}\n")
        cols = {"r": C.row.astype(np.int64) + 1, "c": C.col.astype(np.int64) + 1}
        if not pattern:
            cols["v"] = C.data
        pd.DataFrame(cols).to_csv(f, sep=" ", header=False, index=False, float_format="%.17g")


def read_mm(path: str) -> sp.csc_matrix:
    with open(path) as f:
        f.readline()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(t) for t in line.split())
    if nnz == 0:
        return sp.csc_matrix((m, n))
    d = pd.read_csv(path, sep=r"\s+", skiprows=2, header=None, engine="c",
                    float_precision="round_trip")
    M = sp.csc_matrix((d[2].to_numpy(np.float64), (d[0].to_numpy(np.int64) - 1,
                                                     d[1].to_numpy(np.int64) - 1)), shape=(m, n))
    M.sort_indices()
    return M


def stratified_columns(sizes: np.ndarray, nstrata: int, per: int, seed: int,
                       top: int = 0) -> np.ndarray:
    """`per` seeded random columns from each of `nstrata` equal-count strata of
    `sizes`, plus the `top` largest columns; sorted, unique."""
    rng = np.random.default_rng(seed)
    order = np.argsort(sizes, kind="stable")
    picks = []
    for part in np.array_split(order, nstrata):
        if len(part):
            picks.append(rng.choice(part, size=min(per, len(part)), replace=False))
    if top:
        picks.append(order[-top:])
    return np.unique(np.concatenate(picks))


def restrict(A: sp.csc_matrix, P: sp.csc_matrix, cols: np.ndarray):
    """A sub-problem whose listed columns have exactly the least-squares
    problems of the full one at a fixed pattern: A keeps the columns that the
    listed columns' patterns use (the others become unit columns, never read),
    P keeps the listed columns (diagonal elsewhere)."""
    A = sp.csc_matrix(A)
    P = sp.csc_matrix(P)
    n = P.shape[1]
    keep = np.zeros(A.shape[1], dtype=bool)
    for k in cols:
        keep[P.indices[P.indptr[k]:P.indptr[k + 1]]] = True
    lens = np.diff(A.indptr)
    colmask = np.repeat(keep, lens)
    other = np.nonzero(~keep)[0]
    rows = np.concatenate([A.indices[colmask], other])
    ccol = np.concatenate([np.repeat(np.arange(A.shape[1]), lens)[colmask], other])
    vals = np.concatenate([A.data[colmask], np.ones(len(other))])
    Asub = sp.csc_matrix((vals, (rows, ccol)), shape=A.shape)
    sel = np.zeros(n, dtype=bool)
    sel[cols] = True
    plen = np.diff(P.indptr)
    pmask = np.repeat(sel, plen)
    prow = np.concatenate([P.indices[pmask], np.nonzero(~sel)[0]])
    pcol = np.concatenate([np.repeat(np.arange(n), plen)[pmask], np.nonzero(~sel)[0]])
    Psub = sp.csc_matrix((np.ones(len(prow)), (prow, pcol)), shape=P.shape)
    return Asub, Psub, keep


def run_reference(directory: str, args, cols: np.ndarray, timeout: float = 1200.0) -> sp.csc_matrix:
    """Runs the reference on the listed (block) columns; returns its output."""
    colfile = os.path.join(directory, "cols.txt")
    np.savetxt(colfile, np.asarray(cols, dtype=np.int64), fmt="%d")
    out = os.path.join(directory, "Mref.mtx")
    r = subprocess.run([REF_DRIVER] + [str(a) for a in args] + ["-colfile", colfile, "-out", out],
                       cwd=directory, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return read_mm(out)


def scalar_columns(cols: np.ndarray, bs: int = 1) -> np.ndarray:
    return np.concatenate([np.arange(bs * k, bs * k + bs) for k in cols]) if bs > 1 else cols


def compare_columns(M_gpu: sp.spmatrix, M_ref: sp.spmatrix, cols: np.ndarray, tol: float):
    """(number of columns whose index sets differ, largest per-entry relative
    difference over the columns whose index sets agree)."""
    G = sp.csc_matrix(M_gpu)[:, cols]
    R = sp.csc_matrix(M_ref)[:, cols]
    G.sort_indices()
    R.sort_indices()
    bad = []
    for t in range(len(cols)):
        g = G.indices[G.indptr[t]:G.indptr[t + 1]]
        r = R.indices[R.indptr[t]:R.indptr[t + 1]]
        if not np.array_equal(g, r):
            bad.append(t)
    good = np.setdiff1d(np.arange(len(cols)), bad)
    diff = max_rel_diff(G[:, good], R[:, good]) if len(good) else 0.0
    return len(bad), diff, [int(cols[t]) for t in bad]


def ls_residuals(C: sp.csc_matrix, M: sp.csc_matrix, cols: np.ndarray, B=None) -> np.ndarray:
    """||C(I, J) m_k - b(I)||_2 over I_k = rows of C(:, J_k) (the reference's
    Residual_Norm, src/Spai_Sub.imp:915-941), for the listed columns."""
    C = sp.csc_matrix(C)
    M = sp.csc_matrix(M)
    out = np.zeros(len(cols))
    for t, k in enumerate(cols):
        J = M.indices[M.indptr[k]:M.indptr[k + 1]]
        m = M.data[M.indptr[k]:M.indptr[k + 1]]
        sub = C[:, J]
        I = np.unique(sub.indices)
        r = sub[I, :] @ m
        if B is None:
            r[I == k] -= 1.0
        else:
            r -= np.asarray(sp.csc_matrix(B)[I, k].todense()).ravel()
        out[t] = np.linalg.norm(r)
    return out
