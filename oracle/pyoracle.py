"""ctypes binding of the CPU restatement (oracle/spai_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, to check (never to produce) the GPU results.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libspai_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        lib.oracle_spai_scalar.restype = ctypes.c_int
        lib.oracle_spai_scalar.argtypes = [
            ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, P,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P]
        lib.oracle_spai_block.restype = ctypes.c_int
        lib.oracle_spai_block.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P, P, P, P,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P]
        _lib = lib
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def stack_probing(A: sp.csc_matrix, Ce: Optional[sp.spmatrix], rho: float) -> sp.csc_matrix:
    """C = [A; rho*Ce] (probing rows appended at n..n+p-1)."""
    if Ce is None:
        return sp.csc_matrix(A)
    C = sp.vstack([A, rho * sp.csr_matrix(Ce)], format="csc")
    C.sort_indices()
    return C


def target(n: int, Be: Optional[sp.spmatrix], rho: float) -> sp.csc_matrix:
    """B = [I; rho*Be]."""
    B = sp.identity(n, format="csc")
    if Be is not None:
        B = sp.vstack([B, rho * sp.csr_matrix(Be)], format="csc")
    B = sp.csc_matrix(B)
    B.sort_indices()
    return B


class OracleResult:
    def __init__(self, M, res, steps, info):
        self.M = M            # scipy CSC, n x n
        self.res = res        # per-column ||C(I,J) m - b||_2
        self.steps = steps    # LS solves per column
        self.info = info      # dtrtrs info per column


def spai_scalar(C: sp.csc_matrix, P: sp.csc_matrix, *, B: Optional[sp.csc_matrix] = None,
                UP: Optional[sp.csc_matrix] = None, ep: float = 0.4, mn: int = 5, ns: int = 5,
                um: int = 1, cols: Optional[tuple] = None,
                col_list: Optional[np.ndarray] = None) -> OracleResult:
    """Columns [cols[0], cols[1]) (all when None), or the columns in col_list."""
    lib = load()
    C = sp.csc_matrix(C, dtype=np.float64)
    C.sort_indices()
    nrows, n = C.shape
    cptr = np.ascontiguousarray(C.indptr, dtype=np.int64)
    cidx = np.ascontiguousarray(C.indices, dtype=np.int32)
    cval = np.ascontiguousarray(C.data, dtype=np.float64)
    R = sp.csr_matrix(C[:n, :])
    R.sort_indices()
    rptr = np.ascontiguousarray(R.indptr, dtype=np.int64)
    rcol = np.ascontiguousarray(R.indices, dtype=np.int32)
    P = sp.csc_matrix(P)
    P.sort_indices()
    pptr = np.ascontiguousarray(P.indptr, dtype=np.int64)
    pidx = np.ascontiguousarray(P.indices, dtype=np.int32)
    bptr = bidx = bval = None
    if B is not None:
        B = sp.csc_matrix(B, dtype=np.float64)
        B.sort_indices()
        bptr = np.ascontiguousarray(B.indptr, dtype=np.int64)
        bidx = np.ascontiguousarray(B.indices, dtype=np.int32)
        bval = np.ascontiguousarray(B.data, dtype=np.float64)
    upptr = upidx = None
    if UP is not None:
        UP = sp.csc_matrix(UP)
        UP.sort_indices()
        upptr = np.ascontiguousarray(UP.indptr, dtype=np.int64)
        upidx = np.ascontiguousarray(UP.indices, dtype=np.int32)
    lst = None
    if col_list is not None:
        lst = np.ascontiguousarray(col_list, dtype=np.int32)
        lo, hi = 0, len(lst)
    else:
        lo, hi = (0, n) if cols is None else cols
    stride = int(np.diff(pptr).max()) + mn * ns + 1
    out_len = np.zeros(n, dtype=np.int32)
    out_idx = np.zeros(n * stride, dtype=np.int32)
    out_val = np.zeros(n * stride, dtype=np.float64)
    out_res = np.zeros(n, dtype=np.float64)
    out_steps = np.zeros(n, dtype=np.int32)
    out_info = np.zeros(n, dtype=np.int32)
    rc = lib.oracle_spai_scalar(nrows, n, _ptr(cptr), _ptr(cidx), _ptr(cval), _ptr(rptr),
                                _ptr(rcol), _ptr(bptr), _ptr(bidx), _ptr(bval), _ptr(pptr),
                                _ptr(pidx), _ptr(upptr), _ptr(upidx), float(ep), int(mn),
                                int(ns), int(um), int(lo), int(hi), stride, _ptr(out_len),
                                _ptr(out_idx), _ptr(out_val), _ptr(out_res), _ptr(out_steps),
                                _ptr(out_info), _ptr(lst))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    lens = out_len.astype(np.int64)
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=colptr[1:])
    sel = (np.arange(stride)[None, :] < lens[:, None]).ravel()
    M = sp.csc_matrix((out_val[sel], out_idx[sel], colptr), shape=(n, n))
    return OracleResult(M, out_res, out_steps, out_info)


def spai_block(C: sp.csc_matrix, Pb: sp.csc_matrix, bs: int, *,
               B: Optional[sp.csc_matrix] = None, ep: float = 0.4, mn: int = 5, ns: int = 5,
               um: int = 1, blocks: Optional[tuple] = None,
               block_list: Optional[np.ndarray] = None) -> OracleResult:
    """Block SPAI with constant block size bs; Pb is the (n/bs x n/bs) block pattern.
    Block columns [blocks[0], blocks[1]) (all when None), or those in block_list."""
    lib = load()
    C = sp.csc_matrix(C, dtype=np.float64)
    C.sort_indices()
    nrows, n = C.shape
    cptr = np.ascontiguousarray(C.indptr, dtype=np.int64)
    cidx = np.ascontiguousarray(C.indices, dtype=np.int32)
    cval = np.ascontiguousarray(C.data, dtype=np.float64)
    R = sp.csr_matrix(C[:n, :])
    R.sort_indices()
    rptr = np.ascontiguousarray(R.indptr, dtype=np.int64)
    rcol = np.ascontiguousarray(R.indices, dtype=np.int32)
    Pb = sp.csc_matrix(Pb)
    Pb.sort_indices()
    pptr = np.ascontiguousarray(Pb.indptr, dtype=np.int64)
    pidx = np.ascontiguousarray(Pb.indices, dtype=np.int32)
    bptr = bidx = bval = None
    if B is not None:
        B = sp.csc_matrix(B, dtype=np.float64)
        B.sort_indices()
        bptr = np.ascontiguousarray(B.indptr, dtype=np.int64)
        bidx = np.ascontiguousarray(B.indices, dtype=np.int32)
        bval = np.ascontiguousarray(B.data, dtype=np.float64)
    nb = n // bs
    lst = None
    if block_list is not None:
        lst = np.ascontiguousarray(block_list, dtype=np.int32)
        lo, hi = 0, len(lst)
    else:
        lo, hi = (0, nb) if blocks is None else blocks
    stride = bs * (int(np.diff(pptr).max()) + mn * ns) + 1
    out_len = np.zeros(n, dtype=np.int32)
    out_idx = np.zeros(n * stride, dtype=np.int32)
    out_val = np.zeros(n * stride, dtype=np.float64)
    out_res = np.zeros(n, dtype=np.float64)
    out_steps = np.zeros(n, dtype=np.int32)
    out_info = np.zeros(n, dtype=np.int32)
    rc = lib.oracle_spai_block(nrows, n, bs, _ptr(cptr), _ptr(cidx), _ptr(cval), _ptr(rptr),
                               _ptr(rcol), _ptr(bptr), _ptr(bidx), _ptr(bval), _ptr(pptr),
                               _ptr(pidx), float(ep), int(mn), int(ns), int(um), int(lo),
                               int(hi), stride, _ptr(out_len), _ptr(out_idx), _ptr(out_val),
                               _ptr(out_res), _ptr(out_steps), _ptr(out_info), _ptr(lst))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    lens = out_len.astype(np.int64)
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=colptr[1:])
    sel = (np.arange(stride)[None, :] < lens[:, None]).ravel()
    M = sp.csc_matrix((out_val[sel], out_idx[sel], colptr), shape=(n, n))
    return OracleResult(M, out_res, out_steps, out_info)


def block_pattern(A: sp.spmatrix, bs: int) -> sp.csc_matrix:
    """Block pattern of A for a constant block size: block (I, J) present when
    any scalar entry of A in it is stored (Matrix::Convert_Block_Matrix)."""
    C = sp.coo_matrix(A)
    nb = A.shape[1] // bs
    keep = C.row < nb * bs
    Pb = sp.coo_matrix((np.ones(int(keep.sum())), (C.row[keep] // bs, C.col[keep] // bs)),
                       shape=(nb, nb)).tocsc()
    Pb.sum_duplicates()
    Pb.data[:] = 1.0
    Pb.sort_indices()
    return Pb


def run_reference(args, cwd: str, timeout: float = 600.0) -> None:
    """Runs the compiled reference driver (oracle/_ref/ref_driver) with args."""
    if not os.path.exists(REF_DRIVER):
        raise FileNotFoundError(REF_DRIVER)
    subprocess.run([REF_DRIVER] + [str(a) for a in args], cwd=cwd, check=True,
                   timeout=timeout, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
