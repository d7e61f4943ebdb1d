"""Python interface of the B200 MSPAI setup.

It mirrors the reference's setup entry points: ``Options`` carries the
command-line options of the reference (src/Command_Line.cpp:192-225,
src/imspai.cpp:57-218) with the reference's checks; ``Handle.setup`` is
``Spai<double>::SPAI_Algorithm`` (src/Spai.imp:33-191) on plain CSC arrays;
``mspai`` is the serial command line ``mspai A P|-1|-2 B|-1 [options]``
(probing rows assembled as Read_mm_Matrix does, src/Read_mm_Matrix.cpp:115-420).

Matrices are scipy.sparse (host memory) or ``DeviceCSC`` (torch CUDA tensors,
already resident on the GPU).  All compute runs in the CUDA library; there is
no CPU path.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Tuple, Union

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, MspaiError, mspai_csc, mspai_params, mspai_stats


@dataclasses.dataclass
class Options:
    """Reference options (names and defaults of the reference's command line)."""
    ep: float = 0.4
    mn: int = 5
    ns: int = 5
    um: int = 1
    hs: int = 6
    cs: int = 0
    qr: int = 0
    ch: int = 0
    fg: float = 0.3
    pk: int = 0
    pm: int = 0
    schur: int = 0
    rho: float = 1.0
    bs: int = 1
    target: int = 1
    probing: int = 0
    prec: str = "mixed"        # "fp64" or "mixed"
    refine: int = 4
    batched: bool = True
    verbose: int = 0
    col_begin: int = 0         # solve only columns [col_begin, col_end) (0, 0: all)
    col_end: int = 0
    keep_factors: bool = False  # keep every column's R (adjoint's gbar term, re-setups)
    reuse_factors: int = 0      # > 0: re-setup from the kept factors, at most this many steps

    def to_c(self) -> mspai_params:
        p = mspai_params()
        _lib.load().mspai_default_params(ctypes.byref(p))
        for f in ("ep", "mn", "ns", "um", "hs", "cs", "qr", "ch", "fg", "pk", "pm", "schur",
                  "rho", "bs", "target", "probing", "refine", "verbose", "col_begin", "col_end"):
            setattr(p, f, getattr(self, f))
        p.keep_factors = 1 if self.keep_factors else 0
        p.reuse_factors = int(self.reuse_factors)
        p.prec = _lib.PREC_FP64 if self.prec == "fp64" else _lib.PREC_MIXED
        p.batched = 1 if self.batched else 0
        return p

    def validate(self) -> None:
        """Raises ValueError with the reference's message for invalid options."""
        buf = ctypes.create_string_buffer(1024)
        p = self.to_c()
        rc = _lib.load().mspai_validate_params(ctypes.byref(p), buf, len(buf))
        if rc != _lib.MSPAI_OK:
            raise ValueError(buf.value.decode())


class DeviceCSC:
    """A CSC matrix held in torch tensors (int64 colptr, int32 rowidx, float64
    values or None for a pattern): on the GPU (already resident in HBM) or in
    pinned host memory (copied by the library inside the setup)."""

    def __init__(self, nrows: int, ncols: int, colptr, rowidx, values=None):
        self.nrows, self.ncols = int(nrows), int(ncols)
        self.colptr, self.rowidx, self.values = colptr, rowidx, values

    @property
    def nnz(self) -> int:
        return int(self.rowidx.numel())

    @property
    def on_device(self) -> bool:
        return bool(self.colptr.is_cuda)

    @staticmethod
    def from_scipy(M: sp.spmatrix, device="cuda", pattern: bool = False,
                   pin: bool = False) -> "DeviceCSC":
        import torch

        def conv(a, dt):
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=dt))
            if str(device) == "cpu":
                return t.pin_memory() if pin else t
            return t.to(device)
        M = _canon(M)
        cp = conv(M.indptr, np.int64)
        ri = conv(M.indices, np.int32)
        v = None if pattern else conv(M.data, np.float64)
        return DeviceCSC(M.shape[0], M.shape[1], cp, ri, v)

    def nbytes(self) -> int:
        b = self.colptr.numel() * 8 + self.rowidx.numel() * 4
        return b + (self.values.numel() * 8 if self.values is not None else 0)


def _canon(M: sp.spmatrix) -> sp.csc_matrix:
    M = sp.csc_matrix(M)
    if not M.has_sorted_indices:
        M = M.copy()
        M.sort_indices()
    return M


class _Staged:
    """Keeps the numpy arrays behind a host mspai_csc alive."""

    def __init__(self, M, pattern: bool):
        if isinstance(M, DeviceCSC):
            self.keep = (M.colptr, M.rowidx, M.values)
            self.c = mspai_csc(M.nrows, M.ncols, M.nnz, M.colptr.data_ptr(), M.rowidx.data_ptr(),
                               None if (pattern or M.values is None) else M.values.data_ptr(),
                               MEM_DEVICE if M.on_device else MEM_HOST)
            return
        M = _canon(M)
        cp = np.ascontiguousarray(M.indptr, dtype=np.int64)
        ri = np.ascontiguousarray(M.indices, dtype=np.int32)
        vv = None if pattern else np.ascontiguousarray(M.data, dtype=np.float64)
        self.keep = (cp, ri, vv)
        self.c = mspai_csc(M.shape[0], M.shape[1], M.nnz, cp.ctypes.data, ri.ctypes.data,
                           None if vv is None else vv.ctypes.data, MEM_HOST)


MatrixLike = Union[sp.spmatrix, DeviceCSC]


class Handle:
    """One setup context on one GPU (wraps mspai_create / mspai_free)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self._lib.mspai_create(ctypes.byref(h), int(device), stream)
        if rc != _lib.MSPAI_OK:
            raise MspaiError(rc, "mspai_create failed (is a CUDA device visible?)")
        self._h = h
        self.n = 0

    def close(self) -> None:
        if self._h:
            self._lib.mspai_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != _lib.MSPAI_OK:
            msg = self._lib.mspai_last_error(self._h).decode(errors="replace")
            raise MspaiError(rc, msg)

    def setup(self, C: MatrixLike, P: MatrixLike, B: Optional[MatrixLike] = None,
              UP: Optional[MatrixLike] = None, C_rows: Optional[MatrixLike] = None,
              options: Optional[Options] = None) -> None:
        """Spai<double>::SPAI_Algorithm on CSC inputs (see mspai_setup)."""
        opts = options or Options()
        p = opts.to_c()
        sc = _Staged(C, False)
        sp_ = _Staged(P, True)
        sb = _Staged(B, False) if B is not None else None
        su = _Staged(UP, True) if UP is not None else None
        sr = _Staged(C_rows, True) if C_rows is not None else None
        rc = self._lib.mspai_setup(self._h, ctypes.byref(sc.c),
                                   ctypes.byref(sr.c) if sr else None,
                                   ctypes.byref(sb.c) if sb else None, ctypes.byref(sp_.c),
                                   ctypes.byref(su.c) if su else None, ctypes.byref(p))
        self._check(rc)
        self.n = sc.c.ncols

    def tune(self, C: MatrixLike, P: MatrixLike, B: Optional[MatrixLike] = None,
             UP: Optional[MatrixLike] = None, C_rows: Optional[MatrixLike] = None,
             options: Optional[Options] = None, sample_cols: int = 20000) -> int:
        """Picks the solver's shared-memory area per CTA (KB) by timing setups
        of a sample of columns (mspai_tune); later setups use it."""
        opts = options or Options()
        p = opts.to_c()
        sc = _Staged(C, False)
        sp_ = _Staged(P, True)
        sb = _Staged(B, False) if B is not None else None
        su = _Staged(UP, True) if UP is not None else None
        sr = _Staged(C_rows, True) if C_rows is not None else None
        kb = ctypes.c_int32()
        rc = self._lib.mspai_tune(self._h, ctypes.byref(sc.c), ctypes.byref(sr.c) if sr else None,
                                  ctypes.byref(sb.c) if sb else None, ctypes.byref(sp_.c),
                                  ctypes.byref(su.c) if su else None, ctypes.byref(p),
                                  int(sample_cols), ctypes.byref(kb))
        self._check(rc)
        return int(kb.value)

    def get_tuning(self) -> dict:
        """The handle's launch-shape knobs (mspai_get_tuning)."""
        t = _lib.mspai_tuning()
        self._check(self._lib.mspai_get_tuning(self._h, ctypes.byref(t)))
        return {f: int(getattr(t, f)) for f, _ in _lib.mspai_tuning._fields_}

    def set_tuning(self, **knobs) -> None:
        """Sets some of the knobs (mspai_set_tuning checks the ranges)."""
        t = _lib.mspai_tuning(**self.get_tuning())
        for k, v in knobs.items():
            if not hasattr(t, k):
                raise ValueError(f"unknown tuning knob {k}")
            setattr(t, k, int(v))
        self._check(self._lib.mspai_set_tuning(self._h, ctypes.byref(t)))

    def nnz(self) -> int:
        v = ctypes.c_int64()
        self._check(self._lib.mspai_result_nnz(self._h, ctypes.byref(v)))
        return int(v.value)

    def result(self) -> sp.csc_matrix:
        """M as a host scipy CSC matrix."""
        nnz = self.nnz()
        cp = np.zeros(self.n + 1, dtype=np.int64)
        ri = np.zeros(max(nnz, 1), dtype=np.int32)
        vv = np.zeros(max(nnz, 1), dtype=np.float64)
        self._check(self._lib.mspai_result_copy(self._h, cp.ctypes.data, ri.ctypes.data,
                                                vv.ctypes.data, MEM_HOST))
        return sp.csc_matrix((vv[:nnz], ri[:nnz], cp), shape=(self.n, self.n))

    def result_into(self, colptr=None, rowidx=None, values=None, device: bool = False) -> None:
        """Copies M into caller arrays (numpy, or torch CUDA tensors if device)."""
        def ptr(a):
            if a is None:
                return None
            return a.data_ptr() if device else a.ctypes.data
        self._check(self._lib.mspai_result_copy(self._h, ptr(colptr), ptr(rowidx), ptr(values),
                                                MEM_DEVICE if device else MEM_HOST))

    def apply(self, x):
        """y = M x with the last result (numpy in, numpy out; or a CUDA
        float64 torch tensor in, one out)."""
        try:
            import torch
            if isinstance(x, torch.Tensor) and x.is_cuda:
                xt = x.contiguous().to(torch.float64)
                y = torch.empty_like(xt)
                self._check(self._lib.mspai_apply(self._h, ctypes.c_void_p(xt.data_ptr()),
                                                  ctypes.c_void_p(y.data_ptr()), MEM_DEVICE))
                return y
        except ImportError:
            pass
        xa = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(xa)
        self._check(self._lib.mspai_apply(self._h, xa.ctypes.data, y.ctypes.data, MEM_HOST))
        return y

    def column_info(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        res = np.zeros(self.n, dtype=np.float64)
        steps = np.zeros(self.n, dtype=np.int32)
        status = np.zeros(self.n, dtype=np.int32)
        self._check(self._lib.mspai_column_info(self._h, res.ctypes.data, steps.ctypes.data,
                                                status.ctypes.data))
        return res, steps, status

    def stats(self) -> dict:
        s = mspai_stats()
        self._check(self._lib.mspai_get_stats(self._h, ctypes.byref(s)))
        return {
            "columns": s.columns, "ls_solves": s.ls_solves, "nnz_m": s.nnz_m,
            "singular_columns": s.singular_columns, "capacity_columns": s.capacity_columns,
            "bucket_columns": list(s.bucket_columns), "flops": s.flops,
            "flops_dense": s.flops_dense, "gather_bytes": s.gather_bytes,
            "setup_ms": s.setup_ms, "kernel_ms": list(s.kernel_ms),
            "kernel_launches": s.kernel_launches, "bucket_flops": list(s.bucket_flops),
            "reused_columns": s.reused_columns,
            "factor_reuse_columns": s.factor_reuse_columns,
        }

    def adjoint(self, C: MatrixLike, B: Optional[MatrixLike] = None,
                gbar: Optional[np.ndarray] = None, residual_weight: float = 1.0):
        """Gradient of w ||C M - B||_F^2 + gbar . M (w = residual_weight) with
        respect to the nonzeros of C and B, at the last setup's pattern.

        Returns (dC, dB, loss) as host arrays in C's / B's nonzero order."""
        sc = _Staged(C, False)
        sb = _Staged(B, False) if B is not None else None
        dC = np.zeros(max(sc.c.nnz, 1), dtype=np.float64)
        dB = np.zeros(max(sb.c.nnz, 1), dtype=np.float64) if sb else None
        g = None
        if gbar is not None:
            g = np.ascontiguousarray(gbar, dtype=np.float64)
            if g.size != self.nnz():
                raise ValueError(f"gbar has {g.size} values, M has {self.nnz()}")
        loss = ctypes.c_double()
        rc = self._lib.mspai_adjoint_weighted(self._h, ctypes.byref(sc.c),
                                              ctypes.byref(sb.c) if sb else None,
                                              None if g is None else g.ctypes.data,
                                              float(residual_weight), dC.ctypes.data,
                                              None if dB is None else dB.ctypes.data,
                                              ctypes.byref(loss), MEM_HOST)
        self._check(rc)
        return dC[:sc.c.nnz], (dB[:sb.c.nnz] if dB is not None else None), float(loss.value)

    def adjoint_device(self, C: "DeviceCSC", dC, B: Optional["DeviceCSC"] = None, dB=None,
                       gbar=None, residual_weight: float = 1.0) -> float:
        """mspai_adjoint_weighted with every value array in device memory: C and
        B on the GPU, dC / dB / gbar float64 CUDA tensors (dC: C's nnz
        values).  Returns the loss."""
        sc = _Staged(C, False)
        sb = _Staged(B, False) if B is not None else None
        loss = ctypes.c_double()
        rc = self._lib.mspai_adjoint_weighted(
            self._h, ctypes.byref(sc.c), ctypes.byref(sb.c) if sb else None,
            None if gbar is None else gbar.data_ptr(), float(residual_weight), dC.data_ptr(),
            None if dB is None else dB.data_ptr(), ctypes.byref(loss), MEM_DEVICE)
        self._check(rc)
        return float(loss.value)


def measure_fma_peak(device: int = 0, fp64: bool = False) -> float:
    """FP32 / FP64 CUDA-core FMA throughput in GFLOP/s (mspai_measure_fma_peak)."""
    v = ctypes.c_double()
    rc = _lib.load().mspai_measure_fma_peak(int(device), 1 if fp64 else 0, ctypes.byref(v))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, "FMA peak probe failed")
    return float(v.value)


def assemble_probing(A: sp.spmatrix, Ce: Optional[sp.spmatrix], Be: Optional[sp.spmatrix],
                     rho: float) -> Tuple[sp.csc_matrix, sp.csc_matrix]:
    """C = [A; rho Ce], B = [I; rho Be] (mspai_probing_assemble)."""
    lib = _lib.load()
    sa = _Staged(A, False)
    sce = _Staged(sp.csc_matrix(Ce), False) if Ce is not None else None
    sbe = _Staged(sp.csc_matrix(Be), False) if Be is not None else None
    Cm, Bm = _lib.mspai_matrix(), _lib.mspai_matrix()
    buf = ctypes.create_string_buffer(512)
    rc = lib.mspai_probing_assemble(ctypes.byref(sa.c), ctypes.byref(sce.c) if sce else None,
                                    ctypes.byref(sbe.c) if sbe else None, float(rho),
                                    ctypes.byref(Cm), ctypes.byref(Bm), buf, len(buf))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, buf.value.decode())
    try:
        return _owned_to_scipy(Cm), _owned_to_scipy(Bm)
    finally:
        lib.mspai_matrix_free(ctypes.byref(Cm))
        lib.mspai_matrix_free(ctypes.byref(Bm))


def _owned_to_scipy(m) -> sp.csc_matrix:
    n, nnz = m.ncols, m.nnz
    cp = np.ctypeslib.as_array(m.colptr, shape=(n + 1,)).copy()
    ri = np.ctypeslib.as_array(m.rowidx, shape=(max(nnz, 1),))[:nnz].copy()
    if m.values:
        vv = np.ctypeslib.as_array(m.values, shape=(max(nnz, 1),))[:nnz].copy()
    else:
        vv = np.ones(nnz)
    return sp.csc_matrix((vv, ri, cp), shape=(m.nrows, n))


def read_mm(path: str) -> sp.csc_matrix:
    """Matrix Market reader of the library (mspai_mm_read)."""
    lib = _lib.load()
    m = _lib.mspai_matrix()
    buf = ctypes.create_string_buffer(512)
    rc = lib.mspai_mm_read(path.encode(), ctypes.byref(m), buf, len(buf))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, buf.value.decode())
    try:
        return _owned_to_scipy(m)
    finally:
        lib.mspai_matrix_free(ctypes.byref(m))


def write_mm(path: str, M: sp.spmatrix) -> None:
    """Writes M in the reference's output format (mspai_mm_write)."""
    lib = _lib.load()
    s = _Staged(M, False)
    buf = ctypes.create_string_buffer(512)
    rc = lib.mspai_mm_write(path.encode(), ctypes.byref(s.c), buf, len(buf))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, buf.value.decode())


def start_pattern(C: sp.spmatrix, kind: Union[int, str]) -> sp.csc_matrix:
    """-1 / "diag": diagonal pattern; -2 / "A": pattern of C's first n rows."""
    k = {"diag": 1, -1: 1, 1: 1, "A": 2, -2: 2, 2: 2}[kind]
    lib = _lib.load()
    s = _Staged(C, False)
    m = _lib.mspai_matrix()
    rc = lib.mspai_pattern_generate(ctypes.byref(s.c), k, ctypes.byref(m))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, "pattern generation failed")
    try:
        return _owned_to_scipy(m)
    finally:
        lib.mspai_matrix_free(ctypes.byref(m))


def pattern_power2(C: sp.spmatrix, drop: float = 1e-3, device: int = 0) -> sp.csc_matrix:
    """Start pattern from A^2 on the GPU (mspai_pattern_power2): per column the
    rows i with |(A^2)(i,k)| >= drop * max_i |(A^2)(i,k)|."""
    lib = _lib.load()
    s = _Staged(C, False)
    m = _lib.mspai_matrix()
    buf = ctypes.create_string_buffer(512)
    rc = lib.mspai_pattern_power2(ctypes.byref(s.c), float(drop), int(device), ctypes.byref(m),
                                  buf, len(buf))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, buf.value.decode(errors="replace"))
    try:
        return _owned_to_scipy(m)
    finally:
        lib.mspai_matrix_free(ctypes.byref(m))


def pattern_powers(A: sp.spmatrix, nb_pw: int = 1, device: int = 0) -> sp.csc_matrix:
    """The reference's power pattern with its count-based Sparsify
    (mspai_pattern_powers, To_Pattern_Powers): a CSC matrix whose pattern is
    P and whose values are the magnitudes of the sparsified powers."""
    lib = _lib.load()
    s = _Staged(A, False)
    m = _lib.mspai_matrix()
    buf = ctypes.create_string_buffer(512)
    rc = lib.mspai_pattern_powers(ctypes.byref(s.c), int(nb_pw), int(device), ctypes.byref(m),
                                  buf, len(buf))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, buf.value.decode(errors="replace"))
    try:
        return _owned_to_scipy(m)
    finally:
        lib.mspai_matrix_free(ctypes.byref(m))


def block_pattern(C: sp.spmatrix, bs: int, kind: Union[int, str]) -> sp.csc_matrix:
    """Block start pattern (n/bs x n/bs): -1 / "diag" diagonal blocks, -2 / "A"
    the block pattern of C's first n rows (mspai_block_pattern_generate)."""
    k = {"diag": 1, -1: 1, 1: 1, "A": 2, -2: 2, 2: 2}[kind]
    lib = _lib.load()
    s = _Staged(C, False)
    m = _lib.mspai_matrix()
    rc = lib.mspai_block_pattern_generate(ctypes.byref(s.c), int(bs), k, ctypes.byref(m))
    if rc != _lib.MSPAI_OK:
        raise MspaiError(rc, "block pattern generation failed")
    try:
        return _owned_to_scipy(m)
    finally:
        lib.mspai_matrix_free(ctypes.byref(m))


def mspai(A: sp.spmatrix, pattern: Union[int, str, sp.spmatrix] = -1,
          target: Optional[sp.spmatrix] = None, Ce: Optional[sp.spmatrix] = None,
          Be: Optional[sp.spmatrix] = None, UP: Optional[sp.spmatrix] = None,
          options: Optional[Options] = None, device: int = 0):
    """The serial command line as a function: returns (M, handle)."""
    opts = dataclasses.replace(options or Options())
    opts.probing = 1 if (Ce is not None or Be is not None) else 0
    opts.target = 1 if target is None else 0
    opts.validate()
    C, B = assemble_probing(A, Ce, Be, opts.rho)
    Bin = B if opts.probing else None
    if target is not None:
        Bin = target
    if sp.issparse(pattern):
        P = pattern
    elif opts.bs > 1:
        P = block_pattern(C, opts.bs, pattern)
    else:
        P = start_pattern(C, pattern)
    h = Handle(device)
    h.setup(C, P, B=Bin, UP=UP, options=opts)
    return h.result(), h
