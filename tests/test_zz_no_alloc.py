"""The setup entry point that allocates nothing (mspai_setup_fixed_noalloc).

It exists for callers that cannot call cudaMalloc when they need the
preconditioner -- an application whose GPU memory is owned by its own pool or
by another framework, or a latency-critical path that must not pay for
allocation -- and keeps its scratch in a fixed array inside the library.  This
file checks, through the C ABI, that two consecutive calls give the same M as
the allocating entry point (mspai_setup) within the parity tolerances, and
that inputs beyond its documented limits are refused with a clear error.  It
is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from mspai_b200 import _lib, workloads as W
from mspai_b200.api import _Staged

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}


def noalloc(C, P, B, opts, torch):
    """Calls mspai_setup_fixed_noalloc with device-resident inputs/outputs."""
    lib = _lib.load()
    dC = mb.DeviceCSC.from_scipy(C)
    dP = mb.DeviceCSC.from_scipy(P, pattern=True)
    dB = mb.DeviceCSC.from_scipy(B) if B is not None else None
    sc, spp = _Staged(dC, False), _Staged(dP, True)
    sb = _Staged(dB, False) if dB is not None else None
    n = C.shape[1]
    vals = torch.zeros(max(P.nnz, 1), dtype=torch.float64, device="cuda")
    res = torch.zeros(n, dtype=torch.float64, device="cuda")
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    p = opts.to_c()
    msg = ctypes.create_string_buffer(512)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.mspai_setup_fixed_noalloc(ctypes.byref(sc.c), ctypes.byref(sb.c) if sb else None,
                                       ctypes.byref(spp.c), ctypes.byref(p), vals.data_ptr(),
                                       res.data_ptr(), status.data_ptr(), stream, msg, len(msg))
    torch.cuda.synchronize()
    return rc, msg.value.decode(), vals[:P.nnz].cpu().numpy(), res.cpu().numpy(), \
        status.cpu().numpy()


def with_values(P, values):
    P = sp.csc_matrix(P)
    P.sort_indices()
    return sp.csc_matrix((values, P.indices, P.indptr), shape=P.shape)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["poisson", "probing"])
def test_matches_allocating_entry_point_twice(case, prec):
    torch = pytest.importorskip("torch")
    if case == "poisson":
        w = W.poisson2d(32)
        C, B, opts = w.A, None, mb.Options(ns=0, prec=prec)
    else:
        w = W.aniso2d_probing(24, kinds=("ones", "alt"), rho=10.0)
        C, B = mb.assemble_probing(w.A, w.Ce, w.Be, 10.0)
        opts = mb.Options(ns=0, prec=prec, probing=1, rho=10.0)
    h = mb.Handle(0)
    h.setup(C, w.P, B=B, options=opts)
    ref = h.result()
    ref_res, _, _ = h.column_info()
    h.close()
    scale = np.max(np.abs(ref.data))
    for _ in range(2):  # two calls in a row share the scratch array
        rc, msg, vals, res, status = noalloc(C, w.P, B, opts, torch)
        assert rc == 0, msg
        M = with_values(w.P, vals)
        diff = M - ref
        if diff.nnz:
            assert np.max(np.abs(diff.data)) <= TOL[prec] * scale
        assert np.all(status == 0)
        assert np.allclose(res, ref_res, rtol=1e-8, atol=1e-14)


def test_refuses_columns_beyond_limits():
    torch = pytest.importorskip("torch")
    w = W.ragged(2000)
    rc, msg, *_ = noalloc(w.A, w.P, None, mb.Options(ns=0, prec="mixed"), torch)
    assert rc == 4, msg  # MSPAI_ERR_CAPACITY
    assert "no-allocation limits" in msg


def test_refuses_malformed_pattern_before_indexing():
    """A row index of P outside [0, n) is reported as an input error by the
    structure check, which runs before any kernel indexes with P."""
    torch = pytest.importorskip("torch")
    w = W.poisson2d(8)
    n = w.A.shape[1]
    P = sp.csc_matrix(w.P)
    P.sort_indices()
    rows = P.indices.astype(np.int32).copy()
    rows[P.indptr[3 + 1] - 1] = n + 5  # last row of column 3, out of range (still sorted)
    lib = _lib.load()
    dC = mb.DeviceCSC.from_scipy(w.A)
    dP = mb.DeviceCSC(n, n, torch.from_numpy(P.indptr.astype(np.int64)).cuda(),
                      torch.from_numpy(rows).cuda(), None)
    sc, spp = _Staged(dC, False), _Staged(dP, True)
    vals = torch.zeros(P.nnz, dtype=torch.float64, device="cuda")
    res = torch.zeros(n, dtype=torch.float64, device="cuda")
    status = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = mb.Options(ns=0, prec="mixed").to_c()
    msg = ctypes.create_string_buffer(512)
    rc = lib.mspai_setup_fixed_noalloc(ctypes.byref(sc.c), None, ctypes.byref(spp.c),
                                       ctypes.byref(p), vals.data_ptr(), res.data_ptr(),
                                       status.data_ptr(), torch.cuda.current_stream().cuda_stream,
                                       msg, len(msg))
    torch.cuda.synchronize()
    assert rc == 2, msg.value  # MSPAI_ERR_INPUT
    assert "P: row index" in msg.value.decode() and "column 3" in msg.value.decode()
