"""Column ranges of mspai_setup (col_begin, col_end), the unit of the
multi-GPU sharding (mspai_b200.distributed): the pieces of M solved range by
range make the full M, and the adjoints of the ranges sum to the full
adjoint.  Ranges may land columns in other size buckets than the full setup
does, so values agree within the FP64 tolerance (1e-10 relative)."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import max_rel_diff, same_pattern
from mspai_b200 import distributed as D
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


@pytest.mark.parametrize("case", ["ragged", "convdiff"])
def test_ranges_make_the_full_setup(h, case):
    if case == "ragged":
        w = W.ragged(3000)
        opts = dict(ns=0, prec="fp64")
    else:
        w = W.convdiff3d(8)
        opts = dict(ep=0.4, ns=5, mn=5, prec="fp64")
    n = w.A.shape[1]
    h.setup(w.A, w.P, options=mb.Options(**opts))
    full = h.result()
    res_full, steps_full, _ = h.column_info()
    pieces = []
    ranges = D.balanced_ranges(D.column_work(w.A, w.P), 3)
    for lo, hi in ranges:
        h.setup(w.A, w.P, options=mb.Options(col_begin=lo, col_end=hi, **opts))
        M = h.result()
        res, steps, _ = h.column_info()
        assert np.all(steps[:lo] == 0) and np.all(steps[hi:] == 0)
        assert np.array_equal(steps[lo:hi], steps_full[lo:hi])
        assert np.allclose(res[lo:hi], res_full[lo:hi], rtol=1e-10, atol=1e-14)
        assert h.stats()["columns"] == hi - lo
        pieces.append(D.local_piece(M, lo, hi))
    M = D.assemble(pieces, n)
    assert same_pattern(M, full)
    assert max_rel_diff(M, full) < 1e-10


def test_range_adjoints_sum_to_the_full_adjoint(h):
    w = W.aniso2d_probing(24, kinds=("ones", "alt"), rho=10.0)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, 10.0)
    opts = dict(ns=0, prec="fp64", probing=1, rho=10.0)
    h.setup(C, w.P, B=B, options=mb.Options(**opts))
    dC, dB, L = h.adjoint(C, B)
    n = w.A.shape[1]
    sc, sb, sl = np.zeros_like(dC), np.zeros_like(dB), 0.0
    for lo, hi in ((0, n // 3), (n // 3, n)):
        h.setup(C, w.P, B=B, options=mb.Options(col_begin=lo, col_end=hi, **opts))
        a, b, l = h.adjoint(C, B)
        sc += a
        sb += b
        sl += l
    assert np.allclose(sc, dC, rtol=1e-9, atol=1e-12 * np.abs(dC).max())
    assert np.allclose(sb, dB, rtol=1e-9, atol=1e-12 * np.abs(dB).max())
    assert sl == pytest.approx(L, rel=1e-12)


def test_invalid_range_is_rejected(h):
    w = W.poisson2d(8)
    with pytest.raises(mb.MspaiError, match="range"):
        h.setup(w.A, w.P, options=mb.Options(ns=0, col_begin=10, col_end=5))


def test_tuner_picks_a_candidate_and_keeps_results(h):
    """mspai_tune times column samples under each shared-memory area and keeps
    the fastest; setups after it give the same M (FP64 tolerance)."""
    w = W.ragged(20000)
    h.setup(w.A, w.P, options=mb.Options(ns=0, prec="fp64"))
    before = h.result()
    kb = h.tune(w.A, w.P, options=mb.Options(ns=0, prec="fp64"), sample_cols=4000)
    assert kb in (48, 32, 24)
    with pytest.raises(mb.MspaiError, match="result"):
        h.result()  # the sample runs leave no result
    h.setup(w.A, w.P, options=mb.Options(ns=0, prec="fp64"))
    after = h.result()
    assert same_pattern(after, before) and max_rel_diff(after, before) < 1e-10


@pytest.mark.parametrize("case", ["ragged", "convdiff"])
def test_device_sharded_setup_nccl_one_rank(h, case):
    """sharded_setup_device through a one-rank NCCL group: ranges computed on
    the device, M assembled in HBM by the NCCL collectives, equal to the
    whole setup (fixed pattern: values only; adaptive: lengths, indices and
    values)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    if case == "ragged":
        w = W.ragged(3000)
        opts = dict(ns=0, prec="mixed")
    else:
        w = W.convdiff3d(8)
        opts = dict(ep=0.4, ns=5, mn=5, prec="mixed")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        dA = mb.DeviceCSC.from_scipy(w.A)
        dP = mb.DeviceCSC.from_scipy(w.P, pattern=True)
        M = D.sharded_setup_device(h, dA, dP, options=mb.Options(**opts))
        got = sp.csc_matrix((M.values.cpu().numpy(), M.rowidx.cpu().numpy(),
                                    M.colptr.cpu().numpy()), shape=(w.n, w.n))
        h.setup(w.A, w.P, options=mb.Options(**opts))
        ref = h.result()
        assert same_pattern(got, ref)
        assert max_rel_diff(got, ref) == 0.0
        # the adjoint's device form: gradients summed by NCCL
        h.setup(dA, dP, options=mb.Options(**opts))
        dC = torch.empty(w.A.nnz, dtype=torch.float64, device="cuda")
        L = D.sharded_adjoint_device(h, dA, dC)
        g, _, L2 = h.adjoint(w.A)
        assert L == pytest.approx(L2, rel=1e-12)
        assert np.max(np.abs(dC.cpu().numpy() - g)) <= 1e-12 * np.max(np.abs(g))
    finally:
        dist.destroy_process_group()
