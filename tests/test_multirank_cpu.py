"""The multi-rank path of bench.py on CPU (gloo, world size 2, 127.0.0.1).

The setup shards by columns: each rank solves its own block of columns (weak
scaling), so the only cross-rank steps are the barriers around the timed
region and the max over ranks of the step time.  These run here with the
gloo backend; the reference arm must print from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from mspai_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms, value = bench.whole_job_rate(1000, 100.0 + 50.0 * rank, world)
        w = W.ragged(300, seed=bench.rank_seed(rank))
        out[rank] = (ms, value, float(np.abs(w.A.data).sum()))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        r = dict(out)
    assert set(r) == {0, 1}
    # every rank sees the slowest rank's time and the whole-job rate
    for rank in (0, 1):
        assert r[rank][0] == 150.0
        assert r[rank][1] == pytest.approx(2 * 1000 / 0.150)
    # the ranks' column blocks differ (distinct seeds)
    assert r[0][2] != r[1][2]


def _shard_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from mspai_b200 import distributed as D
    from mspai_b200 import workloads as W
    from oracle import pyoracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        w = W.convdiff3d(6)
        lo, hi = D.shard_range(w.A, w.P, rank, world)
        # the oracle stands in for this rank's GPU solve of its columns
        part = O.spai_scalar(w.A, w.P, ep=0.4, ns=5, mn=5, cols=(lo, hi)).M
        M = D.gather_pieces(D.local_piece(part, lo, hi), w.A.shape[1])
        out[rank] = (lo, hi, M.indptr.copy(), M.indices.copy(), M.data.copy())
    finally:
        dist.destroy_process_group()


def test_sharded_columns_gather_to_the_full_setup():
    """Each of two gloo ranks solves its work-balanced column range and the
    pieces are all-gathered: every rank ends with the whole M."""
    sys.path.insert(0, ROOT)
    from mspai_b200 import workloads as W
    from oracle import pyoracle as O
    world = 2
    port = free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_shard_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        r = dict(out)
    w = W.convdiff3d(6)
    full = O.spai_scalar(w.A, w.P, ep=0.4, ns=5, mn=5).M
    assert r[0][1] == r[1][0] and r[0][0] == 0 and r[1][1] == w.A.shape[1]
    for rank in (0, 1):
        _, _, ip, ix, dv = r[rank]
        assert np.array_equal(ip, full.indptr) and np.array_equal(ix, full.indices)
        assert np.array_equal(dv, full.data)


def test_balanced_ranges():
    sys.path.insert(0, ROOT)
    from mspai_b200 import distributed as D
    from mspai_b200 import workloads as W
    w = W.ragged(3000)
    work = D.column_work(w.A, w.P)
    for world in (1, 2, 3, 8):
        rs = D.balanced_ranges(work, world)
        assert rs[0][0] == 0 and rs[-1][1] == len(work)
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        loads = [work[lo:hi].sum() for lo, hi in rs]
        assert max(loads) - min(loads) <= 2 * work.max() + 1e-9
    # a single heavy column: the other ranges may be empty, none overlaps
    rs = D.balanced_ranges([1.0, 1e9, 1.0], 4)
    assert rs[0][0] == 0 and rs[-1][1] == 3 and sum(hi - lo for lo, hi in rs) == 3


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver")),
                    reason="the reference driver is built from the reference sources")
def test_reference_arm_prints_from_rank_zero_only():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node",
           "2", "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--columns",
           "2000"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def _gather_worker(rank, world, port, out):
    import datetime
    import numpy as np
    import scipy.sparse as sp
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from mspai_b200 import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(42)
        n = 300
        M = sp.random(n, n, density=0.03, format="csc", random_state=7)
        M = (M + sp.identity(n)).tocsc()
        M.sort_indices()
        C = sp.random(n + 2, n, density=0.05, format="csc", random_state=8)
        C = (C + sp.identity(n + 2, format="csc")[:, :n]).tocsc()
        # work and ranges on the "device" (CPU tensors here) equal the host's
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt))
        wdev = D.column_work_device(t(C.indptr, np.int64), t(M.indptr, np.int64),
                                    t(M.indices, np.int32))
        whost = D.column_work(C, M)
        ranges = D.balanced_ranges_device(wdev, world)
        ok_work = bool(np.allclose(wdev.numpy(), whost, rtol=1e-12))
        ok_ranges = ranges == D.balanced_ranges(whost, world)
        lo, hi = ranges[rank]
        # compact result: only this rank's columns are non-empty
        lens = np.diff(M.indptr).copy()
        mask = np.zeros(n, dtype=bool)
        mask[lo:hi] = True
        lens[~mask] = 0
        cp = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(lens, out=cp[1:])
        keep = np.repeat(mask, np.diff(M.indptr))
        ri = M.indices[keep]
        vv = M.data[keep]
        gc, gr, gv = D.gather_csc_device(t(cp, np.int64), t(ri, np.int32), t(vv, np.float64),
                                         ranges, rank)
        G = sp.csc_matrix((gv.numpy(), gr.numpy(), gc.numpy()), shape=(n, n))
        ok_compact = bool((G != M).nnz == 0 and np.array_equal(G.indptr, M.indptr))
        # known structure: values in M's structure, zeros outside the range
        vk = np.where(keep, M.data, 0.0)
        kc, kr, kv = D.gather_csc_device(t(M.indptr, np.int64), None, t(vk, np.float64), ranges,
                                         rank, known_structure=(t(M.indptr, np.int64),
                                                                t(M.indices, np.int32)))
        ok_known = bool(np.array_equal(kv.numpy(), M.data))
        out[rank] = (ok_work, ok_ranges, ok_compact, ok_known, ranges)
    finally:
        dist.destroy_process_group()


def test_device_gather_two_ranks_gloo():
    """The device form of the sharded setup's gather (all_reduce of column
    lengths, padded all_gather of indices and values), on CPU tensors with
    gloo: every rank assembles the whole M; the device work estimate and
    ranges equal the host ones."""
    world = 2
    port = free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_gather_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        r = dict(out)
    assert set(r) == {0, 1}
    for rank in (0, 1):
        ok_work, ok_ranges, ok_compact, ok_known, ranges = r[rank]
        assert ok_work and ok_ranges and ok_compact and ok_known
    assert r[0][4][0][1] == r[0][4][1][0] and r[0][4][1][1] == 300
