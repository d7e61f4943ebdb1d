"""Block SPAI on the GPU (-bs 3): the bs scalar columns of a block column share
J, I and one QR with bs right-hand sides; the residual is a Frobenius norm
against ep * sqrt(bs); block candidates use rho_j^2 = ||R||^2 -
<N, (A_j^T A_j)^-1 N>.  Checked against the reference's block path (golden
fixtures) and, for the probing extension the reference does not support,
against the oracle's block restatement."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from conftest import load_golden
from helpers import max_rel_diff, same_pattern
from mspai_b200 import workloads as W
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}
PRINT_TOL = 5e-12


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name,kind,kw", [
    ("block27_6", -2, dict(ns=0)),
    ("block27_6_upd", -1, dict(ns=3, mn=3, ep=0.05)),
])
def test_block_against_reference(h, prec, name, kind, kw):
    w = W.block27(6, probing=False)
    Pb = mb.block_pattern(w.A, 3, kind)
    h.setup(w.A, Pb, options=mb.Options(bs=3, prec=prec, **kw))
    M = h.result()
    ref = load_golden(name)
    assert same_pattern(M, ref)
    assert max_rel_diff(M, ref) < max(TOL[prec], PRINT_TOL)
    _, steps, status = h.column_info()
    assert np.all(status == 0)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_block_probing_fixed(h, prec):
    """Block SPAI with a probing row e = ones, rho = 10 (fixed block pattern):
    C = [A; rho e^T A], B = [I; rho e^T]; the reference supports no probing in
    block mode, so the oracle's block restatement is the check."""
    rho = 10.0
    w = W.block27(4, rho=rho, probing=True)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    Pb = mb.block_pattern(C, 3, -2)
    h.setup(C, Pb, B=B, options=mb.Options(bs=3, ns=0, prec=prec, probing=1, rho=rho))
    M = h.result()
    o = O.spai_block(C, sp.csc_matrix(Pb), 3, B=B, ns=0)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_block_probing_with_updates(h, prec):
    """Block pattern updates together with the probing row and target (the
    block workload's combination; an extension of the reference, which allows
    probing only without updates).  The option check is the reference's, so
    the extension is requested by passing the probing rows with probing = 0."""
    rho = 10.0
    w = W.block27(4, rho=rho, probing=True)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    Pb = mb.block_pattern(C, 3, -1)
    h.setup(C, Pb, B=B, options=mb.Options(bs=3, ns=3, mn=3, ep=0.05, prec=prec))
    M = h.result()
    o = O.spai_block(C, sp.csc_matrix(Pb), 3, B=B, ns=3, mn=3, ep=0.05)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < TOL[prec]


def test_block_updates_with_target_rows(h):
    """Pattern updates with probing rows present in C (rows >= n carry no row
    structure): the GPU kernel supports it; the oracle agrees."""
    rho = 10.0
    w = W.block27(4, rho=rho, probing=True)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    Pb = mb.block_pattern(C, 3, -1)
    opts = mb.Options(bs=3, ns=3, mn=3, ep=0.05, prec="fp64")
    h.setup(C, Pb, options=opts)
    M = h.result()
    o = O.spai_block(C, sp.csc_matrix(Pb), 3, ns=3, mn=3, ep=0.05)
    assert same_pattern(M, o.M)
    assert max_rel_diff(M, o.M) < TOL["fp64"]


def _block_stencil(nx, bs, seed):
    """A 2-D 5-point block stencil on an nx x nx grid, random bs x bs blocks
    per node (diagonal Q Q^T + 2 bs I, off-diagonal -R / 4)."""
    rng = np.random.default_rng(seed)
    nn = nx * nx
    rows, cols, vals = [], [], []
    for node in range(nn):
        x, y = node % nx, node // nx
        Q = rng.standard_normal((bs, bs))
        blocks = [(node, Q @ Q.T + 2.0 * bs * np.eye(bs))]
        for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
            if 0 <= x + dx < nx and 0 <= y + dy < nx:
                blocks.append((node + dx + dy * nx, -0.25 * rng.standard_normal((bs, bs))))
        for nb, Bk in blocks:
            for i in range(bs):
                for j in range(bs):
                    rows.append(bs * nb + i)
                    cols.append(bs * node + j)
                    vals.append(Bk[i, j])
    A = sp.csc_matrix((vals, (rows, cols)), shape=(bs * nn, bs * nn))
    A.sort_indices()
    return A


@pytest.mark.parametrize("bs", [5, 6, 8])
@pytest.mark.parametrize("kind,kw,args", [
    (-2, dict(ns=0), ["-2", "-1", "-ns", "0"]),
    (-1, dict(ns=2, mn=2, ep=0.05), ["-1", "-1", "-ns", "2", "-mn", "2", "-ep", "0.05"]),
])
def test_block_sizes_up_to_8_against_reference(h, tmp_path, bs, kind, kw, args):
    """Constant block sizes 5, 6 and 8: the GPU's M equals the reference's
    own block run (oracle/_ref/ref_driver -bs k) in FP64 to 1e-10 per entry
    (the reference prints 14 digits)."""
    import os
    import subprocess
    from fullsize import REF_DRIVER, read_mm, write_mm
    if not os.path.exists(REF_DRIVER):
        pytest.skip("oracle/_ref/ref_driver was not built")
    A = _block_stencil(6, bs, seed=bs)
    write_mm(str(tmp_path / "A.mtx"), A)
    r = subprocess.run([REF_DRIVER, "A.mtx"] + args + ["-bs", str(bs), "-out", "ref.mtx"],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-1000:]
    ref = read_mm(str(tmp_path / "ref.mtx"))
    Pb = mb.block_pattern(A, bs, kind)
    h.setup(A, Pb, options=mb.Options(bs=bs, prec="fp64", **kw))
    M = h.result()
    _, steps, status = h.column_info()
    assert np.all(status == 0)
    assert same_pattern(M, ref)
    assert max_rel_diff(M, ref) < max(TOL["fp64"], PRINT_TOL)
    if kind == -1:
        assert steps.max() > 1  # the block patterns grew


def test_block_size_above_8_refused(h):
    A = sp.identity(90, format="csc")
    with pytest.raises(mb.MspaiError, match="block size"):
        h.setup(A, sp.identity(10, format="csc"), options=mb.Options(bs=9, ns=0))
