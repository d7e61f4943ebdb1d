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
