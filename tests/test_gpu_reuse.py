"""GPU reuse table (`-cs` cache size, `-ch` hashing; the reference's
Spai_Caching / Spai_Hashing, src/Spai_Caching.imp:45-332): columns whose
least-squares problems are identical take one solution.  Reuse changes no
value of M: every case is compared bit for bit with the same setup without
reuse, and against the reference's fixtures / the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from conftest import load_golden
from helpers import max_rel_diff, same_pattern
from mspai_b200 import workloads as W
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def run(h, C, P, B=None, **kw):
    h.setup(C, P, B=B, options=mb.Options(**kw))
    M = h.result()
    res, steps, status = h.column_info()
    return M, res.copy(), steps.copy(), status.copy(), h.stats()


def bit_equal(A, B):
    A = sp.csc_matrix(A); B = sp.csc_matrix(B)
    return (same_pattern(A, B)
            and np.array_equal(A.data.view(np.uint64), B.data.view(np.uint64)))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("opt", [dict(ch=1), dict(cs=1000), dict(cs=3)])
def test_poisson_reuse_is_bit_identical(h, prec, opt):
    w = W.poisson2d(64)
    M0, r0, s0, st0, _ = run(h, w.A, w.P, ns=0, prec=prec)
    M1, r1, s1, st1, stats = run(h, w.A, w.P, ns=0, prec=prec, **opt)
    assert bit_equal(M1, M0)
    assert np.array_equal(r1, r0) and np.array_equal(s1, s0) and np.array_equal(st1, st0)
    # the 60 x 60 interior columns of the constant-coefficient stencil share
    # one problem, so do the columns along each edge; with a 3-entry cache
    # which problems are stored depends on the order of insertion
    if opt.get("cs", 10 ** 9) >= 1000:
        assert stats["reused_columns"] >= 3599
    else:
        assert stats["reused_columns"] > 0
    ref = load_golden("poisson2d_64")
    assert same_pattern(M1, ref)
    assert max_rel_diff(M1, ref) < (1e-10 if prec == "fp64" else 1e-8)


@pytest.mark.parametrize("kinds", [("ones",), ("ones", "alt")])
def test_probing_target_reuse(h, kinds):
    """Probing rows are absolute (they do not move with k): columns reuse only
    when the probing values and B's probing entries agree too."""
    rho = 10.0
    w = W.aniso2d_probing(32, kinds=kinds, rho=rho)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    M0, r0, _, _, _ = run(h, C, w.P, B=B, ns=0, probing=1, rho=rho)
    M1, r1, _, _, stats = run(h, C, w.P, B=B, ns=0, probing=1, rho=rho, ch=1)
    assert bit_equal(M1, M0) and np.array_equal(r1, r0)
    assert stats["reused_columns"] > 0
    o = O.spai_scalar(C, w.P, B=B, ns=0)
    assert same_pattern(M1, o.M) and max_rel_diff(M1, o.M) < 1e-8


def test_random_matrix_has_no_reuse(h):
    w = W.ragged(3000)
    M0, r0, _, _, _ = run(h, w.A, w.P, ns=0)
    M1, r1, _, _, stats = run(h, w.A, w.P, ns=0, cs=100000)
    assert stats["reused_columns"] == 0
    assert bit_equal(M1, M0) and np.array_equal(r1, r0)


def test_adaptive_and_block_setups_ignore_the_table(h):
    w = W.convdiff3d(6)
    M0, r0, _, _, _ = run(h, w.A, w.P, ep=0.4, ns=5, mn=5)
    M1, r1, _, _, stats = run(h, w.A, w.P, ep=0.4, ns=5, mn=5, ch=1)
    assert stats["reused_columns"] == 0
    assert bit_equal(M1, M0) and np.array_equal(r1, r0)


@pytest.mark.parametrize("bs", [2, 3])
@pytest.mark.parametrize("opt", [dict(ch=1), dict(cs=50)])
def test_block_problems_reuse(h, bs, opt):
    """Fixed block patterns: a constant-coefficient block stencil (the same
    bs x bs blocks at every node of a 14 x 14 grid) has many identical block
    problems; the block columns that take a representative's solution (its
    values, its rows shifted by its block offset) give the M of the setup
    without reuse, bit for bit."""
    rng = np.random.default_rng(40 + bs)
    Q = rng.standard_normal((bs, bs))
    D = Q @ Q.T + 4.0 * np.eye(bs)
    R = rng.standard_normal((bs, bs))
    T = sp.diags([1.0, 1.0], [-1, 1], shape=(14, 14))
    G = sp.kron(sp.identity(14), T) + sp.kron(T, sp.identity(14))
    A = sp.csc_matrix(sp.kron(sp.identity(196), D) - 0.2 * sp.kron(G, R))
    A.sort_indices()
    P = mb.block_pattern(A, bs, "A")
    M0, r0, s0, st0, _ = run(h, A, P, ns=0, bs=bs, prec="fp64")
    M1, r1, s1, st1, stats = run(h, A, P, ns=0, bs=bs, prec="fp64", **opt)
    assert bit_equal(M1, M0)
    assert np.array_equal(r1.view(np.uint64), r0.view(np.uint64))
    assert np.array_equal(st1, st0) and np.all(st1 == 0)
    assert stats["reused_columns"] >= 100  # the interior nodes share one problem
