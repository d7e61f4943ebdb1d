"""The workloads at their full sizes (C1..C5 of the benchmark description),
checked through properties that hold at any size, since the oracle would take
hours there:
  C2 convection-diffusion 48^3 (110,592 columns), adaptive: mixed and FP64
     choose the same patterns; residual norms agree to 1e-8.
  C3 ragged random, 200,000 columns (the bench runs 1,000,000), fixed
     pattern: ||AM - I||_F of mixed equals FP64's to 1e-8, values to 1e-8.
  C4 anisotropic 1024^2 (1,048,576 columns) with two probing rows, rho = 10:
     mixed equals FP64 to 1e-8; the adjoint's dL/drho equals the closed form
     2 sum_k s_k^2 / rho (s the probing-row residuals) to 1e-9, and its loss
     equals ||CM - B||_F^2.
  C5 27-point block stencil 40^3 x 3 (64,000 block columns), -bs 3 -ns 3
     -mn 3 -ep 0.05: mixed and FP64 choose the same block patterns.
Columns whose setup status is not OK fail every case."""
import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from helpers import column_residuals, max_rel_diff, same_pattern
from mspai_b200 import workloads as W

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
    assert np.all(status == 0)
    return M, res.copy(), steps.copy()


def test_c2_convdiff_48_adaptive(h):
    w = W.convdiff3d(48)
    opts = dict(ep=0.4, ns=5, mn=5, um=1)
    M64, r64, s64 = run(h, w.A, w.P, prec="fp64", **opts)
    M32, r32, s32 = run(h, w.A, w.P, prec="mixed", **opts)
    assert w.A.shape[1] == 110592
    assert same_pattern(M32, M64) and np.array_equal(s32, s64)
    assert np.allclose(r32, r64, rtol=1e-8, atol=1e-14)
    assert max_rel_diff(M32, M64) < 1e-8


def test_c3_ragged_200k_fixed(h):
    w = W.ragged(200000)
    M64, r64, _ = run(h, w.A, w.P, ns=0, prec="fp64")
    M32, r32, _ = run(h, w.A, w.P, ns=0, prec="mixed")
    f64, f32 = np.linalg.norm(r64), np.linalg.norm(r32)
    assert abs(f32 - f64) <= 1e-8 * f64
    assert max_rel_diff(M32, M64) < 1e-8


def test_c4_aniso_1024_probing_and_adjoint(h):
    rho = 10.0
    w = W.aniso2d_probing(1024, kinds=("ones", "alt"), rho=rho)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, rho)
    opts = dict(ns=0, probing=1, rho=rho)
    M32, _, _ = run(h, C, w.P, B=B, prec="mixed", **opts)
    M64, _, _ = run(h, C, w.P, B=B, prec="fp64", **opts)
    assert w.A.shape[1] == 1048576
    assert max_rel_diff(M32, M64) < 1e-8
    dC, dB, L = h.adjoint(C, B)
    n = w.A.shape[1]
    Cc, Bc = sp.csc_matrix(C), sp.csc_matrix(B)
    pc, pb = Cc.indices >= n, Bc.indices >= n
    g = (np.dot(dC[pc], Cc.data[pc]) + np.dot(dB[pb], Bc.data[pb])) / rho
    R = (C @ M64 - B).tocsr()
    s2 = R[n:, :].multiply(R[n:, :]).sum()
    assert abs(g - 2.0 * s2 / rho) <= 1e-9 * abs(g)
    assert abs(L - np.sum(column_residuals(C, M64, B) ** 2)) <= 1e-10 * L


def test_c5_block27_40_updates(h):
    blk = W.block27(40, probing=False)
    bs = 3
    Pb = mb.block_pattern(blk.A, bs, "diag")
    opts = dict(bs=bs, ep=0.05, ns=3, mn=3)
    M64, r64, s64 = run(h, blk.A, Pb, prec="fp64", **opts)
    M32, r32, s32 = run(h, blk.A, Pb, prec="mixed", **opts)
    assert blk.A.shape[1] == 192000
    assert same_pattern(M32, M64) and np.array_equal(s32, s64)
    assert np.allclose(r32, r64, rtol=1e-8, atol=1e-14)
