"""torch.autograd wrapper of the adjoint (mspai_b200.autograd.probing_loss):
gradcheck (central finite differences, FP64) with respect to every nonzero of
A and the probing weight rho, through both places A enters C = [A; rho E^T A];
the loss itself against ||C M - B||_F^2 of the setup's M."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import mspai_b200 as mb
from helpers import column_residuals
from mspai_b200 import workloads as W
from mspai_b200.autograd import probing_loss

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


@pytest.mark.parametrize("kinds,rho", [(("ones",), 2.0), (("ones", "alt"), 10.0)])
def test_gradcheck_probing(h, kinds, rho):
    A = W.aniso2d(6).tocsc()
    A.sort_indices()
    E = W.probing_vectors(A.shape[0], kinds).T           # n x p probing vectors
    Be = sp.csr_matrix(E.T)
    P = sp.csc_matrix(A != 0, dtype=np.float64)
    a = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
    r = torch.tensor(rho, dtype=torch.float64, requires_grad=True)
    f = lambda a_, r_: probing_loss(a_, r_, A, E, Be, P, h)
    assert torch.autograd.gradcheck(f, (a, r), eps=1e-6, atol=1e-6, rtol=1e-5)
    # the loss is ||C M - B||_F^2 of the setup
    L = f(a, r)
    C, B = mb.assemble_probing(A, sp.csr_matrix(E.T @ A), Be, rho)
    h.setup(C, P, B=B, options=mb.Options(ns=0, prec="fp64", probing=1, rho=rho))
    M = h.result()
    assert float(L.detach()) == pytest.approx(float(np.sum(column_residuals(C, M, B) ** 2)), rel=1e-10)


def test_gradcheck_plain_spai(h):
    A = W.ragged_matrix(60).tocsc()
    A.sort_indices()
    P = sp.csc_matrix(A != 0, dtype=np.float64)
    a = torch.tensor(A.data, dtype=torch.float64, requires_grad=True)
    r = torch.tensor(1.0, dtype=torch.float64)
    f = lambda a_: probing_loss(a_, r, A, None, None, P, h)
    assert torch.autograd.gradcheck(f, (a,), eps=1e-6, atol=1e-6, rtol=1e-5)
