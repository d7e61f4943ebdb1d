"""The application phase: M applied by mspai_apply inside right-preconditioned
GMRES on the device (the reference's PETSc KSP loop with Apply_MSPAI).  The
preconditioned solve reaches ||b - Ax|| <= 1e-8 ||b|| in fewer iterations
than the unpreconditioned one, and mspai_apply equals M x."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import mspai_b200 as mb
from mspai_b200 import workloads as W
from mspai_b200.krylov import csr_matvec, gmres

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def test_apply_equals_m_times_x(h):
    w = W.convdiff3d(10)
    h.setup(w.A, w.P, options=mb.Options(ep=0.4, ns=5, mn=5))
    M = h.result()
    x = np.random.default_rng(1).standard_normal(w.A.shape[1])
    y = h.apply(x)
    assert np.allclose(y, M @ x, rtol=1e-12, atol=1e-12 * np.abs(M @ x).max())
    yt = h.apply(torch.from_numpy(x).cuda())
    assert np.allclose(yt.cpu().numpy(), M @ x, rtol=1e-12, atol=1e-12 * np.abs(M @ x).max())


@pytest.mark.parametrize("ns", [0, 5])
def test_preconditioned_gmres(h, ns):
    w = W.convdiff3d(16)
    A = w.A
    P = w.P if ns > 0 else sp.csc_matrix(A != 0, dtype=np.float64)
    h.setup(A, P, options=mb.Options(ep=0.4, ns=ns, mn=5))
    Av = csr_matvec(A)
    b = torch.from_numpy(np.random.default_rng(2).standard_normal(A.shape[0])).cuda()
    x0, it0, r0 = gmres(Av, b, None, tol=1e-8, restart=50, maxiter=3000)
    x1, it1, r1 = gmres(Av, b, lambda v: h.apply(v), tol=1e-8, restart=50, maxiter=3000)
    assert r1 <= 1e-8
    true = float(torch.linalg.vector_norm(b - Av(x1)) / torch.linalg.vector_norm(b))
    assert true <= 1.01e-8
    # fewer iterations with M (pattern(A): less than half)
    assert it1 < (0.5 if ns == 0 else 1.0) * it0, (it0, it1)
