"""Input checks of mspai_setup, run on the device after staging for host and
device inputs alike: column pointers, row range, sorted unique rows and empty
columns of C (the reference rejects those, src/Read_mm_Matrix.cpp:745-751).
A rejected call leaves the handle usable."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import mspai_b200 as mb
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    handle = mb.Handle(0)
    yield handle
    handle.close()


def raw(M, device, pattern=False, edit=None):
    M = sp.csc_matrix(M)
    M.sort_indices()
    cp = torch.from_numpy(M.indptr.astype(np.int64))
    ri = torch.from_numpy(M.indices.astype(np.int32))
    v = None if pattern else torch.from_numpy(M.data.astype(np.float64))
    if edit:
        edit(cp, ri)
    if device == "cuda":
        cp, ri = cp.cuda(), ri.cuda()
        v = v.cuda() if v is not None else None
    return mb.DeviceCSC(M.shape[0], M.shape[1], cp, ri, v)


def swap_first_rows(cp, ri):
    ri[0], ri[1] = int(ri[1]), int(ri[0])


def row_out_of_range(cp, ri):
    ri[-1] = 10 ** 6


def pointer_decrease(cp, ri):
    cp[3] = cp[2] - 1


@pytest.mark.parametrize("device", ["cpu", "cuda"])
@pytest.mark.parametrize("which,edit,match", [
    ("C", swap_first_rows, "not sorted"),
    ("C", row_out_of_range, "out of range"),
    ("C", pointer_decrease, "decrease"),
    ("P", swap_first_rows, "not sorted"),
    ("P", row_out_of_range, "out of range"),
])
def test_invalid_structure_is_rejected(h, device, which, edit, match):
    w = W.poisson2d(8)
    C = raw(w.A, device, edit=edit if which == "C" else None)
    P = raw(w.P, device, pattern=True, edit=edit if which == "P" else None)
    with pytest.raises(mb.MspaiError, match=match):
        h.setup(C, P, options=mb.Options(ns=0))
    # the handle still works
    h.setup(w.A, w.P, options=mb.Options(ns=0))
    assert h.result().nnz == w.P.nnz


@pytest.mark.parametrize("device", ["cpu", "cuda"])
def test_empty_column_rejected_for_device_inputs_too(h, device):
    A = sp.csc_matrix(sp.diags([1.0, 0.0, 2.0]))
    A.eliminate_zeros()
    with pytest.raises(mb.MspaiError, match="empty"):
        h.setup(raw(A, device), raw(sp.identity(3), device, pattern=True),
                options=mb.Options(ns=0))


def test_schur_probing_is_refused(h):
    """-schur 1 is refused with a parameter error instead of silently returning
    the non-Schur M."""
    w = W.aniso2d_probing(8, kinds=("ones",), rho=1.0)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, 1.0)
    with pytest.raises(mb.MspaiError, match="Schur"):
        h.setup(C, w.P, B=B, options=mb.Options(ns=0, probing=1, schur=1))
    h.setup(w.A, w.P, options=mb.Options(ns=0))  # the handle stays usable


@pytest.mark.parametrize("adaptive", [False, True])
def test_apply_is_deterministic_and_exact(h, adaptive):
    """y = M x sums each row in a fixed order: repeated calls agree bit for bit
    (host and device vectors), and y equals the sparse product to rounding."""
    w = W.ragged(5000) if not adaptive else W.convdiff3d(12)
    opts = mb.Options(ns=0) if not adaptive else mb.Options(ns=3, mn=3)
    h.setup(w.A, w.P, options=opts)
    M = h.result()
    x = np.random.default_rng(7).standard_normal(w.n)
    y1 = h.apply(x)
    y2 = h.apply(x)
    assert np.array_equal(y1, y2)
    yd = h.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(y1, yd)
    ref = M @ x
    assert np.max(np.abs(y1 - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
