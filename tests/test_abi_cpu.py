"""C ABI and host layer, without a GPU: the library loads, exports every
symbol the headers declare, checks options like the reference, and its Matrix
Market / probing / pattern helpers agree with independent Python versions."""
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

import mspai_b200 as mb
from mspai_b200 import _lib, workloads as W
from oracle import pyoracle as O

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in ("mspai_b200.h", "mspai_b200_io.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mspai_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = declared_functions()
    assert decl, "no declarations found"
    assert decl <= set(_lib.EXPORTED)
    for name in decl:
        assert hasattr(lib, name), name


def test_defaults_match_reference_command_line():
    p = mb.Options().to_c()
    assert (p.ep, p.mn, p.ns, p.um, p.hs, p.cs, p.qr, p.fg, p.rho, p.bs) == \
        (0.4, 5, 5, 1, 6, 0, 0, 0.3, 1.0, 1)


@pytest.mark.parametrize("kw,msg", [
    (dict(ns=-1), "Illegal number of improvement steps"),
    (dict(ep=-0.1), "Illegal epsilon"),
    (dict(hs=7), "Illegal hash table size"),
    (dict(cs=10, ch=1), "Caching and Hashing cannot be used simultaneously"),
    (dict(cs=10, qr=2), "QR-Updates and Caching"),
    (dict(ch=1, qr=2), "QR-Updates and Hashing"),
    (dict(qr=6), "Illegal parameter for qr"),
    (dict(fg=1.5), "Illegal parameter for fg"),
    (dict(rho=-1.0), "Illegal parameter for rho"),
    (dict(um=2), "Illegal value for using mean value"),
    (dict(probing=1, ns=3), "only supported in static MSPAI"),
    (dict(target=0, ns=0, qr=1), "only supported in static MSPAI"),
    (dict(schur=1, probing=0), "schur"),
    (dict(pm=2), "prerequesting maximum columns"),
])
def test_option_checks_follow_reference(kw, msg):
    with pytest.raises(ValueError, match=msg):
        mb.Options(**kw).validate()


def test_probing_assembly_matches_reader_semantics():
    w = W.aniso2d_probing(8, kinds=("ones", "alt"), rho=10.0)
    C, B = mb.assemble_probing(w.A, w.Ce, w.Be, 10.0)
    assert abs(C - O.stack_probing(w.A, w.Ce, 10.0)).max() == 0
    assert abs(B - O.target(w.n, w.Be, 10.0)).max() == 0
    assert C.shape == (w.n + 2, w.n)


def test_start_patterns():
    w = W.aniso2d_probing(8, kinds=("ones",), rho=1.0)
    C, _ = mb.assemble_probing(w.A, w.Ce, w.Be, 1.0)
    P2 = mb.start_pattern(C, -2)
    assert (P2 != 0).nnz == w.A.nnz and abs((P2 != 0).astype(int) - (w.A != 0).astype(int)).nnz == 0
    P1 = mb.start_pattern(C, -1)
    assert (P1 - sp.identity(w.n)).nnz == 0 or abs(P1 - sp.identity(w.n)).max() == 0


def test_matrix_market_round_trip_in_reference_format(tmp_path):
    w = W.convdiff3d(4)
    path = str(tmp_path / "M.mtx")
    mb.write_mm(path, w.A)
    lines = open(path).read().splitlines()
    assert lines[0] == "%%MatrixMarket matrix coordinate real general"
    assert lines[1] == f"{w.n} {w.n} {w.A.nnz}"
    # "row col" then one space before a negative value, two before a positive one
    pat = re.compile(r"^\d+ \d+(  \d| -\d)\.\d{13}e[+-]\d{2,3}$")
    assert all(pat.match(l) for l in lines[2:])
    assert any("  " in l for l in lines[2:]) and any(" -" in l for l in lines[2:])
    back = mb.read_mm(path)
    assert abs(back - w.A).max() <= 1e-12 * abs(w.A).max()
    py = W.read_mm(path)
    assert abs(back - py).max() == 0


def test_matrix_market_errors(tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text("not a matrix market file\n")
    with pytest.raises(mb.MspaiError, match="INPUT"):
        mb.read_mm(str(bad))
    with pytest.raises(mb.MspaiError, match="IO"):
        mb.read_mm(str(tmp_path / "missing.mtx"))
    trunc = tmp_path / "trunc.mtx"
    trunc.write_text("%%MatrixMarket matrix coordinate real general\n3 3 4\n1 1 1.0\n")
    with pytest.raises(mb.MspaiError, match="Truncated"):
        mb.read_mm(str(trunc))


def test_symmetric_files_are_expanded(tmp_path):
    f = tmp_path / "s.mtx"
    f.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n"
                 "1 1 2.0\n2 1 -1.0\n2 2 2.0\n3 3 1.0\n")
    M = mb.read_mm(str(f)).toarray()
    assert M[0, 1] == -1.0 and M[1, 0] == -1.0


def test_no_device_is_reported_without_gpu(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(mb.MspaiError, match="NO_DEVICE"):
        mb.Handle(0)


def test_pattern_power2_checks_inputs_on_the_host():
    """mspai_pattern_power2 refuses malformed host input and a NaN drop before
    it touches a device (so this runs without a GPU)."""
    import ctypes
    from mspai_b200 import _lib
    lib = _lib.load()

    def call(cp, ri, vv, nrows, drop):
        c = _lib.mspai_csc(nrows, len(cp) - 1, len(ri), cp.ctypes.data, ri.ctypes.data,
                           vv.ctypes.data, _lib.MEM_HOST)
        m = _lib.mspai_matrix()
        buf = ctypes.create_string_buffer(256)
        rc = lib.mspai_pattern_power2(ctypes.byref(c), drop, 0, ctypes.byref(m), buf, len(buf))
        return rc, buf.value.decode()

    cp = np.array([0, 2, 4, 5], dtype=np.int64)
    vv = np.ones(5)
    unsorted = np.array([0, 1, 2, 0, 2], dtype=np.int32)  # column 1 lists rows 2, 0
    rc, msg = call(cp, unsorted, vv, 3, 1e-3)
    assert rc == 2 and "not sorted" in msg and "column 1" in msg
    out_of_range = np.array([0, 1, 0, 1, 7], dtype=np.int32)
    rc, msg = call(cp, out_of_range, vv, 3, 1e-3)
    assert rc == 2 and "row index 7 out of range in column 2" in msg
    good = np.array([0, 1, 0, 1, 2], dtype=np.int32)
    rc, msg = call(cp, good, vv, 3, float("nan"))
    assert rc == 1 and "drop" in msg
