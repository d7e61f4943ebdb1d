"""The library's drop-in inside the reference's own classes.

oracle/_ref/ref_driver_gpu is the reference's serial setup sequence compiled
from its sources (Read_mm_Matrix, Pattern_Switch, Init_Preconditioner,
Write_Matrix_To_File) with include/mspai_b200_reference_shim.hpp's
Spai_GPU_Algorithm in place of alg->SPAI_Algorithm behind -gpu, as a
maintainer would put it into PC_MSPAI::bspai (src/imspai.cpp:831-833).  One
command line runs stock and drop-in; the two files written by the reference's
Write_Matrix_To_File must hold the same matrix: identical index sets and
every value within 1e-10 (FP64) / 1e-8 (mixed) of its own magnitude, entries
below 1e-3 of their column's largest against that floor (the file prints 14
significant digits)."""
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from fullsize import read_mm, write_mm
from helpers import max_rel_diff, same_pattern
from mspai_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_driver_gpu")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(DRIVER),
                                 reason="oracle/_ref/ref_driver_gpu was not built (needs the "
                                        "reference sources at build time)")]

TOL = {"fp64": 1e-10, "mixed": 1e-8}


def run(directory, args, out, gpu=None):
    cmd = [DRIVER] + list(args) + ["-out", out] + (["-gpu", gpu] if gpu else [])
    r = subprocess.run(cmd, cwd=directory, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (cmd, r.stdout[-1000:], r.stderr[-1000:])
    return read_mm(os.path.join(directory, out))


def cases():
    return {
        "poisson64_fixed": (lambda d: write_mm(os.path.join(d, "A.mtx"), W.poisson2d(64).A),
                            ["A.mtx", "-2", "-1", "-ns", "0"]),
        "convdiff10_adaptive": (lambda d: write_mm(os.path.join(d, "A.mtx"), W.convdiff3d(10).A),
                                ["A.mtx", "-1", "-1", "-ep", "0.4", "-ns", "5", "-mn", "5"]),
        "convdiff10_mean0": (lambda d: write_mm(os.path.join(d, "A.mtx"), W.convdiff3d(10).A),
                             ["A.mtx", "-1", "-1", "-ep", "0.3", "-ns", "4", "-mn", "3",
                              "-um", "0"]),
    }


def _probing(d):
    w = W.aniso2d_probing(32, kinds=("ones", "alt"), rho=10.0)
    write_mm(os.path.join(d, "A.mtx"), w.A)
    write_mm(os.path.join(d, "Ce.mtx"), w.Ce)
    write_mm(os.path.join(d, "Be.mtx"), w.Be)


@pytest.mark.parametrize("name", list(cases()) + ["aniso32_probing"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dropin_writes_the_reference_matrix(tmp_path, name, prec):
    d = str(tmp_path)
    if name == "aniso32_probing":
        _probing(d)
        args = ["A.mtx", "-2", "-1", "-ns", "0", "-Ce", "Ce.mtx", "-Be", "Be.mtx", "-rho", "10"]
    else:
        make, args = cases()[name]
        make(d)
    stock = run(d, args, "stock.mtx")
    gpu = run(d, args, "gpu.mtx", gpu=prec)
    assert stock.shape == gpu.shape
    assert same_pattern(stock, gpu), name
    assert max_rel_diff(gpu, stock) < TOL[prec], name
    # the adaptive cases did grow their patterns
    if "adaptive" in name or "mean0" in name:
        assert stock.nnz > stock.shape[1]
