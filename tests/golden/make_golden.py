"""Generates the golden fixtures of the parity tests from the reference itself.

Runs the reference MSPAI sources compiled here (oracle/_ref/ref_driver, built by
`make -C oracle` from the reference tree) on small seeded instances of the five
workloads and stores the reference's output M (as written by its
Write_Matrix_To_File, 13 significant digits) together with the inputs'
recipe.  The fixtures are committed; this script needs the reference tree and
is only run in the build container:

    python tests/golden/make_golden.py

Cases (reference options in brackets):
  poisson2d_16    2-D Poisson 16x16, P = pattern(A)          [-2 -1 -ns 0]
  poisson2d_64    2-D Poisson 64x64 (the full fixed-pattern case) [-2 -1 -ns 0]
  convdiff3d_6    convection-diffusion 6^3, diagonal start,   [-1 -1 -ep 0.4 -ns 5 -mn 5 -um 1]
  convdiff3d_10   convection-diffusion 10^3                   [same]
  convdiff3d_10_um0  same with the sum bound                  [... -um 0]
  convdiff3d_10_qr   QR-update algorithm                       [... -qr 2]
  aniso16_probe   anisotropic 16x16 with probing rows e=ones,alt rho=10: the
                  reference's B-aware path (-cs > 0) crashes on its first
                  column, so this pins C = [A; rho Ce] through its default
                  path, whose right-hand side is e_k     [-2 -1 -ns 0 -Ce -Be -rho 10]
  ragged_3000     random nonsymmetric n=3000, P = dropped pattern(A^2) [file -1 -ns 0]
  block27_6       27-point block stencil 6^3 nodes x 3, block pattern of A
                                                              [-2 -1 -bs 3 -ns 0]
  block27_6_upd   same from the diagonal block pattern with block pattern
                  updates                        [-1 -1 -bs 3 -ns 3 -mn 3 -ep 0.05]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from mspai_b200 import workloads as W  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def run(w, args, name):
    with tempfile.TemporaryDirectory() as d:
        W.write_workload(w, d)
        subprocess.run([DRIVER, "A.mtx"] + args + ["-out", "M.mtx"], cwd=d, check=True,
                       stdout=subprocess.DEVNULL)
        M = W.read_mm(os.path.join(d, "M.mtx"))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), indptr=M.indptr.astype(np.int64),
                        indices=M.indices.astype(np.int32), data=M.data,
                        args=np.array(" ".join(args)))
    print(name, M.shape, M.nnz)


def main():
    if not os.path.exists(DRIVER):
        raise SystemExit("build the reference first: make -C oracle REF=<reference checkout>")
    run(W.poisson2d(16), ["-2", "-1", "-ns", "0"], "poisson2d_16")
    run(W.poisson2d(64), ["-2", "-1", "-ns", "0"], "poisson2d_64")
    adapt = ["-1", "-1", "-ep", "0.4", "-ns", "5", "-mn", "5", "-um", "1"]
    run(W.convdiff3d(6), adapt, "convdiff3d_6")
    run(W.convdiff3d(10), adapt, "convdiff3d_10")
    run(W.convdiff3d(10), adapt[:-1] + ["0"], "convdiff3d_10_um0")
    run(W.convdiff3d(10), adapt + ["-qr", "2"], "convdiff3d_10_qr")
    run(W.aniso2d_probing(16, kinds=("ones", "alt"), rho=10.0),
        ["-2", "-1", "-ns", "0", "-Ce", "Ce.mtx", "-Be", "Be.mtx", "-rho", "10"],
        "aniso16_probe")
    run(W.ragged(3000), ["P.mtx", "-1", "-ns", "0"], "ragged_3000")
    blk = W.block27(6, probing=False)
    run(blk, ["-2", "-1", "-bs", "3", "-ns", "0"], "block27_6")
    run(blk, ["-1", "-1", "-bs", "3", "-ns", "3", "-mn", "3", "-ep", "0.05"], "block27_6_upd")


if __name__ == "__main__":
    main()
