"""The command-line program mspai_b200/bin/mspai (the reference's serial
`mspai A P|-1|-2 B|-1 [options]`, src/main.cpp, src/Command_Line.cpp): same
positional arguments, option checks and Matrix Market output.  The GPU cases
run the workloads of the golden fixtures with the reference's own arguments
and compare M with the reference's output (FP64 mode: identical pattern,
values within 1e-10 relative, or the 13 printed digits)."""
import os
import subprocess

import pytest

from conftest import load_golden
from helpers import max_rel_diff, same_pattern
from mspai_b200 import workloads as W

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "mspai_b200", "bin", "mspai")


def run_cli(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=300)


def test_cli_rejects_invalid_options(tmp_path):
    W.write_workload(W.poisson2d(8), str(tmp_path))
    r = run_cli(["A.mtx", "-2", "-1", "-ep", "-1"], str(tmp_path))
    assert r.returncode != 0
    assert "epsilon" in (r.stderr + r.stdout).lower()
    r = run_cli(["A.mtx", "-2", "-1", "-cs", "5", "-qr", "2"], str(tmp_path))
    assert r.returncode != 0
    assert "simultaneously" in (r.stderr + r.stdout)


@pytest.mark.gpu
@pytest.mark.parametrize("name,work,args", [
    ("poisson2d_16", lambda: W.poisson2d(16), ["-2", "-1", "-ns", "0"]),
    ("convdiff3d_6", lambda: W.convdiff3d(6),
     ["-1", "-1", "-ep", "0.4", "-ns", "5", "-mn", "5", "-um", "1"]),
    ("block27_6", lambda: W.block27(6, probing=False), ["-2", "-1", "-bs", "3", "-ns", "0"]),
    ("block27_6_upd", lambda: W.block27(6, probing=False),
     ["-1", "-1", "-bs", "3", "-ns", "3", "-mn", "3", "-ep", "0.05"]),
])
def test_cli_matches_reference_output(tmp_path, name, work, args):
    W.write_workload(work(), str(tmp_path))
    r = run_cli(["A.mtx"] + args + ["-prec", "fp64", "-out", "M.mtx"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    M = W.read_mm(str(tmp_path / "M.mtx"))
    ref = load_golden(name)
    assert same_pattern(M, ref)
    assert max_rel_diff(M, ref) < 5e-12
