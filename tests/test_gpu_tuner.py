"""The persisted autotuner on the GPU: a sweep on a column sample of a ragged
problem applies a tuning whose setup gives the default tuning's M (mixed
mode: 1e-8 per entry; the knobs only move columns between kernels), a second
call takes the stored choice without timing, and out-of-range knobs are
refused."""
import json

import numpy as np
import pytest

import mspai_b200 as mb
from helpers import max_rel_diff
from mspai_b200 import tuner
from mspai_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_autotune_ragged(tmp_path):
    w = W.ragged(30000, seed=5)
    path = str(tmp_path / "tuning.json")
    h = mb.Handle(0)
    try:
        opts = mb.Options(ns=0, prec="mixed")
        h.setup(w.A, w.P, options=opts)
        M0 = h.result()
        r = tuner.autotune(h, w.A, w.P, opts, sample_cols=8000, cache=path)
        assert not r["cached"] and h.get_tuning() == r["tuning"]
        h.setup(w.A, w.P, options=opts)
        assert max_rel_diff(h.result(), M0) < 1e-8
        table = json.load(open(path))
        assert len(table[r["key"]]["tried"]) == len(tuner.grid_points(True))
        h2 = mb.Handle(0)
        try:
            r2 = tuner.autotune(h2, w.A, w.P, opts, sample_cols=8000, cache=path)
            assert r2["cached"] and h2.get_tuning() == r["tuning"]
        finally:
            h2.close()
        with pytest.raises(mb.MspaiError, match="tuning out of range"):
            h.set_tuning(fixed_arena_kb=200)
        assert h.get_tuning() == r["tuning"]
    finally:
        h.close()


def test_tuning_knobs_move_columns_not_results():
    """Extreme knobs: tiny arenas send every fixed column down the overflow
    chain, a wide tiny bucket takes more columns into the warp kernel."""
    w = W.ragged(6000, seed=8)
    h = mb.Handle(0)
    try:
        opts = mb.Options(ns=0, prec="fp64")
        h.setup(w.A, w.P, options=opts)
        M0 = h.result()
        h.set_tuning(fixed_arena_kb=8, fixed_arena_large_kb=8, warp_emax=256, warp_nmax=32)
        h.setup(w.A, w.P, options=opts)
        st = h.stats()
        assert st["bucket_columns"][1] == 0 and st["bucket_columns"][3] > 0
        assert max_rel_diff(h.result(), M0) < 1e-10
    finally:
        h.close()
