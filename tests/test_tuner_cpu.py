"""The autotuner's sweep, key and JSON store (mspai_b200/tuner.py) with a fake
handle whose setup time is a known function of the knobs (no GPU)."""
import json

import pytest

import mspai_b200 as mb
from mspai_b200 import tuner


class FakeHandle:
    def __init__(self):
        self.t = {"smem_kb": 48, "fixed_arena_kb": 107, "fixed_arena_large_kb": 212,
                  "warp_emax": 64, "warp_nmax": 16, "w_smem_kb": 96}
        self.setups = 0
        self.last = None

    def get_tuning(self):
        return dict(self.t)

    def set_tuning(self, **k):
        self.t.update(k)

    def setup(self, C, P, B=None, options=None):
        self.setups += 1
        self.last = options

    def stats(self):
        t = self.t
        # fastest at warp (128, 24); general: smem 32, w 160
        ms = abs(t["warp_emax"] - 128) + abs(t["warp_nmax"] - 24) \
            + abs(t["smem_kb"] - 32) + abs(t["w_smem_kb"] - 160) + 1.0
        return {"setup_ms": float(ms)}


class P:
    ncols = 1000
    nnz = 130000


def test_sweep_takes_the_minimum():
    pts = [{"a": 1}, {"a": 2}, {"a": 3}]
    best, ms, tried = tuner.sweep(pts, lambda p: (p["a"] - 2) ** 2)
    assert best == {"a": 2} and ms == 0 and len(tried) == 3


def test_key_classes():
    k = tuner.config_key("B200", mb.Options(ns=0, prec="mixed"), 1_000_000, 134.0)
    assert k == "B200|fixed|mixed|bs1|n2^20|J2^7"
    k = tuner.config_key("B200", mb.Options(ns=5, mn=5, prec="fp64", batched=False), 110592, 1)
    assert k == "B200|adaptive|plain|bs1|n2^17|J2^0"


@pytest.mark.parametrize("opts,fixed", [(dict(ns=0, prec="mixed"), True),
                                        (dict(ns=5, mn=5, prec="mixed"), False)])
def test_autotune_sweeps_stores_and_reuses(tmp_path, opts, fixed):
    path = str(tmp_path / "tuning.json")
    h = FakeHandle()
    o = mb.Options(**opts)
    r = tuner.autotune(h, None, P(), o, sample_cols=200, cache=path, gpu_name="FakeGPU")
    npts = len(tuner.grid_points(fixed))
    assert not r["cached"] and h.setups == 2 * npts
    assert h.last.col_begin == 0 and h.last.col_end == 200   # a sample of the columns
    if fixed:
        assert (r["tuning"]["fixed_arena_kb"], r["tuning"]["fixed_arena_large_kb"],
                r["tuning"]["warp_emax"], r["tuning"]["warp_nmax"]) == (107, 212, 128, 24)
    else:
        assert (r["tuning"]["smem_kb"], r["tuning"]["w_smem_kb"]) == (32, 160)
    assert h.get_tuning() == r["tuning"]
    table = json.load(open(path))
    assert r["key"] in table and len(table[r["key"]]["tried"]) == npts
    # the stored choice is applied without timing
    h2 = FakeHandle()
    r2 = tuner.autotune(h2, None, P(), o, sample_cols=200, cache=path, gpu_name="FakeGPU")
    assert r2["cached"] and h2.setups == 0 and h2.get_tuning() == r["tuning"]
    # another GPU is another key
    h3 = FakeHandle()
    r3 = tuner.autotune(h3, None, P(), o, sample_cols=200, cache=path, gpu_name="OtherGPU")
    assert not r3["cached"] and h3.setups == 2 * npts
    assert len(json.load(open(path))) == 2
