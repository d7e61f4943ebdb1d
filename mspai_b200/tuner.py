"""Autotuner of the launch shapes, persisted per GPU and configuration.

The reference's column loop has no launch shape to choose; here the size
buckets and the shared-memory areas of the solvers decide how many columns
run at once per SM and which columns take which kernel.  `autotune` times
setups of a sample of the problem's columns (the first `sample_cols` problem
columns, a column range of the real problem) for each point of a small grid
of knobs (mspai_tuning: the fixed-pattern solver's two arenas, the tiny
bucket's bounds, the general solver's shared-memory area and its bucket
split), keeps the fastest in the handle and stores it in a JSON file under a
key of the GPU's name and the configuration's class:

    {"<gpu>|fixed|mixed|bs1|n2^20|J2^7": {"tuning": {...}, "ms": ..., "tried": [...]}}

A later call with the same key applies the stored choice without timing.  The
file is `cache` if given, else $MSPAI_TUNING_CACHE, else
~/.cache/mspai_b200/tuning.json.  Results do not depend on the knobs beyond
rounding.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from dataclasses import replace
from typing import Callable, Dict, List, Optional

# the grids: every point is a full mspai_tuning (defaults for the rest).  The
# fixed-pattern solver's arenas stay at their largest (107 KB: two CTAs per
# SM; 212 KB): a smaller arena only sends more columns down the overflow chain,
# which a sample of the columns can miss (a sweep that tried 160 KB for the
# second launch chose it on 50,000 columns and lost 2 % on the million)
FIXED_GRID = {"warp_emax": [64, 128], "warp_nmax": [16, 24, 32]}
GENERAL_GRID = {"smem_kb": [24, 32, 48], "w_smem_kb": [64, 96, 160]}


def default_cache() -> str:
    return os.environ.get("MSPAI_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mspai_b200",
                                       "tuning.json"))


def _log2_bucket(x: float) -> int:
    return int(round(math.log2(max(x, 1.0))))


def config_key(gpu: str, options, n_columns: int, mean_pattern: float) -> str:
    """Configuration class: fixed or adaptive, precision, block size, and the
    problem's size and mean |J_k| rounded to powers of two."""
    kind = "fixed" if (options.ns == 0 or options.mn == 0) else "adaptive"
    prec = options.prec if options.batched else "plain"
    return (f"{gpu}|{kind}|{prec}|bs{options.bs}|n2^{_log2_bucket(n_columns)}"
            f"|J2^{_log2_bucket(mean_pattern)}")


def grid_points(fixed: bool) -> List[Dict[str, int]]:
    g = FIXED_GRID if fixed else GENERAL_GRID
    keys = sorted(g)
    return [dict(zip(keys, vals)) for vals in itertools.product(*(g[k] for k in keys))]


def _load(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path: str, table: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def sweep(points: List[Dict[str, int]], measure: Callable[[Dict[str, int]], float]):
    """(best point, its time, every (point, time)) over the grid."""
    tried = []
    for p in points:
        tried.append((p, float(measure(p))))
    best = min(tried, key=lambda t: t[1])
    return best[0], best[1], tried


def autotune(handle, C, P, options, B=None, sample_cols: int = 50000,
             cache: Optional[str] = None, gpu_name: Optional[str] = None,
             refresh: bool = False) -> dict:
    """Chooses and applies the handle's tuning for this configuration; returns
    {"key", "tuning", "ms", "cached"}.  C and P as for Handle.setup."""
    path = cache or default_cache()
    nprob = int(P.ncols) if hasattr(P, "ncols") else int(P.shape[1])
    nnzp = int(P.nnz)
    if gpu_name is None:
        import torch
        gpu_name = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"
    key = config_key(gpu_name, options, nprob, nnzp / max(nprob, 1))
    table = _load(path)
    if key in table and not refresh:
        handle.set_tuning(**table[key]["tuning"])
        return {"key": key, "tuning": table[key]["tuning"], "ms": table[key]["ms"],
                "cached": True}
    fixed = (options.ns == 0 or options.mn == 0) and options.bs == 1 and options.batched
    cols = max(1, min(sample_cols, nprob))
    sample = replace(options, col_begin=0, col_end=cols, keep_factors=False, reuse_factors=0)
    base = handle.get_tuning()

    def measure(point):
        handle.set_tuning(**{**base, **point})
        handle.setup(C, P, B=B, options=sample)          # warm-up
        handle.setup(C, P, B=B, options=sample)
        return handle.stats()["setup_ms"]

    best, ms, tried = sweep(grid_points(fixed), measure)
    choice = {**base, **best}
    handle.set_tuning(**choice)
    table = _load(path)
    table[key] = {"tuning": choice, "ms": ms, "sample_columns": cols,
                  "tried": [{"point": p, "ms": t} for p, t in tried]}
    _store(path, table)
    return {"key": key, "tuning": choice, "ms": ms, "cached": False}
