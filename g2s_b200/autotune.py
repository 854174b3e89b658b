"""Autotuner of the tensor-core form: node batch B (nodes per GEMM launch),
the template-prefix tile (the pattern matrix's K extent: template offsets
scored on the tensor cores; nodes with neighbours beyond it go to the exact
map) and the shortlist width W (candidates kept per node and position
range), chosen per job shape and kept in a JSON cache.

A job shape is the TI grid, variable types, n, k, the tensor mode and the
GPU.  Tuning runs the simulation of that shape on a tuning grid (by default
256^2 in 2-D, 48^3 in 3-D, unconditional, a fixed seed) once per candidate
(after an untimed run that builds each prefix's pattern matrix) and keeps
the fastest by device time whose regret audit (every node re-run on the
plain path) stays within ``max_regret``; only a candidate that would
replace the best (and the automatic choice) is audited.  The search is a
coordinate descent from the automatic choice: width, then prefix, then
batch, each over its candidates with the others held.

The reference has no counterpart: G2S's throughput knobs are the thread
counts of `-j` (src/qs.cpp), chosen by the user.
"""
from __future__ import annotations

import json
import os
from typing import Callable, Dict, Optional, Sequence

import numpy as np

WIDTHS = (8, 16, 32)
BATCHES = (2048, 4096, 8192)
PREFIX_SCALES = (0.125, 0.25, 0.5, 1.0, 2.0)   # times the automatic prefix, rounded to 64 offsets


def default_cache() -> str:
    return os.environ.get("G2S_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "g2s_b200", "tune.json"))


def shape_key(ti_shape: Sequence[int], types: Sequence[int], n: int, k: float, mode: str, device_name: str) -> str:
    return (f"{device_name}|{mode}|ti={'x'.join(str(int(d)) for d in ti_shape)}|"
            f"types={','.join(str(int(t)) for t in types)}|n={int(n)}|k={float(k):g}")


def load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save(path: str, table: Dict[str, dict]) -> None:
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _round64(x: float) -> int:
    return max(64, int(round(x / 64.0)) * 64)


def search(run: Callable[[dict, bool], dict], max_regret: float = 0.0) -> dict:
    """Coordinate descent over width, prefix and batch.  ``run(params,
    audit)`` runs params {"width", "prefix", "batch"} (0: the automatic
    choice) and returns {"ms": device time, "prefix": the prefix used}, with
    audit {"regret": r, "audited": a} as well.  A candidate replaces the best
    only when it is faster and its audit passes (regret <= max_regret of the
    audited nodes); audits run only for such candidates.  Returns the chosen
    params with their time, regret and the number of runs."""
    timed: Dict[tuple, dict] = {}
    audited: Dict[tuple, dict] = {}
    runs = [0]

    def key(p):
        return (p["width"], p["prefix"], p["batch"])

    def t(p):
        if key(p) not in timed:
            timed[key(p)] = run(dict(p), False)
            runs[0] += 1
        return timed[key(p)]

    def ok(p):
        if key(p) not in audited:
            r = run(dict(p), True)
            runs[0] += 1
            audited[key(p)] = dict(r, ok=r["regret"] <= max_regret * max(1, r["audited"]))
        return audited[key(p)]["ok"]

    # the automatic choice is audited first: when it fails, the first
    # candidate that passes replaces it whatever its time
    best = {"width": 0, "prefix": 0, "batch": 4096}
    cur = t(best)["ms"] if ok(best) else float("inf")
    auto_prefix = int(t(best)["prefix"])
    for name, values in (("width", WIDTHS),
                         ("prefix", tuple(sorted({_round64(s * auto_prefix) for s in PREFIX_SCALES}))),
                         ("batch", BATCHES)):
        for v in values:
            p = dict(best, **{name: v})
            r = t(p)
            if r["ms"] < cur and ok(p):
                cur, best = r["ms"], p
    good = ok(best)
    a = audited[key(best)]
    return dict(best, prefix=int(t(best)["prefix"]), ms=float(t(best)["ms"]), regret=int(a["regret"]),
                audited=int(a["audited"]), runs=runs[0], ok=bool(good))


def tuning_grid(ti: np.ndarray, types: Sequence[int]) -> tuple:
    nd = ti.ndim - (1 if len(types) > 1 else 0)
    return (256, 256) if nd <= 2 else (48, 48, 48)


def tune(ti: np.ndarray, types: Sequence[int], n: int, k: float, mode: str = "bf16", device: int = 0,
         grid: Optional[Sequence[int]] = None, cache: Optional[str] = None, max_regret: float = 0.001,
         seed: int = 1234, retune: bool = False, device_name: Optional[str] = None) -> dict:
    """Tuned {"width", "prefix", "batch", "ms", ...} for this job shape, from
    the cache when it holds the shape (unless ``retune``).  ``device_name``
    (default: the CUDA device's name) is part of the shape key."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(device)
    path = cache or default_cache()
    key = shape_key(ti.shape, types, n, k, mode, device_name.replace("|", "/"))
    table = load(path)
    if key in table and not retune:
        return dict(table[key], cached=True)
    from . import Simulation

    g = tuple(grid) if grid is not None else tuning_grid(ti, types)
    di = np.full(g + ((len(types),) if len(types) > 1 else ()), np.nan, np.float32)

    sim = Simulation(ti, di, types, n=n, k=k, seed=seed, device=device)
    built = [None]

    def run(p, audit):
        sim.set_tensor(mode, prefix=p["prefix"], width=p["width"], batch=p["batch"], audit=1.0 if audit else 0.0)
        if not audit and built[0] != p["prefix"]:
            sim.run()   # builds this prefix's pattern matrix (untimed)
            built[0] = p["prefix"]
        sim.run()
        i = sim.info()
        return {"ms": i["ms_total"], "prefix": i["tensor_prefix"], "regret": i["regret"], "audited": i["audited"]}

    try:
        res = search(run, max_regret)
    finally:
        sim.close()
    res.update(grid=list(g), key=key)
    table = load(path)
    table[key] = res
    save(path, table)
    return dict(res, cached=False)


def apply(sim, params: dict, mode: str = "bf16", audit: float = 0.0):
    """Set a simulation's tensor-core form to tuned params."""
    return sim.set_tensor(mode, prefix=int(params["prefix"]), width=int(params["width"]),
                          batch=int(params["batch"]), audit=audit)
