"""Autotuner for the round kernel's launch shape.

Times ``DeviceGames.solve`` for each candidate (resident blocks per SM, which
selects the kernel's register budget, and rounds captured per CUDA graph)
and keeps the fastest.  Results are cached per device and workload label in
``$GEQ_TUNING_CACHE`` (default ``~/.cache/gpuequiv_b200/tuning.json``).
"""
from __future__ import annotations

import json
import os

from .energygame import Context, DeviceGames

CANDIDATES = [(bps, r) for bps in (3, 4, 5) for r in (4, 8, 16)]


def _cache_path() -> str:
    return os.environ.get("GEQ_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "gpuequiv_b200", "tuning.json"))


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db: dict) -> None:
    p = _cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            json.dump(db, f, indent=1)
    except OSError:
        pass


def autotune(dg: DeviceGames, ctx: Context, label: str, repeats: int = 2, use_cache: bool = True) -> dict:
    """Pick (blocks_per_sm, rounds_per_graph) for this workload; returns
    {"best": {...}, "table": [...], "cached": bool} and applies the best."""
    key = f"{ctx.info()['name']}|{label}"
    db = _load() if use_cache else {}
    base_flags = ctx.tuning()["flags"]
    if key in db:
        b = db[key]["best"]
        ctx.set_tuning(blocks_per_sm=b["blocks_per_sm"], rounds_per_graph=b["rounds_per_graph"], flags=base_flags)
        return {**db[key], "cached": True}
    table = []
    for bps, r in CANDIDATES:
        ctx.set_tuning(blocks_per_sm=bps, rounds_per_graph=r, flags=base_flags)
        dg.solve()  # warm the graph for this shape
        ms = min(dg.solve()["device_ms"] for _ in range(repeats))
        table.append({"blocks_per_sm": bps, "rounds_per_graph": r, "device_ms": ms})
    best = min(table, key=lambda t: t["device_ms"])
    ctx.set_tuning(blocks_per_sm=best["blocks_per_sm"], rounds_per_graph=best["rounds_per_graph"], flags=base_flags)
    rec = {"best": best, "table": table}
    if use_cache:
        db[key] = rec
        _store(db)
    return {**rec, "cached": False}
