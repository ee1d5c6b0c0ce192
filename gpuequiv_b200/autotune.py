"""Autotuner for the round kernel's launch shape and lane-path limits.

Times ``DeviceGames.solve`` for each candidate (resident blocks per SM, which
selects the kernel's register budget, and rounds captured per CUDA graph),
keeps the fastest, then times the lane-path limits at that shape: the
largest position (successors, candidates per step, list length) one lane
solves before it goes to a whole warp.  Results are cached per device and
workload label in ``$GEQ_TUNING_CACHE`` (default
``~/.cache/gpuequiv_b200/tuning.json``).
"""
from __future__ import annotations

import json
import os

from .energygame import Context, DeviceGames

CANDIDATES = [(bps, r) for bps in (3, 4, 5) for r in (4, 8, 16, 32)]
# (successors, candidates per step, list length) of the lane path
LANE_LIMITS = [(16, 64, 16), (16, 32, 16), (16, 16, 16), (8, 64, 16), (8, 32, 16), (16, 64, 8), (12, 48, 12)]


def _pack(lim) -> int:
    d, w, k = lim
    return (d & 0xFF) | ((w & 0xFF) << 8) | ((k & 0xFF) << 16)


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
    """Pick (blocks_per_sm, rounds_per_graph, lane_limits) for this workload; returns
    {"best": {...}, "table": [...], "cached": bool} and applies the best."""
    key = f"{ctx.info()['name']}|{label}"
    db = _load() if use_cache else {}
    base_flags = ctx.tuning()["flags"]
    if key in db and "lane_limits" in db[key]["best"]:
        b = db[key]["best"]
        ctx.set_tuning(blocks_per_sm=b["blocks_per_sm"], rounds_per_graph=b["rounds_per_graph"], flags=base_flags,
                       lane_limits=_pack(b["lane_limits"]))
        return {**db[key], "cached": True}
    table = []
    first = _pack(LANE_LIMITS[0])
    for bps, r in CANDIDATES:
        ctx.set_tuning(blocks_per_sm=bps, rounds_per_graph=r, flags=base_flags, lane_limits=first)
        dg.solve()  # warm the graph for this shape
        ms = min(dg.solve()["device_ms"] for _ in range(repeats))
        table.append({"blocks_per_sm": bps, "rounds_per_graph": r, "lane_limits": list(LANE_LIMITS[0]),
                      "device_ms": ms})
    shape = min(table, key=lambda t: t["device_ms"])
    for lim in LANE_LIMITS[1:]:
        ctx.set_tuning(blocks_per_sm=shape["blocks_per_sm"], rounds_per_graph=shape["rounds_per_graph"],
                       flags=base_flags, lane_limits=_pack(lim))
        ms = min(dg.solve()["device_ms"] for _ in range(repeats))
        table.append({"blocks_per_sm": shape["blocks_per_sm"], "rounds_per_graph": shape["rounds_per_graph"],
                      "lane_limits": list(lim), "device_ms": ms})
    best = min(table, key=lambda t: t["device_ms"])
    ctx.set_tuning(blocks_per_sm=best["blocks_per_sm"], rounds_per_graph=best["rounds_per_graph"], flags=base_flags,
                   lane_limits=_pack(best["lane_limits"]))
    rec = {"best": best, "table": table}
    if use_cache:
        db[key] = rec
        _store(db)
    return {**rec, "cached": False}
