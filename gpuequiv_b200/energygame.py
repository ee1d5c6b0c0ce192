"""Energy games solved on the GPU (mirror of src/energygame.rs).

``EnergyGame.run`` hands the CSR game graph, the energies and the to_reach
positions to ``geq_energy_game_run`` of libgeq; the fixpoint runs entirely on
the device.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Sequence

import numpy as np

from ._lib import (GeqError, check, geq_energy_lists, geq_game_graph, geq_solve_stats, geq_tuning, lib)
from .energy import EnergyArray, EnergyConf, Update, UpdateArray, pack_update

_u32 = C.POINTER(C.c_uint32)
_u64 = C.POINTER(C.c_uint64)
_u8 = C.POINTER(C.c_uint8)

_ZERO32 = np.zeros(1, dtype=np.uint32)
_ZERO64 = np.zeros(1, dtype=np.uint64)
_ZERO8 = np.zeros(1, dtype=np.uint8)


def _p(a, t):
    return a.ctypes.data_as(t)


class Context:
    """A CUDA device context of libgeq (replaces GPUCommon, gpuutils.rs:8-31)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.geq_context_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib.geq_context_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        name = C.create_string_buffer(256)
        sms = C.c_int()
        mem = C.c_uint64()
        check(lib.geq_context_info(self.h, name, 256, C.byref(sms), C.byref(mem)))
        return {"name": name.value.decode(), "sms": sms.value, "total_mem": mem.value}

    def tuning(self) -> dict:
        t = geq_tuning()
        lib.geq_context_get_tuning(self.h, C.byref(t))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def set_tuning(self, blocks_per_sm=0, rounds_per_graph=0, small_limit=0, flags=0, lane_limits=0):
        """Zero fields keep their value (flags are always set).  lane_limits:
        (successors, candidates, list length) of the lane path, or its packed
        u32 form."""
        if isinstance(lane_limits, (tuple, list)):
            d, w, k = lane_limits
            lane_limits = (d & 0xFF) | ((w & 0xFF) << 8) | ((k & 0xFF) << 16)
        t = geq_tuning(blocks_per_sm, rounds_per_graph, small_limit, flags, lane_limits)
        check(lib.geq_context_set_tuning(self.h, C.byref(t)))


_default: Context | None = None
_default_lock = threading.Lock()


def default_context() -> Context:
    """Process-wide context on LOCAL_RANK (or device 0), created on first use."""
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(int(os.environ.get("LOCAL_RANK", "0")))
        return _default


class GameGraph:
    """GameGraph (energygame.rs:120-324): CSR successors, weights, attacker flags."""

    def __init__(self, n_vertices: int, edges, attacker_pos: Sequence[bool], conf: EnergyConf):
        """GameGraph::new (energygame.rs:141-194).  ``edges`` = (from, to, update)
        with the update as i32 values (``update(...)``) or an ``Update``."""
        adj = [[] for _ in range(n_vertices)]
        wts = [[] for _ in range(n_vertices)]
        for f, t, u in edges:
            adj[f].append(t)
            wts[f].append(u)
        row = np.zeros(n_vertices + 1, dtype=np.uint32)
        for v in range(n_vertices):
            row[v + 1] = row[v] + len(adj[v])
        col = np.array([t for a in adj for t in a], dtype=np.uint32)
        ua = UpdateArray.from_conf([u for w in wts for u in w], conf)
        self._set(row, col, ua.array, np.array([1 if a else 0 for a in attacker_pos], dtype=np.uint8), conf)

    @classmethod
    def from_csr(cls, row_offsets, column_indices, weights, attacker_pos, conf: EnergyConf) -> "GameGraph":
        g = cls.__new__(cls)
        w = np.ascontiguousarray(weights, dtype=np.uint32).reshape(-1, conf.update_size())
        g._set(np.ascontiguousarray(row_offsets, dtype=np.uint32),
               np.ascontiguousarray(column_indices, dtype=np.uint32), w,
               np.ascontiguousarray(attacker_pos, dtype=np.uint8), conf)
        return g

    @classmethod
    def empty(cls, conf: EnergyConf) -> "GameGraph":
        return cls.from_csr(np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros((0, conf.update_size())),
                            np.zeros(0, np.uint8), conf)

    def _set(self, row, col, wt, att, conf):
        self.row_offsets = row
        self.column_indices = col
        self.weights = UpdateArray(wt, conf)
        self.attacker_pos = att
        self.conf = conf
        self._rev = None

    def get_conf(self) -> EnergyConf:
        return self.conf

    def n_vertices(self) -> int:
        return len(self.attacker_pos)

    def n_edges(self) -> int:
        return int(self.row_offsets[-1])

    def adj(self, v: int) -> np.ndarray:
        return self.column_indices[self.row_offsets[v]:self.row_offsets[v + 1]]

    def make_reverse(self):
        """energygame.rs:235-250 (host copy; the solver builds its own)."""
        n = self.n_vertices()
        src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(self.row_offsets).astype(np.int64))
        order = np.argsort(self.column_indices, kind="stable")
        rcol = src[order]
        cnt = np.bincount(self.column_indices, minlength=n) if n else np.zeros(0, np.int64)
        rrow = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
        self._rev = (rrow, rcol)

    def reverse(self, v: int) -> np.ndarray:
        if self._rev is None:
            self.make_reverse()
        rrow, rcol = self._rev
        return rcol[rrow[v]:rrow[v + 1]]

    @property
    def rev_row_offsets(self):
        if self._rev is None:
            self.make_reverse()
        return self._rev[0]

    @property
    def rev_column_indices(self):
        if self._rev is None:
            self.make_reverse()
        return self._rev[1]

    def standard_reach(self) -> np.ndarray:
        deg = np.diff(self.row_offsets.astype(np.int64))
        return np.nonzero((self.attacker_pos == 0) & (deg == 0))[0].astype(np.uint32)

    def c_view(self):
        """geq_game_graph struct; keep ``self`` alive while it is used."""
        g = geq_game_graph()
        g.conf.elements = self.conf.elements
        g.conf.max = self.conf.max
        g.n_vertices = self.n_vertices()
        g.row_offsets = _p(self.row_offsets, _u32)
        col = self.column_indices if self.column_indices.size else _ZERO32
        wt = self.weights.array if self.weights.array.size else _ZERO32  # contiguous by construction
        att = self.attacker_pos if self.attacker_pos.size else _ZERO8
        g.column_indices = _p(col, _u32)
        g.weights = _p(wt, _u32)
        g.attacker_pos = _p(att, _u8)
        return g


def _lists_from_solution(sol, game: int, conf: EnergyConf) -> list[EnergyArray]:
    view = geq_energy_lists()
    check(lib.geq_solution_lists(sol, game, C.byref(view)))
    n = view.n_vertices
    es = view.energy_size
    offs = np.ctypeslib.as_array(view.offsets, shape=(n + 1,)).copy() if n + 1 else np.zeros(1, np.uint64)
    total = int(offs[-1]) if n + 1 else 0
    data = (np.ctypeslib.as_array(view.data, shape=(total * es,)).copy() if total else np.zeros(0, np.uint32))
    data = data.reshape(-1, es)
    return [EnergyArray(data[int(offs[v]):int(offs[v + 1])], conf) for v in range(n)]


def _stats_of(sol) -> dict:
    st = geq_solve_stats()
    lib.geq_solution_stats(sol, C.byref(st))
    return st.as_dict()


def _pack_lists(energies: Sequence[EnergyArray], conf: EnergyConf):
    es = conf.energy_size()
    counts = np.array([e.n_energies() for e in energies], dtype=np.uint64)
    offs = np.zeros(len(energies) + 1, dtype=np.uint64)
    np.cumsum(counts, out=offs[1:])
    data = (np.ascontiguousarray(np.concatenate([e.array.reshape(-1) for e in energies]), dtype=np.uint32)
            if int(offs[-1]) else np.zeros(1, dtype=np.uint32))
    view = geq_energy_lists()
    view.n_vertices = len(energies)
    view.energy_size = es
    view.offsets = _p(offs, _u64)
    view.data = _p(data, _u32)
    return view, (offs, data)


class EnergyGame:
    """EnergyGame (energygame.rs:329-384)."""

    def __init__(self, graph: GameGraph, energies: list[EnergyArray], to_reach):
        self.graph = graph
        self.energies = energies
        self.to_reach = np.ascontiguousarray(to_reach, dtype=np.uint32)
        self.stats: dict = {}

    @classmethod
    def standard_reach(cls, graph: GameGraph) -> "EnergyGame":
        """Defender positions without successors are the targets (energygame.rs:347-352)."""
        return cls.with_reach(graph, graph.standard_reach())

    @classmethod
    def with_reach(cls, graph: GameGraph, to_reach) -> "EnergyGame":
        """energygame.rs:355-365: {0} at the targets, empty elsewhere."""
        conf = graph.get_conf()
        energies = [EnergyArray.empty(conf) for _ in range(graph.n_vertices())]
        to_reach = np.ascontiguousarray(to_reach, dtype=np.uint32)
        for v in to_reach:
            energies[int(v)] = EnergyArray.zero(1, conf)
        return cls(graph, energies, to_reach)

    def run(self, context: Context | None = None) -> list[EnergyArray]:
        """EnergyGame::run (energygame.rs:379-383): solve on the GPU, store and
        return the winning budgets of every position."""
        ctx = context or default_context()
        conf = self.graph.get_conf()
        g = self.graph.c_view()
        init, keep = _pack_lists(self.energies, conf)
        reach = self.to_reach if self.to_reach.size else _ZERO32
        sol = C.c_void_p()
        check(lib.geq_energy_game_run(ctx.h, C.byref(g), C.byref(init), _p(reach, _u32), len(self.to_reach),
                                      C.byref(sol)))
        try:
            self.energies = _lists_from_solution(sol, 0, conf)
            self.stats = _stats_of(sol)
        finally:
            lib.geq_solution_free(sol)
        del keep
        return self.energies


def run_batch(graphs: Sequence[GameGraph], context: Context | None = None):
    """Solve many games (standard reach) in one set of device rounds.
    Returns (list of per-game energy lists, stats)."""
    ctx = context or default_context()
    n = len(graphs)
    views = (geq_game_graph * n)(*[g.c_view() for g in graphs])
    sol = C.c_void_p()
    check(lib.geq_energy_game_run_batch(ctx.h, n, views, None, None, None, C.byref(sol)))
    try:
        out = [_lists_from_solution(sol, i, graphs[i].get_conf()) for i in range(n)]
        stats = _stats_of(sol)
    finally:
        lib.geq_solution_free(sol)
    return out, stats


class _SolutionOwner:
    """Frees a geq_solution once the last array viewing its memory is gone."""

    def __init__(self, h):
        self.h = h

    def __del__(self):
        if self.h is not None and self.h.value:
            lib.geq_solution_free(self.h)
            self.h = None


def _borrow(ptr, n: int, ctype, dtype, owner: _SolutionOwner) -> np.ndarray:
    """numpy view of n elements at ptr that keeps `owner` alive."""
    if n == 0:
        return np.zeros(0, dtype)
    buf = (ctype * n).from_address(C.cast(ptr, C.c_void_p).value)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dtype)


def run_batch_raw(graphs: Sequence[GameGraph], context: Context | None = None, views=None):
    """geq_energy_game_run_batch with flat results: returns (offsets, data,
    stats) where offsets[g] is game g's (n+1) offset array and data[g] its
    packed energies.  The arrays are views of the solution's page-locked
    memory (no copy, no per-position objects); it is released when the last
    of them is gone."""
    ctx = context or default_context()
    n = len(graphs)
    if views is None:
        views = (geq_game_graph * n)(*[g.c_view() for g in graphs])
    sol = C.c_void_p()
    check(lib.geq_energy_game_run_batch(ctx.h, n, views, None, None, None, C.byref(sol)))
    offs, data = _flat_lists(sol, graphs)
    return offs, data, _stats_of(sol)


def _flat_lists(sol, graphs):
    """Per-game (offsets, data) views of a solution's flat memory; the
    solution is freed once the last view is gone."""
    n = len(graphs)
    owner = _SolutionOwner(sol)
    po, pd = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
    no, nw = C.c_uint64(), C.c_uint64()
    check(lib.geq_solution_flat(sol, C.byref(po), C.byref(no), C.byref(pd), C.byref(nw)))
    flat_o = _borrow(po, no.value, C.c_uint64, np.uint64, owner)
    flat_d = _borrow(pd, nw.value, C.c_uint32, np.uint32, owner)
    nv = np.fromiter((g.n_vertices() for g in graphs), dtype=np.int64, count=n)
    es = graphs[0].get_conf().energy_size() if n else 1
    ob = np.zeros(n + 1, np.int64)
    np.cumsum(nv + 1, out=ob[1:])
    tot = flat_o[ob[1:] - 1].astype(np.int64) * es if n else np.zeros(0, np.int64)
    db = np.zeros(n + 1, np.int64)
    np.cumsum(tot, out=db[1:])
    obl, dbl = ob.tolist(), db.tolist()
    offs = [flat_o[obl[i]:obl[i + 1]] for i in range(n)]
    data = [flat_d[dbl[i]:dbl[i + 1]] for i in range(n)]
    return offs, data


def b_min(graph: GameGraph, offsets) -> int:
    """Schedule-independent byte floor of a solve, from its final lists A*
    (offsets[n+1], STANDARD: one word per energy): every row pair and edge
    read once, the attacker flags once, every final list written once and
    read once per predecessor -- 4(n+1) + 8m + n + sum_v 4|A*_v|(1 + indeg(v))."""
    n = graph.n_vertices()
    m = graph.n_edges()
    indeg = np.bincount(graph.column_indices, minlength=n).astype(np.int64) if m else np.zeros(n, np.int64)
    cnt = np.diff(np.asarray(offsets, dtype=np.int64))
    return int(4 * (n + 1) + 8 * m + n + 4 * int(np.dot(cnt, 1 + indeg)))


def run_static(graph: GameGraph, context: Context | None = None, to_reach=None, data_cap: int | None = None):
    """geq_energy_game_run_static: one game solved inside the library's
    file-scope device scratch, with no allocation in the call.  Returns
    (offsets, data, stats) like one game of run_batch_raw; to_reach None means
    standard reach.  If the result outgrows data_cap the call is repeated
    with the size it reported."""
    ctx = context or default_context()
    n = graph.n_vertices()
    view = graph.c_view()
    reach = None if to_reach is None else np.ascontiguousarray(to_reach, dtype=np.uint32)
    rp = None if reach is None else reach.ctypes.data_as(C.POINTER(C.c_uint32))
    nr = 0 if reach is None else len(reach)
    offs = np.zeros(n + 1, np.uint64)
    cap = 4 * n + 64 if data_cap is None else int(data_cap)
    for _ in range(2):
        data = np.zeros(max(cap, 1), np.uint32)
        nw = C.c_uint64(0)
        st = geq_solve_stats()
        status = lib.geq_energy_game_run_static(ctx.h, C.byref(view), rp, nr,
                                                offs.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                data.ctypes.data_as(C.POINTER(C.c_uint32)), cap, C.byref(nw),
                                                C.byref(st))
        if status == 3 and nw.value > cap and data_cap is None:  # INVALID_INPUT: data_cap too small
            cap = int(nw.value)
            continue
        check(status)
        return offs, data[:nw.value], st.as_dict()
    check(status)


def c_views(graphs: Sequence[GameGraph]):
    """geq_game_graph array of the graphs (keep the graphs alive)."""
    return (geq_game_graph * len(graphs))(*[g.c_view() for g in graphs])


class DeviceGames:
    """Games resident on the device (upload once, solve repeatedly)."""

    def __init__(self, graphs: Sequence[GameGraph], context: Context | None = None):
        self.ctx = context or default_context()
        self.graphs = list(graphs)
        n = len(self.graphs)
        views = (geq_game_graph * n)(*[g.c_view() for g in self.graphs])
        h = C.c_void_p()
        check(lib.geq_device_games_create(self.ctx.h, n, views, None, None, None, C.byref(h)))
        self.h = h

    def solve(self) -> dict:
        st = geq_solve_stats()
        check(lib.geq_device_games_solve(self.ctx.h, self.h, C.byref(st)))
        return st.as_dict()

    def download_raw(self):
        """All games' lists as (offsets, data) per game, views of one flat
        page-locked block (no per-position objects)."""
        sol = C.c_void_p()
        check(lib.geq_device_games_download(self.ctx.h, self.h, C.byref(sol)))
        return _flat_lists(sol, self.graphs)

    def download(self):
        sol = C.c_void_p()
        check(lib.geq_device_games_download(self.ctx.h, self.h, C.byref(sol)))
        try:
            return [_lists_from_solution(sol, i, self.graphs[i].get_conf()) for i in range(len(self.graphs))]
        finally:
            lib.geq_solution_free(sol)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib.geq_device_games_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Context", "default_context", "GameGraph", "EnergyGame", "run_batch", "run_batch_raw", "c_views",
           "DeviceGames", "GeqError", "b_min"]
