"""TransitionSystem, GameBuild and Equivalence (mirror of src/lib.rs,
src/gamebuild.rs and src/equivalence.rs) over libgeq."""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

import numpy as np

from ._lib import check, geq_game_batch_info, geq_game_graph, geq_position, lib
from .energy import Energy, EnergyArray, EnergyConf
from .energygame import Context, GameGraph, _stats_of, default_context

_u32 = C.POINTER(C.c_uint32)
_i32 = C.POINTER(C.c_int32)
_u64 = C.POINTER(C.c_uint64)
_Z32 = np.zeros(1, dtype=np.uint32)
_ZI32 = np.zeros(1, dtype=np.int32)


def _p(a, t):
    return a.ctypes.data_as(t)


class TransitionSystem:
    """Labelled transition system (lib.rs:172-536).  Label 0 is tau."""

    def __init__(self, edges: Iterable[tuple[int, int, int]] | None = None, *, _handle=None):
        if _handle is not None:
            self.h = _handle
            return
        e = np.asarray(list(edges or []), dtype=np.int64).reshape(-1, 3)
        self.h = TransitionSystem._from_arrays(e[:, 0], e[:, 1], e[:, 2])

    @staticmethod
    def _from_arrays(src, dst, lab):
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        l = np.ascontiguousarray(lab, dtype=np.int32)
        h = C.c_void_p()
        n = len(s)
        check(lib.geq_lts_from_edges(n, _p(s if n else _Z32, _u32), _p(d if n else _Z32, _u32),
                                     _p(l if n else _ZI32, _i32), C.byref(h)))
        return h

    @classmethod
    def from_arrays(cls, src, dst, label, n_vertices: int | None = None) -> "TransitionSystem":
        """Edges as arrays; with n_vertices, processes beyond the largest id
        keep empty adjacency lists (From<Vec<Vec<Transition>>>)."""
        if n_vertices is None:
            return cls(_handle=cls._from_arrays(src, dst, label))
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        l = np.ascontiguousarray(label, dtype=np.int32)
        h = C.c_void_p()
        n = len(s)
        check(lib.geq_lts_from_adjacency(n_vertices, n, _p(s if n else _Z32, _u32), _p(d if n else _Z32, _u32),
                                         _p(l if n else _ZI32, _i32), C.byref(h)))
        return cls(_handle=h)

    @classmethod
    def from_csv_file(cls, path: str) -> "TransitionSystem":
        """lib.rs:364-406: lines `from,to,label`; label "i" is tau."""
        h = C.c_void_p()
        check(lib.geq_lts_from_csv_file(str(path).encode(), C.byref(h)))
        return cls(_handle=h)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                lib.geq_lts_free(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def n_vertices(self) -> int:
        return lib.geq_lts_n_vertices(self.h)

    def n_transitions(self) -> int:
        return lib.geq_lts_n_transitions(self.h)

    def inner(self):
        """Label-sorted adjacency as (offsets, targets, labels) arrays."""
        n, m = self.n_vertices(), self.n_transitions()
        off = np.zeros(n + 1, dtype=np.uint64)
        tg = np.zeros(max(m, 1), dtype=np.uint32)
        lb = np.zeros(max(m, 1), dtype=np.int32)
        lib.geq_lts_transitions(self.h, _p(off, _u64), _p(tg, _u32), _p(lb, _i32))
        return off, tg[:m], lb[:m]

    def adj(self, p: int) -> list[tuple[int, int]]:
        off, tg, lb = self.inner()
        return [(int(tg[k]), int(lb[k])) for k in range(int(off[p]), int(off[p + 1]))]

    def signature_refinement(self) -> tuple[np.ndarray, int]:
        """lib.rs:444-464: (partition, number of bisimilarity classes)."""
        n = self.n_vertices()
        part = np.zeros(max(n, 1), dtype=np.uint64)
        cnt = C.c_uint64()
        check(lib.geq_lts_signature_refinement(self.h, _p(part, _u64), C.byref(cnt)))
        return part[:n], cnt.value

    def bisimilar_minimize(self) -> tuple["TransitionSystem", np.ndarray]:
        """lib.rs:413-432: (minimised LTS, process -> class mapping)."""
        n = self.n_vertices()
        mapping = np.zeros(max(n, 1), dtype=np.uint64)
        h = C.c_void_p()
        check(lib.geq_lts_bisimilar_minimize(self.h, C.byref(h), _p(mapping, _u64)))
        return TransitionSystem(_handle=h), mapping[:n]

    def compare(self, p: int, q: int, context: Context | None = None) -> EnergyArray:
        """lib.rs:275-283: energies of Attack(p, {q}) in the minimised system."""
        return compare_batch([(self, p, q)], context=context, minimize=True)[0]

    def compare_unminimized(self, p: int, q: int, context: Context | None = None) -> EnergyArray:
        """lib.rs:291-296."""
        return compare_batch([(self, p, q)], context=context, minimize=False)[0]

    def equivalences(self, context: Context | None = None) -> "Equivalence":
        """lib.rs:329-334."""
        return Equivalence._compute(self, True, context)

    def equivalences_unminimized(self, context: Context | None = None) -> "Equivalence":
        """lib.rs:338-343."""
        return Equivalence._compute(self, False, context)


def signature_refinement_batch(systems: Sequence[TransitionSystem], context: Context | None = None):
    """TransitionSystem::signature_refinement (lib.rs:444-464) of many systems
    at once on the device; returns [(partition, n_classes)] like
    ``TransitionSystem.signature_refinement``."""
    ctx = context or default_context()
    n = len(systems)
    hs = (C.c_void_p * max(n, 1))(*[s.h.value for s in systems])
    sizes = [s.n_vertices() for s in systems]
    part = np.zeros(max(sum(sizes), 1), dtype=np.uint64)
    cnt = np.zeros(max(n, 1), dtype=np.uint64)
    check(lib.geq_lts_signature_refinement_batch(ctx.h, n, hs, _p(part, _u64), _p(cnt, _u64)))
    out, o = [], 0
    for k, m in enumerate(sizes):
        out.append((part[o:o + m].copy(), int(cnt[k])))
        o += m
    return out


def compare_batch(jobs: Sequence[tuple[TransitionSystem, int, int]], context: Context | None = None,
                  minimize: bool = True, return_stats: bool = False):
    """TransitionSystem::compare for many (lts, p, q) jobs, all games solved in
    one set of device rounds."""
    ctx = context or default_context()
    n = len(jobs)
    hs = (C.c_void_p * max(n, 1))(*[j[0].h.value for j in jobs])
    ps = np.array([j[1] for j in jobs] or [0], dtype=np.uint32)
    qs = np.array([j[2] for j in jobs] or [0], dtype=np.uint32)
    sol = C.c_void_p()
    check(lib.geq_compare_batch(ctx.h, n, hs, _p(ps, _u32), _p(qs, _u32), 1 if minimize else 0, C.byref(sol)))
    try:
        # all games' lists at once: game i has one position, offsets (0, count_i)
        po, pd = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
        no, nw = C.c_uint64(), C.c_uint64()
        check(lib.geq_solution_flat(sol, C.byref(po), C.byref(no), C.byref(pd), C.byref(nw)))
        offs = np.ctypeslib.as_array(po, shape=(no.value,)).astype(np.int64) if no.value else np.zeros(0, np.int64)
        data = np.ctypeslib.as_array(pd, shape=(nw.value,)).copy() if nw.value else np.zeros(0, np.uint32)
        stats = _stats_of(sol)
    finally:
        lib.geq_solution_free(sol)
    base = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(offs[1::2][:n], out=base[1:])
    bl = base.tolist()
    out = [EnergyArray(data[bl[i]:bl[i + 1]].reshape(-1, 1), EnergyConf.STANDARD) for i in range(n)]
    return (out, stats) if return_stats else out


# ---- GameBuild ---------------------------------------------------------------
class Position(tuple):
    """Position (gamepos.rs:210-251) as (kind, p, q, qx)."""

    __slots__ = ()

    def __new__(cls, kind: str, p: int, q=(), qx=()):
        return super().__new__(cls, (kind, int(p), tuple(int(x) for x in q), tuple(int(x) for x in qx)))

    @classmethod
    def attack(cls, p, q):
        return cls("attack", p, q)

    @classmethod
    def clause(cls, p, q):
        return cls("clause", p, (q,))

    @classmethod
    def defend(cls, p, q, qx):
        return cls("defend", p, q, qx)

    kind = property(lambda s: s[0])
    p = property(lambda s: s[1])
    q = property(lambda s: s[2])
    qx = property(lambda s: s[3])

    def is_attack(self) -> bool:
        return self[0] in ("attack", "clause")


class StartInfo:
    """StartInfo (equivalence.rs:19-38)."""

    def __init__(self, starting_points, n_processes):
        self.starting_points = starting_points
        self.n_processes = n_processes


class GameBuild:
    """GameBuild (gamebuild.rs:139-266): the generated game and its positions."""

    def __init__(self, handle):
        self.h = handle
        g = geq_game_graph()
        lib.geq_game_build_graph(self.h, C.byref(g))
        n = g.n_vertices
        row = np.ctypeslib.as_array(g.row_offsets, shape=(n + 1,)).copy()
        m = int(row[-1])
        col = np.ctypeslib.as_array(g.column_indices, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        wt = np.ctypeslib.as_array(g.weights, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        att = np.ctypeslib.as_array(g.attacker_pos, shape=(n,)).copy() if n else np.zeros(0, np.uint8)
        self.game = GameGraph.from_csr(row, col, wt.reshape(-1, 1), att, EnergyConf.STANDARD)
        self.n_starting_points = lib.geq_game_build_n_starting_points(self.h)
        self._nodes = None

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                lib.geq_game_build_free(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    @property
    def nodes(self) -> list[Position]:
        if self._nodes is None:
            kinds = ("attack", "clause", "defend")
            out = []
            pos = geq_position()
            for i in range(self.game.n_vertices()):
                check(lib.geq_game_build_position(self.h, i, C.byref(pos)))
                q = [pos.q[k] for k in range(pos.n_q)]
                qx = [pos.qx[k] for k in range(pos.n_qx)]
                out.append(Position(kinds[pos.kind], pos.p, q, qx))
            self._nodes = out
        return self._nodes

    def starting_points(self) -> list[Position]:
        return [p for p in self.nodes[:self.n_starting_points] if p.kind == "attack"]

    @classmethod
    def compare(cls, lts: TransitionSystem, p: int, q: int) -> "GameBuild":
        h = C.c_void_p()
        check(lib.geq_game_build_compare(lts.h, p, q, C.byref(h)))
        return cls(h)

    @classmethod
    def compare_bounded(cls, lts: TransitionSystem, p: int, q: int, max_positions: int) -> "GameBuild":
        """compare() that raises GeqError(OUT_OF_MEMORY) beyond max_positions."""
        h = C.c_void_p()
        check(lib.geq_game_build_compare_bounded(lts.h, p, q, int(max_positions), C.byref(h)))
        return cls(h)

    @classmethod
    def compare_all(cls, lts: TransitionSystem) -> tuple["GameBuild", StartInfo]:
        h = C.c_void_p()
        check(lib.geq_game_build_compare_all(lts.h, C.byref(h)))
        b = cls(h)
        return b, StartInfo(b.starting_points(), lts.n_vertices())

    @classmethod
    def compare_multiple(cls, lts: TransitionSystem, processes: Sequence[int]) -> tuple["GameBuild", StartInfo]:
        pr = np.ascontiguousarray(processes, dtype=np.uint32)
        h = C.c_void_p()
        check(lib.geq_game_build_compare_multiple(lts.h, _p(pr if pr.size else _Z32, _u32), len(pr), C.byref(h)))
        b = cls(h)
        return b, StartInfo(b.starting_points(), lts.n_vertices())


def compare_all_starts(lts: TransitionSystem) -> list[tuple[int, int]]:
    """Start pairs of GameBuild::compare_all (gamebuild.rs:104-133, :200-215):
    every ordered pair of distinct processes with the same set of enabled
    labels, the classes in order of their first process."""
    off, _, lb = lts.inner()
    classes: dict = {}
    for p in range(lts.n_vertices()):
        key = tuple(sorted(set(int(x) for x in lb[int(off[p]):int(off[p + 1])])))
        classes.setdefault(key, []).append(p)
    return [(p, q) for c in classes.values() for p in c for q in c if p != q]


class GameBatch:
    """GameBuild::compare (gamebuild.rs:165-170) for many (lts, p, q) jobs,
    built on the device one breadth-first level of all games at a time
    (geq_game_build_compare_batch).  ``graph(j)`` is job j's GameGraph,
    identical to ``GameBuild.compare(lts, p, q).game``; a job whose game
    exceeds ``max_positions`` raises GeqError(OUT_OF_MEMORY) there, as
    ``GameBuild.compare_bounded`` does."""

    def __init__(self, jobs: Sequence[tuple[TransitionSystem, int, int]], context: Context | None = None,
                 max_positions: int = 0):
        ctx = context or default_context()
        n = len(jobs)
        hs = (C.c_void_p * max(n, 1))(*[j[0].h.value for j in jobs])
        ps = np.array([j[1] for j in jobs] or [0], dtype=np.uint32)
        qs = np.array([j[2] for j in jobs] or [0], dtype=np.uint32)
        h = C.c_void_p()
        check(lib.geq_game_build_compare_batch(ctx.h, n, hs, _p(ps, _u32), _p(qs, _u32), int(max_positions),
                                               C.byref(h)))
        self._adopt(h)

    def _adopt(self, h):
        self.h = h
        info = geq_game_batch_info()
        lib.geq_game_batch_stats(h, C.byref(info))
        self.stats = info.as_dict()

    @classmethod
    def with_starts(cls, systems: Sequence[TransitionSystem], starts: Sequence[Sequence[tuple[int, int]]],
                    context: Context | None = None, max_positions: int = 0) -> "GameBatch":
        """Job j is the game of systems[j] from the start positions
        Attack(p, {q}) for (p, q) in starts[j], numbered in that order (the
        start layout of GameBuild::compare_multiple / compare_all,
        gamebuild.rs:176-215); geq_game_build_starts_batch."""
        ctx = context or default_context()
        n = len(systems)
        hs = (C.c_void_p * max(n, 1))(*[s.h.value for s in systems])
        off = np.zeros(n + 1, dtype=np.uint32)
        np.cumsum([len(x) for x in starts], out=off[1:])
        flat = [pq for x in starts for pq in x]
        ps = np.array([pq[0] for pq in flat] or [0], dtype=np.uint32)
        qs = np.array([pq[1] for pq in flat] or [0], dtype=np.uint32)
        h = C.c_void_p()
        check(lib.geq_game_build_starts_batch(ctx.h, n, hs, _p(off, _u32), _p(ps, _u32), _p(qs, _u32),
                                              int(max_positions), C.byref(h)))
        b = cls.__new__(cls)
        b._adopt(h)
        return b

    @classmethod
    def compare_all(cls, systems: Sequence[TransitionSystem], context: Context | None = None,
                    max_positions: int = 0) -> "GameBatch":
        """GameBuild::compare_all (gamebuild.rs:200-215) of each system on the
        device: every ordered pair of distinct processes with the same enabled
        labels, classes in order of their first process."""
        return cls.with_starts(systems, [compare_all_starts(lts) for lts in systems], context, max_positions)

    def n_starting_points(self, j: int) -> int:
        return lib.geq_game_batch_n_starting_points(self.h, int(j))

    def __len__(self):
        return lib.geq_game_batch_n_jobs(self.h)

    def view(self, j: int) -> geq_game_graph:
        """Borrowed C view of job j's graph (valid while this object lives)."""
        g = geq_game_graph()
        check(lib.geq_game_batch_graph(self.h, int(j), C.byref(g)))
        return g

    def graph(self, j: int) -> GameGraph:
        g = self.view(j)
        n = g.n_vertices
        row = np.ctypeslib.as_array(g.row_offsets, shape=(n + 1,)).copy()
        m = int(row[-1])
        col = np.ctypeslib.as_array(g.column_indices, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        wt = np.ctypeslib.as_array(g.weights, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        att = np.ctypeslib.as_array(g.attacker_pos, shape=(n,)).copy() if n else np.zeros(0, np.uint8)
        return GameGraph.from_csr(row, col, wt.reshape(-1, 1), att, EnergyConf.STANDARD)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                lib.geq_game_batch_free(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass


# ---- Equivalence -------------------------------------------------------------
class EquivalenceRelation:
    """EquivalenceRelation (equivalence.rs:180-247) as class representatives."""

    def __init__(self, classes: np.ndarray, n_classes: int):
        self.classes = classes
        self.n_classes = n_classes

    def __len__(self):
        return len(self.classes)

    def find(self, p: int) -> int:
        return int(self.classes[p])

    def count_classes(self) -> int:
        return self.n_classes

    def class_of(self, proc: int) -> list[int]:
        c = self.classes[proc]
        return [int(i) for i in np.nonzero(self.classes == c)[0]]

    def get_classes(self) -> list[list[int]]:
        order: dict[int, int] = {}
        out: list[list[int]] = []
        for i, c in enumerate(self.classes):
            c = int(c)
            if c not in order:
                order[c] = len(out)
                out.append([])
            out[order[c]].append(i)
        return out

    def equiv(self, p: int, q: int) -> bool:
        return self.classes[p] == self.classes[q]


class Equivalence:
    """Equivalence (equivalence.rs:41-175)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def _compute(cls, lts: TransitionSystem, minimize: bool, context: Context | None):
        ctx = context or default_context()
        h = C.c_void_p()
        check(lib.geq_equivalences(ctx.h, lts.h, 1 if minimize else 0, C.byref(h)))
        return cls(h)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                lib.geq_equivalence_free(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    @property
    def n_processes(self) -> int:
        return lib.geq_equivalence_n_processes(self.h)

    def n_starting_points(self) -> int:
        return lib.geq_equivalence_n_starting_points(self.h)

    def energies(self, p: int, q: int) -> EnergyArray | None:
        d = _u32()
        n = C.c_uint64()
        if not lib.geq_equivalence_energies(self.h, p, q, C.byref(d), C.byref(n)):
            return None
        a = np.ctypeslib.as_array(d, shape=(n.value,)).copy() if n.value else np.zeros(0, np.uint32)
        return EnergyArray(a.reshape(-1, 1), EnergyConf.STANDARD)

    def preorder(self, p: int, q: int, equivalence: Energy) -> bool:
        return bool(lib.geq_equivalence_preorder(self.h, p, q, _p(equivalence.data, _u32)))

    def equiv(self, p: int, q: int, equivalence: Energy) -> bool:
        return bool(lib.geq_equivalence_equiv(self.h, p, q, _p(equivalence.data, _u32)))

    def relation(self, equivalence: Energy) -> EquivalenceRelation:
        n = self.n_processes
        cls_ = np.zeros(max(n, 1), dtype=np.uint32)
        nc = C.c_uint32()
        check(lib.geq_equivalence_relation(self.h, _p(equivalence.data, _u32), _p(cls_, _u32), C.byref(nc)))
        return EquivalenceRelation(cls_[:n], nc.value)


__all__ = ["TransitionSystem", "compare_batch", "Position", "StartInfo", "GameBuild", "Equivalence",
           "EquivalenceRelation"]
