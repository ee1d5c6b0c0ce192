"""ctypes driver for the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by
``__graft_entry__.smoke()`` (as the checker) and by ``bench.py``'s CPU
baseline.  The product package ``gpuequiv_b200`` never imports it.

The oracle restates the reference crate's energy-game path on the CPU; see
``oracle/geq_oracle.h`` for the per-function citations.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)


def build() -> None:
    """Compile liboracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        for name in ("ora_energy_bits", "ora_energy_size", "ora_energy_mask",
                     "ora_update_bits", "ora_update_size", "ora_update_mask"):
            f = getattr(L, name)
            f.argtypes = [C.c_uint32, C.c_uint32]
            f.restype = C.c_uint32
        L.ora_pack_energy.argtypes = [C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p]
        L.ora_pack_energy.restype = C.c_int
        L.ora_unpack_energy.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p]
        L.ora_pack_update.argtypes = [C.c_uint32, C.c_uint32, i32p, C.c_uint32, u32p]
        L.ora_pack_update.restype = C.c_int
        L.ora_unpack_update.argtypes = [C.c_uint32, C.c_uint32, u32p, i32p]
        L.ora_inv_update.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, u32p]
        L.ora_run_game.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p, u32p, u8p,
                                   u64p, u32p, u32p, C.c_uint32]
        L.ora_run_game.restype = C.c_void_p
        L.ora_solution_total.argtypes = [C.c_void_p]
        L.ora_solution_total.restype = C.c_uint64
        L.ora_solution_offsets.argtypes = [C.c_void_p, u64p]
        L.ora_solution_data.argtypes = [C.c_void_p, u32p]
        L.ora_solution_stats.argtypes = [C.c_void_p, u64p]
        L.ora_solution_free.argtypes = [C.c_void_p]
        L.ora_standard_reach.argtypes = [C.c_uint32, u32p, u8p, u32p]
        L.ora_standard_reach.restype = C.c_uint32
        L.ora_defend_intersection.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, C.c_uint32,
                                              C.c_uint32, u32p]
        L.ora_defend_intersection.restype = C.c_int32
        L.ora_lts_from_edges.argtypes = [C.c_uint64, u32p, u32p, i32p]
        L.ora_lts_from_edges.restype = C.c_void_p
        L.ora_lts_from_csv.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        L.ora_lts_from_csv.restype = C.c_void_p
        L.ora_lts_n_vertices.argtypes = [C.c_void_p]
        L.ora_lts_n_vertices.restype = C.c_uint32
        L.ora_lts_n_transitions.argtypes = [C.c_void_p]
        L.ora_lts_n_transitions.restype = C.c_uint64
        L.ora_lts_transitions.argtypes = [C.c_void_p, u64p, u32p, i32p]
        L.ora_lts_signature_refinement.argtypes = [C.c_void_p, u64p]
        L.ora_lts_signature_refinement.restype = C.c_uint64
        L.ora_lts_minimize.argtypes = [C.c_void_p, u64p]
        L.ora_lts_minimize.restype = C.c_void_p
        L.ora_lts_free.argtypes = [C.c_void_p]
        L.ora_build_compare.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.ora_build_compare.restype = C.c_void_p
        L.ora_build_compare_all.argtypes = [C.c_void_p]
        L.ora_build_compare_all.restype = C.c_void_p
        L.ora_build_n_nodes.argtypes = [C.c_void_p]
        L.ora_build_n_nodes.restype = C.c_uint32
        L.ora_build_n_edges.argtypes = [C.c_void_p]
        L.ora_build_n_edges.restype = C.c_uint64
        L.ora_build_n_starting.argtypes = [C.c_void_p]
        L.ora_build_n_starting.restype = C.c_uint32
        L.ora_build_graph.argtypes = [C.c_void_p, u32p, u32p, u32p, u8p]
        L.ora_build_position.argtypes = [C.c_void_p, C.c_uint32, u32p, u32p, u32p, u32p]
        L.ora_build_position_sets.argtypes = [C.c_void_p, C.c_uint32, u32p, u32p]
        L.ora_build_free.argtypes = [C.c_void_p]
        L.ora_compare_batch.argtypes = [C.c_uint32, C.POINTER(C.c_void_p), u32p, u32p, C.c_uint32,
                                        u64p, u64p]
        L.ora_run_games_parallel.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p,
                                             C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p),
                                             C.POINTER(u8p), C.c_uint32, u64p]
        L.ora_solve_games.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p,
                                      C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p),
                                      C.POINTER(u8p), C.c_uint32, u32p, u64p, C.POINTER(C.c_void_p)]
        L.ora_b_min.argtypes = [C.c_uint32, u32p, u32p, u64p]
        L.ora_b_min.restype = C.c_uint64
        L.ora_check_fixpoint.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p, u32p, u8p, u64p, u32p,
                                         C.c_uint32, u32p]
        L.ora_check_fixpoint.restype = C.c_uint64
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def conf_sizes(elements: int, max_: int) -> dict:
    L = lib()
    return dict(
        energy_bits=L.ora_energy_bits(elements, max_), energy_size=L.ora_energy_size(elements, max_),
        energy_mask=L.ora_energy_mask(elements, max_), update_bits=L.ora_update_bits(elements, max_),
        update_size=L.ora_update_size(elements, max_), update_mask=L.ora_update_mask(elements, max_))


def pack_energy(elements, max_, values):
    es = lib().ora_energy_size(elements, max_)
    v = np.ascontiguousarray(values, dtype=np.uint32)
    out = np.zeros(es, dtype=np.uint32)
    if lib().ora_pack_energy(elements, max_, _p(v, C.c_uint32), len(v), _p(out, C.c_uint32)) != 0:
        return None
    return out


def unpack_energy(elements, max_, words):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.zeros(elements, dtype=np.uint32)
    lib().ora_unpack_energy(elements, max_, _p(w, C.c_uint32), _p(out, C.c_uint32))
    return out


def pack_update(elements, max_, values):
    us = lib().ora_update_size(elements, max_)
    v = np.ascontiguousarray(values, dtype=np.int32)
    out = np.zeros(us, dtype=np.uint32)
    if lib().ora_pack_update(elements, max_, _p(v, C.c_int32), len(v), _p(out, C.c_uint32)) != 0:
        return None
    return out


def unpack_update(elements, max_, words):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.zeros(elements, dtype=np.int32)
    lib().ora_unpack_update(elements, max_, _p(w, C.c_uint32), _p(out, C.c_int32))
    return out


def inv_update(elements, max_, energy_words, update_words):
    es = lib().ora_energy_size(elements, max_)
    e = np.ascontiguousarray(energy_words, dtype=np.uint32)
    u = np.ascontiguousarray(update_words, dtype=np.uint32)
    out = np.zeros(es, dtype=np.uint32)
    lib().ora_inv_update(elements, max_, _p(e, C.c_uint32), _p(u, C.c_uint32), _p(out, C.c_uint32))
    return out


class Solution:
    """Final energies of an oracle run: ``offsets[n+1]`` and ``data``."""

    def __init__(self, handle, n, esize):
        L = lib()
        total = L.ora_solution_total(handle)
        self.offsets = np.zeros(n + 1, dtype=np.uint64)
        self.data = np.zeros(int(total) * esize, dtype=np.uint32)
        L.ora_solution_offsets(handle, _p(self.offsets, C.c_uint64))
        if total:
            L.ora_solution_data(handle, _p(self.data, C.c_uint32))
        st = np.zeros(6, dtype=np.uint64)
        L.ora_solution_stats(handle, _p(st, C.c_uint64))
        self.stats = dict(zip(("rounds", "attack_visits", "defend_visits", "defend_retries",
                               "edges_relaxed", "bytes"), (int(x) for x in st)))
        L.ora_solution_free(handle)
        self.esize = esize

    def lists(self):
        """Per-position energy lists, each an (k, esize) uint32 array."""
        o = self.offsets
        es = self.esize
        return [self.data[int(o[v]) * es:int(o[v + 1]) * es].reshape(-1, es) for v in range(len(o) - 1)]


def run_game(elements, max_, row_offsets, col, weights, attacker, to_reach, init=None):
    """EnergyGame::run on a CSR graph.  ``init`` = (offsets[n+1], data) or None."""
    L = lib()
    row = np.ascontiguousarray(row_offsets, dtype=np.uint32)
    n = len(row) - 1
    col = np.ascontiguousarray(col, dtype=np.uint32)
    wt = np.ascontiguousarray(weights, dtype=np.uint32)
    att = np.ascontiguousarray(attacker, dtype=np.uint8)
    reach = np.ascontiguousarray(to_reach, dtype=np.uint32)
    if init is not None:
        io = np.ascontiguousarray(init[0], dtype=np.uint64)
        idata = np.ascontiguousarray(init[1], dtype=np.uint32)
        if idata.size == 0:
            idata = np.zeros(1, dtype=np.uint32)
        iop, idp = _p(io, C.c_uint64), _p(idata, C.c_uint32)
    else:
        iop, idp = None, None
    colp = col if col.size else np.zeros(1, dtype=np.uint32)
    wtp = wt if wt.size else np.zeros(1, dtype=np.uint32)
    attp = att if att.size else np.zeros(1, dtype=np.uint8)
    rp = reach if reach.size else np.zeros(1, dtype=np.uint32)
    h = L.ora_run_game(elements, max_, n, _p(row, C.c_uint32), _p(colp, C.c_uint32), _p(wtp, C.c_uint32),
                       _p(attp, C.c_uint8), iop, idp, _p(rp, C.c_uint32), len(reach))
    return Solution(h, n, L.ora_energy_size(elements, max_))


def standard_reach(row_offsets, attacker):
    row = np.ascontiguousarray(row_offsets, dtype=np.uint32)
    att = np.ascontiguousarray(attacker, dtype=np.uint8)
    n = len(row) - 1
    out = np.zeros(max(n, 1), dtype=np.uint32)
    c = lib().ora_standard_reach(n, _p(row, C.c_uint32), _p(att if att.size else np.zeros(1, np.uint8), C.c_uint8),
                                 _p(out, C.c_uint32))
    return out[:c].copy()


def defend_intersection(elements, max_, energies, succ_offsets, mem):
    es = lib().ora_energy_size(elements, max_)
    e = np.ascontiguousarray(energies, dtype=np.uint32)
    so = np.ascontiguousarray(succ_offsets, dtype=np.uint32)
    out = np.zeros(max(mem, 1) * es, dtype=np.uint32)
    st = lib().ora_defend_intersection(elements, max_, _p(e, C.c_uint32), _p(so, C.c_uint32),
                                       len(so) - 1, mem, _p(out, C.c_uint32))
    if st < 0:
        return st, None
    return st, out[:st * es].reshape(-1, es)


class Lts:
    """TransitionSystem of the oracle (owns a native handle)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_edges(cls, edges):
        e = np.asarray(edges, dtype=np.int64).reshape(-1, 3)
        src = np.ascontiguousarray(e[:, 0], dtype=np.uint32)
        dst = np.ascontiguousarray(e[:, 1], dtype=np.uint32)
        lab = np.ascontiguousarray(e[:, 2], dtype=np.int32)
        if len(e) == 0:
            src = dst = np.zeros(1, np.uint32)
            lab = np.zeros(1, np.int32)
        return cls(lib().ora_lts_from_edges(len(e), _p(src, C.c_uint32), _p(dst, C.c_uint32),
                                            _p(lab, C.c_int32)))

    @classmethod
    def from_arrays(cls, src, dst, lab):
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32)
        lab = np.ascontiguousarray(lab, dtype=np.int32)
        return cls(lib().ora_lts_from_edges(len(src), _p(src, C.c_uint32), _p(dst, C.c_uint32),
                                            _p(lab, C.c_int32)))

    @classmethod
    def from_csv(cls, path):
        err = C.c_int(0)
        h = lib().ora_lts_from_csv(path.encode(), C.byref(err))
        if not h:
            raise ValueError(f"csv error {err.value}")
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ora_lts_free(self.h)
            self.h = None

    @property
    def n_vertices(self):
        return lib().ora_lts_n_vertices(self.h)

    def transitions(self):
        n = self.n_vertices
        m = lib().ora_lts_n_transitions(self.h)
        off = np.zeros(n + 1, dtype=np.uint64)
        tg = np.zeros(max(m, 1), dtype=np.uint32)
        lb = np.zeros(max(m, 1), dtype=np.int32)
        lib().ora_lts_transitions(self.h, _p(off, C.c_uint64), _p(tg, C.c_uint32), _p(lb, C.c_int32))
        return off, tg[:m], lb[:m]

    def signature_refinement(self):
        n = self.n_vertices
        part = np.zeros(max(n, 1), dtype=np.uint64)
        cnt = lib().ora_lts_signature_refinement(self.h, _p(part, C.c_uint64))
        return part[:n], int(cnt)

    def bisimilar_minimize(self):
        n = self.n_vertices
        mapping = np.zeros(max(n, 1), dtype=np.uint64)
        h = lib().ora_lts_minimize(self.h, _p(mapping, C.c_uint64))
        return Lts(h), mapping[:n]


class Build:
    """GameBuild of the oracle: positions and the CSR game graph."""

    def __init__(self, handle, positions=True):
        L = lib()
        self.n = L.ora_build_n_nodes(handle)
        m = L.ora_build_n_edges(handle)
        self.n_starting = L.ora_build_n_starting(handle)
        self.row = np.zeros(self.n + 1, dtype=np.uint32)
        self.col = np.zeros(max(m, 1), dtype=np.uint32)
        self.wt = np.zeros(max(m, 1), dtype=np.uint32)
        self.attacker = np.zeros(max(self.n, 1), dtype=np.uint8)
        L.ora_build_graph(handle, _p(self.row, C.c_uint32), _p(self.col, C.c_uint32),
                          _p(self.wt, C.c_uint32), _p(self.attacker, C.c_uint8))
        self.col, self.wt, self.attacker = self.col[:m], self.wt[:m], self.attacker[:self.n]
        self.positions = []
        k, p, nq, nqx = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        for i in range(self.n if positions else 0):
            L.ora_build_position(handle, i, C.byref(k), C.byref(p), C.byref(nq), C.byref(nqx))
            q = np.zeros(max(nq.value, 1), dtype=np.uint32)
            qx = np.zeros(max(nqx.value, 1), dtype=np.uint32)
            L.ora_build_position_sets(handle, i, _p(q, C.c_uint32), _p(qx, C.c_uint32))
            self.positions.append((("attack", "clause", "defend")[k.value], p.value,
                                   tuple(int(x) for x in q[:nq.value]), tuple(int(x) for x in qx[:nqx.value])))
        L.ora_build_free(handle)

    @classmethod
    def compare(cls, lts: Lts, p: int, q: int, positions=True):
        """GameBuild::compare; positions=False skips reading the positions
        back (only the graph)."""
        return cls(lib().ora_build_compare(lts.h, p, q), positions)

    @classmethod
    def compare_all(cls, lts: Lts):
        return cls(lib().ora_build_compare_all(lts.h))

    def adj(self, v):
        return self.col[self.row[v]:self.row[v + 1]]


def compare_batch(lts_list, ps, qs, threads=1):
    n = len(lts_list)
    hs = (C.c_void_p * n)(*[l.h for l in lts_list])
    p = np.ascontiguousarray(ps, dtype=np.uint32)
    q = np.ascontiguousarray(qs, dtype=np.uint32)
    cnt = np.zeros(n, dtype=np.uint64)
    nodes = np.zeros(n, dtype=np.uint64)
    lib().ora_compare_batch(n, hs, _p(p, C.c_uint32), _p(q, C.c_uint32), threads,
                            _p(cnt, C.c_uint64), _p(nodes, C.c_uint64))
    return cnt, nodes


def _game_arrays(games):
    n = len(games)
    keep = []
    npos = np.array([len(g[0]) - 1 for g in games], dtype=np.uint32)
    rows = (u32p * n)()
    cols = (u32p * n)()
    wts = (u32p * n)()
    atts = (u8p * n)()
    for i, (r, c, w, a) in enumerate(games):
        r = np.ascontiguousarray(r, dtype=np.uint32)
        c = np.ascontiguousarray(c if len(c) else np.zeros(1), dtype=np.uint32)
        w = np.ascontiguousarray(w if len(w) else np.zeros(1), dtype=np.uint32)
        a = np.ascontiguousarray(a if len(a) else np.zeros(1), dtype=np.uint8)
        keep += [r, c, w, a]
        rows[i], cols[i], wts[i], atts[i] = _p(r, C.c_uint32), _p(c, C.c_uint32), _p(w, C.c_uint32), _p(a, C.c_uint8)
    return npos, rows, cols, wts, atts, keep


def solve_games(games, threads=1, largest_first=False, elements=6, max_=3):
    """Oracle solve of many games (standard reach) on `threads` threads that
    share one work counter (largest games first when asked, so that one big
    game does not end up last).  Returns one Solution per game."""
    n = len(games)
    if n == 0:
        return []
    npos, rows, cols, wts, atts, keep = _game_arrays(games)
    order = None
    if largest_first:
        size = np.array([len(g[1]) + len(g[0]) for g in games], dtype=np.int64)
        order = np.ascontiguousarray(np.argsort(-size, kind="stable"), dtype=np.uint32)
    handles = (C.c_void_p * n)()
    lib().ora_solve_games(n, elements, max_, _p(npos, C.c_uint32), rows, cols, wts, atts, threads,
                          None if order is None else _p(order, C.c_uint32), None, handles)
    es = lib().ora_energy_size(elements, max_)
    return [Solution(handles[i], int(npos[i]), es) for i in range(n)]


def b_min(row_offsets, col, offsets):
    """The schedule-independent byte floor 4(n+1) + 8m + n + sum_v 4|A*_v|(1 +
    indeg(v)) of a game from its final list offsets (STANDARD conf)."""
    r = np.ascontiguousarray(row_offsets, dtype=np.uint32)
    c = np.ascontiguousarray(col if len(col) else np.zeros(1), dtype=np.uint32)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    return int(lib().ora_b_min(len(r) - 1, _p(r, C.c_uint32), _p(c, C.c_uint32), _p(o, C.c_uint64)))


def run_games_parallel(games, threads=1, elements=6, max_=3):
    """games: list of (row, col, wt, attacker) CSR arrays; standard reach."""
    n = len(games)
    keep = []
    npos = np.array([len(g[0]) - 1 for g in games], dtype=np.uint32)
    rows = (u32p * n)()
    cols = (u32p * n)()
    wts = (u32p * n)()
    atts = (u8p * n)()
    for i, (r, c, w, a) in enumerate(games):
        r = np.ascontiguousarray(r, dtype=np.uint32)
        c = np.ascontiguousarray(c if len(c) else np.zeros(1), dtype=np.uint32)
        w = np.ascontiguousarray(w if len(w) else np.zeros(1), dtype=np.uint32)
        a = np.ascontiguousarray(a if len(a) else np.zeros(1), dtype=np.uint8)
        keep += [r, c, w, a]
        rows[i], cols[i], wts[i], atts[i] = _p(r, C.c_uint32), _p(c, C.c_uint32), _p(w, C.c_uint32), _p(a, C.c_uint8)
    out = np.zeros(n, dtype=np.uint64)
    lib().ora_run_games_parallel(n, elements, max_, _p(npos, C.c_uint32), rows, cols, wts, atts, threads,
                                 _p(out, C.c_uint64))
    return out


def check_fixpoint(row, col, wt, att, offsets, data, threads=0, elements=6, max_=3):
    """(count, first) of positions whose list one more worklist step would
    change; (0, None) when the lists are a fixpoint (test support for sizes
    the sequential solve would take too long for)."""
    import os
    r = np.ascontiguousarray(row, dtype=np.uint32)
    c = np.ascontiguousarray(col if len(col) else np.zeros(1), dtype=np.uint32)
    w = np.ascontiguousarray(wt if len(wt) else np.zeros(1), dtype=np.uint32)
    a = np.ascontiguousarray(att, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    d = np.ascontiguousarray(data if len(data) else np.zeros(1), dtype=np.uint32)
    first = C.c_uint32(0)
    n_bad = lib().ora_check_fixpoint(elements, max_, len(r) - 1, _p(r, C.c_uint32), _p(c, C.c_uint32),
                                     _p(w, C.c_uint32), _p(a, C.c_uint8), _p(o, C.c_uint64), _p(d, C.c_uint32),
                                     threads or (os.cpu_count() or 1), C.byref(first))
    return int(n_bad), (None if n_bad == 0 else int(first.value))


# ---------------------------------------------------------------------------
# Verdicts: restatement of src/equivalence.rs and EnergyArray::test_equivalence
# (src/energy.rs:307-318) for small cases.
# ---------------------------------------------------------------------------
def test_equivalence(lists_packed, eq_values, elements=6, max_=3):
    """True iff no energy of the list is <= the equivalence tuple (energy.rs:317)."""
    eq = list(eq_values) + [0] * (elements - len(eq_values))
    for row in np.asarray(lists_packed, dtype=np.uint32).reshape(-1, lib().ora_energy_size(elements, max_)):
        vals = unpack_energy(elements, max_, row)
        if all(int(a) <= b for a, b in zip(vals, eq)):
            return False
    return True


def compare(lts: Lts, p: int, q: int):
    """TransitionSystem::compare (lib.rs:275-296): energies of Attack(p,{q})."""
    red, mapping = lts.bisimilar_minimize()
    pm, qm = int(mapping[p]), int(mapping[q])
    if pm == qm:
        return np.zeros((0, 1), dtype=np.uint32)
    b = Build.compare(red, pm, qm)
    reach = standard_reach(b.row, b.attacker)
    sol = run_game(6, 3, b.row, b.col, b.wt, b.attacker, reach)
    return sol.lists()[0]


class _UnionFind:
    def __init__(self, n):
        self.parent = list(range(n))

    def find(self, x):
        while self.parent[x] != x:
            self.parent[x] = self.parent[self.parent[x]]
            x = self.parent[x]
        return x

    def union(self, a, b):
        ra, rb = self.find(a), self.find(b)
        if ra != rb:
            self.parent[max(ra, rb)] = min(ra, rb)


class Relation:
    """EquivalenceRelation (equivalence.rs:180-247)."""

    def __init__(self, uf: _UnionFind):
        self.uf = uf

    def __len__(self):
        return len(self.uf.parent)

    def count_classes(self):
        return len({self.uf.find(i) for i in range(len(self))})

    def class_of(self, p):
        c = self.uf.find(p)
        return [i for i in range(len(self)) if self.uf.find(i) == c]

    def get_classes(self):
        order, classes = {}, []
        for i in range(len(self)):
            c = self.uf.find(i)
            if c not in order:
                order[c] = len(classes)
                classes.append([])
            classes[order[c]].append(i)
        return classes

    def with_mapping(self, mapping):
        uf = _UnionFind(len(mapping))
        rep = {}
        for proc, m in enumerate(mapping):
            part = self.uf.find(int(m))
            if part in rep:
                uf.union(proc, rep[part])
            else:
                rep[part] = proc
        return Relation(uf)


class Equivalence:
    """Equivalence (equivalence.rs:41-175) over oracle energies."""

    def __init__(self, starting_points, energies, n_processes, minimization=None):
        self.starting_points = list(starting_points)
        self.energies = list(energies[:len(self.starting_points)])
        self.n_processes = n_processes
        self.pos_to_idx = {sp: i for i, sp in enumerate(self.starting_points)}
        self.minimization = minimization

    def _mapped(self, p):
        return int(self.minimization[p]) if self.minimization is not None else p

    def energies_minimized(self, p, q):
        idx = self.pos_to_idx.get((p, q))
        return None if idx is None else self.energies[idx]

    def energies_of(self, p, q):
        return self.energies_minimized(self._mapped(p), self._mapped(q))

    def preorder(self, p, q, eq_values):
        p, q = self._mapped(p), self._mapped(q)
        if p == q:
            return True
        e = self.energies_minimized(p, q)
        return e is not None and test_equivalence(e, eq_values)

    def equiv(self, p, q, eq_values):
        return self.preorder(p, q, eq_values) and self.preorder(q, p, eq_values)

    def relation(self, eq_values):
        uf = _UnionFind(self.n_processes)
        for (p, q), e in zip(self.starting_points, self.energies):
            e2 = self.energies_minimized(q, p)
            if test_equivalence(e, eq_values) and test_equivalence(e2, eq_values):
                uf.union(p, q)
        rel = Relation(uf)
        return rel.with_mapping(self.minimization) if self.minimization is not None else rel


def equivalences(lts: Lts, minimize=True):
    """TransitionSystem::equivalences / equivalences_unminimized (lib.rs:329-343)."""
    if minimize:
        red, mapping = lts.bisimilar_minimize()
    else:
        red, mapping = lts, None
    b = Build.compare_all(red)
    reach = standard_reach(b.row, b.attacker)
    sol = run_game(6, 3, b.row, b.col, b.wt, b.attacker, reach)
    starts = [(pos[1], pos[2][0]) for pos in b.positions[:b.n_starting]]
    return Equivalence(starts, sol.lists(), red.n_vertices, mapping)
