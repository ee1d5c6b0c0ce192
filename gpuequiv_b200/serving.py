"""The serving loop (``geq_server_*``): submit games, poll for their lists.

Requests are queued and solved in batches by pipeline threads inside
libgeq, each with its own CUDA stream, while the caller keeps submitting
(continuous batching).  A result equals ``EnergyGame.standard_reach(graph).run()``
of the same game.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import GeqError, check, geq_server_config, geq_server_stats, lib
from .energygame import Context, GameGraph, _borrow, _SolutionOwner, _stats_of, default_context

TIMEOUT = 4  # GEQ_ERR_TIMEOUT


class Server:
    """geq_server: ``submit(graph)`` / ``submit_compare(lts, p, q) -> ticket``,
    ``poll(ticket, timeout_ms)``."""

    def __init__(self, context: Context | None = None, n_pipelines: int = 0, max_batch_games: int = 0,
                 max_wait_us: int = 0, hbm_budget_bytes: int = 0, max_queued: int = 0, max_game_positions: int = 0):
        """max_game_positions: a compare query whose game would have more
        positions fails alone with OUT_OF_MEMORY (0: no bound)."""
        ctx = context or default_context()
        cfg = geq_server_config(n_pipelines, max_batch_games, max_wait_us, max_game_positions, hbm_budget_bytes,
                                max_queued)
        h = C.c_void_p()
        check(lib.geq_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h

    def submit(self, graph: GameGraph) -> int:
        """Queue one game (copied by the library); returns its ticket."""
        t = C.c_uint64()
        view = graph.c_view()
        check(lib.geq_server_submit(self.h, C.byref(view), C.byref(t)))
        return t.value

    def submit_compare(self, lts, p: int, q: int) -> int:
        """Queue one ``TransitionSystem.compare(p, q)`` query (the LTS is
        copied); its result is the start position's energies, as
        ``lts.compare(p, q)``."""
        t = C.c_uint64()
        check(lib.geq_server_submit_compare(self.h, lts.h, int(p), int(q), C.byref(t)))
        return t.value

    def poll(self, ticket: int, timeout_ms: int = -1):
        """(offsets, data, stats) of the request, or None if it is not done
        within timeout_ms (< 0: wait).  Arrays view the solution's memory."""
        sol = C.c_void_p()
        st = lib.geq_server_poll(self.h, ticket, timeout_ms, C.byref(sol))
        if st == TIMEOUT:
            return None
        check(st)
        owner = _SolutionOwner(sol)
        po, pd = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
        no, nw = C.c_uint64(), C.c_uint64()
        check(lib.geq_solution_flat(sol, C.byref(po), C.byref(no), C.byref(pd), C.byref(nw)))
        return (_borrow(po, no.value, C.c_uint64, np.uint64, owner),
                _borrow(pd, nw.value, C.c_uint32, np.uint32, owner), _stats_of(sol))

    def poll_any(self, timeout_ms: int = -1):
        """(ticket, (offsets, data, stats)) of whichever request finished
        first, or None if none finishes within timeout_ms (< 0: wait).  A
        failed request raises GeqError (its ticket in ``.ticket``)."""
        sol = C.c_void_p()
        t = C.c_uint64()
        st = lib.geq_server_poll_any(self.h, timeout_ms, C.byref(t), C.byref(sol))
        if st == TIMEOUT and t.value == 0:
            return None
        try:
            check(st)
        except GeqError as e:
            e.ticket = t.value
            raise
        owner = _SolutionOwner(sol)
        po, pd = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)()
        no, nw = C.c_uint64(), C.c_uint64()
        check(lib.geq_solution_flat(sol, C.byref(po), C.byref(no), C.byref(pd), C.byref(nw)))
        return t.value, (_borrow(po, no.value, C.c_uint64, np.uint64, owner),
                         _borrow(pd, nw.value, C.c_uint32, np.uint32, owner), _stats_of(sol))

    def stats(self) -> dict:
        st = geq_server_stats()
        lib.geq_server_get_stats(self.h, C.byref(st))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib.geq_server_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Server", "GeqError"]
