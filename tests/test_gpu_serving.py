"""The serving loop (geq_server_*): every result, solved in a mix of
concurrently submitted requests, equals the same game solved alone."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import csr_from_edges

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def geq():
    import gpuequiv_b200 as geq
    return geq


@pytest.fixture(scope="module")
def ctx(geq):
    c = geq.Context(0)
    yield c
    c.close()


def _canon(offs, data):
    offs = np.asarray(offs, np.int64)
    return [tuple(sorted(int(x) for x in data[offs[v]:offs[v + 1]])) for v in range(len(offs) - 1)]


def _games(geq, n):
    from gpuequiv_b200 import synth
    rows = synth.batched_manifest()["jobs"]
    seeds = [r[0] for r in rows if r[1] <= 60_000][:n]
    out = []
    for seed in seeds:
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        out.append(geq.GameBuild.compare(red, int(mp[p]), int(mp[q])).game)
    return out


def _alone(geq, ctx, g):
    offs, data, _ = geq.run_batch_raw([g], ctx)
    return _canon(offs[0], data[0])


def test_results_alone_equal_in_the_mix(geq, ctx):
    from gpuequiv_b200.serving import Server
    games = _games(geq, 160)
    expect = [_alone(geq, ctx, g) for g in games]
    with Server(ctx, n_pipelines=2, max_wait_us=500) as srv:
        # submissions interleaved with polls: batches start while requests keep arriving
        tickets = []
        got = {}
        for i, g in enumerate(games):
            tickets.append(srv.submit(g))
            if i % 16 == 15:
                r = srv.poll(tickets[i - 15], timeout_ms=0)
                if r is not None:
                    got[i - 15] = _canon(r[0], r[1])
        for i, t in enumerate(tickets):
            if i not in got:
                r = srv.poll(t, timeout_ms=60_000)
                assert r is not None, f"request {i} not done"
                got[i] = _canon(r[0], r[1])
        st = srv.stats()
    for i in range(len(games)):
        assert got[i] == expect[i], f"game {i} differs from its solve alone"
    assert st["completed"] == len(games) and st["failed"] == 0
    assert st["games_in_batches"] == len(games)


def test_admission_budget_splits_batches(geq, ctx):
    from gpuequiv_b200.serving import Server
    games = _games(geq, 40)
    expect = [_alone(geq, ctx, g) for g in games]
    budget = 2 * (40 << 20)  # two pipelines, about 40 MB each: several batches
    with Server(ctx, n_pipelines=2, hbm_budget_bytes=budget, max_wait_us=2000) as srv:
        tickets = [srv.submit(g) for g in games]
        got = [_canon(*srv.poll(t)[:2]) for t in tickets]
        st = srv.stats()
    assert got == expect
    assert st["batches"] > 1
    assert st["max_batch_footprint"] <= budget // 2 or st["games_in_batches"] == st["batches"]


def test_faulty_request_fails_alone(geq, ctx):
    from gpuequiv_b200 import GeqError
    from gpuequiv_b200.serving import Server
    games = _games(geq, 6)
    expect = [_alone(geq, ctx, g) for g in games]
    # a successor index beyond the game: caught on the device at upload
    row, col, wt, att = csr_from_edges(3, [(0, 1, [-1]), (1, 2, [0])], [True, False, False])
    col = np.array(col, np.uint32)
    col[1] = 7
    bad = geq.GameGraph.from_csr(row, col, wt, att, geq.EnergyConf(6, 3))
    with Server(ctx, n_pipelines=1, max_wait_us=20_000) as srv:
        tickets = [srv.submit(g) for g in games[:3]] + [srv.submit(bad)] + [srv.submit(g) for g in games[3:]]
        results = []
        for t in tickets:
            try:
                r = srv.poll(t)
                results.append(_canon(r[0], r[1]))
            except GeqError as e:
                results.append(e.name)
    assert results[3] == "INVALID_INPUT"
    assert results[:3] + results[4:] == expect


def test_unknown_ticket_and_busy(geq, ctx):
    from gpuequiv_b200 import GeqError
    from gpuequiv_b200.serving import Server
    with Server(ctx, n_pipelines=1) as srv:
        with pytest.raises(GeqError) as e:
            srv.poll(12345, timeout_ms=0)
        assert e.value.name == "INVALID_INPUT"


def test_compare_queries_alone_equal_in_the_mix(geq, ctx):
    """LTS equivalence queries (geq_server_submit_compare) mixed with game
    requests: each query's energies equal compare() of the query alone and
    the oracle's TransitionSystem::compare; bisimilar pairs give no energies."""
    from gpuequiv_b200 import synth
    from gpuequiv_b200.serving import Server
    from helpers import random_lts
    from oracle import ora
    queries, oracle_of = [], {}
    for seed, npos, _ in synth.batched_manifest()["jobs"][:400]:
        if npos <= 20_000 and len(queries) < 96:
            src, dst, lab, p, q = synth.batched_lts(seed)
            queries.append((geq.TransitionSystem.from_arrays(src, dst, lab), int(p), int(q)))
    rng = np.random.default_rng(31)
    for k in range(24):
        n = int(rng.integers(2, 10))
        edges = random_lts(rng, n, 2, int(rng.integers(n, 2 * n + 1)))
        lts = geq.TransitionSystem(edges)
        p = int(rng.integers(0, lts.n_vertices()))
        q = p if k % 6 == 0 else int(rng.integers(0, lts.n_vertices()))
        oracle_of[len(queries)] = ora.compare(ora.Lts.from_edges(edges), p, q)
        queries.append((lts, p, q))
    alone = [sorted(int(x) for x in np.asarray(geq.compare_batch([qq], context=ctx)[0].array).reshape(-1))
             for qq in queries]
    games = _games(geq, 16)
    with Server(ctx, n_pipelines=2, max_wait_us=1000) as srv:
        tickets = []
        for i, (lts, p, q) in enumerate(queries):
            tickets.append(srv.submit_compare(lts, p, q))
            if i % 8 == 0:
                srv.submit(games[(i // 8) % len(games)])
        got = []
        for t in tickets:
            offs, data, _ = srv.poll(t, timeout_ms=120_000)
            assert len(offs) == 2
            got.append(sorted(int(x) for x in data[int(offs[0]):int(offs[1])]))
        st = srv.stats()
    assert got == alone
    for i, ref in oracle_of.items():
        assert got[i] == sorted(int(x) for x in np.asarray(ref).reshape(-1)), i
    assert st["failed"] == 0


def test_compare_query_position_bound(geq, ctx):
    """With max_game_positions, a query whose game would be larger fails alone
    (OUT_OF_MEMORY) while the queries of its batch that fit are answered as
    compare() alone answers them."""
    from gpuequiv_b200 import GeqError, synth
    from gpuequiv_b200.serving import Server
    rows = synth.batched_manifest()["jobs"]
    big = [r for r in rows if r[1] > 50_000][:2]
    small = [r for r in rows if r[1] <= 5_000][:12]
    bound = 20_000
    jobs = []
    for seed, npos, _ in small[:6] + big[:1] + small[6:] + big[1:]:
        src, dst, lab, p, q = synth.batched_lts(seed)
        jobs.append((geq.TransitionSystem.from_arrays(src, dst, lab), int(p), int(q), npos > bound))
    alone = {i: sorted(int(x) for x in np.asarray(geq.compare_batch([j[:3]], context=ctx)[0].array).reshape(-1))
             for i, j in enumerate(jobs) if not j[3]}
    with Server(ctx, n_pipelines=1, max_wait_us=20_000, max_game_positions=bound) as srv:
        tickets = [srv.submit_compare(*j[:3]) for j in jobs]
        for i, (t, j) in enumerate(zip(tickets, jobs)):
            if j[3]:
                with pytest.raises(GeqError) as e:
                    srv.poll(t, timeout_ms=120_000)
                assert e.value.name == "OUT_OF_MEMORY"
            else:
                offs, data, _ = srv.poll(t, timeout_ms=120_000)
                assert sorted(int(x) for x in data[int(offs[0]):int(offs[1])]) == alone[i], i
        st = srv.stats()
    assert st["failed"] == 2 and st["completed"] == len(jobs) - 2


def test_games_retire_at_their_own_fixpoint(geq, ctx):
    """Games of one resident batch are answered when their own part of the
    frontier empties: a small game solved beside a deep one comes back after
    fewer rounds than the deep one (the rounds its batch had run when it was
    read back), and every list equals the game solved alone and the oracle."""
    from gpuequiv_b200 import synth
    from gpuequiv_b200.serving import Server
    from oracle import ora
    rows = synth.batched_manifest()["jobs"]

    def game(seed):
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        return geq.GameBuild.compare(red, int(mp[p]), int(mp[q])).game

    def alone_rounds(g):
        return geq.run_batch_raw([g], ctx)[2]["rounds"]

    R = ctx.tuning()["rounds_per_graph"]
    deep = next(g for g in (game(r[0]) for r in sorted(rows[:800], key=lambda r: -r[1])[:40])
                if alone_rounds(g) >= 3 * R)
    small = [g for g in (game(r[0]) for r in rows[:400] if 30 <= r[1] <= 400) if alone_rounds(g) < R][:24]
    assert len(small) >= 8
    games = [deep] + small
    expect = [_alone(geq, ctx, g) for g in games]
    with Server(ctx, n_pipelines=1, max_wait_us=50_000) as srv:
        tickets = [srv.submit(g) for g in games]
        res = [srv.poll(t, timeout_ms=120_000) for t in tickets]
        st = srv.stats()
    assert st["batches"] == 1 and st["failed"] == 0
    rounds = [r[2]["rounds"] for r in res]
    assert max(rounds[1:]) < rounds[0], rounds
    for i, (g, (offs, data, _)) in enumerate(zip(games, res)):
        assert _canon(offs, data) == expect[i], i
    for i in (1, 2, 3):
        g = games[i]
        sol = ora.run_game(6, 3, g.row_offsets, g.column_indices, g.weights.array.reshape(-1), g.attacker_pos,
                           ora.standard_reach(g.row_offsets, g.attacker_pos))
        assert _canon(sol.offsets, sol.data) == expect[i], i


def test_requests_admitted_while_batches_run(geq, ctx):
    """Requests submitted while earlier batches are resident join as new
    batches between steps; all results equal the games solved alone."""
    from gpuequiv_b200.serving import Server
    games = _games(geq, 200)
    expect = [_alone(geq, ctx, g) for g in games]
    with Server(ctx, n_pipelines=1, max_wait_us=100) as srv:
        tickets = []
        for k in range(0, len(games), 25):
            tickets += [srv.submit(g) for g in games[k:k + 25]]
        got = [srv.poll(t, timeout_ms=120_000) for t in tickets]
        st = srv.stats()
    assert st["failed"] == 0 and st["completed"] == len(games)
    for i, (offs, data, _) in enumerate(got):
        assert _canon(offs, data) == expect[i], i


def test_poll_any_returns_each_request_once(geq, ctx):
    """The completion queue (geq_server_poll_any) hands out every request
    exactly once, in the order they finish, with the lists of the game solved
    alone; a ticket taken by geq_server_poll is not handed out again."""
    from gpuequiv_b200.serving import Server
    games = _games(geq, 60)
    expect = [_alone(geq, ctx, g) for g in games]
    with Server(ctx, n_pipelines=2, max_wait_us=300) as srv:
        tickets = [srv.submit(g) for g in games]
        first = srv.poll(tickets[0], timeout_ms=60_000)
        got = {tickets[0]: _canon(first[0], first[1])}
        while len(got) < len(games):
            r = srv.poll_any(timeout_ms=60_000)
            assert r is not None
            t, (offs, data, _) = r
            assert t not in got
            got[t] = _canon(offs, data)
        assert srv.poll_any(timeout_ms=0) is None
    for i, t in enumerate(tickets):
        assert got[t] == expect[i], i
