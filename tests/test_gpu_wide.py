"""The multi-word solver (wide.cu): EnergyConfs without a thermometer codec
-- several energy words ({30, 3}, {16, 7}, {100, 1}), 32-bit fields
(ONE_DIMENSION = {1, u32::MAX}, energy.rs:46), fields of 16 bits ({3, 1000}),
several update words -- against the oracle, which restates the arithmetic
shadergen.rs:55-157 generates for any conf.  The same solver forced onto
STANDARD and SILENT_STEP games is checked against the thermometer-codec path
and the reference's own known answers.  Lists are compared as sorted
multisets of packed energies (EnergyArray equality is set equality)."""
from __future__ import annotations

import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import canon, csr_from_edges, earray, ref_eq
from oracle import ora

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


@pytest.fixture(scope="module")
def ctx_wide(geq):
    from gpuequiv_b200._lib import TUNE_FORCE_WIDE
    c = geq.Context(0)
    c.set_tuning(flags=TUNE_FORCE_WIDE)
    yield c
    c.close()


def random_update(rng, el):
    u = [0] * el
    r = rng.random()
    if r < 0.4:
        return u
    pos = int(rng.integers(el))
    if r < 0.75 or el == 1:
        u[pos] = -1
    else:
        t = int(rng.integers(1, el))  # Min(k), 1-indexed, k != pos + 1
        if t >= pos + 1:
            t += 1
        u[pos] = t
    if rng.random() < 0.15:  # a second component
        u[int(rng.integers(el))] = -1
    return u


def random_game(seed, n, conf, avg_deg=2.2, p_att=0.6, bipartite=True):
    rng = np.random.default_rng(seed)
    el = conf[0]
    att = rng.random(n) < p_att
    A, D = np.nonzero(att)[0], np.nonzero(~att)[0]
    edges = []
    for v in range(n):
        pool = (D if att[v] else A) if bipartite else np.arange(n)
        deg = int(rng.geometric(1.0 / avg_deg)) - (0 if att[v] else 1)
        for _ in range(max(deg, 0) if len(pool) else 0):
            edges.append((v, int(pool[rng.integers(len(pool))]), random_update(rng, el)))
    return csr_from_edges(n, edges, att, conf=conf)


def solve(geq, ctx, conf, row, col, wt, att, to_reach=None, init=None):
    C = geq.EnergyConf(*conf)
    g = geq.GameGraph.from_csr(row, col, wt, att, C)
    reach = g.standard_reach() if to_reach is None else to_reach
    if init is None:
        game = geq.EnergyGame.with_reach(g, reach)
    else:
        game = geq.EnergyGame(g, [geq.EnergyArray(a, C) for a in init], reach)
    return [r.array for r in game.run(ctx)], game.stats


def oracle(conf, row, col, wt, att, to_reach=None, init=None):
    reach = ora.standard_reach(row, att) if to_reach is None else np.asarray(to_reach, np.uint32)
    iarg = None
    if init is not None:
        offs = np.zeros(len(init) + 1, np.uint64)
        offs[1:] = np.cumsum([len(a) for a in init])
        data = (np.concatenate([np.asarray(a, np.uint32).reshape(-1) for a in init]) if offs[-1]
                else np.zeros(0, np.uint32))
        iarg = (offs, data)
    return ora.run_game(conf[0], conf[1], row, col, np.asarray(wt).reshape(-1), att, reach, init=iarg).lists()


def assert_parity(got, exp, what):
    assert len(got) == len(exp)
    for v, (g, e) in enumerate(zip(got, exp)):
        assert canon(g) == canon(e), f"{what}: position {v}: gpu {canon(g)} oracle {canon(e)}"


CONFS = [(1, 0xFFFFFFFF), (30, 3), (3, 1000), (16, 7), (100, 1), (2, 65535)]


def test_confs_take_the_multiword_solver(geq):
    for conf in CONFS:
        C = geq.EnergyConf(*conf)
        assert not C.supported() and C.solvable(), conf
    assert geq.EnergyConf(30, 3).energy_size() == 2 and geq.EnergyConf(30, 3).update_size() == 8
    assert not geq.EnergyConf(300, 0xFFFFFFFF).solvable()


@pytest.mark.parametrize("conf", CONFS)
@pytest.mark.parametrize("seed,n,bip", [(1, 40, True), (2, 400, True), (3, 1500, True), (4, 300, False)])
def test_random_games_vs_oracle(geq, ctx, conf, seed, n, bip):
    row, col, wt, att = random_game(seed * 7 + conf[0], n, conf, bipartite=bip)
    got, stats = solve(geq, ctx, conf, row, col, wt, att)
    assert_parity(got, oracle(conf, row, col, wt, att), f"conf {conf} seed {seed}")
    assert stats["kernel_launches"] > 0


def test_one_dimension_wraps_like_u32(geq, ctx):
    """ONE_DIMENSION: +1 on a 32-bit field is u32 arithmetic, so a decrement
    edge maps u32::MAX to 0 before the min with max (UPDATE1,
    shadergen.rs:103-111); explicit initial lists carry u32::MAX."""
    conf = (1, 0xFFFFFFFF)
    dec = [-1]
    # 0 (att) -> 1 (def) -> 2 (att, own list {u32::MAX}) ; 0 -> 3 (def sink)
    row, col, wt, att = csr_from_edges(4, [(0, 1, dec), (1, 2, dec), (0, 3, [0])], [1, 0, 1, 0], conf=conf)
    init = [np.zeros((0, 1), np.uint32), np.zeros((0, 1), np.uint32),
            np.array([[0xFFFFFFFF]], np.uint32), np.array([[5]], np.uint32)]
    reach = np.array([2, 3], np.uint32)
    got, _ = solve(geq, ctx, conf, row, col, wt, att, to_reach=reach, init=init)
    exp = oracle(conf, row, col, wt, att, to_reach=reach, init=init)
    assert_parity(got, exp, "one dimension, wrap")
    assert canon(got[1]) == [(0,)]  # u32::MAX + 1 wraps to 0


def test_forced_onto_standard_matches_codec_path(geq, ctx, ctx_wide):
    """STANDARD and SILENT_STEP games through the multi-word solver equal the
    thermometer-codec path and the oracle; the reference's known answers of
    tests/energygame.rs hold."""
    att = [i in G.SIMPLE_ATTACKERS for i in range(18)]
    got, st = solve(geq, ctx_wide, (6, 3), *csr_from_edges(18, G.SIMPLE_EDGES, att))
    for v, (g, rows) in enumerate(zip(got, G.SIMPLE_EXPECTED)):
        assert ref_eq(g, earray(rows)), f"simple: position {v}"
    c = G.COMBINATIONS
    att = [i in c["attackers"] for i in range(c["n"])]
    got, _ = solve(geq, ctx_wide, (6, 3), *csr_from_edges(c["n"], c["edges"], att))
    for v, (g, rows) in enumerate(zip(got, c["expected"])):
        assert ref_eq(g, earray(rows)), f"combinations: position {v}"
    for conf, seeds in (((6, 3), (11, 12, 13)), ((8, 2), (14, 15))):
        for seed in seeds:
            row, col, wt, att = random_game(seed, 1200, conf)
            a, _ = solve(geq, ctx_wide, conf, row, col, wt, att)
            b, _ = solve(geq, ctx, conf, row, col, wt, att)
            assert_parity(a, b, f"forced wide vs codec, conf {conf} seed {seed}")
            assert_parity(a, oracle(conf, row, col, wt, att), f"forced wide vs oracle, conf {conf} seed {seed}")


def test_forced_onto_spectroscopy_games(geq, ctx, ctx_wide):
    """GameBuild games of the batched workload (defenders with many
    successors and wide antichains) through the multi-word solver."""
    from gpuequiv_b200 import synth
    rows = synth.batched_manifest()["jobs"]
    for seed, npos, _ in [r for r in rows if 200 <= r[1] <= 20_000][:6]:
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        g = geq.GameBuild.compare(red, int(mp[p]), int(mp[q])).game
        a = geq.EnergyGame.standard_reach(g).run(ctx_wide)
        offs, data, _ = geq.run_batch_raw([g], ctx)
        for v in range(npos):
            assert canon(a[v].array) == canon(data[0][offs[0][v]:offs[0][v + 1]]), f"seed {seed} position {v}"


def test_batch_and_server_take_wide_games(geq, ctx):
    """run_batch of several wide games and the serving loop's game requests."""
    from gpuequiv_b200.serving import Server
    conf = (30, 3)
    C = geq.EnergyConf(*conf)
    games = [random_game(50 + i, 200 + 50 * i, conf) for i in range(4)]
    graphs = [geq.GameGraph.from_csr(r, c, w, a, C) for r, c, w, a in games]
    lists, _ = geq.run_batch(graphs, ctx)
    exp = [oracle(conf, *g) for g in games]
    for i in range(len(games)):
        assert_parity([x.array for x in lists[i]], exp[i], f"batch game {i}")
    with Server(ctx, n_pipelines=1) as srv:
        tickets = [srv.submit(g) for g in graphs]
        for i, t in enumerate(tickets):
            offs, data, _ = srv.poll(t, timeout_ms=120_000)
            es = C.energy_size()
            got = [data[int(offs[v]) * es:int(offs[v + 1]) * es].reshape(-1, es) for v in range(len(offs) - 1)]
            assert_parity(got, exp[i], f"served game {i}")
