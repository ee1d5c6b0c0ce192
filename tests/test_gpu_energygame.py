"""CUDA path vs the oracle and the reference's known answers (EnergyGame::run).

Every case runs under several solver modes so that each kernel path is
checked: the default (lane-per-position path, warp register paths, 4096-bit
bitmap paths, CUDA graphs), the warp paths only, the bitmap/list paths only,
the generic codec (with and without the register paths), and round-by-round
launches.
Bit-exact: per-position energy lists are compared as sorted multisets.
"""
import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import canon, csr_from_edges, earray, pack_u, ref_eq
from oracle import ora

pytestmark = pytest.mark.gpu

MODES = {
    "default": dict(),
    "warp": dict(flags=16),
    "large": dict(flags=2),
    "generic": dict(flags=1),
    "generic_large": dict(flags=3),
    "nograph": dict(flags=4),
    # every register budget of the round kernel
    "bps2": dict(blocks_per_sm=2, rounds_per_graph=3),
    "bps5": dict(blocks_per_sm=5, rounds_per_graph=16),
    # tighter lane-path limits: more positions take the warp routines
    "lanes_small": dict(lane_limits=(4, 8, 4)),
    # defenders pushed only once every successor has energies
    "ready": dict(flags=256),
}


@pytest.fixture(scope="module")
def geq():
    import gpuequiv_b200 as geq
    return geq


@pytest.fixture(scope="module", params=list(MODES))
def ctx(request, geq):
    c = geq.Context(0)
    c.set_tuning(**MODES[request.param])
    yield c
    c.close()


def gpu_run(geq, ctx, row, col, wt, att, to_reach=None, init=None, conf=(6, 3)):
    C = geq.EnergyConf(*conf)
    g = geq.GameGraph.from_csr(row, col, wt, att, C)
    if init is None:
        game = geq.EnergyGame.with_reach(g, g.standard_reach() if to_reach is None else to_reach)
    else:
        game = geq.EnergyGame(g, [geq.EnergyArray(a, C) for a in init],
                              g.standard_reach() if to_reach is None else to_reach)
    res = game.run(ctx)
    return [r.array for r in res], game.stats


def oracle_run(row, col, wt, att, to_reach=None, init=None, conf=(6, 3)):
    reach = ora.standard_reach(row, att) if to_reach is None else np.asarray(to_reach, np.uint32)
    iarg = None
    if init is not None:
        offs = np.zeros(len(init) + 1, np.uint64)
        offs[1:] = np.cumsum([len(a) for a in init])
        data = np.concatenate([np.asarray(a, np.uint32).reshape(-1) for a in init]) if offs[-1] else np.zeros(0, np.uint32)
        iarg = (offs, data)
    return ora.run_game(conf[0], conf[1], row, col, wt, att, reach, init=iarg).lists()


def assert_parity(got, exp, what):
    assert len(got) == len(exp)
    for v, (g, e) in enumerate(zip(got, exp)):
        assert canon(g) == canon(e), f"{what}: position {v}: gpu {canon(g)} oracle {canon(e)}"


def check_expected(got, expected_values, what):
    for v, (g, rows) in enumerate(zip(got, expected_values)):
        e = earray(rows)
        assert ref_eq(g, e), f"{what}: position {v}: {canon(g)} != {canon(e)}"


def _simple():
    att = [i in G.SIMPLE_ATTACKERS for i in range(18)]
    return csr_from_edges(18, G.SIMPLE_EDGES, att)


def test_simple(geq, ctx):
    got, _ = gpu_run(geq, ctx, *_simple())
    check_expected(got, G.SIMPLE_EXPECTED, "simple")
    assert_parity(got, oracle_run(*_simple()), "simple")


def test_simple_one_dimension(geq, ctx):
    row, col, wt, att = _simple()
    wt = np.full_like(wt, pack_u([-1])[0])
    got, _ = gpu_run(geq, ctx, row, col, wt, att)
    check_expected(got, G.SIMPLE_1D_EXPECTED, "simple_one_dimension")


def test_fork(geq, ctx):
    f = G.FORK
    got, _ = gpu_run(geq, ctx, *csr_from_edges(f["n"], f["edges"], f["attacker"]))
    check_expected(got, f["expected"], "fork")


def test_combinations(geq, ctx):
    c = G.COMBINATIONS
    att = [i in c["attackers"] for i in range(c["n"])]
    got, _ = gpu_run(geq, ctx, *csr_from_edges(c["n"], c["edges"], att))
    check_expected(got, c["expected"], "combinations")


def test_wide_game(geq, ctx):
    n, edges, att, expected = G.wide(*G.WIDE_GAME)
    got, stats = gpu_run(geq, ctx, *csr_from_edges(n, edges, att))
    check_expected(got, expected, "wide_game")
    assert stats["rounds"] >= 2


def _defender_over(lists, weights):
    """A defender (node 0) over attacker successors 1..k that start with the
    given lists and are the to_reach set (so node 0 is computed once)."""
    k = len(lists)
    edges = [(0, i + 1, w) for i, w in enumerate(weights)]
    att = [False] + [True] * k
    row, col, wt, a = csr_from_edges(k + 1, edges, att)
    init = [np.zeros((0, 1), np.uint32)] + [np.asarray(l, np.uint32).reshape(-1, 1) for l in lists]
    return row, col, wt, a, list(range(1, k + 1)), init


def test_defend_intersection_fixture(geq, ctx):
    # src/energygame/tests.rs:62-111 as a game
    lists, so = earray(G.DEF_ENERGIES).reshape(-1), G.DEF_SUCC_OFFSETS
    succ = [lists[so[i]:so[i + 1]] for i in range(4)]
    row, col, wt, att, reach, init = _defender_over(succ, G.DEF_WEIGHTS)
    got, _ = gpu_run(geq, ctx, row, col, wt, att, reach, init)
    assert canon(got[0]) == canon(earray(G.DEF_EXPECTED))


def test_defend_antichain(geq, ctx):
    # src/energygame/tests.rs:230-343: four copies of a 141-antichain -> itself
    ac = earray(G.ANTICHAIN_141).reshape(-1)
    ac2 = (ac + np.uint32(ora.pack_energy(6, 3, [1] * 6)[0])).astype(np.uint32)
    for lst in (ac, ac2):
        row, col, wt, att, reach, init = _defender_over([lst] * 4, [[0]] * 4)
        got, _ = gpu_run(geq, ctx, row, col, wt, att, reach, init)
        assert len(got[0]) == 141 and canon(got[0]) == canon(lst.reshape(-1, 1))


def test_defend_mixed(geq, ctx):
    # src/energygame/tests.rs:346-483: three defenders in one round
    ac = earray(G.ANTICHAIN_141).reshape(-1)
    ac2 = (ac + np.uint32(ora.pack_energy(6, 3, [1] * 6)[0])).astype(np.uint32)
    lists0, so = earray(G.DEF_ENERGIES).reshape(-1), G.DEF_SUCC_OFFSETS
    succ0 = [lists0[so[i]:so[i + 1]] for i in range(4)]
    n = 15
    edges, init = [], [np.zeros((0, 1), np.uint32)] * n
    init = list(init)
    for i, w in enumerate(G.DEF_WEIGHTS):
        edges.append((0, 1 + i, w))
        init[1 + i] = succ0[i].reshape(-1, 1)
    for base, lst in ((5, ac), (10, ac2)):
        for i in range(4):
            edges.append((base, base + 1 + i, [0]))
            init[base + 1 + i] = lst.reshape(-1, 1)
    att = [i not in (0, 5, 10) for i in range(n)]
    row, col, wt, a = csr_from_edges(n, edges, att)
    reach = [i for i in range(n) if i not in (0, 5, 10)]
    got, _ = gpu_run(geq, ctx, row, col, wt, a, reach, init)
    assert canon(got[0]) == canon(earray(G.DEF_EXPECTED))
    assert canon(got[5]) == canon(ac.reshape(-1, 1))
    assert canon(got[10]) == canon(ac2.reshape(-1, 1))


def _random_update(rng, n_el=6):
    """Single-component updates like the reference's graphgen.py:14-27, plus zero."""
    u = [0] * n_el
    r = rng.random()
    if r < 0.45:
        return u
    pos = int(rng.integers(n_el))
    if r < 0.75:
        u[pos] = -1
    else:
        t = int(rng.integers(1, n_el))
        if t >= pos + 1:
            t += 1
        u[pos] = t
    return u


def random_bipartite_game(seed, n, avg_deg=2.5, p_att=0.6):
    rng = np.random.default_rng(seed)
    att = rng.random(n) < p_att
    A = np.nonzero(att)[0]
    D = np.nonzero(~att)[0]
    edges = []
    for v in range(n):
        deg = int(rng.geometric(1.0 / avg_deg)) - (1 if not att[v] else 0)
        pool = D if att[v] else A
        if len(pool) == 0:
            continue
        for _ in range(max(deg, 0)):
            edges.append((v, int(pool[rng.integers(len(pool))]), _random_update(rng)))
    return csr_from_edges(n, edges, att)


@pytest.mark.parametrize("seed,n", [(1, 30), (2, 200), (3, 1000), (4, 3000), (5, 5000)])
def test_random_bipartite_vs_oracle(geq, ctx, seed, n):
    row, col, wt, att = random_bipartite_game(seed, n)
    got, _ = gpu_run(geq, ctx, row, col, wt, att)
    assert_parity(got, oracle_run(row, col, wt, att), f"bipartite seed {seed}")


def random_graphgen_game(seed, n):
    """Like graphgen/graphgen.py:40-51: a reversed random tree with random
    attacker flags and one non-zero update component per edge, plus extra
    random edges so that the game has cycles."""
    rng = np.random.default_rng(seed)
    edges = []
    for v in range(1, n):
        edges.append((int(rng.integers(v)), v, _random_update(rng)))
    for _ in range(n // 2):
        edges.append((int(rng.integers(n)), int(rng.integers(n)), _random_update(rng)))
    att = rng.random(n) < 0.5
    return csr_from_edges(n, edges, att)


@pytest.mark.parametrize("seed,n", [(11, 50), (12, 400), (13, 2000)])
def test_random_graphgen_vs_oracle(geq, ctx, seed, n):
    row, col, wt, att = random_graphgen_game(seed, n)
    got, _ = gpu_run(geq, ctx, row, col, wt, att)
    assert_parity(got, oracle_run(row, col, wt, att), f"graphgen seed {seed}")


def test_with_reach_explicit_empty(geq, ctx):
    # to_reach = [] : no visit lists, every position stays empty
    row, col, wt, att = _simple()
    got, st = gpu_run(geq, ctx, row, col, wt, att, to_reach=[])
    assert all(len(g) == 0 for g in got)


def test_other_conf_silent_step(geq, ctx):
    # EnergyConf::SILENT_STEP {8, 2}: generic codec on the device
    conf = (8, 2)
    rng = np.random.default_rng(7)
    n = 300
    att = rng.random(n) < 0.6
    edges = []
    for v in range(n):
        for _ in range(int(rng.integers(0, 4))):
            u = [0] * 8
            pos = int(rng.integers(8))
            if rng.random() < 0.5:
                u[pos] = -1
            else:
                u[pos] = int(rng.integers(1, 9))
            edges.append((v, int(rng.integers(n)), u))
    row, col, wt, a = csr_from_edges(n, edges, att, conf=conf)
    got, _ = gpu_run(geq, ctx, row, col, wt, a, conf=conf)
    assert_parity(got, oracle_run(row, col, wt, a, conf=conf), "silent_step")


def test_batch_equals_single(geq, ctx):
    games = [random_bipartite_game(100 + i, 50 + 37 * i) for i in range(12)]
    C = geq.EnergyConf.STANDARD
    graphs = [geq.GameGraph.from_csr(r, c, w, a, C) for r, c, w, a in games]
    batch, stats = geq.run_batch(graphs, ctx)
    for i, (r, c, w, a) in enumerate(games):
        single, _ = gpu_run(geq, ctx, r, c, w, a)
        assert_parity([x.array for x in batch[i]], single, f"batch game {i}")
        assert_parity(single, oracle_run(r, c, w, a), f"oracle game {i}")


def test_device_games_repeatable(geq, ctx):
    r, c, w, a = random_bipartite_game(77, 2000)
    C = geq.EnergyConf.STANDARD
    dg = geq.DeviceGames([geq.GameGraph.from_csr(r, c, w, a, C)], ctx)
    s1 = dg.solve()
    out1 = dg.download()[0]
    s2 = dg.solve()
    out2 = dg.download()[0]
    dg.close()
    assert s1["rounds"] == s2["rounds"]
    assert_parity([x.array for x in out1], [x.array for x in out2], "repeat")
    assert_parity([x.array for x in out1], oracle_run(r, c, w, a), "repeat vs oracle")


def test_invalid_inputs(geq, ctx):
    C = geq.EnergyConf.STANDARD
    g = geq.GameGraph.from_csr(np.array([0, 1], np.uint32), np.array([5], np.uint32),
                               np.array([0], np.uint32), np.array([1], np.uint8), C)
    with pytest.raises(geq.GeqError) as e:
        geq.EnergyGame.standard_reach(g).run(ctx)
    assert e.value.name == "INVALID_INPUT"
    g = geq.GameGraph.from_csr(np.array([0, 1], np.uint32), np.array([0], np.uint32),
                               np.array([0xF], np.uint32), np.array([1], np.uint8), C)
    with pytest.raises(geq.GeqError):
        geq.EnergyGame.standard_reach(g).run(ctx)
    # a conf beyond the multi-word solver (300 words per energy)
    big = geq.EnergyConf(300, 0xFFFFFFFF)
    g1 = geq.GameGraph.from_csr(np.array([0, 0], np.uint32), np.zeros(0, np.uint32),
                                np.zeros((0, big.update_size()), np.uint32), np.array([1], np.uint8), big)
    with pytest.raises(geq.GeqError) as e:
        geq.EnergyGame.standard_reach(g1).run(ctx)
    assert e.value.name == "UNSUPPORTED"


def test_invalid_inputs_large_batch(geq, ctx):
    """Batches of 64 games and more leave the row checks and the standard
    reach to the device: a faulty game still fails the call cleanly, and the
    context solves the next batch correctly."""
    games = [random_bipartite_game(100 + i, 40) for i in range(70)]
    graphs = [geq.GameGraph.from_csr(r, c, w, a, geq.EnergyConf.STANDARD) for r, c, w, a in games]
    good = geq.run_batch_raw(graphs, ctx)
    for i in (0, 41, 69):
        o = oracle_run(*games[i])
        got = [np.asarray(good[1][i][good[0][i][v]:good[0][i][v + 1]], np.uint32) for v in range(len(good[0][i]) - 1)]
        assert_parity(got, o, f"batch game {i}")

    def with_bad(i, fix):
        r, c, w, a = [np.array(x) for x in games[i]]
        r, c = fix(r.astype(np.uint32), c.astype(np.uint32))
        bad = geq.GameGraph.from_csr(r, c, w, a, geq.EnergyConf.STANDARD)
        return graphs[:i] + [bad] + graphs[i + 1:]

    def unsorted_rows(r, c):
        r = r.copy()
        k = int(np.argmax(np.diff(r)[1:] > 0))  # position k+1 has successors: r[k+1] < r[k+2]
        r[k + 1], r[k + 2] = r[k + 2], r[k + 1]
        return r, c

    def far_successor(r, c):
        c = c.copy()
        c[0] = 0xFFFFFF00
        return r, c

    def other_games_successor(r, c):
        c = c.copy()
        c[0] = 41  # beyond this 40-position game, inside the batch's id space
        return r, c

    for i, fix in ((40, unsorted_rows), (3, far_successor), (5, other_games_successor)):
        with pytest.raises(geq.GeqError) as e:
            geq.run_batch_raw(with_bad(i, fix), ctx)
        assert e.value.name == "INVALID_INPUT", fix.__name__
    again = geq.run_batch_raw(graphs, ctx)
    assert all(np.array_equal(a, b) for a, b in zip(again[1], good[1]))
