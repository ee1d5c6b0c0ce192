"""The stress configuration (energy game only: 2,000,000 positions, 10,000,000
edges, 60 % attackers, geometric out-degree, single-component updates,
standard reach) on the device against the oracle: exact lists at scaled-down
and at full size, and the fixpoint property of the full-size result."""
from __future__ import annotations

import numpy as np
import pytest

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


def canonical(offsets, data):
    """Every position's list sorted, as (offsets, data)."""
    o = np.asarray(offsets, np.int64)
    d = np.asarray(data, np.uint32)
    seg = np.repeat(np.arange(len(o) - 1), np.diff(o))
    return o, d[np.lexsort((d, seg))]


def solve_both(geq, ctx, row, col, wt, att):
    g = geq.GameGraph.from_csr(row, col, wt, att, geq.EnergyConf.STANDARD)
    offs, data, stats = geq.run_batch_raw([g], ctx)
    got = canonical(offs[0], data[0])
    sol = ora.run_game(6, 3, row, col, wt, att, ora.standard_reach(row, att))
    exp = canonical(sol.offsets, sol.data)
    return got, exp, stats, sol


@pytest.mark.parametrize("seed,n,m", [(5, 20_000, 100_000), (6, 200_000, 1_000_000)])
def test_stress_scaled_vs_oracle(geq, ctx, seed, n, m):
    from gpuequiv_b200 import synth
    row, col, wt, att = synth.scaled_stress_game(seed, n, m)
    got, exp, _, _ = solve_both(geq, ctx, row, col, wt, att)
    assert np.array_equal(got[0], exp[0]), "list lengths differ"
    assert np.array_equal(got[1], exp[1]), "energies differ"


def test_stress_full_size(geq, ctx):
    from gpuequiv_b200 import synth
    row, col, wt, att = synth.stress_game()  # seed 2, 2M positions, 10M edges
    assert len(row) - 1 == 2_000_000 and len(col) == 10_000_000
    got, exp, stats, sol = solve_both(geq, ctx, row, col, wt, att)
    assert np.array_equal(got[0], exp[0]), "list lengths differ"
    assert np.array_equal(got[1], exp[1]), "energies differ"
    # size-independent property of the device's lists: one more worklist step
    # changes no position
    assert ora.check_fixpoint(row, col, wt, att, got[0].astype(np.uint64), got[1]) == (0, None)
    # every position that ends with a list and is not a target was computed at
    # least once with all of its successors read
    deg = np.diff(np.asarray(row, np.int64))
    need = (np.diff(got[0]) > 0) & (deg > 0)
    assert stats["positions_computed"] >= int(need.sum())
    assert stats["edges_relaxed"] >= int(deg[need].sum())
    assert stats["rounds"] >= 1


def test_split_batch_matches_one_engine(geq, ctx):
    """A batch of at least 2**21 positions runs as two halves on two engines
    (the second half uploads while the first solves): every game's lists
    equal those of the same batch on one engine, and the oracle's for a game
    of each half."""
    from gpuequiv_b200 import synth
    from gpuequiv_b200._lib import TUNE_NO_SPLIT
    games = [synth.scaled_stress_game(20 + i, 200_000, 1_000_000) for i in range(12)]
    graphs = [geq.GameGraph.from_csr(r, c, w, a, geq.EnergyConf.STANDARD) for r, c, w, a in games]
    offs, data, stats = geq.run_batch_raw(graphs, ctx)
    ctx.set_tuning(flags=TUNE_NO_SPLIT)
    try:
        offs1, data1, stats1 = geq.run_batch_raw(graphs, ctx)
    finally:
        ctx.set_tuning()
    assert stats["positions_computed"] == stats1["positions_computed"]
    for i in range(len(games)):
        a, b = canonical(offs[i], data[i]), canonical(offs1[i], data1[i])
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), f"game {i} differs"
    for i in (0, len(games) - 1):
        row, col, wt, att = games[i]
        sol = ora.run_game(6, 3, row, col, wt, att, ora.standard_reach(row, att))
        exp = canonical(sol.offsets, sol.data)
        got = canonical(offs[i], data[i])
        assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1]), f"game {i} differs from the oracle"


def test_split_batch_result_block_grows(geq, ctx):
    """The two-halves form copies the first half's lists to the host while
    the second half solves, into a block sized from the first half; here the
    first half has no energies at all and the second many (every attacker
    ends with six incomparable unit energies), so the block must grow: the
    lists still equal those of one engine, and the expected ones."""
    from gpuequiv_b200._lib import TUNE_NO_SPLIT
    conf = geq.EnergyConf.STANDARD
    graphs = []
    for _ in range(2):  # attackers without moves: empty lists
        n = 600_000
        graphs.append(geq.GameGraph.from_csr(np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32),
                                             np.zeros(0, np.uint32), np.ones(n, np.uint8), conf))
    m = 180_000  # attackers, each with six defender sinks behind decrements of dims 0..5
    n = 7 * m
    row = np.zeros(n + 1, np.uint32)
    row[1:m + 1] = 6 * np.arange(1, m + 1, dtype=np.uint32)
    row[m + 1:] = 6 * m
    col = (m + np.arange(6 * m, dtype=np.uint32)).astype(np.uint32)
    wt = (np.uint32(1) << (4 * np.tile(np.arange(6, dtype=np.uint32), m))).astype(np.uint32)
    att = np.zeros(n, np.uint8)
    att[:m] = 1
    graphs.append(geq.GameGraph.from_csr(row, col, wt, att, conf))
    assert sum(g.n_vertices() for g in graphs) >= 2 ** 21
    offs, data, stats = geq.run_batch_raw(graphs, ctx)
    ctx.set_tuning(flags=TUNE_NO_SPLIT)
    try:
        offs1, data1, _ = geq.run_batch_raw(graphs, ctx)
    finally:
        ctx.set_tuning()
    for i in range(len(graphs)):
        a, b = canonical(offs[i], data[i]), canonical(offs1[i], data1[i])
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), f"game {i} differs"
    assert int(offs[0][-1]) == 0 and int(offs[1][-1]) == 0
    o, d = np.asarray(offs[2], np.int64), np.asarray(data[2]).reshape(-1)
    assert np.all(np.diff(o[:m + 1]) == 6) and np.all(np.diff(o[m:]) == 1)
    units = sorted(1 << (2 * k) for k in range(6))
    for v in (0, m // 2, m - 1):
        assert sorted(int(x) for x in d[o[v]:o[v + 1]]) == units
    assert not d[o[m]:].any()  # the sinks: the zero energy
