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
