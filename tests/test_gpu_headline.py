"""Parity on the headline workload: the 4,096 games of the batched
configuration (gpuequiv_b200/data/batched_seeds.json), solved together on the
device through the timed path (DeviceGames: upload once, solve, download) and
through geq_energy_game_run_batch, against the oracle's own GameBuild and
EnergyGame::run of every 16th job; and manifest LTSs through compare_batch
and the serving loop's equivalence queries against the oracle's
TransitionSystem::compare (src/lib.rs:275-283, src/energygame.rs:379-383)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import ora

pytestmark = pytest.mark.gpu

STRIDE = 16  # every 16th job of the batch is checked against the oracle


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
    """Every position's list sorted: (offsets, data) with data ordered by
    (position, word)."""
    o = np.asarray(offsets, np.int64)
    d = np.asarray(data, np.uint32)
    seg = np.repeat(np.arange(len(o) - 1), np.diff(o))
    return o, d[np.lexsort((d, seg))]


@pytest.fixture(scope="module")
def batch(geq):
    """All jobs of the manifest, minimised and built by the library's host
    builder (as the benchmark does), plus the oracle's build and solve of
    every 16th job."""
    from concurrent.futures import ThreadPoolExecutor

    from gpuequiv_b200 import synth
    rows = synth.batched_manifest()["jobs"]
    seeds = [r[0] for r in rows]

    def build(seed):
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        return geq.GameBuild.compare(red, int(mp[p]), int(mp[q])).game

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        graphs = list(ex.map(build, seeds))
    assert [g.n_vertices() for g in graphs] == [r[1] for r in rows]
    sample = list(range(0, len(seeds), STRIDE))
    ora_games = []
    for i in sample:
        src, dst, lab, p, q = synth.batched_lts(seeds[i])
        red, mp = ora.Lts.from_arrays(src, dst, lab).bisimilar_minimize()
        b = ora.Build.compare(red, int(mp[p]), int(mp[q]), positions=False)
        g = graphs[i]
        # the graph itself: the oracle's GameBuild and the library's agree
        assert np.array_equal(b.row, g.row_offsets) and np.array_equal(b.col, g.column_indices), i
        assert np.array_equal(b.wt, g.weights.array.reshape(-1)) and np.array_equal(b.attacker, g.attacker_pos), i
        ora_games.append((b.row, b.col, b.wt, b.attacker))
    sols = ora.solve_games(ora_games, threads=os.cpu_count() or 4, largest_first=True)
    expect = {i: canonical(s.offsets, s.data) for i, s in zip(sample, sols)}
    return graphs, sample, expect


def _check(offs, data, sample, expect, what):
    bad = []
    for i in sample:
        go, gd = canonical(offs[i], data[i])
        eo, ed = expect[i]
        if not (np.array_equal(go, eo) and np.array_equal(gd, ed)):
            bad.append(i)
    assert not bad, f"{what}: jobs {bad[:10]} differ from the oracle ({len(bad)} of {len(sample)})"


def test_resident_solve_matches_oracle(geq, ctx, batch):
    """The path `value` times: games resident in HBM, solved repeatedly
    (every solve restarts from the uploaded initial lists)."""
    graphs, sample, expect = batch
    dg = geq.DeviceGames(graphs, ctx)
    try:
        for _ in range(2):
            st = dg.solve()
        assert st["rounds"] >= 1 and st["kernel_launches"] > 0
        offs, data = dg.download_raw()
    finally:
        dg.close()
    _check(offs, data, sample, expect, "DeviceGames.solve")


def test_run_batch_matches_oracle(geq, ctx, batch):
    """The path `e2e` times: host buffers through geq_energy_game_run_batch."""
    graphs, sample, expect = batch
    offs, data, st = geq.run_batch_raw(graphs, ctx)
    _check(offs, data, sample, expect, "geq_energy_game_run_batch")
    # the byte floor of the final lists is below what the solve moved
    bmin = sum(geq.b_min(graphs[i], offs[i]) for i in range(len(graphs)))
    assert 0 < bmin <= st["algorithmic_bytes"]
    for i in sample[:8]:
        assert geq.b_min(graphs[i], offs[i]) == ora.b_min(graphs[i].row_offsets, graphs[i].column_indices, offs[i])


def test_compare_and_serving_queries_match_oracle(geq, ctx):
    """compare(p, q) of 64 manifest LTSs (unminimised: minimisation, GameBuild
    and solve on the device) through compare_batch and through the serving
    loop's geq_server_submit_compare, against the oracle's compare."""
    from gpuequiv_b200 import synth
    from gpuequiv_b200.serving import Server
    rows = synth.batched_manifest()["jobs"]
    picks = [r[0] for r in rows[::64]][:64]
    jobs, ora_games = [], []
    for seed in picks:
        src, dst, lab, p, q = synth.batched_lts(seed)
        jobs.append((geq.TransitionSystem.from_arrays(src, dst, lab), int(p), int(q)))
        red, mp = ora.Lts.from_arrays(src, dst, lab).bisimilar_minimize()
        assert mp[p] != mp[q]  # the manifest holds no bisimilar pairs
        b = ora.Build.compare(red, int(mp[p]), int(mp[q]), positions=False)
        ora_games.append((b.row, b.col, b.wt, b.attacker))
    sols = ora.solve_games(ora_games, threads=os.cpu_count() or 4, largest_first=True)
    expect = [sorted(int(x) for x in s.data[int(s.offsets[0]):int(s.offsets[1])]) for s in sols]
    got = [sorted(int(x) for x in np.asarray(r.array).reshape(-1)) for r in geq.compare_batch(jobs, context=ctx)]
    assert got == expect
    with Server(ctx, n_pipelines=2, max_wait_us=500) as srv:
        tickets = [srv.submit_compare(*j) for j in jobs]
        served = []
        for t in tickets:
            offs, data, _ = srv.poll(t, timeout_ms=120_000)
            served.append(sorted(int(x) for x in data[int(offs[0]):int(offs[1])]))
        assert srv.stats()["failed"] == 0
    assert served == expect
