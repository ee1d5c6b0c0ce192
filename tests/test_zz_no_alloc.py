"""geq_energy_game_run_static (the allocation-free entry point) against
geq_energy_game_run (the existing entry point) and the oracle.

Each game is solved twice in a row through the static entry point, whose
scratch is one file-scope device array reused by every call: both results
must hold the existing entry point's lists (as sets, like the crate's
EnergyArray equality) and be identical to each other.  The existing entry
point runs on a second context whose tuning turns off its one-block path for
small games, which launches the same kernel as the static entry point: the
expected lists then come from the general round kernels, and small games are
also checked against the oracle.  The file is named to be collected last, so
that in a full run it also exercises the scratch after every other GPU test
of the session.
"""
from __future__ import annotations

import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import csr_from_edges
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
def ctx_general(geq):
    """A context whose geq_energy_game_run takes the general round kernels
    for every game: any tuning flag turns the one-block path off, and
    GEQ_TUNE_NO_SPLIT changes nothing else for one game."""
    from gpuequiv_b200._lib import TUNE_NO_SPLIT
    c = geq.Context(0)
    c.set_tuning(flags=TUNE_NO_SPLIT)
    yield c
    c.close()


def _oracle(g, to_reach=None):
    conf = g.get_conf()
    reach = ora.standard_reach(g.row_offsets, g.attacker_pos) if to_reach is None else to_reach
    sol = ora.run_game(conf.elements, conf.max, g.row_offsets, g.column_indices, g.weights.array.reshape(-1),
                       g.attacker_pos, reach)
    return sol.offsets, sol.data


def _random_update(rng, n_el=6):
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


def _bipartite(seed, n, avg_deg=2.5, p_att=0.6):
    rng = np.random.default_rng(seed)
    att = rng.random(n) < p_att
    A, D = np.nonzero(att)[0], np.nonzero(~att)[0]
    edges = []
    for v in range(n):
        pool = D if att[v] else A
        deg = int(rng.geometric(1.0 / avg_deg)) - (0 if att[v] else 1)
        for _ in range(max(deg, 0) if len(pool) else 0):
            edges.append((v, int(pool[rng.integers(len(pool))]), _random_update(rng)))
    return csr_from_edges(n, edges, att)


def _graph(geq, row, col, wt, att, conf=(6, 3)):
    return geq.GameGraph.from_csr(row, col, wt, att, geq.EnergyConf(*conf))


def _games(geq):
    att = [i in G.SIMPLE_ATTACKERS for i in range(18)]
    yield "simple", _graph(geq, *csr_from_edges(18, G.SIMPLE_EDGES, att))
    c = G.COMBINATIONS
    att = [i in c["attackers"] for i in range(c["n"])]
    yield "combinations", _graph(geq, *csr_from_edges(c["n"], c["edges"], att))
    for seed, n in ((1, 30), (2, 1000), (3, 5000)):
        yield f"bipartite-{seed}-{n}", _graph(geq, *_bipartite(seed, n))
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    yield "spectroscopy-example", geq.GameBuild.compare(lts, 0, 1).game
    from gpuequiv_b200 import synth
    for seed in (11, 71):  # 453 and 35,734 positions
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        yield f"spectroscopy-batched-{seed}", geq.GameBuild.compare(red, int(mp[p]), int(mp[q])).game


def _canon(offsets, data):
    """Each position's list sorted: lists are compared as sets, as the
    crate's EnergyArray equality does (the order inside a list depends on
    the order in which a path meets the candidates)."""
    o = np.asarray(offsets, np.int64)
    d = np.asarray(data, np.uint32)
    seg = np.repeat(np.arange(len(o) - 1), np.diff(o))
    return o, d[np.lexsort((d, seg))]


def _same(a, b, what):
    (ao, ad), (bo, bd) = _canon(*a), _canon(*b)
    assert np.array_equal(ao, bo), f"{what}: list lengths differ"
    assert np.array_equal(ad, bd), f"{what}: energies differ"


def _identical(a, b, what):
    assert np.array_equal(np.asarray(a[0], np.uint64), np.asarray(b[0], np.uint64)), f"{what}: offsets differ"
    assert np.array_equal(np.asarray(a[1], np.uint32), np.asarray(b[1], np.uint32)), f"{what}: energies differ"


def test_static_equals_existing_entry_point(geq, ctx, ctx_general):
    for name, g in _games(geq):
        offs, data, st = geq.run_batch_raw([g], ctx_general)
        ref = (offs[0].copy(), data[0].copy())
        del offs, data
        assert st["kernel_launches"] > 1, f"{name}: the existing entry point took the one-block path"
        first = geq.run_static(g, ctx)
        second = geq.run_static(g, ctx)
        _same(first[:2], ref, f"{name}, first call")
        _same(second[:2], ref, f"{name}, second call")
        _identical(first[:2], second[:2], f"{name}, second call against the first")
        if g.n_vertices() <= 5000:
            _same(first[:2], _oracle(g), f"{name}, oracle")
        assert first[2]["kernel_launches"] == 1
        assert first[2]["rounds"] == second[2]["rounds"]


def test_static_allocates_nothing(geq, ctx):
    """After one call, a second call leaves the device's free memory as it
    was: no cudaMalloc, no pool growth, no graph or module load."""
    import torch
    g = _graph(geq, *_bipartite(9, 3000))
    first = geq.run_static(g, ctx)
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    second = geq.run_static(g, ctx)
    torch.cuda.synchronize(0)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"
    _identical(first[:2], second[:2], "second call against the first")


def test_static_explicit_reach(geq, ctx, ctx_general):
    g = _graph(geq, *_bipartite(7, 800))
    reach = np.array([3, 17, 400], np.uint32)
    res = geq.EnergyGame.with_reach(g, reach).run(ctx_general)
    o_off, o_data = _oracle(g, reach)
    for _ in range(2):
        offs, data, _ = geq.run_static(g, ctx, to_reach=reach)
        for v, e in enumerate(res):
            assert np.array_equal(np.sort(data[offs[v]:offs[v + 1]]), np.sort(e.array.reshape(-1))), f"position {v}"
        _same((offs, data), (o_off, o_data), "explicit reach, oracle")
    offs, data, _ = geq.run_static(g, ctx, to_reach=[])
    assert int(offs[-1]) == 0


def test_static_generic_codec(geq, ctx, ctx_general):
    rng = np.random.default_rng(5)
    n, conf = 300, (8, 2)
    att = rng.random(n) < 0.6
    edges = []
    for v in range(n):
        for _ in range(int(rng.integers(0, 4))):
            u = [0] * 8
            pos = int(rng.integers(8))
            u[pos] = -1 if rng.random() < 0.5 else int(rng.integers(1, 9))
            edges.append((v, int(rng.integers(n)), u))
    g = _graph(geq, *csr_from_edges(n, edges, att, conf=conf), conf=conf)
    offs, data, _ = geq.run_batch_raw([g], ctx_general)
    ref = (offs[0].copy(), data[0].copy())
    _same(ref, _oracle(g), "generic codec, existing entry point against the oracle")
    for k in range(2):
        _same(geq.run_static(g, ctx)[:2], ref, f"silent-step call {k}")


def test_static_limits(geq, ctx):
    from gpuequiv_b200 import GeqError
    g = _graph(geq, *_bipartite(2, 1000))
    offs, data, _ = geq.run_static(g, ctx)
    need = int(offs[-1])
    assert need > 1
    with pytest.raises(GeqError) as e:
        geq.run_static(g, ctx, data_cap=need - 1)
    assert e.value.name == "INVALID_INPUT"
    # a game larger than the scratch is refused before any device work
    n = 400_000
    row = np.arange(n + 1, dtype=np.uint32)
    col = np.roll(np.arange(n, dtype=np.uint32), 1)
    big = geq.GameGraph.from_csr(row, col, np.zeros(n, np.uint32), np.ones(n, bool), geq.EnergyConf(6, 3))
    with pytest.raises(GeqError) as e:
        geq.run_static(big, ctx)
    assert e.value.name == "UNSUPPORTED"
    # the scratch is still good afterwards
    _same(geq.run_static(g, ctx)[:2], (offs, data), "after refusals")
