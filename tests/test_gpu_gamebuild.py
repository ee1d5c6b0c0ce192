"""GameBuild::compare on the device (geq_game_build_compare_batch) against the
reference's example game (tests/complete.rs:24-75), the oracle's GameBuild
(src/gamebuild.rs:139-266 restated) and the host builder: the same position
numbering, adjacency order, weights and attacker flags, bit for bit."""
import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import random_lts
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


def arrays(g):
    return (np.asarray(g.row_offsets), np.asarray(g.column_indices), np.asarray(g.weights.array).reshape(-1),
            np.asarray(g.attacker_pos))


def assert_same(a, b, what=""):
    for x, y, name in zip(a, b, ("row_offsets", "column_indices", "weights", "attacker_pos")):
        assert np.array_equal(np.asarray(x, dtype=np.int64), np.asarray(y, dtype=np.int64)), (what, name)


def test_example_game(geq, ctx):
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    b = geq.GameBatch([(lts, 0, 1)], context=ctx)
    g = b.graph(0)
    assert g.n_vertices() == len(G.EXAMPLE_NODES)
    assert [sorted(int(x) for x in g.adj(v)) for v in range(g.n_vertices())] == G.EXAMPLE_ADJ
    assert list(g.attacker_pos) == [int(k != "defend") for k, *_ in G.EXAMPLE_NODES]
    assert_same(arrays(g), arrays(geq.GameBuild.compare(lts, 0, 1).game))


@pytest.mark.parametrize("seed", range(4))
def test_random_vs_oracle(geq, ctx, seed):
    rng = np.random.default_rng(100 + seed)
    jobs, ora_builds = [], []
    for _ in range(24):
        n = int(rng.integers(1, 14))
        edges = random_lts(rng, n, int(rng.integers(1, 5)), int(rng.integers(0, 3 * n + 1)))
        p, q = int(rng.integers(0, n)), int(rng.integers(0, n))
        lts = geq.TransitionSystem(edges) if edges else geq.TransitionSystem.from_arrays([], [], [], n_vertices=n)
        if lts.n_vertices() <= max(p, q):
            continue
        jobs.append((lts, p, q))
        ol = ora.Lts.from_edges(edges) if edges else None
        ora_builds.append(ora.Build.compare(ol, p, q) if ol is not None else None)
    b = geq.GameBatch(jobs, context=ctx)
    assert len(b) == len(jobs)
    for j, (lts, p, q) in enumerate(jobs):
        g = arrays(b.graph(j))
        ob = ora_builds[j]
        if ob is not None:
            assert_same(g, (ob.row, ob.col, ob.wt, ob.attacker), f"job {j}")
        assert_same(g, arrays(geq.GameBuild.compare(lts, p, q).game), f"job {j}")


@pytest.mark.parametrize("flags", [0, 4], ids=["graph_loop", "plain_launches"])
def test_batched_workload_vs_host(geq, ctx, flags):
    """Minimised LTSs of the batched configuration (every 32nd accepted seed),
    with the level loop in a CUDA graph and as plain launches (GEQ_TUNE_NO_GRAPH)."""
    from gpuequiv_b200 import synth
    rows = synth.batched_manifest()["jobs"][::32]
    jobs = []
    for seed, npos, _ in rows:
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        jobs.append((red, int(mp[p]), int(mp[q]), npos))
    try:
        ctx.set_tuning(flags=flags)
        b = geq.GameBatch([j[:3] for j in jobs], context=ctx)
    finally:
        ctx.set_tuning(flags=0)
    assert b.stats["attempts"] == 1
    assert b.stats["positions"] == sum(j[3] for j in jobs)
    for k, (red, p, q, npos) in enumerate(jobs):
        g = b.graph(k)
        assert g.n_vertices() == npos
        assert_same(arrays(g), arrays(geq.GameBuild.compare(red, p, q).game), f"seed {rows[k][0]}")


def test_warp_path_vs_host(geq, ctx):
    """Every attack position through the warp path (bitmap unions, ballot
    placement), on random LTSs with much nondeterminism and on a slice of the
    batched workload."""
    from gpuequiv_b200._lib import TUNE_BUILD_WARP_ALL
    from gpuequiv_b200 import synth
    rng = np.random.default_rng(11)
    jobs = []
    for _ in range(48):
        n = int(rng.integers(2, 40))
        lts = geq.TransitionSystem(random_lts(rng, n, int(rng.integers(1, 4)), int(rng.integers(n, 4 * n + 1))))
        jobs.append((lts, int(rng.integers(0, lts.n_vertices())), int(rng.integers(0, lts.n_vertices()))))
    for seed, _, _ in synth.batched_manifest()["jobs"][1::64]:
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        jobs.append((red, int(mp[p]), int(mp[q])))
    try:
        ctx.set_tuning(flags=TUNE_BUILD_WARP_ALL)
        b = geq.GameBatch(jobs, context=ctx, max_positions=300_000)
    finally:
        ctx.set_tuning(flags=0)
    for j, (lts, p, q) in enumerate(jobs):
        try:
            host = geq.GameBuild.compare_bounded(lts, p, q, 300_000)
        except geq.GeqError:
            with pytest.raises(geq.GeqError):
                b.graph(j)
            continue
        assert_same(arrays(b.graph(j)), arrays(host.game), f"job {j}")


def test_position_bound(geq, ctx):
    """Jobs beyond max_positions are refused exactly when compare_bounded refuses."""
    rng = np.random.default_rng(7)
    jobs = []
    for _ in range(40):
        n = int(rng.integers(4, 30))
        lts = geq.TransitionSystem(random_lts(rng, n, 3, 3 * n))
        jobs.append((lts, int(rng.integers(0, lts.n_vertices())), int(rng.integers(0, lts.n_vertices()))))
    bound = 300
    b = geq.GameBatch(jobs, context=ctx, max_positions=bound)
    refused = 0
    for j, (lts, p, q) in enumerate(jobs):
        try:
            host = geq.GameBuild.compare_bounded(lts, p, q, bound)
        except geq.GeqError as e:
            assert e.status == 2
            with pytest.raises(geq.GeqError) as ei:
                b.graph(j)
            assert ei.value.status == 2
            refused += 1
            continue
        assert_same(arrays(b.graph(j)), arrays(host.game), f"job {j}")
    assert 0 < refused < len(jobs)


def test_bad_input(geq, ctx):
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    with pytest.raises(geq.GeqError) as ei:
        geq.GameBatch([(lts, 0, 7)], context=ctx)
    assert ei.value.status == 3
    with pytest.raises(geq.GeqError):
        geq.GameBatch([], context=ctx)


def test_compare_all_vs_host(geq, ctx):
    """GameBuild::compare_all on the device (many start positions per job)
    against the host builder and the oracle: same start numbering, CSR and
    weights."""
    rng = np.random.default_rng(21)
    systems, edges_of = [], []
    for _ in range(12):
        n = int(rng.integers(2, 9))
        edges = random_lts(rng, n, 2, int(rng.integers(n, 2 * n + 1)))
        systems.append(geq.TransitionSystem(edges))
        edges_of.append(edges)
    systems.append(geq.TransitionSystem(G.EXAMPLE_LTS))
    edges_of.append(G.EXAMPLE_LTS)
    b = geq.GameBatch.compare_all(systems, context=ctx, max_positions=2_000_000)
    for j, lts in enumerate(systems):
        host, info = geq.GameBuild.compare_all(lts)
        assert b.n_starting_points(j) == host.n_starting_points
        assert_same(arrays(b.graph(j)), arrays(host.game), f"job {j}")
        ob = ora.Build.compare_all(ora.Lts.from_edges(edges_of[j]))
        assert ob.n_starting == host.n_starting_points
        assert_same(arrays(b.graph(j)), (ob.row, ob.col, ob.wt, ob.attacker), f"job {j} (oracle)")
