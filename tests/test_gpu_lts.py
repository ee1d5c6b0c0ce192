"""Whole-algorithm parity on the GPU: TransitionSystem::compare / equivalences
(src/lib.rs:275-343) against the reference's known answers and the oracle."""
import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import canon, earray, random_lts, ref_eq
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


def eqv(geq, name):
    return geq.std_equivalences.get(name)


def test_example_energies(geq, ctx):
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    b = geq.GameBuild.compare(lts, 0, 1)
    assert [tuple(p) for p in b.nodes] == G.EXAMPLE_NODES
    game = geq.EnergyGame.standard_reach(b.game)
    got = game.run(ctx)
    for v, (g, rows) in enumerate(zip(got, G.EXAMPLE_ENERGIES)):
        assert ref_eq(g.array, earray(rows)), (v, g.canonical())


def test_bisimilar(geq, ctx):
    lts = geq.TransitionSystem(G.BISIMILAR_LTS)
    part, _ = lts.signature_refinement()
    assert part[0] == part[5]
    e = lts.compare(0, 5, ctx)
    assert e.is_empty()
    assert e.test_equivalence(eqv(geq, "bisimulation"))


def test_failure_trace(geq, ctx):
    lts = geq.TransitionSystem(G.FAILURE_TRACE_LTS)
    e = lts.compare(0, 9, ctx)
    for name, holds in G.FAILURE_TRACE_VERDICTS.items():
        assert e.test_equivalence(eqv(geq, name)) == holds, name


def test_doc_examples(geq, ctx):
    lts = geq.TransitionSystem(G.DOC_LTS)
    e = lts.compare(0, 4, ctx)
    for name, holds in G.DOC_COMPARE_0_4:
        assert e.test_equivalence(eqv(geq, name)) == holds
    eq = lts.equivalences(ctx)
    for kind, p, q, name, expect in G.DOC_EQUIVALENCES:
        f = eq.preorder if kind == "preorder" else eq.equiv
        assert f(p, q, eqv(geq, name)) == expect, (kind, p, q, name)
    traces = eq.relation(eqv(geq, "traces"))
    assert traces.count_classes() == G.DOC_TRACES_CLASSES
    assert traces.class_of(0) == G.DOC_TRACES_CLASS_OF_0


@pytest.mark.parametrize("seed", range(6))
def test_compare_random_vs_oracle(geq, ctx, seed):
    rng = np.random.default_rng(seed)
    edges = random_lts(rng, 40, 4, 120)  # the "small" configuration
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    jobs = []
    for _ in range(8):
        p, q = (int(x) for x in rng.integers(0, lts.n_vertices(), 2))
        jobs.append((lts, p, q))
    got = geq.compare_batch(jobs, ctx)
    for (l, p, q), g in zip(jobs, got):
        assert canon(g.array) == canon(ora.compare(olts, p, q)), (seed, p, q)
        single = lts.compare(p, q, ctx)
        assert canon(single.array) == canon(g.array)


@pytest.mark.parametrize("seed", range(4))
def test_compare_unminimized_vs_oracle(geq, ctx, seed):
    rng = np.random.default_rng(100 + seed)
    edges = random_lts(rng, 25, 3, 60)
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    n = lts.n_vertices()
    for _ in range(4):
        p, q = (int(x) for x in rng.integers(0, n, 2))
        if p == q:
            continue
        got = lts.compare_unminimized(p, q, ctx)
        b = ora.Build.compare(olts, p, q)
        sol = ora.run_game(6, 3, b.row, b.col, b.wt, b.attacker, ora.standard_reach(b.row, b.attacker))
        assert canon(got.array) == canon(sol.lists()[0])


@pytest.mark.parametrize("seed", range(4))
def test_equivalences_vs_oracle(geq, ctx, seed):
    rng = np.random.default_rng(200 + seed)
    edges = random_lts(rng, 40, 4, 120)
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    eq = lts.equivalences(ctx)
    oeq = ora.equivalences(olts)
    n = lts.n_vertices()
    names = G.STD_EQUIVALENCES
    for name, tup in names.items():
        e = eqv(geq, name)
        for p in range(n):
            for q in range(n):
                assert eq.preorder(p, q, e) == oeq.preorder(p, q, tup), (name, p, q)
        rel = eq.relation(e)
        orel = oeq.relation(tup)
        assert rel.count_classes() == orel.count_classes(), name
        assert sorted(map(tuple, rel.get_classes())) == sorted(map(tuple, orel.get_classes())), name
    for p in range(n):
        for q in range(n):
            a, b = eq.energies(p, q), oeq.energies_of(p, q)
            assert (a is None) == (b is None)
            if a is not None:
                assert canon(a.array) == canon(b)


def test_equivalences_unminimized_vs_oracle(geq, ctx):
    rng = np.random.default_rng(300)
    edges = random_lts(rng, 30, 3, 80)
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    eq = lts.equivalences_unminimized(ctx)
    oeq = ora.equivalences(olts, minimize=False)
    n = lts.n_vertices()
    for name, tup in G.STD_EQUIVALENCES.items():
        e = eqv(geq, name)
        for p in range(n):
            for q in range(n):
                assert eq.preorder(p, q, e) == oeq.preorder(p, q, tup), (name, p, q)


def test_compare_all_game_vs_oracle(geq, ctx):
    """The compare_all game keyed by position content (start order differs
    from the reference's hash order, so indices are not compared)."""
    rng = np.random.default_rng(400)
    edges = random_lts(rng, 30, 3, 90)
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    b, _ = geq.GameBuild.compare_all(lts)
    ob = ora.Build.compare_all(olts)
    assert b.game.n_vertices() == ob.n and b.n_starting_points == ob.n_starting
    got = geq.EnergyGame.standard_reach(b.game).run(ctx)
    osol = ora.run_game(6, 3, ob.row, ob.col, ob.wt, ob.attacker, ora.standard_reach(ob.row, ob.attacker)).lists()
    mine = {tuple(p): canon(g.array) for p, g in zip(b.nodes, got)}
    theirs = {p: canon(l) for p, l in zip(ob.positions, osol)}
    assert mine == theirs
