"""Signature refinement on the device (geq_lts_signature_refinement_batch)
against the oracle's restatement of TransitionSystem::signature_refinement
(src/lib.rs:444-478) and the host implementation: identical partitions (class
ids handed out in process order) and class counts."""
import numpy as np
import pytest

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


@pytest.mark.parametrize("seed", range(3))
def test_random_vs_oracle(geq, ctx, seed):
    rng = np.random.default_rng(500 + seed)
    systems, edges_of = [], []
    for _ in range(64):
        n = int(rng.integers(1, 60))
        # few labels and sparse rows give many bisimilar processes
        edges = random_lts(rng, n, int(rng.integers(1, 4)), int(rng.integers(0, 2 * n + 1)))
        if not edges:
            continue
        systems.append(geq.TransitionSystem(edges))
        edges_of.append(edges)
    got = geq.signature_refinement_batch(systems, context=ctx)
    merged = 0
    for k, (part, cnt) in enumerate(got):
        opart, ocnt = ora.Lts.from_edges(edges_of[k]).signature_refinement()
        assert cnt == ocnt, k
        assert np.array_equal(part, opart.astype(np.uint64)), k
        hpart, hcnt = systems[k].signature_refinement()
        assert cnt == hcnt and np.array_equal(part, np.asarray(hpart, dtype=np.uint64)), k
        merged += cnt < systems[k].n_vertices()
    assert merged > 0


def test_batched_workload_vs_host(geq, ctx):
    from gpuequiv_b200 import synth
    systems = []
    for seed, _, _ in synth.batched_manifest()["jobs"][:256:4]:
        src, dst, lab, _, _ = synth.batched_lts(seed)
        systems.append(geq.TransitionSystem.from_arrays(src, dst, lab))
    got = geq.signature_refinement_batch(systems, context=ctx)
    for k, (part, cnt) in enumerate(got):
        hpart, hcnt = systems[k].signature_refinement()
        assert cnt == hcnt and np.array_equal(part, np.asarray(hpart, dtype=np.uint64)), k


def test_edge_cases(geq, ctx):
    """A system without transitions, a self loop, a cycle of equal processes."""
    systems = [geq.TransitionSystem.from_arrays([], [], [], n_vertices=5),
               geq.TransitionSystem([(0, 0, 1)]),
               geq.TransitionSystem([(0, 1, 1), (1, 2, 1), (2, 0, 1), (3, 3, 2)])]
    got = geq.signature_refinement_batch(systems, context=ctx)
    for k, (part, cnt) in enumerate(got):
        hpart, hcnt = systems[k].signature_refinement()
        assert cnt == hcnt and np.array_equal(part, np.asarray(hpart, dtype=np.uint64)), k
    assert got[0][1] == 1 and got[2][1] == 2


def test_compare_batch_minimised_on_device(geq, ctx):
    """compare_batch (device minimisation, build, solve) against the oracle's
    TransitionSystem::compare, including bisimilar pairs (empty lists)."""
    rng = np.random.default_rng(77)
    jobs, oras = [], []
    for _ in range(48):
        n = int(rng.integers(2, 16))
        edges = random_lts(rng, n, 3, int(rng.integers(n, 3 * n + 1)))
        lts = geq.TransitionSystem(edges)
        p, q = int(rng.integers(0, lts.n_vertices())), int(rng.integers(0, lts.n_vertices()))
        jobs.append((lts, p, q))
        oras.append(ora.compare(ora.Lts.from_edges(edges), p, q))
    jobs.append((jobs[0][0], 0, 0))  # p == q: bisimilar, no game, no energies
    oras.append([])
    got = geq.compare_batch(jobs, context=ctx)
    for k in range(len(jobs)):
        mine = sorted(int(x) for x in np.asarray(got[k].array).reshape(-1))
        ref = sorted(int(x) for x in np.asarray(oras[k]).reshape(-1))
        assert mine == ref, k
