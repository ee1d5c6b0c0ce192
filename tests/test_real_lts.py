"""Real inputs: the VLTS systems the reference benchmarks on
(benches/benchmark.rs:16-28, CSV files of benches/lts/, loaded with
TransitionSystem::from_csv_file, src/lib.rs:364-420).  The files are not part
of this repository; the tests read them from the directory named by the
environment variable GEQ_LTS_DIR and are skipped when it is absent.  The CPU
tests also look in the reference's own checkout.

- CPU: the library's CSV loader and host minimisation against the oracle's,
  and the host GameBuild::compare_all of the minimised system against the
  oracle's, position for position (src/gamebuild.rs:139-266).
- GPU: equivalences() through the device pipeline (minimisation, compare_all
  built and solved on the device) against the oracle's equivalences() of the
  same file: the energies of every starting pair (a seeded sample of 200,000
  pairs where there are more) and, for systems with at most 20,000 starting
  pairs, the 13 standard relations as partitions.  The reference's own list
  (vasy_18_73 is skipped there as too large, benchmark.rs:27) is used, with a
  position cap (GEQ_LTS_MAX_POSITIONS, default 3,000,000) on the oracle's
  sequential solve.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import ora

# benches/benchmark.rs:16-28, smallest games first
FILES = ["vasy_25_25.csv", "peterson_mutex_weak.csv", "vasy_0_1.csv", "vasy_1_4.csv", "vasy_5_9.csv",
         "vasy_8_38.csv", "cwi_3_14.csv", "vasy_8_24.csv", "vasy_10_56.csv", "cwi_1_2.csv"]
# host builds the CPU suite compares (the oracle builds cwi_1_2 in minutes)
CPU_FILES = FILES[:8]


def _dir(gpu: bool) -> str | None:
    d = os.environ.get("GEQ_LTS_DIR")
    if not d and not gpu:
        d = "/root/reference/benches/lts"
    return d if d and os.path.isdir(d) else None


def _path(name: str, gpu: bool) -> str:
    d = _dir(gpu)
    if d is None or not os.path.isfile(os.path.join(d, name)):
        pytest.skip(f"{name}: no directory of VLTS files (GEQ_LTS_DIR)")
    return os.path.join(d, name)


@pytest.fixture(scope="module")
def geq():
    import gpuequiv_b200 as geq
    return geq


def _canon(labels) -> np.ndarray:
    """Partition as first-occurrence class numbers (independent of naming)."""
    first: dict[int, int] = {}
    return np.array([first.setdefault(int(c), len(first)) for c in labels], dtype=np.int64)


@pytest.mark.parametrize("name", CPU_FILES)
def test_host_minimise_and_compare_all(geq, name):
    path = _path(name, gpu=False)
    lts, olts = geq.TransitionSystem.from_csv_file(path), ora.Lts.from_csv(path)
    assert lts.n_vertices() == olts.n_vertices
    red, mp = lts.bisimilar_minimize()
    ored, omp = olts.bisimilar_minimize()
    assert red.n_vertices() == ored.n_vertices
    assert np.array_equal(np.asarray(mp, dtype=np.int64), np.asarray(omp, dtype=np.int64))
    b, info = geq.GameBuild.compare_all(red)
    ob = ora.Build.compare_all(ored)
    g = b.game
    assert np.array_equal(np.asarray(g.row_offsets, dtype=np.int64), np.asarray(ob.row, dtype=np.int64))
    assert np.array_equal(np.asarray(g.column_indices, dtype=np.int64), np.asarray(ob.col, dtype=np.int64))
    assert np.array_equal(np.asarray(g.weights.array).reshape(-1).astype(np.int64),
                          np.asarray(ob.wt, dtype=np.int64))
    assert np.array_equal(np.asarray(g.attacker_pos, dtype=np.int64), np.asarray(ob.attacker, dtype=np.int64))
    assert len(info.starting_points) == ob.n_starting


@pytest.mark.gpu
@pytest.mark.parametrize("name", FILES)
def test_device_equivalences(geq, name):
    path = _path(name, gpu=True)
    cap = int(os.environ.get("GEQ_LTS_MAX_POSITIONS", "3000000"))
    olts = ora.Lts.from_csv(path)
    ored, omp = olts.bisimilar_minimize()
    ob = ora.Build.compare_all(ored)
    if len(ob.row) - 1 > cap:
        pytest.skip(f"{name}: {len(ob.row) - 1} positions > GEQ_LTS_MAX_POSITIONS")
    sol = ora.run_game(6, 3, ob.row, ob.col, ob.wt, ob.attacker, ora.standard_reach(ob.row, ob.attacker))
    lists = sol.lists()
    starts = [(pos[1], pos[2][0]) for pos in ob.positions[:ob.n_starting]]
    oeq = ora.Equivalence(starts, lists, ored.n_vertices, omp)

    ctx = geq.Context(0)
    try:
        eq = geq.TransitionSystem.from_csv_file(path).equivalences(ctx)
        assert eq.n_starting_points() == len(starts)
        # an original process of each minimised class (the oracle's mapping)
        rep = np.full(ored.n_vertices, -1, dtype=np.int64)
        for proc in range(len(omp) - 1, -1, -1):
            rep[int(omp[proc])] = proc
        idx = np.arange(len(starts))
        if len(idx) > 200_000:
            idx = np.sort(np.random.default_rng(7).choice(len(idx), 200_000, replace=False))
        bad = 0
        for i in idx:
            pm, qm = starts[i]
            mine = eq.energies(int(rep[pm]), int(rep[qm]))
            ref = np.asarray(lists[i]).reshape(-1)
            if mine is None or sorted(mine.array.reshape(-1).tolist()) != sorted(ref.tolist()):
                bad += 1
        assert bad == 0, f"{bad} of {len(idx)} starting pairs differ"
        if len(starts) <= 20_000:
            for rel in geq.std_equivalences.names():
                r = eq.relation(geq.std_equivalences.get(rel))
                o = oeq.relation(geq.std_equivalences._T[rel])
                assert r.count_classes() == o.count_classes(), rel
                assert np.array_equal(_canon(r.classes), _canon([o.uf.find(i) for i in range(len(o))])), rel
    finally:
        ctx.close()
