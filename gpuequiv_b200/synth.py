"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference benchmarks on VLTS files (benches/benchmark.rs:16-28); these
generators stand in for them with fixed seeds:

* small_lts    40 states, 4 labels, 120 transitions, tau with p = 0.2
* large_lts    25,000 states, 12 labels (tau p = 0.15), 100,000 transitions,
               power-law out-degree (exponent 2.1, 1..64), 10% of the states
               in one strongly connected core
* stress_game  bipartite attacker/defender game, 2M positions (60% attacker,
               shuffled), 10M edges, geometric out-degree of mean 5; updates
               55% zero, 30% one decrement, 15% one min-merge
* batched_lts  states log-uniform in [20, 5000], 2..16 labels, 1.5..5
               transitions per state, tau p = 0.2, one pair p != q
* serving      Poisson arrivals of batched-style queries with 20..20,000 states
"""
from __future__ import annotations

import numpy as np

STANDARD_UPDATE_BITS = 4


def _labels(rng, m, n_labels, tau_p):
    lab = rng.integers(1, max(n_labels, 2), m)
    lab[rng.random(m) < tau_p] = 0
    return lab.astype(np.int32)


def small_lts(seed: int):
    """(src, dst, label) arrays of the small configuration."""
    rng = np.random.default_rng(seed)
    m, n = 120, 40
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    return src, dst, _labels(rng, m, 4, 0.2)


def _power_law_degrees(rng, n, total, exponent=2.1, dmax=64):
    d = np.arange(1, dmax + 1, dtype=np.float64)
    p = d ** -exponent
    p /= p.sum()
    deg = rng.choice(np.arange(1, dmax + 1), size=n, p=p).astype(np.int64)
    # rescale to exactly `total`
    deg = np.clip(np.round(deg * (total / deg.sum())), 1, dmax).astype(np.int64)
    diff = total - int(deg.sum())
    while diff != 0:
        idx = rng.integers(0, n, abs(diff))
        if diff > 0:
            ok = idx[deg[idx] < dmax]
            np.add.at(deg, ok, 1)
        else:
            ok = idx[deg[idx] > 1]
            np.add.at(deg, ok, -1)
        deg = np.clip(deg, 1, dmax)
        diff = total - int(deg.sum())
    return deg


def large_lts(seed: int = 1, n: int = 25_000, m: int = 100_000, n_labels: int = 12, tau_p: float = 0.15,
              core_frac: float = 0.10):
    rng = np.random.default_rng(seed)
    deg = _power_law_degrees(rng, n, m)
    core = int(n * core_frac)
    src = np.repeat(np.arange(n, dtype=np.uint32), deg)
    dst = rng.integers(0, n, m).astype(np.uint32)
    starts = np.concatenate([[0], np.cumsum(deg)[:-1]])
    # core states: first edge closes a Hamiltonian cycle, the others stay in the core
    in_core = src < core
    dst[in_core] = rng.integers(0, core, int(in_core.sum())).astype(np.uint32)
    cyc = starts[:core]
    dst[cyc] = (np.arange(core, dtype=np.uint32) + 1) % core
    return src, dst, _labels(rng, m, n_labels, tau_p)


def batched_lts(seed: int, smin: int = 20, smax: int = 5000):
    """One job of the batched configuration: (src, dst, label, p, q)."""
    rng = np.random.default_rng(seed)
    n = int(round(np.exp(rng.uniform(np.log(smin), np.log(smax)))))
    n_labels = int(rng.integers(2, 17))
    m = max(1, int(round(n * rng.uniform(1.5, 5.0))))
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    lab = _labels(rng, m, n_labels, 0.2)
    # make sure the LTS has exactly n states (the vertex count is the largest id + 1)
    src[0] = n - 1
    p = int(rng.integers(0, n))
    q = int(rng.integers(0, n - 1))
    if q >= p:
        q += 1
    return src, dst, lab, p, q


def serving_trace(seed: int, rate: float, duration_s: float, smin: int = 20, smax: int = 20_000):
    """Poisson arrival times (s) and one job seed per arrival."""
    rng = np.random.default_rng(seed)
    n = rng.poisson(rate * duration_s)
    t = np.sort(rng.uniform(0, duration_s, n))
    seeds = rng.integers(0, 2**31 - 1, n)
    return t, seeds


def _pack_updates(kind, pos, tgt):
    """Packed STANDARD update words: kind 0 zero, 1 decrement at pos,
    2 min-merge of pos into tgt (code tgt+2 at pos)."""
    w = np.zeros(kind.shape, dtype=np.uint32)
    dec = kind == 1
    w[dec] = (np.uint32(1) << (STANDARD_UPDATE_BITS * pos[dec]).astype(np.uint32))
    mn = kind == 2
    w[mn] = ((tgt[mn] + 2).astype(np.uint32) << (STANDARD_UPDATE_BITS * pos[mn]).astype(np.uint32))
    return w


def stress_game(seed: int = 2, n: int = 2_000_000, m: int = 10_000_000, p_att: float = 0.6, mean_deg: float = 5.0):
    """CSR (row, col, weights, attacker) of the energy-game-only stress config."""
    rng = np.random.default_rng(seed)
    att = np.zeros(n, dtype=np.uint8)
    att[:int(n * p_att)] = 1
    rng.shuffle(att)
    # geometric out-degree with support >= 0 and mean `mean_deg`
    deg = rng.geometric(1.0 / (mean_deg + 1.0), n).astype(np.int64) - 1
    diff = m - int(deg.sum())
    while diff != 0:
        idx = rng.integers(0, n, abs(diff))
        if diff > 0:
            np.add.at(deg, idx, 1)
        else:
            ok = idx[deg[idx] > 0]
            np.add.at(deg, ok, -1)
            np.maximum(deg, 0, out=deg)  # a position drawn twice
        diff = m - int(deg.sum())
    row = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(deg, out=row[1:])
    A = np.nonzero(att)[0].astype(np.uint32)
    D = np.nonzero(att == 0)[0].astype(np.uint32)
    src_att = np.repeat(att, deg).astype(bool)
    col = np.empty(m, dtype=np.uint32)
    na = int(src_att.sum())
    col[src_att] = D[rng.integers(0, len(D), na)]          # attacker -> defender
    col[~src_att] = A[rng.integers(0, len(A), m - na)]     # defender -> attacker
    r = rng.random(m)
    kind = np.where(r < 0.55, 0, np.where(r < 0.85, 1, 2)).astype(np.int64)
    pos = rng.integers(0, 6, m)
    tgt = rng.integers(0, 5, m)
    tgt = tgt + (tgt >= pos)  # uniform target != pos
    wt = _pack_updates(kind, pos, tgt)
    return row, col, wt, att


def scaled_stress_game(seed: int, n: int, m: int):
    """The stress generator at another size (parity tests)."""
    return stress_game(seed=seed, n=n, m=m)


def select_batched_jobs(n_jobs: int, max_positions: int = 200_000, first_seed: int = 0, threads: int | None = None):
    """Jobs of the batched configuration, in seed order, keeping those whose
    pair is not bisimilar and whose game has at most ``max_positions``
    positions (the spectroscopy game is exponential in the nondeterminism of
    the LTS; about a quarter of the specified jobs exceed a million
    positions).  Returns a list of dicts with the LTS arrays, the pair, the
    minimised LTS, the built game and its seed."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    from gpuequiv_b200 import GameBuild, GeqError, TransitionSystem

    threads = threads or min(32, os.cpu_count() or 4)

    def one(seed):
        src, dst, lab, p, q = batched_lts(seed)
        lts = TransitionSystem.from_arrays(src, dst, lab)
        red, mapping = lts.bisimilar_minimize()
        pm, qm = int(mapping[p]), int(mapping[q])
        if pm == qm:
            return None
        try:
            b = GameBuild.compare_bounded(red, pm, qm, max_positions)
        except GeqError:
            return None
        return dict(seed=seed, src=src, dst=dst, lab=lab, p=p, q=q, lts=lts, red=red, pm=pm, qm=qm, build=b)

    out = []
    seed = first_seed
    chunk = max(64, threads * 8)
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while len(out) < n_jobs:
            res = list(ex.map(one, range(seed, seed + chunk)))
            seed += chunk
            out.extend(r for r in res if r is not None)
    return out[:n_jobs]


MANIFEST = __import__("os").path.join(__import__("os").path.dirname(__file__), "data", "batched_seeds.json")


def write_batched_manifest(n_jobs: int = 4096, max_positions: int = 200_000, path: str = MANIFEST) -> None:
    """Record the accepted seeds of the batched configuration (with their game
    sizes) so that every consumer solves exactly the same jobs."""
    import json
    jobs = select_batched_jobs(n_jobs, max_positions)
    rows = [[j["seed"], int(j["build"].game.n_vertices()), int(j["build"].game.n_edges())] for j in jobs]
    with open(path, "w") as f:
        json.dump({"generator": "synth.batched_lts", "max_positions": max_positions,
                   "fields": ["seed", "positions", "edges"], "jobs": rows}, f, separators=(",", ":"))


def batched_manifest(path: str = MANIFEST) -> dict:
    import json
    with open(path) as f:
        return json.load(f)


if __name__ == "__main__":
    write_batched_manifest()
