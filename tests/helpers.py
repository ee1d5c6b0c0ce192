"""Shared test helpers: CSR construction, packing and list comparison.

The oracle (``oracle.ora``) is the checker; these helpers only shape inputs.
"""
from __future__ import annotations

import numpy as np

from oracle import ora

STD = (6, 3)


def pack_e(values, conf=STD):
    w = ora.pack_energy(conf[0], conf[1], values)
    assert w is not None, values
    return w


def pack_u(values, conf=STD):
    w = ora.pack_update(conf[0], conf[1], values)
    assert w is not None, values
    return w


def earray(rows, conf=STD):
    """earray! macro of the reference tests: value lists -> (k, esize) words."""
    es = ora.lib().ora_energy_size(*conf)
    if not rows:
        return np.zeros((0, es), dtype=np.uint32)
    return np.stack([pack_e(r, conf) for r in rows]).astype(np.uint32)


def csr_from_edges(n, edges, attacker, conf=STD):
    """GameGraph::new (energygame.rs:141-194): successors grouped per source
    in edge order.  ``edges`` = (from, to, update-values)."""
    us = ora.lib().ora_update_size(*conf)
    adj = [[] for _ in range(n)]
    wts = [[] for _ in range(n)]
    for f, t, u in edges:
        adj[f].append(t)
        wts[f].append(pack_u(u, conf) if not isinstance(u, np.ndarray) else u)
    row = np.zeros(n + 1, dtype=np.uint32)
    for v in range(n):
        row[v + 1] = row[v] + len(adj[v])
    col = np.array([t for a in adj for t in a], dtype=np.uint32)
    wt = (np.concatenate([w for ws in wts for w in ws]).astype(np.uint32)
          if row[n] else np.zeros(0, dtype=np.uint32))
    assert wt.size == row[n] * us
    att = np.array([1 if a else 0 for a in attacker], dtype=np.uint8)
    return row, col, wt, att


def canon(lst):
    """Canonical (sorted) form of one position's energy list, as tuples."""
    a = np.asarray(lst, dtype=np.uint32)
    if a.size == 0:
        return []
    if a.ndim == 1:
        a = a.reshape(-1, 1)
    return sorted(tuple(int(x) for x in r) for r in a)


def ref_eq(self_rows, other_rows):
    """EnergyArray == (energy.rs:334-350): same row count and every row of
    ``other`` occurs in ``self``."""
    a = canon(self_rows)
    b = canon(other_rows)
    if len(a) != len(b):
        return False
    s = set(a)
    return all(r in s for r in b)


def assert_same_lists(got, expected, what=""):
    assert len(got) == len(expected), f"{what}: {len(got)} positions vs {len(expected)}"
    for v, (g, e) in enumerate(zip(got, expected)):
        assert canon(g) == canon(e), f"{what}: position {v}: {canon(g)} != {canon(e)}"


def random_lts(rng, n_states, n_labels, n_trans, tau_p=0.2):
    src = rng.integers(0, n_states, n_trans)
    dst = rng.integers(0, n_states, n_trans)
    lab = np.where(rng.random(n_trans) < tau_p, 0, rng.integers(1, max(n_labels, 2), n_trans))
    return [(int(a), int(b), int(c)) for a, b, c in zip(src, dst, lab)]
