"""serde JSON of GameGraph and TransitionSystem in the crate's layouts.

With the crate's `serde` feature, `GameGraph` (de)serialises through
`SerdeGameGraph` (energygame.rs:34-109)::

    {"conf": {"elements": 6, "max": 3},
     "adj": [[successor, ...], ...],              # per position
     "weights": [[[update value, ...], ...], ...], # per position, per edge
     "attacker_pos": [true, false, ...]}

with update values as in `Update::new` (0 = Zero, -1 = Decrement, k = Min(k)),
and `TransitionSystem` (lib.rs:171-219) as
``{"adj": [[{"process": p, "label": l}, ...], ...]}``.  Reading checks what
`TryFrom<SerdeGameGraph>` checks (energygame.rs:65-83) and fails with its
messages (as ValueError).
"""
from __future__ import annotations

import json

import numpy as np

from .energy import EnergyConf, UpdateArray
from .energygame import GameGraph


def _update_values(weights: UpdateArray) -> np.ndarray:
    """(m, elements) int32 update values of packed update rows."""
    conf = weights.conf
    m = weights.n_updates()
    ub, um = conf.update_bits(), conf.update_mask()
    per_word = 32 // ub
    out = np.zeros((m, conf.elements), dtype=np.int32)
    for i in range(conf.elements):
        w = weights.array[:, i // per_word].astype(np.int64)
        code = (w >> (ub * (i % per_word))) & um
        out[:, i] = np.where(code == 0, 0, np.where(code == 1, -1, code - 1))
    return out


def game_graph_to_serde(g: GameGraph) -> dict:
    """SerdeGameGraph of a GameGraph (From<GameGraph>, energygame.rs:46-63)."""
    row = g.row_offsets.astype(np.int64)
    col = g.column_indices.tolist()
    vals = _update_values(g.weights).tolist()
    adj, weights = [], []
    for v in range(g.n_vertices()):
        a, b = int(row[v]), int(row[v + 1])
        adj.append(col[a:b])
        weights.append(vals[a:b])
    return {"conf": {"elements": g.conf.elements, "max": g.conf.max}, "adj": adj, "weights": weights,
            "attacker_pos": [bool(x) for x in g.attacker_pos]}


def game_graph_from_serde(d: dict) -> GameGraph:
    """GameGraph of a SerdeGameGraph (TryFrom, energygame.rs:65-109)."""
    conf = EnergyConf(int(d["conf"]["elements"]), int(d["conf"]["max"]))
    adj, weights, att = d["adj"], d["weights"], d["attacker_pos"]
    n = len(adj)
    if len(weights) != n:
        raise ValueError("Weight list size doesn't match adjacecy list size")
    if len(att) != n:
        raise ValueError("attacker_pos list has wrong length")
    for succ, wts in zip(adj, weights):
        if len(succ) != len(wts):
            raise ValueError("Out-degree in adjacency list doesn't match out-degree in weight list")
        if not all(0 <= s < n for s in succ):
            raise ValueError("Node index too high")
    row = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum([len(a) for a in adj], out=row[1:])
    col = np.array([s for a in adj for s in a], dtype=np.uint32)
    ua = UpdateArray.from_conf([u for w in weights for u in w], conf)
    return GameGraph.from_csr(row, col, ua.array, np.array([1 if a else 0 for a in att], np.uint8), conf)


def game_graph_to_json(g: GameGraph) -> str:
    return json.dumps(game_graph_to_serde(g))


def game_graph_from_json(s: str) -> GameGraph:
    return game_graph_from_serde(json.loads(s))


def transition_system_to_serde(lts) -> dict:
    """The crate's TransitionSystem layout: adjacency lists sorted by label."""
    off, tgt, lab = lts.inner()
    adj = []
    for p in range(lts.n_vertices()):
        a, b = int(off[p]), int(off[p + 1])
        adj.append([{"process": int(t), "label": int(l)} for t, l in zip(tgt[a:b], lab[a:b])])
    return {"adj": adj}


def transition_system_from_serde(d: dict):
    from .lts import TransitionSystem
    adj = d["adj"]
    n = len(adj)
    src = np.array([p for p, ts in enumerate(adj) for _ in ts], dtype=np.uint32)
    dst = np.array([t["process"] for ts in adj for t in ts], dtype=np.uint32)
    lab = np.array([t["label"] for ts in adj for t in ts], dtype=np.int32)
    if len(dst) and int(dst.max()) >= n:
        raise ValueError("Node index too high")
    lts = TransitionSystem.from_arrays(src, dst, lab, n_vertices=n)
    return lts


def transition_system_to_json(lts) -> str:
    return json.dumps(transition_system_to_serde(lts))


def transition_system_from_json(s: str):
    return transition_system_from_serde(json.loads(s))
