"""serde JSON layouts of GameGraph (SerdeGameGraph, energygame.rs:34-109) and
TransitionSystem (lib.rs:171-219): exact layout on a small game, round trips,
and the TryFrom error messages."""
from __future__ import annotations

import json

import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import csr_from_edges


@pytest.fixture(scope="module")
def geq():
    import gpuequiv_b200 as geq
    return geq


def test_game_graph_layout(geq):
    from gpuequiv_b200 import serde
    edges = [(0, 1, [-1]), (0, 2, [0, -1]), (1, 2, [0, 0, 0, 3]), (2, 0, [4, 0, 0, 0, 0, -1])]
    row, col, wt, att = csr_from_edges(3, edges, [True, False, True])
    g = geq.GameGraph.from_csr(row, col, wt, att, geq.EnergyConf.STANDARD)
    d = serde.game_graph_to_serde(g)
    assert d == {
        "conf": {"elements": 6, "max": 3},
        "adj": [[1, 2], [2], [0]],
        "weights": [[[-1, 0, 0, 0, 0, 0], [0, -1, 0, 0, 0, 0]], [[0, 0, 0, 3, 0, 0]], [[4, 0, 0, 0, 0, -1]]],
        "attacker_pos": [True, False, True],
    }
    back = serde.game_graph_from_json(json.dumps(d))
    assert np.array_equal(back.row_offsets, g.row_offsets)
    assert np.array_equal(back.column_indices, g.column_indices)
    assert np.array_equal(back.weights.array, g.weights.array)
    assert np.array_equal(back.attacker_pos, g.attacker_pos)


def test_game_graph_round_trip_built_game(geq):
    from gpuequiv_b200 import serde
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    g = geq.GameBuild.compare(lts, 0, 1).game
    back = serde.game_graph_from_json(serde.game_graph_to_json(g))
    for a in ("row_offsets", "column_indices", "attacker_pos"):
        assert np.array_equal(getattr(back, a), getattr(g, a))
    assert back.weights == g.weights and back.get_conf() == g.get_conf()


@pytest.mark.parametrize("mutate,msg", [
    (lambda d: d["weights"].pop(), "Weight list size doesn't match adjacecy list size"),
    (lambda d: d["attacker_pos"].pop(), "attacker_pos list has wrong length"),
    (lambda d: d["adj"][0].append(1), "Out-degree in adjacency list doesn't match out-degree in weight list"),
    (lambda d: d["adj"][1].__setitem__(0, 9), "Node index too high"),
])
def test_game_graph_try_from_errors(geq, mutate, msg):
    from gpuequiv_b200 import serde
    d = {"conf": {"elements": 6, "max": 3}, "adj": [[1], [0]],
         "weights": [[[-1, 0, 0, 0, 0, 0]], [[0, 0, 0, 0, 0, 0]]], "attacker_pos": [True, False]}
    serde.game_graph_from_serde(d)
    mutate(d)
    with pytest.raises(ValueError, match=msg):
        serde.game_graph_from_serde(d)


def test_transition_system_layout_and_round_trip(geq):
    from gpuequiv_b200 import serde
    lts = geq.TransitionSystem([(0, 1, 2), (0, 2, 1), (1, 2, 0)])
    d = serde.transition_system_to_serde(lts)
    # adjacency lists sorted by label (lib.rs sort_labels)
    assert d == {"adj": [[{"process": 2, "label": 1}, {"process": 1, "label": 2}],
                         [{"process": 2, "label": 0}], []]}
    # trailing processes without transitions survive the round trip
    d["adj"].append([])
    back = serde.transition_system_from_json(json.dumps(d))
    assert back.n_vertices() == 4
    assert serde.transition_system_to_serde(back) == d
    with pytest.raises(ValueError, match="Node index too high"):
        serde.transition_system_from_serde({"adj": [[{"process": 3, "label": 0}]]})
