"""Golden vectors transcribed from the reference crate's own tests.

Every constant cites the file:line of Gobbel2000/gpuequiv (v1.0.0) it was
copied from.  The reference is Rust + WGSL and cannot run in this image (no
Rust toolchain, no graphics stack), so these known answers are the pin for the
CPU oracle and, through it, for the CUDA path.

Energies are given as value lists (shorter lists are zero-padded, as
``Energy::new`` does); updates in the crate's i32 form (0 Zero, -1 Decrement,
k>=1 Min(k)).
"""

STANDARD = (6, 3)

# ---------------------------------------------------------------------------
# src/energy.rs unit tests
# ---------------------------------------------------------------------------
# test_energy_conf, src/energy.rs:810-842
# (elements, max) -> energy_size, energy_bits, energy_mask, update_size, update_bits, update_mask
CONF_SIZES = [
    ((4, 3), (1, 2, 0x3, 1, 4, 0xf)),
    ((6, 100), (2, 8, 0xff, 1, 4, 0xf)),
    ((30, 3), (2, 2, 0x3, 8, 8, 0xff)),
    ((4, 0xFFFFFFFF), (4, 32, 0xFFFFFFFF, 1, 4, 0xf)),
]

# test_energy, src/energy.rs:845-856
ENERGY_PACK = dict(conf=(12, 15), values=[0, 1, 2, 3, 4, 5, 6, 7, 8, 13, 14, 15],
                   words=[0x76543210, 0xfed8])

# test_energy_array, src/energy.rs:858-871: row 2 of a 4x1 array set to
# Energy::new([0,1,2,0,3]) -> bytes of the whole array.
ENERGY_ARRAY = dict(conf=(6, 3), values=[0, 1, 2, 0, 3], word=0x324,
                    unpacked=[0, 1, 2, 0, 3, 0],
                    array_bytes=[0, 0, 0, 0, 0, 0, 0, 0, 0x24, 0x3, 0, 0, 0, 0, 0, 0])

# test_energy_ord, src/energy.rs:873-886 (None = incomparable)
ENERGY_ORD = [
    ([0, 0, 0, 0, 0, 0], [1, 1, 1, 1, 1, 1], "lt"),
    ([0, 0, 0, 0, 0, 0], [0, 0, 0, 0, 0, 1], "lt"),
    ([0, 0, 0, 0, 0, 1], [1, 1, 1, 1, 1, 1], "lt"),
    ([0, 0, 0, 0, 0, 1], [1, 0, 0, 0, 0, 0], None),
    ([1, 0, 0, 0, 0, 0], [0, 0, 0, 0, 0, 1], None),
    ([0, 0, 0, 0, 0, 1], [0, 0, 0, 0, 0, 1], "eq"),
]

# std_equivalences, src/energy.rs:212-224 (test_equivalences, :888-895)
STD_EQUIVALENCES = {
    "enabledness": [1, 1],
    "traces": [3, 1],
    "failures": [3, 2, 0, 0, 1, 1],
    "failure_traces": [3, 3, 3, 0, 1, 1],
    "readiness": [3, 2, 1, 1, 1, 1],
    "readiness_traces": [3, 3, 3, 1, 1, 1],
    "revivals": [3, 2, 1, 0, 1, 1],
    "impossible_futures": [3, 2, 0, 0, 3, 1],
    "possible_futures": [3, 2, 3, 3, 3, 1],
    "simulation": [3, 3, 3, 3, 0, 0],
    "ready_simulation": [3, 3, 3, 3, 1, 1],
    "nested_2simulation": [3, 3, 3, 3, 3, 1],
    "bisimulation": [3, 3, 3, 3, 3, 3],
}

# test_update, src/energy.rs:911-929
UPDATE_PACK = dict(conf=(12, 3), values=[0, -1, 1, 2, 3, 4, 5, 6, 9, 10, 11, 12],
                   words=[0x76543210, 0xdcba])

# test_update_array, src/energy.rs:931-936
UPDATE_ARRAY = dict(conf=(6, 3), values=[0, -1, 2])

# ---------------------------------------------------------------------------
# tests/energygame.rs
# ---------------------------------------------------------------------------
# simple_graph, tests/energygame.rs:4-37
SIMPLE_ATTACKERS = [0, 2, 4, 6, 9, 11, 12, 14, 17]
SIMPLE_EDGES = [
    (0, 1, [0, 0, -1]),
    (1, 2, [0, -1, 0]),
    (2, 3, [0, 1]),
    (3, 4, [0, 0, 0, -1]),
    (4, 5, [-1, 0]),
    (5, 6, [0, -1]),
    (6, 7, [-1, 0]),
    (6, 8, [0, 0, 1]),
    (8, 4, [0, -1, 0]),
    (1, 9, [0, 0, -1]),
    (9, 10, [0, 0, -1]),
    (10, 11, [0, 0, 0, -1]),
    (11, 3, [3]),
    (10, 12, [0, 0, -1]),
    (12, 10, [0, 0, -1]),
    (0, 13, [2]),
    (13, 14, [-1]),
    (14, 15, [0, -1]),
    (14, 16, [0, 0, -1]),
    (16, 17, [0, 0, -1]),
]
# expected energies of `simple`, tests/energygame.rs:45-71
SIMPLE_EXPECTED = [
    [[1, 1]],
    [],
    [[2, 1, 0, 1]],
    [[2, 1, 0, 1]],
    [[2, 1]],
    [[1, 1]],
    [[1]],
    [[0]],
    [[2, 2]],
    [],
    [],
    [[2, 1, 2, 1]],
    [],
    [[1, 1]],
    [[0, 1]],
    [[0]],
    [],
    [],
]
# simple_one_dimension, tests/energygame.rs:73-104 (all weights -> [-1])
SIMPLE_1D_EXPECTED = [
    [[3]], [], [[3]], [[3]], [[3]], [[2]], [[1]], [[0]], [[3]],
    [], [], [[3]], [], [[2]], [[1]], [[0]], [], [],
]

# fork, tests/energygame.rs:107-129
FORK = dict(
    n=4,
    edges=[(0, 1, [0, 0, 0, -1]), (1, 2, [-1, 0]), (1, 3, [0, -1])],
    attacker=[False, True, False, False],
    expected=[
        [[1, 0, 0, 1], [0, 1, 0, 1]],
        [[1], [0, 1]],
        [[0]],
        [[0]],
    ],
)

# combinations_graph, tests/energygame.rs:132-169; expected :171-199
COMBINATIONS = dict(
    n=20,
    attackers=[1, 2, 3, 4, 6, 10, 16],
    edges=[
        (0, 1, [-1]),
        (0, 2, [0, -1]),
        (0, 3, [0, 0, 0, -1]),
        (0, 4, [0, 0, 0, 0, 0, -1]),
        (1, 5, [-1]),
        (5, 6, [-1]),
        (6, 7, [0, -1]),
        (6, 8, [-1, 0]),
        (5, 10, [3]),
        (1, 9, [0, 0, -1]),
        (9, 10, [0, 0, -1]),
        (10, 11, [-1]),
        (2, 12, [0, 0, -1]),
        (2, 13, [0, -1]),
        (3, 14, [0, 0, -1]),
        (3, 15, [0, 0, 0, 5]),
        (15, 16, [0, 0, 0, -1]),
        (16, 17, [0, 0, 0, -1]),
        (3, 18, [0, -1]),
        (4, 19, [0, 0, 0, 0, 0, -1]),
    ],
    expected=[
        [[3, 1, 1, 1, 0, 2], [2, 1, 2, 1, 0, 2]],
        [[2, 1, 1], [3, 0, 1], [1, 0, 2]],
        [[0, 0, 1], [0, 1]],
        [[0, 0, 0, 2, 2], [0, 0, 1], [0, 1]],
        [[0, 0, 0, 0, 0, 1]],
        [[1, 1, 1], [2, 0, 1]],
        [[0, 1], [1]],
        [[0]],
        [[0]],
        [[1, 0, 1]],
        [[1]],
        [[0]],
        [[0]],
        [[0]],
        [[0]],
        [[0, 0, 0, 2]],
        [[0, 0, 0, 1]],
        [[0]],
        [[0]],
        [[0]],
    ],
)


def wide(single, double):
    """`wide`, tests/energygame.rs:209-237: a defender root over `single`
    two-deep paths and `double` subtrees with two leaves each (2**double
    combinations at the root).  Returns (n, edges, attacker, expected)."""
    n = 2 * single + 3 * double + 1
    edges = []
    attacker = [False] * n
    expected = [[[0]] for _ in range(n)]
    expected[0] = [[1, 1, 2], [1, 1, 1, 1]]
    for i in range(1, single + 1):
        edges.append((0, i, [2]))
        edges.append((i, i + single, [-1]))
        attacker[i] = True
        expected[i] = [[1]]
    for i in range(1, double + 1):
        edges.append((0, 2 * single + i, [0, 0, -1]))
        edges.append((2 * single + i, 2 * single + double + i, [0, 0, -1]))
        edges.append((2 * single + i, 2 * single + double + i + 1, [0, 0, 0, -1]))
        attacker[2 * single + i] = True
        expected[2 * single + i] = [[0, 0, 1], [0, 0, 0, 1]]
    return n, edges, attacker, expected


# wide_game, tests/energygame.rs:239-243
WIDE_GAME = (1200, 150)

# ---------------------------------------------------------------------------
# src/energygame/tests.rs (defend intersection shader)
# ---------------------------------------------------------------------------
# game(), src/energygame/tests.rs:30-60: gathered energies of the four
# successors of node 0 (before the edge update) and the successor offsets
# used at :75.
DEF_ENERGIES = [
    [2, 1, 1], [3, 0, 1], [1, 0, 2],
    [0, 0, 1], [0, 1],
    [0, 0, 0, 2, 2], [0, 0, 1], [0, 1],
    [0, 0, 0, 0, 0, 1],
]
DEF_SUCC_OFFSETS = [0, 3, 5, 8, 9]
# edge weights of node 0 in game(), src/energygame/tests.rs:34-37; the
# compute pass applies them (defend_update.wgsl) before the intersection.
DEF_WEIGHTS = [[-1], [0, -1], [0, 0, 0, -1], [0, 0, 0, 0, 0, -1]]
# test_defend_intersection_shader, :96-104
DEF_EXPECTED = [[3, 1, 1, 1, 0, 2], [2, 1, 2, 1, 0, 2]]

# antichain(), src/energygame/tests.rs:176-218 (141 elements)
ANTICHAIN_141 = [
    [0, 0, 0, 2, 2, 2], [0, 0, 1, 1, 2, 2], [0, 0, 1, 2, 1, 2], [0, 0, 1, 2, 2, 1],
    [0, 0, 2, 0, 2, 2], [0, 0, 2, 1, 1, 2], [0, 0, 2, 1, 2, 1], [0, 0, 2, 2, 0, 2],
    [0, 0, 2, 2, 1, 1], [0, 0, 2, 2, 2, 0], [0, 1, 0, 1, 2, 2], [0, 1, 0, 2, 1, 2],
    [0, 1, 0, 2, 2, 1], [0, 1, 1, 0, 2, 2], [0, 1, 1, 1, 1, 2], [0, 1, 1, 1, 2, 1],
    [0, 1, 1, 2, 0, 2], [0, 1, 1, 2, 1, 1], [0, 1, 1, 2, 2, 0], [0, 1, 2, 0, 1, 2],
    [0, 1, 2, 0, 2, 1], [0, 1, 2, 1, 0, 2], [0, 1, 2, 1, 1, 1], [0, 1, 2, 1, 2, 0],
    [0, 1, 2, 2, 0, 1], [0, 1, 2, 2, 1, 0], [0, 2, 0, 0, 2, 2], [0, 2, 0, 1, 1, 2],
    [0, 2, 0, 1, 2, 1], [0, 2, 0, 2, 0, 2], [0, 2, 0, 2, 1, 1], [0, 2, 0, 2, 2, 0],
    [0, 2, 1, 0, 1, 2], [0, 2, 1, 0, 2, 1], [0, 2, 1, 1, 0, 2], [0, 2, 1, 1, 1, 1],
    [0, 2, 1, 1, 2, 0], [0, 2, 1, 2, 0, 1], [0, 2, 1, 2, 1, 0], [0, 2, 2, 0, 0, 2],
    [0, 2, 2, 0, 1, 1], [0, 2, 2, 0, 2, 0], [0, 2, 2, 1, 0, 1], [0, 2, 2, 1, 1, 0],
    [0, 2, 2, 2, 0, 0], [1, 0, 0, 1, 2, 2], [1, 0, 0, 2, 1, 2], [1, 0, 0, 2, 2, 1],
    [1, 0, 1, 0, 2, 2], [1, 0, 1, 1, 1, 2], [1, 0, 1, 1, 2, 1], [1, 0, 1, 2, 0, 2],
    [1, 0, 1, 2, 1, 1], [1, 0, 1, 2, 2, 0], [1, 0, 2, 0, 1, 2], [1, 0, 2, 0, 2, 1],
    [1, 0, 2, 1, 0, 2], [1, 0, 2, 1, 1, 1], [1, 0, 2, 1, 2, 0], [1, 0, 2, 2, 0, 1],
    [1, 0, 2, 2, 1, 0], [1, 1, 0, 0, 2, 2], [1, 1, 0, 1, 1, 2], [1, 1, 0, 1, 2, 1],
    [1, 1, 0, 2, 0, 2], [1, 1, 0, 2, 1, 1], [1, 1, 0, 2, 2, 0], [1, 1, 1, 0, 1, 2],
    [1, 1, 1, 0, 2, 1], [1, 1, 1, 1, 0, 2], [1, 1, 1, 1, 1, 1], [1, 1, 1, 1, 2, 0],
    [1, 1, 1, 2, 0, 1], [1, 1, 1, 2, 1, 0], [1, 1, 2, 0, 0, 2], [1, 1, 2, 0, 1, 1],
    [1, 1, 2, 0, 2, 0], [1, 1, 2, 1, 0, 1], [1, 1, 2, 1, 1, 0], [1, 1, 2, 2, 0, 0],
    [1, 2, 0, 0, 1, 2], [1, 2, 0, 0, 2, 1], [1, 2, 0, 1, 0, 2], [1, 2, 0, 1, 1, 1],
    [1, 2, 0, 1, 2, 0], [1, 2, 0, 2, 0, 1], [1, 2, 0, 2, 1, 0], [1, 2, 1, 0, 0, 2],
    [1, 2, 1, 0, 1, 1], [1, 2, 1, 0, 2, 0], [1, 2, 1, 1, 0, 1], [1, 2, 1, 1, 1, 0],
    [1, 2, 1, 2, 0, 0], [1, 2, 2, 0, 0, 1], [1, 2, 2, 0, 1, 0], [1, 2, 2, 1, 0, 0],
    [2, 0, 0, 0, 2, 2], [2, 0, 0, 1, 1, 2], [2, 0, 0, 1, 2, 1], [2, 0, 0, 2, 0, 2],
    [2, 0, 0, 2, 1, 1], [2, 0, 0, 2, 2, 0], [2, 0, 1, 0, 1, 2], [2, 0, 1, 0, 2, 1],
    [2, 0, 1, 1, 0, 2], [2, 0, 1, 1, 1, 1], [2, 0, 1, 1, 2, 0], [2, 0, 1, 2, 0, 1],
    [2, 0, 1, 2, 1, 0], [2, 0, 2, 0, 0, 2], [2, 0, 2, 0, 1, 1], [2, 0, 2, 0, 2, 0],
    [2, 0, 2, 1, 0, 1], [2, 0, 2, 1, 1, 0], [2, 0, 2, 2, 0, 0], [2, 1, 0, 0, 1, 2],
    [2, 1, 0, 0, 2, 1], [2, 1, 0, 1, 0, 2], [2, 1, 0, 1, 1, 1], [2, 1, 0, 1, 2, 0],
    [2, 1, 0, 2, 0, 1], [2, 1, 0, 2, 1, 0], [2, 1, 1, 0, 0, 2], [2, 1, 1, 0, 1, 1],
    [2, 1, 1, 0, 2, 0], [2, 1, 1, 1, 0, 1], [2, 1, 1, 1, 1, 0], [2, 1, 1, 2, 0, 0],
    [2, 1, 2, 0, 0, 1], [2, 1, 2, 0, 1, 0], [2, 1, 2, 1, 0, 0], [2, 2, 0, 0, 0, 2],
    [2, 2, 0, 0, 1, 1], [2, 2, 0, 0, 2, 0], [2, 2, 0, 1, 0, 1], [2, 2, 0, 1, 1, 0],
    [2, 2, 0, 2, 0, 0], [2, 2, 1, 0, 0, 1], [2, 2, 1, 0, 1, 0], [2, 2, 1, 1, 0, 0],
    [2, 2, 2, 0, 0, 0],
]
# test_defend_intersection_antichain, src/energygame/tests.rs:230-343:
# four copies of the antichain; status with 64 / 256 / 512 slots of memory.
ANTICHAIN_STATUS = [(64, -141), (256, -257), (512, 141)]

# ---------------------------------------------------------------------------
# tests/complete.rs
# ---------------------------------------------------------------------------
# example(), tests/complete.rs:9-22 (Bisping 2023, Fig. 4); label 0 = tau
EXAMPLE_LTS = [(0, 0, 0), (0, 2, 0), (0, 2, 1), (1, 1, 0), (1, 2, 1), (2, 2, 0)]
# example_game_graph, tests/complete.rs:24-75: node order of
# GameBuild::compare(0, 1) and the sorted adjacency lists.
EXAMPLE_NODES = [
    ("attack", 0, (1,), ()),
    ("attack", 2, (1,), ()),
    ("defend", 0, (1,), ()),
    ("defend", 2, (1,), ()),
    ("clause", 0, (1,), ()),
    ("clause", 2, (1,), ()),
    ("attack", 1, (0,), ()),
    ("attack", 1, (2,), ()),
    ("attack", 1, (0, 2), ()),
    ("defend", 1, (0,), ()),
    ("attack", 2, (), ()),
    ("defend", 1, (2,), ()),
    ("defend", 1, (0, 2), ()),
    ("defend", 1, (2,), (0,)),
    ("clause", 1, (0,), ()),
    ("defend", 2, (), ()),
    ("clause", 1, (2,), ()),
]
EXAMPLE_ADJ = [
    [0, 1, 2], [1, 3], [4], [5], [0, 6], [1, 7], [8, 9], [7, 10, 11],
    [8, 12, 13], [14], [15], [16], [14, 16], [6, 16], [0, 6], [], [1, 7],
]
# example_energies, tests/complete.rs:83-112
EXAMPLE_ENERGIES = [
    [[2, 2, 0, 0, 1, 1]],
    [[1, 2, 0, 0, 1, 1]],
    [[2, 2, 2, 2, 1, 1], [2, 3, 0, 0, 2, 3]],
    [[1, 1, 0, 0, 1, 1]],
    [[2, 2, 0, 2, 1, 1], [2, 3, 0, 0, 2, 3]],
    [[1, 1, 0, 0, 1, 1]],
    [[2, 3, 0, 0, 2, 2]],
    [[1, 1]],
    [[2, 3, 0, 0, 2, 2]],
    [[2, 2, 0, 0, 2, 2]],
    [[0, 1]],
    [[1, 1, 1, 1], [1, 2, 0, 0, 1, 2]],
    [[2, 2, 0, 0, 2, 2]],
    [[2, 3, 2, 0, 2, 2]],
    [[2, 2, 0, 0, 2, 2]],
    [[0]],
    [[1, 1, 0, 1], [1, 2, 0, 0, 1, 2]],
]

# bisimilar(), tests/complete.rs:116-138; test_bisimilar :140-148
BISIMILAR_LTS = [
    (0, 1, 0), (0, 2, 0), (1, 3, 0), (1, 4, 1), (2, 4, 0), (3, 0, 0), (4, 0, 0),
    (5, 6, 0), (5, 8, 0), (6, 7, 0), (6, 7, 1), (7, 5, 0), (8, 9, 0), (9, 0, 0),
]

# failure_trace(), tests/complete.rs:160-185; test_failure_trace :187-201
FAILURE_TRACE_LTS = [
    (0, 1, 0), (0, 5, 0), (1, 2, 1), (1, 3, 2), (3, 4, 3),
    (5, 6, 5), (5, 7, 2), (7, 8, 4),
    (9, 10, 0), (9, 14, 0), (10, 11, 1), (10, 12, 2), (12, 13, 4),
    (14, 15, 5), (14, 16, 2), (16, 17, 3),
]
FAILURE_TRACE_VERDICTS = {
    "failures": True, "readiness": True, "revivals": True, "traces": True,
    "failure_traces": False, "readiness_traces": False, "ready_simulation": False,
    "bisimulation": False,
}

# ---------------------------------------------------------------------------
# src/lib.rs doctests (:63-82, :94-127, :248-266, :305-324)
# ---------------------------------------------------------------------------
DOC_LTS = [(0, 1, 0), (1, 2, 1), (1, 3, 2), (4, 5, 0), (5, 7, 1), (4, 6, 0), (6, 8, 2)]
# compare(0, 4): (equivalence, holds)
DOC_COMPARE_0_4 = [("simulation", False), ("traces", True)]
# equivalences(): (kind, p, q, equivalence, expected)
DOC_EQUIVALENCES = [
    ("preorder", 4, 0, "simulation", True),
    ("equiv", 4, 0, "simulation", False),
    ("equiv", 1, 5, "enabledness", False),
    ("equiv", 3, 7, "bisimulation", True),
    ("preorder", 0, 4, "simulation", False),
    ("equiv", 0, 4, "traces", True),
]
DOC_TRACES_CLASSES = 5
DOC_TRACES_CLASS_OF_0 = [0, 4]
