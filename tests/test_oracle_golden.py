"""Pin the CPU oracle against every known answer of the reference's tests.

The oracle is then the checker for the CUDA path (tests/test_gpu_*.py).
No GPU needed.
"""
import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import STD, csr_from_edges, earray, pack_e, pack_u, ref_eq, canon, assert_same_lists
from oracle import ora


# ---- src/energy.rs unit tests ---------------------------------------------
@pytest.mark.parametrize("conf,expect", G.CONF_SIZES)
def test_conf_sizes(conf, expect):
    s = ora.conf_sizes(*conf)
    got = (s["energy_size"], s["energy_bits"], s["energy_mask"],
           s["update_size"], s["update_bits"], s["update_mask"])
    assert got == expect


def test_energy_pack_golden():
    c = G.ENERGY_PACK["conf"]
    w = ora.pack_energy(*c, G.ENERGY_PACK["values"])
    assert list(w) == G.ENERGY_PACK["words"]
    assert list(ora.unpack_energy(*c, w)) == G.ENERGY_PACK["values"]
    assert list(ora.pack_energy(*c, [])) == [0, 0]


def test_energy_array_bytes():
    c = G.ENERGY_ARRAY["conf"]
    w = ora.pack_energy(*c, G.ENERGY_ARRAY["values"])
    assert list(w) == [G.ENERGY_ARRAY["word"]]
    assert list(ora.unpack_energy(*c, w)) == G.ENERGY_ARRAY["unpacked"]
    arr = np.zeros(4, dtype=np.uint32)
    arr[2] = w[0]
    assert list(arr.view(np.uint8)) == G.ENERGY_ARRAY["array_bytes"]


def test_energy_pack_rejects():
    assert ora.pack_energy(6, 3, [4]) is None          # > max
    assert ora.pack_energy(6, 3, [0] * 7) is None      # too many values
    assert ora.pack_update(6, 3, [7]) is None          # Min(7) > elements
    assert ora.pack_update(6, 3, [-2]) is None         # invalid entry


@pytest.mark.parametrize("a,b,rel", G.ENERGY_ORD)
def test_energy_order(a, b, rel):
    ea, eb = ora.unpack_energy(6, 3, pack_e(a)), ora.unpack_energy(6, 3, pack_e(b))
    le = all(x <= y for x, y in zip(ea, eb))
    ge = all(x >= y for x, y in zip(ea, eb))
    got = "eq" if le and ge else ("lt" if le else ("gt" if ge else None))
    assert got == rel


def test_std_equivalences_pack():
    assert list(pack_e(G.STD_EQUIVALENCES["enabledness"])) == list(pack_e([1, 1]))
    assert list(pack_e(G.STD_EQUIVALENCES["bisimulation"])) == [0xfff]


def test_update_pack_golden():
    c = G.UPDATE_PACK["conf"]
    w = ora.pack_update(*c, G.UPDATE_PACK["values"])
    assert list(w) == G.UPDATE_PACK["words"]
    assert list(ora.unpack_update(*c, w)) == G.UPDATE_PACK["values"]
    assert list(ora.pack_update(*c, [])) == [0, 0]


def test_update_array():
    w = pack_u(G.UPDATE_ARRAY["values"])
    assert list(ora.unpack_update(6, 3, w)) == [0, -1, 2, 0, 0, 0]


def test_inv_update_semantics():
    # shadergen.rs:103-128: decrements first, then min-merges in index order.
    e = pack_e([1, 2, 0, 3, 0, 0])
    assert list(ora.unpack_energy(6, 3, ora.inv_update(6, 3, e, pack_u([-1, -1, 0, -1])))) == [2, 3, 0, 3, 0, 0]
    # Min(3) at dim 0: e[2] = max(e[2], e[0])
    assert list(ora.unpack_energy(6, 3, ora.inv_update(6, 3, e, pack_u([3])))) == [1, 2, 1, 3, 0, 0]
    # chained merges: dim0 -> dim1, then dim1 -> dim2 (sequential)
    e2 = pack_e([3, 0, 0])
    assert list(ora.unpack_energy(6, 3, ora.inv_update(6, 3, e2, pack_u([2, 3])))) == [3, 3, 3, 0, 0, 0]


# ---- tests/energygame.rs ---------------------------------------------------
def _simple_graph():
    att = [i in G.SIMPLE_ATTACKERS for i in range(18)]
    return csr_from_edges(18, G.SIMPLE_EDGES, att)


def _run_std(row, col, wt, att):
    reach = ora.standard_reach(row, att)
    return ora.run_game(6, 3, row, col, wt, att, reach)


def _check(sol, expected_values):
    got = sol.lists()
    exp = [earray(rows) for rows in expected_values]
    assert len(got) == len(exp)
    for v, (g, e) in enumerate(zip(got, exp)):
        assert ref_eq(g, e), (v, canon(g), canon(e))
        assert canon(g) == canon(e), v


def test_simple():
    _check(_run_std(*_simple_graph()), G.SIMPLE_EXPECTED)


def test_simple_one_dimension():
    row, col, wt, att = _simple_graph()
    wt = np.full_like(wt, pack_u([-1])[0])
    _check(_run_std(row, col, wt, att), G.SIMPLE_1D_EXPECTED)


def test_fork():
    f = G.FORK
    _check(_run_std(*csr_from_edges(f["n"], f["edges"], f["attacker"])), f["expected"])


def test_combinations():
    c = G.COMBINATIONS
    att = [i in c["attackers"] for i in range(c["n"])]
    _check(_run_std(*csr_from_edges(c["n"], c["edges"], att)), c["expected"])


def test_wide_game():
    n, edges, att, expected = G.wide(*G.WIDE_GAME)
    sol = _run_std(*csr_from_edges(n, edges, att))
    _check(sol, expected)
    # the reference's defender overflow protocol fires for the 2**150 root
    assert sol.stats["defend_retries"] >= 0


# ---- src/energygame/tests.rs -----------------------------------------------
def _def_updated():
    """DEF_ENERGIES after defend_update.wgsl applied the edge weights."""
    en = earray(G.DEF_ENERGIES).reshape(-1)
    so = G.DEF_SUCC_OFFSETS
    out = en.copy()
    for s, w in enumerate(G.DEF_WEIGHTS):
        for i in range(so[s], so[s + 1]):
            out[i] = ora.inv_update(6, 3, en[i:i + 1], pack_u(w))[0]
    return out


def test_defend_intersection_shader():
    en = _def_updated()
    st, res = ora.defend_intersection(6, 3, en, G.DEF_SUCC_OFFSETS, 64)
    assert st == 2
    assert ref_eq(res, earray(G.DEF_EXPECTED)) and canon(res) == canon(earray(G.DEF_EXPECTED))


def test_defend_intersection_large():
    # 5 identical nodes (:113-174): each node is computed independently.
    en = _def_updated()
    for _ in range(5):
        st, res = ora.defend_intersection(6, 3, en, G.DEF_SUCC_OFFSETS, 64)
        assert st == 2 and canon(res) == canon(earray(G.DEF_EXPECTED))


def test_defend_intersection_antichain_overflow_protocol():
    ac = earray(G.ANTICHAIN_141)
    assert len(ac) == 141
    en = np.concatenate([ac] * 4).reshape(-1)
    so = [0, 141, 282, 423, 564]
    for mem, status in G.ANTICHAIN_STATUS:
        st, res = ora.defend_intersection(6, 3, en, so, mem)
        assert st == status, (mem, st)
        if st >= 0:
            assert ref_eq(res, ac) and canon(res) == canon(ac)


def test_defend_intersection_mixed():
    ac = earray(G.ANTICHAIN_141)
    ac2 = ac + pack_e([1] * 6)[0]  # antichain2: every field + 1 (:220-228)
    so = [0, 141, 282, 423, 564]
    st, res = ora.defend_intersection(6, 3, np.concatenate([ac] * 4).reshape(-1), so, 512)
    assert st == 141 and ref_eq(res, ac)
    st, res = ora.defend_intersection(6, 3, np.concatenate([ac2] * 4).reshape(-1), so, 512)
    assert st == 141 and ref_eq(res, ac2)
    st, res = ora.defend_intersection(6, 3, _def_updated(), G.DEF_SUCC_OFFSETS, 64)
    assert st == 2 and canon(res) == canon(earray(G.DEF_EXPECTED))


# ---- tests/complete.rs -----------------------------------------------------
def test_example_game_graph():
    lts = ora.Lts.from_edges(G.EXAMPLE_LTS)
    b = ora.Build.compare(lts, 0, 1)
    assert b.positions == G.EXAMPLE_NODES
    assert b.n == len(G.EXAMPLE_ADJ)
    for v, exp in enumerate(G.EXAMPLE_ADJ):
        assert sorted(int(x) for x in b.adj(v)) == exp, v


def test_example_energies():
    lts = ora.Lts.from_edges(G.EXAMPLE_LTS)
    b = ora.Build.compare(lts, 0, 1)
    sol = _run_std(b.row, b.col, b.wt, b.attacker)
    _check(sol, G.EXAMPLE_ENERGIES)


def test_bisimilar():
    lts = ora.Lts.from_edges(G.BISIMILAR_LTS)
    part, _ = lts.signature_refinement()
    assert part[0] == part[5]
    e = ora.compare(lts, 0, 5)
    assert len(e) == 0
    assert ora.test_equivalence(e, G.STD_EQUIVALENCES["bisimulation"])


def test_failure_trace():
    lts = ora.Lts.from_edges(G.FAILURE_TRACE_LTS)
    e = ora.compare(lts, 0, 9)
    for name, holds in G.FAILURE_TRACE_VERDICTS.items():
        assert ora.test_equivalence(e, G.STD_EQUIVALENCES[name]) == holds, name


# ---- src/lib.rs doctests ---------------------------------------------------
def test_doc_compare():
    lts = ora.Lts.from_edges(G.DOC_LTS)
    e = ora.compare(lts, 0, 4)
    for name, holds in G.DOC_COMPARE_0_4:
        assert ora.test_equivalence(e, G.STD_EQUIVALENCES[name]) == holds


def test_doc_equivalences():
    lts = ora.Lts.from_edges(G.DOC_LTS)
    eq = ora.equivalences(lts)
    for kind, p, q, name, expect in G.DOC_EQUIVALENCES:
        f = eq.preorder if kind == "preorder" else eq.equiv
        assert f(p, q, G.STD_EQUIVALENCES[name]) == expect, (kind, p, q, name)
    traces = eq.relation(G.STD_EQUIVALENCES["traces"])
    assert traces.count_classes() == G.DOC_TRACES_CLASSES
    assert traces.class_of(0) == G.DOC_TRACES_CLASS_OF_0


def test_signature_refinement_shape():
    lts = ora.Lts.from_edges(G.DOC_LTS)
    part, cnt = lts.signature_refinement()
    # processes 2,3,7,8 are deadlocks -> one class; ids assigned in process order
    assert part[0] == 0
    assert part[2] == part[3] == part[7] == part[8]
    assert cnt == len(set(int(x) for x in part))
