"""The C ABI without a GPU: symbols, packing, host modules against the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from golden import reference_vectors as G
from helpers import random_lts
from oracle import ora

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def geq():
    import gpuequiv_b200 as geq
    return geq


def header_functions():
    txt = open(os.path.join(ROOT, "include", "geq.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(geq_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(geq):
    from gpuequiv_b200 import _lib
    declared = header_functions()
    assert len(declared) >= 50
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.library_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (geq_[a-z0-9_]+)", out))
    assert set(declared) <= exported, set(declared) - exported
    assert set(declared) <= set(_lib.EXPORTED), set(declared) - set(_lib.EXPORTED)
    assert exported <= set(declared), exported - set(declared)
    assert _lib.lib.geq_abi_version() == 2


def test_conf_sizes(geq):
    for conf, expect in G.CONF_SIZES:
        c = geq.EnergyConf(*conf)
        assert (c.energy_size(), c.energy_bits(), c.energy_mask(), c.update_size(), c.update_bits(),
                c.update_mask()) == expect
    assert geq.EnergyConf.STANDARD.supported()
    assert not geq.EnergyConf.ONE_DIMENSION.supported()
    # every conf of the crate's own tests is solvable; those without a
    # thermometer codec by the multi-word solver
    for conf, _ in G.CONF_SIZES:
        assert geq.EnergyConf(*conf).solvable(), conf
    assert geq.EnergyConf.ONE_DIMENSION.solvable() and geq.EnergyConf(30, 3).solvable()
    assert not geq.EnergyConf(300, 0xFFFFFFFF).solvable()  # 300 energy words
    assert not geq.EnergyConf(0, 3).solvable()


def test_packing_golden(geq):
    c = geq.EnergyConf(*G.ENERGY_PACK["conf"])
    e = geq.Energy.new(G.ENERGY_PACK["values"], c)
    assert list(e.data) == G.ENERGY_PACK["words"]
    assert e.to_vec() == G.ENERGY_PACK["values"]
    c = geq.EnergyConf(*G.UPDATE_PACK["conf"])
    u = geq.Update.new(G.UPDATE_PACK["values"], c)
    assert list(u.data) == G.UPDATE_PACK["words"]
    assert u.to_vec() == G.UPDATE_PACK["values"]
    assert geq.Energy.new([4], geq.EnergyConf.STANDARD) is None
    assert geq.Update.new([7], geq.EnergyConf.STANDARD) is None
    assert geq.Update.new([-2], geq.EnergyConf.STANDARD) is None


def test_energy_order_and_equivalences(geq):
    c = geq.EnergyConf.STANDARD
    for a, b, rel in G.ENERGY_ORD:
        got = geq.Energy.new(a, c).partial_cmp(geq.Energy.new(b, c))
        assert got == {"lt": -1, "eq": 0, "gt": 1, None: None}[rel]
    for name, tup in G.STD_EQUIVALENCES.items():
        assert geq.std_equivalences.get(name).to_vec() == tup + [0] * (6 - len(tup))


def test_packing_random_vs_oracle(geq):
    rng = np.random.default_rng(0)
    for conf in [(6, 3), (8, 2), (4, 7), (12, 15), (3, 100)]:
        c = geq.EnergyConf(*conf)
        for _ in range(50):
            vals = [int(x) for x in rng.integers(0, conf[1] + 1, conf[0])]
            assert list(geq.Energy.new(vals, c).data) == list(ora.pack_energy(*conf, vals))
            upd = [int(x) for x in rng.integers(-1, conf[0] + 1, conf[0])]
            assert list(geq.Update.new(upd, c).data) == list(ora.pack_update(*conf, upd))


def test_test_equivalence(geq):
    c = geq.EnergyConf.STANDARD
    a = geq.EnergyArray.from_conf([[1, 1], [2]], c)
    assert not a.test_equivalence(geq.std_equivalences.traces())
    assert a.test_equivalence(geq.Energy.new([0, 3, 3, 3, 3, 3], c))
    assert geq.EnergyArray.empty(c).test_equivalence(geq.std_equivalences.enabledness())


def test_energy_array_eq_semantics(geq):
    c = geq.EnergyConf.STANDARD
    a = geq.EnergyArray.from_conf([[1], [2]], c)
    b = geq.EnergyArray.from_conf([[2], [1]], c)
    d = geq.EnergyArray.from_conf([[1], [1]], c)
    assert a == b and b == a
    # energy.rs:334-350: same length, rows of the right side among the left's
    assert a == d and not (d == a)


def test_context_without_gpu_fails_loudly(geq):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(geq.GeqError) as e:
        geq.Context(0)
    assert e.value.name == "NO_DEVICE"


def test_invalid_lts_inputs(geq):
    with pytest.raises(geq.GeqError):
        geq.TransitionSystem.from_csv_file("/nonexistent/file.csv")


@pytest.mark.parametrize("seed", range(8))
def test_lts_and_minimisation_vs_oracle(geq, seed, tmp_path):
    rng = np.random.default_rng(seed)
    edges = random_lts(rng, int(rng.integers(5, 60)), int(rng.integers(2, 6)), int(rng.integers(5, 150)))
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    assert lts.n_vertices() == olts.n_vertices
    off, tg, lb = lts.inner()
    ooff, otg, olb = olts.transitions()
    assert np.array_equal(off, ooff) and np.array_equal(tg, otg) and np.array_equal(lb, olb)
    part, cnt = lts.signature_refinement()
    opart, ocnt = olts.signature_refinement()
    assert cnt == ocnt and np.array_equal(part, opart)
    red, mp = lts.bisimilar_minimize()
    ored, omp = olts.bisimilar_minimize()
    assert np.array_equal(mp, omp)
    r1, r2 = red.inner(), ored.transitions()
    assert all(np.array_equal(x, y) for x, y in zip(r1, r2))
    # CSV round trip (lib.rs:372-406), labels written as names
    names = {0: "i"}
    path = tmp_path / "lts.csv"
    with open(path, "w") as f:
        for s, d, l in edges:
            nm = names.setdefault(l, f"act{l}")
            f.write(f'{s},{d},"{nm}"\n' if l % 2 else f"{s},{d},{nm}\n")
    a = geq.TransitionSystem.from_csv_file(str(path))
    b = ora.Lts.from_csv(str(path))
    assert all(np.array_equal(x, y) for x, y in zip(a.inner(), b.transitions()))


@pytest.mark.parametrize("seed", range(10))
def test_gamebuild_compare_exact_vs_oracle(geq, seed):
    """Same node numbering, positions and adjacency order as the reference."""
    rng = np.random.default_rng(50 + seed)
    edges = random_lts(rng, int(rng.integers(3, 25)), int(rng.integers(2, 5)), int(rng.integers(3, 50)))
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    n = lts.n_vertices()
    for _ in range(3):
        p, q = (int(x) for x in rng.integers(0, n, 2))
        if p == q:
            continue
        b = geq.GameBuild.compare(lts, p, q)
        ob = ora.Build.compare(olts, p, q)
        assert [tuple(x) for x in b.nodes] == ob.positions
        assert np.array_equal(b.game.row_offsets, ob.row)
        assert np.array_equal(b.game.column_indices, ob.col)
        assert np.array_equal(b.game.weights.array.reshape(-1), ob.wt)
        assert np.array_equal(b.game.attacker_pos, ob.attacker)


def test_gamebuild_example_exact(geq):
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    b = geq.GameBuild.compare(lts, 0, 1)
    assert [tuple(x) for x in b.nodes] == G.EXAMPLE_NODES
    for v, exp in enumerate(G.EXAMPLE_ADJ):
        assert sorted(int(x) for x in b.game.adj(v)) == exp


@pytest.mark.parametrize("seed", range(5))
def test_gamebuild_compare_all_vs_oracle(geq, seed):
    rng = np.random.default_rng(80 + seed)
    edges = random_lts(rng, int(rng.integers(5, 30)), 3, int(rng.integers(10, 60)))
    lts = geq.TransitionSystem(edges)
    olts = ora.Lts.from_edges(edges)
    b, info = geq.GameBuild.compare_all(lts)
    ob = ora.Build.compare_all(olts)
    assert b.game.n_vertices() == ob.n and b.n_starting_points == ob.n_starting
    # identical start order (classes by first process), hence identical numbering
    assert [tuple(x) for x in b.nodes] == ob.positions
    assert np.array_equal(b.game.column_indices, ob.col)


@pytest.mark.parametrize("seed", range(5))
def test_compare_all_start_pairs(geq, seed):
    """The start pairs the device build of compare_all is given
    (lts.compare_all_starts) are the host builder's start positions, in order,
    and the oracle's."""
    from gpuequiv_b200.lts import compare_all_starts
    rng = np.random.default_rng(90 + seed)
    edges = random_lts(rng, int(rng.integers(5, 30)), 3, int(rng.integers(10, 60)))
    lts = geq.TransitionSystem(edges)
    pairs = compare_all_starts(lts)
    b, _ = geq.GameBuild.compare_all(lts)
    starts = [(int(x[1]), tuple(int(v) for v in x[2])) for x in b.nodes[:b.n_starting_points]]
    assert [(p, (q,)) for p, q in pairs] == starts
    ob = ora.Build.compare_all(ora.Lts.from_edges(edges))
    assert [(p, (q,)) for p, q in pairs] == [(pos[1], pos[2]) for pos in ob.positions[:ob.n_starting]]


def test_gamebuild_bounded(geq):
    lts = geq.TransitionSystem(G.EXAMPLE_LTS)
    with pytest.raises(geq.GeqError) as e:
        geq.GameBuild.compare_bounded(lts, 0, 1, 5)
    assert e.value.name == "OUT_OF_MEMORY"
    b = geq.GameBuild.compare_bounded(lts, 0, 1, 100)
    assert b.game.n_vertices() == 17


def test_device_codec_host_exhaustive(tmp_path):
    """The thermometer codecs of codec.cuh, compiled for the host, against the
    oracle's field-wise arithmetic on every STANDARD energy."""
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstdint>
#include "codec.cuh"
using namespace geq;
int main() {
  CodecStd s; CodecGen g(6, 3, 2, 3, 4, 15);
  unsigned bad = 0;
  for (uint32_t p = 0; p < 4096; p++) {
    if (s.to_p(s.to_t(p)) != p) bad++;
    if (g.to_p(g.to_t(p)) != p) bad++;
  }
  // print updates applied to all energies for the Python side to compare
  const uint32_t ups[] = {0u, 0x1u, 0x10u, 0x4u, 0x4000u, 0x5u, 0x100006u, 0x111111u, 0x234567u, 0x765432u,
                          0x32u, 0x2003u, 0x700000u, 0x11u};
  for (uint32_t u : ups)
    for (uint32_t p = 0; p < 4096; p++)
      std::printf("%u %u %u %u\n", u, p, s.to_p(s.upd(s.to_t(p), u)), g.to_p(g.upd(g.to_t(p), u)));
  // pseudo-random valid STANDARD updates (every field code 0..7)
  uint32_t r = 12345u;
  for (int k = 0; k < 48; k++) {
    uint32_t u = 0;
    for (int i = 0; i < 6; i++) {
      r = r * 1664525u + 1013904223u;
      const uint32_t c = (r >> 24) % 10u;
      u |= (c < 8u ? c : 0u) << (4 * i);
    }
    for (uint32_t p = 0; p < 4096; p++)
      std::printf("%u %u %u %u\n", u, p, s.to_p(s.upd(s.to_t(p), u)), g.to_p(g.upd(g.to_t(p), u)));
  }
  // order: (a & ~b) == 0 iff field-wise <=
  for (uint32_t a = 0; a < 4096; a += 7)
    for (uint32_t b = 0; b < 4096; b += 5) {
      bool le = true;
      for (int i = 0; i < 6; i++) if (((a >> 2*i) & 3) > ((b >> 2*i) & 3)) le = false;
      if (t_leq(s.to_t(a), s.to_t(b)) != le) bad++;
      if (t_leq(g.to_t(a), g.to_t(b)) != le) bad++;
      uint32_t mx = 0;
      for (int i = 0; i < 6; i++) { uint32_t x = (a >> 2*i) & 3, y = (b >> 2*i) & 3; mx |= (x > y ? x : y) << 2*i; }
      if (s.to_p(s.to_t(a) | s.to_t(b)) != mx) bad++;
      if (g.to_p(g.to_t(a) | g.to_t(b)) != mx) bad++;
    }
  std::fprintf(stderr, "bad=%u\n", bad);
  return bad ? 1 : 0;
}
''')
    exe = tmp_path / "t"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "gpuequiv_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rows = np.array([list(map(int, l.split())) for l in r.stdout.splitlines()], dtype=np.uint64)
    # oracle inverse update on the same (update, energy) pairs
    for u in np.unique(rows[:, 0]):
        sel = rows[rows[:, 0] == u]
        for p, a, b in sel[::17, 1:]:
            want = ora.inv_update(6, 3, [int(p)], [int(u)])[0]
            assert a == want and b == want, (hex(int(u)), int(p), int(a), int(b), int(want))
