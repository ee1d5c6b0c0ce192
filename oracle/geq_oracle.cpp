// geq_oracle.cpp - CPU restatement of gpuequiv's energy-game path.
//
// TEST INFRASTRUCTURE ONLY (the parity oracle and the CPU baseline).  The
// product library never links or calls this file.  Each function below cites
// the reference file:line (paths inside the Gobbel2000/gpuequiv crate) whose
// behaviour it restates.  The restatement is deliberately plain and
// sequential: it mirrors the reference's algorithm (Jacobi worklist, O(K^2)
// attacker minimisation, chunked defender fold with its memory protocol), not
// an optimised one.

#include "geq_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// EnergyConf (src/energy.rs:36-78)
// ---------------------------------------------------------------------------
uint32_t leading_zeros(uint32_t x) { return x == 0 ? 32u : (uint32_t)__builtin_clz(x); }
uint32_t next_pow2(uint32_t x) {  // u32::next_power_of_two (0 -> 1)
  if (x <= 1) return 1;
  return 1u << (32 - leading_zeros(x - 1));
}

struct Conf {
  uint32_t elements, max;
  // energy.rs:56-59
  uint32_t energy_bits() const { return next_pow2(32 - leading_zeros(max)); }
  // energy.rs:61-63
  uint32_t energy_mask() const { return 0xffffffffu >> (32 - energy_bits()); }
  // energy.rs:49-53
  uint32_t energy_size() const { return (energy_bits() * elements + 31) / 32; }
  // energy.rs:70-73
  uint32_t update_bits() const { return next_pow2(32 - leading_zeros(elements + 2)); }
  uint32_t update_mask() const { return 0xffffffffu >> (32 - update_bits()); }
  // energy.rs:65-68
  uint32_t update_size() const { return (update_bits() * elements + 31) / 32; }
};

// Field extraction as generated by shadergen.rs:87-101 (`unpack`): the shift
// advances by `bits` and wraps to the next word once it reaches 32.
void unpack_fields(const uint32_t *w, uint32_t n, uint32_t bits, uint32_t mask,
                   uint32_t *out) {
  uint32_t shift = 0, word = 0;
  for (uint32_t i = 0; i < n; i++) {
    out[i] = (w[word] >> shift) & mask;
    shift += bits;
    if (shift >= 32) { shift = 0; word++; }
  }
}

// pack_energy, src/energy.rs:143-162.
bool pack_energy(const Conf &c, const uint32_t *vals, uint32_t n, uint32_t *out) {
  if (n > c.elements) return false;
  uint32_t es = c.energy_size(), bits = c.energy_bits();
  for (uint32_t i = 0; i < es; i++) out[i] = 0;
  uint32_t shift = 0, word = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (vals[i] > c.max) return false;
    out[word] |= vals[i] << shift;
    shift += bits;
    if (shift + bits > 32) { shift = 0; word++; }
  }
  return true;
}

// Upd::packed_repr (energy.rs:454-460) and From<i32> (energy.rs:474-490),
// pack_upd (energy.rs:543-565).
bool pack_update(const Conf &c, const int32_t *vals, uint32_t n, uint32_t *out) {
  if (n > c.elements) return false;
  uint32_t us = c.update_size(), bits = c.update_bits();
  for (uint32_t i = 0; i < us; i++) out[i] = 0;
  uint32_t shift = 0, word = 0;
  for (uint32_t i = 0; i < n; i++) {
    int32_t v = vals[i];
    uint32_t repr;
    if (v == 0) repr = 0;
    else if (v == -1) repr = 1;
    else if (v < -1) return false;  // "Invalid update entry" panics in the crate
    else {
      if ((uint32_t)v > c.elements) return false;  // Min is 1-indexed, energy.rs:551-556
      repr = (uint32_t)v + 1;
    }
    out[word] |= repr << shift;
    shift += bits;
    if (shift + bits > 32) { shift = 0; word++; }
  }
  return true;
}

// Generated arithmetic of shadergen.rs: UNPACK_ENERGY/UNPACK_UPDATE (:87-101),
// UPDATE1 (:103-111), UPDATE_MIN (:113-128), PACK_ENERGY (:130-149), applied
// as inv_update in attack_update.wgsl:45-61 / defend_update.wgsl:41-57.
struct Arith {
  Conf c;
  uint32_t es, us, ebits, emask, ubits, umask;
  explicit Arith(Conf cc) : c(cc) {
    es = c.energy_size(); us = c.update_size();
    ebits = c.energy_bits(); emask = c.energy_mask();
    ubits = c.update_bits(); umask = c.update_mask();
  }
  void inv_update(const uint32_t *e, const uint32_t *u, uint32_t *out) const {
    std::vector<uint32_t> v(c.elements), upd(c.elements);
    unpack_fields(e, c.elements, ebits, emask, v.data());
    unpack_fields(u, c.elements, ubits, umask, upd.data());
    for (uint32_t i = 0; i < c.elements; i++) {
      uint32_t x = v[i] + (upd[i] == 1u ? 1u : 0u);  // u32 arithmetic wraps
      v[i] = std::min(x, c.max);
    }
    for (uint32_t i = 0; i < c.elements; i++) {
      uint32_t k = upd[i];
      if (k > 1u) {
        k -= 2u;
        // Codes that name no element cannot be produced by pack_upd; such
        // targets are ignored here (the C ABI rejects them as invalid input).
        if (k < c.elements) v[k] = std::max(v[k], v[i]);
      }
    }
    pack(v.data(), out);
  }
  // PACK_ENERGY (shadergen.rs:130-149)
  void pack(const uint32_t *v, uint32_t *out) const {
    uint32_t i = 0;
    for (uint32_t w = 0; w < es; w++) {
      uint32_t word = 0;
      for (uint32_t shift = 0; shift < 32; shift += ebits) {
        word |= v[i] << shift;
        i++;
        if (i >= c.elements) break;
      }
      out[w] = word;
      if (i >= c.elements) {
        for (uint32_t r = w + 1; r < es; r++) out[r] = 0;
        break;
      }
    }
  }
  // IMPL_LESS_EQ (shadergen.rs:55-73): masked field-wise <=.
  bool less_eq(const uint32_t *a, const uint32_t *b) const {
    uint32_t shift = 0, word = 0;
    for (uint32_t i = 0; i < c.elements; i++) {
      uint32_t m = emask << shift;
      if ((a[word] & m) > (b[word] & m)) return false;
      shift += ebits;
      if (shift >= 32) { shift = 0; word++; }
    }
    return true;
  }
  // IMPL_EQ (shadergen.rs:75-85)
  bool eq(const uint32_t *a, const uint32_t *b) const {
    for (uint32_t i = 0; i < es; i++)
      if (a[i] != b[i]) return false;
    return true;
  }
  // MAX_SUPREMUM (shadergen.rs:151-157) on unpacked fields, repacked.
  void supremum(const uint32_t *a, const uint32_t *b, uint32_t *out) const {
    std::vector<uint32_t> va(c.elements), vb(c.elements);
    unpack_fields(a, c.elements, ebits, emask, va.data());
    unpack_fields(b, c.elements, ebits, emask, vb.data());
    for (uint32_t i = 0; i < c.elements; i++) va[i] = std::max(va[i], vb[i]);
    pack(va.data(), out);
  }
};

// ---------------------------------------------------------------------------
// Game graph (src/energygame.rs:120-250)
// ---------------------------------------------------------------------------
struct Graph {
  Conf conf;
  uint32_t n = 0;
  std::vector<uint32_t> row, col, wt;   // CSR, wt has m*update_size words
  std::vector<uint32_t> rrow, rcol;     // reverse CSR (make_reverse, :235-250)
  std::vector<uint8_t> attacker;

  void make_reverse() {
    std::vector<uint32_t> cnt(n + 1, 0);
    for (uint32_t v = 0; v < n; v++)
      for (uint32_t k = row[v]; k < row[v + 1]; k++) cnt[col[k] + 1]++;
    rrow.assign(n + 1, 0);
    for (uint32_t v = 0; v < n; v++) rrow[v + 1] = rrow[v] + cnt[v + 1];
    rcol.assign(rrow[n], 0);
    std::vector<uint32_t> fill(rrow.begin(), rrow.end() - 1);
    // predecessors are listed in increasing source order, like the
    // Vec::push loop in make_reverse.
    for (uint32_t v = 0; v < n; v++)
      for (uint32_t k = row[v]; k < row[v + 1]; k++) rcol[fill[col[k]]++] = v;
  }
};

using EList = std::vector<uint32_t>;  // flat list of packed energies

struct Stats {
  uint64_t rounds = 0, atk_visits = 0, def_visits = 0, def_retries = 0;
  uint64_t edges_relaxed = 0, bytes = 0;
};

// EnergyArray: PartialEq<ArrayBase> (energy.rs:334-350): `self == other` iff
// the shapes match and every row of `other` occurs among the rows of `self`.
bool earray_eq(const Arith &ar, const EList &self, const EList &other) {
  if (self.size() != other.size()) return false;
  uint32_t es = ar.es;
  size_t n = self.size() / es;
  for (size_t i = 0; i < n; i++) {
    bool found = false;
    for (size_t j = 0; j < n && !found; j++)
      found = ar.eq(&self[j * es], &other[i * es]);
    if (!found) return false;
  }
  return true;
}

// defend_iterative.wgsl:123-180 `minimize`, executed for one workgroup of 64
// invocations.  All reads of a chunk happen before its writes, as the
// workgroup/storage barriers in the shader guarantee.
uint32_t wg_minimize(const Arith &ar, std::vector<uint32_t> &sup, uint32_t sbase,
                     uint32_t extra_shift, uint32_t size) {
  const uint32_t es = ar.es;
  uint32_t n_minimized = 0;
  uint32_t nbase = sbase + extra_shift;
  std::vector<uint32_t> val(64 * es);
  uint32_t flag[64];
  for (uint32_t chunk = 0; chunk < size; chunk += 64) {
    for (uint32_t l = 0; l < 64; l++) {
      uint32_t i = chunk + l;
      uint32_t extra_i = i + extra_shift;
      flag[l] = 0;
      if (i >= size) continue;
      const uint32_t *energy = &sup[(nbase + i) * es];
      std::copy(energy, energy + es, &val[l * es]);
      uint32_t is_minimal = 1;
      for (uint32_t j = 0; j < n_minimized; j++) {
        const uint32_t *e2 = &sup[(sbase + j) * es];
        bool eq = ar.eq(e2, energy);
        if (j != extra_i && ((eq && extra_i > j) || (!eq && ar.less_eq(e2, energy))))
          is_minimal = 0;
      }
      if (is_minimal) {
        for (uint32_t j = chunk; j < size; j++) {
          const uint32_t *e2 = &sup[(nbase + j) * es];
          bool eq = ar.eq(e2, energy);
          if (j != i && ((eq && i > j) || (!eq && ar.less_eq(e2, energy))))
            is_minimal = 0;
        }
      }
      flag[l] = is_minimal;
    }
    // prefix_sum (defend_iterative.wgsl:81-113): exclusive scan + total.
    uint32_t prefix = 0;
    for (uint32_t l = 0; l < 64; l++) {
      if (flag[l]) {
        std::copy(&val[l * es], &val[l * es] + es, &sup[(sbase + n_minimized + prefix) * es]);
        prefix++;
      }
    }
    n_minimized += prefix;
  }
  return n_minimized;
}

// defend_iterative.wgsl:182-267 `intersection` for one defender node.
// `en` holds the already inv-updated energies of the successors back to back,
// `so` the n_succ+1 region offsets (relative to en).  Returns the status.
int32_t wg_intersection(const Arith &ar, const uint32_t *en, const uint32_t *so,
                        uint32_t n_succ, uint32_t available_mem, EList &result) {
  const uint32_t es = ar.es;
  if (n_succ == 0) return 0;  // :291-293, never reached from the worklist
  std::vector<uint32_t> sup((size_t)available_mem * es + 64 * es, 0);
  uint32_t slen = so[1] - so[0];
  if (slen > available_mem) return -(int32_t)slen;  // :303-307
  for (uint32_t i = 0; i < slen; i++)
    std::copy(&en[(so[0] + i) * es], &en[(so[0] + i) * es] + es, &sup[i * es]);
  std::vector<uint32_t> tmp(es);
  for (uint32_t suc = 1; suc < n_succ; suc++) {
    uint32_t suc_width = so[suc + 1] - so[suc];
    uint32_t comb_size = slen * suc_width;
    uint32_t n_minimized = 0;
    for (uint32_t chunk = 0; chunk < comb_size; chunk += 64) {
      uint32_t required = slen + n_minimized + std::min(comb_size - chunk, 64u);
      if (required > available_mem) return -(int32_t)required;  // :329-334
      for (uint32_t l = 0; l < 64; l++) {
        uint32_t i = chunk + l;
        if (i >= comb_size) continue;
        uint32_t prev_pick = i % slen, next_pick = i / slen;
        ar.supremum(&sup[prev_pick * es], &en[(so[suc] + next_pick) * es], tmp.data());
        std::copy(tmp.begin(), tmp.end(), &sup[(slen + n_minimized + l) * es]);
      }
      if (chunk + 64 >= comb_size) {
        uint32_t size = n_minimized + comb_size - chunk;
        slen = wg_minimize(ar, sup, 0, slen, size);
      } else {
        n_minimized = wg_minimize(ar, sup, slen, 0, n_minimized + 64);
      }
    }
  }
  result.assign(sup.begin(), sup.begin() + (size_t)slen * es);
  return (int32_t)slen;
}

// DefendIterShader::DEFAULT_SUPREMA_MEMORY (energygame.rs:505)
constexpr uint32_t DEFAULT_SUPREMA_MEMORY = 64;

// GPURunner::execute_gpu and the collect/process steps of AttackShader and
// DefendIterShader (energygame.rs:1258-1426, :774-944, :1461-1523).
// The dispatch/binding-size limits that make the reference split a round
// (:783-825, :1282-1295) are not modelled: they only move work to a later
// round.
void run_game(const Graph &g, std::vector<EList> &E, const std::vector<uint32_t> &to_reach,
              Stats &st) {
  const Arith ar(g.conf);
  const uint32_t es = ar.es, us = ar.us;
  const uint32_t n = g.n;
  std::vector<uint8_t> atk_in(n, 0);
  std::vector<uint32_t> atk_list;
  std::vector<uint32_t> def_mem(n, 0);  // 0 = not in the visit map
  std::vector<uint32_t> def_list;

  // changed_nodes (:1467-1479)
  auto changed_nodes = [&](const std::vector<uint32_t> &nodes) {
    for (uint32_t v : nodes) {
      for (uint32_t k = g.rrow[v]; k < g.rrow[v + 1]; k++) {
        uint32_t w = g.rcol[k];
        if (g.attacker[w]) {
          if (!atk_in[w]) { atk_in[w] = 1; atk_list.push_back(w); }
        } else if (def_mem[w] == 0) {  // entry(w).or_insert(DEFAULT)
          def_mem[w] = DEFAULT_SUPREMA_MEMORY;
          def_list.push_back(w);
        }
      }
    }
  };
  changed_nodes(to_reach);  // initialize_visit_lists (:1461-1465)

  std::vector<uint32_t> cand, upd_tmp(es);
  std::vector<uint8_t> keep;
  for (;;) {
    st.rounds++;
    // ---- collect (snapshot of E at round start) ----
    std::vector<uint32_t> atk_nodes;
    atk_nodes.swap(atk_list);
    for (uint32_t v : atk_nodes) atk_in[v] = 0;
    std::vector<std::pair<uint32_t, uint32_t>> def_nodes;
    for (uint32_t v : def_list) {
      uint32_t mem = def_mem[v];
      def_mem[v] = 0;
      bool any_empty = false;  // :789-792
      for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++)
        if (E[g.col[k]].empty()) { any_empty = true; break; }
      if (!any_empty) def_nodes.emplace_back(v, mem);
    }
    def_list.clear();

    // ---- attack: update + minimize (attack_update.wgsl:77-113,
    //      attack_minimize.wgsl:69-122) ----
    std::vector<std::pair<uint32_t, EList>> atk_res;
    for (uint32_t v : atk_nodes) {
      st.atk_visits++;
      cand.clear();
      for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++) {
        const EList &ew = E[g.col[k]];
        st.edges_relaxed++;
        st.bytes += 16 + 4ull * (ew.size() / es);
        for (size_t x = 0; x < ew.size(); x += es) {
          ar.inv_update(&ew[x], &g.wt[(size_t)k * us], upd_tmp.data());
          cand.insert(cand.end(), upd_tmp.begin(), upd_tmp.end());
        }
      }
      size_t own_start = cand.size() / es;
      std::vector<uint32_t> zero(us, 0);
      for (size_t x = 0; x < E[v].size(); x += es) {  // own energies, zero update
        ar.inv_update(&E[v][x], zero.data(), upd_tmp.data());
        cand.insert(cand.end(), upd_tmp.begin(), upd_tmp.end());
      }
      size_t K = cand.size() / es;
      keep.assign(K, 1);
      bool changed = false;
      for (size_t i = 0; i < K; i++) {
        const uint32_t *ei = &cand[i * es];
        for (size_t j = 0; j < K; j++) {
          const uint32_t *e2 = &cand[j * es];
          bool eq = ar.eq(e2, ei);
          if (j != i && ((eq && i < j) || (!eq && ar.less_eq(e2, ei)))) { keep[i] = 0; break; }
        }
        if (keep[i] && i < own_start) changed = true;
      }
      st.bytes += 8 + 4ull * (E[v].size() / es) + 4;
      if (changed) {
        EList nw;
        for (size_t i = 0; i < K; i++)
          if (keep[i]) nw.insert(nw.end(), &cand[i * es], &cand[i * es] + es);
        st.bytes += 4ull * (nw.size() / es);
        atk_res.emplace_back(v, std::move(nw));
      }
    }

    // ---- defend: defend_update.wgsl:73-101 + intersection ----
    struct DefRes { uint32_t v; int32_t status; EList list; };
    std::vector<DefRes> def_res;
    for (auto &vm : def_nodes) {
      uint32_t v = vm.first;
      st.def_visits++;
      EList en;
      std::vector<uint32_t> so;
      for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++) {
        const EList &ew = E[g.col[k]];
        st.edges_relaxed++;
        st.bytes += 16 + 4ull * (ew.size() / es);
        so.push_back((uint32_t)(en.size() / es));
        for (size_t x = 0; x < ew.size(); x += es) {
          ar.inv_update(&ew[x], &g.wt[(size_t)k * us], upd_tmp.data());
          en.insert(en.end(), upd_tmp.begin(), upd_tmp.end());
        }
      }
      so.push_back((uint32_t)(en.size() / es));
      DefRes r{v, 0, {}};
      r.status = wg_intersection(ar, en.data(), so.data(), (uint32_t)so.size() - 1, vm.second, r.list);
      st.bytes += 8 + 4;
      def_res.push_back(std::move(r));
    }

    // ---- process_results (:1372-1426 then :896-944) ----
    std::vector<uint32_t> changed;
    for (auto &r : atk_res) {
      E[r.first] = std::move(r.second);
      changed.push_back(r.first);
    }
    changed_nodes(changed);
    changed.clear();
    for (auto &r : def_res) {
      if (r.status < 0) {  // insufficient suprema memory: retry with more
        st.def_retries++;
        uint32_t need = (uint32_t)(-(int64_t)r.status);
        uint32_t next = std::max(next_pow2(need), 128u);
        if (def_mem[r.v] == 0) def_list.push_back(r.v);
        def_mem[r.v] = next;  // visit_list.insert overwrites
        continue;
      }
      if (!earray_eq(ar, E[r.v], r.list)) {  // `new_array != energies[node]`
        st.bytes += 4ull * (r.list.size() / es);
        E[r.v] = std::move(r.list);
        changed.push_back(r.v);
      }
    }
    changed_nodes(changed);
    if (atk_list.empty() && def_list.empty()) break;
  }
}

// ---------------------------------------------------------------------------
// TransitionSystem (src/lib.rs)
// ---------------------------------------------------------------------------
struct Tr { uint32_t process; int32_t label; };

struct Lts {
  std::vector<std::vector<Tr>> adj;
  uint32_t n() const { return (uint32_t)adj.size(); }
  // TransitionSystem::sort_labels (lib.rs:489-493): stable sort by label.
  void sort_labels() {
    for (auto &row : adj)
      std::stable_sort(row.begin(), row.end(), [](const Tr &a, const Tr &b) { return a.label < b.label; });
  }
};

// FromIterator<Edge> (lib.rs:523-536)
Lts lts_from_edges(uint64_t m, const uint32_t *src, const uint32_t *dst, const int32_t *lab) {
  Lts l;
  for (uint64_t i = 0; i < m; i++) {
    size_t mx = std::max<size_t>(src[i], dst[i]);
    if (mx >= l.adj.size()) l.adj.resize(mx + 1);
    l.adj[src[i]].push_back(Tr{dst[i], lab[i]});
  }
  l.sort_labels();
  return l;
}

// signatures (lib.rs:468-478) / signature_refinement (lib.rs:444-464)
std::vector<uint64_t> signature_refinement(const Lts &l, uint64_t &count) {
  uint32_t n = l.n();
  std::vector<uint64_t> part(n, 0);
  uint64_t prev = 0, cur = 1;
  while (prev != cur) {
    prev = cur;
    cur = 0;
    std::vector<std::vector<std::pair<int32_t, uint64_t>>> sig(n);
    for (uint32_t p = 0; p < n; p++) {
      for (const Tr &t : l.adj[p]) sig[p].emplace_back(t.label, part[t.process]);
      std::sort(sig[p].begin(), sig[p].end());
      sig[p].erase(std::unique(sig[p].begin(), sig[p].end()), sig[p].end());
    }
    std::map<std::vector<std::pair<int32_t, uint64_t>>, uint64_t> sigmap;
    for (uint32_t p = 0; p < n; p++)
      if (!sigmap.count(sig[p])) sigmap.emplace(sig[p], cur++);
    for (uint32_t p = 0; p < n; p++) part[p] = sigmap[sig[p]];
  }
  count = cur;
  return part;
}

// bisimilar_minimize (lib.rs:413-432)
Lts minimize(const Lts &l, std::vector<uint64_t> &mapping) {
  uint64_t count = 0;
  mapping = signature_refinement(l, count);
  Lts r;
  r.adj.assign(count, {});
  std::vector<uint8_t> represented(count, 0);
  for (uint32_t p = 0; p < l.n(); p++) {
    uint64_t part = mapping[p];
    if (!represented[part]) {
      for (const Tr &t : l.adj[p]) r.adj[part].push_back(Tr{(uint32_t)mapping[t.process], t.label});
      represented[part] = 1;
    }
  }
  r.sort_labels();
  return r;
}

// ---------------------------------------------------------------------------
// GameBuild (src/gamebuild.rs, src/gamebuild/gamepos.rs)
// ---------------------------------------------------------------------------
enum Kind : uint8_t { ATTACK = 0, CLAUSE = 1, DEFEND = 2 };
struct Pos {
  uint8_t kind;
  uint32_t p;
  std::vector<uint32_t> q, qx;  // Clause: q = {q}
  bool operator==(const Pos &o) const { return kind == o.kind && p == o.p && q == o.q && qx == o.qx; }
};
struct PosHash {
  size_t operator()(const Pos &x) const {
    uint64_t h = 1469598103934665603ull ^ x.kind;
    auto mix = [&](uint64_t v) { h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); };
    mix(x.p);
    mix(x.q.size());
    for (uint32_t v : x.q) mix(v);
    mix(x.qx.size());
    for (uint32_t v : x.qx) mix(v);
    return (size_t)h;
  }
};

// TransitionSystem::compare_enabled (gamebuild.rs:23-98)
std::pair<bool, bool> compare_enabled(const Lts &l, uint32_t p, uint32_t q) {
  if (p == q) return {true, true};
  bool subset = true, superset = true;
  const auto &pl = l.adj[p], &ql = l.adj[q];
  size_t pp = 0, qp = 0, pm = pl.size(), qm = ql.size();
  for (;;) {
    if (!(subset || superset)) break;
    if (pp == pm && qp == qm) break;
    if (pp == pm) { subset = false; break; }
    if (qp == qm) { superset = false; break; }
    int32_t pa = pl[pp].label, qa = ql[qp].label;
    bool ap = false, aq = false;
    if (pa == qa) { ap = aq = true; }
    else if (pa < qa) { superset = false; ap = true; }
    else { subset = false; aq = true; }
    if (ap) { pp++; while (pp < pm && pl[pp].label == pa) pp++; }
    if (aq) { qp++; while (qp < qm && ql[qp].label == qa) qp++; }
  }
  return {subset, superset};
}

struct Builder {
  Conf conf{6, 3};  // GameBuild::ENERGY_CONF = STANDARD (gamebuild.rs:152)
  std::vector<Pos> nodes;
  std::unordered_map<Pos, uint32_t, PosHash> node_map;
  uint32_t n_starting = 0;
  std::vector<uint32_t> row, col, wt;
  std::vector<uint8_t> attacker;
  uint32_t upd_obs, upd_chal, upd_rev, upd_ans, upd_cl1, upd_cl2;

  Builder() {
    auto mk = [&](std::initializer_list<int32_t> v) {
      std::vector<int32_t> vv(v);
      uint32_t w = 0;
      pack_update(conf, vv.data(), (uint32_t)vv.size(), &w);
      return w;
    };
    upd_obs = mk({-1});                  // observation_update (gamepos.rs:21)
    upd_chal = mk({0, -1});              // challenge_update (gamepos.rs:22)
    upd_rev = mk({3});                   // revival_update: Min(3) (gamepos.rs:183)
    upd_ans = mk({0, 0, 0, 3});          // answer_update (gamepos.rs:184)
    upd_cl1 = mk({4});                   // Min(4) (gamepos.rs:145)
    upd_cl2 = mk({5, 0, 0, 0, 0, -1});   // Min(5),0,0,0,0,-1 (gamepos.rs:146)
  }

  // new_node (gamebuild.rs:255-265)
  uint32_t new_node(const Pos &pos) {
    uint32_t idx = (uint32_t)nodes.size();
    attacker.push_back(pos.kind != DEFEND);
    nodes.push_back(pos);
    node_map[pos] = idx;
    return idx;
  }

  // AttackPosition::set_transition (gamepos.rs:111-120)
  static std::vector<uint32_t> set_transition(const Lts &l, const std::vector<uint32_t> &Q, int32_t a) {
    std::vector<uint32_t> r;
    for (uint32_t q : Q)
      for (const Tr &t : l.adj[q])
        if (t.label == a) r.push_back(t.process);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    return r;
  }

  // Position::successors (gamepos.rs:244-250 and the three impls)
  void successors(const Lts &l, const Pos &x, std::vector<Pos> &pos, std::vector<uint32_t> &w) {
    pos.clear();
    w.clear();
    if (x.kind == ATTACK) {  // gamepos.rs:17-106
      if (x.q.empty()) {
        pos.push_back(Pos{DEFEND, x.p, {}, {}});
        w.push_back(upd_chal);
        return;
      }
      for (const Tr &t : l.adj[x.p]) {
        std::vector<uint32_t> q2 = set_transition(l, x.q, t.label);
        if (std::find(q2.begin(), q2.end(), t.process) == q2.end())
          pos.push_back(Pos{ATTACK, t.process, std::move(q2), {}});
      }
      w.assign(pos.size(), upd_obs);
      size_t cs = pos.size();
      pos.push_back(Pos{DEFEND, x.p, x.q, {}});
      std::vector<uint32_t> q_sub, qx_sub, q_sup, qx_sup, q_eq, qx_eq;
      for (uint32_t q : x.q) {
        auto se = compare_enabled(l, x.p, q);
        (se.first ? qx_sub : q_sub).push_back(q);
        (se.second ? qx_sup : q_sup).push_back(q);
        ((se.first && se.second) ? qx_eq : q_eq).push_back(q);
      }
      auto contains = [&](const Pos &c) {
        for (size_t i = cs + 1; i < pos.size(); i++)
          if (pos[i] == c) return true;
        return false;
      };
      if (!qx_sub.empty() && !q_sub.empty()) pos.push_back(Pos{DEFEND, x.p, q_sub, qx_sub});
      if (!qx_sup.empty() && !q_sup.empty()) {
        Pos c{DEFEND, x.p, q_sup, qx_sup};
        if (!contains(c)) pos.push_back(c);
      }
      if (!qx_eq.empty() && !q_eq.empty()) {
        Pos c{DEFEND, x.p, q_eq, qx_eq};
        if (!contains(c)) pos.push_back(c);
      }
      for (size_t i = cs; i < pos.size(); i++) w.push_back(upd_chal);
    } else if (x.kind == CLAUSE) {  // gamepos.rs:139-158
      pos.push_back(Pos{ATTACK, x.p, {x.q[0]}, {}});
      pos.push_back(Pos{ATTACK, x.q[0], {x.p}, {}});
      w.push_back(upd_cl1);
      w.push_back(upd_cl2);
    } else {  // DefendPosition::successors (gamepos.rs:179-198)
      for (uint32_t q : x.q) {
        pos.push_back(Pos{CLAUSE, x.p, {q}, {}});
        w.push_back(upd_ans);
      }
      if (!x.qx.empty()) {
        pos.push_back(Pos{ATTACK, x.p, x.qx, {}});
        w.push_back(upd_rev);
      }
    }
  }

  // build_internal (gamebuild.rs:229-239) + add_nodes (:242-252)
  void build(const Lts &l) {
    n_starting = (uint32_t)nodes.size();
    std::vector<Pos> ps;
    std::vector<uint32_t> ws;
    for (size_t idx = 0; idx < nodes.size(); idx++) {
      Pos cur = nodes[idx];
      successors(l, cur, ps, ws);
      row.push_back((uint32_t)col.size());
      for (auto &p : ps) {
        auto it = node_map.find(p);
        uint32_t s = (it != node_map.end()) ? it->second : new_node(p);
        col.push_back(s);
      }
      wt.insert(wt.end(), ws.begin(), ws.end());
    }
    row.push_back((uint32_t)col.size());
  }
};

Graph builder_graph(const Builder &b) {
  Graph g;
  g.conf = b.conf;
  g.n = (uint32_t)b.nodes.size();
  g.row = b.row;
  if (g.row.empty()) g.row.push_back(0);
  g.col = b.col;
  g.wt = b.wt;
  g.attacker = b.attacker;
  g.make_reverse();
  return g;
}

// EnergyGame::standard_reach (energygame.rs:347-352)
std::vector<uint32_t> standard_reach(const Graph &g) {
  std::vector<uint32_t> r;
  for (uint32_t v = 0; v < g.n; v++)
    if (!g.attacker[v] && g.row[v + 1] == g.row[v]) r.push_back(v);
  return r;
}

// TransitionSystem::compare (lib.rs:275-283) -> size of energies[0]
void compare_job(const Lts &l, uint32_t p, uint32_t q, uint64_t &count, uint64_t &nodes) {
  std::vector<uint64_t> mapping;
  Lts red = minimize(l, mapping);
  uint32_t pm = (uint32_t)mapping[p], qm = (uint32_t)mapping[q];
  if (pm == qm) { count = 0; nodes = 0; return; }
  Builder b;
  b.new_node(Pos{ATTACK, pm, {qm}, {}});
  b.build(red);
  Graph g = builder_graph(b);
  std::vector<uint32_t> reach = standard_reach(g);
  std::vector<EList> E(g.n);
  for (uint32_t v : reach) E[v].assign(g.conf.energy_size(), 0);
  Stats st;
  run_game(g, E, reach, st);
  count = E[0].size() / g.conf.energy_size();
  nodes = g.n;
}

template <class F>
void parallel_for(uint32_t n, uint32_t threads, F f) {
  if (threads <= 1 || n <= 1) {
    for (uint32_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; t++)
    pool.emplace_back([&]() {
      for (;;) {
        uint32_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto &th : pool) th.join();
}

// One worklist step of position v against the lists E, as a round of
// run_game applies it (energygame.rs:774-944, attack_update.wgsl:77-113,
// attack_minimize.wgsl:69-122, defend_iterative.wgsl:182-267): true when
// the reference would change v's list.  Defenders whose suprema outgrow the
// preallocated memory are retried with more, as run_game does in a later
// round.
bool step_changes(const Graph &g, const Arith &ar, const std::vector<EList> &E, uint32_t v) {
  const uint32_t es = ar.es, us = ar.us;
  if (g.row[v] == g.row[v + 1]) return false;  // never visited: no successors
  std::vector<uint32_t> upd_tmp(es), cand;
  if (g.attacker[v]) {
    for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++) {
      const EList &ew = E[g.col[k]];
      for (size_t x = 0; x < ew.size(); x += es) {
        ar.inv_update(&ew[x], &g.wt[(size_t)k * us], upd_tmp.data());
        cand.insert(cand.end(), upd_tmp.begin(), upd_tmp.end());
      }
    }
    const size_t own_start = cand.size() / es;
    std::vector<uint32_t> zero(us, 0);
    for (size_t x = 0; x < E[v].size(); x += es) {
      ar.inv_update(&E[v][x], zero.data(), upd_tmp.data());
      cand.insert(cand.end(), upd_tmp.begin(), upd_tmp.end());
    }
    const size_t K = cand.size() / es;
    for (size_t i = 0; i < own_start; i++) {
      bool keep = true;
      for (size_t j = 0; j < K && keep; j++) {
        bool eq = ar.eq(&cand[j * es], &cand[i * es]);
        if (j != i && ((eq && i < j) || (!eq && ar.less_eq(&cand[j * es], &cand[i * es])))) keep = false;
      }
      if (keep) return true;  // a kept candidate from a successor
    }
    return false;
  }
  for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++)
    if (E[g.col[k]].empty()) return false;  // :789-792, not visited
  EList en;
  std::vector<uint32_t> so;
  for (uint32_t k = g.row[v]; k < g.row[v + 1]; k++) {
    const EList &ew = E[g.col[k]];
    so.push_back((uint32_t)(en.size() / es));
    for (size_t x = 0; x < ew.size(); x += es) {
      ar.inv_update(&ew[x], &g.wt[(size_t)k * us], upd_tmp.data());
      en.insert(en.end(), upd_tmp.begin(), upd_tmp.end());
    }
  }
  so.push_back((uint32_t)(en.size() / es));
  EList res;
  uint32_t mem = DEFAULT_SUPREMA_MEMORY;
  for (;;) {
    const int32_t stt = wg_intersection(ar, en.data(), so.data(), (uint32_t)so.size() - 1, mem, res);
    if (stt >= 0) break;
    mem = std::max(next_pow2((uint32_t)(-(int64_t)stt)), 128u);
  }
  return !earray_eq(ar, E[v], res);
}

}  // namespace

struct OraSolution {
  uint32_t esize;
  std::vector<EList> E;
  Stats st;
};
struct OraLts { Lts l; };
struct OraBuild { Builder b; Graph g; };

extern "C" {

uint32_t ora_energy_bits(uint32_t e, uint32_t m) { return Conf{e, m}.energy_bits(); }
uint32_t ora_energy_size(uint32_t e, uint32_t m) { return Conf{e, m}.energy_size(); }
uint32_t ora_energy_mask(uint32_t e, uint32_t m) { return Conf{e, m}.energy_mask(); }
uint32_t ora_update_bits(uint32_t e, uint32_t m) { return Conf{e, m}.update_bits(); }
uint32_t ora_update_size(uint32_t e, uint32_t m) { return Conf{e, m}.update_size(); }
uint32_t ora_update_mask(uint32_t e, uint32_t m) { return Conf{e, m}.update_mask(); }

int ora_pack_energy(uint32_t e, uint32_t m, const uint32_t *vals, uint32_t n, uint32_t *out) {
  return pack_energy(Conf{e, m}, vals, n, out) ? 0 : -1;
}
// From<&Energy> for Vec<u32> (energy.rs:164-179)
void ora_unpack_energy(uint32_t e, uint32_t m, const uint32_t *words, uint32_t *out) {
  Conf c{e, m};
  unpack_fields(words, c.elements, c.energy_bits(), c.energy_mask(), out);
}
int ora_pack_update(uint32_t e, uint32_t m, const int32_t *vals, uint32_t n, uint32_t *out) {
  return pack_update(Conf{e, m}, vals, n, out) ? 0 : -1;
}
// From<&Update> for Vec<Upd> / Vec<i32> (energy.rs:567-602)
void ora_unpack_update(uint32_t e, uint32_t m, const uint32_t *words, int32_t *out) {
  Conf c{e, m};
  std::vector<uint32_t> raw(c.elements);
  unpack_fields(words, c.elements, c.update_bits(), c.update_mask(), raw.data());
  for (uint32_t i = 0; i < c.elements; i++)
    out[i] = raw[i] == 0 ? 0 : (raw[i] == 1 ? -1 : (int32_t)(raw[i] - 1));
}
void ora_inv_update(uint32_t e, uint32_t m, const uint32_t *energy, const uint32_t *update,
                    uint32_t *out) {
  Arith(Conf{e, m}).inv_update(energy, update, out);
}

OraSolution *ora_run_game(uint32_t elements, uint32_t max, uint32_t n, const uint32_t *row_offsets,
                          const uint32_t *col, const uint32_t *weights, const uint8_t *attacker,
                          const uint64_t *init_offsets, const uint32_t *init_data,
                          const uint32_t *to_reach, uint32_t n_reach) {
  Graph g;
  g.conf = Conf{elements, max};
  g.n = n;
  g.row.assign(row_offsets, row_offsets + n + 1);
  uint32_t m = g.row[n];
  g.col.assign(col, col + m);
  g.wt.assign(weights, weights + (size_t)m * g.conf.update_size());
  g.attacker.assign(attacker, attacker + n);
  g.make_reverse();
  auto *s = new OraSolution;
  s->esize = g.conf.energy_size();
  s->E.assign(n, {});
  std::vector<uint32_t> reach(to_reach, to_reach + n_reach);
  if (init_offsets) {
    for (uint32_t v = 0; v < n; v++)
      s->E[v].assign(init_data + init_offsets[v] * s->esize, init_data + init_offsets[v + 1] * s->esize);
  } else {
    for (uint32_t v : reach) s->E[v].assign(s->esize, 0);  // with_reach (:355-365)
  }
  run_game(g, s->E, reach, s->st);
  return s;
}

uint64_t ora_solution_total(const OraSolution *s) {
  uint64_t t = 0;
  for (auto &e : s->E) t += e.size() / s->esize;
  return t;
}
void ora_solution_offsets(const OraSolution *s, uint64_t *out) {
  uint64_t t = 0;
  out[0] = 0;
  for (size_t v = 0; v < s->E.size(); v++) {
    t += s->E[v].size() / s->esize;
    out[v + 1] = t;
  }
}
void ora_solution_data(const OraSolution *s, uint32_t *out) {
  for (auto &e : s->E) {
    std::copy(e.begin(), e.end(), out);
    out += e.size();
  }
}
void ora_solution_stats(const OraSolution *s, uint64_t *out) {
  out[0] = s->st.rounds;
  out[1] = s->st.atk_visits;
  out[2] = s->st.def_visits;
  out[3] = s->st.def_retries;
  out[4] = s->st.edges_relaxed;
  out[5] = s->st.bytes;
}
void ora_solution_free(OraSolution *s) { delete s; }

uint32_t ora_standard_reach(uint32_t n, const uint32_t *row, const uint8_t *attacker, uint32_t *out) {
  uint32_t c = 0;
  for (uint32_t v = 0; v < n; v++)
    if (!attacker[v] && row[v + 1] == row[v]) out[c++] = v;
  return c;
}

int32_t ora_defend_intersection(uint32_t elements, uint32_t max, const uint32_t *energies,
                                const uint32_t *succ_offsets, uint32_t n_succ, uint32_t mem,
                                uint32_t *sup_out) {
  Arith ar(Conf{elements, max});
  EList res;
  int32_t st = wg_intersection(ar, energies, succ_offsets, n_succ, mem, res);
  if (st >= 0) std::copy(res.begin(), res.end(), sup_out);
  return st;
}

OraLts *ora_lts_from_edges(uint64_t m, const uint32_t *src, const uint32_t *dst, const int32_t *label) {
  return new OraLts{lts_from_edges(m, src, dst, label)};
}

// TransitionSystem::from_csv_lines (lib.rs:372-406)
OraLts *ora_lts_from_csv(const char *path, int *err) {
  *err = 0;
  std::ifstream f(path);
  if (!f) { *err = 1; return nullptr; }
  std::vector<std::vector<Tr>> adj;
  std::unordered_map<std::string, int32_t> labels;
  labels["i"] = 0;
  int32_t max_label = 0;
  std::string line;
  auto parse_uint = [](const std::string &s, uint64_t lim, uint64_t &out) {
    size_t i = 0;
    if (i < s.size() && s[i] == '+') i++;
    if (i >= s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); i++) {
      if (s[i] < '0' || s[i] > '9') return false;
      v = v * 10 + (uint64_t)(s[i] - '0');
      if (v > lim) return false;
    }
    out = v;
    return true;
  };
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    size_t c1 = line.find(',');
    if (c1 == std::string::npos) { *err = 2; return nullptr; }
    size_t c2 = line.find(',', c1 + 1);
    if (c2 == std::string::npos) { *err = 2; return nullptr; }
    uint64_t from, to;
    if (!parse_uint(line.substr(0, c1), UINT64_MAX / 10, from) ||
        !parse_uint(line.substr(c1 + 1, c2 - c1 - 1), 0xffffffffull, to)) {
      *err = 3;
      return nullptr;
    }
    std::string label = line.substr(c2 + 1);
    if (label.size() >= 2 && label.front() == '"' && label.back() == '"')
      label = label.substr(1, label.size() - 2);
    int32_t ln;
    auto it = labels.find(label);
    if (it != labels.end()) ln = it->second;
    else { ln = ++max_label; labels[label] = ln; }
    size_t mx = std::max<uint64_t>(from, to);
    if (mx >= adj.size()) adj.resize(mx + 1);
    adj[from].push_back(Tr{(uint32_t)to, ln});
  }
  auto *o = new OraLts;
  o->l.adj = std::move(adj);
  o->l.sort_labels();
  return o;
}

uint32_t ora_lts_n_vertices(const OraLts *l) { return l->l.n(); }
uint64_t ora_lts_n_transitions(const OraLts *l) {
  uint64_t t = 0;
  for (auto &r : l->l.adj) t += r.size();
  return t;
}
void ora_lts_transitions(const OraLts *l, uint64_t *offsets, uint32_t *targets, int32_t *labels) {
  uint64_t t = 0;
  offsets[0] = 0;
  for (size_t p = 0; p < l->l.adj.size(); p++) {
    for (const Tr &x : l->l.adj[p]) {
      targets[t] = x.process;
      labels[t] = x.label;
      t++;
    }
    offsets[p + 1] = t;
  }
}
uint64_t ora_lts_signature_refinement(const OraLts *l, uint64_t *partition) {
  uint64_t count = 0;
  auto part = signature_refinement(l->l, count);
  std::copy(part.begin(), part.end(), partition);
  return count;
}
OraLts *ora_lts_minimize(const OraLts *l, uint64_t *mapping) {
  std::vector<uint64_t> m;
  Lts r = minimize(l->l, m);
  std::copy(m.begin(), m.end(), mapping);
  return new OraLts{std::move(r)};
}
void ora_lts_free(OraLts *l) { delete l; }

// GameBuild::compare (gamebuild.rs:165-170)
OraBuild *ora_build_compare(const OraLts *l, uint32_t p, uint32_t q) {
  auto *o = new OraBuild;
  o->b.new_node(Pos{ATTACK, p, {q}, {}});
  o->b.build(l->l);
  o->g = builder_graph(o->b);
  return o;
}

// GameBuild::compare_all (gamebuild.rs:200-215).  The reference walks the
// enabledness partitions in FxHashMap iteration order; here the partitions
// are visited in order of their first process, so start indices differ from
// the reference's while the set of positions and the game are the same.
OraBuild *ora_build_compare_all(const OraLts *l) {
  auto *o = new OraBuild;
  std::map<std::vector<int32_t>, size_t> idx;
  std::vector<std::vector<uint32_t>> parts;
  for (uint32_t p = 0; p < l->l.n(); p++) {  // enabledness_partitions (:104-117)
    std::vector<int32_t> en;
    for (const Tr &t : l->l.adj[p]) en.push_back(t.label);
    std::sort(en.begin(), en.end());
    en.erase(std::unique(en.begin(), en.end()), en.end());
    auto it = idx.find(en);
    if (it == idx.end()) { idx.emplace(en, parts.size()); parts.push_back({p}); }
    else parts[it->second].push_back(p);
  }
  for (auto &part : parts)
    for (uint32_t p : part)
      for (uint32_t q : part)
        if (p != q) o->b.new_node(Pos{ATTACK, p, {q}, {}});
  o->b.build(l->l);
  o->g = builder_graph(o->b);
  return o;
}
uint32_t ora_build_n_nodes(const OraBuild *b) { return b->g.n; }
uint64_t ora_build_n_edges(const OraBuild *b) { return b->g.col.size(); }
uint32_t ora_build_n_starting(const OraBuild *b) { return b->b.n_starting; }
void ora_build_graph(const OraBuild *b, uint32_t *row, uint32_t *col, uint32_t *wt, uint8_t *att) {
  std::copy(b->g.row.begin(), b->g.row.end(), row);
  std::copy(b->g.col.begin(), b->g.col.end(), col);
  std::copy(b->g.wt.begin(), b->g.wt.end(), wt);
  std::copy(b->g.attacker.begin(), b->g.attacker.end(), att);
}
void ora_build_position(const OraBuild *b, uint32_t idx, uint32_t *kind, uint32_t *p, uint32_t *nq,
                        uint32_t *nqx) {
  const Pos &x = b->b.nodes[idx];
  *kind = x.kind;
  *p = x.p;
  *nq = (uint32_t)x.q.size();
  *nqx = (uint32_t)x.qx.size();
}
void ora_build_position_sets(const OraBuild *b, uint32_t idx, uint32_t *q, uint32_t *qx) {
  const Pos &x = b->b.nodes[idx];
  std::copy(x.q.begin(), x.q.end(), q);
  std::copy(x.qx.begin(), x.qx.end(), qx);
}
void ora_build_free(OraBuild *b) { delete b; }

void ora_compare_batch(uint32_t n_jobs, const OraLts *const *lts, const uint32_t *p, const uint32_t *q,
                       uint32_t n_threads, uint64_t *out_counts, uint64_t *out_nodes) {
  parallel_for(n_jobs, n_threads, [&](uint32_t i) {
    compare_job(lts[i]->l, p[i], q[i], out_counts[i], out_nodes[i]);
  });
}

uint64_t ora_check_fixpoint(uint32_t elements, uint32_t max, uint32_t n, const uint32_t *row_offsets,
                            const uint32_t *col, const uint32_t *weights, const uint8_t *attacker,
                            const uint64_t *offsets, const uint32_t *data, uint32_t n_threads, uint32_t *first_bad) {
  Graph g;
  g.conf = Conf{elements, max};
  g.n = n;
  g.row.assign(row_offsets, row_offsets + n + 1);
  const uint32_t m = g.row[n];
  g.col.assign(col, col + m);
  g.wt.assign(weights, weights + (size_t)m * g.conf.update_size());
  g.attacker.assign(attacker, attacker + n);
  const Arith ar(g.conf);
  const uint32_t es = ar.es;
  std::vector<EList> E(n);
  for (uint32_t v = 0; v < n; v++) E[v].assign(data + offsets[v] * es, data + offsets[v + 1] * es);
  const uint32_t chunks = (n + 4095) / 4096;
  std::vector<uint64_t> bad(chunks, 0);
  std::vector<uint32_t> first(chunks, 0xFFFFFFFFu);
  parallel_for(chunks, n_threads, [&](uint32_t c) {
    const uint32_t b = c * 4096, e = std::min(n, b + 4096);
    for (uint32_t v = b; v < e; v++)
      if (step_changes(g, ar, E, v)) {
        if (!bad[c]) first[c] = v;
        bad[c]++;
      }
  });
  uint64_t total = 0;
  uint32_t f = 0xFFFFFFFFu;
  for (uint32_t c = 0; c < chunks; c++) {
    total += bad[c];
    if (bad[c] && f == 0xFFFFFFFFu) f = first[c];
  }
  if (first_bad) *first_bad = f;
  return total;
}

void ora_run_games_parallel(uint32_t n_games, uint32_t elements, uint32_t max, const uint32_t *n_pos,
                            const uint32_t *const *row_offsets, const uint32_t *const *col,
                            const uint32_t *const *weights, const uint8_t *const *attacker,
                            uint32_t n_threads, uint64_t *out_total) {
  ora_solve_games(n_games, elements, max, n_pos, row_offsets, col, weights, attacker, n_threads, nullptr,
                  out_total, nullptr);
}

void ora_solve_games(uint32_t n_games, uint32_t elements, uint32_t max, const uint32_t *n_pos,
                     const uint32_t *const *row_offsets, const uint32_t *const *col,
                     const uint32_t *const *weights, const uint8_t *const *attacker, uint32_t n_threads,
                     const uint32_t *order, uint64_t *out_total, OraSolution **out_sol) {
  // one shared work counter over the whole set: a thread takes the next game
  // (in `order` when given) as soon as it is free
  parallel_for(n_games, n_threads, [&](uint32_t k) {
    const uint32_t i = order ? order[k] : k;
    Graph g;
    g.conf = Conf{elements, max};
    g.n = n_pos[i];
    g.row.assign(row_offsets[i], row_offsets[i] + g.n + 1);
    uint32_t m = g.row[g.n];
    g.col.assign(col[i], col[i] + m);
    g.wt.assign(weights[i], weights[i] + (size_t)m * g.conf.update_size());
    g.attacker.assign(attacker[i], attacker[i] + g.n);
    g.make_reverse();
    std::vector<uint32_t> reach = standard_reach(g);
    std::vector<EList> E(g.n);
    for (uint32_t v : reach) E[v].assign(g.conf.energy_size(), 0);
    Stats st;
    run_game(g, E, reach, st);
    uint64_t t = 0;
    for (auto &e : E) t += e.size() / g.conf.energy_size();
    if (out_total) out_total[i] = t;
    if (out_sol) {
      auto *s = new OraSolution;
      s->esize = g.conf.energy_size();
      s->E = std::move(E);
      s->st = st;
      out_sol[i] = s;
    }
  });
}

uint64_t ora_b_min(uint32_t n, const uint32_t *row_offsets, const uint32_t *col, const uint64_t *offsets) {
  const uint64_t m = row_offsets[n];
  std::vector<uint64_t> indeg(n, 0);
  for (uint64_t k = 0; k < m; k++) indeg[col[k]]++;
  uint64_t b = 4ull * (n + 1) + 8ull * m + n;
  for (uint32_t v = 0; v < n; v++) b += 4ull * (offsets[v + 1] - offsets[v]) * (1ull + indeg[v]);
  return b;
}

}  // extern "C"
