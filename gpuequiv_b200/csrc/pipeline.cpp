// pipeline.cpp - the whole algorithm: minimise, build, solve, interpret
// (TransitionSystem::compare / equivalences, src/lib.rs:275-343, and
// Equivalence, src/equivalence.rs).
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>
#include <unordered_map>

#include "gamebuild.h"
#include "geq_internal.h"
#include "lts.h"

struct geq_equivalence {
  uint32_t n_processes = 0;        // processes of the LTS the game was built on
  bool minimized = false;
  std::vector<uint64_t> mapping;   // original process -> class (when minimized)
  std::vector<std::pair<uint32_t, uint32_t>> starts;
  std::vector<uint64_t> offsets;   // per start position
  std::vector<uint32_t> data;
  std::unordered_map<uint64_t, uint32_t> pos_to_idx;
};

namespace geq {
namespace {

geq_status engine_of(geq_context *ctx, Engine *&e) {
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  e = ctx->engine.get();
  return GEQ_OK;
}

// EnergyArray::test_equivalence (energy.rs:307-318) for STANDARD energies.
bool holds(const uint32_t *e, uint64_t n, uint32_t eq) {
  for (uint64_t k = 0; k < n; k++) {
    bool le = true;
    for (int i = 0; i < 6 && le; i++)
      if (((e[k] >> (2 * i)) & 3u) > ((eq >> (2 * i)) & 3u)) le = false;
    if (le) return false;
  }
  return true;
}

struct UnionFind {
  std::vector<uint32_t> parent;
  explicit UnionFind(size_t n) : parent(n) { std::iota(parent.begin(), parent.end(), 0u); }
  uint32_t find(uint32_t x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  }
  void unite(uint32_t a, uint32_t b) {
    a = find(a);
    b = find(b);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
};

}  // namespace
}  // namespace geq

using namespace geq;

extern "C" {

geq_status geq_compare_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts, const uint32_t *p,
                             const uint32_t *q, int minimize, geq_solution **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  Engine *e;
  geq_status st = engine_of(ctx, e);
  if (st) return st;
  if (n_jobs && (!lts || !p || !q)) return fail(GEQ_ERR_INVALID_INPUT, "NULL job arrays");
  for (uint32_t i = 0; i < n_jobs; i++) {
    if (!lts[i]) return fail(GEQ_ERR_INVALID_INPUT, "job %u: LTS is NULL", i);
    if (p[i] >= lts[i]->l.n || q[i] >= lts[i]->l.n) return fail(GEQ_ERR_INVALID_INPUT, "job %u: process out of range", i);
  }
  // everything on the device: the LTSs staged once, minimised (signature
  // refinement), the bisimilar short cut decided, the games built and solved
  std::vector<const Lts *> L(n_jobs);
  std::vector<uint32_t> start_off(n_jobs + 1);
  for (uint32_t i = 0; i < n_jobs; i++) L[i] = &lts[i]->l;
  for (uint32_t i = 0; i <= n_jobs; i++) start_off[i] = i;
  std::vector<uint8_t> trivial(n_jobs, 0);
  std::unique_ptr<geq_solution> sol(new geq_solution());
  geq_solution part;
  if (n_jobs) {
    GamesPtr dg;
    if ((st = build_and_upload(*e, ctx->device, n_jobs, L.data(), start_off.data(), p, q, 0, dg, nullptr,
                               minimize ? &trivial : nullptr)))
      return st;
    if (dg) {
      if ((st = e->solve(*dg, &sol->stats))) return st;
      const uint32_t n_games = (uint32_t)(std::count(trivial.begin(), trivial.end(), 0));
      std::vector<uint32_t> first(n_games, 0), count(n_games, 1);
      if ((st = e->download_selected(*dg, first, count, part))) return st;
    }
  }
  // assemble: one game of one position per job
  sol->energy_size = 1;
  sol->n_vertices.assign(n_jobs, 1);
  sol->offsets_base.resize(n_jobs);
  sol->data_base.resize(n_jobs);
  sol->offsets.resize(2 * (size_t)n_jobs);
  size_t k = 0;
  for (uint32_t i = 0; i < n_jobs; i++) {
    sol->offsets_base[i] = 2 * (size_t)i;
    sol->offsets[2 * i] = 0;
    if (trivial[i]) {
      sol->offsets[2 * i + 1] = 0;
      sol->data_base[i] = sol->data.size();
      continue;
    }
    const uint64_t cnt = part.offsets[part.offsets_base[k] + 1];
    sol->offsets[2 * i + 1] = cnt;
    sol->data_base[i] = sol->data.size();
    sol->data.insert(sol->data.end(), part.data.begin() + part.data_base[k],
                     part.data.begin() + part.data_base[k] + cnt);
    k++;
  }
  *out = sol.release();
  return GEQ_OK;
}

geq_status geq_compare(geq_context *ctx, const geq_lts *l, uint32_t p, uint32_t q, int minimize, geq_solution **out) {
  const geq_lts *ls[1] = {l};
  return geq_compare_batch(ctx, 1, ls, &p, &q, minimize, out);
}

geq_status geq_equivalences(geq_context *ctx, const geq_lts *l, int minimize, geq_equivalence **out) {
  if (!out || !l) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  *out = nullptr;
  Engine *e;
  geq_status st = engine_of(ctx, e);
  if (st) return st;
  std::unique_ptr<geq_equivalence> eq(new geq_equivalence());
  Lts red;
  const Lts *base = &l->l;
  if (minimize) {
    l->l.minimize(eq->mapping, red);
    base = &red;
    eq->minimized = true;
  }
  eq->n_processes = base->n;
  // GameBuild::compare_all (gamebuild.rs:200-215): the start pairs on the
  // host, the game built on the device
  std::vector<uint32_t> all(base->n);
  for (uint32_t i = 0; i < base->n; i++) all[i] = i;
  GameBuilder::start_pairs(*base, all.data(), base->n, eq->starts);
  const uint32_t n_starting = (uint32_t)eq->starts.size();
  if (n_starting) {
    std::vector<uint32_t> sp(n_starting), sq(n_starting), start_off{0, n_starting};
    for (uint32_t i = 0; i < n_starting; i++) {
      sp[i] = eq->starts[i].first;
      sq[i] = eq->starts[i].second;
    }
    const Lts *L[1] = {base};
    GamesPtr dg;
    if ((st = build_and_upload(*e, ctx->device, 1, L, start_off.data(), sp.data(), sq.data(), 0, dg, nullptr)))
      return st;
    if ((st = e->solve(*dg, nullptr))) return st;
    geq_solution part;
    std::vector<uint32_t> first{0}, count{n_starting};
    if ((st = e->download_selected(*dg, first, count, part))) return st;
    eq->offsets.assign(part.offsets.begin(), part.offsets.end());
    eq->data = std::move(part.data);
  } else {
    eq->offsets.assign(1, 0);
  }
  for (uint32_t i = 0; i < eq->starts.size(); i++)
    eq->pos_to_idx.emplace(((uint64_t)eq->starts[i].first << 32) | eq->starts[i].second, i);
  *out = eq.release();
  return GEQ_OK;
}

static uint32_t mapped(const geq_equivalence *e, uint32_t p) {
  return e->minimized ? (uint32_t)e->mapping[p] : p;
}

static bool energies_min(const geq_equivalence *e, uint32_t p, uint32_t q, const uint32_t *&d, uint64_t &n) {
  auto it = e->pos_to_idx.find(((uint64_t)p << 32) | q);
  if (it == e->pos_to_idx.end()) return false;
  d = e->data.data() + e->offsets[it->second];
  n = e->offsets[it->second + 1] - e->offsets[it->second];
  return true;
}

int geq_equivalence_energies(const geq_equivalence *e, uint32_t p, uint32_t q, const uint32_t **data, uint64_t *n) {
  if (!e) return 0;
  uint32_t n_orig = e->minimized ? (uint32_t)e->mapping.size() : e->n_processes;
  if (p >= n_orig || q >= n_orig) return 0;
  const uint32_t *d;
  uint64_t c;
  if (!energies_min(e, mapped(e, p), mapped(e, q), d, c)) return 0;
  if (data) *data = d;
  if (n) *n = c;
  return 1;
}

// Equivalence::preorder (equivalence.rs:125-132)
int geq_equivalence_preorder(const geq_equivalence *e, uint32_t p, uint32_t q, const uint32_t *equivalence) {
  if (!e || !equivalence) return 0;
  uint32_t n_orig = e->minimized ? (uint32_t)e->mapping.size() : e->n_processes;
  if (p >= n_orig || q >= n_orig) return 0;
  p = mapped(e, p);
  q = mapped(e, q);
  if (p == q) return 1;
  const uint32_t *d;
  uint64_t c;
  if (!energies_min(e, p, q, d, c)) return 0;
  return holds(d, c, equivalence[0]) ? 1 : 0;
}

// Equivalence::equiv (equivalence.rs:142-144)
int geq_equivalence_equiv(const geq_equivalence *e, uint32_t p, uint32_t q, const uint32_t *equivalence) {
  return geq_equivalence_preorder(e, p, q, equivalence) && geq_equivalence_preorder(e, q, p, equivalence);
}

// Equivalence::relation + EquivalenceRelation::with_mapping
// (equivalence.rs:154-170, :234-246).
geq_status geq_equivalence_relation(const geq_equivalence *e, const uint32_t *equivalence, uint32_t *classes,
                                    uint32_t *n_classes) {
  if (!e || !equivalence || !n_classes) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  UnionFind uf(e->n_processes);
  for (size_t i = 0; i < e->starts.size(); i++) {
    const uint32_t p = e->starts[i].first, q = e->starts[i].second;
    const uint32_t *d2;
    uint64_t c2;
    if (!energies_min(e, q, p, d2, c2))
      return fail(GEQ_ERR_INTERNAL, "symmetric position not included in starting points");
    const uint32_t *d = e->data.data() + e->offsets[i];
    const uint64_t c = e->offsets[i + 1] - e->offsets[i];
    if (holds(d, c, equivalence[0]) && holds(d2, c2, equivalence[0])) uf.unite(p, q);
  }
  const size_t n_orig = e->minimized ? e->mapping.size() : e->n_processes;
  std::vector<uint32_t> cls(n_orig);
  std::unordered_map<uint32_t, uint32_t> rep;  // class root -> smallest process
  for (size_t proc = 0; proc < n_orig; proc++) {
    uint32_t root = uf.find(e->minimized ? (uint32_t)e->mapping[proc] : (uint32_t)proc);
    auto it = rep.find(root);
    if (it == rep.end()) {
      rep.emplace(root, (uint32_t)proc);
      cls[proc] = (uint32_t)proc;
    } else {
      cls[proc] = it->second;
    }
  }
  if (classes) std::copy(cls.begin(), cls.end(), classes);
  *n_classes = (uint32_t)rep.size();
  return GEQ_OK;
}

uint32_t geq_equivalence_n_processes(const geq_equivalence *e) {
  if (!e) return 0;
  return e->minimized ? (uint32_t)e->mapping.size() : e->n_processes;
}
uint32_t geq_equivalence_n_starting_points(const geq_equivalence *e) { return e ? (uint32_t)e->starts.size() : 0; }
void geq_equivalence_free(geq_equivalence *e) { delete e; }

}  // extern "C"
