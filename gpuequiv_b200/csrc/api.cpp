// api.cpp - the extern "C" boundary of libgeq.so (declared in include/geq.h).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <unordered_map>

#include "gamebuild.h"
#include "geq_internal.h"
#include "lts.h"

namespace geq {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

geq_status fail(geq_status st, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

// TryFrom<SerdeGameGraph> (energygame.rs:65-83): CSR shape, successor ids,
// and update codes that name an element (pack_upd rejects others, energy.rs:551-556).
geq_status validate_graph(const geq_game_graph &g, bool check_rows) {
  Conf c(g.conf);
  if (c.elements == 0) return fail(GEQ_ERR_INVALID_INPUT, "EnergyConf with zero elements");
  if (!g.row_offsets) return fail(GEQ_ERR_INVALID_INPUT, "row_offsets is NULL");
  if (g.row_offsets[0] != 0) return fail(GEQ_ERR_INVALID_INPUT, "row_offsets[0] must be 0");
  for (uint32_t v = 0; check_rows && v < g.n_vertices; v++)
    if (g.row_offsets[v + 1] < g.row_offsets[v]) return fail(GEQ_ERR_INVALID_INPUT, "row_offsets not monotone at %u", v);
  const uint64_t m = g.row_offsets[g.n_vertices];
  if (m && (!g.column_indices || !g.weights)) return fail(GEQ_ERR_INVALID_INPUT, "edges without column_indices/weights");
  if (g.n_vertices && !g.attacker_pos) return fail(GEQ_ERR_INVALID_INPUT, "attacker_pos is NULL");
  // Successor ids and update codes are checked on the device during the
  // upload (k_fix_cols, k_check_weights), which reports GEQ_ERR_INVALID_INPUT.
  return GEQ_OK;
}

geq_status validate_lists(const geq_game_graph &g, const geq_energy_lists *l) {
  if (!l) return GEQ_OK;
  Conf c(g.conf);
  if (l->n_vertices != g.n_vertices) return fail(GEQ_ERR_INVALID_INPUT, "energies cover %u positions, graph has %u", l->n_vertices, g.n_vertices);
  if (l->energy_size != c.energy_size()) return fail(GEQ_ERR_INVALID_INPUT, "energy_size %u does not match the conf (%u)", l->energy_size, c.energy_size());
  if (!l->offsets || l->offsets[0] != 0) return fail(GEQ_ERR_INVALID_INPUT, "energy offsets must start at 0");
  for (uint32_t v = 0; v < l->n_vertices; v++) {
    if (l->offsets[v + 1] < l->offsets[v]) return fail(GEQ_ERR_INVALID_INPUT, "energy offsets not monotone");
    if (l->offsets[v + 1] - l->offsets[v] > 0xFFFFFFull) return fail(GEQ_ERR_INVALID_INPUT, "energy list too long");
  }
  if (l->offsets[l->n_vertices] && !l->data) return fail(GEQ_ERR_INVALID_INPUT, "energy data is NULL");
  if (c.energy_bits() * c.elements < 32) {
    const uint32_t pad = ~0u << (c.energy_bits() * c.elements);
    for (uint64_t i = 0; i < l->offsets[l->n_vertices]; i++)
      if (l->data[i] & pad) return fail(GEQ_ERR_INVALID_INPUT, "energy padding bits set");
  }
  return GEQ_OK;
}

std::vector<uint32_t> standard_reach_of(const geq_game_graph &g) {
  std::vector<uint32_t> r;
  for (uint32_t v = 0; v < g.n_vertices; v++)
    if (!g.attacker_pos[v] && g.row_offsets[v + 1] == g.row_offsets[v]) r.push_back(v);
  return r;
}

// Batches of at least this many positions run as two pipelined halves.
static constexpr unsigned long long SPLIT_MIN_POSITIONS = 1ull << 21;

static geq_status ctx_engine(geq_context *ctx, Engine *&e) {
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  e = ctx->engine.get();
  return GEQ_OK;
}

static geq_status make_inputs(uint32_t n_games, const geq_game_graph *graphs, const geq_energy_lists *const *initial,
                              const uint32_t *const *to_reach, const uint32_t *n_to_reach,
                              std::vector<GameInput> &in) {
  if (n_games == 0 || !graphs) return fail(GEQ_ERR_INVALID_INPUT, "no games");
  in.resize(n_games);
  // large batches: row monotonicity and the standard reach are left to the
  // device (k_check_rows, k_std_reach), which reads every row anyway
  const bool on_device = n_games >= 64 && !initial;
  auto one = [&](uint32_t g) -> geq_status {
    GameInput &gi = in[g];
    gi.g = graphs[g];
    gi.rows_unchecked = on_device;
    geq_status st = validate_graph(gi.g, !on_device);
    if (st) return st;
    if (!(Conf(gi.g.conf) == Conf(graphs[0].conf))) return fail(GEQ_ERR_INVALID_INPUT, "games of one batch need one EnergyConf");
    gi.init = initial ? initial[g] : nullptr;
    if ((st = validate_lists(gi.g, gi.init))) return st;
    if (to_reach && to_reach[g]) {
      gi.to_reach = to_reach[g];
      gi.n_reach = n_to_reach ? n_to_reach[g] : 0;
      for (uint32_t i = 0; i < gi.n_reach; i++)
        if (gi.to_reach[i] >= gi.g.n_vertices) return fail(GEQ_ERR_INVALID_INPUT, "to_reach index out of range");
    } else if (to_reach && !to_reach[g] && n_to_reach && n_to_reach[g]) {
      return fail(GEQ_ERR_INVALID_INPUT, "to_reach is NULL with a non-zero count");
    } else if (!to_reach && on_device) {
      gi.std_reach = true;
    } else if (!to_reach) {
      gi.reach_storage = standard_reach_of(gi.g);
      gi.to_reach = gi.reach_storage.data();
      gi.n_reach = (uint32_t)gi.reach_storage.size();
    }
    return GEQ_OK;
  };
  if (n_games < 64) {
    for (uint32_t g = 0; g < n_games; g++) {
      const geq_status st = one(g);
      if (st) return st;
    }
  } else {
    // large batches: games checked on all host cores; the first failing game
    // (in batch order) decides the status and message
    std::vector<geq_status> sts(n_games, GEQ_OK);
    std::vector<std::string> msgs(n_games);
    parallel_for(n_games, [&](uint32_t g) {
      sts[g] = one(g);
      if (sts[g]) msgs[g] = geq_last_error();
    });
    for (uint32_t g = 0; g < n_games; g++)
      if (sts[g]) {
        set_last_error(msgs[g]);
        return sts[g];
      }
  }
  return GEQ_OK;
}

// The solver path of a batch's conf: true for the multi-word solver.
static geq_status wide_path(const Engine &e, const geq_energy_conf &c, bool &wide) {
  const Conf conf(c);
  wide = !conf.supported() || (e.tuning.flags & GEQ_TUNE_FORCE_WIDE);
  std::string why;
  if (wide && !wide_supported(conf, &why)) return fail(GEQ_ERR_UNSUPPORTED, "%s", why.c_str());
  return GEQ_OK;
}

}  // namespace geq

using namespace geq;

extern "C" {

const char *geq_status_string(geq_status s) {
  switch (s) {
    case GEQ_OK: return "ok";
    case GEQ_ERR_NO_DEVICE: return "no CUDA device";
    case GEQ_ERR_OUT_OF_MEMORY: return "out of memory";
    case GEQ_ERR_INVALID_INPUT: return "invalid input";
    case GEQ_ERR_TIMEOUT: return "timeout";
    case GEQ_ERR_UNSUPPORTED: return "unsupported energy configuration";
    case GEQ_ERR_CUDA: return "CUDA error";
    case GEQ_ERR_IO: return "I/O error";
    case GEQ_ERR_PARSE: return "parse error";
    case GEQ_ERR_BUSY: return "busy";
    case GEQ_ERR_INTERNAL: return "internal error";
  }
  return "unknown";
}
const char *geq_last_error(void) { return g_last_error.c_str(); }
int geq_abi_version(void) { return GEQ_ABI_VERSION; }

uint32_t geq_conf_energy_bits(geq_energy_conf c) { return Conf(c).energy_bits(); }
uint32_t geq_conf_energy_size(geq_energy_conf c) { return Conf(c).energy_size(); }
uint32_t geq_conf_energy_mask(geq_energy_conf c) { return Conf(c).energy_mask(); }
uint32_t geq_conf_update_bits(geq_energy_conf c) { return Conf(c).update_bits(); }
uint32_t geq_conf_update_size(geq_energy_conf c) { return Conf(c).update_size(); }
uint32_t geq_conf_update_mask(geq_energy_conf c) { return Conf(c).update_mask(); }
int geq_conf_supported(geq_energy_conf c) { return Conf(c).supported() ? 1 : 0; }
int geq_conf_solvable(geq_energy_conf c) { return Conf(c).supported() || wide_supported(Conf(c)) ? 1 : 0; }

// pack_energy (energy.rs:143-162)
geq_status geq_energy_pack(geq_energy_conf cc, const uint32_t *values, uint32_t n, uint32_t *out) {
  Conf c(cc);
  if (n > c.elements) return fail(GEQ_ERR_INVALID_INPUT, "%u values for %u elements", n, c.elements);
  const uint32_t es = c.energy_size(), bits = c.energy_bits();
  for (uint32_t i = 0; i < es; i++) out[i] = 0;
  uint32_t shift = 0, word = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (values[i] > c.max) return fail(GEQ_ERR_INVALID_INPUT, "value %u exceeds max %u", values[i], c.max);
    out[word] |= values[i] << shift;
    shift += bits;
    if (shift + bits > 32) { shift = 0; word++; }
  }
  return GEQ_OK;
}

// From<&Energy> for Vec<u32> (energy.rs:164-179)
void geq_energy_unpack(geq_energy_conf cc, const uint32_t *words, uint32_t *out) {
  Conf c(cc);
  uint32_t shift = 0, word = 0, bits = c.energy_bits(), mask = c.energy_mask();
  for (uint32_t i = 0; i < c.elements; i++) {
    out[i] = (words[word] >> shift) & mask;
    shift += bits;
    if (shift >= 32) { shift = 0; word++; }
  }
}

// Upd::from(i32) + pack_upd (energy.rs:474-490, :543-565)
geq_status geq_update_pack(geq_energy_conf cc, const int32_t *values, uint32_t n, uint32_t *out) {
  Conf c(cc);
  if (n > c.elements) return fail(GEQ_ERR_INVALID_INPUT, "%u updates for %u elements", n, c.elements);
  const uint32_t us = c.update_size(), bits = c.update_bits();
  for (uint32_t i = 0; i < us; i++) out[i] = 0;
  uint32_t shift = 0, word = 0;
  for (uint32_t i = 0; i < n; i++) {
    int32_t v = values[i];
    uint32_t repr;
    if (v == 0) repr = 0;
    else if (v == -1) repr = 1;
    else if (v < -1) return fail(GEQ_ERR_INVALID_INPUT, "invalid update entry %d", v);
    else if ((uint32_t)v > c.elements) return fail(GEQ_ERR_INVALID_INPUT, "Min(%d) names no element", v);
    else repr = (uint32_t)v + 1;
    out[word] |= repr << shift;
    shift += bits;
    if (shift + bits > 32) { shift = 0; word++; }
  }
  return GEQ_OK;
}

// From<&Update> for Vec<i32> (energy.rs:567-602)
void geq_update_unpack(geq_energy_conf cc, const uint32_t *words, int32_t *out) {
  Conf c(cc);
  uint32_t shift = 0, word = 0, bits = c.update_bits(), mask = c.update_mask();
  for (uint32_t i = 0; i < c.elements; i++) {
    uint32_t raw = (words[word] >> shift) & mask;
    out[i] = raw == 0 ? 0 : (raw == 1 ? -1 : (int32_t)(raw - 1));
    shift += bits;
    if (shift >= 32) { shift = 0; word++; }
  }
}

// EnergyArray::test_equivalence (energy.rs:307-318)
int geq_test_equivalence(geq_energy_conf cc, const uint32_t *energies, uint64_t n, const uint32_t *eq) {
  Conf c(cc);
  const uint32_t es = c.energy_size(), bits = c.energy_bits(), mask = c.energy_mask();
  for (uint64_t k = 0; k < n; k++) {
    const uint32_t *e = energies + k * es;
    bool le = true;
    uint32_t shift = 0, word = 0;
    for (uint32_t i = 0; i < c.elements && le; i++) {
      if (((e[word] >> shift) & mask) > ((eq[word] >> shift) & mask)) le = false;
      shift += bits;
      if (shift >= 32) { shift = 0; word++; }
    }
    if (le) return 0;
  }
  return 1;
}

uint32_t geq_standard_reach(const geq_game_graph *g, uint32_t *out) {
  uint32_t c = 0;
  for (uint32_t v = 0; v < g->n_vertices; v++)
    if (!g->attacker_pos[v] && g->row_offsets[v + 1] == g->row_offsets[v]) out[c++] = v;
  return c;
}

geq_status geq_context_create(int device, geq_context **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  std::unique_ptr<Engine> e;
  geq_status st = Engine::create(device, e);
  if (st) return st;
  geq_context *ctx = new (std::nothrow) geq_context();
  if (!ctx) return fail(GEQ_ERR_OUT_OF_MEMORY, "context");
  ctx->device = device;
  ctx->engine = std::move(e);
  *out = ctx;
  return GEQ_OK;
}

void geq_context_destroy(geq_context *ctx) { delete ctx; }

geq_status geq_context_info(const geq_context *ctx, char *name, size_t name_len, int *n_sms, uint64_t *total_mem) {
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  if (name && name_len) {
    std::strncpy(name, ctx->engine->name.c_str(), name_len - 1);
    name[name_len - 1] = 0;
  }
  if (n_sms) *n_sms = ctx->engine->n_sms;
  if (total_mem) *total_mem = ctx->engine->total_mem;
  return GEQ_OK;
}

geq_status geq_context_set_tuning(geq_context *ctx, const geq_tuning *t) {
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  if (!t) return fail(GEQ_ERR_INVALID_INPUT, "tuning is NULL");
  if (t->blocks_per_sm) e->tuning.blocks_per_sm = std::min<uint32_t>(std::max<uint32_t>(t->blocks_per_sm, 2), 5);
  if (t->rounds_per_graph) e->tuning.rounds_per_graph = std::min<uint32_t>(t->rounds_per_graph, 256);
  if (t->small_limit) e->tuning.small_limit = std::min<uint32_t>(t->small_limit, 32);
  if (t->lane_limits) e->tuning.lane_limits = t->lane_limits;
  e->tuning.flags = t->flags;
  return GEQ_OK;
}

void geq_context_get_tuning(const geq_context *ctx, geq_tuning *t) {
  if (ctx && ctx->engine && t) *t = ctx->engine->tuning;
}

uint32_t geq_solution_n_games(const geq_solution *s) { return s ? (uint32_t)s->n_vertices.size() : 0; }

geq_status geq_solution_lists(const geq_solution *s, uint32_t game, geq_energy_lists *out) {
  if (!s || !out || game >= s->n_vertices.size()) return fail(GEQ_ERR_INVALID_INPUT, "no such game");
  out->n_vertices = s->n_vertices[game];
  out->energy_size = s->energy_size;
  out->offsets = s->off_ptr() + s->offsets_base[game];
  out->data = s->data_ptr() + s->data_base[game] * s->energy_size;
  return GEQ_OK;
}

geq_status geq_solution_flat(const geq_solution *s, const uint64_t **offsets, uint64_t *n_offsets,
                             const uint32_t **data, uint64_t *n_words) {
  if (!s || !offsets || !n_offsets || !data || !n_words) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  // the flat layout holds when each game's offsets and words follow the previous game's
  uint64_t ob = 0, db = 0;
  for (size_t g = 0; g < s->n_vertices.size(); g++) {
    if (s->offsets_base[g] != ob || s->data_base[g] != db)
      return fail(GEQ_ERR_UNSUPPORTED, "solution is not laid out flat");
    db += s->off_ptr()[ob + s->n_vertices[g]];
    ob += (uint64_t)s->n_vertices[g] + 1;
  }
  *offsets = s->off_ptr();
  *n_offsets = s->offsets_len();
  *data = s->data_ptr();
  *n_words = s->data_len();
  return GEQ_OK;
}

void geq_solution_stats(const geq_solution *s, geq_solve_stats *out) {
  if (s && out) *out = s->stats;
}
void geq_solution_free(geq_solution *s) { delete s; }

geq_status geq_device_games_create(geq_context *ctx, uint32_t n_games, const geq_game_graph *graphs,
                                   const geq_energy_lists *const *initial, const uint32_t *const *to_reach,
                                   const uint32_t *n_to_reach, geq_device_games **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  std::vector<GameInput> in;
  if ((st = make_inputs(n_games, graphs, initial, to_reach, n_to_reach, in))) return st;
  if (!Conf(graphs[0].conf).supported())
    return fail(GEQ_ERR_UNSUPPORTED,
                "device-resident games need a conf of the thermometer codecs (EnergyConf {%u, %u} is solved by "
                "geq_energy_game_run / geq_energy_game_run_batch)", graphs[0].conf.elements, graphs[0].conf.max);
  std::unique_ptr<geq_device_games> dg(new geq_device_games());
  if ((st = e->upload(in, dg->impl))) return st;
  *out = dg.release();
  return GEQ_OK;
}

geq_status geq_device_games_solve(geq_context *ctx, geq_device_games *dg, geq_solve_stats *stats) {
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  if (!dg || !dg->impl) return fail(GEQ_ERR_INVALID_INPUT, "device games is NULL");
  return e->solve(*dg->impl, stats);
}

geq_status geq_device_games_download(geq_context *ctx, geq_device_games *dg, geq_solution **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  if (!dg || !dg->impl) return fail(GEQ_ERR_INVALID_INPUT, "device games is NULL");
  std::unique_ptr<geq_solution> sol(new geq_solution());
  if ((st = e->download(*dg->impl, *sol))) return st;
  *out = sol.release();
  return GEQ_OK;
}

void geq_device_games_free(geq_device_games *dg) {
  if (!dg) return;
  delete dg;  // DeviceGamesImpl releases its device memory
}

geq_status geq_energy_game_run_batch(geq_context *ctx, uint32_t n_games, const geq_game_graph *graphs,
                                     const geq_energy_lists *const *initial, const uint32_t *const *to_reach,
                                     const uint32_t *n_to_reach, geq_solution **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  std::vector<GameInput> in;
  if ((st = make_inputs(n_games, graphs, initial, to_reach, n_to_reach, in))) return st;
  bool wide = false;
  if ((st = wide_path(*e, graphs[0].conf, wide))) return st;
  if (wide) {
    std::unique_ptr<geq_solution> sol(new geq_solution());
    if ((st = solve_wide(*e, ctx->device, in, *sol))) return st;
    *out = sol.release();
    return GEQ_OK;
  }
  if (n_games == 1) {
    // a small single game: one launch of the one-block solver
    std::unique_ptr<geq_solution> sol(new geq_solution());
    bool handled = false;
    if ((st = e->solve_small(in[0], *sol, handled))) return st;
    if (handled) {
      *out = sol.release();
      return GEQ_OK;
    }
  }
  unsigned long long positions = 0;
  for (auto &gi : in) positions += gi.g.n_vertices;
  if (n_games >= 2 && positions >= SPLIT_MIN_POSITIONS &&
      !(e->tuning.flags & (GEQ_TUNE_NO_SPLIT | GEQ_TUNE_PROFILE))) {
    // two halves on two engines: the second half's upload overlaps the
    // first half's rounds
    if (!ctx->engine2) {
      std::unique_ptr<Engine> e2;
      if ((st = Engine::create(ctx->device, e2))) return st;
      ctx->engine2 = std::move(e2);
    }
    ctx->engine2->tuning = e->tuning;
    std::unique_ptr<geq_solution> sol(new geq_solution());
    if ((st = run_batch_pipelined(ctx->device, *e, *ctx->engine2, in, *sol))) return st;
    *out = sol.release();
    return GEQ_OK;
  }
  GamesPtr dg;
  if ((st = e->upload(in, dg))) return st;
  std::unique_ptr<geq_solution> sol(new geq_solution());
  st = e->solve(*dg, &sol->stats);
  if (!st) st = e->download(*dg, *sol);
  if (st) return st;
  *out = sol.release();
  return GEQ_OK;
}

geq_status geq_energy_game_run(geq_context *ctx, const geq_game_graph *graph, const geq_energy_lists *initial,
                               const uint32_t *to_reach, uint32_t n_to_reach, geq_solution **out) {
  if (!graph) return fail(GEQ_ERR_INVALID_INPUT, "graph is NULL");
  if (!to_reach && n_to_reach) return fail(GEQ_ERR_INVALID_INPUT, "to_reach is NULL with a non-zero count");
  // an explicit (possibly empty) to_reach list, as in EnergyGame { to_reach, .. }
  const geq_energy_lists *const init[1] = {initial};
  const uint32_t *const reach[1] = {to_reach};
  uint32_t nr[1] = {n_to_reach};
  return geq_energy_game_run_batch(ctx, 1, graph, initial ? init : nullptr, reach, nr, out);
}

geq_status geq_energy_game_run_static(geq_context *ctx, const geq_game_graph *graph, const uint32_t *to_reach,
                                      uint32_t n_to_reach, uint64_t *offsets, uint32_t *data,
                                      uint64_t data_cap, uint64_t *n_words, geq_solve_stats *stats) {
  Engine *e;
  geq_status st = ctx_engine(ctx, e);
  if (st) return st;
  if (!graph || !offsets || !n_words) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (data_cap && !data) return fail(GEQ_ERR_INVALID_INPUT, "data is NULL with a non-zero data_cap");
  if ((st = validate_graph(*graph))) return st;
  if (!to_reach && n_to_reach) return fail(GEQ_ERR_INVALID_INPUT, "to_reach is NULL with a non-zero count");
  for (uint32_t i = 0; to_reach && i < n_to_reach; i++)
    if (to_reach[i] >= graph->n_vertices) return fail(GEQ_ERR_INVALID_INPUT, "to_reach index out of range");
  return e->run_static(ctx->device, *graph, to_reach, n_to_reach, offsets, data, data_cap, n_words, stats);
}

// ---- TransitionSystem -------------------------------------------------------
geq_status geq_lts_from_edges(uint64_t n_edges, const uint32_t *src, const uint32_t *dst, const int32_t *label,
                              geq_lts **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  if (n_edges && (!src || !dst || !label)) return fail(GEQ_ERR_INVALID_INPUT, "edge arrays are NULL");
  std::unique_ptr<geq_lts> l(new geq_lts());
  geq_status st = Lts::from_edges(n_edges, src, dst, label, l->l);
  if (st) return st;
  *out = l.release();
  return GEQ_OK;
}

geq_status geq_lts_from_adjacency(uint32_t n_vertices, uint64_t n_edges, const uint32_t *src, const uint32_t *dst,
                                  const int32_t *label, geq_lts **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  if (n_edges && (!src || !dst || !label)) return fail(GEQ_ERR_INVALID_INPUT, "edge arrays are NULL");
  for (uint64_t i = 0; i < n_edges; i++)
    if (src[i] >= n_vertices || dst[i] >= n_vertices) return fail(GEQ_ERR_INVALID_INPUT, "Node index too high");
  std::unique_ptr<geq_lts> l(new geq_lts());
  geq_status st = Lts::from_edges(n_edges, src, dst, label, l->l, n_vertices);
  if (st) return st;
  *out = l.release();
  return GEQ_OK;
}

geq_status geq_lts_from_csv_file(const char *path, geq_lts **out) {
  if (!out || !path) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  *out = nullptr;
  std::unique_ptr<geq_lts> l(new geq_lts());
  geq_status st = Lts::from_csv_file(path, l->l);
  if (st) return st;
  *out = l.release();
  return GEQ_OK;
}

uint32_t geq_lts_n_vertices(const geq_lts *l) { return l ? l->l.n : 0; }
uint64_t geq_lts_n_transitions(const geq_lts *l) { return l ? l->l.n_transitions() : 0; }
void geq_lts_transitions(const geq_lts *l, uint64_t *offsets, uint32_t *targets, int32_t *labels) {
  std::copy(l->l.off.begin(), l->l.off.end(), offsets);
  std::copy(l->l.tgt.begin(), l->l.tgt.end(), targets);
  std::copy(l->l.lab_.begin(), l->l.lab_.end(), labels);
}

geq_status geq_lts_signature_refinement(const geq_lts *l, uint64_t *partition, uint64_t *n_classes) {
  if (!l || !partition || !n_classes) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  std::vector<uint64_t> part;
  *n_classes = l->l.signature_refinement(part);
  std::copy(part.begin(), part.end(), partition);
  return GEQ_OK;
}

geq_status geq_lts_bisimilar_minimize(const geq_lts *l, geq_lts **reduced, uint64_t *mapping) {
  if (!l || !reduced) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  std::unique_ptr<geq_lts> r(new geq_lts());
  std::vector<uint64_t> m;
  l->l.minimize(m, r->l);
  if (mapping) std::copy(m.begin(), m.end(), mapping);
  *reduced = r.release();
  return GEQ_OK;
}

void geq_lts_free(geq_lts *l) { delete l; }

// ---- GameBuild ----------------------------------------------------------------
geq_status geq_game_build_compare(const geq_lts *l, uint32_t p, uint32_t q, geq_game_build **out) {
  if (!l || !out) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (p >= l->l.n || q >= l->l.n) return fail(GEQ_ERR_INVALID_INPUT, "process out of range");
  std::unique_ptr<geq_game_build> b(new geq_game_build());
  GameBuilder::compare(l->l, p, q, b->b);
  *out = b.release();
  return GEQ_OK;
}

geq_status geq_game_build_compare_bounded(const geq_lts *l, uint32_t p, uint32_t q, uint64_t max_positions,
                                          geq_game_build **out) {
  if (!l || !out) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  *out = nullptr;
  if (p >= l->l.n || q >= l->l.n) return fail(GEQ_ERR_INVALID_INPUT, "process out of range");
  std::unique_ptr<geq_game_build> b(new geq_game_build());
  b->b.max_positions = max_positions;
  GameBuilder::compare(l->l, p, q, b->b);
  if (b->b.truncated) return fail(GEQ_ERR_OUT_OF_MEMORY, "game exceeds %llu positions", (unsigned long long)max_positions);
  *out = b.release();
  return GEQ_OK;
}

geq_status geq_game_build_compare_all(const geq_lts *l, geq_game_build **out) {
  if (!l || !out) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  std::unique_ptr<geq_game_build> b(new geq_game_build());
  GameBuilder::compare_all(l->l, b->b);
  *out = b.release();
  return GEQ_OK;
}

geq_status geq_game_build_compare_multiple(const geq_lts *l, const uint32_t *procs, uint32_t n, geq_game_build **out) {
  if (!l || !out || (n && !procs)) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  for (uint32_t i = 0; i < n; i++)
    if (procs[i] >= l->l.n) return fail(GEQ_ERR_INVALID_INPUT, "process out of range");
  std::unique_ptr<geq_game_build> b(new geq_game_build());
  GameBuilder::compare_processes(l->l, procs, n, b->b);
  *out = b.release();
  return GEQ_OK;
}

void geq_game_build_graph(const geq_game_build *b, geq_game_graph *out) {
  out->conf = geq_energy_conf{6, 3};
  out->n_vertices = (uint32_t)b->b.nodes.size();
  out->row_offsets = b->b.row.data();
  out->column_indices = b->b.col.data();
  out->weights = b->b.wt.data();
  out->attacker_pos = b->b.attacker.data();
}

uint32_t geq_game_build_n_starting_points(const geq_game_build *b) { return b ? b->b.n_starting : 0; }

geq_status geq_game_build_position(const geq_game_build *b, uint32_t idx, geq_position *out) {
  if (!b || !out || idx >= b->b.nodes.size()) return fail(GEQ_ERR_INVALID_INPUT, "no such position");
  const PosKey &k = b->b.nodes[idx];
  out->kind = k.kind;
  out->p = k.p;
  if (k.kind == POS_CLAUSE) {
    out->q = &k.a;
    out->n_q = 1;
    out->qx = nullptr;
    out->n_qx = 0;
  } else {
    out->q = b->b.sets.ptr(k.a);
    out->n_q = b->b.sets.size(k.a);
    out->qx = b->b.sets.ptr(k.b);
    out->n_qx = b->b.sets.size(k.b);
  }
  return GEQ_OK;
}

void geq_game_build_free(geq_game_build *b) { delete b; }

}  // extern "C"
