// server.cpp - the serving loop: queued single-game requests solved in
// batches by pipeline threads, each owning an Engine (stream, staging,
// device pool, CUDA graphs).  While one pipeline solves its batch on the
// device, another stages and uploads the next, so the device always has a
// batch in flight (continuous batching over alternating pipelines).
//
// A request is one game with standard initialisation, as EnergyGame::run
// after EnergyGame::standard_reach (energygame.rs:347-352, :379-383), or one
// TransitionSystem::compare query (lib.rs:275-283) that is minimised, built
// and solved on the device with the other queries of its batch.  Inside a
// batch every game keeps its own positions and frontier, so each result is
// the result of solving that game or query alone.

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include <cuda_runtime.h>

#include "geq_internal.h"
#include "lts.h"

namespace geq {
namespace {

// Estimated device bytes of a batch: per position the CSR row, flags,
// descriptors (3 x 8 B), reverse row, frontier slots and lists, arena words;
// per edge successor, update and reverse entry; doubled for the pool's
// power-of-two blocks, plus the fixed minimum arena.
constexpr uint64_t BATCH_BASE_BYTES = 32ull << 20;
uint64_t game_footprint(uint64_t n, uint64_t m) { return 2 * (70 * n + 12 * m) + 4096; }
// A compare query's game is not known before it is built: estimated at 16
// positions and 64 edges per state and transition of its LTS, plus the
// builder's and the minimisation's per-state and per-transition arrays.
uint64_t compare_footprint(uint64_t n, uint64_t m) {
  return game_footprint(16 * (n + m) + 64, 64 * (n + m) + 256) + 64 * (n + m);
}

struct Request {
  uint64_t ticket = 0;
  int kind = 0;  // 0: a game (geq_server_submit), 1: a compare query (geq_server_submit_compare)
  Lts lts;
  uint32_t p = 0, q = 0;
  geq_energy_conf conf{};
  uint32_t n = 0;
  std::vector<uint32_t> row, col, wt, reach;
  std::vector<uint8_t> att;
  uint64_t footprint = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  geq_status st = GEQ_OK;
  std::string err;
  std::unique_ptr<geq_solution> sol;
};

}  // namespace
}  // namespace geq

using namespace geq;

struct geq_server {
  int device = 0;
  geq_server_config cfg{};
  uint64_t budget = 0;  // per pipeline
  std::vector<std::unique_ptr<Engine>> engines;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  geq_server_stats stats{};
};

namespace {

// One game of a batch solution as a solution of its own.
std::unique_ptr<geq_solution> split_one(const geq_solution &all, uint32_t g) {
  std::unique_ptr<geq_solution> s(new geq_solution());
  const uint32_t n = all.n_vertices[g];
  const uint64_t *o = all.off_ptr() + all.offsets_base[g];
  const uint64_t words = o[n];
  s->energy_size = all.energy_size;
  s->n_vertices.assign(1, n);
  s->offsets_base.assign(1, 0);
  s->data_base.assign(1, 0);
  s->offsets.assign(o, o + n + 1);
  const uint32_t *d = all.data_ptr() + all.data_base[g] * all.energy_size;
  s->data.assign(d, d + words * all.energy_size);
  s->stats = all.stats;
  return s;
}

// Compare queries of a batch: minimised, built and solved together on the
// device (the path of geq_compare_batch); each request gets the energies of
// its start position.  On failure of several, each is retried alone.
void run_compares(Engine &e, int device, std::vector<Request *> &batch) {
  const uint32_t n = (uint32_t)batch.size();
  std::vector<const Lts *> L(n);
  std::vector<uint32_t> p(n), q(n), start_off(n + 1);
  for (uint32_t i = 0; i < n; i++) {
    L[i] = &batch[i]->lts;
    p[i] = batch[i]->p;
    q[i] = batch[i]->q;
  }
  for (uint32_t i = 0; i <= n; i++) start_off[i] = i;
  std::vector<uint8_t> trivial;
  GamesPtr dg;
  geq_solution part;
  geq_status st = build_and_upload(e, device, n, L.data(), start_off.data(), p.data(), q.data(), 0, dg, nullptr,
                                   &trivial);
  if (!st && dg) st = e.solve(*dg, &part.stats);
  if (!st && dg) {
    const uint32_t games = (uint32_t)std::count(trivial.begin(), trivial.end(), 0);
    std::vector<uint32_t> first(games, 0), count(games, 1);
    st = e.download_selected(*dg, first, count, part);
  }
  dg.reset();
  if (st) {
    if (n > 1) {
      for (Request *r : batch) {
        std::vector<Request *> one{r};
        run_compares(e, device, one);
      }
      return;
    }
    batch[0]->st = st;
    batch[0]->err = geq_last_error();
    return;
  }
  uint32_t k = 0;
  for (uint32_t i = 0; i < n; i++) {
    std::unique_ptr<geq_solution> sol(new geq_solution());
    sol->energy_size = 1;
    sol->n_vertices.assign(1, 1);
    sol->offsets_base.assign(1, 0);
    sol->data_base.assign(1, 0);
    sol->stats = part.stats;
    if (trivial[i]) {
      sol->offsets = {0, 0};  // bisimilar: lib.rs:279-281
    } else {
      const uint64_t cnt = part.offsets[part.offsets_base[k] + 1];
      sol->offsets = {0, cnt};
      sol->data.assign(part.data.begin() + part.data_base[k], part.data.begin() + part.data_base[k] + cnt);
      k++;
    }
    batch[i]->sol = std::move(sol);
  }
}

// Upload, solve and download one batch on engine `e`; on failure of a batch
// of several games each game is retried alone so that only the faulty one
// fails.
void run_batch(Engine &e, std::vector<Request *> &batch) {
  std::vector<GameInput> in(batch.size());
  for (size_t i = 0; i < batch.size(); i++) {
    Request &r = *batch[i];
    GameInput &gi = in[i];
    gi.g.conf = r.conf;
    gi.g.n_vertices = r.n;
    gi.g.row_offsets = r.row.data();
    gi.g.column_indices = r.col.data();
    gi.g.weights = r.wt.data();
    gi.g.attacker_pos = r.att.data();
    gi.to_reach = r.reach.data();
    gi.n_reach = (uint32_t)r.reach.size();
  }
  if (batch.size() == 1) {
    // a lone small game: one launch of the one-block solver
    std::unique_ptr<geq_solution> one(new geq_solution());
    bool handled = false;
    const geq_status st = e.solve_small(in[0], *one, handled);
    if (st) {
      batch[0]->st = st;
      batch[0]->err = geq_last_error();
      return;
    }
    if (handled) {
      batch[0]->sol = std::move(one);
      return;
    }
  }
  GamesPtr dg;
  geq_solution sol;
  geq_status st = e.upload(in, dg);
  if (!st) st = e.solve(*dg, &sol.stats);
  if (!st) st = e.download(*dg, sol);
  dg.reset();
  if (st) {
    if (batch.size() > 1) {
      for (Request *r : batch) {
        std::vector<Request *> one{r};
        run_batch(e, one);
      }
      return;
    }
    batch[0]->st = st;
    batch[0]->err = geq_last_error();
    return;
  }
  parallel_for((uint32_t)batch.size(), [&](uint32_t i) { batch[i]->sol = split_one(sol, i); },
               batch.size() >= 256 ? 0u : 1u);
}

void pipeline(geq_server *s, Engine *e) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Request *> batch;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->stop) break;
      // batching window: a few hundred microseconds for more requests
      if (s->queue.size() < s->cfg.max_batch_games)
        s->cv_work.wait_for(lk, std::chrono::microseconds(s->cfg.max_wait_us),
                            [&] { return s->stop || s->queue.size() >= s->cfg.max_batch_games; });
      if (s->stop) break;
      uint64_t fp = BATCH_BASE_BYTES;
      while (!s->queue.empty() && batch.size() < s->cfg.max_batch_games) {
        Request *r = s->queue.front();
        if (!batch.empty() && fp + r->footprint > s->budget) break;
        fp += r->footprint;
        s->queue.pop_front();
        r->state = 1;
        batch.push_back(r);
      }
      if (batch.empty()) continue;
      s->stats.batches++;
      s->stats.games_in_batches += batch.size();
      s->stats.running += batch.size();
      s->stats.queued = s->queue.size();
      if (fp > s->stats.max_batch_footprint) s->stats.max_batch_footprint = fp;
    }
    {
      std::vector<Request *> games, compares;
      for (Request *r : batch) (r->kind ? compares : games).push_back(r);
      if (!games.empty()) run_batch(*e, games);
      if (!compares.empty()) run_compares(*e, s->device, compares);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (Request *r : batch) {
        r->state = 2;
        if (r->st) s->stats.failed++;
        else s->stats.completed++;
      }
      s->stats.running -= batch.size();
    }
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

geq_status geq_server_create(geq_context *ctx, const geq_server_config *cfg, geq_server **out) {
  if (!out) return fail(GEQ_ERR_INVALID_INPUT, "out is NULL");
  *out = nullptr;
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  std::unique_ptr<geq_server> s(new geq_server());
  s->device = ctx->device;
  if (cfg) s->cfg = *cfg;
  if (!s->cfg.n_pipelines) s->cfg.n_pipelines = 2;
  if (s->cfg.n_pipelines > 8) return fail(GEQ_ERR_INVALID_INPUT, "at most 8 pipelines");
  if (!s->cfg.max_batch_games) s->cfg.max_batch_games = 4096;
  if (!s->cfg.max_wait_us) s->cfg.max_wait_us = 200;
  if (!s->cfg.hbm_budget_bytes) s->cfg.hbm_budget_bytes = 150ull * 1000 * 1000 * 1000;
  if (!s->cfg.max_queued) s->cfg.max_queued = 1000000;
  s->budget = s->cfg.hbm_budget_bytes / s->cfg.n_pipelines;
  for (uint32_t i = 0; i < s->cfg.n_pipelines; i++) {
    std::unique_ptr<Engine> e;
    geq_status st = Engine::create(ctx->device, e);
    if (st) return st;
    e->tuning = ctx->engine->tuning;
    s->engines.push_back(std::move(e));
  }
  for (auto &e : s->engines) s->threads.emplace_back(pipeline, s.get(), e.get());
  *out = s.release();
  return GEQ_OK;
}

geq_status geq_server_submit(geq_server *s, const geq_game_graph *graph, uint64_t *ticket) {
  if (!s || !graph || !ticket) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  geq_status st = validate_graph(*graph);
  if (st) return st;
  if (!Conf(graph->conf).supported())
    return fail(GEQ_ERR_UNSUPPORTED, "EnergyConf {%u, %u} is outside the device codecs", graph->conf.elements,
                graph->conf.max);
  const uint64_t n = graph->n_vertices, m = graph->row_offsets[n];
  std::unique_ptr<Request> r(new Request());
  r->conf = graph->conf;
  r->n = graph->n_vertices;
  r->row.assign(graph->row_offsets, graph->row_offsets + n + 1);
  r->col.assign(graph->column_indices, graph->column_indices + m);
  r->wt.assign(graph->weights, graph->weights + m);
  r->att.assign(graph->attacker_pos, graph->attacker_pos + n);
  for (auto &a : r->att) a = a ? 1 : 0;
  r->reach = standard_reach_of(*graph);
  r->footprint = game_footprint(n, m);
  if (BATCH_BASE_BYTES + r->footprint > s->budget)
    return fail(GEQ_ERR_OUT_OF_MEMORY, "game of %llu positions needs ~%llu device bytes, a pipeline may use %llu",
                (unsigned long long)n, (unsigned long long)(BATCH_BASE_BYTES + r->footprint),
                (unsigned long long)s->budget);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(GEQ_ERR_BUSY, "server is shutting down");
    if (s->queue.size() >= s->cfg.max_queued) return fail(GEQ_ERR_BUSY, "%llu requests queued",
                                                          (unsigned long long)s->queue.size());
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->queue.push_back(r.get());
    s->reqs.emplace(r->ticket, std::move(r));
    s->stats.submitted++;
    s->stats.queued = s->queue.size();
  }
  s->cv_work.notify_one();
  return GEQ_OK;
}

geq_status geq_server_submit_compare(geq_server *s, const geq_lts *lts, uint32_t p, uint32_t q, uint64_t *ticket) {
  if (!s || !lts || !ticket) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (p >= lts->l.n || q >= lts->l.n) return fail(GEQ_ERR_INVALID_INPUT, "process out of range");
  std::unique_ptr<Request> r(new Request());
  r->kind = 1;
  r->lts = lts->l;
  r->p = p;
  r->q = q;
  r->footprint = compare_footprint(lts->l.n, lts->l.n_transitions());
  if (BATCH_BASE_BYTES + r->footprint > s->budget)
    return fail(GEQ_ERR_OUT_OF_MEMORY, "query of %u processes needs ~%llu device bytes, a pipeline may use %llu",
                lts->l.n, (unsigned long long)(BATCH_BASE_BYTES + r->footprint), (unsigned long long)s->budget);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(GEQ_ERR_BUSY, "server is shutting down");
    if (s->queue.size() >= s->cfg.max_queued) return fail(GEQ_ERR_BUSY, "%llu requests queued",
                                                          (unsigned long long)s->queue.size());
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->queue.push_back(r.get());
    s->reqs.emplace(r->ticket, std::move(r));
    s->stats.submitted++;
    s->stats.queued = s->queue.size();
  }
  s->cv_work.notify_one();
  return GEQ_OK;
}

geq_status geq_server_poll(geq_server *s, uint64_t ticket, int32_t timeout_ms, geq_solution **out) {
  if (!s || !out) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  *out = nullptr;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(GEQ_ERR_INVALID_INPUT, "unknown ticket %llu", (unsigned long long)ticket);
  Request *r = it->second.get();
  auto done = [&] { return r->state == 2; };
  if (timeout_ms < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
    return fail(GEQ_ERR_TIMEOUT, "request %llu not finished", (unsigned long long)ticket);
  const geq_status st = r->st;
  if (st) set_last_error(r->err);
  else *out = r->sol.release();
  s->reqs.erase(it);
  return st;
}

void geq_server_get_stats(geq_server *s, geq_server_stats *out) {
  if (!s || !out) return;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
}

void geq_server_destroy(geq_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Request *r : s->queue) {
      r->state = 2;
      r->st = GEQ_ERR_BUSY;
      r->err = "server destroyed before the request ran";
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto &t : s->threads) t.join();
  s->engines.clear();
  delete s;
}

}  // extern "C"
