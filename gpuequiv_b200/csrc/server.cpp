// server.cpp - the serving loop: queued single-game requests solved in
// batches by pipeline threads, each owning an Engine (stream, staging,
// device pool, CUDA graphs).  A pipeline keeps up to MAX_SESSIONS admitted
// batches resident and runs one step (a CUDA graph of worklist rounds) of
// each in turn: requests that arrive while batches are on the device are
// admitted at the next step boundary, as device memory (the admission budget)
// allows, and every game is answered as soon as its own part of the frontier
// is empty, not when its batch ends.  Several pipelines do this on their own
// streams, so one stages and uploads while another's rounds run.
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
// resident batches per pipeline (more arrivals wait and are batched together)
constexpr size_t MAX_SESSIONS = 4;
// equivalence queries per batch: a batch's device GameBuild runs as many
// levels as its deepest game, which every query of the batch waits for
constexpr size_t MAX_COMPARE_BATCH = 128;
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
  // a game's copy: row | col | wt | attacker bytes | reach in one page-locked
  // block from the server's pool (back to the pool when the request is
  // answered); the pipeline copies it to the device as it is
  HostBuf blk;
  const uint32_t *row = nullptr, *col = nullptr, *wt = nullptr, *reach = nullptr;
  const uint8_t *att = nullptr;
  uint32_t n_reach = 0;
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
  std::deque<uint64_t> done_q;  // tickets in the order their requests finished
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  geq_server_stats stats{};
  // page-locked input blocks, reused: a fresh heap block of a few hundred KB
  // costs page faults on every request (and unmapping it a TLB flush on
  // every thread), and a pageable block would be copied once more to reach
  // the device
  std::shared_ptr<HostPool> inpool;
};

namespace {

constexpr size_t INPOOL_IDLE_BYTES = (size_t)4 << 30;  // idle page-locked input blocks kept

// A request's input block from the server's page-locked pool (heap memory
// when none can be had); a new block is allocated with the server's device
// current, so the caller's current device is left as it was.
bool take_block(geq_server *s, Request &r, size_t words) {
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != s->device) cudaSetDevice(s->device);
  const bool ok = r.blk.alloc(s->inpool, words * 4);
  if (dev != s->device && dev >= 0) cudaSetDevice(dev);
  cudaGetLastError();
  return ok;
}

// One game of a batch solution as a solution of its own that views the
// batch's lists (no copy; the batch lives until its last view is freed).
std::unique_ptr<geq_solution> view_one(const std::shared_ptr<const geq_solution> &all, uint32_t g) {
  std::unique_ptr<geq_solution> s(new geq_solution());
  const uint32_t n = all->n_vertices[g], es = all->energy_size;
  s->energy_size = es;
  s->n_vertices.assign(1, n);
  s->offsets_base.assign(1, 0);
  s->data_base.assign(1, 0);
  s->view_off = all->off_ptr() + all->offsets_base[g];
  s->view_noff = (uint64_t)n + 1;
  s->view_data = all->data_ptr() + all->data_base[g] * es;
  s->view_nwords = s->view_off[n] * es;
  s->shared = all;
  s->stats = all->stats;
  return s;
}


// Games of confs without a thermometer codec: the multi-word solver, one
// request at a time.
void run_wide(Engine &e, int device, std::vector<Request *> &batch) {
  for (Request *r : batch) {
    std::vector<GameInput> in(1);
    GameInput &gi = in[0];
    gi.g.conf = r->conf;
    gi.g.n_vertices = r->n;
    gi.g.row_offsets = r->row;
    gi.g.column_indices = r->col;
    gi.g.weights = r->wt;
    gi.g.attacker_pos = r->att;
    gi.to_reach = r->reach;
    gi.n_reach = r->n_reach;
    std::unique_ptr<geq_solution> sol(new geq_solution());
    const geq_status st = solve_wide(e, device, in, *sol);
    if (st) {
      r->st = st;
      r->err = geq_last_error();
    } else {
      r->sol = std::move(sol);
    }
  }
}

// ---- sessions: uploaded batches that are solved a step at a time ------------
// A pipeline keeps every batch it has admitted resident as a session and runs
// one step (one CUDA graph of worklist rounds) of each session in turn, so a
// batch admitted while others are on the device starts at the next step
// boundary instead of after them.  After every step the games whose part of
// the frontier is empty have reached their fixpoint (games share no edges):
// their lists are read back and their requests answered at once.
struct Session {
  GamesPtr dg;
  std::vector<Request *> req;    // game g -> its request (null: nobody waits for it)
  std::vector<uint8_t> retired;  // per game
  bool first_only = false;       // compare queries: only the start position's energies
  uint64_t footprint = 0;
  uint32_t live = 0;             // games not retired
};

void finish(geq_server *s, const std::vector<Request *> &done) {
  if (done.empty()) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (Request *r : done) {
      r->state = 2;
      s->done_q.push_back(r->ticket);
      if (r->st) s->stats.failed++;
      else s->stats.completed++;
    }
    s->stats.running -= done.size();
  }
  s->cv_done.notify_all();
}

void fail_req(Request *r, geq_status st, const std::string &msg, std::vector<Request *> &done) {
  r->st = st;
  r->err = msg;
  done.push_back(r);
}

// Read back and answer the listed games of a session.
geq_status retire(Engine &e, Session &ss, const std::vector<uint32_t> &games, std::vector<Request *> &done) {
  std::vector<uint32_t> want;
  for (uint32_t g : games)
    if (ss.req[g]) want.push_back(g);
  geq_solve_stats stt{};
  geq_status st = e.solve_stats(*ss.dg, &stt);
  std::shared_ptr<geq_solution> part = std::make_shared<geq_solution>();
  if (!st && !want.empty()) st = e.download_games(*ss.dg, want, ss.first_only, *part);
  for (uint32_t g : games) {
    ss.retired[g] = 1;
    ss.live--;
  }
  if (st) {
    const std::string msg = geq_last_error();
    for (uint32_t g : want) fail_req(ss.req[g], st, msg, done);
    return st;
  }
  part->stats = stt;
  const std::shared_ptr<const geq_solution> all = part;
  for (uint32_t i = 0; i < want.size(); i++) {
    Request *r = ss.req[want[i]];
    r->sol = view_one(all, i);
    done.push_back(r);
  }
  return GEQ_OK;
}

// Games of one conf with a thermometer codec: a lone small game in one
// launch of the one-block solver, else an upload that becomes a session.  An
// upload of several games that fails is retried game by game, so that a
// malformed game fails alone.
void start_games(Engine &e, std::vector<Request *> &batch, uint64_t footprint,
                 std::vector<std::unique_ptr<Session>> &out, std::vector<Request *> &done) {
  std::vector<GameInput> in(batch.size());
  for (size_t i = 0; i < batch.size(); i++) {
    Request &r = *batch[i];
    GameInput &gi = in[i];
    gi.g.conf = r.conf;
    gi.g.n_vertices = r.n;
    gi.g.row_offsets = r.row;
    gi.g.column_indices = r.col;
    gi.g.weights = r.wt;
    gi.g.attacker_pos = r.att;
    gi.to_reach = r.reach;
    gi.n_reach = r.n_reach;
    gi.block = (const uint32_t *)r.blk.p;  // one word per update (a device codec conf)
    gi.block_words = packed_game_words(r.n, r.row[r.n], r.n_reach);
  }
  if (batch.size() == 1) {
    std::unique_ptr<geq_solution> one(new geq_solution());
    bool handled = false;
    const geq_status st = e.solve_small(in[0], *one, handled);
    if (st) return fail_req(batch[0], st, geq_last_error(), done);
    if (handled) {
      batch[0]->sol = std::move(one);
      done.push_back(batch[0]);
      return;
    }
  }
  std::unique_ptr<Session> ss(new Session());
  geq_status st = e.upload(in, ss->dg);
  if (!st) st = e.solve_begin(*ss->dg);
  if (st) {
    if (batch.size() > 1) {
      for (Request *r : batch) {
        std::vector<Request *> one{r};
        start_games(e, one, r->footprint, out, done);
      }
      return;
    }
    return fail_req(batch[0], st, geq_last_error(), done);
  }
  ss->req.assign(batch.begin(), batch.end());
  ss->retired.assign(batch.size(), 0);
  ss->live = (uint32_t)batch.size();
  ss->footprint = footprint;
  out.push_back(std::move(ss));
}

// Compare queries: minimised and built together on the device (the path of
// geq_compare_batch), then a session whose games answer with their start
// position.  Bisimilar pairs are answered at once with no energies
// (lib.rs:279-281); a query whose game exceeds the position bound fails
// alone.  If the build of several fails, each query is tried alone.
void start_compares(Engine &e, int device, uint64_t max_positions, std::vector<Request *> &batch, uint64_t footprint,
                    std::vector<std::unique_ptr<Session>> &out, std::vector<Request *> &done) {
  const uint32_t n = (uint32_t)batch.size();
  std::vector<const Lts *> L(n);
  std::vector<uint32_t> p(n), q(n), start_off(n + 1);
  for (uint32_t i = 0; i < n; i++) {
    L[i] = &batch[i]->lts;
    p[i] = batch[i]->p;
    q[i] = batch[i]->q;
  }
  for (uint32_t i = 0; i <= n; i++) start_off[i] = i;
  std::vector<uint8_t> trivial, over;
  std::unique_ptr<Session> ss(new Session());
  geq_status st = build_and_upload(e, device, n, L.data(), start_off.data(), p.data(), q.data(), max_positions, ss->dg,
                                   nullptr, &trivial, &over);
  if (!st && ss->dg) {
    // the games cut at the position bound are never solved
    std::vector<uint32_t> skip;
    for (uint32_t i = 0, k = 0; i < n; i++)
      if (!trivial[i]) {
        if (over[i]) skip.push_back(k);
        k++;
      }
    if (!skip.empty()) e.skip_games(*ss->dg, skip);
    st = e.solve_begin(*ss->dg);
  }
  if (st) {
    if (n > 1) {
      for (Request *r : batch) {
        std::vector<Request *> one{r};
        start_compares(e, device, max_positions, one, r->footprint, out, done);
      }
      return;
    }
    return fail_req(batch[0], st, geq_last_error(), done);
  }
  for (uint32_t i = 0; i < n; i++) {
    Request *r = batch[i];
    if (trivial[i]) {
      std::unique_ptr<geq_solution> sol(new geq_solution());
      sol->energy_size = 1;
      sol->n_vertices.assign(1, 1);
      sol->offsets_base.assign(1, 0);
      sol->data_base.assign(1, 0);
      sol->offsets = {0, 0};  // bisimilar: no game, no energies
      r->sol = std::move(sol);
      done.push_back(r);
    } else {
      // its game is in the upload (cut at the bound when over[i]): game k
      if (over[i]) fail_req(r, GEQ_ERR_OUT_OF_MEMORY, "game exceeds " + std::to_string(max_positions) + " positions",
                            done);
      ss->req.push_back(over[i] ? nullptr : r);
    }
  }
  if (!ss->dg) return;
  ss->retired.assign(ss->req.size(), 0);
  ss->live = (uint32_t)ss->req.size();
  ss->first_only = true;
  ss->footprint = footprint;
  out.push_back(std::move(ss));
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// The second half of a session's step (its graph of rounds was enqueued and
// the stream synchronised): the games that reached their fixpoint retire.
// false: the session is finished (or failed) and can be dropped.
bool finish_session(Engine &e, Session &ss, geq_status enq, std::vector<Request *> &done, double &retire_ms) {
  bool fin = false;
  const uint8_t *active = nullptr;
  geq_status st = enq ? enq : e.step_finish(*ss.dg, fin, active);
  std::vector<uint32_t> ret;
  if (!st && (fin || active))
    for (uint32_t g = 0; g < ss.retired.size(); g++)
      if (!ss.retired[g] && (fin || !active[g])) ret.push_back(g);
  if (st) {
    const std::string msg = geq_last_error();
    for (uint32_t g = 0; g < ss.retired.size(); g++)
      if (!ss.retired[g]) {
        ss.retired[g] = 1;
        if (ss.req[g]) fail_req(ss.req[g], st, msg, done);
      }
    ss.live = 0;
    return false;
  }
  if (!ret.empty()) {
    const auto t0 = std::chrono::steady_clock::now();
    retire(e, ss, ret, done);
    retire_ms += ms_since(t0);
  }
  return ss.live > 0;
}

// One step of every resident session, in two halves: enqueue_steps puts all
// their graphs back to back on the pipeline's stream; finish_steps
// synchronises once and retires, for the first n sessions (sessions admitted
// in between are appended behind them and step from the next turn).
std::vector<geq_status> enqueue_steps(Engine &e, std::vector<std::unique_ptr<Session>> &active) {
  std::vector<geq_status> enq(active.size(), GEQ_OK);
  for (size_t k = 0; k < active.size(); k++) enq[k] = e.step_enqueue(*active[k]->dg, true);
  return enq;
}
void finish_steps(Engine &e, std::vector<std::unique_ptr<Session>> &active, size_t n,
                  const std::vector<geq_status> &enq, uint64_t &used, std::vector<Request *> &done,
                  double &retire_ms) {
  if (!n) return;
  const geq_status sy = e.sync();
  for (size_t k = 0, j = 0; j < n; j++) {
    if (finish_session(e, *active[k], sy ? sy : enq[j], done, retire_ms)) {
      k++;
    } else {
      used -= std::min(used, active[k]->footprint);
      active.erase(active.begin() + k);
    }
  }
}

void pipeline(geq_server *s, Engine *e) {
  cudaSetDevice(s->device);
  std::vector<std::unique_ptr<Session>> active;
  uint64_t used = 0;  // footprint of the resident sessions
  for (;;) {
    std::vector<Request *> batch;
    uint64_t fp = BATCH_BASE_BYTES;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (active.empty()) {
        s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
        if (s->stop) break;
        // batching window: a few hundred microseconds for more requests
        if (s->queue.size() < s->cfg.max_batch_games)
          s->cv_work.wait_for(lk, std::chrono::microseconds(s->cfg.max_wait_us),
                              [&] { return s->stop || s->queue.size() >= s->cfg.max_batch_games; });
        if (s->stop) break;
      }
      // admit what has arrived, while it fits beside the resident sessions
      // (a pipeline without sessions always takes the first request)
      size_t n_compares = 0;
      while (!s->queue.empty() && batch.size() < s->cfg.max_batch_games && active.size() < MAX_SESSIONS) {
        Request *r = s->queue.front();
        if (r->kind && n_compares >= MAX_COMPARE_BATCH) break;
        n_compares += r->kind ? 1 : 0;
        if ((!batch.empty() || !active.empty()) && used + fp + r->footprint > s->budget) break;
        fp += r->footprint;
        s->queue.pop_front();
        r->state = 1;
        batch.push_back(r);
      }
      if (!batch.empty()) {
        s->stats.batches++;
        s->stats.games_in_batches += batch.size();
        s->stats.running += batch.size();
        s->stats.queued = s->queue.size();
        if (used + fp > s->stats.max_batch_footprint) s->stats.max_batch_footprint = used + fp;
      }
    }
    std::vector<Request *> done;
    double admit_ms = 0, step_ms = 0, retire_ms = 0;
    // the resident sessions' next step goes to the device first; the new
    // batch is staged on the host and uploaded behind it on the same stream,
    // so its packing overlaps their rounds
    const auto t1 = std::chrono::steady_clock::now();
    const size_t n_old = active.size();
    const std::vector<geq_status> enq = enqueue_steps(*e, active);
    if (!batch.empty()) {
      const auto t0 = std::chrono::steady_clock::now();
      std::vector<Request *> games, compares, wide;
      uint64_t fg = 0, fc = 0;
      for (Request *r : batch) {
        if (r->kind) {
          compares.push_back(r);
          fc += r->footprint;
        } else if (Conf(r->conf).supported()) {
          games.push_back(r);
          fg += r->footprint;
        } else {
          wide.push_back(r);
        }
      }
      const size_t before = active.size();
      if (!games.empty()) start_games(*e, games, fg, active, done);
      if (!compares.empty()) start_compares(*e, s->device, s->cfg.max_game_positions, compares, fc, active, done);
      for (size_t k = before; k < active.size(); k++) used += active[k]->footprint;
      if (!wide.empty()) {
        run_wide(*e, s->device, wide);
        done.insert(done.end(), wide.begin(), wide.end());
      }
      admit_ms = ms_since(t0);
    }
    finish_steps(*e, active, n_old, enq, used, done, retire_ms);
    step_ms = ms_since(t1) - retire_ms - admit_ms;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stats.admit_ms += admit_ms;
      s->stats.step_ms += step_ms;
      s->stats.retire_ms += retire_ms;
    }
    finish(s, done);
  }
  // stopped: the sessions in flight finish
  while (!active.empty()) {
    std::vector<Request *> done;
    double retire_ms = 0;
    const std::vector<geq_status> enq = enqueue_steps(*e, active);
    finish_steps(*e, active, active.size(), enq, used, done, retire_ms);
    finish(s, done);
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
  // 3: measured against 2 and 4 at the saturation and arrival-rate runs
  if (!s->cfg.n_pipelines) s->cfg.n_pipelines = 3;
  if (s->cfg.n_pipelines > 8) return fail(GEQ_ERR_INVALID_INPUT, "at most 8 pipelines");
  // 512: at saturation (a deep queue) batches of 512 games gave more games/s
  // and a shorter tail than batches of 256 or 4,096
  if (!s->cfg.max_batch_games) s->cfg.max_batch_games = 512;
  if (!s->cfg.max_wait_us) s->cfg.max_wait_us = 200;
  if (!s->cfg.hbm_budget_bytes) s->cfg.hbm_budget_bytes = 150ull * 1000 * 1000 * 1000;
  if (!s->cfg.max_queued) s->cfg.max_queued = 1000000;
  s->budget = s->cfg.hbm_budget_bytes / s->cfg.n_pipelines;
  s->inpool = std::make_shared<HostPool>(cudaHostAllocPortable, INPOOL_IDLE_BYTES);
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
  std::string why;
  if (!Conf(graph->conf).supported() && !wide_supported(Conf(graph->conf), &why))
    return fail(GEQ_ERR_UNSUPPORTED, "%s", why.c_str());
  const uint64_t n = graph->n_vertices, m = graph->row_offsets[n];
  const uint64_t us = Conf(graph->conf).update_size();
  std::unique_ptr<Request> r(new Request());
  r->conf = graph->conf;
  r->n = graph->n_vertices;
  if (!take_block(s, *r, (n + 1) + m + m * us + (n + 3) / 4 + n))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for a game of %llu positions", (unsigned long long)n);
  uint32_t *w = (uint32_t *)r->blk.p;
  std::memcpy(w, graph->row_offsets, (n + 1) * 4);
  r->row = w;
  w += n + 1;
  if (m) std::memcpy(w, graph->column_indices, m * 4);
  r->col = w;
  w += m;
  if (m) std::memcpy(w, graph->weights, m * us * 4);
  r->wt = w;
  w += m * us;
  uint8_t *att = (uint8_t *)w;
  for (uint64_t v = 0; v < n; v++) att[v] = graph->attacker_pos[v] ? 1 : 0;
  r->att = att;
  w += (n + 3) / 4;
  // standard reach: the defenders without successors (energygame.rs:347-352)
  uint32_t nr = 0;
  for (uint64_t v = 0; v < n; v++)
    if (!att[v] && graph->row_offsets[v + 1] == graph->row_offsets[v]) w[nr++] = (uint32_t)v;
  r->reach = w;
  r->n_reach = nr;
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

geq_status geq_server_poll_any(geq_server *s, int32_t timeout_ms, uint64_t *ticket, geq_solution **out) {
  if (!s || !out || !ticket) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  *out = nullptr;
  *ticket = 0;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    // tickets already taken by geq_server_poll are passed over
    while (!s->done_q.empty() && !s->reqs.count(s->done_q.front())) s->done_q.pop_front();
    if (!s->done_q.empty()) break;
    auto ready = [&] { return !s->done_q.empty(); };
    if (timeout_ms < 0) {
      s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
      return fail(GEQ_ERR_TIMEOUT, "no request finished");
    }
  }
  const uint64_t t = s->done_q.front();
  s->done_q.pop_front();
  auto it = s->reqs.find(t);
  Request *r = it->second.get();
  *ticket = t;
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
