// loadgen.cpp - request load for a serving loop (geq_server) from native
// threads, the way a native client drives the C ABI: an open loop (request i
// submitted at its arrival time) and a closed loop (a fixed number of
// requests kept in flight).  Finished requests are taken in completion order
// (geq_server_poll_any).  The server is reached through function pointers,
// so the same driver runs against libgeq or against a stand-in on the CPU.
// Built as its own library (libgeq_load.so); it is measurement tooling for
// the serving loop, not part of the solver.
//
// Per request, in submission order: the latency from just before the submit
// call to the moment its answer was taken (ms), and its status (the
// geq_status of the submit or of the answer; -1 = not answered before the
// drain deadline).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

extern "C" {

// submit(ctx, item, &ticket) -> status; poll_any(ctx, timeout_ms, &ticket,
// &answer) -> status with ticket 0 when nothing finished in time;
// free_answer(answer) releases an answer (the solution).
typedef int32_t (*geq_load_submit_fn)(void *ctx, uint32_t item, uint64_t *ticket);
typedef int32_t (*geq_load_poll_fn)(void *ctx, int32_t timeout_ms, uint64_t *ticket, void **answer);
typedef void (*geq_load_free_fn)(void *answer);

typedef struct geq_load_api {
  void *ctx;
  geq_load_submit_fn submit;
  geq_load_poll_fn poll_any;
  geq_load_free_fn free_answer;
} geq_load_api;

// A geq_server reached through libgeq's entry points (their addresses, so
// that this library does not link libgeq): items are game views
// (geq_server_submit of games[item]) or compare queries
// (geq_server_submit_compare of lts[item], p[item], q[item]).
typedef struct geq_load_server {
  void *server;
  const void *games;  // geq_game_graph array, or NULL
  size_t game_stride;  // sizeof(geq_game_graph)
  const void *const *lts;
  const uint32_t *p, *q;
  int32_t (*server_submit)(void *srv, const void *graph, uint64_t *ticket);
  int32_t (*server_submit_compare)(void *srv, const void *lts, uint32_t p, uint32_t q, uint64_t *ticket);
  int32_t (*server_poll_any)(void *srv, int32_t timeout_ms, uint64_t *ticket, void **solution);
  void (*solution_free)(void *solution);
} geq_load_server;

}  // extern "C"

namespace {

int32_t srv_submit(void *ctx, uint32_t item, uint64_t *ticket) {
  const geq_load_server *s = (const geq_load_server *)ctx;
  if (s->games) return s->server_submit(s->server, (const char *)s->games + (size_t)item * s->game_stride, ticket);
  return s->server_submit_compare(s->server, s->lts[item], s->p[item], s->q[item], ticket);
}
int32_t srv_poll(void *ctx, int32_t timeout_ms, uint64_t *ticket, void **answer) {
  const geq_load_server *s = (const geq_load_server *)ctx;
  return s->server_poll_any(s->server, timeout_ms, ticket, answer);
}

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct Run {
  const geq_load_api &api;
  double *lat_ms;
  int32_t *status;
  uint64_t cap;
  Clock::time_point t0;
  std::vector<Clock::time_point> t_sub;
  std::atomic<uint64_t> next{0}, submitted{0}, answered{0};
  std::atomic<int64_t> inflight{0};
  std::atomic<bool> submit_done{false};
  std::mutex mu;
  std::unordered_map<uint64_t, uint64_t> index;    // ticket -> request index
  std::unordered_map<uint64_t, std::pair<Clock::time_point, int32_t>> early;  // answered before indexed
  std::atomic<int64_t> last_ns{0};

  Run(const geq_load_api &a, double *l, int32_t *s, uint64_t c) : api(a), lat_ms(l), status(s), cap(c), t_sub(c) {
    for (uint64_t i = 0; i < c; i++) {
      lat_ms[i] = 0.0;
      status[i] = -1;
    }
  }
  void record(uint64_t i, Clock::time_point t, int32_t st) {
    lat_ms[i] = secs(t_sub[i], t) * 1e3;
    status[i] = st;
    const int64_t ns = std::chrono::duration_cast<std::chrono::nanoseconds>(t - t0).count();
    int64_t prev = last_ns.load();
    while (ns > prev && !last_ns.compare_exchange_weak(prev, ns)) {
    }
  }
  // request i with item `item` (`reserved`: its place in flight is taken)
  void submit(uint64_t i, uint32_t item, bool reserved = false) {
    uint64_t ticket = 0;
    t_sub[i] = Clock::now();
    if (!reserved) inflight.fetch_add(1);
    const int32_t st = api.submit(api.ctx, item, &ticket);
    submitted.fetch_add(1);
    if (st != 0 || ticket == 0) {
      record(i, Clock::now(), st ? st : -2);
      inflight.fetch_sub(1);
      answered.fetch_add(1);
      return;
    }
    std::lock_guard<std::mutex> lk(mu);
    auto e = early.find(ticket);
    if (e != early.end()) {
      record(i, e->second.first, e->second.second);
      early.erase(e);
      inflight.fetch_sub(1);
      answered.fetch_add(1);
    } else {
      index.emplace(ticket, i);
    }
  }
  void poller(Clock::time_point *deadline, std::atomic<bool> *deadline_set) {
    for (;;) {
      if (submit_done.load() && answered.load() >= submitted.load()) return;
      if (deadline_set->load() && Clock::now() > *deadline) return;
      uint64_t ticket = 0;
      void *ans = nullptr;
      const int32_t st = api.poll_any(api.ctx, 20, &ticket, &ans);
      if (!ticket) continue;
      const Clock::time_point t = Clock::now();
      if (st == 0 && ans) api.free_answer(ans);
      std::lock_guard<std::mutex> lk(mu);
      auto it = index.find(ticket);
      if (it == index.end()) {
        early.emplace(ticket, std::make_pair(t, st));
        continue;
      }
      record(it->second, t, st);
      index.erase(it);
      inflight.fetch_sub(1);
      answered.fetch_add(1);
    }
  }
};

uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

// The driver's callbacks for a geq_load_server (api->ctx = s).
void geq_load_server_api(geq_load_server *s, geq_load_api *api) {
  api->ctx = s;
  api->submit = srv_submit;
  api->poll_any = srv_poll;
  api->free_answer = s->solution_free;
}

// Open loop: request i (item pick[i]) is submitted at t0 + arrivals[i]
// seconds by one of `submit_threads` threads; after the last submit the
// pollers wait at most drain_s for the rest.  lat_ms / status: n entries.
// *span_s: t0 to the last answer.  Returns the number answered.
int64_t geq_load_open(const geq_load_api *api, const uint32_t *pick, const double *arrivals, uint64_t n,
                      uint32_t submit_threads, uint32_t poll_threads, double drain_s, double *lat_ms,
                      int32_t *status, double *span_s) {
  if (!api || !api->submit || !api->poll_any || !api->free_answer || (n && (!pick || !arrivals || !lat_ms || !status)))
    return -1;
  Run r(*api, lat_ms, status, n);
  submit_threads = std::max(1u, submit_threads);
  poll_threads = std::max(1u, poll_threads);
  r.t0 = Clock::now() + std::chrono::milliseconds(20);
  Clock::time_point deadline;
  std::atomic<bool> deadline_set{false};
  std::vector<std::thread> pol, sub;
  for (uint32_t k = 0; k < poll_threads; k++) pol.emplace_back([&]() { r.poller(&deadline, &deadline_set); });
  for (uint32_t k = 0; k < submit_threads; k++)
    sub.emplace_back([&, k]() {
      for (uint64_t i = k; i < n; i += submit_threads) {
        const auto at = r.t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrivals[i]));
        std::this_thread::sleep_until(at);
        r.submit(i, pick[i]);
      }
    });
  for (auto &t : sub) t.join();
  deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(drain_s));
  deadline_set.store(true);
  r.submit_done.store(true);
  for (auto &t : pol) t.join();
  if (span_s) *span_s = r.last_ns.load() * 1e-9;
  return (int64_t)r.answered.load();
}

// Closed loop: `outstanding` requests kept in flight for `seconds` (items
// drawn uniformly, seeded, from pick[0..n_pick)), at most `cap` requests;
// then at most drain_s for the rest.  lat_ms / status: cap entries, the
// first *n_submitted used.  Returns the number answered.
int64_t geq_load_closed(const geq_load_api *api, const uint32_t *pick, uint32_t n_pick, uint32_t outstanding,
                        double seconds, uint64_t cap, uint32_t submit_threads, uint32_t poll_threads, uint64_t seed,
                        double drain_s, double *lat_ms, int32_t *status, uint64_t *n_submitted, double *span_s) {
  if (!api || !api->submit || !api->poll_any || !api->free_answer || !pick || !n_pick || !lat_ms || !status ||
      !n_submitted)
    return -1;
  Run r(*api, lat_ms, status, cap);
  submit_threads = std::max(1u, submit_threads);
  poll_threads = std::max(1u, poll_threads);
  r.t0 = Clock::now();
  const Clock::time_point t_end =
      r.t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(seconds));
  Clock::time_point deadline;
  std::atomic<bool> deadline_set{false};
  std::vector<std::thread> pol, sub;
  for (uint32_t k = 0; k < poll_threads; k++) pol.emplace_back([&]() { r.poller(&deadline, &deadline_set); });
  for (uint32_t k = 0; k < submit_threads; k++)
    sub.emplace_back([&, k]() {
      uint64_t rng = seed * 0x100000001B3ull + k + 1;
      while (Clock::now() < t_end) {
        if (r.inflight.fetch_add(1) >= (int64_t)outstanding) {  // a place in flight
          r.inflight.fetch_sub(1);
          std::this_thread::sleep_for(std::chrono::microseconds(20));
          continue;
        }
        const uint64_t i = r.next.fetch_add(1);
        if (i >= r.cap) {
          r.inflight.fetch_sub(1);
          return;
        }
        r.submit(i, pick[splitmix(rng) % n_pick], true);
      }
    });
  for (auto &t : sub) t.join();
  *n_submitted = std::min<uint64_t>(r.next.load(), r.cap);
  deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(drain_s));
  deadline_set.store(true);
  r.submit_done.store(true);
  for (auto &t : pol) t.join();
  if (span_s) *span_s = r.last_ns.load() * 1e-9;
  return (int64_t)r.answered.load();
}

}  // extern "C"
