// geq_internal.h - declarations shared by the sources of libgeq.so.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/geq.h"

namespace geq {

// ---- EnergyConf arithmetic (src/energy.rs:36-78) --------------------------
inline uint32_t lzcnt32(uint32_t x) { return x == 0 ? 32u : (uint32_t)__builtin_clz(x); }
inline uint32_t next_pow2(uint32_t x) { return x <= 1 ? 1u : 1u << (32 - lzcnt32(x - 1)); }
struct Conf {
  uint32_t elements = 6, max = 3;
  Conf() = default;
  Conf(uint32_t e, uint32_t m) : elements(e), max(m) {}
  explicit Conf(geq_energy_conf c) : elements(c.elements), max(c.max) {}
  uint32_t energy_bits() const { return next_pow2(32 - lzcnt32(max)); }
  uint32_t energy_mask() const { return 0xffffffffu >> (32 - energy_bits()); }
  uint32_t energy_size() const { return (energy_bits() * elements + 31) / 32; }
  uint32_t update_bits() const { return next_pow2(32 - lzcnt32(elements + 2)); }
  uint32_t update_mask() const { return 0xffffffffu >> (32 - update_bits()); }
  uint32_t update_size() const { return (update_bits() * elements + 31) / 32; }
  bool standard() const { return elements == 6 && max == 3; }
  // Device codecs: one energy word, one update word, thermometer code of
  // elements*max bits in a u32.
  bool supported() const {
    return elements >= 1 && max >= 1 && energy_size() == 1 && update_size() == 1 &&
           (uint64_t)elements * max <= 32;
  }
  bool operator==(const Conf &o) const { return elements == o.elements && max == o.max; }
};

// ---- errors -----------------------------------------------------------------
void set_last_error(const std::string &msg);
geq_status fail(geq_status st, const char *fmt, ...);

// ---- host-side game description handed to the device engine --------------
struct GameInput {
  geq_game_graph g{};
  const geq_energy_lists *init = nullptr;  // may be null
  const uint32_t *to_reach = nullptr;
  uint32_t n_reach = 0;
  std::vector<uint32_t> reach_storage;  // standard reach when none was given
  bool std_reach = false;       // standard reach, to be computed on the device (no list)
  bool rows_unchecked = false;  // row monotonicity left to the device (large batches)
  // optional: the game packed in one host block, row (n+1) | col (m) | wt (m)
  // | attacker bytes ((n+3)/4 words) | reach (n_reach), that g and to_reach
  // point into; a batch whose games all have one is copied block by block
  // and unpacked on the device (no host staging copy)
  const uint32_t *block = nullptr;
  size_t block_words = 0;
};
// Words of a packed game block (see GameInput::block).
inline size_t packed_game_words(uint64_t n, uint64_t m, uint64_t n_reach) {
  return (n + 1) + 2 * m + (n + 3) / 4 + n_reach;
}

// Validation of a graph view (TryFrom<SerdeGameGraph> checks,
// energygame.rs:65-83, plus update-code checks).
geq_status validate_graph(const geq_game_graph &g, bool check_rows = true);
geq_status validate_lists(const geq_game_graph &g, const geq_energy_lists *l);
// EnergyGame::standard_reach (energygame.rs:347-352): defenders without successors.
std::vector<uint32_t> standard_reach_of(const geq_game_graph &g);

// ---- host threads -----------------------------------------------------------
// f(i) for i < n on up to `max_threads` host threads (all cores when 0).
template <class F>
void parallel_for(uint32_t n, F f, uint32_t max_threads = 0) {
  uint32_t threads = std::max(1u, std::min<uint32_t>(std::thread::hardware_concurrency(), n));
  if (max_threads) threads = std::min(threads, max_threads);
  if (threads <= 1) {
    for (uint32_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; t++)
    pool.emplace_back([&]() {
      for (;;) {
        const uint32_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto &th : pool) th.join();
}

// ---- page-locked host memory for results -------------------------------------
// Blocks are cached by size class so that downloads copy straight into
// page-locked memory at full link speed without paying for the page locking
// on every call.  A block lent to a solution returns to the cache when the
// solution is freed; the cache lives as long as its engine or its last
// lent block, whichever is later.
class HostPool {
 public:
  HostPool() = default;
  // flags: cudaHostAlloc flags of new blocks; limit: bytes of idle blocks kept
  HostPool(unsigned flags, size_t limit) : flags_(flags), limit_(limit) {}
  static size_t round_size(size_t bytes);
  void *get(size_t bytes, size_t &cap);  // nullptr when page-locked memory is unavailable
  void put(void *p, size_t cap);
  ~HostPool();

 private:
  std::mutex mu_;
  std::map<size_t, std::vector<void *>> free_;
  size_t cached_ = 0;
  unsigned flags_ = 0;
  size_t limit_ = (size_t)4 << 30;
};

// One host array: a HostPool block, or heap memory when none could be had.
// The contents start uninitialised.
struct HostBuf {
  std::shared_ptr<HostPool> pool;
  void *p = nullptr;
  size_t cap = 0;
  bool alloc(const std::shared_ptr<HostPool> &hp, size_t bytes);
  void reset();
  HostBuf() = default;
  HostBuf(const HostBuf &) = delete;
  HostBuf &operator=(const HostBuf &) = delete;
  ~HostBuf() { reset(); }
};

}  // namespace geq

// ---- opaque objects of the C ABI ------------------------------------------
// A solution's lists live either in the vectors (results assembled on the
// host) or in the HostBufs (a whole batch copied back from the device).
struct geq_solution {
  uint32_t energy_size = 1;
  std::vector<uint32_t> n_vertices;     // per game
  std::vector<uint64_t> offsets_base;   // per game: index into the offsets
  std::vector<uint64_t> data_base;      // per game: first word in the data
  std::vector<uint64_t> offsets;        // per game n+1 entries, relative
  std::vector<uint32_t> data;
  geq::HostBuf off_buf, data_buf;
  uint64_t n_offsets = 0, n_words = 0;  // sizes when the HostBufs are used
  // a view of one game of another solution (the serving loop's answers):
  // its lists stay where they are, kept alive by `shared`
  std::shared_ptr<const geq_solution> shared;
  const uint64_t *view_off = nullptr;
  const uint32_t *view_data = nullptr;
  uint64_t view_noff = 0, view_nwords = 0;
  geq_solve_stats stats{};
  const uint64_t *off_ptr() const {
    return view_off ? view_off : off_buf.p ? (const uint64_t *)off_buf.p : offsets.data();
  }
  const uint32_t *data_ptr() const {
    return view_off ? view_data : data_buf.p ? (const uint32_t *)data_buf.p : data.data();
  }
  uint64_t offsets_len() const { return view_off ? view_noff : off_buf.p ? n_offsets : offsets.size(); }
  uint64_t data_len() const { return view_off ? view_nwords : data_buf.p ? n_words : data.size(); }
};

namespace geq {
class Engine;
struct DeviceGamesImpl;
// Releases the device memory of uploaded games and the object itself.
void destroy_games(DeviceGamesImpl *p);
struct GamesDeleter {
  void operator()(DeviceGamesImpl *p) const { destroy_games(p); }
};
using GamesPtr = std::unique_ptr<DeviceGamesImpl, GamesDeleter>;
}  // namespace geq

struct geq_context {
  int device = 0;
  std::unique_ptr<geq::Engine> engine;
  // second engine for large batches, created on first use
  std::unique_ptr<geq::Engine> engine2;
};

struct geq_device_games {
  geq::GamesPtr impl;
};

namespace geq {

// Games built on the device (device game builder) in the solver's input
// layout: per game, positions in order with row offsets relative to the game,
// successor ids local to the game.  Device pointers on the engine's stream.
struct BuiltGames {
  uint32_t n_games = 0;
  const uint32_t *n_nodes = nullptr, *n_edges = nullptr;  // host, per game
  unsigned long long N = 0, M = 0;
  const uint32_t *row_rel = nullptr, *col = nullptr, *wt = nullptr;
  const uint8_t *att = nullptr;
};

// Engine: owns the CUDA stream, events, pinned staging and the kernels.
class Engine {
 public:
  static geq_status create(int device, std::unique_ptr<Engine> &out);
  ~Engine();
  geq_status upload(std::vector<GameInput> &games, GamesPtr &out);
  geq_status upload_blocks(std::vector<GameInput> &games, GamesPtr &out);
  // games already on the device (BuiltGames), standard reach
  geq_status upload_built(const BuiltGames &b, GamesPtr &out);
  geq_status solve(DeviceGamesImpl &dg, geq_solve_stats *stats);
  // the same in steps: restart from the uploaded state, then one graph of
  // rounds per step (done: the frontier is empty); counters of the solve so far
  geq_status solve_begin(DeviceGamesImpl &dg);
  geq_status solve_step(DeviceGamesImpl &dg, bool &done);
  // one step in two halves around a synchronisation of the engine's stream
  // (several uploads' steps back to back): with `active`, the games that
  // still have frontier positions are read back too (null when unknown)
  geq_status step_enqueue(DeviceGamesImpl &dg, bool active);
  geq_status step_finish(DeviceGamesImpl &dg, bool &done, const uint8_t *&active);
  geq_status sync();
  geq_status solve_stats(DeviceGamesImpl &dg, geq_solve_stats *stats);
  // active[g] = 1 while game g has a position in the frontier
  geq_status active_games(DeviceGamesImpl &dg, std::vector<uint8_t> &active);
  // games never to be solved from the next solve_begin on (their lists stay initial)
  void skip_games(DeviceGamesImpl &dg, const std::vector<uint32_t> &games);
  // the lists of the listed games (all positions, or the first only), one
  // solution game per listed game, in page-locked memory
  geq_status download_games(DeviceGamesImpl &dg, const std::vector<uint32_t> &games, bool first_only,
                            geq_solution &sol);
  static uint32_t game_positions(const DeviceGamesImpl &dg, uint32_t g);
  static uint32_t n_games_of(const DeviceGamesImpl &dg);
  // All positions of all games.
  geq_status download(DeviceGamesImpl &dg, geq_solution &sol);
  // download in two steps: prepare gathers every list on the device and
  // counts the words; copy reads offsets (relative to each game) and words
  // into the given host memory and releases the device buffers.
  struct Readback {
    unsigned long long *goff = nullptr, *rel = nullptr;
    uint32_t *out = nullptr;
    unsigned long long total = 0;
  };
  geq_status download_prepare(DeviceGamesImpl &dg, Readback &rb);
  geq_status download_copy(DeviceGamesImpl &dg, Readback &rb, uint64_t *off_dst, uint32_t *data_dst);
  void download_release(DeviceGamesImpl &dg, Readback &rb);
  // Only the listed positions: game g's local positions first_g .. first_g+count_g-1
  // become game g of the solution.
  geq_status download_selected(DeviceGamesImpl &dg, const std::vector<uint32_t> &first,
                               const std::vector<uint32_t> &count, geq_solution &sol);
  // One small game (no initial lists, default tuning) by the one-block
  // solver in a pooled block; handled = false leaves it to upload/solve.
  geq_status solve_small(const GameInput &gi, geq_solution &sol, bool &handled);
  // geq_energy_game_run_static: one game in the file-scope scratch, no allocation.
  geq_status run_static(int device, const geq_game_graph &g, const uint32_t *to_reach, uint32_t n_reach,
                        uint64_t *offsets, uint32_t *data, uint64_t data_cap, uint64_t *n_words,
                        geq_solve_stats *stats);
  // Node id of game g's first position inside the uploaded batch.
  static uint64_t game_node_base(const DeviceGamesImpl &dg, uint32_t g);
  // The engine's CUDA stream (a cudaStream_t) and page-locked host pool, for
  // the other device passes of the library (the device game builder).
  void *stream_handle() const;
  std::shared_ptr<HostPool> host_pool() const;
  geq_tuning tuning{};
  int n_sms = 0;
  uint64_t total_mem = 0;
  std::string name;

  struct State;
  std::unique_ptr<State> st;

 private:
  geq_status clear_off_ranges(DeviceGamesImpl &dg, uint32_t stamp);
  geq_status alloc_work(DeviceGamesImpl &D, bool any_init);
  geq_status finish_upload(GamesPtr &dg, bool any_init, GamesPtr &out);
};

// The games of jobs L[j] with start positions Attack(p[t], {q[t]}) for t in
// start_off[j] .. start_off[j+1]-1 (GameBuild::compare with one start,
// compare_all with the pairs of start_pairs), built by the device game builder
// and uploaded on eng's stream as standard-reach games; the graphs never pass
// through the host.
struct Lts;
// With `trivial` set the LTSs are minimised on the device first and a
// one-start job whose processes are bisimilar gets no game (trivial[j] = 1);
// the games of out are the jobs with positions, in order (out is empty when
// there are none).
geq_status build_and_upload(Engine &eng, int device, uint32_t n_jobs, const Lts *const *L, const uint32_t *start_off,
                            const uint32_t *p, const uint32_t *q, uint64_t max_positions, GamesPtr &out,
                            double *build_ms, std::vector<uint8_t> *trivial = nullptr,
                            std::vector<uint8_t> *over = nullptr);

// Games whose EnergyConf is outside the thermometer codecs (Conf::supported
// false), or every game under GEQ_TUNE_FORCE_WIDE: the multi-word solver of
// wide.cu, one game after the other on the engine's stream.
bool wide_supported(const Conf &c, std::string *why = nullptr);
geq_status solve_wide(Engine &e, int device, std::vector<GameInput> &in, geq_solution &sol);

// A large batch split in two halves by positions on engines ea and eb: the
// upload of the second half overlaps the solve of the first.
geq_status run_batch_pipelined(int device, Engine &ea, Engine &eb, std::vector<GameInput> &in, geq_solution &sol);

}  // namespace geq
