/*
 * geq.h - C ABI of the B200 energy-game solver (libgeq.so).
 *
 * This is the drop-in boundary for the energy-game path of the gpuequiv
 * crate: a Rust (or any FFI) host that owns `GameGraph`/`EnergyGame`/
 * `TransitionSystem` values passes plain pointers and sizes here instead of
 * running the wgpu pipelines.  Every entry point names the reference
 * interface (file:line inside the crate) it replaces.
 *
 * Conventions
 *  - Energies and updates use the crate's packed layout (src/energy.rs:143-179,
 *    :543-588): an energy is `energy_size` u32 words, an update `update_size`
 *    words.  Energy lists are CSR: position v owns energies
 *    offsets[v] .. offsets[v+1] (counted in energies, not words).
 *  - Host buffers passed in are borrowed for the duration of the call.
 *    Objects returned through `**out` are owned by the caller and released
 *    with the matching *_free function.  Views filled by *_view / *_lists
 *    functions point into the owning object and live as long as it does.
 *  - Every function that can fail returns a geq_status; the detail message of
 *    the last failure on the calling thread is geq_last_error().
 *  - A geq_context is bound to one CUDA device and one stream.  It may be used
 *    from one thread at a time; create one context per host thread for
 *    concurrency.
 *  - There is no CPU fallback: without a usable CUDA device the solver entry
 *    points return GEQ_ERR_NO_DEVICE.
 */
#ifndef GEQ_H
#define GEQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* 2: geq_tuning.lane_limits, geq_server_config.max_game_positions,
 *    geq_conf_solvable, GEQ_TUNE_FORCE_WIDE */
#define GEQ_ABI_VERSION 2

/* Error codes.  Replaces gpuequiv::Error (src/error.rs:3-40) and the
 * TryFrom<SerdeGameGraph> checks (src/energygame.rs:65-83). */
typedef enum geq_status {
  GEQ_OK = 0,
  GEQ_ERR_NO_DEVICE = 1,     /* Error::NoAdapter / Error::NoDevice */
  GEQ_ERR_OUT_OF_MEMORY = 2, /* device or pinned host allocation failed */
  GEQ_ERR_INVALID_INPUT = 3, /* malformed graph / energies / arguments */
  GEQ_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  GEQ_ERR_UNSUPPORTED = 5,   /* EnergyConf outside the device codecs */
  GEQ_ERR_CUDA = 6,          /* other CUDA runtime failure (~Error::BufferMap) */
  GEQ_ERR_IO = 7,            /* CSVError::IOError */
  GEQ_ERR_PARSE = 8,         /* CSVError::MissingField / ParseError */
  GEQ_ERR_BUSY = 9,          /* serving: admission budget exhausted */
  GEQ_ERR_INTERNAL = 10
} geq_status;

const char *geq_status_string(geq_status s);
/* Detail of the last failure on this thread ("" if none). */
const char *geq_last_error(void);
int geq_abi_version(void);

/* ---- EnergyConf (src/energy.rs:36-78) ---------------------------------- */
typedef struct geq_energy_conf {
  uint32_t elements;
  uint32_t max;
} geq_energy_conf;
/* EnergyConf::STANDARD = {6, 3} (energy.rs:44) */
uint32_t geq_conf_energy_bits(geq_energy_conf c);  /* energy.rs:56-59 */
uint32_t geq_conf_energy_size(geq_energy_conf c);  /* energy.rs:49-53 */
uint32_t geq_conf_energy_mask(geq_energy_conf c);  /* energy.rs:61-63 */
uint32_t geq_conf_update_bits(geq_energy_conf c);  /* energy.rs:70-73 */
uint32_t geq_conf_update_size(geq_energy_conf c);  /* energy.rs:65-68 */
uint32_t geq_conf_update_mask(geq_energy_conf c);  /* energy.rs:75-77 */
/* 1 if the conf has a thermometer codec (energy and update fit one word and
 * elements*max <= 32): the batched round kernels, device-resident games and
 * geq_energy_game_run_static take it.  Else 0. */
int geq_conf_supported(geq_energy_conf c);
/* 1 if geq_energy_game_run / _batch and the serving loop solve games of this
 * conf: every conf with elements >= 1, an energy of at most 64 words and an
 * update of at most 128 words (e.g. ONE_DIMENSION {1, u32::MAX}: one 32-bit
 * field; {30, 3}: 2 energy words, 8 update words); the confs without a
 * thermometer codec take the multi-word solver.  EnergyConf itself has no
 * limit (energy.rs:36-78); the reference generates its shaders per conf
 * (shadergen.rs:159-189). */
int geq_conf_solvable(geq_energy_conf c);

/* ---- Energy / Update packing ------------------------------------------- */
/* Energy::new (energy.rs:88-93, pack_energy :143-162).  n_values <= elements;
 * missing values are 0.  GEQ_ERR_INVALID_INPUT where the crate returns None. */
geq_status geq_energy_pack(geq_energy_conf c, const uint32_t *values, uint32_t n_values,
                           uint32_t *out_words);
/* From<&Energy> for Vec<u32> (energy.rs:164-179): `elements` values. */
void geq_energy_unpack(geq_energy_conf c, const uint32_t *words, uint32_t *out_values);
/* Update::new via Upd::from(i32) (energy.rs:474-490, :510-515, pack_upd
 * :543-565): 0 Zero, -1 Decrement, k >= 1 Min(k). */
geq_status geq_update_pack(geq_energy_conf c, const int32_t *values, uint32_t n_values,
                           uint32_t *out_words);
/* From<&Update> for Vec<i32> (energy.rs:567-602). */
void geq_update_unpack(geq_energy_conf c, const uint32_t *words, int32_t *out_values);
/* EnergyArray::test_equivalence (energy.rs:307-318): 1 if no energy of the
 * list is <= `equivalence` (the equivalence holds), else 0. */
int geq_test_equivalence(geq_energy_conf c, const uint32_t *energies, uint64_t n_energies,
                         const uint32_t *equivalence_words);

/* ---- GameGraph (src/energygame.rs:120-138) ------------------------------ */
/* CSR view of a game graph in host memory.  Mirrors the pub fields
 * column_indices / row_offsets / weights / attacker_pos; the reverse graph is
 * derived on the device. */
typedef struct geq_game_graph {
  geq_energy_conf conf;
  uint32_t n_vertices;
  const uint32_t *row_offsets;    /* n_vertices + 1 */
  const uint32_t *column_indices; /* row_offsets[n_vertices] */
  const uint32_t *weights;        /* row_offsets[n_vertices] * update_size words */
  const uint8_t *attacker_pos;    /* n_vertices, 0 or 1 */
} geq_game_graph;

/* Energy lists (Vec<EnergyArray>). */
typedef struct geq_energy_lists {
  uint32_t n_vertices;
  uint32_t energy_size;    /* words per energy */
  const uint64_t *offsets; /* n_vertices + 1 */
  const uint32_t *data;    /* offsets[n_vertices] * energy_size words */
} geq_energy_lists;

/* EnergyGame::standard_reach (energygame.rs:347-352): writes the defender
 * positions without successors to out (capacity n_vertices), returns count. */
uint32_t geq_standard_reach(const geq_game_graph *g, uint32_t *out);

/* ---- device context ----------------------------------------------------- */
/* Replaces GPUCommon::get_gpu (src/energygame/gpuutils.rs:15-31). */
typedef struct geq_context geq_context;
geq_status geq_context_create(int device, geq_context **out);
void geq_context_destroy(geq_context *ctx);
/* Name of the device, number of SMs and total memory (for reports). */
geq_status geq_context_info(const geq_context *ctx, char *name, size_t name_len, int *n_sms,
                            uint64_t *total_mem);

/* ---- solving ------------------------------------------------------------ */
typedef struct geq_solve_stats {
  uint64_t rounds;              /* worklist rounds until the fixpoint */
  uint64_t positions_computed;  /* position recomputations */
  uint64_t edges_relaxed;       /* (v, w) relaxations */
  uint64_t algorithmic_bytes;   /* bytes the algorithm must move: per edge
                                   relaxation 16 + 4|A_w|, per recomputed
                                   position 12 (+4|A_v| for an attacker's own
                                   list), +4 per energy written */
  uint64_t arena_compactions;   /* energy-arena garbage collections */
  uint64_t kernel_launches;     /* kernels launched by the solve */
  double device_ms;             /* device time of the solve (CUDA events) */
  double round_kernel_ms;       /* GEQ_TUNE_PROFILE only: summed duration of the
                                   round kernel launches (CUDA events around each) */
  uint64_t round_kernel_launches;
} geq_solve_stats;

/* Result of a solve: one or more games, each with its per-position lists. */
typedef struct geq_solution geq_solution;
uint32_t geq_solution_n_games(const geq_solution *s);
/* Lists of game `game` (borrowed from the solution). */
geq_status geq_solution_lists(const geq_solution *s, uint32_t game, geq_energy_lists *out);
/* All games' lists at once (borrowed): game g's n_vertices(g)+1 offsets start
 * at offsets[first_offset(g)] where first_offset(g) = sum over h < g of
 * (n_vertices(h) + 1); they count energies from game g's first energy, and
 * game g's energies follow game g-1's in `data`; *n_words is the number of
 * words in `data` (energies x energy_size).  Lets a binding hand the whole
 * batch to its caller without per-game calls.  No counterpart in the crate,
 * whose results are per EnergyGame. */
geq_status geq_solution_flat(const geq_solution *s, const uint64_t **offsets, uint64_t *n_offsets,
                             const uint32_t **data, uint64_t *n_words);
void geq_solution_stats(const geq_solution *s, geq_solve_stats *out);
void geq_solution_free(geq_solution *s);

/* EnergyGame::run (energygame.rs:379-383) on EnergyGame { graph, energies,
 * to_reach } (:329-338).  `initial` may be NULL: then every position starts
 * empty except the to_reach positions, which start with {0}
 * (EnergyGame::with_reach, :355-365).  Host buffers in, host buffers out. */
geq_status geq_energy_game_run(geq_context *ctx, const geq_game_graph *graph,
                               const geq_energy_lists *initial, const uint32_t *to_reach,
                               uint32_t n_to_reach, geq_solution **out);

/* geq_energy_game_run_static: geq_energy_game_run for one game with no initial
 * lists, computed without allocating any memory -- no cudaMalloc/cudaFree, no
 * page-locked or heap buffers, no CUDA graph.  The game, its reverse CSR, the
 * energy lists and the frontiers live in one file-scope device array of
 * GEQ_STATIC_SCRATCH_BYTES per device, and one single-block kernel runs the
 * whole solve.  For callers that cannot allocate device memory when they
 * solve: a process whose own allocator has reserved the device's memory (a
 * serving framework or caching allocator that preallocates HBM, where a
 * cudaMalloc fails), and latency-bound callers whose other streams would be
 * stalled by the implicit device-wide synchronisation of cudaFree.
 *
 * to_reach: NULL = standard reach (EnergyGame::standard_reach), else the
 *   n_to_reach positions that start with {0}.
 * offsets (n_vertices + 1 entries) and data (data_cap words) receive the
 *   lists in the layout of geq_energy_lists; *n_words = result words, set
 *   also when data_cap is too small (then GEQ_ERR_INVALID_INPUT and data is
 *   not written).  After any other error offsets and data are unspecified.
 * Limit: the game takes 45 bytes per position + 12 per edge + 4 per
 *   explicit to_reach entry of the scratch, plus up to 4 KiB of alignment
 *   (each of its 15 arrays starts on a 256-byte boundary); the rest (at least
 *   16 KiB) holds the energy lists.  A larger game gives GEQ_ERR_UNSUPPORTED,
 *   lists that outgrow the rest GEQ_ERR_OUT_OF_MEMORY.
 * The scratch is reserved on a device when a context is created there
 * (geq_context_create loads the module that holds it): create the context
 * before the caller's own allocator reserves the device's memory.  Every call
 * looks the scratch's device address up (cudaGetSymbolAddress) with the
 * context's device current.  All contexts of a device share the scratch:
 * calls that overlap in time on one device race on it, so the caller must
 * serialise them.
 * No counterpart in the reference, whose runs create their buffers per run
 * (GPURunner::with_game and the shader constructors, energygame.rs:1442,
 * :507-540). */
#define GEQ_STATIC_SCRATCH_BYTES (16u << 20)
geq_status geq_energy_game_run_static(geq_context *ctx, const geq_game_graph *graph, const uint32_t *to_reach,
                                      uint32_t n_to_reach, uint64_t *offsets, uint32_t *data,
                                      uint64_t data_cap, uint64_t *n_words, geq_solve_stats *stats);

/* Many independent games solved together in one set of device rounds (the
 * batched form; no reference counterpart beyond calling EnergyGame::run once
 * per game).  initial / to_reach / n_to_reach are arrays of n_games entries;
 * initial may be NULL (all games with_reach-initialised) and
 * to_reach may be NULL (all games standard_reach). */
geq_status geq_energy_game_run_batch(geq_context *ctx, uint32_t n_games,
                                     const geq_game_graph *graphs,
                                     const geq_energy_lists *const *initial,
                                     const uint32_t *const *to_reach,
                                     const uint32_t *n_to_reach, geq_solution **out);

/* Device-resident games: upload once, solve repeatedly (each solve restarts
 * from the uploaded initial energies), download on demand.  Used to time the
 * solver with inputs already in HBM. */
typedef struct geq_device_games geq_device_games;
geq_status geq_device_games_create(geq_context *ctx, uint32_t n_games,
                                   const geq_game_graph *graphs,
                                   const geq_energy_lists *const *initial,
                                   const uint32_t *const *to_reach,
                                   const uint32_t *n_to_reach, geq_device_games **out);
geq_status geq_device_games_solve(geq_context *ctx, geq_device_games *dg,
                                  geq_solve_stats *stats);
geq_status geq_device_games_download(geq_context *ctx, geq_device_games *dg,
                                     geq_solution **out);
void geq_device_games_free(geq_device_games *dg);

/* ---- serving loop ---------------------------------------------------------
 * Requests (one game each, standard initialisation) are queued by
 * geq_server_submit and solved by pipeline threads, each with its own CUDA
 * stream, staging and device memory: a pipeline takes every queued request
 * that fits, uploads them as one batch (one id space) and keeps up to four
 * such batches resident, running one CUDA graph of worklist rounds of each in
 * turn -- requests that arrive while others are on the device are admitted at
 * the next step boundary, and each game's lists are returned as soon as its
 * own part of the frontier is empty (its fixpoint), not when its batch ends
 * (continuous batching).  The resident batches of a pipeline stay within an
 * estimated device footprint of hbm_budget_bytes / n_pipelines.
 * Results are identical to geq_energy_game_run of the same game: every game
 * keeps its own positions and frontier inside a batch.  The crate has no
 * server; its callers run EnergyGame::run per request (energygame.rs:379-383),
 * which geq_energy_game_run replaces one to one. */
typedef struct geq_server geq_server;
typedef struct geq_server_config {
  uint32_t n_pipelines;       /* pipeline threads/streams (0: 3) */
  uint32_t max_batch_games;   /* requests per batch at most (0: 512) */
  uint32_t max_wait_us;       /* a pipeline waits this long for more requests
                                 once it holds fewer than max_batch_games (0: 200) */
  uint32_t max_game_positions; /* compare queries: a query whose game would have more
                                 positions fails alone with GEQ_ERR_OUT_OF_MEMORY
                                 (0: no bound; the game is exponential in the
                                 nondeterminism of the LTS) */
  uint64_t hbm_budget_bytes;  /* device footprint of all in-flight batches (0: 150 GB) */
  uint64_t max_queued;        /* queued requests before submit answers BUSY (0: 1,000,000) */
} geq_server_config;
typedef struct geq_server_stats {
  uint64_t submitted, completed, failed, batches, queued, running;
  uint64_t games_in_batches;     /* sum of batch sizes */
  uint64_t max_batch_footprint;  /* bytes, largest resident footprint estimate */
  double admit_ms;               /* pipeline threads' wall time: staging, upload (and
                                    minimisation + GameBuild of queries) of batches,
                                    which queue behind the resident batches' rounds */
  double step_ms;                /* ... rounds of resident batches (the rest of them) */
  double retire_ms;              /* ... reading back and answering finished games */
} geq_server_stats;
/* The server solves on the device of `ctx` and copies its tuning; ctx may be
 * destroyed afterwards.  cfg may be NULL (defaults). */
geq_status geq_server_create(geq_context *ctx, const geq_server_config *cfg, geq_server **out);
/* Queue one game (copied; the caller's buffers may be reused at once).
 * GEQ_ERR_BUSY when max_queued requests wait; GEQ_ERR_INVALID_INPUT for a
 * malformed graph (the same checks as geq_energy_game_run); a game whose
 * estimated footprint alone exceeds a pipeline's budget: GEQ_ERR_OUT_OF_MEMORY. */
geq_status geq_server_submit(geq_server *srv, const geq_game_graph *graph, uint64_t *ticket);
/* Queue one equivalence query TransitionSystem::compare(p, q) (lib.rs:275-283;
 * the LTS is copied).  The queries of a batch are minimised, built and solved
 * together on the device; the solution equals geq_compare's: one game of one
 * position, the energies of Attack(p, {q}) (none for bisimilar processes).
 * Admission uses an estimate of the game from the LTS's size. */
geq_status geq_server_submit_compare(geq_server *srv, const struct geq_lts *lts, uint32_t p, uint32_t q,
                                     uint64_t *ticket);
/* Wait up to timeout_ms (< 0: forever) for request `ticket`.  GEQ_OK: *out
 * is its solution (one game; free with geq_solution_free) and the ticket is
 * retired.  GEQ_ERR_TIMEOUT: not finished yet (poll again).  Any other
 * status: the request failed with that status (message in geq_last_error)
 * and the ticket is retired.  GEQ_ERR_INVALID_INPUT for an unknown ticket. */
geq_status geq_server_poll(geq_server *srv, uint64_t ticket, int32_t timeout_ms, geq_solution **out);
/* The same for whichever request finished first (a completion queue):
 * waits up to timeout_ms (< 0: forever) for a finished request not yet
 * polled, writes its ticket to *ticket and retires it; the status and *out
 * are those geq_server_poll would give for that ticket.  GEQ_ERR_TIMEOUT
 * (and *ticket = 0) when none finished in time. */
geq_status geq_server_poll_any(geq_server *srv, int32_t timeout_ms, uint64_t *ticket, geq_solution **out);
void geq_server_get_stats(geq_server *srv, geq_server_stats *out);
/* Finishes the batches in flight, fails the queued requests, frees all. */
void geq_server_destroy(geq_server *srv);

/* Solver tuning (autotuner output).  Zero fields keep the current value. */
typedef struct geq_tuning {
  uint32_t blocks_per_sm;     /* resident 256-thread blocks per SM of the round kernel
                                 (2 to 5: selects the register budget) */
  uint32_t rounds_per_graph;  /* worklist rounds captured per CUDA graph launch */
  uint32_t small_limit;       /* candidates handled in registers per position (1..32) */
  uint32_t flags;             /* GEQ_TUNE_* bits */
  uint32_t lane_limits;       /* positions the round kernel solves one per lane (the
                                 others go to one warp each): at most bits 0-7
                                 successors (1..16), bits 8-15 candidates per step
                                 (1..64), bits 16-23 energies in the own / first list
                                 (1..16); 0 keeps the current value, a zero field
                                 means the largest */
} geq_tuning;
#define GEQ_TUNE_FORCE_GENERIC 1u /* generic codec even for STANDARD (cross-check) */
#define GEQ_TUNE_FORCE_LARGE 2u   /* bypass the register paths (cross-check) */
#define GEQ_TUNE_NO_GRAPH 4u      /* launch rounds (and GameBuild levels) one by one instead of graphs */
#define GEQ_TUNE_PROFILE 8u       /* time every round-kernel launch (implies no graphs) */
#define GEQ_TUNE_NO_THREAD_PATH 16u /* no lane-per-position path (cross-check) */
#define GEQ_TUNE_NO_SPLIT 32u     /* a large batch on one engine, not as two pipelined halves */
#define GEQ_TUNE_BUILD_WARP_ALL 64u /* device GameBuild: every attack position by the warp path (cross-check) */
#define GEQ_TUNE_FORCE_WIDE 128u  /* geq_energy_game_run(_batch): the multi-word solver for every conf (cross-check) */
#define GEQ_TUNE_READY 256u       /* count per defender the successors without energies and push a defender
                                     only once it has none (the reference visits and skips it); measured
                                     slower on the spectroscopy batch, off by default */
#define GEQ_TUNE_NO_EDGE_PAIRS 512u /* the lane path reads col / wt and decodes updates (cross-check) */
geq_status geq_context_set_tuning(geq_context *ctx, const geq_tuning *t);
void geq_context_get_tuning(const geq_context *ctx, geq_tuning *t);

/* ---- TransitionSystem (src/lib.rs) -------------------------------------- */
typedef struct geq_lts geq_lts;
/* FromIterator<(u32, u32, i32)> (lib.rs:523-536): edges (src, dst, label). */
geq_status geq_lts_from_edges(uint64_t n_edges, const uint32_t *src, const uint32_t *dst,
                              const int32_t *label, geq_lts **out);
/* From<Vec<Vec<Transition>>> (lib.rs:507-514): n_vertices adjacency lists
 * given as edges (src, dst, label); processes beyond the largest id in the
 * edges keep empty lists (the serde layout's trailing isolated processes). */
geq_status geq_lts_from_adjacency(uint32_t n_vertices, uint64_t n_edges, const uint32_t *src,
                                  const uint32_t *dst, const int32_t *label, geq_lts **out);
/* TransitionSystem::from_csv_file (lib.rs:364-406). */
geq_status geq_lts_from_csv_file(const char *path, geq_lts **out);
uint32_t geq_lts_n_vertices(const geq_lts *l);
uint64_t geq_lts_n_transitions(const geq_lts *l);
/* Adjacency lists sorted by label (inner(), lib.rs:496-499):
 * offsets[n+1], targets[m], labels[m]. */
void geq_lts_transitions(const geq_lts *l, uint64_t *offsets, uint32_t *targets,
                         int32_t *labels);
/* TransitionSystem::signature_refinement (lib.rs:444-464). */
geq_status geq_lts_signature_refinement(const geq_lts *l, uint64_t *partition,
                                        uint64_t *n_classes);
/* TransitionSystem::bisimilar_minimize (lib.rs:413-432). */
geq_status geq_lts_bisimilar_minimize(const geq_lts *l, geq_lts **reduced, uint64_t *mapping);
/* TransitionSystem::signature_refinement (lib.rs:444-464) of n_lts systems at
 * once on the context's device: partitions holds each system's per-process
 * class ids in turn (sum of the process counts), n_classes one count per
 * system; both identical to geq_lts_signature_refinement's. */
geq_status geq_lts_signature_refinement_batch(geq_context *ctx, uint32_t n_lts, const geq_lts *const *lts,
                                              uint64_t *partitions, uint64_t *n_classes);
void geq_lts_free(geq_lts *l);

/* ---- GameBuild (src/gamebuild.rs) --------------------------------------- */
typedef struct geq_game_build geq_game_build;
/* GameBuild::compare (gamebuild.rs:165-170) */
geq_status geq_game_build_compare(const geq_lts *l, uint32_t p, uint32_t q,
                                  geq_game_build **out);
/* GameBuild::compare_all (gamebuild.rs:200-215) */
geq_status geq_game_build_compare_all(const geq_lts *l, geq_game_build **out);
/* GameBuild::compare_multiple (gamebuild.rs:176-194) */
geq_status geq_game_build_compare_multiple(const geq_lts *l, const uint32_t *processes,
                                           uint32_t n_processes, geq_game_build **out);
/* GameBuild::compare with a bound: GEQ_ERR_OUT_OF_MEMORY if the game would
 * have more than max_positions positions (the game is exponential in the
 * nondeterminism of the LTS; the reference has no such guard). */
geq_status geq_game_build_compare_bounded(const geq_lts *l, uint32_t p, uint32_t q,
                                          uint64_t max_positions, geq_game_build **out);
/* The generated GameGraph (borrowed view). */
void geq_game_build_graph(const geq_game_build *b, geq_game_graph *out);
uint32_t geq_game_build_n_starting_points(const geq_game_build *b);
/* Position (gamepos.rs:210-215): kind 0 Attack, 1 Clause, 2 Defend.  For a
 * Clause, q has one element. */
typedef struct geq_position {
  uint32_t kind;
  uint32_t p;
  const uint32_t *q;
  uint32_t n_q;
  const uint32_t *qx;
  uint32_t n_qx;
} geq_position;
geq_status geq_game_build_position(const geq_game_build *b, uint32_t idx, geq_position *out);
void geq_game_build_free(geq_game_build *b);

/* ---- GameBuild on the device ----------------------------------------------
 * GameBuild::compare (gamebuild.rs:165-170, successors gamepos.rs:17-198) for
 * n_jobs (lts[j], p[j], q[j]) jobs at once, built on the context's device:
 * every breadth-first level of all jobs' games is expanded by one group of
 * kernels.  Each job's game is identical to geq_game_build_compare's (same
 * position numbering, adjacency order and weights).  A job whose game would
 * exceed max_positions positions (0 = no bound) is marked and its graph
 * refused with GEQ_ERR_OUT_OF_MEMORY, as geq_game_build_compare_bounded does. */
typedef struct geq_game_batch geq_game_batch;
geq_status geq_game_build_compare_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts,
                                        const uint32_t *p, const uint32_t *q, uint64_t max_positions,
                                        geq_game_batch **out);
/* The same with any start positions: job j starts from Attack(p[t], {q[t]}) for
 * t in start_off[j] .. start_off[j+1]-1 (start_off has n_jobs + 1 entries,
 * start_off[0] = 0), numbered 0.. in that order, as GameBuild::new_node does
 * for compare_multiple / compare_all (gamebuild.rs:176-215; the start pairs of
 * compare_all are every ordered pair of distinct processes inside each
 * enabledness class, classes in order of their first process).  The start
 * positions of one job must be distinct. */
geq_status geq_game_build_starts_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts,
                                       const uint32_t *start_off, const uint32_t *p, const uint32_t *q,
                                       uint64_t max_positions, geq_game_batch **out);
uint32_t geq_game_batch_n_jobs(const geq_game_batch *b);
uint32_t geq_game_batch_n_starting_points(const geq_game_batch *b, uint32_t job);
/* Job's GameGraph (borrowed view, STANDARD conf). */
geq_status geq_game_batch_graph(const geq_game_batch *b, uint32_t job, geq_game_graph *out);
typedef struct geq_game_batch_info {
  uint64_t positions, edges; /* all jobs */
  uint32_t levels;           /* breadth-first levels of the deepest game */
  uint32_t kernel_launches;
  uint32_t attempts;         /* 1 unless a fingerprint collision forced a new hash seed */
  double upload_ms, build_ms, download_ms; /* host wall time of each phase */
} geq_game_batch_info;
void geq_game_batch_stats(const geq_game_batch *b, geq_game_batch_info *out);
void geq_game_batch_free(geq_game_batch *b);

/* ---- whole algorithm (lib.rs:275-343, src/equivalence.rs) --------------- */
/* TransitionSystem::compare (minimize != 0) / compare_unminimized: the
 * solution holds one game with a single position: the energies of the start
 * position Attack(p, {q}).  Minimisation, game construction and solving all
 * run on the device. */
geq_status geq_compare(geq_context *ctx, const geq_lts *l, uint32_t p, uint32_t q, int minimize,
                       geq_solution **out);
/* compare() for many (lts, p, q) jobs; every game solved in one batch.  The
 * solution holds n_jobs games of one position each. */
geq_status geq_compare_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts,
                             const uint32_t *p, const uint32_t *q, int minimize,
                             geq_solution **out);

/* TransitionSystem::equivalences (minimize != 0) / equivalences_unminimized. */
typedef struct geq_equivalence geq_equivalence;
geq_status geq_equivalences(geq_context *ctx, const geq_lts *l, int minimize,
                            geq_equivalence **out);
/* Equivalence::energies (equivalence.rs:96-98): 0 if (p, q) was no start. */
int geq_equivalence_energies(const geq_equivalence *e, uint32_t p, uint32_t q,
                             const uint32_t **data, uint64_t *n_energies);
/* Equivalence::preorder / equiv (equivalence.rs:125-144); `equivalence` is a
 * packed STANDARD energy (std_equivalences, energy.rs:212-224). */
int geq_equivalence_preorder(const geq_equivalence *e, uint32_t p, uint32_t q,
                             const uint32_t *equivalence);
int geq_equivalence_equiv(const geq_equivalence *e, uint32_t p, uint32_t q,
                          const uint32_t *equivalence);
/* Equivalence::relation (equivalence.rs:154-170): class representative of
 * every (original) process, written to classes[n_processes]; returns the
 * number of classes in *n_classes.  Representatives are the smallest member
 * of each class. */
geq_status geq_equivalence_relation(const geq_equivalence *e, const uint32_t *equivalence,
                                    uint32_t *classes, uint32_t *n_classes);
uint32_t geq_equivalence_n_processes(const geq_equivalence *e);
uint32_t geq_equivalence_n_starting_points(const geq_equivalence *e);
void geq_equivalence_free(geq_equivalence *e);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* GEQ_H */
