/*
 * geq_oracle.h - CPU restatement of gpuequiv's energy-game path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: it is loaded
 * by tests/, by __graft_entry__.smoke() (as the checker) and by bench.py's
 * cpu_baseline / --impl reference leg.  Nothing in the product
 * (gpuequiv_b200/, libgeq.so) links, loads or calls it.
 *
 * Every function restates the reference crate (Gobbel2000/gpuequiv 1.0.0,
 * Rust + WGSL) and cites the file:line it follows.  The reference cannot be
 * built in this image (no cargo/rustc; wgpu 0.20 is not vendored), so the
 * restatement is pinned against the golden vectors of the reference's own
 * tests (tests/energygame.rs, tests/complete.rs, src/energygame/tests.rs,
 * src/energy.rs tests, the lib.rs doctests); see tests/golden/.
 *
 * Plain C ABI so that ctypes can drive it.
 */
#ifndef GEQ_ORACLE_H
#define GEQ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- EnergyConf (src/energy.rs:36-78) ---------------------------------- */
uint32_t ora_energy_bits(uint32_t elements, uint32_t max);
uint32_t ora_energy_size(uint32_t elements, uint32_t max);
uint32_t ora_energy_mask(uint32_t elements, uint32_t max);
uint32_t ora_update_bits(uint32_t elements, uint32_t max);
uint32_t ora_update_size(uint32_t elements, uint32_t max);
uint32_t ora_update_mask(uint32_t elements, uint32_t max);

/* ---- packing (src/energy.rs:143-179, :543-588) -------------------------- */
/* returns 0 on success, -1 if the values do not fit the conf (pack_* -> None) */
int ora_pack_energy(uint32_t elements, uint32_t max, const uint32_t *vals,
                    uint32_t n, uint32_t *out);
void ora_unpack_energy(uint32_t elements, uint32_t max, const uint32_t *words,
                       uint32_t *out);
/* updates in the crate's i32 form: 0 Zero, -1 Decrement, k>=1 Min(k) */
int ora_pack_update(uint32_t elements, uint32_t max, const int32_t *vals,
                    uint32_t n, uint32_t *out);
void ora_unpack_update(uint32_t elements, uint32_t max, const uint32_t *words,
                       int32_t *out);
/* inv_update of one packed energy (attack_update.wgsl:45-61) */
void ora_inv_update(uint32_t elements, uint32_t max, const uint32_t *energy,
                    const uint32_t *update, uint32_t *out);

/* ---- EnergyGame::run (src/energygame.rs:379-383, :1461-1523) ------------ */
typedef struct OraSolution OraSolution;
/* init_offsets/init_data may be NULL: then energies start empty except the
 * to_reach positions, which get {0} (EnergyGame::with_reach, :355-365). */
OraSolution *ora_run_game(uint32_t elements, uint32_t max, uint32_t n,
                          const uint32_t *row_offsets, const uint32_t *col,
                          const uint32_t *weights, const uint8_t *attacker,
                          const uint64_t *init_offsets, const uint32_t *init_data,
                          const uint32_t *to_reach, uint32_t n_reach);
uint64_t ora_solution_total(const OraSolution *s);
void ora_solution_offsets(const OraSolution *s, uint64_t *out);
void ora_solution_data(const OraSolution *s, uint32_t *out);
/* stats: [rounds, attack visits, defend visits, defend overflow retries,
 *         edges relaxed, algorithmic bytes] */
void ora_solution_stats(const OraSolution *s, uint64_t *out);
void ora_solution_free(OraSolution *s);

/* Standard reach of a graph (EnergyGame::standard_reach, :347-352).
 * Writes the defender sinks to out (capacity n) and returns their count. */
uint32_t ora_standard_reach(uint32_t n, const uint32_t *row_offsets,
                            const uint8_t *attacker, uint32_t *out);

/* One workgroup of defend_iterative.wgsl:182-267 on already-updated
 * energies.  succ_offsets has n_succ+1 entries (relative to energies).
 * Returns the shader's status (>=0: size of the result written to sup_out,
 * <0: -required memory).  sup_out needs room for `mem` energies. */
int32_t ora_defend_intersection(uint32_t elements, uint32_t max,
                                const uint32_t *energies,
                                const uint32_t *succ_offsets, uint32_t n_succ,
                                uint32_t mem, uint32_t *sup_out);

/* ---- TransitionSystem (src/lib.rs) -------------------------------------- */
typedef struct OraLts OraLts;
OraLts *ora_lts_from_edges(uint64_t n_edges, const uint32_t *src,
                           const uint32_t *dst, const int32_t *label);
/* err: 0 ok, 1 io, 2 missing field, 3 parse error */
OraLts *ora_lts_from_csv(const char *path, int *err);
uint32_t ora_lts_n_vertices(const OraLts *l);
uint64_t ora_lts_n_transitions(const OraLts *l);
void ora_lts_transitions(const OraLts *l, uint64_t *offsets, uint32_t *targets,
                         int32_t *labels);
uint64_t ora_lts_signature_refinement(const OraLts *l, uint64_t *partition);
OraLts *ora_lts_minimize(const OraLts *l, uint64_t *mapping);
void ora_lts_free(OraLts *l);

/* ---- GameBuild (src/gamebuild.rs, src/gamebuild/gamepos.rs) ------------- */
typedef struct OraBuild OraBuild;
OraBuild *ora_build_compare(const OraLts *l, uint32_t p, uint32_t q);
OraBuild *ora_build_compare_all(const OraLts *l);
uint32_t ora_build_n_nodes(const OraBuild *b);
uint64_t ora_build_n_edges(const OraBuild *b);
uint32_t ora_build_n_starting(const OraBuild *b);
void ora_build_graph(const OraBuild *b, uint32_t *row_offsets, uint32_t *col,
                     uint32_t *weights, uint8_t *attacker);
/* kind: 0 Attack, 1 Clause, 2 Defend */
void ora_build_position(const OraBuild *b, uint32_t idx, uint32_t *kind,
                        uint32_t *p, uint32_t *nq, uint32_t *nqx);
void ora_build_position_sets(const OraBuild *b, uint32_t idx, uint32_t *q,
                             uint32_t *qx);
void ora_build_free(OraBuild *b);

/* ---- whole pipelines, used for CPU baselines ---------------------------- */
/* TransitionSystem::compare (lib.rs:275-283) for many (lts, p, q) jobs on
 * n_threads host threads.  out_counts[i] = number of energies of the start
 * position; out_nodes[i] = game size (0 when the pair is bisimilar). */
void ora_compare_batch(uint32_t n_jobs, const OraLts *const *lts,
                       const uint32_t *p, const uint32_t *q, uint32_t n_threads,
                       uint64_t *out_counts, uint64_t *out_nodes);
/* EnergyGame::run on many games in parallel (graph given as CSR arrays). */
/* Test support, at sizes the sequential solve would take too long for:
 * the number of positions whose list one more worklist step (the update of
 * a run_game round) would change, given final lists (offsets[n+1] in
 * energies, data packed); 0 for a fixpoint.  *first_bad = the first such
 * position (0xFFFFFFFF when none). */
uint64_t ora_check_fixpoint(uint32_t elements, uint32_t max, uint32_t n, const uint32_t *row_offsets,
                            const uint32_t *col, const uint32_t *weights, const uint8_t *attacker,
                            const uint64_t *offsets, const uint32_t *data, uint32_t n_threads,
                            uint32_t *first_bad);
void ora_run_games_parallel(uint32_t n_games, uint32_t elements, uint32_t max,
                            const uint32_t *n_pos, /* positions per game */
                            const uint32_t *const *row_offsets,
                            const uint32_t *const *col,
                            const uint32_t *const *weights,
                            const uint8_t *const *attacker, uint32_t n_threads,
                            uint64_t *out_total);
/* The same with the lists kept: games are taken from one shared counter in
 * `order` (NULL: index order) by n_threads threads; out_total and out_sol
 * (one OraSolution per game, freed by ora_solution_free) may each be NULL. */
void ora_solve_games(uint32_t n_games, uint32_t elements, uint32_t max, const uint32_t *n_pos,
                     const uint32_t *const *row_offsets, const uint32_t *const *col,
                     const uint32_t *const *weights, const uint8_t *const *attacker, uint32_t n_threads,
                     const uint32_t *order, uint64_t *out_total, OraSolution **out_sol);
/* Schedule-independent byte floor of a solve from its final lists A*:
 * 4(n+1) + 8m + n + sum_v 4|A*_v|(1 + indeg(v)) -- every row pair and edge
 * read once, the attacker flags once, every final list written once and read
 * once per predecessor (STANDARD: one word per energy). */
uint64_t ora_b_min(uint32_t n, const uint32_t *row_offsets, const uint32_t *col, const uint64_t *offsets);

#ifdef __cplusplus
}
#endif
#endif
