// engine.cu - the energy-game fixpoint on the B200.
//
// Reference path: EnergyGame::run -> GPURunner::execute_gpu
// (src/energygame.rs:379-383, :1461-1523) with the attack shaders
// (attack_update.wgsl:77-113, attack_minimize.wgsl:69-122) and the defend
// shaders (defend_update.wgsl:73-101, defend_iterative.wgsl:182-267).
//
// The reference runs a Jacobi worklist: every round it gathers the successor
// energies of all queued positions on the host, uploads them, runs the four
// shaders, maps the results back and rebuilds the queues from the reverse
// graph.  Here the whole loop stays on the device:
//
//   * The game (CSR + reverse CSR), the per-position energy lists and the
//     frontier are resident in HBM.  A list of up to 5 energies sits inline
//     in its position's 64-bit descriptor; longer ones are slices of one
//     energy arena (offset << 24 | count).
//   * k_round: each lane of a warp solves one frontier position (the lane
//     path: the successors' lists read straight from HBM, the inverse edge
//     update applied, candidates streamed into an antichain in shared
//     memory), stores the new list in a per-slot buffer and, if the list
//     changed, marks its predecessors in the next-frontier bitmap.  Positions
//     too large for a lane are queued for k_round_big, one warp each.
//   * k_commit: publishes the new descriptors (Jacobi: every position of a
//     round reads the lists of the previous round), counts the bitmap, and
//     flips the round; k_ffill turns the bitmap into the next frontier list
//     (attackers first, each kind in position order).
//   * Rounds are launched as CUDA graphs of several rounds each; the host
//     reads one small counter block per graph launch to detect termination.
//
// Results are identical to the reference's: the same positions are recomputed
// in the same rounds from the same inputs.  The one scheduling difference is
// that the reference delays a defender by a round when its preallocated
// suprema list overflows (energygame.rs:919-923); here the combination is
// bounded by a 4096-bit up-set bitmap and never needs a retry.  Such delays
// cannot change the final lists: both update operators are monotone on
// up-closed sets, every position is recomputed after its successors' last
// change, so the worklist ends in the least fixpoint whatever the round in
// which a position is recomputed; the attacker and multi-successor defender
// lists are the minimal elements of that fixpoint, and a single-successor
// defender's list is the image of its successor's list.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "codec.cuh"
#include "geq_internal.h"

namespace geq {

#ifndef GEQ_CHECKED
#define GEQ_CHECKED 0
#endif
// GEQ_PATH_PROFILE=1: k_round counts positions and SM cycles per code path
// into Ctr::prof and solve() prints them to stderr (diagnostic builds only).
#ifndef GEQ_PATH_PROFILE
#define GEQ_PATH_PROFILE 0
#endif

constexpr uint32_t FULL = 0xffffffffu;
constexpr unsigned long long NONE_DESC = ~0ull;
constexpr uint32_t CNT_MASK = (1u << 24) - 1u;
constexpr uint32_t ALLOC_CHUNK = 256;
constexpr int WARPS_PER_BLOCK = 8;
constexpr int BLOCK = 32 * WARPS_PER_BLOCK;
// per-warp shared memory (u32 words)
constexpr int SM_BM = 0;      // 128 words: bitmap
constexpr int SM_BM2 = 128;   // 128 words: second bitmap (own / old list)
constexpr int SM_TMP = 256;   // 32 words: segment map / compaction
constexpr int SM_PINC = 288;  // 32 words: predecessor counts (inclusive scan)
constexpr int SM_PBEG = 320;  // 32 words: predecessor row starts
constexpr int SM_WORDS = 352;
// device error bits (Ctr::error)
constexpr uint32_t DERR_LIST = 1u;     // a list longer than 2^24 - 1 energies
constexpr uint32_t DERR_BOUNDS = 2u;   // checked build: index out of range
constexpr uint32_t DERR_SCRATCH = 4u;  // list-path combination too large

// Device-resident control block.  Mutable pointers live here (not in the
// kernel parameters) so that captured CUDA graphs stay valid across arena
// compactions.
struct Ctr {
  uint32_t *arena;
  unsigned long long arena_cap;
  unsigned long long arena_top;
  uint32_t fsize[2];
  uint32_t cur;
  uint32_t stamp;  // stamp of the current frontier
  uint32_t overflow;
  uint32_t halt;
  uint32_t error;
  uint32_t err_line;
  uint32_t done_blocks;
  uint32_t pad;
  uint32_t next_slot;  // k_round: next frontier slot to hand out (32 per grab)
  uint32_t nbig;       // large positions queued by k_round for k_round_big
  uint32_t next_big;   // k_round_big: next queue entry to hand out
  uint32_t pad3;
  unsigned long long positions, edges, bytes, rounds;
#if GEQ_PATH_PROFILE
  unsigned long long prof[32];
#endif
};
#if GEQ_PATH_PROFILE
enum : int {
  PF_CYC_THREAD, PF_CYC_BIG, PF_CYC_PUSH, PF_T_ATT, PF_T_DEF, PF_B_ATT, PF_B_DEF, PF_T_CAND, PF_T_DEG,
  PF_SKIP, PF_SLOTS, PF_CYC_ALL, PF_ITERS, PF_T_UNCH, PF_B_DEG, PF_PUSHED,
  // warp routines: calls and cycles (lane 0, straight into Ctr::prof)
  PF_AS_N, PF_AS_C, PF_AB_N, PF_AB_C, PF_D1_N, PF_D1_C, PF_DS_N, PF_DS_C, PF_DB_N, PF_DB_C, PF_DK_N, PF_DK_C,
  PF_DT_N, PF_DT_C
};
#define PROF_WARP(c, n_idx, t0)                                           \
  do {                                                                    \
    if ((threadIdx.x & 31u) == 0) {                                       \
      atomicAdd(&(c)->prof[n_idx], 1ull);                                 \
      atomicAdd(&(c)->prof[(n_idx) + 1], (unsigned long long)(clock64() - (t0))); \
    }                                                                     \
  } while (0)
#define PROF_ADD(i, v) prof_acc[i] += (v)
#else
#define PROF_ADD(i, v) ((void)0)
#define PROF_WARP(c, n_idx, t0) ((void)0)
#endif

struct KParams {
  const uint32_t *row, *col, *wt, *rrow, *rcol;
  const uint8_t *flags;
  unsigned long long *desc;
  uint32_t *mark;
  uint32_t *front0, *front1;
  unsigned long long *slot_new;
  Ctr *ctr;
  unsigned long long n_nodes, n_edges;
  uint32_t el, mx, eb, em, ub, um;
  uint32_t small_limit;
  uint32_t thread_path;  // 1: lane-per-position path for small positions
  uint32_t ib, ibm, inl; // inline descriptors: bits per energy, its mask, capacity
  uint32_t mwords;       // words of one half of the frontier bitmap `mark`
  uint32_t *fpart;       // per-block set-bit counts of the bitmap (k_commit / k_fcount): attackers, defenders
  uint32_t fblocks;      // blocks of k_commit, k_fcount, k_ffill
  const uint32_t *abits; // attacker positions as a bitmap (mwords words)
  uint32_t *bigq;        // frontier slots of the large positions of the round
  // edge pairs for the lane path: successor id (low word) and the update in
  // the codec's pack_edge form (high word); null: read col / wt
  const unsigned long long *cw;
  uint32_t td, tw, tk;   // lane-path limits: successors, candidates per step, list length
  // per defender: successors whose list is still empty (null: not counted,
  // every predecessor of a changed position is pushed)
  uint32_t *missing;
};

// Energy-list descriptors (one u64 per position):
//   inline (bit 63 set): count in bits 60..62, energy i in bits [i*ib, i*ib+ib)
//          with ib = elements * energy_bits (12 for STANDARD: up to 5 energies)
//   arena  (bit 63 clear): arena offset in bits 24..62, count in bits 0..23
// Almost every list of the spectroscopy games fits inline, so reading a
// successor's list is one 8-byte load and writing a result needs no arena.
constexpr unsigned long long INLINE_BIT = 1ull << 63;
__device__ __forceinline__ unsigned long long mkdesc(unsigned long long off, uint32_t cnt) {
  return (off << 24) | (unsigned long long)cnt;
}
__device__ __forceinline__ bool dinl(unsigned long long d) { return (d >> 63) != 0ull; }
__device__ __forceinline__ uint32_t dcnt(unsigned long long d) {
  return dinl(d) ? (uint32_t)((d >> 60) & 7ull) : (uint32_t)(d & CNT_MASK);
}
__device__ __forceinline__ unsigned long long doff(unsigned long long d) { return (d >> 24) & ((1ull << 39) - 1ull); }
__device__ __forceinline__ unsigned long long inl_hdr(uint32_t n) { return INLINE_BIT | ((unsigned long long)n << 60); }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

#if GEQ_CHECKED
__device__ __noinline__ void report_bounds(Ctr *c, int line) {
  atomicOr(&c->error, DERR_BOUNDS);
  atomicMax(&c->err_line, (uint32_t)line);
  atomicExch(&c->halt, 1u);
}
#define CHECK_IDX(c, idx, size) \
  (((unsigned long long)(idx) < (unsigned long long)(size)) ? true : (report_bounds((c), __LINE__), false))
#else
#define CHECK_IDX(c, idx, size) true
#endif

// Guarded loads: in the checked build an out-of-range index records an
// error and reads 0 instead of touching memory.
template <class T>
__device__ __forceinline__ T ld(const T *a, unsigned long long i, unsigned long long n, Ctr *c) {
  return CHECK_IDX(c, i, n) ? a[i] : T(0);
}

// Energy q of the list behind descriptor d.
__device__ __forceinline__ uint32_t lelem(unsigned long long d, uint32_t q, const uint32_t *arena,
                                          unsigned long long cap, Ctr *c, uint32_t ib, uint32_t ibm) {
  return dinl(d) ? ((uint32_t)(d >> (q * ib)) & ibm) : ld(arena, doff(d) + q, cap, c);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}

// ---- per-warp arena allocator ------------------------------------------
struct WarpAlloc {
  unsigned long long cur, end;
  // Reserve `cnt` energies.  Lane-uniform.  false on arena overflow.
  __device__ __forceinline__ bool alloc(uint32_t cnt, Ctr *c, unsigned long long cap, uint32_t lane,
                                        unsigned long long &out) {
    if (cur + cnt > end) {
      unsigned long long grab = cnt > ALLOC_CHUNK ? cnt : ALLOC_CHUNK;
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&c->arena_top, grab);
      base = __shfl_sync(FULL, base, 0);
      if (base + grab > cap) {
        if (lane == 0) atomicExch(&c->overflow, 1u);
        cur = end = 0;
        return false;
      }
      cur = base;
      end = base + grab;
    }
    out = cur;
    cur += cnt;
    return true;
  }
};

// ---- bitmap up-set algebra over {0..3}^6 (CodecStd) ----------------------
// A 4096-bit set indexed by the packed energy is spread over the warp: lane l
// holds bits [128l, 128l+128) as w0 (low 64) and w1.  Element i of the
// energy is bits [2i, 2i+2) of the index, so dims 0-2 move bits inside a
// word, dim 3 moves between w0/w1 and between lane pairs, dims 4-5 move
// between lanes.
struct BM {
  unsigned long long w0, w1;
};
__device__ __forceinline__ unsigned long long cl012(unsigned long long x) {
  x |= (x & 0x7777777777777777ull) << 1;
  x |= (x & 0x3333333333333333ull) << 2;
  x |= (x & 0x0FFF0FFF0FFF0FFFull) << 4;
  x |= (x & 0x00FF00FF00FF00FFull) << 8;
  x |= (x & 0x0000FFFFFFFFFFFFull) << 16;
  x |= (x & 0x00000000FFFFFFFFull) << 32;
  return x;
}
// Upward closure: every energy >= some member.
__device__ __forceinline__ BM up_closure(BM b, uint32_t lane) {
  b.w0 = cl012(b.w0);
  b.w1 = cl012(b.w1);
  b.w1 |= b.w0;
  unsigned long long t = __shfl_up_sync(FULL, b.w1, 1);
  if (lane & 1u) { b.w0 |= t; b.w1 |= t; }
  const uint32_t v4 = (lane >> 1) & 3u, v5 = (lane >> 3) & 3u;
  unsigned long long t0 = __shfl_up_sync(FULL, b.w0, 2), t1 = __shfl_up_sync(FULL, b.w1, 2);
  if (v4 >= 1u) { b.w0 |= t0; b.w1 |= t1; }
  t0 = __shfl_up_sync(FULL, b.w0, 4);
  t1 = __shfl_up_sync(FULL, b.w1, 4);
  if (v4 >= 2u) { b.w0 |= t0; b.w1 |= t1; }
  t0 = __shfl_up_sync(FULL, b.w0, 8);
  t1 = __shfl_up_sync(FULL, b.w1, 8);
  if (v5 >= 1u) { b.w0 |= t0; b.w1 |= t1; }
  t0 = __shfl_up_sync(FULL, b.w0, 16);
  t1 = __shfl_up_sync(FULL, b.w1, 16);
  if (v5 >= 2u) { b.w0 |= t0; b.w1 |= t1; }
  return b;
}
__device__ __forceinline__ unsigned long long st012(unsigned long long x) {
  return ((x & 0x7777777777777777ull) << 1) | ((x & 0x0FFF0FFF0FFF0FFFull) << 4) |
         ((x & 0x0000FFFFFFFFFFFFull) << 16);
}
// One step up in any single element: {e + unit_i}.
__device__ __forceinline__ BM step_up(BM b, uint32_t lane) {
  BM s;
  s.w0 = st012(b.w0);
  s.w1 = st012(b.w1) | b.w0;
  unsigned long long t = __shfl_up_sync(FULL, b.w1, 1);
  if (lane & 1u) s.w0 |= t;
  const uint32_t v4 = (lane >> 1) & 3u, v5 = (lane >> 3) & 3u;
  unsigned long long t0 = __shfl_up_sync(FULL, b.w0, 2), t1 = __shfl_up_sync(FULL, b.w1, 2);
  if (v4 >= 1u) { s.w0 |= t0; s.w1 |= t1; }
  t0 = __shfl_up_sync(FULL, b.w0, 8);
  t1 = __shfl_up_sync(FULL, b.w1, 8);
  if (v5 >= 1u) { s.w0 |= t0; s.w1 |= t1; }
  return s;
}
__device__ __forceinline__ BM bm_load(const uint32_t *sm, uint32_t lane) {
  BM b;
  b.w0 = (unsigned long long)sm[4 * lane] | ((unsigned long long)sm[4 * lane + 1] << 32);
  b.w1 = (unsigned long long)sm[4 * lane + 2] | ((unsigned long long)sm[4 * lane + 3] << 32);
  return b;
}
__device__ __forceinline__ void bm_set(uint32_t *sm, uint32_t idx) {
  idx &= 0xFFFu;
  atomicOr(&sm[idx >> 5], 1u << (idx & 31u));
}

template <class Cd>
__device__ __forceinline__ Cd make_codec(const KParams &p);
template <>
__device__ __forceinline__ CodecStd make_codec<CodecStd>(const KParams &) { return CodecStd{}; }
template <>
__device__ __forceinline__ CodecGen make_codec<CodecGen>(const KParams &p) {
  return CodecGen(p.el, p.mx, p.eb, p.em, p.ub, p.um);
}

enum : int { R_UNCHANGED = 0, R_CHANGED = 1, R_OVERFLOW = 2, R_SKIPPED = 3, R_ERROR = 4 };
struct Res {
  int st;
  unsigned long long d;  // the new descriptor when st == R_CHANGED
};

struct WarpCtx {
  const KParams &p;
  Ctr *c;
  uint32_t *arena;
  unsigned long long cap;
  uint32_t lane;
  uint32_t *sm;
  WarpAlloc &wa;
  unsigned long long &edges, &bytes;
  uint32_t *scr;  // this lane's scratch column (free while the warp routines run)
  __device__ __forceinline__ uint32_t elem(unsigned long long d, uint32_t q) const {
    return lelem(d, q, arena, cap, c, p.ib, p.ibm);
  }
};

// Successor of edge k: its update and list descriptor (lane-local).
// ---- antichains in lane-private shared-memory columns ----------------------
// blocks per SM of k_commit / k_fcount / k_ffill (each owns a slice of the
// frontier bitmap)
#ifndef GEQ_FRONTIER_BLOCKS_PER_SM
#define GEQ_FRONTIER_BLOCKS_PER_SM 8  // measured: 1 → 36.7 ms, 2 → 35.3, 4 → 34.5-34.7, 6 → 34.4, 8 → 34.1-34.3 per solve of the batch
#endif
// resident blocks per SM of k_round_big (its register budget and grid)
#ifndef GEQ_BIG_BLOCKS_PER_SM
#define GEQ_BIG_BLOCKS_PER_SM 4  // measured: 2 → 36.2 ms, 3 → 34.2, 4 → 33.5-33.7, 5 → 33.55 (with spills) per solve of the batch
#endif
#ifndef GEQ_LANE_TK
#define GEQ_LANE_TK 16
#endif
constexpr uint32_t TK = GEQ_LANE_TK;  // antichain members per column
constexpr uint32_t TD = 16;   // successors per lane
constexpr uint32_t TW = 64;   // candidates (attacker) / combinations per step (defender)
constexpr int TSCR = 2 * TK;  // scratch words per lane: two antichain columns
enum : int { T_NONE = 0, T_UNCHANGED = 1, T_CHANGED = 2, T_SKIPPED = 3, T_BIG = 4, T_OVERFLOW = 5 };

// scratch column of this lane: word i at scr[i * 32]
#define SCR(i) scr[(uint32_t)(i) * 32u]

// Insert thermometer code x into the antichain at column words [b, b+n).
// om bit k: member k equals an own energy (the attacker's tie rule keeps the
// own copy, the later one).  false if the antichain would exceed TK members.
__device__ __forceinline__ bool ac_insert(uint32_t *scr, uint32_t b, uint32_t &n, uint32_t &om, uint32_t x,
                                          bool own) {
  uint32_t j = 0, om2 = 0;
  for (uint32_t k = 0; k < n; k++) {
    const uint32_t a = SCR(b + k);
    if ((a & ~x) == 0u) {
      // a <= x: x is not minimal.  No member was removed before this one:
      // a member above x would be above a, and members form an antichain.
      if (own && a == x) om |= 1u << k;
      return true;
    }
    if ((x & ~a) != 0u) {  // a is not above x: keep it
      if (j != k) SCR(b + j) = a;
      om2 |= ((om >> k) & 1u) << j;
      j++;
    }
  }
  if (j >= TK) return false;
  SCR(b + j) = x;
  om = om2 | ((own ? 1u : 0u) << j);
  n = j + 1;
  return true;
}

struct EdgeInfo {
  uint32_t u, cw;
  unsigned long long d;
};
__device__ __forceinline__ EdgeInfo edge_info(const WarpCtx &x, unsigned long long k) {
  EdgeInfo e{0, 0, 0};
  const uint32_t w = ld(x.p.col, k, x.p.n_edges, x.c);
  e.u = ld(x.p.wt, k, x.p.n_edges, x.c);
  e.d = ld(x.p.desc, w, x.p.n_nodes, x.c);
  e.cw = dcnt(e.d);
  return e;
}
__device__ __forceinline__ EdgeInfo shfl_edge(const EdgeInfo &e, uint32_t src) {
  EdgeInfo r;
  r.u = __shfl_sync(FULL, e.u, src);
  r.cw = __shfl_sync(FULL, e.cw, src);
  r.d = __shfl_sync(FULL, e.d, src);
  return r;
}

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long x) {
  const uint32_t lo = __reduce_or_sync(FULL, (uint32_t)x), hi = __reduce_or_sync(FULL, (uint32_t)(x >> 32));
  return ((unsigned long long)hi << 32) | lo;
}

// Store a new list of `cnt` energies held one per lane (`val` at `rank` where
// `has`): inline when it fits, else in fresh arena space.
__device__ Res warp_store(const WarpCtx &x, uint32_t val, bool has, uint32_t rank, uint32_t cnt) {
  x.bytes += 4ull * cnt;
  if (cnt <= x.p.inl) {
    const unsigned long long part = has ? ((unsigned long long)val << (rank * x.p.ib)) : 0ull;
    return Res{R_CHANGED, inl_hdr(cnt) | warp_or64(part)};
  }
  unsigned long long off = 0;
  if (!x.wa.alloc(cnt, x.c, x.cap, x.lane, off)) return Res{R_OVERFLOW, 0};
  if (has && CHECK_IDX(x.c, off + rank, x.cap)) x.arena[off + rank] = val;
  return Res{R_CHANGED, mkdesc(off, cnt)};
}

// Store the members of bitmap `m` (ascending index order).
__device__ Res bm_store(const WarpCtx &x, BM m) {
  const uint32_t lane = x.lane;
  const uint32_t c = (uint32_t)(__popcll(m.w0) + __popcll(m.w1));
  const uint32_t incl = warp_incl_scan(c, lane);
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  uint32_t rank = incl - c;
  x.bytes += 4ull * total;
  if (total <= x.p.inl) {
    unsigned long long part = 0;
    for (unsigned long long w = m.w0; w; w &= w - 1ull, rank++)
      part |= (unsigned long long)(lane * 128u + (uint32_t)__ffsll((long long)w) - 1u) << (rank * x.p.ib);
    for (unsigned long long w = m.w1; w; w &= w - 1ull, rank++)
      part |= (unsigned long long)(lane * 128u + 64u + (uint32_t)__ffsll((long long)w) - 1u) << (rank * x.p.ib);
    return Res{R_CHANGED, inl_hdr(total) | warp_or64(part)};
  }
  unsigned long long off = 0;
  if (!x.wa.alloc(total, x.c, x.cap, lane, off)) return Res{R_OVERFLOW, 0};
  if (CHECK_IDX(x.c, off + total - 1, x.cap)) {
    unsigned long long k = off + rank;
    for (unsigned long long w = m.w0; w; w &= w - 1ull) x.arena[k++] = lane * 128u + (uint32_t)__ffsll((long long)w) - 1u;
    for (unsigned long long w = m.w1; w; w &= w - 1ull) x.arena[k++] = lane * 128u + 64u + (uint32_t)__ffsll((long long)w) - 1u;
  }
  return Res{R_CHANGED, mkdesc(off, total)};
}

// Store a list of `cnt` packed energies that sits in arena scratch at `src`.
__device__ Res scratch_store(const WarpCtx &x, unsigned long long src, uint32_t cnt) {
  if (cnt <= x.p.inl) {
    const uint32_t lane = x.lane;
    const uint32_t v = lane < cnt ? ld(x.arena, src + lane, x.cap, x.c) : 0u;
    return warp_store(x, v, lane < cnt, lane, cnt);
  }
  unsigned long long off = 0;
  if (!x.wa.alloc(cnt, x.c, x.cap, x.lane, off)) return Res{R_OVERFLOW, 0};
  for (uint32_t q = x.lane; q < cnt; q += 32u)
    if (CHECK_IDX(x.c, off + q, x.cap)) x.arena[off + q] = ld(x.arena, src + q, x.cap, x.c);
  x.bytes += 4ull * cnt;
  return Res{R_CHANGED, mkdesc(off, cnt)};
}

// ---- attacker (warp routines) ------------------------------------------------
// attack_update.wgsl:77-113 + attack_minimize.wgsl:69-122: candidates are
// the inverse-updated successor energies followed by the own energies; keep
// the minimal ones (on ties the later copy, so own energies win); the
// position changed iff a kept candidate came from a successor.
template <class Cd>
__device__ Res attack_small(const WarpCtx &x, const Cd &cd, unsigned long long e0, uint32_t d,
                            unsigned long long dv, bool &fits) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  EdgeInfo ei{0, 0, 0};
  if (lane < d) ei = edge_info(x, e0 + lane);
  const uint32_t incl = warp_incl_scan(ei.cw, lane);
  const uint32_t tot = __shfl_sync(FULL, incl, 31);
  const uint32_t K = tot + cv;
  if (K > x.p.small_limit) {
    fits = false;
    return Res{R_UNCHANGED, 0};
  }
  fits = true;
  x.bytes += 16ull * d + 4ull * tot;
  const uint32_t excl = incl - ei.cw;
  for (uint32_t k = excl; k < incl; k++) x.sm[SM_TMP + k] = lane;
  __syncwarp();
  const uint32_t i = lane;
  const uint32_t ed = (i < tot) ? x.sm[SM_TMP + i] : 0u;
  __syncwarp();
  const unsigned long long d_e = __shfl_sync(FULL, ei.d, ed);
  const uint32_t ex_e = __shfl_sync(FULL, excl, ed);
  const uint32_t u_e = __shfl_sync(FULL, ei.u, ed);
  const bool valid = i < K;
  uint32_t cnd = 0;
  if (i < tot) cnd = cd.upd(cd.to_t(x.elem(d_e, i - ex_e)), u_e);
  else if (valid) cnd = cd.to_t(x.elem(dv, i - tot));
  bool killed = false;
  for (uint32_t j = 0; j < K; j++) {
    const uint32_t cj = __shfl_sync(FULL, cnd, j);
    if (valid && j != i) {
      const bool eq = cj == cnd;
      if ((eq && i < j) || (!eq && t_leq(cj, cnd))) killed = true;
    }
  }
  const bool kept = valid && !killed;
  const uint32_t bal = __ballot_sync(FULL, kept);
  const bool changed = __ballot_sync(FULL, kept && i < tot) != 0u;
  if (!changed) return Res{R_UNCHANGED, 0};
  return warp_store(x, cd.to_p(cnd), kept, __popc(bal & lanemask_lt()), __popc(bal));
}

// Large attacker positions on STANDARD: candidates go into a 4096-bit set;
// minimal members = set minus the strict up-closure of the set.
__device__ __noinline__ Res attack_bitmap(const WarpCtx &x, const CodecStd &cd, unsigned long long e0, unsigned long long e1,
                             unsigned long long dv) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  for (uint32_t k = lane; k < 256u; k += 32u) x.sm[SM_BM + k] = 0u;
  __syncwarp();
  unsigned long long tot = 0;
  for (unsigned long long k0 = e0; k0 < e1; k0 += 32) {
    EdgeInfo ei{0, 0, 0};
    if (k0 + lane < e1) ei = edge_info(x, k0 + lane);
    const uint32_t nk = (uint32_t)min(32ull, e1 - k0);
    for (uint32_t j = 0; j < nk; j++) {
      const EdgeInfo e = shfl_edge(ei, j);
      tot += e.cw;
      for (uint32_t q = lane; q < e.cw; q += 32u) bm_set(x.sm + SM_BM, cd.to_p(cd.upd(cd.to_t(x.elem(e.d, q)), e.u)));
    }
  }
  x.bytes += 16ull * (e1 - e0) + 4ull * tot;
  for (uint32_t q = lane; q < cv; q += 32u) {
    const uint32_t idx = x.elem(dv, q);
    bm_set(x.sm + SM_BM, idx);
    bm_set(x.sm + SM_BM2, idx);
  }
  __syncwarp();
  const BM b = bm_load(x.sm + SM_BM, lane);
  const BM own = bm_load(x.sm + SM_BM2, lane);
  __syncwarp();
  const BM su = up_closure(step_up(b, lane), lane);
  BM m;
  m.w0 = b.w0 & ~su.w0;
  m.w1 = b.w1 & ~su.w1;
  const bool changed = __ballot_sync(FULL, ((m.w0 & ~own.w0) | (m.w1 & ~own.w1)) != 0ull) != 0u;
  if (!changed) return Res{R_UNCHANGED, 0};
  return bm_store(x, m);
}

// Large attacker positions on other confs: candidates in arena scratch,
// pairwise minimisation (same tie rule).
template <class Cd>
__device__ __noinline__ Res attack_list(const WarpCtx &x, const Cd &cd, unsigned long long e0, unsigned long long e1,
                           unsigned long long dv) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  unsigned long long K = cv;
  for (unsigned long long k0 = e0; k0 < e1; k0 += 32) {
    EdgeInfo ei{0, 0, 0};
    if (k0 + lane < e1) ei = edge_info(x, k0 + lane);
    const uint32_t incl = warp_incl_scan(ei.cw, lane);
    K += __shfl_sync(FULL, incl, 31);
  }
  if (K > CNT_MASK) {
    if (lane == 0) { atomicOr(&x.c->error, DERR_SCRATCH); atomicExch(&x.c->halt, 1u); }
    return Res{R_ERROR, 0};
  }
  unsigned long long sc = 0;
  if (!x.wa.alloc((uint32_t)K, x.c, x.cap, lane, sc)) return Res{R_OVERFLOW, 0};
  unsigned long long pos = 0;
  for (unsigned long long k0 = e0; k0 < e1; k0 += 32) {
    EdgeInfo ei{0, 0, 0};
    if (k0 + lane < e1) ei = edge_info(x, k0 + lane);
    const uint32_t nk = (uint32_t)min(32ull, e1 - k0);
    for (uint32_t j = 0; j < nk; j++) {
      const EdgeInfo e = shfl_edge(ei, j);
      for (uint32_t q = lane; q < e.cw; q += 32u)
        if (CHECK_IDX(x.c, sc + pos + q, x.cap)) x.arena[sc + pos + q] = cd.upd(cd.to_t(x.elem(e.d, q)), e.u);
      pos += e.cw;
    }
  }
  x.bytes += 16ull * (e1 - e0) + 4ull * pos;
  const unsigned long long tot = pos;
  for (uint32_t q = lane; q < cv; q += 32u)
    if (CHECK_IDX(x.c, sc + tot + q, x.cap)) x.arena[sc + tot + q] = cd.to_t(x.elem(dv, q));
  __syncwarp();
  unsigned long long out = 0;
  if (!x.wa.alloc((uint32_t)K, x.c, x.cap, lane, out)) return Res{R_OVERFLOW, 0};
  uint32_t cnt = 0;
  bool changed = false;
  for (unsigned long long i0 = 0; i0 < K; i0 += 32) {
    const unsigned long long i = i0 + lane;
    bool kept = false;
    uint32_t ci = 0;
    if (i < K) {
      ci = ld(x.arena, sc + i, x.cap, x.c);
      kept = true;
      for (unsigned long long j = 0; j < K; j++) {
        if (j == i) continue;
        const uint32_t cj = ld(x.arena, sc + j, x.cap, x.c);
        const bool eq = cj == ci;
        if ((eq && i < j) || (!eq && t_leq(cj, ci))) { kept = false; break; }
      }
    }
    const uint32_t bal = __ballot_sync(FULL, kept);
    if (__ballot_sync(FULL, kept && i < tot)) changed = true;
    if (kept) {
      const unsigned long long k = out + cnt + __popc(bal & lanemask_lt());
      if (CHECK_IDX(x.c, k, x.cap)) x.arena[k] = cd.to_p(ci);
    }
    cnt += __popc(bal);
  }
  __syncwarp();
  if (!changed) return Res{R_UNCHANGED, 0};
  return scratch_store(x, out, cnt);
}

// ---- defender (warp routines) --------------------------------------------------
// Reference semantics (energygame.rs:896-944 with defend_iterative.wgsl):
// the new list is min{ a_1 v ... v a_d : a_k in upd_k(A_{w_k}) } (the first
// successor's updated list is taken as is when there is only one successor);
// the position changed iff the new list is not equal to the old one under
// EnergyArray's PartialEq (energy.rs:334-350: same length and every new
// energy occurs in the old list).

// changed-test for a new list held in lanes (n <= 32) against the old list.
__device__ bool differs_small(const WarpCtx &x, uint32_t newp, uint32_t n, unsigned long long dv) {
  const uint32_t cv = dcnt(dv);
  if (n != cv) return true;
  const uint32_t lane = x.lane;
  const uint32_t o = (lane < cv) ? x.elem(dv, lane) : 0u;
  bool found = false;
  for (uint32_t j = 0; j < cv; j++) found |= (__shfl_sync(FULL, o, j) == newp);
  return __ballot_sync(FULL, lane < n && !found) != 0u;
}

template <class Cd>
__device__ Res defend_single(const WarpCtx &x, const Cd &cd, const EdgeInfo &e, unsigned long long dv) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  const uint32_t n = e.cw;
  x.bytes += 16ull + 4ull * n;
  bool changed;
  if (n != cv) {
    changed = true;
  } else if (n <= 32u) {
    const uint32_t np = (lane < n) ? cd.to_p(cd.upd(cd.to_t(x.elem(e.d, lane)), e.u)) : 0u;
    changed = differs_small(x, np, n, dv);
  } else if (Cd::kBitmap) {
    for (uint32_t k = lane; k < 128u; k += 32u) x.sm[SM_BM2 + k] = 0u;
    __syncwarp();
    for (uint32_t q = lane; q < cv; q += 32u) bm_set(x.sm + SM_BM2, x.elem(dv, q));
    __syncwarp();
    bool miss = false;
    for (uint32_t q = lane; q < n; q += 32u) {
      const uint32_t idx = cd.to_p(cd.upd(cd.to_t(x.elem(e.d, q)), e.u)) & 0xFFFu;
      miss |= ((x.sm[SM_BM2 + (idx >> 5)] >> (idx & 31u)) & 1u) == 0u;
    }
    changed = __ballot_sync(FULL, miss) != 0u;
    __syncwarp();
  } else {
    bool miss = false;
    for (uint32_t q = lane; q < n; q += 32u) {
      const uint32_t np = cd.to_p(cd.upd(cd.to_t(x.elem(e.d, q)), e.u));
      bool found = false;
      for (uint32_t j = 0; j < cv && !found; j++) found = x.elem(dv, j) == np;
      miss |= !found;
    }
    changed = __ballot_sync(FULL, miss) != 0u;
  }
  if (!changed) return Res{R_UNCHANGED, 0};
  if (n <= 32u)
    return warp_store(x, lane < n ? cd.to_p(cd.upd(cd.to_t(x.elem(e.d, lane)), e.u)) : 0u, lane < n, lane, n);
  unsigned long long off = 0;
  if (!x.wa.alloc(n, x.c, x.cap, lane, off)) return Res{R_OVERFLOW, 0};
  for (uint32_t q = lane; q < n; q += 32u)
    if (CHECK_IDX(x.c, off + q, x.cap)) x.arena[off + q] = cd.to_p(cd.upd(cd.to_t(x.elem(e.d, q)), e.u));
  x.bytes += 4ull * n;
  return Res{R_CHANGED, mkdesc(off, n)};
}

// Fold of up to 32 successors whose pairwise combinations stay <= 32: the
// running antichain lives in one register per lane.
template <class Cd>
__device__ __noinline__ Res defend_small(const WarpCtx &x, const Cd &cd, unsigned long long e0, uint32_t d,
                            unsigned long long dv, bool &fits) {
  const uint32_t lane = x.lane;
  EdgeInfo ei{0, 0, 0};
  if (lane < d) ei = edge_info(x, e0 + lane);
  uint32_t s = __shfl_sync(FULL, ei.cw, 0);
  fits = false;
  if (s > x.p.small_limit) return Res{R_UNCHANGED, 0};
  const EdgeInfo e0i = shfl_edge(ei, 0);
  uint32_t S = (lane < s) ? cd.upd(cd.to_t(x.elem(e0i.d, lane)), e0i.u) : 0u;
  for (uint32_t k = 1; k < d; k++) {
    const EdgeInfo b = shfl_edge(ei, k);
    const uint32_t combos = s * b.cw;
    if (combos > x.p.small_limit) return Res{R_UNCHANGED, 0};  // fits stays false
    const uint32_t l = lane;
    const bool valid = l < combos;
    const uint32_t a = __shfl_sync(FULL, S, valid ? (l % s) : 0u);
    uint32_t cc = 0;
    if (valid) cc = a | cd.upd(cd.to_t(x.elem(b.d, l / s)), b.u);
    bool killed = false;
    for (uint32_t j = 0; j < combos; j++) {
      const uint32_t cj = __shfl_sync(FULL, cc, j);
      if (valid && j != l) {
        const bool eq = cj == cc;
        if ((eq && l > j) || (!eq && t_leq(cj, cc))) killed = true;
      }
    }
    const bool kept = valid && !killed;
    const uint32_t bal = __ballot_sync(FULL, kept);
    if (kept) x.sm[SM_TMP + __popc(bal & lanemask_lt())] = cc;
    __syncwarp();
    s = __popc(bal);
    S = (lane < s) ? x.sm[SM_TMP + lane] : 0u;
    __syncwarp();
  }
  fits = true;
  unsigned long long tot = (lane < d) ? ei.cw : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(FULL, tot, o);
  x.bytes += 16ull * d + 4ull * tot;
  const uint32_t np = (lane < s) ? cd.to_p(S) : 0u;
  if (!differs_small(x, np, s, dv)) return Res{R_UNCHANGED, 0};
  return warp_store(x, np, lane < s, lane, s);
}

// Defender fold across the warp: lane l folds the updated lists of
// successors l, l+32, ... into an antichain in its scratch column, then the
// lanes' antichains are combined pairwise in five steps.  The suprema fold
// is associative and commutative once minimised, so the result is the set of
// minimal suprema of the reference's sequential fold.  fits = false when an
// antichain outgrows TK members or one combination step TW pairs.
template <class Cd>
__device__ Res defend_tree(const WarpCtx &x, const Cd &cd, unsigned long long e0, unsigned long long e1,
                           unsigned long long dv, bool &fits, bool &empty) {
  const uint32_t lane = x.lane;
  uint32_t *scr = x.scr;
  uint32_t n = 0, om = 0, tot = 0;
  bool ok = true, first = true, emp = false;
  for (unsigned long long k = e0 + lane; k < e1; k += 32) {
    const EdgeInfo e = edge_info(x, k);
    tot += e.cw;
    emp |= e.cw == 0u;
    if (!ok) continue;
    const auto pu = cd.prep(e.u);
    if (first) {
      for (uint32_t q = 0; q < e.cw && ok; q++) ok = ac_insert(scr, 0, n, om, cd.apply(cd.to_t(x.elem(e.d, q)), pu), false);
      first = false;
    } else if (n * e.cw > TW) {
      ok = false;
    } else {
      uint32_t nn = 0;
      for (uint32_t q = 0; q < e.cw && ok; q++) {
        const uint32_t bq = cd.apply(cd.to_t(x.elem(e.d, q)), pu);
        for (uint32_t i = 0; i < n && ok; i++) ok = ac_insert(scr, TK, nn, om, SCR(i) | bq, false);
      }
      for (uint32_t q = 0; q < nn && ok; q++) SCR(q) = SCR(TK + q);
      n = nn;
    }
  }
  fits = false;
  // skipped while a successor has no energies (energygame.rs:789-792)
  empty = __any_sync(FULL, emp);
  if (empty) return Res{R_SKIPPED, 0};
  if (__any_sync(FULL, !ok)) return Res{R_UNCHANGED, 0};
  const uint32_t dl = (uint32_t)min(32ull, e1 - e0);
  for (uint32_t st = 1; st < dl; st <<= 1) {
    __syncwarp();
    const uint32_t np = __shfl_down_sync(FULL, n, st);
    if ((lane & (2u * st - 1u)) == 0u && lane + st < dl) {
      if (n * np > TW) {
        ok = false;
      } else {
        uint32_t nn = 0;
        for (uint32_t j = 0; j < np && ok; j++) {
          const uint32_t b = scr[st + j * 32u];  // partner lane's column
          for (uint32_t i = 0; i < n && ok; i++) ok = ac_insert(scr, TK, nn, om, SCR(i) | b, false);
        }
        for (uint32_t q = 0; q < nn && ok; q++) SCR(q) = SCR(TK + q);
        n = nn;
      }
    }
    if (__any_sync(FULL, !ok)) return Res{R_UNCHANGED, 0};
  }
  __syncwarp();
  fits = true;
  x.bytes += 16ull * (e1 - e0) + 4ull * __reduce_add_sync(FULL, tot);
  const uint32_t r = __shfl_sync(FULL, n, 0);
  const uint32_t np = lane < r ? cd.to_p((scr - lane)[lane * 32u]) : 0u;  // word `lane` of lane 0's column
  __syncwarp();
  if (!differs_small(x, np, r, dv)) return Res{R_UNCHANGED, 0};
  return warp_store(x, np, lane < r, lane, r);
}

// STANDARD defender with large lists: intersect the up-closures of the
// updated successor lists in a 4096-bit set, then take its minimal members.
__device__ __noinline__ Res defend_bitmap(const WarpCtx &x, const CodecStd &cd, unsigned long long e0, unsigned long long e1,
                             unsigned long long dv) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  BM acc;
  acc.w0 = ~0ull;
  acc.w1 = ~0ull;
  unsigned long long tot = 0;
  for (unsigned long long k0 = e0; k0 < e1; k0 += 32) {
    EdgeInfo ei{0, 0, 0};
    if (k0 + lane < e1) ei = edge_info(x, k0 + lane);
    const uint32_t nk = (uint32_t)min(32ull, e1 - k0);
    for (uint32_t j = 0; j < nk; j++) {
      const EdgeInfo e = shfl_edge(ei, j);
      tot += e.cw;
      for (uint32_t k = lane; k < 128u; k += 32u) x.sm[SM_BM + k] = 0u;
      __syncwarp();
      for (uint32_t q = lane; q < e.cw; q += 32u) bm_set(x.sm + SM_BM, cd.to_p(cd.upd(cd.to_t(x.elem(e.d, q)), e.u)));
      __syncwarp();
      const BM u = up_closure(bm_load(x.sm + SM_BM, lane), lane);
      __syncwarp();
      acc.w0 &= u.w0;
      acc.w1 &= u.w1;
    }
  }
  x.bytes += 16ull * (e1 - e0) + 4ull * tot;
  const BM st = step_up(acc, lane);
  BM m;
  m.w0 = acc.w0 & ~st.w0;
  m.w1 = acc.w1 & ~st.w1;
  for (uint32_t k = lane; k < 128u; k += 32u) x.sm[SM_BM2 + k] = 0u;
  __syncwarp();
  for (uint32_t q = lane; q < cv; q += 32u) bm_set(x.sm + SM_BM2, x.elem(dv, q));
  __syncwarp();
  const BM old = bm_load(x.sm + SM_BM2, lane);
  __syncwarp();
  const uint32_t total = (uint32_t)__reduce_add_sync(FULL, (uint32_t)(__popcll(m.w0) + __popcll(m.w1)));
  const bool changed =
      total != cv || __ballot_sync(FULL, ((m.w0 & ~old.w0) | (m.w1 & ~old.w1)) != 0ull) != 0u;
  if (!changed) return Res{R_UNCHANGED, 0};
  return bm_store(x, m);
}

// Other confs with large lists: the fold of defend_iterative.wgsl with the
// running list and the combinations in arena scratch.
template <class Cd>
__device__ __noinline__ Res defend_list(const WarpCtx &x, const Cd &cd, unsigned long long e0, unsigned long long e1,
                           unsigned long long dv) {
  const uint32_t lane = x.lane;
  const uint32_t cv = dcnt(dv);
  EdgeInfo f{0, 0, 0};
  if (lane == 0) f = edge_info(x, e0);
  f = shfl_edge(f, 0);
  unsigned long long S = 0;
  uint32_t s = f.cw;
  if (!x.wa.alloc(s, x.c, x.cap, lane, S)) return Res{R_OVERFLOW, 0};
  for (uint32_t q = lane; q < s; q += 32u)
    if (CHECK_IDX(x.c, S + q, x.cap)) x.arena[S + q] = cd.upd(cd.to_t(x.elem(f.d, q)), f.u);
  unsigned long long tot = s;
  __syncwarp();
  for (unsigned long long k = e0 + 1; k < e1; k++) {
    EdgeInfo b{0, 0, 0};
    if (lane == 0) b = edge_info(x, k);
    b = shfl_edge(b, 0);
    tot += b.cw;
    const unsigned long long combos = (unsigned long long)s * b.cw;
    if (combos > (1ull << 22)) {
      if (lane == 0) { atomicOr(&x.c->error, DERR_SCRATCH); atomicExch(&x.c->halt, 1u); }
      return Res{R_ERROR, 0};
    }
    unsigned long long C = 0, N = 0;
    if (!x.wa.alloc((uint32_t)combos, x.c, x.cap, lane, C)) return Res{R_OVERFLOW, 0};
    if (!x.wa.alloc((uint32_t)combos, x.c, x.cap, lane, N)) return Res{R_OVERFLOW, 0};
    for (unsigned long long l = lane; l < combos; l += 32)
      if (CHECK_IDX(x.c, C + l, x.cap))
        x.arena[C + l] = ld(x.arena, S + l % s, x.cap, x.c) | cd.upd(cd.to_t(x.elem(b.d, (uint32_t)(l / s))), b.u);
    __syncwarp();
    uint32_t cnt = 0;
    for (unsigned long long l0 = 0; l0 < combos; l0 += 32) {
      const unsigned long long l = l0 + lane;
      bool kept = false;
      uint32_t cl = 0;
      if (l < combos) {
        cl = ld(x.arena, C + l, x.cap, x.c);
        kept = true;
        for (unsigned long long j = 0; j < combos; j++) {
          if (j == l) continue;
          const uint32_t cj = ld(x.arena, C + j, x.cap, x.c);
          const bool eq = cj == cl;
          if ((eq && l > j) || (!eq && t_leq(cj, cl))) { kept = false; break; }
        }
      }
      const uint32_t bal = __ballot_sync(FULL, kept);
      if (kept) {
        const unsigned long long kk = N + cnt + __popc(bal & lanemask_lt());
        if (CHECK_IDX(x.c, kk, x.cap)) x.arena[kk] = cl;
      }
      cnt += __popc(bal);
    }
    __syncwarp();
    S = N;
    s = cnt;
  }
  x.bytes += 16ull * (e1 - e0) + 4ull * tot;
  // packed copies for the comparison and the store
  for (uint32_t q = lane; q < s; q += 32u)
    if (CHECK_IDX(x.c, S + q, x.cap)) x.arena[S + q] = cd.to_p(ld(x.arena, S + q, x.cap, x.c));
  __syncwarp();
  bool changed = s != cv;
  if (!changed) {
    bool miss = false;
    for (uint32_t q = lane; q < s; q += 32u) {
      const uint32_t np = ld(x.arena, S + q, x.cap, x.c);
      bool found = false;
      for (uint32_t j = 0; j < cv && !found; j++) found = x.elem(dv, j) == np;
      miss |= !found;
    }
    changed = __ballot_sync(FULL, miss) != 0u;
  }
  if (!changed) return Res{R_UNCHANGED, 0};
  return scratch_store(x, S, s);
}

template <class Cd>
__device__ Res solve_position(const WarpCtx &x, const Cd &cd, uint32_t v) {
  const uint32_t lane = x.lane;
  const unsigned long long e0 = ld(x.p.row, v, x.p.n_nodes + 1, x.c);
  const unsigned long long e1 = ld(x.p.row, (unsigned long long)v + 1, x.p.n_nodes + 1, x.c);
  const uint32_t d = (uint32_t)(e1 - e0);
  const unsigned long long dv = ld(x.p.desc, v, x.p.n_nodes, x.c);
  const bool attacker = ld(x.p.flags, v, x.p.n_nodes, x.c) & 1u;
  if (d == 0) return Res{R_SKIPPED, 0};
#if GEQ_PATH_PROFILE
  const long long t0 = clock64();
#endif
  if (attacker) {
    x.edges += d;
    x.bytes += 12ull + 4ull * dcnt(dv);
    if (d <= 32u && x.p.small_limit > 0) {
      bool fits = false;
      const Res r = attack_small(x, cd, e0, d, dv, fits);
      if (fits) { PROF_WARP(x.c, PF_AS_N, t0); return r; }
    }
    if constexpr (Cd::kBitmap) { const Res r = attack_bitmap(x, cd, e0, e1, dv); PROF_WARP(x.c, PF_AB_N, t0); return r; }
    else return attack_list(x, cd, e0, e1, dv);
  }
  if (d >= 2u && x.p.small_limit > 0) {
    // the tree fold reads every successor's list and sees the empty ones
    bool fits = false, emp = false;
    const Res r = defend_tree(x, cd, e0, e1, dv, fits, emp);
    if (emp) { PROF_WARP(x.c, PF_DK_N, t0); return Res{R_SKIPPED, 0}; }
    if (fits) {
      x.edges += d;
      x.bytes += 12ull;
      PROF_WARP(x.c, PF_DT_N, t0);
      return r;
    }
  }
  // defender: skipped while a successor has no energies (energygame.rs:789-792)
  bool empty = false;
  for (unsigned long long k0 = e0; k0 < e1; k0 += 32) {
    bool e = false;
    if (k0 + lane < e1) {
      const uint32_t w = ld(x.p.col, k0 + lane, x.p.n_edges, x.c);
      e = dcnt(ld(x.p.desc, w, x.p.n_nodes, x.c)) == 0u;
    }
    if (__ballot_sync(FULL, e)) { empty = true; break; }
  }
  if (empty) { PROF_WARP(x.c, PF_DK_N, t0); return Res{R_SKIPPED, 0}; }
  x.edges += d;
  x.bytes += 12ull;
  if (d == 1u) {
    EdgeInfo e{0, 0, 0};
    if (lane == 0) e = edge_info(x, e0);
    const Res r = defend_single(x, cd, shfl_edge(e, 0), dv);
    PROF_WARP(x.c, PF_D1_N, t0);
    return r;
  }
  if (d <= 32u && x.p.small_limit > 0) {
    bool fits = false;
    const Res r = defend_small(x, cd, e0, d, dv, fits);
    if (fits) { PROF_WARP(x.c, PF_DS_N, t0); return r; }
  }
  if constexpr (Cd::kBitmap) { const Res r = defend_bitmap(x, cd, e0, e1, dv); PROF_WARP(x.c, PF_DB_N, t0); return r; }
  else return defend_list(x, cd, e0, e1, dv);
}

// ---- thread path: one lane per small position -----------------------------
// Successor and update of edge k: one 8-byte load of the edge pair, or the
// col / wt arrays where there are none (the one-block solver).
__device__ __forceinline__ void load_edge(const KParams &p, Ctr *c, unsigned long long k, uint32_t &w, uint32_t &u) {
  if (p.cw) {
    const unsigned long long e = ld(p.cw, k, p.n_edges, c);
    w = (uint32_t)e;
    u = (uint32_t)(e >> 32);
  } else {
    w = ld(p.col, k, p.n_edges, c);
    u = ld(p.wt, k, p.n_edges, c);
  }
}
// up to four consecutive edges k0 .. k0+min(left,4)-1
__device__ __forceinline__ void load_edges4(const KParams &p, Ctr *c, unsigned long long k0, uint32_t left,
                                            uint32_t (&w)[4], uint32_t (&u)[4]) {
#pragma unroll
  for (int t = 0; t < 4; t++)
    if ((uint32_t)t < left) load_edge(p, c, k0 + t, w[t], u[t]);
}
template <class Cd>
__device__ __forceinline__ typename Cd::Upd edge_upd(const KParams &p, const Cd &cd, uint32_t u) {
  return p.cw ? cd.unpack_edge(u) : cd.prep(u);
}

// Most positions have a handful of successors with one or two energies each.
// Every lane of a warp solves its own such position.  Candidates stream into
// an antichain held in a lane-private column of shared memory (bank = lane):
// a candidate is dropped when a member lies below or equals it, and removes
// the members above it.  What remains is the set of minimal candidates
// whatever the insertion order, so the lists equal the reference's as sets
// (the order inside a list may differ).  Positions beyond TD successors, TK
// members or TW candidates (per defender step: combinations) go to the warp
// routines.
template <class Cd>
__device__ int thread_solve(const KParams &p, Ctr *c, const Cd &cd, const uint32_t *arena, unsigned long long cap,
                            uint32_t v, uint32_t *scr, uint32_t &out_cnt, uint32_t &edges, uint32_t &bytes,
                            uint32_t &old_cnt) {
  const uint32_t e0 = ld(p.row, v, p.n_nodes + 1, c), e1 = ld(p.row, (unsigned long long)v + 1, p.n_nodes + 1, c);
  const uint32_t d = e1 - e0;
  if (d == 0) return T_SKIPPED;
  if (d > p.td) return T_BIG;
  const unsigned long long dv = ld(p.desc, v, p.n_nodes, c);
  const uint32_t cv = dcnt(dv);
  old_cnt = cv;
  const bool attacker = ld(p.flags, v, p.n_nodes, c) & 1u;
  if (attacker) {
    // attack_update.wgsl + attack_minimize.wgsl: successor candidates, then
    // the own energies; changed iff a minimal value has no own copy
    if (cv > p.tk) return T_BIG;
    // the own energies first (the old minimal set, all flagged own): in the
    // common case that nothing changes, every successor candidate then meets
    // a member below it at once.  The minimal set is the same in any order;
    // a candidate equal to an own member is dropped, so the own copy stays
    // (the later copy wins, attack_minimize.wgsl:84-92).
    uint32_t n = 0, om = 0, tot = 0;
    for (uint32_t q = 0; q < cv; q++)
      if (!ac_insert(scr, 0, n, om, cd.to_t(lelem(dv, q, arena, cap, c, p.ib, p.ibm)), true)) return T_BIG;
    for (uint32_t j0 = 0; j0 < d; j0 += 4) {
      uint32_t w[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
      unsigned long long dw[4] = {0, 0, 0, 0};
      load_edges4(p, c, e0 + j0, d - j0, w, u);
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (j0 + t < d) dw[t] = ld(p.desc, w[t], p.n_nodes, c);
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (j0 + t < d) {
          const uint32_t cw = dcnt(dw[t]);
          tot += cw;
          if (tot > p.tw) return T_BIG;
          const auto pu = edge_upd(p, cd, u[t]);
          for (uint32_t q = 0; q < cw; q++)
            if (!ac_insert(scr, 0, n, om, cd.apply(cd.to_t(lelem(dw[t], q, arena, cap, c, p.ib, p.ibm)), pu), false))
              return T_BIG;
        }
    }
    edges += d;
    bytes += 12u + 4u * cv + 16u * d + 4u * tot;
    if (om == (1u << n) - 1u) return T_UNCHANGED;
    for (uint32_t q = 0; q < n; q++) SCR(TK + q) = cd.to_p(SCR(q));
    out_cnt = n;
    return T_CHANGED;
  }
  // defender: skipped while a successor has no energies
  // (energygame.rs:789-792); successors read four at a time, each group
  // checked for an empty list before it is folded in.  d == 1: the
  // successor's updated list as is (defend_iterative.wgsl:200-211); else the
  // fold of pairwise suprema, minimised after every step
  // (defend_iterative.wgsl:215-262) -- the first list minimised too, which
  // leaves the minimal suprema unchanged.
  uint32_t n = 0;
  {
    uint32_t sb = 0, nb = TK, ns = 0, om = 0;
    unsigned long long tot = 0;
    for (uint32_t j0 = 0; j0 < d; j0 += 4) {
      uint32_t w[4] = {0, 0, 0, 0}, u[4] = {0, 0, 0, 0};
      unsigned long long dw[4] = {0, 0, 0, 0};
      load_edges4(p, c, e0 + j0, d - j0, w, u);
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (j0 + t < d) dw[t] = ld(p.desc, w[t], p.n_nodes, c);
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (j0 + t < d && dcnt(dw[t]) == 0u) return T_SKIPPED;
#pragma unroll
      for (int t = 0; t < 4; t++) {
        if (j0 + t >= d) continue;
        const uint32_t cb = dcnt(dw[t]);
        tot += cb;
        const auto pu = edge_upd(p, cd, u[t]);
        if (j0 + t == 0) {
          if (d == 1) {
            if (cb > p.tk) return T_BIG;
            for (uint32_t q = 0; q < cb; q++)
              SCR(TK + q) = cd.to_p(cd.apply(cd.to_t(lelem(dw[t], q, arena, cap, c, p.ib, p.ibm)), pu));
            n = cb;
          } else {
            if (cb > p.tw) return T_BIG;
            for (uint32_t q = 0; q < cb; q++)
              if (!ac_insert(scr, sb, ns, om, cd.apply(cd.to_t(lelem(dw[t], q, arena, cap, c, p.ib, p.ibm)), pu),
                             false))
                return T_BIG;
          }
          continue;
        }
        if (ns * cb > p.tw) return T_BIG;
        uint32_t nn = 0;
        for (uint32_t q = 0; q < cb; q++) {
          const uint32_t bq = cd.apply(cd.to_t(lelem(dw[t], q, arena, cap, c, p.ib, p.ibm)), pu);
          for (uint32_t k = 0; k < ns; k++)
            if (!ac_insert(scr, nb, nn, om, SCR(sb + k) | bq, false)) return T_BIG;
        }
        const uint32_t tmp = sb;
        sb = nb;
        nb = tmp;
        ns = nn;
      }
    }
    if (d > 1) {
      for (uint32_t q = 0; q < ns; q++) SCR(TK + q) = cd.to_p(SCR(sb + q));
      n = ns;
    }
    edges += d;
    bytes += 12u + 16u * d + 4u * (uint32_t)tot;
  }
  // EnergyArray PartialEq (energy.rs:334-350) against the old list
  bool changed = n != cv;
  for (uint32_t i = 0; i < n && !changed; i++) {
    const uint32_t x = SCR(TK + i);
    bool found = false;
    for (uint32_t j = 0; j < cv && !found; j++) found = lelem(dv, j, arena, cap, c, p.ib, p.ibm) == x;
    changed = !found;
  }
  if (!changed) return T_UNCHANGED;
  out_cnt = n;
  return T_CHANGED;
}

// The next frontier is a bitmap: one bit per position in each of two halves
// of `mark`, chosen by the parity of the stamp of the round that pushes.
// After the round k_commit counts the half's bits per block and clears the
// half that the round after next uses, and k_ffill turns the half into the
// frontier list in position order.  The bitmap (N/16 bytes) stays in L2.
__device__ __forceinline__ void mark_push(const KParams &p, uint32_t u, uint32_t stamp) {
  atomicOr(p.mark + (stamp & 1u) * p.mwords + (u >> 5), 1u << (u & 31u));
}

// Push predecessor u of a changed position.  A defender is computed only once
// every successor has energies (energygame.rs:789-792), so with `missing`
// counted it is pushed only then: the change that fills its last empty
// successor (`first`: the changed list was empty before) pushes it, and later
// changes push it as any predecessor.  The reference visits it and skips it
// meanwhile; the lists are the same.
__device__ __forceinline__ void push_one(const KParams &p, uint32_t u, uint32_t stamp, uint32_t first) {
  if (p.missing && !((p.abits[u >> 5] >> (u & 31u)) & 1u)) {
    if (first) {
      if (atomicSub(&p.missing[u], 1u) != 1u) return;
    } else if (*(volatile const uint32_t *)&p.missing[u] != 0u) {
      return;
    }
  }
  mark_push(p, u, stamp);
}

// Put the predecessors of the flagged lanes' positions into the next
// frontier.  The reverse-CSR ranges of all flagged lanes are concatenated and
// walked 32 entries at a time, so a position with many predecessors is spread
// over the whole warp.
__device__ void push_preds_warp(const KParams &p, Ctr *c, uint32_t *sm, uint32_t v, bool flagged, uint32_t stamp,
                                uint32_t lane, bool first = false) {
  const uint32_t firsts = __ballot_sync(FULL, flagged && first);
  uint32_t b = 0, n = 0;
  if (flagged) {
    b = ld(p.rrow, v, p.n_nodes + 1, c);
    n = ld(p.rrow, (unsigned long long)v + 1, p.n_nodes + 1, c) - b;
  }
  const uint32_t incl = warp_incl_scan(n, lane);
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  if (total == 0u) return;
  sm[SM_PINC + lane] = incl;
  sm[SM_PBEG + lane] = b;
  __syncwarp();
  for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
    const uint32_t t = t0 + lane;
    if (t < total) {
      // owner lane: the first whose inclusive end exceeds t
      uint32_t lo = 0, hi = 31;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sm[SM_PINC + mid] > t) hi = mid; else lo = mid + 1;
      }
      const uint32_t start = lo ? sm[SM_PINC + lo - 1] : 0u;
      const unsigned long long k = (unsigned long long)sm[SM_PBEG + lo] + (t - start);
      const uint32_t u = ld(p.rcol, k, p.n_edges, c);
      if (CHECK_IDX(c, u, p.n_nodes)) push_one(p, u, stamp, (firsts >> lo) & 1u);
    }
  }
  __syncwarp();
}

template <class Cd, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_round(const KParams p) {
  __shared__ uint32_t smem[WARPS_PER_BLOCK * SM_WORDS];
  __shared__ uint32_t tscr[WARPS_PER_BLOCK * TSCR * 32];
  Ctr *c = p.ctr;
  if (c->halt) return;
  const uint32_t cur = c->cur;
  const uint32_t fs = c->fsize[cur];
  if (fs == 0) return;
  const uint32_t *F = cur ? p.front1 : p.front0;
  const uint32_t stamp = c->stamp + 1u;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t *sm = smem + (threadIdx.x >> 5) * SM_WORDS;
  uint32_t *scr = tscr + (threadIdx.x >> 5) * (TSCR * 32) + lane;
  const Cd cd = make_codec<Cd>(p);
  uint32_t *arena = c->arena;
  const unsigned long long cap = c->arena_cap;
  WarpAlloc wa{0, 0};
  uint32_t t_edges = 0, t_bytes = 0, t_pos = 0;  // per lane, this launch
#if GEQ_PATH_PROFILE
  unsigned long long prof_acc[16] = {};
  const long long t_all0 = clock64();
#endif
  for (;;) {
    // 32 slots at a time from a shared counter: warps that drew heavy
    // positions take fewer slots
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&c->next_slot, 32u);
    base = __shfl_sync(FULL, base, 0);
    if (base >= fs) break;
#if GEQ_PATH_PROFILE
    const long long tq0 = clock64();
#endif
    const uint32_t slot = base + lane;
    const bool active = slot < fs;
    const uint32_t v = active ? ld(F, slot, p.n_nodes, c) : 0u;
    int ts = T_NONE;
    uint32_t cnt = 0, old_cnt = 0;
    if (active)
      ts = p.thread_path ? thread_solve(p, c, cd, arena, cap, v, scr, cnt, t_edges, t_bytes, old_cnt) : T_BIG;
    if (ts != T_NONE && ts != T_BIG && ts != T_SKIPPED) t_pos++;
    // inline results need no arena; one reservation for the others
    unsigned long long nd = NONE_DESC;
    if (ts == T_CHANGED && cnt <= p.inl) {
      nd = inl_hdr(cnt);
      for (uint32_t q = 0; q < cnt; q++) nd |= (unsigned long long)SCR(TK + q) << (q * p.ib);
    }
    const uint32_t need = (ts == T_CHANGED && cnt > p.inl) ? cnt : 0u;
    const uint32_t incl = warp_incl_scan(need, lane);
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    unsigned long long obase = 0;
    const bool ok = total == 0u || wa.alloc(total, c, cap, lane, obase);
    if (need) {
      if (!ok) {
        ts = T_OVERFLOW;
      } else {
        const unsigned long long off = obase + incl - need;
        for (uint32_t q = 0; q < need; q++)
          if (CHECK_IDX(c, off + q, cap)) arena[off + q] = SCR(TK + q);
        nd = mkdesc(off, need);
      }
    }
    if (ts == T_CHANGED) t_bytes += 4u * cnt;
    if (active && ts != T_BIG && CHECK_IDX(c, slot, p.n_nodes)) p.slot_new[slot] = (ts == T_CHANGED) ? nd : NONE_DESC;
    // large positions go to k_round_big (a whole warp per position)
    const uint32_t big = __ballot_sync(FULL, ts == T_BIG);
    if (big) {
      uint32_t b0 = 0;
      if (lane == 0) b0 = atomicAdd(&c->nbig, (uint32_t)__popc(big));
      b0 = __shfl_sync(FULL, b0, 0);
      if (ts == T_BIG) {
        const uint32_t k = b0 + (uint32_t)__popc(big & lanemask_lt());
        if (CHECK_IDX(c, k, p.n_nodes)) p.bigq[k] = slot;
      }
    }
#if GEQ_PATH_PROFILE
    const long long tq1 = clock64();
    if (lane == 0) { PROF_ADD(PF_CYC_THREAD, tq1 - tq0); PROF_ADD(PF_ITERS, 1); }
    if (active) {
      PROF_ADD(PF_SLOTS, 1);
      if (ts == T_SKIPPED) PROF_ADD(PF_SKIP, 1);
      if (ts == T_CHANGED || ts == T_UNCHANGED) {
        PROF_ADD((p.flags[v] & 1u) ? PF_T_ATT : PF_T_DEF, 1);
        PROF_ADD(PF_T_DEG, p.row[v + 1] - p.row[v]);
        if (ts == T_UNCHANGED) PROF_ADD(PF_T_UNCH, 1);
      }
    }
#endif
    push_preds_warp(p, c, sm, v, ts == T_CHANGED, stamp, lane, old_cnt == 0u);
    if (ts == T_OVERFLOW) mark_push(p, v, stamp);
#if GEQ_PATH_PROFILE
    if (lane == 0) PROF_ADD(PF_CYC_PUSH, clock64() - tq1);
    if (ts == T_CHANGED) PROF_ADD(PF_PUSHED, p.rrow[v + 1] - p.rrow[v]);
#endif
  }
#if GEQ_PATH_PROFILE
  if (lane == 0) PROF_ADD(PF_CYC_ALL, clock64() - t_all0);
#pragma unroll
  for (int i = 0; i < 16; i++) {
    unsigned long long a = prof_acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(FULL, a, o);
    if (lane == 0 && a) atomicAdd(&c->prof[i], a);
  }
#endif
  unsigned long long te = t_edges, tb = t_bytes, tp = t_pos;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    te += __shfl_xor_sync(FULL, te, o);
    tb += __shfl_xor_sync(FULL, tb, o);
    tp += __shfl_xor_sync(FULL, tp, o);
  }
  if (lane == 0 && tp) {
    atomicAdd(&c->positions, tp);
    atomicAdd(&c->edges, te);
    atomicAdd(&c->bytes, tb);
  }
}

// The large positions k_round queued: one warp per position with the warp
// routines (tree fold, register and bitmap paths), then its predecessors.
template <class Cd>
__global__ void __launch_bounds__(BLOCK, GEQ_BIG_BLOCKS_PER_SM) k_round_big(const KParams p) {
  __shared__ uint32_t smem[WARPS_PER_BLOCK * SM_WORDS];
  __shared__ uint32_t tscr[WARPS_PER_BLOCK * TSCR * 32];
  Ctr *c = p.ctr;
  if (c->halt) return;
  const uint32_t nb = c->nbig;
  if (nb == 0) return;
  const uint32_t cur = c->cur;
  const uint32_t *F = cur ? p.front1 : p.front0;
  const uint32_t stamp = c->stamp + 1u;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t *sm = smem + (threadIdx.x >> 5) * SM_WORDS;
  uint32_t *scr = tscr + (threadIdx.x >> 5) * (TSCR * 32) + lane;
  const Cd cd = make_codec<Cd>(p);
  uint32_t *arena = c->arena;
  const unsigned long long cap = c->arena_cap;
  WarpAlloc wa{0, 0};
  unsigned long long w_edges = 0, w_bytes = 0, w_pos = 0;  // lane-uniform
  WarpCtx x{p, c, arena, cap, lane, sm, wa, w_edges, w_bytes, scr};
#if GEQ_PATH_PROFILE
  const long long t0 = clock64();
#endif
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(&c->next_big, 1u);
    i = __shfl_sync(FULL, i, 0);
    if (i >= nb) break;
    const uint32_t slot = ld(p.bigq, i, p.n_nodes, c);
    const uint32_t v = ld(F, slot, p.n_nodes, c);
#if GEQ_PATH_PROFILE
    if (lane == 0) {
      atomicAdd(&c->prof[(p.flags[v] & 1u) ? PF_B_ATT : PF_B_DEF], 1ull);
      atomicAdd(&c->prof[PF_B_DEG], (unsigned long long)(p.row[v + 1] - p.row[v]));
    }
#endif
    const bool was_empty = dcnt(ld(p.desc, v, p.n_nodes, c)) == 0u;  // committed list, before this round
    const Res r = solve_position(x, cd, v);
    if (r.st != R_SKIPPED) w_pos++;
    if (lane == 0 && CHECK_IDX(c, slot, p.n_nodes)) p.slot_new[slot] = (r.st == R_CHANGED) ? r.d : NONE_DESC;
    push_preds_warp(p, c, sm, v, lane == 0 && r.st == R_CHANGED, stamp, lane, was_empty);
    if (r.st == R_OVERFLOW && lane == 0) mark_push(p, v, stamp);  // retried after compaction
  }
#if GEQ_PATH_PROFILE
  if (lane == 0) atomicAdd(&c->prof[PF_CYC_BIG], (unsigned long long)(clock64() - t0));
#endif
  if (lane == 0 && w_pos) {
    atomicAdd(&c->positions, w_pos);
    atomicAdd(&c->edges, w_edges);
    atomicAdd(&c->bytes, w_bytes);
  }
}

// Publish the round's new descriptors, clear the bitmap half of the round
// after next, count this round's pushes per block (for k_ffill) and advance
// to the next round.  Launched with exactly fblocks blocks.
__global__ void k_commit(const KParams p) {
  Ctr *c = p.ctr;
  // k_round only raises `overflow` (never `halt`) for arena exhaustion, so
  // the round that overflowed still commits its finished positions; k_ffill
  // then halts the remaining rounds of the graph until the host has
  // compacted the arena.
  if (c->halt) return;
  __shared__ uint32_t wsum[2 * WARPS_PER_BLOCK];
  __shared__ bool last;
  const uint32_t cur = c->cur;
  const uint32_t fs = c->fsize[cur];
  const uint32_t stamp = c->stamp;
  if (fs) {
    const uint32_t *F = cur ? p.front1 : p.front0;
    // the round after next pushes with stamp + 2: clear that half
    uint32_t *mh = p.mark + (stamp & 1u) * p.mwords;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.mwords; i += gridDim.x * blockDim.x) mh[i] = 0u;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < fs; s += gridDim.x * blockDim.x) {
      const unsigned long long d = p.slot_new[s];
      if (d != NONE_DESC) {
        const uint32_t v = F[s];
        if (CHECK_IDX(c, v, p.n_nodes)) p.desc[v] = d;
      }
    }
  }
  // this round's pushes (stamp + 1 half): attackers and defenders per block.
  // With an empty frontier both halves are clear and the counts are zero.
  {
    const uint32_t *mh = p.mark + ((stamp + 1u) & 1u) * p.mwords;
    const uint32_t per = (p.mwords + gridDim.x - 1u) / gridDim.x;
    const uint32_t b = min(p.mwords, blockIdx.x * per), e = min(p.mwords, b + per);
    uint32_t sa = 0, sd = 0;
    for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) {
      const uint32_t w = mh[i], a = p.abits[i];
      sa += (uint32_t)__popc(w & a);
      sd += (uint32_t)__popc(w & ~a);
    }
    sa = __reduce_add_sync(FULL, sa);
    sd = __reduce_add_sync(FULL, sd);
    if ((threadIdx.x & 31u) == 0u) {
      wsum[threadIdx.x >> 5] = sa;
      wsum[WARPS_PER_BLOCK + (threadIdx.x >> 5)] = sd;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ta = 0, td = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      ta += wsum[w];
      td += wsum[WARPS_PER_BLOCK + w];
    }
    p.fpart[2 * blockIdx.x] = ta;
    p.fpart[2 * blockIdx.x + 1] = td;
  }
  if (!fs) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&c->done_blocks, 1u) == gridDim.x - 1u;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    c->fsize[cur] = 0u;
    c->cur = cur ^ 1u;
    c->stamp = stamp + 1u;
    c->rounds = c->rounds + 1ull;
    c->done_blocks = 0u;
    __threadfence();
  }
}

// Ids of the set bits of words [b, e) of `mh` (and of `mask` ^ flip when a
// mask is given), in order, to F[base ...]; every thread of the block calls
// it.  Returns the count.  wsum: 33 words of shared memory.
__device__ uint32_t block_fill_bits(const uint32_t *mh, uint32_t b, uint32_t e, uint32_t base, uint32_t *F,
                                    uint32_t nmax, Ctr *c, uint32_t *wsum, const uint32_t *mask = nullptr,
                                    uint32_t flip = 0u) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarps = blockDim.x >> 5;
  uint32_t total = 0;
  for (uint32_t t0 = b; t0 < e; t0 += blockDim.x) {
    const uint32_t i = t0 + tid;
    const uint32_t w = i < e ? (mh[i] & (mask ? (mask[i] ^ flip) : ~0u)) : 0u;
    const uint32_t cnt = (uint32_t)__popc(w);
    const uint32_t incl = warp_incl_scan(cnt, lane);
    if (lane == 31u) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t x = lane < nwarps ? wsum[lane] : 0u;
      const uint32_t xi = warp_incl_scan(x, lane);
      if (lane < nwarps) wsum[lane] = xi - x;
      if (lane == 31u) wsum[32] = xi;
    }
    __syncthreads();
    uint32_t off = base + total + wsum[warp] + incl - cnt;
    for (uint32_t x = w; x; x &= x - 1u, off++)
      if (CHECK_IDX(c, off, nmax)) F[off] = i * 32u + (uint32_t)__ffs((int)x) - 1u;
    total += wsum[32];
    __syncthreads();
  }
  return total;
}

// k_fcount (after the initial pushes; k_commit counts after a round) +
// k_ffill: the next frontier (stamp parity half of the bitmap)
// as a list in position order, attackers first, then defenders, so that a
// warp of the next round mostly meets one kind of position.  The last k_ffill
// block publishes its size, resets the slot counter and, after an arena
// overflow, halts the remaining rounds of the graph until the host has
// compacted the arena.
__global__ void k_fcount(const KParams p) {
  Ctr *c = p.ctr;
  if (c->halt) return;
  __shared__ uint32_t wsum[2 * WARPS_PER_BLOCK];
  const uint32_t *mh = p.mark + (c->stamp & 1u) * p.mwords;
  const uint32_t per = (p.mwords + gridDim.x - 1u) / gridDim.x;
  const uint32_t b = min(p.mwords, blockIdx.x * per), e = min(p.mwords, b + per);
  uint32_t sa = 0, sd = 0;
  for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) {
    const uint32_t w = mh[i], a = p.abits[i];
    sa += (uint32_t)__popc(w & a);
    sd += (uint32_t)__popc(w & ~a);
  }
  sa = __reduce_add_sync(FULL, sa);
  sd = __reduce_add_sync(FULL, sd);
  if ((threadIdx.x & 31u) == 0u) {
    wsum[threadIdx.x >> 5] = sa;
    wsum[WARPS_PER_BLOCK + (threadIdx.x >> 5)] = sd;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ta = 0, td = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      ta += wsum[w];
      td += wsum[WARPS_PER_BLOCK + w];
    }
    p.fpart[2 * blockIdx.x] = ta;
    p.fpart[2 * blockIdx.x + 1] = td;
  }
}
__global__ void k_ffill(const KParams p) {
  Ctr *c = p.ctr;
  if (c->halt) return;
  __shared__ uint32_t wsum[33];
  __shared__ uint32_t s_pa, s_pd, s_ta;
  const uint32_t cur = c->cur;
  uint32_t *F = cur ? p.front1 : p.front0;
  const uint32_t *mh = p.mark + (c->stamp & 1u) * p.mwords;
  // attackers before this block, defenders before this block, all attackers
  uint32_t pa = 0, pd = 0, ta = 0;
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    const uint32_t a = p.fpart[2 * i], d = p.fpart[2 * i + 1];
    ta += a;
    if (i < blockIdx.x) {
      pa += a;
      pd += d;
    }
  }
  pa = __reduce_add_sync(FULL, pa);
  pd = __reduce_add_sync(FULL, pd);
  ta = __reduce_add_sync(FULL, ta);
  if (threadIdx.x == 0) {
    s_pa = 0u;
    s_pd = 0u;
    s_ta = 0u;
  }
  __syncthreads();
  if ((threadIdx.x & 31u) == 0u) {
    atomicAdd(&s_pa, pa);
    atomicAdd(&s_pd, pd);
    atomicAdd(&s_ta, ta);
  }
  __syncthreads();
  const uint32_t per = (p.mwords + gridDim.x - 1u) / gridDim.x;
  const uint32_t b = min(p.mwords, blockIdx.x * per), e = min(p.mwords, b + per);
  block_fill_bits(mh, b, e, s_pa, F, (uint32_t)p.n_nodes, c, wsum, p.abits, 0u);
  block_fill_bits(mh, b, e, s_ta + s_pd, F, (uint32_t)p.n_nodes, c, wsum, p.abits, ~0u);
  if (blockIdx.x == gridDim.x - 1u && threadIdx.x == 0) {
    c->fsize[cur] = s_ta + s_pd + p.fpart[2 * blockIdx.x + 1];
    c->next_slot = 0u;
    c->nbig = 0u;
    c->next_big = 0u;
    if (c->overflow) c->halt = 1u;
  }
}
// Attacker positions as a bitmap (frontier ordering by kind).
__global__ void k_abits(const uint8_t *flags, unsigned long long n, uint32_t words, uint32_t *abits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
    uint32_t w = 0;
    for (uint32_t k = 0; k < 32u; k++) {
      const unsigned long long v = (unsigned long long)i * 32u + k;
      if (v < n && (flags[v] & 1u)) w |= 1u << k;
    }
    abits[i] = w;
  }
}

}  // namespace geq

// ===========================================================================
// Support kernels: scan, reverse CSR, initial state, compaction, download.
// ===========================================================================
namespace geq {

constexpr int SCAN_T = 1024;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_T * SCAN_ITEMS;

__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long x, unsigned long long *ws,
                                                              unsigned long long &total) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  unsigned long long incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(FULL, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  if (lane == 31u) ws[w] = incl;
  __syncthreads();
  if (w == 0) {
    unsigned long long s = (lane < blockDim.x / 32) ? ws[lane] : 0ull;
    unsigned long long si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(FULL, si, o);
      if (lane >= (uint32_t)o) si += y;
    }
    ws[lane] = si - s;
    if (lane == 31u) ws[32] = si;
  }
  __syncthreads();
  total = ws[32];
  unsigned long long r = ws[w] + incl - x;
  __syncthreads();
  return r;
}

__global__ void k_scan_reduce(const uint32_t *in, unsigned long long n, unsigned long long *part) {
  __shared__ unsigned long long ws[33];
  unsigned long long base = (unsigned long long)blockIdx.x * SCAN_TILE + (unsigned long long)threadIdx.x * SCAN_ITEMS;
  unsigned long long s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++)
    if (base + i < n) s += in[base + i];
  unsigned long long total;
  block_excl_scan(s, ws, total);
  if (threadIdx.x == 0) part[blockIdx.x] = total;
}

// Exclusive scan of the per-tile sums, one block.
__global__ void k_scan_partials(unsigned long long *part, unsigned long long nb) {
  __shared__ unsigned long long ws[33];
  unsigned long long carry = 0;
  for (unsigned long long b0 = 0; b0 < nb; b0 += SCAN_T) {
    unsigned long long i = b0 + threadIdx.x;
    unsigned long long x = i < nb ? part[i] : 0ull;
    unsigned long long total;
    unsigned long long e = block_excl_scan(x, ws, total);
    if (i < nb) part[i] = carry + e;
    carry += total;
  }
}

__global__ void k_scan_apply(const uint32_t *in, unsigned long long n, const unsigned long long *part,
                             unsigned long long *out) {
  __shared__ unsigned long long ws[33];
  unsigned long long base = (unsigned long long)blockIdx.x * SCAN_TILE + (unsigned long long)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  unsigned long long s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = (base + i < n) ? in[base + i] : 0u;
    s += v[i];
  }
  unsigned long long total;
  unsigned long long e = block_excl_scan(s, ws, total) + part[blockIdx.x];
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) out[base + i] = e;
    e += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = e;
}

__global__ void k_desc_counts(const unsigned long long *desc, unsigned long long n, uint32_t *cnt) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x)
    cnt[v] = dcnt(desc[v]);
}

__global__ void k_indegree(const uint32_t *col, unsigned long long m, unsigned long long n, uint32_t *indeg,
                           uint32_t *err) {
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < m;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t w = col[k];
    if (w < n) atomicAdd(&indeg[w], 1u);
    else atomicOr(err, 1u);
  }
}

__global__ void k_u64_to_u32(const unsigned long long *in, unsigned long long n, uint32_t *out) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    out[i] = (uint32_t)in[i];
}

// Predecessor lists.  Successor ids and row offsets are not trusted yet (the
// error flags of the checks are read after the upload): edges outside
// [0, m) and successors outside [0, n) are skipped, as k_indegree skips them,
// so every write stays inside the lists counted for it.
__global__ void k_fill_reverse(const uint32_t *row, const uint32_t *col, unsigned long long n,
                               unsigned long long m, uint32_t *cursor, uint32_t *rcol) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long e = min((unsigned long long)row[v + 1], m);
    for (unsigned long long k = row[v]; k < e; k++) {
      const uint32_t w = col[k];
      if (w >= n) continue;
      const uint32_t pos = atomicAdd(&cursor[w], 1u);
      if (pos < m) rcol[pos] = (uint32_t)v;
    }
  }
}

__device__ __forceinline__ uint32_t game_of(const unsigned long long *base, uint32_t n_games,
                                            unsigned long long x) {
  // largest g with base[g] <= x
  uint32_t lo = 0, hi = n_games;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// Shift per-game local ids of a concatenated batch into the global id space.
// Row offsets of every game, before they are made global: each game's first
// offset is 0 and offsets do not decrease up to the game's edge count.
__global__ void k_check_rows(const uint32_t *row, unsigned long long n, const unsigned long long *node_base,
                             const unsigned long long *edge_base, uint32_t n_games, uint32_t *err) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t g = game_of(node_base, n_games, v);
    const uint32_t r = row[v];
    const unsigned long long next =
        (v + 1 < node_base[g + 1]) ? row[v + 1] : (edge_base[g + 1] - edge_base[g]);
    if ((v == node_base[g] && r != 0u) || r > next) atomicOr(err, 4u);
  }
}
// EnergyGame::standard_reach + with_reach (energygame.rs:347-365) on the
// device: {0} at every defender without successors.
__global__ void k_std_reach(const uint32_t *row, const uint8_t *flags, unsigned long long n,
                            unsigned long long *desc) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x)
    if (!(flags[v] & 1u) && row[v] == row[v + 1]) desc[v] = inl_hdr(1u);
}
__global__ void k_fix_rows(uint32_t *row, unsigned long long n, const unsigned long long *node_base,
                           const unsigned long long *edge_base, uint32_t n_games) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x)
    row[v] += (uint32_t)edge_base[game_of(node_base, n_games, v)];
}
__global__ void k_fix_cols(uint32_t *col, unsigned long long m, const unsigned long long *node_base,
                           const unsigned long long *edge_base, uint32_t n_games,
                           const unsigned long long *game_nodes, uint32_t *err) {
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < m;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t g = game_of(edge_base, n_games, k);
    uint32_t w = col[k];
    if (w >= game_nodes[g]) atomicOr(err, 1u);
    col[k] = w + (uint32_t)node_base[g];
  }
}

// TryFrom checks on the device: every update code names an element and the
// padding bits above the last element are clear (pack_upd, energy.rs:543-565).
__global__ void k_check_weights(const uint32_t *wt, unsigned long long m, uint32_t elements, uint32_t ubits,
                                uint32_t umask, uint32_t *err) {
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < m;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t u = wt[k];
    bool bad = elements * ubits < 32u && (u >> (elements * ubits)) != 0u;
    for (uint32_t i = 0; i < elements; i++)
      if (((u >> (i * ubits)) & umask) > elements + 1u) bad = true;
    if (bad) atomicOr(err, 2u);
  }
}

// EnergyGame::with_reach (energygame.rs:355-365): {0} at every target.
// Successors with an empty initial list, per defender (attackers: 0).
__global__ void k_missing_init(const KParams p, const unsigned long long *desc0, uint32_t *miss) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < p.n_nodes;
       v += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t m = 0;
    if (!(p.flags[v] & 1u))
      for (uint32_t k = p.row[v]; k < p.row[v + 1]; k++) m += dcnt(desc0[p.col[k]]) == 0u ? 1u : 0u;
    miss[v] = m;
  }
}

// Edge pairs of the lane path: successor id and the update in the codec's
// pack_edge form (after k_fix_cols / k_check_weights).
template <class Cd>
__global__ void k_pack_edges(const uint32_t *col, const uint32_t *wt, unsigned long long m, unsigned long long *cw) {
  for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < m;
       k += (unsigned long long)gridDim.x * blockDim.x)
    cw[k] = (unsigned long long)col[k] | ((unsigned long long)Cd::pack_edge(wt[k]) << 32);
}

// Packed game blocks (row | col | wt | attacker bytes | reach, one after the
// other in `raw`, game g from word boff[g]) into the batch's arrays: rows and
// columns stay game-local (k_fix_rows / k_fix_cols rebase them), reach
// entries get the game's position base.  One thread per word of `raw`.
__global__ void k_unpack_games(const uint32_t *raw, const unsigned long long *boff, const unsigned long long *nb,
                               const unsigned long long *eb, const unsigned long long *rb, uint32_t n_games,
                               unsigned long long words, uint32_t *row, uint32_t *col, uint32_t *wt,
                               uint8_t *flags, uint32_t *reach, unsigned long long N, unsigned long long M) {
  if (blockIdx.x == 0 && threadIdx.x == 0) row[N] = (uint32_t)M;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < words;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n_games - 1;  // the game whose block holds word i
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (boff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const uint32_t g = lo;
    const unsigned long long n = nb[g + 1] - nb[g], m = eb[g + 1] - eb[g];
    unsigned long long k = i - boff[g];
    const uint32_t x = raw[i];
    if (k < n + 1) {
      if (k < n) row[nb[g] + k] = x;
      continue;
    }
    k -= n + 1;
    if (k < m) { col[eb[g] + k] = x; continue; }
    k -= m;
    if (k < m) { wt[eb[g] + k] = x; continue; }
    k -= m;
    const unsigned long long aw = (n + 3) / 4;
    if (k < aw) {
      for (unsigned long long b = 0; b < 4 && 4 * k + b < n; b++) flags[nb[g] + 4 * k + b] = (uint8_t)(x >> (8 * b));
      continue;
    }
    k -= aw;
    if (k < rb[g + 1] - rb[g]) reach[rb[g] + k] = x + (uint32_t)nb[g];
  }
}
__global__ void k_init_reach(unsigned long long *desc, const uint32_t *reach, unsigned long long n_reach) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n_reach;
       i += (unsigned long long)gridDim.x * blockDim.x)
    desc[reach[i]] = inl_hdr(1u);  // one energy, all elements 0
}

// initialize_visit_lists (energygame.rs:1461-1465): predecessors of to_reach.
// The initial frontier of the standard reach: predecessors of every defender
// without successors.
__global__ void k_init_frontier_std(const KParams p) {
  __shared__ uint32_t smem[(256 / 32) * SM_WORDS];
  Ctr *c = p.ctr;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t *sm = smem + (threadIdx.x >> 5) * SM_WORDS;
  const unsigned long long gw = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long i0 = gw * 32ull; i0 < p.n_nodes; i0 += nw * 32ull) {
    const unsigned long long v = i0 + lane;
    const bool f = v < p.n_nodes && !(p.flags[v] & 1u) && p.row[v] == p.row[v + 1];
    push_preds_warp(p, c, sm, (uint32_t)(v < p.n_nodes ? v : 0u), f, c->stamp, lane);
  }
}
__global__ void k_init_frontier(const KParams p, const uint32_t *reach, unsigned long long n_reach) {
  __shared__ uint32_t smem[(256 / 32) * SM_WORDS];
  Ctr *c = p.ctr;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t *sm = smem + (threadIdx.x >> 5) * SM_WORDS;
  const unsigned long long gw = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long i0 = gw * 32ull; i0 < n_reach; i0 += nw * 32ull) {
    const unsigned long long i = i0 + lane;
    push_preds_warp(p, c, sm, i < n_reach ? reach[i] : 0u, i < n_reach, c->stamp, lane);
  }
}

// Arena compaction: live arena lists move to `dst`; inline lists stay.
__global__ void k_compact(unsigned long long *desc, unsigned long long n, const unsigned long long *noff,
                          const uint32_t *src, uint32_t *dst) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long gw = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long v = gw; v < n; v += nw) {
    const unsigned long long d = desc[v];
    if (dinl(d)) continue;
    const uint32_t c = dcnt(d);
    const unsigned long long o = doff(d), no = noff[v];
    for (uint32_t q = lane; q < c; q += 32u) dst[no + q] = src[o + q];
    if (lane == 0) desc[v] = mkdesc(no, c);
  }
}

// Arena words held by arena (non-inline) lists.
__global__ void k_arena_counts(const unsigned long long *desc, unsigned long long n, uint32_t *cnt) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n;
       v += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long d = desc[v];
    cnt[v] = dinl(d) ? 0u : dcnt(d);
  }
}

__global__ void k_gather(const unsigned long long *desc, unsigned long long n, const unsigned long long *goff,
                         const uint32_t *arena, uint32_t ib, uint32_t ibm, uint32_t *out) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long gw = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long v = gw; v < n; v += nw) {
    const unsigned long long d = desc[v];
    const uint32_t c = dcnt(d);
    const unsigned long long go = goff[v];
    for (uint32_t q = lane; q < c; q += 32u)
      out[go + q] = dinl(d) ? ((uint32_t)(d >> (q * ib)) & ibm) : arena[doff(d) + q];
  }
}

// Per-game offsets relative to the game's first energy: game g owns entries
// [node_base[g] + g, node_base[g+1] + g] of `rel`.
__global__ void k_rel_offsets(const unsigned long long *goff, unsigned long long n,
                              const unsigned long long *node_base, uint32_t n_games, unsigned long long *rel) {
  for (unsigned long long v = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; v < n + n_games;
       v += (unsigned long long)gridDim.x * blockDim.x) {
    if (v < n) {
      uint32_t g = game_of(node_base, n_games, v);
      rel[v + g] = goff[v] - goff[node_base[g]];
    } else {
      uint32_t g = (uint32_t)(v - n);
      rel[node_base[g + 1] + g] = goff[node_base[g + 1]] - goff[node_base[g]];
    }
  }
}

// Selection of whole games: position i of the selection is position
// i - pre[g] of selected game g (first id base[g]).
__global__ void k_sel_expand(const unsigned long long *base, const unsigned long long *pre, uint32_t g_count,
                             unsigned long long k, uint32_t *sel) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t g = game_of(pre, g_count, i);
    sel[i] = (uint32_t)(base[g] + (i - pre[g]));
  }
}

// Clear the frontier-bitmap bits of position ranges [b, e) (games that must
// not be solved): words at a range's ends are shared with its neighbours.
__global__ void k_clear_ranges(uint32_t *mh, const unsigned long long *ranges, uint32_t n_ranges) {
  for (uint32_t r = blockIdx.x; r < n_ranges; r += gridDim.x) {
    const unsigned long long b = ranges[2 * r], e = ranges[2 * r + 1];
    if (b >= e) continue;
    const unsigned long long w0 = b >> 5, w1 = (e - 1) >> 5;
    for (unsigned long long w = w0 + threadIdx.x; w <= w1; w += blockDim.x) {
      uint32_t m = ~0u;
      if (w == w0) m &= ~0u << (uint32_t)(b & 31u);
      if (w == w1) m &= ~0u >> (31u - (uint32_t)((e - 1) & 31u));
      atomicAnd(&mh[w], ~m);
    }
  }
}

// Counts of selected positions (sel = global ids).
__global__ void k_sel_counts(const unsigned long long *desc, const uint32_t *sel, unsigned long long k,
                             uint32_t *cnt) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x)
    cnt[i] = dcnt(desc[sel[i]]);
}
__global__ void k_sel_gather(const unsigned long long *desc, const uint32_t *sel, unsigned long long k,
                             const unsigned long long *goff, const uint32_t *arena, uint32_t ib, uint32_t ibm,
                             uint32_t *out) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long gw = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long i = gw; i < k; i += nw) {
    const unsigned long long d = desc[sel[i]];
    const uint32_t c = dcnt(d);
    const unsigned long long go = goff[i];
    for (uint32_t q = lane; q < c; q += 32u)
      out[go + q] = dinl(d) ? ((uint32_t)(d >> (q * ib)) & ibm) : arena[doff(d) + q];
  }
}

__global__ void k_set_arena(Ctr *c, uint32_t *arena, unsigned long long cap, unsigned long long top) {
  c->arena = arena;
  c->arena_cap = cap;
  c->arena_top = top;
  c->overflow = 0u;
  c->halt = 0u;
}

// ===========================================================================
// Host side
// ===========================================================================
#define CU(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? GEQ_ERR_OUT_OF_MEMORY : GEQ_ERR_CUDA,    \
                  "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));        \
  } while (0)

// Device memory cache.  Solving one small game per call (the plain drop-in)
// would otherwise pay a cudaMalloc/cudaFree pair per buffer and call; cached
// blocks are reused by later uploads.
class DevPool {
 public:
  static size_t round_size(size_t b) {
    b = std::max<size_t>(b, 512);
    if (b <= (8u << 20)) {
      size_t r = 512;
      while (r < b) r <<= 1;
      return r;
    }
    return (b + (8u << 20) - 1) & ~size_t((8u << 20) - 1);
  }
  // A cached block of the request's size class, or of a larger class up to
  // 4x: a serving loop's batches vary in size, and reusing a larger block
  // avoids a cudaMalloc for every new size.
  void *get(size_t bytes) {
    const size_t r = round_size(bytes);
    for (auto it = free_.lower_bound(r); it != free_.end() && it->first <= 4 * r; ++it)
      if (!it->second.empty()) {
        void *p = it->second.back();
        it->second.pop_back();
        cached_ -= it->first;
        size_[p] = it->first;
        return p;
      }
    void *p = nullptr;
    if (cudaMalloc(&p, r) != cudaSuccess) {
      cudaGetLastError();
      trim();
      if (cudaMalloc(&p, r) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
    }
    size_[p] = r;
    return p;
  }
  // Back to the cache under the block's real size (`bytes` is the request).
  void put(void *p, size_t bytes) {
    if (!p) return;
    auto it = size_.find(p);
    const size_t r = it != size_.end() ? it->second : round_size(bytes);
    if (it != size_.end()) size_.erase(it);
    if (cached_ + r > limit_) {
      cudaFree(p);
      return;
    }
    free_[r].push_back(p);
    cached_ += r;
  }
  void trim() {
    for (auto &kv : free_)
      for (void *p : kv.second) cudaFree(p);
    free_.clear();
    cached_ = 0;
  }
  ~DevPool() { trim(); }

 private:
  std::map<size_t, std::vector<void *>> free_;
  std::unordered_map<void *, size_t> size_;  // blocks handed out: real size
  size_t cached_ = 0;
  size_t limit_ = (size_t)16 << 30;
};

size_t HostPool::round_size(size_t b) {
  b = std::max<size_t>(b, 4096);
  if (b <= (64u << 20)) {
    size_t r = 4096;
    while (r < b) r <<= 1;
    return r;
  }
  return (b + (64u << 20) - 1) & ~size_t((64u << 20) - 1);
}
void *HostPool::get(size_t bytes, size_t &cap) {
  cap = round_size(bytes);
  {
    // the request's size class or a larger one up to 4x (see DevPool::get)
    std::lock_guard<std::mutex> g(mu_);
    for (auto it = free_.lower_bound(cap); it != free_.end() && it->first <= 4 * cap; ++it)
      if (!it->second.empty()) {
        void *p = it->second.back();
        it->second.pop_back();
        cached_ -= it->first;
        cap = it->first;
        return p;
      }
  }
  void *p = nullptr;
  if (cudaHostAlloc(&p, cap, flags_) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void HostPool::put(void *p, size_t cap) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> g(mu_);
    if (cached_ + cap <= limit_) {
      free_[cap].push_back(p);
      cached_ += cap;
      return;
    }
  }
  cudaFreeHost(p);
}
HostPool::~HostPool() {
  for (auto &kv : free_)
    for (void *p : kv.second) cudaFreeHost(p);
}
bool HostBuf::alloc(const std::shared_ptr<HostPool> &hp, size_t bytes) {
  reset();
  bytes = std::max<size_t>(bytes, 8);
  if (hp && (p = hp->get(bytes, cap)) != nullptr) {
    pool = hp;
    return true;
  }
  p = std::malloc(bytes);
  cap = bytes;
  return p != nullptr;
}
void HostBuf::reset() {
  if (p) {
    if (pool) pool->put(p, cap);
    else std::free(p);
  }
  p = nullptr;
  cap = 0;
  pool.reset();
}

struct Engine::State {
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, eva = nullptr, evb = nullptr;
  Ctr *h_ctr = nullptr;     // pinned
  // one captured graph of rounds per codec [CodecStd, CodecGen], shared by all
  // uploads; its kernel nodes get the parameters of the games being solved
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  std::vector<cudaGraphNode_t> gnodes[2];
  uint32_t g_rounds[2] = {0, 0}, g_bps[2] = {0, 0};
  KParams g_kp[2] = {};              // the parameters the graph's nodes hold
  bool g_kp_valid[2] = {false, false};
  unsigned long long *part = nullptr;
  size_t part_cap = 0;
  uint32_t *cnt = nullptr;
  size_t cnt_cap = 0;
  char *stage = nullptr;
  size_t stage_cap = 0;
  uint32_t *d_err = nullptr;
  DevPool pool;
  std::shared_ptr<HostPool> hpool = std::make_shared<HostPool>();
  std::set<DeviceGamesImpl *> live;
};

struct DeviceGamesImpl {
  Engine::State *owner = nullptr;  // pool the buffers return to
  std::vector<std::pair<void *, size_t>> bufs;
  Conf conf;
  bool generic = false;
  uint32_t n_games = 0;
  std::vector<unsigned long long> node_base, edge_base;  // n_games + 1
  unsigned long long N = 0, M = 0;
  uint32_t *row = nullptr, *col = nullptr, *wt = nullptr, *rrow = nullptr, *rcol = nullptr;
  uint8_t *flags = nullptr;
  unsigned long long *desc = nullptr, *desc_init = nullptr, *slot_new = nullptr;
  unsigned long long *cw = nullptr;  // edge pairs (successor, packed update)
  uint32_t *missing = nullptr, *missing_init = nullptr;  // defenders: successors with no energies yet
  std::vector<unsigned long long> off_ranges;  // position ranges of games that are not solved (pairs)
  uint32_t *mark = nullptr, *front0 = nullptr, *front1 = nullptr, *fpart = nullptr, *abits = nullptr, *bigq = nullptr;
  uint32_t *init_data = nullptr;
  unsigned long long init_total = 0;
  char *inbuf = nullptr;  // row, col, wt, flags, reach, init_data, [desc_init], node bases
  bool std_reach = false;       // standard reach computed on the device (no reach list)
  bool rows_on_device = false;  // row offsets checked by k_check_rows
  uint32_t *arena[2] = {nullptr, nullptr};
  unsigned long long arena_cap[2] = {0, 0};
  int arena_cur = 0;
  uint32_t *reach = nullptr;
  unsigned long long n_reach = 0;
  unsigned long long *d_node_base = nullptr;
  Ctr *ctr = nullptr;
  uint32_t next_stamp = 1;
  KParams kp{};
  // bookkeeping of the solve in progress (Engine::solve_begin / solve_step)
  struct Progress {
    unsigned long long launches = 0, compactions = 0, round_launches = 0;
    double round_ms = 0.0;
    std::chrono::steady_clock::time_point t_start{};
  } prog;
  HostBuf hstep;            // page-locked: the control block and active flags read back by a step
  uint8_t *d_act = nullptr; // active flags on the device
  bool step_active = false;

  template <class T>
  bool alloc(T *&p, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    p = (T *)(owner ? owner->pool.get(bytes) : nullptr);
    if (!p) return false;
    bufs.emplace_back((void *)p, bytes);
    return true;
  }
  template <class T>
  void release(T *&p) {
    for (size_t i = 0; i < bufs.size(); i++)
      if (bufs[i].first == (void *)p) {
        if (owner) owner->pool.put(p, bufs[i].second);
        else cudaFree(p);
        bufs.erase(bufs.begin() + i);
        break;
      }
    p = nullptr;
  }
  void release_all() {
    for (auto &b : bufs) {
      if (owner) owner->pool.put(b.first, b.second);
      else cudaFree(b.first);
    }
    bufs.clear();
  }
};

void destroy_games(DeviceGamesImpl *p) {
  if (!p) return;
  if (p->owner) {
    cudaStreamSynchronize(p->owner->stream);
    p->owner->live.erase(p);
  }
  p->release_all();
  delete p;
}

template <class T>
static geq_status dalloc(T *&p, size_t n) {
  p = nullptr;
  if (n == 0) n = 1;
  CU(cudaMalloc((void **)&p, n * sizeof(T)));
  return GEQ_OK;
}
template <class T>
static void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

static geq_status scan_u32(Engine::State &s, const uint32_t *in, unsigned long long n, unsigned long long *out,
                           unsigned long long &launches) {
  unsigned long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 0) nb = 1;
  if (s.part_cap < nb) {
    dfree(s.part);
    size_t cap = std::max<size_t>(nb, 1024);
    geq_status st = dalloc(s.part, cap);
    if (st) return st;
    s.part_cap = cap;
  }
  k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, s.stream>>>(in, n, s.part);
  k_scan_partials<<<1, SCAN_T, 0, s.stream>>>(s.part, nb);
  k_scan_apply<<<(unsigned)nb, SCAN_T, 0, s.stream>>>(in, n, s.part, out);
  launches += 3;
  CU(cudaGetLastError());
  return GEQ_OK;
}

static geq_status ensure_cnt(Engine::State &s, size_t n) {
  if (s.cnt_cap >= n) return GEQ_OK;
  dfree(s.cnt);
  size_t cap = std::max<size_t>(n, 1 << 16);
  geq_status st = dalloc(s.cnt, cap);
  if (st) return st;
  s.cnt_cap = cap;
  return GEQ_OK;
}

static geq_status ensure_stage(Engine::State &s, size_t bytes) {
  if (s.stage_cap >= bytes) return GEQ_OK;
  if (s.stage) cudaFreeHost(s.stage);
  s.stage = nullptr;
  size_t cap = std::max<size_t>(bytes, 1 << 20);
  cap = std::max(cap, s.stage_cap * 3 / 2);
  CU(cudaHostAlloc((void **)&s.stage, cap, cudaHostAllocDefault));
  s.stage_cap = cap;
  return GEQ_OK;
}

// Host-to-device upload of the staging buffer.  Small uploads are packed
// serially and sent with one copy.  Large ones are split into windows of the
// staging buffer: host threads pack the pieces in address order and each
// window is sent as soon as all its pieces are in, so packing overlaps the
// link transfer.
struct CopyJob {
  void *dst;
  const void *src;
  size_t bytes;
};
static geq_status staged_upload(std::vector<CopyJob> &jobs, const char *stage, char *dev, size_t total,
                                cudaStream_t S) {
  size_t payload = 0;
  for (auto &j : jobs) payload += j.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  if (payload < (16u << 20) || hw < 2) {
    for (auto &j : jobs)
      if (j.bytes) std::memcpy(j.dst, j.src, j.bytes);
    if (total) CU(cudaMemcpyAsync(dev, stage, total, cudaMemcpyHostToDevice, S));
    return GEQ_OK;
  }
  constexpr size_t WIN = 32u << 20, PIECE = 2u << 20;
  const size_t n_win = (total + WIN - 1) / WIN;
  struct Piece {
    size_t off;  // offset in the staging buffer
    const char *src;
    size_t bytes;
  };
  std::vector<Piece> pieces;
  pieces.reserve(jobs.size() + payload / PIECE + n_win);
  for (auto &j : jobs) {
    size_t o = (size_t)((const char *)j.dst - stage), left = j.bytes;
    const char *src = (const char *)j.src;
    while (left) {
      const size_t win_end = (o / WIN + 1) * WIN;
      const size_t b = std::min({left, PIECE, win_end - o});
      pieces.push_back(Piece{o, src, b});
      o += b; src += b; left -= b;
    }
  }
  std::sort(pieces.begin(), pieces.end(), [](const Piece &a, const Piece &b) { return a.off < b.off; });
  std::unique_ptr<std::atomic<size_t>[]> pending(new std::atomic<size_t>[n_win]);
  for (size_t w = 0; w < n_win; w++) pending[w].store(0, std::memory_order_relaxed);
  for (auto &pc : pieces) pending[pc.off / WIN].fetch_add(1, std::memory_order_relaxed);
  std::atomic<size_t> next{0};
  const unsigned T = std::min(16u, hw);
  std::vector<std::thread> pool;
  pool.reserve(T);
  for (unsigned t = 0; t < T; t++)
    pool.emplace_back([&]() {
      for (;;) {
        const size_t i = next.fetch_add(1, std::memory_order_relaxed);
        if (i >= pieces.size()) break;
        std::memcpy((char *)stage + pieces[i].off, pieces[i].src, pieces[i].bytes);
        pending[pieces[i].off / WIN].fetch_sub(1, std::memory_order_release);
      }
    });
  cudaError_t ce = cudaSuccess;
  for (size_t w = 0; w < n_win; w++) {
    while (pending[w].load(std::memory_order_acquire) != 0) std::this_thread::yield();
    const size_t o = w * WIN, b = std::min(WIN, total - o);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dev + o, stage + o, b, cudaMemcpyHostToDevice, S);
  }
  for (auto &th : pool) th.join();
  if (ce != cudaSuccess) return fail(GEQ_ERR_CUDA, "upload copy: %s", cudaGetErrorString(ce));
  return GEQ_OK;
}

void *Engine::stream_handle() const { return (void *)st->stream; }
std::shared_ptr<HostPool> Engine::host_pool() const { return st->hpool; }

static geq_status static_scratch(int device, unsigned char *&out);

geq_status Engine::create(int device, std::unique_ptr<Engine> &out) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(GEQ_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  if (device < 0 || device >= n) return fail(GEQ_ERR_NO_DEVICE, "device %d out of range (%d)", device, n);
  CU(cudaSetDevice(device));
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, device));
  {
    // reserve the scratch of geq_energy_game_run_static now (module load)
    unsigned char *scratch = nullptr;
    const geq_status rs = static_scratch(device, scratch);
    if (rs) return rs;
  }
  std::unique_ptr<Engine> eng(new Engine());
  eng->st.reset(new State());
  eng->n_sms = prop.multiProcessorCount;
  eng->total_mem = prop.totalGlobalMem;
  eng->name = prop.name;
  State &s = *eng->st;
  CU(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  CU(cudaEventCreate(&s.ev0));
  CU(cudaEventCreate(&s.ev1));
  CU(cudaEventCreate(&s.eva));
  CU(cudaEventCreate(&s.evb));
  CU(cudaHostAlloc((void **)&s.h_ctr, sizeof(Ctr), cudaHostAllocDefault));
  CU(cudaMalloc((void **)&s.d_err, sizeof(uint32_t)));
  // the round kernels want shared memory for several resident blocks
  CU(cudaFuncSetAttribute(k_round<CodecStd, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecStd, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecStd, 4>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecStd, 5>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecGen, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecGen, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecGen, 4>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round<CodecGen, 5>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round_big<CodecStd>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  CU(cudaFuncSetAttribute(k_round_big<CodecGen>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int bps = 0;
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_round<CodecStd, 4>, BLOCK, 0));
  eng->tuning.blocks_per_sm = (uint32_t)std::max(2, std::min(bps, 4));
  eng->tuning.rounds_per_graph = 8;
  eng->tuning.small_limit = 32;
  out = std::move(eng);
  return GEQ_OK;
}

Engine::~Engine() {
  if (!st) return;
  State &s = *st;
  if (s.stream) cudaStreamSynchronize(s.stream);
  // games still alive keep their memory but lose the pool
  for (DeviceGamesImpl *g : s.live) {
    g->release_all();
    g->owner = nullptr;
  }
  s.live.clear();
  for (auto &g : s.gexec)
    if (g) cudaGraphExecDestroy(g);
  for (auto &g : s.graph)
    if (g) cudaGraphDestroy(g);
  dfree(s.part);
  dfree(s.cnt);
  dfree(s.d_err);
  s.pool.trim();
  if (s.stage) cudaFreeHost(s.stage);
  if (s.h_ctr) cudaFreeHost(s.h_ctr);
  if (s.ev0) cudaEventDestroy(s.ev0);
  if (s.ev1) cudaEventDestroy(s.ev1);
  if (s.eva) cudaEventDestroy(s.eva);
  if (s.evb) cudaEventDestroy(s.evb);
  if (s.stream) cudaStreamDestroy(s.stream);
}

uint64_t Engine::game_node_base(const DeviceGamesImpl &dg, uint32_t g) { return dg.node_base[g]; }

// Pack the games into pinned staging and move them to the device.
geq_status Engine::upload(std::vector<GameInput> &games, GamesPtr &out) {
  State &s = *st;
  if (games.empty()) return fail(GEQ_ERR_INVALID_INPUT, "no games");
  bool packed = true;
  for (const GameInput &gi : games) packed = packed && gi.block && !gi.init;
  if (packed) return upload_blocks(games, out);
#if GEQ_PATH_PROFILE
  const auto tu0 = std::chrono::steady_clock::now();
  auto tsince = [&]() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tu0).count(); };
#endif
  GamesPtr dg(new DeviceGamesImpl());
  dg->owner = &s;
  s.live.insert(dg.get());
  dg->conf = Conf(games[0].g.conf);
  if (!dg->conf.supported())
    return fail(GEQ_ERR_UNSUPPORTED, "EnergyConf {%u, %u} is outside the device codecs", dg->conf.elements,
                dg->conf.max);
  dg->generic = !dg->conf.standard() || (tuning.flags & GEQ_TUNE_FORCE_GENERIC);
  dg->n_games = (uint32_t)games.size();
  dg->node_base.assign(dg->n_games + 1, 0);
  dg->edge_base.assign(dg->n_games + 1, 0);
  unsigned long long init_total = 0, n_reach = 0;
  bool any_init = false;
  // standard reach and row checks on the device when every game asks for it
  dg->std_reach = true;
  dg->rows_on_device = true;
  for (const GameInput &gi : games) {
    dg->std_reach = dg->std_reach && gi.std_reach;
    dg->rows_on_device = dg->rows_on_device && gi.rows_unchecked;
  }
  for (uint32_t g = 0; g < dg->n_games; g++) {
    const GameInput &gi = games[g];
    if (!(Conf(gi.g.conf) == dg->conf)) return fail(GEQ_ERR_INVALID_INPUT, "games of one batch need one EnergyConf");
    dg->node_base[g + 1] = dg->node_base[g] + gi.g.n_vertices;
    dg->edge_base[g + 1] = dg->edge_base[g] + gi.g.row_offsets[gi.g.n_vertices];
    if (gi.init) { any_init = true; init_total += gi.init->offsets[gi.init->n_vertices]; }
    n_reach += gi.n_reach;
  }
  dg->N = dg->node_base.back();
  dg->M = dg->edge_base.back();
  if (dg->N >= 0xFFFFFFF0ull || dg->M >= 0xFFFFFFF0ull)
    return fail(GEQ_ERR_INVALID_INPUT, "too many positions/edges for 32-bit ids (%llu, %llu)", dg->N, dg->M);
  const unsigned long long N = dg->N, M = dg->M;
  // arena layout: [zero energy][initial lists ...]
  dg->init_total = 1 + init_total;
  dg->n_reach = n_reach;
  // staging layout
  size_t off_row = 0, off_col = off_row + (N + 1) * 4, off_wt = off_col + M * 4, off_flags = off_wt + M * 4;
  size_t off_reach = (off_flags + N + 15) & ~size_t(15);
  size_t off_init = off_reach + n_reach * 4;
  size_t off_desc = off_init + dg->init_total * 4;
  off_desc = (off_desc + 15) & ~size_t(15);
  size_t off_base = off_desc + (any_init ? N * 8 : 0);
  size_t total_bytes = off_base + (dg->n_games + 1) * 8 * 3;
  geq_status stt = ensure_stage(s, total_bytes);
  if (stt) return stt;
  char *H = s.stage;
  uint32_t *h_row = (uint32_t *)(H + off_row), *h_col = (uint32_t *)(H + off_col), *h_wt = (uint32_t *)(H + off_wt);
  uint8_t *h_flags = (uint8_t *)(H + off_flags);
  uint32_t *h_reach = (uint32_t *)(H + off_reach), *h_init = (uint32_t *)(H + off_init);
  unsigned long long *h_desc = (unsigned long long *)(H + off_desc);
  unsigned long long *h_nb = (unsigned long long *)(H + off_base);
  unsigned long long *h_eb = h_nb + (dg->n_games + 1);
  unsigned long long *h_gn = h_eb + (dg->n_games + 1);
  std::vector<CopyJob> copies;
  copies.reserve(4 * (size_t)dg->n_games);
  unsigned long long ri = 0, ii = 1;
  h_init[0] = 0;  // the zero energy of standard initialisation
  for (uint32_t g = 0; g < dg->n_games; g++) {
    const GameInput &gi = games[g];
    const uint32_t n = gi.g.n_vertices;
    const unsigned long long nb = dg->node_base[g], eb = dg->edge_base[g], m = dg->edge_base[g + 1] - eb;
    copies.push_back(CopyJob{h_row + nb, gi.g.row_offsets, (size_t)n * 4});
    if (m) {
      copies.push_back(CopyJob{h_col + eb, gi.g.column_indices, (size_t)m * 4});
      copies.push_back(CopyJob{h_wt + eb, gi.g.weights, (size_t)m * 4});
    }
    copies.push_back(CopyJob{h_flags + nb, gi.g.attacker_pos, n});
    for (uint32_t i = 0; i < gi.n_reach; i++) h_reach[ri++] = gi.to_reach[i] + (uint32_t)nb;
    if (any_init) {
      if (gi.init) {
        const unsigned long long t = gi.init->offsets[n];
        copies.push_back(CopyJob{h_init + ii, gi.init->data, (size_t)t * 4});
        for (uint32_t v = 0; v < n; v++) {
          unsigned long long o = gi.init->offsets[v], c = gi.init->offsets[v + 1] - o;
          h_desc[nb + v] = ((ii + o) << 24) | c;
        }
        ii += t;
      } else {
        for (uint32_t v = 0; v < n; v++) h_desc[nb + v] = 0ull;
        for (uint32_t i = 0; i < gi.n_reach; i++) h_desc[nb + gi.to_reach[i]] = (0ull << 24) | 1ull;
      }
    }
    h_nb[g] = nb;
    h_eb[g] = eb;
    h_gn[g] = n;
  }
  h_row[N] = (uint32_t)M;
  h_nb[dg->n_games] = N;
  h_eb[dg->n_games] = M;
  h_gn[dg->n_games] = 0;

  // device allocations (pooled); the uploaded inputs share one block laid
  // out like the staging buffer, so any window of it is one copy
  DeviceGamesImpl &D = *dg;
  if (!D.alloc(D.inbuf, total_bytes))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "device allocation of %zu input bytes failed", total_bytes);
  D.row = (uint32_t *)(D.inbuf + off_row);
  D.col = (uint32_t *)(D.inbuf + off_col);
  D.wt = (uint32_t *)(D.inbuf + off_wt);
  D.flags = (uint8_t *)(D.inbuf + off_flags);
  D.reach = (uint32_t *)(D.inbuf + off_reach);
  D.init_data = (uint32_t *)(D.inbuf + off_init);
  D.d_node_base = (unsigned long long *)(D.inbuf + off_base);
  if (any_init) D.desc_init = (unsigned long long *)(D.inbuf + off_desc);
  geq_status ast = alloc_work(D, any_init);
  if (ast) return ast;
  cudaStream_t S = s.stream;
#if GEQ_PATH_PROFILE
  const double t_stage0 = tsince();
#endif
  geq_status ust = staged_upload(copies, H, D.inbuf, total_bytes, S);
#if GEQ_PATH_PROFILE
  const double t_stage1 = tsince();
  std::fprintf(stderr, "GEQ_UPLOAD host_prep_ms %.2f staged_ms %.2f bytes %zu\n", t_stage0, t_stage1 - t_stage0,
               total_bytes);
#endif
  if (ust) return ust;
  return finish_upload(dg, any_init, out);
}

// Games that each sit in one packed host block (GameInput::block, page-locked
// when the caller could get it so): one copy per block into a device scratch
// area, unpacked there into the batch's arrays by k_unpack_games, so the
// host copies nothing; the small per-game tables go through the staging
// buffer.  The device half is the one of upload().
geq_status Engine::upload_blocks(std::vector<GameInput> &games, GamesPtr &out) {
  State &s = *st;
  const uint32_t G = (uint32_t)games.size();
  GamesPtr dg(new DeviceGamesImpl());
  dg->owner = &s;
  s.live.insert(dg.get());
  dg->conf = Conf(games[0].g.conf);
  if (!dg->conf.supported())
    return fail(GEQ_ERR_UNSUPPORTED, "EnergyConf {%u, %u} is outside the device codecs", dg->conf.elements,
                dg->conf.max);
  dg->generic = !dg->conf.standard() || (tuning.flags & GEQ_TUNE_FORCE_GENERIC);
  dg->n_games = G;
  dg->node_base.assign(G + 1, 0);
  dg->edge_base.assign(G + 1, 0);
  dg->std_reach = true;
  dg->rows_on_device = true;
  unsigned long long n_reach = 0, words = 0;
  for (uint32_t g = 0; g < G; g++) {
    const GameInput &gi = games[g];
    if (!(Conf(gi.g.conf) == dg->conf)) return fail(GEQ_ERR_INVALID_INPUT, "games of one batch need one EnergyConf");
    const uint64_t n = gi.g.n_vertices, m = gi.g.row_offsets[n];
    if (gi.block_words != packed_game_words(n, m, gi.n_reach))
      return fail(GEQ_ERR_INTERNAL, "packed block of game %u has %zu words, expected %zu", g, gi.block_words,
                  packed_game_words(n, m, gi.n_reach));
    dg->std_reach = dg->std_reach && gi.std_reach;
    dg->rows_on_device = dg->rows_on_device && gi.rows_unchecked;
    dg->node_base[g + 1] = dg->node_base[g] + n;
    dg->edge_base[g + 1] = dg->edge_base[g] + m;
    n_reach += gi.n_reach;
    words += gi.block_words;
  }
  dg->N = dg->node_base.back();
  dg->M = dg->edge_base.back();
  if (dg->N >= 0xFFFFFFF0ull || dg->M >= 0xFFFFFFF0ull)
    return fail(GEQ_ERR_INVALID_INPUT, "too many positions/edges for 32-bit ids (%llu, %llu)", dg->N, dg->M);
  const unsigned long long N = dg->N, M = dg->M;
  dg->init_total = 1;  // the zero energy of standard initialisation
  dg->n_reach = n_reach;
  // the input block's layout is upload()'s (no initial lists); two tables
  // follow it: each game's first word in the scratch area and reach base
  const size_t off_row = 0, off_col = off_row + (N + 1) * 4, off_wt = off_col + M * 4, off_flags = off_wt + M * 4;
  const size_t off_reach = (off_flags + N + 15) & ~size_t(15);
  const size_t off_init = off_reach + n_reach * 4;
  const size_t off_base = (off_init + 4 + 15) & ~size_t(15);
  const size_t off_boff = off_base + (G + 1) * 8 * 3;
  const size_t off_rb = off_boff + (G + 1) * 8;
  const size_t total_bytes = off_rb + (G + 1) * 8;
  const size_t tail = total_bytes - off_init;  // staged: init word and the tables
  geq_status stt = ensure_stage(s, tail);
  if (stt) return stt;
  char *H = s.stage;
  ((uint32_t *)H)[0] = 0;
  unsigned long long *h_nb = (unsigned long long *)(H + (off_base - off_init));
  unsigned long long *h_eb = h_nb + (G + 1), *h_gn = h_eb + (G + 1);
  unsigned long long *h_boff = (unsigned long long *)(H + (off_boff - off_init));
  unsigned long long *h_rb = (unsigned long long *)(H + (off_rb - off_init));
  unsigned long long w = 0, r = 0;
  for (uint32_t g = 0; g < G; g++) {
    h_nb[g] = dg->node_base[g];
    h_eb[g] = dg->edge_base[g];
    h_gn[g] = games[g].g.n_vertices;
    h_boff[g] = w;
    h_rb[g] = r;
    w += games[g].block_words;
    r += games[g].n_reach;
  }
  h_nb[G] = N;
  h_eb[G] = M;
  h_gn[G] = 0;
  h_boff[G] = w;
  h_rb[G] = r;
  DeviceGamesImpl &D = *dg;
  if (!D.alloc(D.inbuf, total_bytes))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "device allocation of %zu input bytes failed", total_bytes);
  D.row = (uint32_t *)(D.inbuf + off_row);
  D.col = (uint32_t *)(D.inbuf + off_col);
  D.wt = (uint32_t *)(D.inbuf + off_wt);
  D.flags = (uint8_t *)(D.inbuf + off_flags);
  D.reach = (uint32_t *)(D.inbuf + off_reach);
  D.init_data = (uint32_t *)(D.inbuf + off_init);
  D.d_node_base = (unsigned long long *)(D.inbuf + off_base);
  geq_status ast = alloc_work(D, false);
  if (ast) return ast;
  uint32_t *raw = (uint32_t *)s.pool.get(std::max<size_t>(words, 1) * 4);
  if (!raw) return fail(GEQ_ERR_OUT_OF_MEMORY, "device scratch of %llu words for the game blocks", words);
  struct Give {
    DevPool &pool;
    void *p;
    size_t b;
    ~Give() { pool.put(p, b); }  // later users of the pool run behind this upload on the stream
  } give{s.pool, raw, std::max<size_t>(words, 1) * 4};
  cudaStream_t S = s.stream;
  for (uint32_t g = 0; g < G; g++)
    if (games[g].block_words)
      CU(cudaMemcpyAsync(raw + h_boff[g], games[g].block, games[g].block_words * 4, cudaMemcpyHostToDevice, S));
  CU(cudaMemcpyAsync(D.inbuf + off_init, H, tail, cudaMemcpyHostToDevice, S));
  if (words) {
    const unsigned grid = (unsigned)std::max<unsigned long long>(
        1, std::min<unsigned long long>((words + 255) / 256, (unsigned long long)n_sms * 8));
    k_unpack_games<<<grid, 256, 0, S>>>(raw, (const unsigned long long *)(D.inbuf + off_boff), D.d_node_base,
                                        D.d_node_base + (G + 1), (const unsigned long long *)(D.inbuf + off_rb), G,
                                        words, D.row, D.col, D.wt, D.flags, D.reach, N, M);
  }
  return finish_upload(dg, false, out);
}

// Games already on the device in the solver's input layout (built by the
// device game builder on this engine's stream): copied into one input block
// like a host upload, then the same device half.
geq_status Engine::upload_built(const BuiltGames &b, GamesPtr &out) {
  State &s = *st;
  if (b.n_games == 0) return fail(GEQ_ERR_INVALID_INPUT, "no games");
  GamesPtr dg(new DeviceGamesImpl());
  dg->owner = &s;
  s.live.insert(dg.get());
  dg->conf = Conf(6, 3);
  dg->generic = (tuning.flags & GEQ_TUNE_FORCE_GENERIC) != 0;
  dg->n_games = b.n_games;
  dg->node_base.assign(dg->n_games + 1, 0);
  dg->edge_base.assign(dg->n_games + 1, 0);
  for (uint32_t g = 0; g < b.n_games; g++) {
    dg->node_base[g + 1] = dg->node_base[g] + b.n_nodes[g];
    dg->edge_base[g + 1] = dg->edge_base[g] + b.n_edges[g];
  }
  dg->N = dg->node_base.back();
  dg->M = dg->edge_base.back();
  if (dg->N != b.N || dg->M != b.M) return fail(GEQ_ERR_INTERNAL, "built games: sizes disagree");
  if (dg->N >= 0xFFFFFFF0ull || dg->M >= 0xFFFFFFF0ull)
    return fail(GEQ_ERR_INVALID_INPUT, "too many positions/edges for 32-bit ids (%llu, %llu)", dg->N, dg->M);
  dg->std_reach = true;
  dg->rows_on_device = false;  // rows are valid by construction
  dg->init_total = 1;
  dg->n_reach = 0;
  const unsigned long long N = dg->N, M = dg->M;
  const size_t off_row = 0, off_col = off_row + (N + 1) * 4, off_wt = off_col + M * 4, off_flags = off_wt + M * 4;
  const size_t off_init = (off_flags + N + 15) & ~size_t(15);
  const size_t off_base = (off_init + 4 + 15) & ~size_t(15);
  const size_t total_bytes = off_base + (dg->n_games + 1) * 8 * 3;
  const size_t small = 16 + (dg->n_games + 1) * 8 * 3;
  geq_status stt = ensure_stage(s, small);
  if (stt) return stt;
  uint32_t *h_tail = (uint32_t *)s.stage;  // row[N] = M, init[0] = 0
  h_tail[0] = (uint32_t)M;
  h_tail[1] = 0;
  unsigned long long *h_nb = (unsigned long long *)(s.stage + 16);
  unsigned long long *h_eb = h_nb + (dg->n_games + 1), *h_gn = h_eb + (dg->n_games + 1);
  for (uint32_t g = 0; g <= dg->n_games; g++) {
    h_nb[g] = dg->node_base[g];
    h_eb[g] = dg->edge_base[g];
    h_gn[g] = g < dg->n_games ? b.n_nodes[g] : 0;
  }
  DeviceGamesImpl &D = *dg;
  if (!D.alloc(D.inbuf, total_bytes))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "device allocation of %zu input bytes failed", total_bytes);
  D.row = (uint32_t *)(D.inbuf + off_row);
  D.col = (uint32_t *)(D.inbuf + off_col);
  D.wt = (uint32_t *)(D.inbuf + off_wt);
  D.flags = (uint8_t *)(D.inbuf + off_flags);
  D.reach = (uint32_t *)(D.inbuf + off_init);
  D.init_data = (uint32_t *)(D.inbuf + off_init);
  D.d_node_base = (unsigned long long *)(D.inbuf + off_base);
  geq_status ast = alloc_work(D, false);
  if (ast) return ast;
  cudaStream_t S = s.stream;
  CU(cudaMemcpyAsync(D.row, b.row_rel, N * 4, cudaMemcpyDeviceToDevice, S));
  CU(cudaMemcpyAsync(D.row + N, h_tail, 4, cudaMemcpyHostToDevice, S));
  if (M) {
    CU(cudaMemcpyAsync(D.col, b.col, M * 4, cudaMemcpyDeviceToDevice, S));
    CU(cudaMemcpyAsync(D.wt, b.wt, M * 4, cudaMemcpyDeviceToDevice, S));
  }
  CU(cudaMemcpyAsync(D.flags, b.att, N, cudaMemcpyDeviceToDevice, S));
  CU(cudaMemcpyAsync(D.init_data, h_tail + 1, 4, cudaMemcpyHostToDevice, S));
  CU(cudaMemcpyAsync(D.d_node_base, h_nb, (dg->n_games + 1) * 8 * 3, cudaMemcpyHostToDevice, S));
  return finish_upload(dg, false, out);
}

// Work arrays of an upload: reverse CSR, descriptors, frontier, arena.
geq_status Engine::alloc_work(DeviceGamesImpl &D, bool any_init) {
  const unsigned long long N = D.N, M = D.M;
  if (!D.alloc(D.rrow, N + 1) || !D.alloc(D.rcol, M) || !D.alloc(D.desc, N) ||
      (!any_init && !D.alloc(D.desc_init, N)) || !D.alloc(D.slot_new, N) || !D.alloc(D.mark, 2 * ((N + 31) / 32)) ||
      !D.alloc(D.front0, N) || !D.alloc(D.front1, N) || !D.alloc(D.ctr, 1) ||
      !D.alloc(D.fpart, 2 * (size_t)std::max(1, n_sms * GEQ_FRONTIER_BLOCKS_PER_SM)) || !D.alloc(D.abits, (N + 31) / 32) ||
      !D.alloc(D.bigq, N) || !D.alloc(D.cw, M))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "device allocation for %llu positions / %llu edges failed", N, M);
  unsigned long long cap = std::max<unsigned long long>(4ull * (D.init_total + N) + (1ull << 20), 1ull << 22);
  if (!D.alloc(D.arena[0], cap)) return fail(GEQ_ERR_OUT_OF_MEMORY, "energy arena of %llu words", cap);
  D.arena_cap[0] = DevPool::round_size(cap * 4) / 4;
  return GEQ_OK;
}

// Device half of an upload, once the inputs are in D.inbuf: row and column
// ids into the global id space, checks, initial state, reverse CSR.
geq_status Engine::finish_upload(GamesPtr &dg, bool any_init, GamesPtr &out) {
  State &s = *st;
  DeviceGamesImpl &D = *dg;
  const unsigned long long N = D.N, M = D.M, n_reach = D.n_reach;
  cudaStream_t S = s.stream;
  CU(cudaMemsetAsync(D.mark, 0, 2 * ((N + 31) / 32) * 4, S));
  CU(cudaMemsetAsync(s.d_err, 0, 4, S));
  const unsigned grid = (unsigned)std::max(1, n_sms * 8);
  if (N && D.rows_on_device)
    k_check_rows<<<grid, 256, 0, S>>>(D.row, N, D.d_node_base, D.d_node_base + (D.n_games + 1), D.n_games,
                                      s.d_err);
  if (D.n_games > 1)
    k_fix_rows<<<grid, 256, 0, S>>>(D.row, N, D.d_node_base, D.d_node_base + (D.n_games + 1), D.n_games);
  if (!any_init) {
    if (N) CU(cudaMemsetAsync(D.desc_init, 0, N * 8, S));
    if (D.std_reach && N) k_std_reach<<<grid, 256, 0, S>>>(D.row, D.flags, N, D.desc_init);
    else if (n_reach)
      k_init_reach<<<(unsigned)std::min<unsigned long long>((n_reach + 255) / 256, 4096), 256, 0, S>>>(
          D.desc_init, D.reach, n_reach);
  }
  // successor ids into the global id space, checked against each game's size
  k_fix_cols<<<grid, 256, 0, S>>>(D.col, M, D.d_node_base, D.d_node_base + (D.n_games + 1), D.n_games,
                                  D.d_node_base + 2 * (D.n_games + 1), s.d_err);
  k_check_weights<<<grid, 256, 0, S>>>(D.wt, M, D.conf.elements, D.conf.update_bits(), D.conf.update_mask(),
                                       s.d_err);
  // reverse CSR
  geq_status es = ensure_cnt(s, N + 1);
  if (es) return es;
  CU(cudaMemsetAsync(s.cnt, 0, (N + 1) * 4, S));
  k_indegree<<<grid, 256, 0, S>>>(D.col, M, N, s.cnt, s.d_err);
  unsigned long long *roff = (unsigned long long *)s.pool.get((N + 1) * 8);
  if (!roff) return fail(GEQ_ERR_OUT_OF_MEMORY, "reverse offsets");
  unsigned long long launches = 0;
  geq_status a = scan_u32(s, s.cnt, N, roff, launches);
  if (a) { s.pool.put(roff, (N + 1) * 8); return a; }
  k_u64_to_u32<<<grid, 256, 0, S>>>(roff, N + 1, D.rrow);
  CU(cudaMemcpyAsync(s.cnt, D.rrow, N * 4, cudaMemcpyDeviceToDevice, S));
  k_fill_reverse<<<grid, 256, 0, S>>>(D.row, D.col, N, M, s.cnt, D.rcol);
  if (N) k_abits<<<grid, 256, 0, S>>>(D.flags, N, (uint32_t)((N + 31) / 32), D.abits);
  if (M) {
    if (D.generic) k_pack_edges<CodecGen><<<grid, 256, 0, S>>>(D.col, D.wt, M, D.cw);
    else k_pack_edges<CodecStd><<<grid, 256, 0, S>>>(D.col, D.wt, M, D.cw);
  }
  CU(cudaMemcpyAsync(&s.h_ctr->pad, s.d_err, 4, cudaMemcpyDeviceToHost, S));
#if GEQ_PATH_PROFILE
  const auto tw0 = std::chrono::steady_clock::now();
#endif
  CU(cudaStreamSynchronize(S));
#if GEQ_PATH_PROFILE
  std::fprintf(stderr, "GEQ_UPLOAD wait_ms %.2f\n",
               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw0).count());
#endif
  s.pool.put(roff, (N + 1) * 8);
  CU(cudaGetLastError());
  const uint32_t h_err = s.h_ctr->pad;
  if (h_err & 1u) return fail(GEQ_ERR_INVALID_INPUT, "Node index too high: a successor index is out of range");
  if (h_err & 2u) return fail(GEQ_ERR_INVALID_INPUT, "an edge update names no element or sets padding bits");
  if (h_err & 4u) return fail(GEQ_ERR_INVALID_INPUT, "row_offsets must start at 0 and must not decrease");
  KParams &kp = D.kp;
  kp.row = D.row; kp.col = D.col; kp.wt = D.wt; kp.rrow = D.rrow; kp.rcol = D.rcol;
  kp.flags = D.flags; kp.desc = D.desc; kp.mark = D.mark; kp.front0 = D.front0; kp.front1 = D.front1;
  kp.slot_new = D.slot_new; kp.ctr = D.ctr; kp.n_nodes = N; kp.n_edges = M;
  kp.mwords = (uint32_t)((N + 31) / 32);
  kp.fpart = D.fpart;
  kp.fblocks = (uint32_t)std::max(1, n_sms * GEQ_FRONTIER_BLOCKS_PER_SM);
  kp.abits = D.abits;
  kp.bigq = D.bigq;
  kp.cw = D.cw;
  kp.missing = nullptr;
  kp.el = D.conf.elements; kp.mx = D.conf.max; kp.eb = D.conf.energy_bits(); kp.em = D.conf.energy_mask();
  kp.ub = D.conf.update_bits(); kp.um = D.conf.update_mask();
  kp.small_limit = (tuning.flags & GEQ_TUNE_FORCE_LARGE) ? 0u : std::min<uint32_t>(tuning.small_limit, 32);
  kp.thread_path = (tuning.flags & (GEQ_TUNE_FORCE_LARGE | GEQ_TUNE_NO_THREAD_PATH)) ? 0u : 1u;
  kp.ib = D.conf.elements * D.conf.energy_bits();
  kp.ibm = kp.ib >= 32 ? 0xFFFFFFFFu : ((1u << kp.ib) - 1u);
  kp.inl = std::min<uint32_t>(7u, 60u / kp.ib);
  out = std::move(dg);
  return GEQ_OK;
}

static geq_status compact(Engine &E, DeviceGamesImpl &dg, unsigned long long &launches) {
  Engine::State &s = *E.st;
  cudaStream_t S = s.stream;
  const unsigned long long N = dg.N;
  geq_status a = ensure_cnt(s, N + 1);
  if (a) return a;
  unsigned long long *noff = (unsigned long long *)s.pool.get((N + 1) * 8);
  if (!noff) return fail(GEQ_ERR_OUT_OF_MEMORY, "compaction offsets");
  const unsigned grid = (unsigned)std::max(1, E.n_sms * 8);
  k_arena_counts<<<grid, 256, 0, S>>>(dg.desc, N, s.cnt);
  launches++;
  if ((a = scan_u32(s, s.cnt, N, noff, launches))) { s.pool.put(noff, (N + 1) * 8); return a; }
  unsigned long long total = 0;
  CU(cudaMemcpyAsync(&s.h_ctr->positions, noff + N, 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  total = s.h_ctr->positions;
  const int alt = dg.arena_cur ^ 1;
  unsigned long long need = std::max<unsigned long long>(dg.arena_cap[dg.arena_cur], 4 * total + (1ull << 20));
  if (dg.arena_cap[alt] < need) {
    if (dg.arena[alt]) dg.release(dg.arena[alt]);
    dg.arena_cap[alt] = 0;
    if (!dg.alloc(dg.arena[alt], need)) { s.pool.put(noff, (N + 1) * 8); return fail(GEQ_ERR_OUT_OF_MEMORY, "arena"); }
    dg.arena_cap[alt] = DevPool::round_size(need * 4) / 4;
  }
  k_compact<<<grid, 256, 0, S>>>(dg.desc, N, noff, dg.arena[dg.arena_cur], dg.arena[alt]);
  k_set_arena<<<1, 1, 0, S>>>(dg.ctr, dg.arena[alt], dg.arena_cap[alt], total);
  launches += 2;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(S));
  s.pool.put(noff, (N + 1) * 8);
  dg.arena_cur = alt;
  return GEQ_OK;
}

// Lane-path limits from geq_tuning.lane_limits (a zero field: the largest).
static void set_lane_limits(KParams &kp, const geq_tuning &t) {
  const uint32_t d = t.lane_limits & 0xFFu, w = (t.lane_limits >> 8) & 0xFFu, k = (t.lane_limits >> 16) & 0xFFu;
  kp.td = d ? std::min(d, TD) : TD;
  kp.tw = w ? std::min(w, TW) : TW;
  kp.tk = k ? std::min(k, TK) : TK;
}

template <class Cd>
static void launch_round(Engine &E, const KParams &kp, cudaStream_t S, cudaEvent_t ea = nullptr,
                         cudaEvent_t eb = nullptr) {
  const uint32_t bps = std::min<uint32_t>(std::max<uint32_t>(E.tuning.blocks_per_sm, 2), 5);
  const unsigned grid = (unsigned)std::max<uint32_t>(1, E.n_sms * bps);
  if (ea) cudaEventRecord(ea, S);
  if (bps == 2) k_round<Cd, 2><<<grid, BLOCK, 0, S>>>(kp);
  else if (bps == 3) k_round<Cd, 3><<<grid, BLOCK, 0, S>>>(kp);
  else if (bps == 4) k_round<Cd, 4><<<grid, BLOCK, 0, S>>>(kp);
  else k_round<Cd, 5><<<grid, BLOCK, 0, S>>>(kp);
  k_round_big<Cd><<<(unsigned)std::max(1, E.n_sms * GEQ_BIG_BLOCKS_PER_SM), BLOCK, 0, S>>>(kp);
  if (eb) cudaEventRecord(eb, S);
  k_commit<<<kp.fblocks, 256, 0, S>>>(kp);
  k_ffill<<<kp.fblocks, 256, 0, S>>>(kp);
}

// One captured graph of R rounds per codec, shared by every upload: before a
// solve its kernel nodes are pointed at the parameters of that upload.
static geq_status round_graph(Engine &E, const KParams &kp, bool generic, uint32_t R, cudaGraphExec_t &out) {
  Engine::State &s = *E.st;
  const int k = generic ? 1 : 0;
  if (!(s.gexec[k] && s.g_rounds[k] == R && s.g_bps[k] == E.tuning.blocks_per_sm)) {
    if (s.gexec[k]) { cudaGraphExecDestroy(s.gexec[k]); s.gexec[k] = nullptr; }
    if (s.graph[k]) { cudaGraphDestroy(s.graph[k]); s.graph[k] = nullptr; }
    cudaStream_t cs;
    CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      for (uint32_t r = 0; r < R; r++) {
        if (generic) launch_round<CodecGen>(E, kp, cs);
        else launch_round<CodecStd>(E, kp, cs);
      }
      ce = cudaStreamEndCapture(cs, &s.graph[k]);
    }
    cudaStreamDestroy(cs);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&s.gexec[k], s.graph[k], 0);
    size_t n = 0;
    if (ce == cudaSuccess) ce = cudaGraphGetNodes(s.graph[k], nullptr, &n);
    s.gnodes[k].assign(n, nullptr);
    if (ce == cudaSuccess && n) ce = cudaGraphGetNodes(s.graph[k], s.gnodes[k].data(), &n);
    if (ce != cudaSuccess) return fail(GEQ_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    s.g_rounds[k] = R;
    s.g_bps[k] = E.tuning.blocks_per_sm;
    s.g_kp[k] = kp;
    s.g_kp_valid[k] = true;
  } else if (!(s.g_kp_valid[k] && std::memcmp(&s.g_kp[k], &kp, sizeof(KParams)) == 0)) {
    s.g_kp_valid[k] = false;
    for (cudaGraphNode_t node : s.gnodes[k]) {
      cudaGraphNodeType t;
      CU(cudaGraphNodeGetType(node, &t));
      if (t != cudaGraphNodeTypeKernel) continue;
      cudaKernelNodeParams np;
      CU(cudaGraphKernelNodeGetParams(node, &np));
      void *args[1] = {(void *)&kp};
      np.kernelParams = args;
      np.extra = nullptr;
      CU(cudaGraphExecKernelNodeSetParams(s.gexec[k], node, &np));
    }
    s.g_kp[k] = kp;
    s.g_kp_valid[k] = true;
  }
  out = s.gexec[k];
  return GEQ_OK;
}

// A solve in steps: solve_begin restarts from the uploaded initial state and
// builds the first frontier; every solve_step runs one CUDA graph of R
// worklist rounds (or one round as plain launches), compacts the arena when
// needed and reports whether the frontier is empty.  solve() is begin + steps
// until done; the serving loop interleaves the steps of several uploads on one
// stream and retires games as their part of the frontier empties.
geq_status Engine::solve_begin(DeviceGamesImpl &dg) {
  State &s = *st;
  cudaStream_t S = s.stream;
  DeviceGamesImpl::Progress &pr = dg.prog;
  pr = DeviceGamesImpl::Progress{};
  pr.t_start = std::chrono::steady_clock::now();
  // restart from the uploaded initial state
  const int a0 = dg.arena_cur;
  CU(cudaEventRecord(s.ev0, S));
  if (dg.N) CU(cudaMemcpyAsync(dg.desc, dg.desc_init, dg.N * 8, cudaMemcpyDeviceToDevice, S));
  CU(cudaMemcpyAsync(dg.arena[a0], dg.init_data, dg.init_total * 4, cudaMemcpyDeviceToDevice, S));
  if (dg.next_stamp > 0xF0000000u) dg.next_stamp = 1;
  CU(cudaMemsetAsync(dg.mark, 0, 2ull * dg.kp.mwords * 4, S));
  dg.kp.cw = (tuning.flags & GEQ_TUNE_NO_EDGE_PAIRS) ? nullptr : dg.cw;
  // GEQ_TUNE_READY: defenders wait for their successors' lists (counted per
  // defender, set up at the first such solve); else every predecessor of a
  // changed position is pushed, as the reference's visit lists do
  dg.kp.missing = nullptr;
  if ((tuning.flags & GEQ_TUNE_READY) && dg.N) {
    if (!dg.missing) {
      if (!dg.alloc(dg.missing, dg.N) || !dg.alloc(dg.missing_init, dg.N))
        return fail(GEQ_ERR_OUT_OF_MEMORY, "defender counts for %llu positions", dg.N);
      k_missing_init<<<(unsigned)std::max(1, n_sms * 8), 256, 0, S>>>(dg.kp, dg.desc_init, dg.missing_init);
    }
    CU(cudaMemcpyAsync(dg.missing, dg.missing_init, dg.N * 4, cudaMemcpyDeviceToDevice, S));
    dg.kp.missing = dg.missing;
  }
  Ctr h{};
  h.arena = dg.arena[a0];
  h.arena_cap = dg.arena_cap[a0];
  h.arena_top = dg.init_total;
  h.stamp = dg.next_stamp;
  *s.h_ctr = h;
  CU(cudaMemcpyAsync(dg.ctr, s.h_ctr, sizeof(Ctr), cudaMemcpyHostToDevice, S));
  if (dg.std_reach && dg.N) {
    k_init_frontier_std<<<(unsigned)std::max(1, n_sms * 16), 256, 0, S>>>(dg.kp);
    if (!dg.off_ranges.empty()) {
      geq_status cr = clear_off_ranges(dg, h.stamp);
      if (cr) return cr;
      pr.launches++;
    }
    k_fcount<<<dg.kp.fblocks, 256, 0, S>>>(dg.kp);
    k_ffill<<<dg.kp.fblocks, 256, 0, S>>>(dg.kp);
    pr.launches += 3;
  } else if (dg.n_reach) {
    const unsigned grid = (unsigned)std::max<unsigned long long>(
        1, std::min<unsigned long long>((dg.n_reach + 7) / 8, (unsigned long long)n_sms * 16));
    k_init_frontier<<<grid, 256, 0, S>>>(dg.kp, dg.reach, dg.n_reach);
    if (!dg.off_ranges.empty()) {
      geq_status cr = clear_off_ranges(dg, h.stamp);
      if (cr) return cr;
      pr.launches++;
    }
    k_fcount<<<dg.kp.fblocks, 256, 0, S>>>(dg.kp);
    k_ffill<<<dg.kp.fblocks, 256, 0, S>>>(dg.kp);
    pr.launches += 3;
  }
  CU(cudaGetLastError());
  return GEQ_OK;
}

// Games that are not to be solved: their initial frontier is cleared, so no
// position of theirs is ever computed (games share no edges).
void Engine::skip_games(DeviceGamesImpl &dg, const std::vector<uint32_t> &games) {
  for (uint32_t g : games) {
    dg.off_ranges.push_back(dg.node_base[g]);
    dg.off_ranges.push_back(dg.node_base[g + 1]);
  }
}
geq_status Engine::clear_off_ranges(DeviceGamesImpl &dg, uint32_t stamp) {
  State &s = *st;
  const size_t bytes = dg.off_ranges.size() * 8;
  unsigned long long *d = (unsigned long long *)s.pool.get(bytes);
  if (!d) return fail(GEQ_ERR_OUT_OF_MEMORY, "skipped games");
  CU(cudaMemcpyAsync(d, dg.off_ranges.data(), bytes, cudaMemcpyHostToDevice, s.stream));
  const uint32_t n = (uint32_t)(dg.off_ranges.size() / 2);
  k_clear_ranges<<<std::min<uint32_t>(n, 1024), 256, 0, s.stream>>>(dg.mark + (stamp & 1u) * dg.kp.mwords, d, n);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(s.stream));  // the ranges are pageable host memory
  s.pool.put(d, bytes);
  return GEQ_OK;
}

// Lists of whole games (or only their first position): the selection is
// expanded, counted, scanned and gathered on the device and read back into
// page-locked blocks; solution game i is games[i].
geq_status Engine::download_games(DeviceGamesImpl &dg, const std::vector<uint32_t> &games, bool first_only,
                                  geq_solution &sol) {
  State &s = *st;
  cudaStream_t S = s.stream;
  const uint32_t G = (uint32_t)games.size();
  std::vector<unsigned long long> hb(2 * (size_t)G + 1);  // bases, then prefix of counts
  unsigned long long K = 0;
  for (uint32_t i = 0; i < G; i++) {
    const uint32_t g = games[i];
    hb[i] = dg.node_base[g];
    hb[G + i] = K;
    K += first_only ? 1ull : dg.node_base[g + 1] - dg.node_base[g];
  }
  hb[2 * (size_t)G] = K;
  unsigned long long launches = 0;
  geq_status a = ensure_cnt(s, K + 1);
  if (a) return a;
  const size_t hb_bytes = hb.size() * 8;
  unsigned long long *d_hb = (unsigned long long *)s.pool.get(hb_bytes);
  uint32_t *d_sel = (uint32_t *)s.pool.get(std::max<unsigned long long>(K, 1) * 4);
  unsigned long long *goff = (unsigned long long *)s.pool.get((K + 1) * 8);
  unsigned long long *rel = (unsigned long long *)s.pool.get((K + G) * 8);
  struct Give {
    State &s;
    std::vector<std::pair<void *, size_t>> v;
    ~Give() {
      for (auto &x : v)
        if (x.first) s.pool.put(x.first, x.second);
    }
  } give{s, {{d_hb, hb_bytes}, {d_sel, std::max<unsigned long long>(K, 1) * 4}, {goff, (K + 1) * 8},
             {rel, (K + G) * 8}}};
  if (!d_hb || !d_sel || !goff || !rel) return fail(GEQ_ERR_OUT_OF_MEMORY, "selection of %u games", G);
  CU(cudaMemcpyAsync(d_hb, hb.data(), hb_bytes, cudaMemcpyHostToDevice, S));
  const unsigned grid = (unsigned)std::max(1, n_sms * 8);
  if (K) {
    k_sel_expand<<<grid, 256, 0, S>>>(d_hb, d_hb + G, G, K, d_sel);
    k_sel_counts<<<grid, 256, 0, S>>>(dg.desc, d_sel, K, s.cnt);
  }
  if ((a = scan_u32(s, s.cnt, K, goff, launches))) return a;
  k_rel_offsets<<<grid, 256, 0, S>>>(goff, K, d_hb + G, G, rel);
  unsigned long long total = 0;
  CU(cudaMemcpyAsync(&s.h_ctr->positions, goff + K, 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  total = s.h_ctr->positions;
  uint32_t *out = (uint32_t *)s.pool.get(std::max<unsigned long long>(total, 1) * 4);
  if (!out) return fail(GEQ_ERR_OUT_OF_MEMORY, "selection data");
  give.v.push_back({out, std::max<unsigned long long>(total, 1) * 4});
  if (K) k_sel_gather<<<grid, 256, 0, S>>>(dg.desc, d_sel, K, goff, dg.arena[dg.arena_cur], dg.kp.ib, dg.kp.ibm, out);
  CU(cudaGetLastError());
  sol.energy_size = 1;
  sol.offsets.clear();
  sol.data.clear();
  const bool pinned = sol.off_buf.alloc(s.hpool, (K + G) * 8) && sol.data_buf.alloc(s.hpool, std::max<unsigned long long>(total, 1) * 4);
  if (!pinned) return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for %llu offsets", K + G);
  CU(cudaMemcpyAsync(sol.off_buf.p, rel, (K + G) * 8, cudaMemcpyDeviceToHost, S));
  if (total) CU(cudaMemcpyAsync(sol.data_buf.p, out, total * 4, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  sol.n_offsets = K + G;
  sol.n_words = total;
  sol.n_vertices.resize(G);
  sol.offsets_base.resize(G);
  sol.data_base.resize(G);
  const unsigned long long *ro = (const unsigned long long *)sol.off_buf.p;
  unsigned long long db = 0;
  for (uint32_t i = 0; i < G; i++) {
    const unsigned long long n = hb[G + i + 1] - hb[G + i];
    sol.n_vertices[i] = (uint32_t)n;
    sol.offsets_base[i] = hb[G + i] + i;
    sol.data_base[i] = db;
    db += ro[hb[G + i] + i + n];
  }
  return GEQ_OK;
}

__global__ void k_active_games(const KParams p, const unsigned long long *node_base, uint32_t n_games,
                               uint8_t *active);

// One step in two halves: step_enqueue launches a CUDA graph of R rounds (or
// one round as plain launches) and the read-back of the control block -- and,
// with `active`, of the games that still have frontier positions -- into
// page-locked memory of the upload, without waiting; step_finish, once the
// stream has been synchronised, handles errors and arena compaction and
// reports whether the frontier is empty.  Several uploads' steps can be
// enqueued back to back and finished after one synchronisation.
geq_status Engine::step_enqueue(DeviceGamesImpl &dg, bool active) {
  State &s = *st;
  cudaStream_t S = s.stream;
  DeviceGamesImpl::Progress &pr = dg.prog;
  set_lane_limits(dg.kp, tuning);
  const bool profile = (tuning.flags & GEQ_TUNE_PROFILE) != 0;
  const bool use_graph = !(tuning.flags & (GEQ_TUNE_NO_GRAPH | GEQ_TUNE_PROFILE));
  const uint32_t R = use_graph ? std::max<uint32_t>(1, tuning.rounds_per_graph) : 1;
  const size_t hbytes = sizeof(Ctr) + dg.n_games;
  if (!dg.hstep.p && !dg.hstep.alloc(s.hpool, hbytes)) return fail(GEQ_ERR_OUT_OF_MEMORY, "step read-back");
  if (use_graph) {
    // the shared graph is pointed at this upload's parameters when they differ
    cudaGraphExec_t gexec = nullptr;
    geq_status g = round_graph(*this, dg.kp, dg.generic, R, gexec);
    if (g) return g;
    CU(cudaGraphLaunch(gexec, S));
  } else {
    cudaEvent_t ea = profile ? s.eva : nullptr, eb = profile ? s.evb : nullptr;
    if (dg.generic) launch_round<CodecGen>(*this, dg.kp, S, ea, eb);
    else launch_round<CodecStd>(*this, dg.kp, S, ea, eb);
  }
  pr.launches += 4ull * R;
  CU(cudaMemcpyAsync(dg.hstep.p, dg.ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
  dg.step_active = active && dg.n_games > 0;
  if (dg.step_active) {
    if (!dg.d_act && !dg.alloc(dg.d_act, dg.n_games)) return fail(GEQ_ERR_OUT_OF_MEMORY, "active flags");
    CU(cudaMemsetAsync(dg.d_act, 0, dg.n_games, S));
    k_active_games<<<(unsigned)std::max(1, n_sms * 4), 256, 0, S>>>(dg.kp, dg.d_node_base, dg.n_games, dg.d_act);
    CU(cudaMemcpyAsync((char *)dg.hstep.p + sizeof(Ctr), dg.d_act, dg.n_games, cudaMemcpyDeviceToHost, S));
  }
  CU(cudaGetLastError());
  return GEQ_OK;
}

geq_status Engine::step_finish(DeviceGamesImpl &dg, bool &done, const uint8_t *&active) {
  State &s = *st;
  DeviceGamesImpl::Progress &pr = dg.prog;
  done = false;
  active = nullptr;
  const Ctr c = *(const Ctr *)dg.hstep.p;
  if (tuning.flags & GEQ_TUNE_PROFILE) {
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, s.eva, s.evb));
    pr.round_ms += ms;
    pr.round_launches++;
  }
  if (c.error) {
    const char *what = (c.error & DERR_BOUNDS) ? "index out of range" :
                       (c.error & DERR_LIST) ? "energy list too long" : "combination too large";
    return fail((c.error & DERR_BOUNDS) ? GEQ_ERR_INTERNAL : GEQ_ERR_OUT_OF_MEMORY,
                "device error %u (%s, line %u)", c.error, what, c.err_line);
  }
  if (c.overflow || c.arena_top > c.arena_cap - c.arena_cap / 4) {
    geq_status a = compact(*this, dg, pr.launches);
    if (a) return a;
    pr.compactions++;
    if (c.overflow) return GEQ_OK;  // the halted rounds run at the next step; nothing retires now
  }
  if (c.fsize[c.cur] == 0) {
    done = true;
    dg.next_stamp = c.stamp + 2u;
    return GEQ_OK;
  }
  // The device work of every launch is bounded; this bounds the host loop in
  // case the frontier never empties (GEQ_SOLVE_TIMEOUT_S seconds, default 600).
  const char *lim_env = std::getenv("GEQ_SOLVE_TIMEOUT_S");
  const double limit_s = lim_env ? std::atof(lim_env) : 600.0;
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - pr.t_start).count();
  if (el > limit_s) return fail(GEQ_ERR_TIMEOUT, "no fixpoint after %llu rounds (%.0f s)", c.rounds, el);
  if (dg.step_active) active = (const uint8_t *)dg.hstep.p + sizeof(Ctr);
  return GEQ_OK;
}

geq_status Engine::sync() {
  CU(cudaStreamSynchronize(st->stream));
  return GEQ_OK;
}

geq_status Engine::solve_step(DeviceGamesImpl &dg, bool &done) {
  geq_status r = step_enqueue(dg, false);
  if (!r) r = sync();
  const uint8_t *active = nullptr;
  if (!r) r = step_finish(dg, done, active);
  return r;
}

geq_status Engine::solve_stats(DeviceGamesImpl &dg, geq_solve_stats *stats) {
  State &s = *st;
  cudaStream_t S = s.stream;
  CU(cudaMemcpyAsync(s.h_ctr, dg.ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  const Ctr c = *s.h_ctr;
  if (stats) {
    *stats = geq_solve_stats{};
    stats->rounds = c.rounds;
    stats->positions_computed = c.positions;
    stats->edges_relaxed = c.edges;
    stats->algorithmic_bytes = c.bytes;
    stats->arena_compactions = dg.prog.compactions;
    stats->kernel_launches = dg.prog.launches;
    stats->round_kernel_ms = dg.prog.round_ms;
    stats->round_kernel_launches = dg.prog.round_launches;
  }
  return GEQ_OK;
}

geq_status Engine::solve(DeviceGamesImpl &dg, geq_solve_stats *stats) {
  State &s = *st;
  cudaStream_t S = s.stream;
  geq_status st_ = solve_begin(dg);
  if (st_) return st_;
  for (bool done = false; !done;)
    if ((st_ = solve_step(dg, done))) return st_;
  CU(cudaEventRecord(s.ev1, S));
  if ((st_ = solve_stats(dg, stats))) return st_;
#if GEQ_PATH_PROFILE
  {
    const Ctr c = *s.h_ctr;
    std::fprintf(stderr, "GEQ_PROF");
    for (int i = 0; i < 32; i++) std::fprintf(stderr, " %llu", c.prof[i]);
    std::fprintf(stderr, "\n");
  }
#endif
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s.ev0, s.ev1);
    stats->device_ms = ms;
  }
  return GEQ_OK;
}

// Games with at least one position in the current frontier; the others
// have reached their fixpoint (games share no edges, so a game without a
// frontier position never changes again).
__global__ void k_active_games(const KParams p, const unsigned long long *node_base, uint32_t n_games,
                               uint8_t *active) {
  const Ctr *c = p.ctr;
  const uint32_t cur = c->cur, fs = c->fsize[cur];
  const uint32_t *F = cur ? p.front1 : p.front0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < fs; i += gridDim.x * blockDim.x) {
    const uint32_t v = F[i];
    if (v < p.n_nodes) active[game_of(node_base, n_games, v)] = 1;
  }
}

geq_status Engine::active_games(DeviceGamesImpl &dg, std::vector<uint8_t> &active) {
  State &s = *st;
  cudaStream_t S = s.stream;
  const uint32_t G = dg.n_games;
  uint8_t *d_act = (uint8_t *)s.pool.get(std::max<uint32_t>(G, 1));
  if (!d_act) return fail(GEQ_ERR_OUT_OF_MEMORY, "active flags");
  CU(cudaMemsetAsync(d_act, 0, G, S));
  k_active_games<<<(unsigned)std::max(1, n_sms * 4), 256, 0, S>>>(dg.kp, dg.d_node_base, G, d_act);
  active.assign(G, 0);
  CU(cudaMemcpyAsync(active.data(), d_act, G, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  s.pool.put(d_act, std::max<uint32_t>(G, 1));
  CU(cudaGetLastError());
  return GEQ_OK;
}

uint32_t Engine::game_positions(const DeviceGamesImpl &dg, uint32_t g) {
  return (uint32_t)(dg.node_base[g + 1] - dg.node_base[g]);
}
uint32_t Engine::n_games_of(const DeviceGamesImpl &dg) { return dg.n_games; }

// Result lists of all positions: gathered on the device (counts, scan,
// gather into one buffer, per-game relative offsets), then read back.  The
// two steps are separate so that two uploads' results can be read into one
// host buffer (run_batch_pipelined).
geq_status Engine::download_prepare(DeviceGamesImpl &dg, Readback &rb) {
  State &s = *st;
  cudaStream_t S = s.stream;
  const unsigned long long N = dg.N;
  unsigned long long launches = 0;
  geq_status a = ensure_cnt(s, N + 1);
  if (a) return a;
  rb.goff = (unsigned long long *)s.pool.get((N + 1) * 8);
  rb.rel = (unsigned long long *)s.pool.get((N + dg.n_games) * 8);
  if (!rb.goff || !rb.rel) {
    download_release(dg, rb);
    return fail(GEQ_ERR_OUT_OF_MEMORY, "download offsets");
  }
  const unsigned grid = (unsigned)std::max(1, n_sms * 8);
  k_desc_counts<<<grid, 256, 0, S>>>(dg.desc, N, s.cnt);
  if ((a = scan_u32(s, s.cnt, N, rb.goff, launches))) return a;
  CU(cudaMemcpyAsync(&s.h_ctr->positions, rb.goff + N, 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  rb.total = s.h_ctr->positions;
  rb.out = (uint32_t *)s.pool.get(std::max<unsigned long long>(rb.total, 1) * 4);
  if (!rb.out) return fail(GEQ_ERR_OUT_OF_MEMORY, "download data");
  k_gather<<<grid, 256, 0, S>>>(dg.desc, N, rb.goff, dg.arena[dg.arena_cur], dg.kp.ib, dg.kp.ibm, rb.out);
  k_rel_offsets<<<grid, 256, 0, S>>>(rb.goff, N, dg.d_node_base, dg.n_games, rb.rel);
  CU(cudaGetLastError());
  return GEQ_OK;
}
geq_status Engine::download_copy(DeviceGamesImpl &dg, Readback &rb, uint64_t *off_dst, uint32_t *data_dst) {
  State &s = *st;
  cudaStream_t S = s.stream;
  CU(cudaMemcpyAsync(off_dst, rb.rel, (dg.N + dg.n_games) * 8, cudaMemcpyDeviceToHost, S));
  if (rb.total) CU(cudaMemcpyAsync(data_dst, rb.out, rb.total * 4, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  CU(cudaGetLastError());
  download_release(dg, rb);
  return GEQ_OK;
}
void Engine::download_release(DeviceGamesImpl &dg, Readback &rb) {
  State &s = *st;
  s.pool.put(rb.goff, (dg.N + 1) * 8);
  s.pool.put(rb.rel, (dg.N + dg.n_games) * 8);
  s.pool.put(rb.out, std::max<unsigned long long>(rb.total, 1) * 4);
  rb.goff = rb.rel = nullptr;
  rb.out = nullptr;
}

// Per-game bases of a solution whose offsets are in place, starting at game
// g0 with offset index ob and word db.
static void fill_bases(const DeviceGamesImpl &dg, geq_solution &sol, uint32_t g0, uint64_t ob, uint64_t db) {
  const uint64_t *offs = sol.off_ptr();
  for (uint32_t g = 0; g < dg.n_games; g++) {
    const uint32_t n = (uint32_t)(dg.node_base[g + 1] - dg.node_base[g]);
    sol.n_vertices[g0 + g] = n;
    sol.offsets_base[g0 + g] = ob;
    sol.data_base[g0 + g] = db;
    db += offs[ob + n];
    ob += (uint64_t)n + 1;
  }
}

geq_status Engine::download(DeviceGamesImpl &dg, geq_solution &sol) {
  State &s = *st;
  Readback rb;
  geq_status a = download_prepare(dg, rb);
  if (a) {
    download_release(dg, rb);
    return a;
  }
  sol.energy_size = 1;
  // straight into page-locked host memory (no staging copy, no zero fill)
  sol.n_offsets = dg.N + dg.n_games;
  sol.n_words = rb.total;
  if (!sol.off_buf.alloc(s.hpool, sol.n_offsets * 8) || !sol.data_buf.alloc(s.hpool, rb.total * 4)) {
    download_release(dg, rb);
    return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for %llu result words", rb.total);
  }
  if ((a = download_copy(dg, rb, (uint64_t *)sol.off_buf.p, (uint32_t *)sol.data_buf.p))) return a;
  sol.n_vertices.resize(dg.n_games);
  sol.offsets_base.resize(dg.n_games);
  sol.data_base.resize(dg.n_games);
  fill_bases(dg, sol, 0, 0, 0);
  return GEQ_OK;
}

// A large batch on two engines: the first half is uploaded, then solved
// while the second half uploads on the other engine's stream, so the link
// transfer of one half overlaps the rounds of the other; both halves' lists
// are read back into one flat solution.
geq_status run_batch_pipelined(int device, Engine &ea, Engine &eb, std::vector<GameInput> &in, geq_solution &sol) {
  const uint32_t n_games = (uint32_t)in.size();
  unsigned long long total = 0;
  for (auto &gi : in) total += gi.g.n_vertices;
  uint32_t k = 0;
  unsigned long long acc = 0;
  while (k + 1 < n_games && acc < total / 2) acc += in[k++].g.n_vertices;
  auto part = [&](uint32_t b, uint32_t e) {
    std::vector<GameInput> v(e - b);
    for (uint32_t i = b; i < e; i++) {
      GameInput &d = v[i - b];
      d.g = in[i].g;
      d.init = in[i].init;
      d.to_reach = in[i].to_reach;  // points into in[i], alive for the call
      d.n_reach = in[i].n_reach;
      d.std_reach = in[i].std_reach;
      d.rows_unchecked = in[i].rows_unchecked;
    }
    return v;
  };
  std::vector<GameInput> ia = part(0, k), ib = part(k, n_games);
  GamesPtr da, db;
  Engine::Readback ra, rb;
  geq_solve_stats sa{}, sb{};
  geq_status st_a = GEQ_OK, st_b = GEQ_OK;
  std::string err_b;
  std::promise<void> a_up;
  std::future<void> a_up_done = a_up.get_future();
#if GEQ_PATH_PROFILE
  const auto tp0 = std::chrono::steady_clock::now();
  double tl[12] = {};
  auto mark = [&](int i) { tl[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp0).count(); };
#else
  auto mark = [](int) {};
#endif
  std::thread tb([&]() {
    cudaSetDevice(device);
    a_up_done.wait();
    mark(5);
    st_b = eb.upload(ib, db);
    mark(6);
    if (!st_b) st_b = eb.solve(*db, &sb);
    mark(7);
    if (!st_b) st_b = eb.download_prepare(*db, rb);
    mark(8);
    if (st_b) err_b = geq_last_error();
  });
  st_a = ea.upload(ia, da);
  mark(0);
  a_up.set_value();
  if (!st_a) st_a = ea.solve(*da, &sa);
  mark(1);
  if (!st_a) st_a = ea.download_prepare(*da, ra);
  mark(2);
  // the first half's lists go to the host while the second half may still
  // be solving: the offsets' size is known (every position of the batch),
  // the words are not, so the data block is sized from the first half's
  // total scaled to the second half's positions, with headroom, and
  // replaced below when the second half needs more
  const uint64_t na = da ? da->N + da->n_games : 0;
  const uint64_t n_off = total + n_games;
  if (!st_a) {
    const double scale = (double)(total - da->N) / (double)std::max<uint64_t>(1, da->N);
    const uint64_t guess = ra.total + (uint64_t)((double)ra.total * scale * 1.25) + (1u << 20);
    if (!sol.off_buf.alloc(ea.st->hpool, n_off * 8) || !sol.data_buf.alloc(ea.st->hpool, guess * 4))
      st_a = fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for %llu result words", (unsigned long long)guess);
    else
      st_a = ea.download_copy(*da, ra, (uint64_t *)sol.off_buf.p, (uint32_t *)sol.data_buf.p);
  }
  mark(3);
  tb.join();
  mark(4);
  if (st_a || st_b) {
    if (da) ea.download_release(*da, ra);
    if (db) eb.download_release(*db, rb);
    if (!st_a) set_last_error(err_b);
    return st_a ? st_a : st_b;
  }
  sol.energy_size = 1;
  sol.n_offsets = n_off;
  sol.n_words = ra.total + rb.total;
  if (sol.data_buf.cap < sol.n_words * 4) {
    HostBuf bigger;
    if (!bigger.alloc(ea.st->hpool, sol.n_words * 4)) {
      eb.download_release(*db, rb);
      return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for %llu result words", (unsigned long long)sol.n_words);
    }
    std::memcpy(bigger.p, sol.data_buf.p, ra.total * 4);
    std::swap(sol.data_buf.p, bigger.p);
    std::swap(sol.data_buf.cap, bigger.cap);
    std::swap(sol.data_buf.pool, bigger.pool);
  }
  uint64_t *off = (uint64_t *)sol.off_buf.p;
  uint32_t *data = (uint32_t *)sol.data_buf.p;
  geq_status st = eb.download_copy(*db, rb, off + na, data + ra.total);
  if (st) return st;
  mark(9);
#if GEQ_PATH_PROFILE
  std::fprintf(stderr,
               "GEQ_SPLIT a_up %.1f a_solve %.1f a_prep %.1f a_copy %.1f join %.1f | b_start %.1f b_up %.1f b_solve %.1f "
               "b_prep %.1f | b_copy %.1f\n",
               tl[0], tl[1], tl[2], tl[3], tl[4], tl[5], tl[6], tl[7], tl[8], tl[9]);
#endif
  sol.n_vertices.resize(n_games);
  sol.offsets_base.resize(n_games);
  sol.data_base.resize(n_games);
  fill_bases(*da, sol, 0, 0, 0);
  fill_bases(*db, sol, k, na, ra.total);
  sol.stats = sa;
  sol.stats.rounds = std::max(sa.rounds, sb.rounds);
  sol.stats.positions_computed += sb.positions_computed;
  sol.stats.edges_relaxed += sb.edges_relaxed;
  sol.stats.algorithmic_bytes += sb.algorithmic_bytes;
  sol.stats.arena_compactions += sb.arena_compactions;
  sol.stats.kernel_launches += sb.kernel_launches;
  sol.stats.device_ms = std::max(sa.device_ms, sb.device_ms);
  return GEQ_OK;
}

geq_status Engine::download_selected(DeviceGamesImpl &dg, const std::vector<uint32_t> &first,
                                     const std::vector<uint32_t> &count, geq_solution &sol) {
  State &s = *st;
  cudaStream_t S = s.stream;
  const uint32_t G = (uint32_t)first.size();
  std::vector<uint32_t> sel;
  for (uint32_t g = 0; g < G; g++)
    for (uint32_t i = 0; i < count[g]; i++) sel.push_back((uint32_t)(dg.node_base[g] + first[g] + i));
  const unsigned long long K = sel.size();
  unsigned long long launches = 0;
  geq_status a = ensure_cnt(s, K + 1);
  if (a) return a;
  uint32_t *d_sel = (uint32_t *)s.pool.get(std::max<unsigned long long>(K, 1) * 4);
  unsigned long long *goff = (unsigned long long *)s.pool.get((K + 1) * 8);
  if (!d_sel || !goff) return fail(GEQ_ERR_OUT_OF_MEMORY, "selection");
  if (K) CU(cudaMemcpyAsync(d_sel, sel.data(), K * 4, cudaMemcpyHostToDevice, S));
  const unsigned grid = (unsigned)std::max(1, n_sms * 8);
  k_sel_counts<<<grid, 256, 0, S>>>(dg.desc, d_sel, K, s.cnt);
  if ((a = scan_u32(s, s.cnt, K, goff, launches))) return a;
  std::vector<unsigned long long> off(K + 1);
  CU(cudaMemcpyAsync(off.data(), goff, (K + 1) * 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  const unsigned long long total = off[K];
  uint32_t *out = (uint32_t *)s.pool.get(std::max<unsigned long long>(total, 1) * 4);
  if (!out) return fail(GEQ_ERR_OUT_OF_MEMORY, "selection data");
  k_sel_gather<<<grid, 256, 0, S>>>(dg.desc, d_sel, K, goff, dg.arena[dg.arena_cur], dg.kp.ib, dg.kp.ibm, out);
  sol.energy_size = 1;
  sol.data.resize(total);
  if (total) CU(cudaMemcpyAsync(sol.data.data(), out, total * 4, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  CU(cudaGetLastError());
  s.pool.put(d_sel, std::max<unsigned long long>(K, 1) * 4);
  s.pool.put(goff, (K + 1) * 8);
  s.pool.put(out, std::max<unsigned long long>(total, 1) * 4);
  sol.n_vertices.assign(count.begin(), count.end());
  sol.offsets_base.resize(G);
  sol.data_base.resize(G);
  sol.offsets.clear();
  sol.offsets.reserve(K + G);
  unsigned long long k = 0;
  for (uint32_t g = 0; g < G; g++) {
    sol.offsets_base[g] = sol.offsets.size();
    sol.data_base[g] = off[k];
    for (uint32_t i = 0; i <= count[g]; i++) sol.offsets.push_back(off[k + i] - off[k]);
    k += count[g];
  }
  return GEQ_OK;
}

// ---- allocation-free solve of one game (geq_energy_game_run_static) -------
// All device memory of this solve is one file-scope array: the game, its
// reverse CSR, descriptors, frontiers, control block and energy arena.  One
// block of BLOCK threads runs the whole solve in one launch -- validation,
// reverse CSR, initialisation, the rounds (the position routines of k_round,
// with block barriers between a round and its commit) and the gather of the
// result lists -- so the call allocates nothing and launches one kernel.
static __device__ __align__(256) unsigned char g_static_scratch[GEQ_STATIC_SCRATCH_BYTES];

struct StaticArgs {
  const uint32_t *reach;        // explicit to_reach list, or null: standard reach
  uint32_t n_reach;
  uint32_t max_rounds;
  uint32_t *arena;
  unsigned long long arena_cap;  // words
  unsigned long long *out_off;   // n_nodes + 1 result offsets
};
// Games up to these sizes take the one-block path in geq_energy_game_run.
constexpr unsigned long long SMALL_GAME_POSITIONS = 4096, SMALL_GAME_EDGES = 65536;
// Ctr::pad bits of the static solve
constexpr uint32_t SERR_COL = 1u, SERR_WEIGHT = 2u, SERR_ARENA = 4u, SERR_ROUNDS = 8u;

// out[v] = sum of cnt(u) for u < v, out[n] = the total; one block.
template <class T, class F>
__device__ void block_excl_scan_n(unsigned long long n, F cnt, T *out, unsigned long long *ws) {
  const uint32_t t = threadIdx.x;
  const unsigned long long chunk = (n + BLOCK - 1) / BLOCK;
  const unsigned long long b = min(n, (unsigned long long)t * chunk), e = min(n, b + chunk);
  unsigned long long sum = 0;
  for (unsigned long long v = b; v < e; v++) sum += cnt(v);
  ws[t] = sum;
  __syncthreads();
  if (t == 0) {
    unsigned long long acc = 0;
    for (int i = 0; i < BLOCK; i++) {
      const unsigned long long x = ws[i];
      ws[i] = acc;
      acc += x;
    }
    out[n] = (T)acc;
  }
  __syncthreads();
  unsigned long long acc = ws[t];
  for (unsigned long long v = b; v < e; v++) {
    out[v] = (T)acc;
    acc += cnt(v);
  }
  __syncthreads();
}

template <class Cd>
__global__ void __launch_bounds__(BLOCK, 1) k_solve_static(const KParams p, const StaticArgs a) {
  __shared__ uint32_t smem[WARPS_PER_BLOCK * SM_WORDS];
  __shared__ uint32_t tscr[WARPS_PER_BLOCK * TSCR * 32];
  __shared__ unsigned long long ws[BLOCK];
  __shared__ uint32_t s_err;
  Ctr *c = p.ctr;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const unsigned long long N = p.n_nodes, M = p.n_edges;
  uint32_t *rrow = const_cast<uint32_t *>(p.rrow), *rcol = const_cast<uint32_t *>(p.rcol);
  // -- everything that must start at zero, and the control block
  if (tid == 0) {
    Ctr h{};
    h.arena = a.arena;
    h.arena_cap = a.arena_cap;
    h.arena_top = 1;  // word 0: the zero energy
    h.stamp = 1;
    *c = h;
    a.arena[0] = 0u;
    s_err = 0u;
  }
  for (unsigned long long v = tid; v < N; v += BLOCK) {
    p.desc[v] = 0ull;
    p.mark[v] = 0u;
  }
  __syncthreads();
  // -- successor ids and update codes (k_indegree, k_check_weights); in-degrees into mark
  uint32_t bad = 0;
  for (unsigned long long k = tid; k < M; k += BLOCK) {
    const uint32_t w = p.col[k];
    if (w < N) atomicAdd(&p.mark[w], 1u);
    else bad |= SERR_COL;
    const uint32_t u = p.wt[k];
    if (p.el * p.ub < 32u && (u >> (p.el * p.ub)) != 0u) bad |= SERR_WEIGHT;
    for (uint32_t i = 0; i < p.el; i++)
      if (((u >> (i * p.ub)) & p.um) > p.el + 1u) bad |= SERR_WEIGHT;
  }
  if (bad) atomicOr(&s_err, bad);
  __syncthreads();
  if (s_err) {
    if (tid == 0) c->pad = s_err;
    return;
  }
  // -- reverse CSR: offsets, then predecessors through a cursor kept in mark
  block_excl_scan_n<uint32_t>(N, [&](unsigned long long v) { return (unsigned long long)p.mark[v]; }, rrow, ws);
  for (unsigned long long v = tid; v < N; v += BLOCK) p.mark[v] = rrow[v];
  __syncthreads();
  for (unsigned long long v = tid; v < N; v += BLOCK)
    for (uint32_t k = p.row[v]; k < p.row[v + 1]; k++) rcol[atomicAdd(&p.mark[p.col[k]], 1u)] = (uint32_t)v;
  __syncthreads();
  for (unsigned long long v = tid; v < 2ull * p.mwords; v += BLOCK) p.mark[v] = 0u;
  __syncthreads();
  // -- standard initialisation: {0} at the positions to reach (EnergyGame::with_reach)
  auto is_reach = [&](unsigned long long v) { return !(p.flags[v] & 1u) && p.row[v + 1] == p.row[v]; };
  const unsigned long long n_src = a.reach ? a.n_reach : N;
  for (unsigned long long i = tid; i < n_src; i += BLOCK) {
    if (a.reach) p.desc[a.reach[i]] = inl_hdr(1u);
    else if (is_reach(i)) p.desc[i] = inl_hdr(1u);
  }
  __syncthreads();
  uint32_t *sm = smem + warp * SM_WORDS;
  for (unsigned long long b0 = (unsigned long long)warp * 32u; b0 < n_src; b0 += BLOCK) {
    const unsigned long long i = b0 + lane;
    bool f = false;
    uint32_t v = 0;
    if (i < n_src) {
      v = a.reach ? a.reach[i] : (uint32_t)i;
      f = a.reach ? true : is_reach(i);
    }
    push_preds_warp(p, c, sm, v, f, c->stamp, lane);
  }
  __syncthreads();
  __shared__ uint32_t s_wsum[33];
  {
    const uint32_t n0 = block_fill_bits(p.mark + (c->stamp & 1u) * p.mwords, 0u, p.mwords, 0u, p.front0,
                                        (uint32_t)N, c, s_wsum);
    if (tid == 0) c->fsize[0] = n0;
    __syncthreads();
  }
  // -- rounds (k_round + k_commit + k_fcount/k_ffill in one block)
  uint32_t *scr = tscr + warp * (TSCR * 32) + lane;
  const Cd cd = make_codec<Cd>(p);
  uint32_t *arena = a.arena;
  const unsigned long long cap = a.arena_cap;
  WarpAlloc wa{0, 0};
  unsigned long long w_edges = 0, w_bytes = 0, w_pos = 0;
  uint32_t t_edges = 0, t_bytes = 0, t_pos = 0;
  WarpCtx x{p, c, arena, cap, lane, sm, wa, w_edges, w_bytes, scr};
  __shared__ uint32_t s_cur, s_fs, s_stop;
  for (uint32_t r = 0;; r++) {
    // one thread decides, so that every warp leaves the loop in the same round
    if (tid == 0) {
      s_cur = c->cur;
      s_fs = c->fsize[s_cur];
      s_stop = (s_fs == 0u || c->overflow || c->error) ? 1u : (r >= a.max_rounds ? 2u : 0u);
      if (s_stop == 2u) c->pad = SERR_ROUNDS;
    }
    __syncthreads();
    if (s_stop) break;
    const uint32_t cur = s_cur, fs = s_fs;
    const uint32_t *F = cur ? p.front1 : p.front0;
    const uint32_t stamp = c->stamp + 1u;
    for (uint32_t base = warp * 32u; base < fs; base += BLOCK) {
      const uint32_t slot = base + lane;
      const bool active = slot < fs;
      const uint32_t v = active ? ld(F, slot, p.n_nodes, c) : 0u;
      int ts = T_NONE;
      uint32_t cnt = 0, old_cnt = 0;
      if (active)
        ts = p.thread_path ? thread_solve(p, c, cd, arena, cap, v, scr, cnt, t_edges, t_bytes, old_cnt) : T_BIG;
      if (ts != T_NONE && ts != T_BIG && ts != T_SKIPPED) t_pos++;
      unsigned long long nd = NONE_DESC;
      if (ts == T_CHANGED && cnt <= p.inl) {
        nd = inl_hdr(cnt);
        for (uint32_t q = 0; q < cnt; q++) nd |= (unsigned long long)SCR(TK + q) << (q * p.ib);
      }
      const uint32_t need = (ts == T_CHANGED && cnt > p.inl) ? cnt : 0u;
      const uint32_t incl = warp_incl_scan(need, lane);
      const uint32_t total = __shfl_sync(FULL, incl, 31);
      unsigned long long obase = 0;
      const bool ok = total == 0u || wa.alloc(total, c, cap, lane, obase);
      if (need) {
        if (!ok) {
          ts = T_OVERFLOW;
        } else {
          const unsigned long long off = obase + incl - need;
          for (uint32_t q = 0; q < need; q++)
            if (CHECK_IDX(c, off + q, cap)) arena[off + q] = SCR(TK + q);
          nd = mkdesc(off, need);
        }
      }
      if (ts == T_CHANGED) t_bytes += 4u * cnt;
      if (active && ts != T_BIG && CHECK_IDX(c, slot, p.n_nodes)) p.slot_new[slot] = (ts == T_CHANGED) ? nd : NONE_DESC;
      uint32_t big = __ballot_sync(FULL, ts == T_BIG);
      bool big_changed = false;
      while (big) {
        const uint32_t l = __ffs(big) - 1u;
        big &= big - 1u;
        const uint32_t vb = __shfl_sync(FULL, v, l);
        const Res rs = solve_position(x, cd, vb);
        if (rs.st != R_SKIPPED) w_pos++;
        if (lane == 0 && CHECK_IDX(c, base + l, p.n_nodes))
          p.slot_new[base + l] = (rs.st == R_CHANGED) ? rs.d : NONE_DESC;
        if (lane == l) big_changed = rs.st == R_CHANGED;
      }
      push_preds_warp(p, c, sm, v, ts == T_CHANGED || big_changed, stamp, lane);
    }
    __syncthreads();
    for (uint32_t i = tid; i < p.mwords; i += BLOCK) p.mark[(c->stamp & 1u) * p.mwords + i] = 0u;
    for (uint32_t s2 = tid; s2 < fs; s2 += BLOCK) {
      const unsigned long long d = p.slot_new[s2];
      if (d != NONE_DESC) {
        const uint32_t v = F[s2];
        if (CHECK_IDX(c, v, p.n_nodes)) p.desc[v] = d;
      }
    }
    __syncthreads();
    if (tid == 0) {
      c->fsize[cur] = 0u;
      c->cur = cur ^ 1u;
      c->stamp = c->stamp + 1u;
      c->rounds = c->rounds + 1ull;
    }
    __syncthreads();
    // the next frontier, in position order, from the half this round filled
    const uint32_t nn = block_fill_bits(p.mark + (c->stamp & 1u) * p.mwords, 0u, p.mwords, 0u,
                                        cur ? p.front0 : p.front1, (uint32_t)N, c, s_wsum);
    if (tid == 0) c->fsize[cur ^ 1u] = nn;
    __syncthreads();
  }
  unsigned long long te = t_edges, tb = t_bytes, tp = t_pos;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    te += __shfl_xor_sync(FULL, te, o);
    tb += __shfl_xor_sync(FULL, tb, o);
    tp += __shfl_xor_sync(FULL, tp, o);
  }
  if (lane == 0) {
    atomicAdd(&c->positions, tp + w_pos);
    atomicAdd(&c->edges, te + w_edges);
    atomicAdd(&c->bytes, tb + w_bytes);
  }
  __syncthreads();
  if (c->overflow) {
    if (tid == 0) c->pad |= SERR_ARENA;
    return;
  }
  if (c->pad || c->error) return;
  // -- result lists (k_desc_counts + scan + k_gather) behind the arena's used part
  block_excl_scan_n<unsigned long long>(N, [&](unsigned long long v) { return (unsigned long long)dcnt(p.desc[v]); },
                                        a.out_off, ws);
  const unsigned long long top = c->arena_top, total = a.out_off[N];
  if (top + total > cap) {
    if (tid == 0) c->pad = SERR_ARENA;
    return;
  }
  uint32_t *out = arena + top;
  for (unsigned long long v = warp; v < N; v += WARPS_PER_BLOCK) {
    const unsigned long long d = p.desc[v];
    const uint32_t n = dcnt(d);
    const unsigned long long go = a.out_off[v];
    for (uint32_t q = lane; q < n; q += 32u)
      out[go + q] = dinl(d) ? ((uint32_t)(d >> (q * p.ib)) & p.ibm) : arena[doff(d) + q];
  }
}

// Device address of the scratch on the current device.  Looked up on every
// call (cheap once the module is loaded), so that no address outlives the
// context it belongs to (a cudaDeviceReset makes a new one).  The first
// lookup on a device loads the module and with it reserves the array:
// Engine::create does that lookup, so the scratch is reserved when a
// context is created and not inside a later geq_energy_game_run_static.
static geq_status static_scratch(int device, unsigned char *&out) {
  (void)device;
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
  if (e != cudaSuccess || !ptr)
    return fail(GEQ_ERR_CUDA, "cudaGetSymbolAddress of the static scratch: %s", cudaGetErrorString(e));
  out = (unsigned char *)ptr;
  return GEQ_OK;
}

// Layout of a one-block solve (k_solve_static) inside one memory block:
// control block, the game, reverse CSR, descriptors, frontiers, result
// offsets, 256-byte aligned, then the energy arena up to the block's end.
struct BlockLayout {
  size_t ctr, row, col, wt, flags, reach, rrow, rcol, desc, slot, mark, f0, f1, out, top;
};
static BlockLayout block_layout(unsigned long long N, unsigned long long M, uint32_t n_reach) {
  BlockLayout L{};
  size_t top = 0;
  auto take = [&](size_t bytes) {
    const size_t o = top;
    top = (top + std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return o;
  };
  L.ctr = take(sizeof(Ctr));
  L.row = take((N + 1) * 4);
  L.col = take(M * 4);
  L.wt = take(M * 4);
  L.flags = take(N);
  L.reach = take((size_t)n_reach * 4);
  L.rrow = take((N + 1) * 4);
  L.rcol = take(M * 4);
  L.desc = take(N * 8);
  L.slot = take(N * 8);
  L.mark = take(std::max<unsigned long long>(N, 2 * ((N + 31) / 32)) * 4);
  L.f0 = take(N * 4);
  L.f1 = take(N * 4);
  L.out = take((N + 1) * 8);
  L.top = top;
  return L;
}
static void block_params(const BlockLayout &L, unsigned char *base, size_t bytes, unsigned long long N,
                         unsigned long long M, const Conf &conf, const geq_tuning &t, bool explicit_reach,
                         uint32_t n_reach, KParams &kp, StaticArgs &sa) {
  kp = KParams{};
  kp.row = (const uint32_t *)(base + L.row);
  kp.col = (const uint32_t *)(base + L.col);
  kp.wt = (const uint32_t *)(base + L.wt);
  kp.rrow = (const uint32_t *)(base + L.rrow);
  kp.rcol = (const uint32_t *)(base + L.rcol);
  kp.flags = (const uint8_t *)(base + L.flags);
  kp.desc = (unsigned long long *)(base + L.desc);
  kp.mark = (uint32_t *)(base + L.mark);
  kp.front0 = (uint32_t *)(base + L.f0);
  kp.front1 = (uint32_t *)(base + L.f1);
  kp.slot_new = (unsigned long long *)(base + L.slot);
  kp.ctr = (Ctr *)(base + L.ctr);
  kp.n_nodes = N;
  kp.n_edges = M;
  kp.mwords = (uint32_t)((N + 31) / 32);
  kp.el = conf.elements; kp.mx = conf.max; kp.eb = conf.energy_bits(); kp.em = conf.energy_mask();
  kp.ub = conf.update_bits(); kp.um = conf.update_mask();
  kp.small_limit = (t.flags & GEQ_TUNE_FORCE_LARGE) ? 0u : std::min<uint32_t>(t.small_limit, 32);
  kp.thread_path = (t.flags & (GEQ_TUNE_FORCE_LARGE | GEQ_TUNE_NO_THREAD_PATH)) ? 0u : 1u;
  kp.ib = conf.elements * conf.energy_bits();
  kp.ibm = kp.ib >= 32 ? 0xFFFFFFFFu : ((1u << kp.ib) - 1u);
  kp.inl = std::min<uint32_t>(7u, 60u / kp.ib);
  kp.cw = nullptr;
  set_lane_limits(kp, geq_tuning{});
  sa = StaticArgs{};
  sa.reach = explicit_reach ? (const uint32_t *)(base + L.reach) : nullptr;
  sa.n_reach = explicit_reach ? n_reach : 0u;
  sa.max_rounds = 1u << 20;
  sa.arena = (uint32_t *)(base + L.top);
  sa.arena_cap = (bytes - L.top) / 4;
  sa.out_off = (unsigned long long *)(base + L.out);
}

geq_status Engine::run_static(int device, const geq_game_graph &g, const uint32_t *to_reach, uint32_t n_reach,
                              uint64_t *offsets, uint32_t *data, uint64_t data_cap, uint64_t *n_words,
                              geq_solve_stats *stats) {
  State &s = *st;
  cudaStream_t S = s.stream;
  int prev = -1;
  CU(cudaGetDevice(&prev));
  if (prev != device) CU(cudaSetDevice(device));
  struct Restore {
    int prev, dev;
    ~Restore() { if (prev != dev && prev >= 0) cudaSetDevice(prev); }
  } restore{prev, device};
  const Conf conf(g.conf);
  if (!conf.supported())
    return fail(GEQ_ERR_UNSUPPORTED, "EnergyConf {%u, %u} is outside the device codecs", conf.elements, conf.max);
  const unsigned long long N = g.n_vertices, M = g.row_offsets[g.n_vertices];
  const BlockLayout L = block_layout(N, M, n_reach);
  const size_t min_arena = 4096 * 4;
  if (N >= 0xFFFFFFF0ull || M >= 0xFFFFFFF0ull || L.top + min_arena > GEQ_STATIC_SCRATCH_BYTES)
    return fail(GEQ_ERR_UNSUPPORTED,
                "game of %llu positions / %llu edges needs %zu bytes of the %u-byte static scratch",
                N, M, L.top + min_arena, (unsigned)GEQ_STATIC_SCRATCH_BYTES);
  unsigned char *base = nullptr;
  geq_status rc = static_scratch(device, base);
  if (rc) return rc;
  KParams kp;
  StaticArgs sa;
  block_params(L, base, GEQ_STATIC_SCRATCH_BYTES, N, M, conf, tuning, to_reach != nullptr, n_reach, kp, sa);
  // the game, straight from the caller's buffers
  CU(cudaEventRecord(s.ev0, S));
  CU(cudaMemcpyAsync(base + L.row, g.row_offsets, (N + 1) * 4, cudaMemcpyHostToDevice, S));
  if (M) {
    CU(cudaMemcpyAsync(base + L.col, g.column_indices, M * 4, cudaMemcpyHostToDevice, S));
    CU(cudaMemcpyAsync(base + L.wt, g.weights, M * 4, cudaMemcpyHostToDevice, S));
  }
  if (N) CU(cudaMemcpyAsync(base + L.flags, g.attacker_pos, N, cudaMemcpyHostToDevice, S));
  if (to_reach && n_reach) CU(cudaMemcpyAsync(base + L.reach, to_reach, (size_t)n_reach * 4, cudaMemcpyHostToDevice, S));
  const bool generic = !conf.standard() || (tuning.flags & GEQ_TUNE_FORCE_GENERIC);
  if (generic) k_solve_static<CodecGen><<<1, BLOCK, 0, S>>>(kp, sa);
  else k_solve_static<CodecStd><<<1, BLOCK, 0, S>>>(kp, sa);
  CU(cudaGetLastError());
  Ctr h{};
  CU(cudaMemcpyAsync(&h, kp.ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
  CU(cudaMemcpyAsync(offsets, sa.out_off, (N + 1) * 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  if (h.pad & SERR_COL) return fail(GEQ_ERR_INVALID_INPUT, "Node index too high: a successor index is out of range");
  if (h.pad & SERR_WEIGHT) return fail(GEQ_ERR_INVALID_INPUT, "an edge update names no element or sets padding bits");
  if (h.error)
    return fail((h.error & DERR_BOUNDS) ? GEQ_ERR_INTERNAL : GEQ_ERR_OUT_OF_MEMORY, "device error %u (line %u)",
                h.error, h.err_line);
  if (h.pad & SERR_ARENA)
    return fail(GEQ_ERR_OUT_OF_MEMORY, "the energy lists outgrew the static scratch (%llu words)", sa.arena_cap);
  if (h.pad & SERR_ROUNDS) return fail(GEQ_ERR_TIMEOUT, "no fixpoint after %u rounds", sa.max_rounds);
  const unsigned long long total = offsets[N];
  if (n_words) *n_words = total;
  if (total > data_cap)
    return fail(GEQ_ERR_INVALID_INPUT, "data_cap %llu is below the %llu result words", (unsigned long long)data_cap,
                total);
  if (total) CU(cudaMemcpyAsync(data, sa.arena + h.arena_top, total * 4, cudaMemcpyDeviceToHost, S));
  CU(cudaEventRecord(s.ev1, S));
  CU(cudaStreamSynchronize(S));
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s.ev0, s.ev1);
    *stats = geq_solve_stats{};
    stats->rounds = h.rounds;
    stats->positions_computed = h.positions;
    stats->edges_relaxed = h.edges;
    stats->algorithmic_bytes = h.bytes;
    stats->kernel_launches = 1;
    stats->device_ms = ms;
  }
  return GEQ_OK;
}


// One small game in one launch of the one-block solver, in a pooled device
// block: one upload from page-locked staging, one kernel, two read-backs.  A
// game whose lists outgrow the block's arena is left to the general path
// (handled = false), as is everything outside the limits.
geq_status Engine::solve_small(const GameInput &gi, geq_solution &sol, bool &handled) {
  handled = false;
  State &s = *st;
  cudaStream_t S = s.stream;
  const Conf conf(gi.g.conf);
  const unsigned long long N = gi.g.n_vertices, M = gi.g.row_offsets[gi.g.n_vertices];
  if (gi.init || tuning.flags || N > SMALL_GAME_POSITIONS || M > SMALL_GAME_EDGES || !conf.supported())
    return GEQ_OK;
  const BlockLayout L = block_layout(N, M, gi.n_reach);
  const size_t bytes = L.top + 4 * (16 * (size_t)(N + M) + 65536);
  unsigned char *base = (unsigned char *)s.pool.get(bytes);
  if (!base) return GEQ_OK;
  struct Give {
    DevPool &pool;
    void *p;
    size_t b;
    ~Give() { pool.put(p, b); }
  } give{s.pool, base, bytes};
  geq_status rc = ensure_stage(s, L.rrow);
  if (rc) return rc;
  char *H = s.stage;
  std::memcpy(H + L.row, gi.g.row_offsets, (N + 1) * 4);
  if (M) {
    std::memcpy(H + L.col, gi.g.column_indices, M * 4);
    std::memcpy(H + L.wt, gi.g.weights, M * 4);
  }
  if (N) std::memcpy(H + L.flags, gi.g.attacker_pos, N);
  if (gi.n_reach) std::memcpy(H + L.reach, gi.to_reach, (size_t)gi.n_reach * 4);
  KParams kp;
  StaticArgs sa;
  block_params(L, base, bytes, N, M, conf, tuning, true, gi.n_reach, kp, sa);
  CU(cudaEventRecord(s.ev0, S));
  CU(cudaMemcpyAsync(base, H, L.rrow, cudaMemcpyHostToDevice, S));
  if (!conf.standard()) k_solve_static<CodecGen><<<1, BLOCK, 0, S>>>(kp, sa);
  else k_solve_static<CodecStd><<<1, BLOCK, 0, S>>>(kp, sa);
  CU(cudaGetLastError());
  sol.n_offsets = N + 1;
  if (!sol.off_buf.alloc(s.hpool, (N + 1) * 8)) return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for offsets");
  CU(cudaMemcpyAsync(s.h_ctr, kp.ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
  CU(cudaMemcpyAsync(sol.off_buf.p, sa.out_off, (N + 1) * 8, cudaMemcpyDeviceToHost, S));
  CU(cudaStreamSynchronize(S));
  const Ctr h = *s.h_ctr;
  if ((h.pad & SERR_ARENA) || (h.error & ~DERR_BOUNDS)) {
    sol.off_buf.reset();
    return GEQ_OK;  // the general path grows its arena
  }
  handled = true;
  if (h.pad & SERR_COL) return fail(GEQ_ERR_INVALID_INPUT, "Node index too high: a successor index is out of range");
  if (h.pad & SERR_WEIGHT) return fail(GEQ_ERR_INVALID_INPUT, "an edge update names no element or sets padding bits");
  if (h.error) return fail(GEQ_ERR_INTERNAL, "device error %u (line %u)", h.error, h.err_line);
  if (h.pad & SERR_ROUNDS) return fail(GEQ_ERR_TIMEOUT, "no fixpoint after %u rounds", sa.max_rounds);
  const unsigned long long total = ((const uint64_t *)sol.off_buf.p)[N];
  sol.n_words = total;
  if (!sol.data_buf.alloc(s.hpool, total * 4)) return fail(GEQ_ERR_OUT_OF_MEMORY, "host memory for %llu words", total);
  if (total) CU(cudaMemcpyAsync(sol.data_buf.p, sa.arena + h.arena_top, total * 4, cudaMemcpyDeviceToHost, S));
  CU(cudaEventRecord(s.ev1, S));
  CU(cudaStreamSynchronize(S));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s.ev0, s.ev1);
  sol.energy_size = 1;
  sol.n_vertices.assign(1, (uint32_t)N);
  sol.offsets_base.assign(1, 0);
  sol.data_base.assign(1, 0);
  sol.stats = geq_solve_stats{};
  sol.stats.rounds = h.rounds;
  sol.stats.positions_computed = h.positions;
  sol.stats.edges_relaxed = h.edges;
  sol.stats.algorithmic_bytes = h.bytes;
  sol.stats.kernel_launches = 1;
  sol.stats.device_ms = ms;
  return GEQ_OK;
}

}  // namespace geq
