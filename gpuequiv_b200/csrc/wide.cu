// wide.cu - the energy-game fixpoint for every EnergyConf outside the
// thermometer codecs of codec.cuh: energies of several words (e.g. {30, 3},
// two words), fields too wide for a thermometer code (ONE_DIMENSION =
// {1, u32::MAX}), updates of several words.
//
// Reference: the same path as engine.cu -- EnergyGame::run ->
// GPURunner::execute_gpu (src/energygame.rs:379-383, :1461-1523) with the
// arithmetic the shader preprocessor generates for any conf
// (src/energygame/shadergen.rs:55-157): IMPL_LESS_EQ / IMPL_EQ field-wise on
// the packed words, UPDATE1 (+1 in u32 arithmetic, then min with max),
// UPDATE_MIN (merges in index order), MAX_SUPREMUM.
//
// Layout: energies stay in the crate's packed form (energy_size words, a
// field never straddles a word since energy_bits is a power of two).  Every
// position's list is a slice of one energy arena (descriptor = first energy
// << 24 | count).  The rounds are the reference's Jacobi rounds: a round
// reads only committed lists and writes new lists to fresh arena space; the
// commit publishes them and marks the predecessors of changed positions for
// the next frontier (a bitmap turned into a list).
//
// One warp per frontier position.  A position's new list is built as an
// antichain in the warp's slice of a global scratch: each candidate (an
// inverse-updated successor energy, a supremum) is tested against the
// members by the 32 lanes at once and either dropped or inserted while the
// members it dominates are removed.  Field-wise <= and max run word by word
// with SWAR arithmetic (fields of 1-16 bits in guarded 2k-bit slots; 32-bit
// fields directly).  A position whose antichain outgrows its scratch is
// recorded and computed again in the same round with a larger scratch; a
// round whose results outgrow the arena is run again after the arena has
// been compacted and grown.  Either way only committed lists are read, so a
// repeated computation gives the same lists.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>

#include "geq_internal.h"
#include "wide_arith.cuh"

namespace geq {
namespace wide {

constexpr uint32_t ES_MAX = 64;   // words per energy
constexpr uint32_t US_MAX = 128;  // words per update
constexpr uint32_t WARPS = 4;
constexpr uint32_t BLOCK_T = 32 * WARPS;
constexpr unsigned long long NOCHANGE = ~0ull;
constexpr uint32_t CNT_BITS = 24;
constexpr unsigned long long CNT_MASK = (1ull << CNT_BITS) - 1ull;

struct Ctr {
  unsigned long long arena_top;  // energies in use
  unsigned long long positions, edges, bytes;
  uint32_t next_slot;   // slots handed out to warps
  uint32_t n_ovf;       // slots whose antichain outgrew the warp scratch
  uint32_t arena_full;  // a new list found no arena space
  uint32_t next_size;   // size of the next frontier
};

struct P {
  const uint32_t *row, *col, *wt, *rrow, *rcol;
  const uint8_t *att;
  unsigned long long *desc;
  uint32_t *arena;
  unsigned long long arena_cap;  // energies
  const uint32_t *front;
  const uint32_t *slots;  // null: item i is slot i
  uint32_t n_items;
  unsigned long long *slot_new;
  uint32_t *ovf;
  uint32_t *scratch;
  unsigned long long scratch_words;  // per warp
  Ctr *ctr;
  uint32_t *mark, *next;
  uint32_t n_nodes, mwords;
  uint32_t n_warps;  // warps with a scratch slice (the others of the last block idle)
  uint32_t el, mx, eb, em, ub, um, es, us;
  Swar sw;
  WideConf wc;
};

// Inverse update of one energy in place (UPDATE1 then UPDATE_MIN); u = the
// edge's update words, null for the zero update of an attacker's own list.
__device__ __forceinline__ void inv_update(const P &p, uint32_t *x, const uint32_t *u) { wide_inv_update(p.wc, x, u); }
__device__ __forceinline__ bool leq_w(uint32_t a, uint32_t b, const Swar &s) { return swar_leq(a, b, s); }
__device__ __forceinline__ uint32_t max_w(uint32_t a, uint32_t b, const Swar &s) { return swar_max(a, b, s); }

// The warp's antichain: members in `ac` (es words each), an "own energy" flag
// per member in `fl` (attacker tie rule).
struct Ac {
  uint32_t *ac;
  uint8_t *fl;
  uint32_t n, cap;
};

// Insert candidate x (shared memory, es words): dropped when a member is <=
// x (an equal member takes x's own flag when x is own, as the later copy
// wins); else the members above x leave and x joins.  false: no room.
__device__ bool ac_insert(const P &p, Ac &a, const uint32_t *x, bool own, uint32_t lane) {
  const uint32_t es = p.es;
  bool dom = false, rm = false;
  int eqi = -1;
  for (uint32_t j = lane; j < a.n; j += 32) {
    const uint32_t *m = a.ac + (size_t)j * es;
    bool le = true, ge = true, eq = true;
    for (uint32_t w = 0; w < es && (le || ge); w++) {
      const uint32_t mv = m[w], xv = x[w];
      le = le && leq_w(mv, xv, p.sw);
      ge = ge && leq_w(xv, mv, p.sw);
      eq = eq && mv == xv;
    }
    if (le) {
      dom = true;
      if (eq) eqi = (int)j;
    } else if (ge) {
      rm = true;
    }
  }
  if (__any_sync(0xffffffffu, dom)) {
    if (own && eqi >= 0) a.fl[eqi] = 1;
    return true;
  }
  uint32_t n = a.n;
  if (__any_sync(0xffffffffu, rm)) {
    // remove the members above x, keeping the order (reads of a chunk's word
    // before its writes; destinations never pass their sources)
    uint32_t out = 0;
    for (uint32_t base = 0; base < a.n; base += 32) {
      const uint32_t j = base + lane;
      bool keep = false;
      if (j < a.n) {
        const uint32_t *m = a.ac + (size_t)j * es;
        bool ge = true;
        for (uint32_t w = 0; w < es && ge; w++) ge = leq_w(x[w], m[w], p.sw);
        keep = !ge;
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, keep);
      const uint32_t dst = out + __popc(bal & ((1u << lane) - 1u));
      for (uint32_t w = 0; w < es; w++) {
        const uint32_t val = keep ? a.ac[(size_t)j * es + w] : 0u;
        __syncwarp();
        if (keep) a.ac[(size_t)dst * es + w] = val;
        __syncwarp();
      }
      const uint8_t f = keep ? a.fl[j] : 0;
      __syncwarp();
      if (keep) a.fl[dst] = f;
      __syncwarp();
      out += __popc(bal);
    }
    n = out;
  }
  if (n >= a.cap) return false;
  for (uint32_t w = lane; w < es; w += 32) a.ac[(size_t)n * es + w] = x[w];
  if (lane == 0) a.fl[n] = own ? 1 : 0;
  __syncwarp();
  a.n = n + 1;
  return true;
}

// Append x without a dominance test (a single-successor defender's list is
// its successor's updated list as is).
__device__ bool ac_append(const P &p, Ac &a, const uint32_t *x, uint32_t lane) {
  if (a.n >= a.cap) return false;
  for (uint32_t w = lane; w < p.es; w += 32) a.ac[(size_t)a.n * p.es + w] = x[w];
  if (lane == 0) a.fl[a.n] = 0;
  __syncwarp();
  a.n++;
  return true;
}

__device__ __forceinline__ uint32_t dcnt(unsigned long long d) { return (uint32_t)(d & CNT_MASK); }
__device__ __forceinline__ unsigned long long doff(unsigned long long d) { return d >> CNT_BITS; }

// shared memory of one warp: the update words, 32 staged energies, one candidate
__device__ __forceinline__ uint32_t *warp_smem(const P &p, uint32_t *base, uint32_t wib) {
  return base + (size_t)wib * (p.us + 33u * p.es);
}

// Stage energies [b0, b0+32) of list d, each inverse-updated by u (null: own
// list, clamped); returns how many were staged.
__device__ uint32_t stage(const P &p, uint32_t *stg, unsigned long long d, uint32_t b0, const uint32_t *u,
                          uint32_t lane) {
  const uint32_t cnt = dcnt(d), k = min(32u, cnt - b0);
  if (lane < k) {
    uint32_t *x = stg + (size_t)lane * p.es;
    const uint32_t *src = p.arena + (doff(d) + b0 + lane) * p.es;
    for (uint32_t w = 0; w < p.es; w++) x[w] = src[w];
    inv_update(p, x, u);
  }
  __syncwarp();
  return k;
}

__device__ void load_update(const P &p, uint32_t *ush, unsigned long long k, uint32_t lane) {
  __syncwarp();
  for (uint32_t w = lane; w < p.us; w += 32) ush[w] = p.wt[k * p.us + w];
  __syncwarp();
}

// One position; returns false when its antichain outgrew the scratch.
__device__ bool solve_one(const P &p, uint32_t slot, uint32_t *sm, uint32_t lane, unsigned long long &edges,
                          unsigned long long &bytes) {
  const uint32_t v = p.front[slot];
  const uint32_t e0 = p.row[v], e1 = p.row[v + 1], deg = e1 - e0;
  const bool attacker = p.att[v] != 0;
  uint32_t *ush = sm, *stg = sm + p.us, *xb = stg + 32u * p.es;
  uint32_t *ws = p.scratch + (size_t)(((blockIdx.x * BLOCK_T) + threadIdx.x) >> 5) * p.scratch_words;
  // scratch: two antichains of cap energies and their flags
  const unsigned long long cap_e = p.scratch_words / (2ull * p.es + 1ull);
  const uint32_t cap = (uint32_t)(cap_e < 0xFFFFFFull ? cap_e : 0xFFFFFFull);
  Ac A{ws, (uint8_t *)(ws + 2ull * cap * p.es), 0, cap};
  Ac B{ws + (size_t)cap * p.es, A.fl + cap, 0, cap};
  const unsigned long long esb = 4ull * p.es;
  if (attacker) {
    for (uint32_t k = e0; k < e1; k++) {
      const unsigned long long d = p.desc[p.col[k]];
      bytes += 16 + esb * dcnt(d);
      load_update(p, ush, k, lane);
      for (uint32_t b0 = 0; b0 < dcnt(d); b0 += 32) {
        const uint32_t n = stage(p, stg, d, b0, ush, lane);
        for (uint32_t t = 0; t < n; t++)
          if (!ac_insert(p, A, stg + (size_t)t * p.es, false, lane)) return false;
        __syncwarp();
      }
    }
    edges += deg;
    const unsigned long long dv = p.desc[v];
    bytes += 12 + esb * dcnt(dv);
    for (uint32_t b0 = 0; b0 < dcnt(dv); b0 += 32) {
      const uint32_t n = stage(p, stg, dv, b0, nullptr, lane);
      for (uint32_t t = 0; t < n; t++)
        if (!ac_insert(p, A, stg + (size_t)t * p.es, true, lane)) return false;
      __syncwarp();
    }
    // changed iff a kept energy came from a successor (attack_minimize.wgsl:95-101)
    bool from_succ = false;
    for (uint32_t j = lane; j < A.n; j += 32) from_succ |= A.fl[j] == 0;
    if (!__any_sync(0xffffffffu, from_succ)) {
      if (lane == 0) p.slot_new[slot] = NOCHANGE;
      return true;
    }
  } else {
    // defenders wait until every successor has a list (energygame.rs:789-792)
    bool empty = false;
    for (uint32_t k = e0 + lane; k < e1; k += 32) empty |= dcnt(p.desc[p.col[k]]) == 0;
    if (deg == 0 || __any_sync(0xffffffffu, empty)) {
      if (lane == 0) p.slot_new[slot] = NOCHANGE;
      return true;
    }
    edges += deg;
    bytes += 12;
    {
      const unsigned long long d = p.desc[p.col[e0]];
      bytes += 16 + esb * dcnt(d);
      load_update(p, ush, e0, lane);
      for (uint32_t b0 = 0; b0 < dcnt(d); b0 += 32) {
        const uint32_t n = stage(p, stg, d, b0, ush, lane);
        for (uint32_t t = 0; t < n; t++) {
          const uint32_t *x = stg + (size_t)t * p.es;
          if (!(deg == 1 ? ac_append(p, A, x, lane) : ac_insert(p, A, x, false, lane))) return false;
        }
        __syncwarp();
      }
    }
    // fold: minimal elements of the pairwise suprema, successor by successor
    for (uint32_t k = e0 + 1; k < e1; k++) {
      const unsigned long long d = p.desc[p.col[k]];
      bytes += 16 + esb * dcnt(d);
      load_update(p, ush, k, lane);
      B.n = 0;
      for (uint32_t b0 = 0; b0 < dcnt(d); b0 += 32) {
        const uint32_t n = stage(p, stg, d, b0, ush, lane);
        for (uint32_t t = 0; t < n; t++) {
          const uint32_t *y = stg + (size_t)t * p.es;
          for (uint32_t i = 0; i < A.n; i++) {
            const uint32_t *a = A.ac + (size_t)i * p.es;
            for (uint32_t w = lane; w < p.es; w += 32) xb[w] = max_w(a[w], y[w], p.sw);
            __syncwarp();
            if (!ac_insert(p, B, xb, false, lane)) return false;
            __syncwarp();
          }
        }
        __syncwarp();
      }
      Ac t = A;
      A = B;
      B = t;
    }
    // changed iff the list differs from the old one (EnergyArray ==,
    // energy.rs:334-350: same length and every new energy in the old list)
    const unsigned long long dv = p.desc[v];
    bool same = dcnt(dv) == A.n;
    if (same) {
      bool miss = false;
      for (uint32_t j = lane; j < A.n; j += 32) {
        const uint32_t *x = A.ac + (size_t)j * p.es;
        bool found = false;
        for (uint32_t q = 0; q < dcnt(dv) && !found; q++) {
          const uint32_t *o = p.arena + (doff(dv) + q) * p.es;
          bool eq = true;
          for (uint32_t w = 0; w < p.es && eq; w++) eq = o[w] == x[w];
          found = eq;
        }
        miss |= !found;
      }
      same = !__any_sync(0xffffffffu, miss);
    }
    if (same) {
      if (lane == 0) p.slot_new[slot] = NOCHANGE;
      return true;
    }
  }
  // the new list into fresh arena space
  unsigned long long off = 0;
  if (lane == 0) off = atomicAdd(&p.ctr->arena_top, (unsigned long long)A.n);
  off = __shfl_sync(0xffffffffu, off, 0);
  if (off + A.n > p.arena_cap) {
    if (lane == 0) {
      atomicExch(&p.ctr->arena_full, 1u);
      p.slot_new[slot] = NOCHANGE;
    }
    return true;
  }
  for (size_t w = lane; w < (size_t)A.n * p.es; w += 32) p.arena[off * p.es + w] = A.ac[w];
  bytes += esb * A.n;
  if (lane == 0) p.slot_new[slot] = (off << CNT_BITS) | A.n;
  return true;
}

__global__ void __launch_bounds__(BLOCK_T) k_wide_round(const P p) {
  extern __shared__ uint32_t smem[];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  if (blockIdx.x * WARPS + wib >= p.n_warps) return;
  uint32_t *sm = warp_smem(p, smem, wib);
  unsigned long long edges = 0, bytes = 0, pos = 0;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(&p.ctr->next_slot, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= p.n_items) break;
    const uint32_t slot = p.slots ? p.slots[i] : i;
    if (!solve_one(p, slot, sm, lane, edges, bytes)) {
      if (lane == 0) p.ovf[atomicAdd(&p.ctr->n_ovf, 1u)] = slot;
    } else {
      pos++;
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(&p.ctr->positions, pos);
    atomicAdd(&p.ctr->edges, edges);
    atomicAdd(&p.ctr->bytes, bytes);
  }
}

// publish the round's lists and mark the predecessors of changed positions
__global__ void k_wide_commit(const P p, uint32_t n_slots) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  const unsigned long long d = p.slot_new[s];
  if (d == NOCHANGE) return;
  const uint32_t v = p.front[s];
  p.desc[v] = d;
  for (uint32_t k = p.rrow[v]; k < p.rrow[v + 1]; k++) {
    const uint32_t u = p.rcol[k];
    atomicOr(&p.mark[u >> 5], 1u << (u & 31u));
  }
}

// the next frontier from the bitmap (clears it)
__global__ void k_wide_fill(const P p) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= p.mwords) return;
  uint32_t b = p.mark[w];
  if (!b) return;
  p.mark[w] = 0;
  uint32_t at = atomicAdd(&p.ctr->next_size, (uint32_t)__popc(b));
  while (b) {
    const uint32_t i = (uint32_t)__ffs((int)b) - 1u;
    b &= b - 1u;
    p.next[at++] = w * 32u + i;
  }
}

// initial visit lists: predecessors of the to_reach positions (energygame.rs:1461-1465)
__global__ void k_wide_mark_reach(const P p, const uint32_t *reach, uint32_t n_reach) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_reach) return;
  const uint32_t v = reach[i];
  for (uint32_t k = p.rrow[v]; k < p.rrow[v + 1]; k++) {
    const uint32_t u = p.rcol[k];
    atomicOr(&p.mark[u >> 5], 1u << (u & 31u));
  }
}

// arena compaction: every position's list copied to its new place
__global__ void k_wide_move(const unsigned long long *desc, const unsigned long long *noff, uint32_t n,
                            const uint32_t *src, uint32_t *dst, uint32_t es) {
  const uint32_t v = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
  if (v >= n) return;
  const unsigned long long d = desc[v];
  const size_t words = (size_t)dcnt(d) * es;
  for (size_t w = lane; w < words; w += 32) dst[noff[v] * es + w] = src[doff(d) * es + w];
}

__global__ void k_wide_redesc(unsigned long long *desc, const unsigned long long *noff, uint32_t n) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) desc[v] = (noff[v] << CNT_BITS) | dcnt(desc[v]);
}

// ---- host side ----------------------------------------------------------------
#define WCU(x)                                                                          \
  do {                                                                                  \
    const cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) return fail(e_ == cudaErrorMemoryAllocation ? GEQ_ERR_OUT_OF_MEMORY : GEQ_ERR_CUDA, \
                                       "%s: %s", #x, cudaGetErrorString(e_));           \
  } while (0)

// device buffers of one solve, released with the stream
struct Bufs {
  cudaStream_t S;
  std::vector<void *> ptrs;
  template <class T>
  geq_status get(T *&p, size_t n) {
    void *q = nullptr;
    const cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(n, 1) * sizeof(T), S);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(GEQ_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes for the wide solver failed",
                  std::max<size_t>(n, 1) * sizeof(T));
    }
    ptrs.push_back(q);
    p = (T *)q;
    return GEQ_OK;
  }
  void put(void *q) {
    for (auto &x : ptrs)
      if (x == q) {
        cudaFreeAsync(q, S);
        x = nullptr;
      }
  }
  ~Bufs() {
    for (void *q : ptrs)
      if (q) cudaFreeAsync(q, S);
  }
};

static geq_status check_game(const GameInput &gi, const Conf &c) {
  const geq_game_graph &g = gi.g;
  const uint32_t n = g.n_vertices, us = c.update_size(), ub = c.update_bits(), um = c.update_mask();
  const uint64_t m = g.row_offsets[n];
  for (uint32_t v = 0; v < n; v++)
    if (g.row_offsets[v + 1] < g.row_offsets[v]) return fail(GEQ_ERR_INVALID_INPUT, "row_offsets not monotone at %u", v);
  for (uint64_t k = 0; k < m; k++)
    if (g.column_indices[k] >= n) return fail(GEQ_ERR_INVALID_INPUT, "Node index too high: successor %u of %u positions",
                                              g.column_indices[k], n);
  // update codes: 0 Zero, 1 Decrement, k+2 Min into element k < elements;
  // bits past the last field are padding and must be clear
  const uint64_t fields_bits = (uint64_t)ub * c.elements;
  for (uint64_t k = 0; k < m; k++) {
    const uint32_t *u = g.weights + k * us;
    for (uint32_t i = 0; i < c.elements; i++) {
      const uint32_t bit = i * ub, code = (u[bit >> 5] >> (bit & 31u)) & um;
      if (code >= 2 && code - 2 >= c.elements)
        return fail(GEQ_ERR_INVALID_INPUT, "edge %llu: update code %u names no element", (unsigned long long)k, code);
    }
    if (fields_bits % 32) {
      const uint32_t pad = ~0u << (fields_bits % 32);
      if (u[us - 1] & pad) return fail(GEQ_ERR_INVALID_INPUT, "edge %llu: update padding bits set", (unsigned long long)k);
    }
  }
  return GEQ_OK;
}

// One game on the engine's stream.
static geq_status solve_one_game(cudaStream_t S, int n_sms, const GameInput &gi, const Conf &c, geq_solution &sol,
                                 uint32_t g_index) {
  const geq_game_graph &g = gi.g;
  const uint32_t n = g.n_vertices, es = c.energy_size(), us = c.update_size();
  const uint64_t m = g.row_offsets[n];
  geq_status st = check_game(gi, c);
  if (st) return st;
  // reverse CSR (energygame.rs:235-250), predecessors in increasing order
  std::vector<uint32_t> rrow(n + 1, 0), rcol(m);
  for (uint64_t k = 0; k < m; k++) rrow[g.column_indices[k] + 1]++;
  for (uint32_t v = 0; v < n; v++) rrow[v + 1] += rrow[v];
  {
    std::vector<uint32_t> fill(rrow.begin(), rrow.end() - 1);
    for (uint32_t v = 0; v < n; v++)
      for (uint32_t k = g.row_offsets[v]; k < g.row_offsets[v + 1]; k++) rcol[fill[g.column_indices[k]]++] = v;
  }
  // initial lists: given, or {0} at the to_reach positions (with_reach, energygame.rs:355-365)
  std::vector<unsigned long long> desc(n, 0);
  std::vector<uint32_t> init_words;
  if (gi.init) {
    for (uint32_t v = 0; v < n; v++) {
      const uint64_t a = gi.init->offsets[v], b = gi.init->offsets[v + 1];
      desc[v] = ((unsigned long long)a << CNT_BITS) | (b - a);
    }
    init_words.assign(gi.init->data, gi.init->data + gi.init->offsets[n] * es);
  } else {
    for (uint32_t i = 0; i < gi.n_reach; i++) {
      const uint32_t v = gi.to_reach[i];
      if (desc[v]) continue;
      desc[v] = ((unsigned long long)(init_words.size() / es) << CNT_BITS) | 1ull;
      init_words.insert(init_words.end(), es, 0u);
    }
  }
  const unsigned long long init_e = init_words.size() / es;

  Bufs B{S, {}};
  P p{};
  uint32_t *d_row, *d_col, *d_wt, *d_rrow, *d_rcol, *d_front, *d_next, *d_ovf, *d_mark, *d_reach, *d_arena,
      *d_scratch;
  uint8_t *d_att;
  unsigned long long *d_desc, *d_slot;
  Ctr *d_ctr;
  const uint32_t mwords = (n + 31) / 32;
  if ((st = B.get(d_row, n + 1)) || (st = B.get(d_col, m)) || (st = B.get(d_wt, m * us)) ||
      (st = B.get(d_rrow, n + 1)) || (st = B.get(d_rcol, m)) || (st = B.get(d_att, n)) ||
      (st = B.get(d_desc, n)) || (st = B.get(d_front, n)) || (st = B.get(d_next, n)) ||
      (st = B.get(d_ovf, n)) || (st = B.get(d_mark, mwords)) || (st = B.get(d_slot, n)) ||
      (st = B.get(d_ctr, 1)) || (st = B.get(d_reach, gi.n_reach)))
    return st;
  unsigned long long arena_cap = std::max<unsigned long long>(4 * init_e + 16ull * (n + m), 1ull << 16);
  if ((st = B.get(d_arena, arena_cap * es))) return st;
  const uint32_t max_warps = (uint32_t)n_sms * 16;
  unsigned long long scratch_words = 1ull << 14;  // per warp
  uint32_t scratch_warps = max_warps;
  if ((st = B.get(d_scratch, scratch_words * scratch_warps))) return st;

  WCU(cudaMemcpyAsync(d_row, g.row_offsets, (n + 1) * 4ull, cudaMemcpyHostToDevice, S));
  if (m) {
    WCU(cudaMemcpyAsync(d_col, g.column_indices, m * 4, cudaMemcpyHostToDevice, S));
    WCU(cudaMemcpyAsync(d_wt, g.weights, m * us * 4, cudaMemcpyHostToDevice, S));
    WCU(cudaMemcpyAsync(d_rcol, rcol.data(), m * 4, cudaMemcpyHostToDevice, S));
  }
  WCU(cudaMemcpyAsync(d_rrow, rrow.data(), (n + 1) * 4ull, cudaMemcpyHostToDevice, S));
  std::vector<uint8_t> att(n);
  for (uint32_t v = 0; v < n; v++) att[v] = g.attacker_pos[v] ? 1 : 0;
  if (n) {
    WCU(cudaMemcpyAsync(d_att, att.data(), n, cudaMemcpyHostToDevice, S));
    WCU(cudaMemcpyAsync(d_desc, desc.data(), n * 8ull, cudaMemcpyHostToDevice, S));
  }
  if (!init_words.empty())
    WCU(cudaMemcpyAsync(d_arena, init_words.data(), init_words.size() * 4, cudaMemcpyHostToDevice, S));
  if (gi.n_reach) WCU(cudaMemcpyAsync(d_reach, gi.to_reach, gi.n_reach * 4ull, cudaMemcpyHostToDevice, S));
  WCU(cudaMemsetAsync(d_mark, 0, mwords * 4ull, S));
  {
    // new lists go after the initial ones
    Ctr h0{};
    h0.arena_top = init_e;
    WCU(cudaMemcpyAsync(d_ctr, &h0, sizeof(Ctr), cudaMemcpyHostToDevice, S));
    WCU(cudaStreamSynchronize(S));  // h0 is on the stack
  }

  p.row = d_row; p.col = d_col; p.wt = d_wt; p.rrow = d_rrow; p.rcol = d_rcol; p.att = d_att;
  p.desc = d_desc; p.arena = d_arena; p.arena_cap = arena_cap;
  p.front = d_front; p.slots = nullptr; p.slot_new = d_slot; p.ovf = d_ovf;
  p.scratch = d_scratch; p.scratch_words = scratch_words; p.ctr = d_ctr;
  p.mark = d_mark; p.next = d_next; p.n_nodes = n; p.mwords = mwords;
  p.el = c.elements; p.mx = c.max; p.eb = c.energy_bits(); p.em = c.energy_mask();
  p.ub = c.update_bits(); p.um = c.update_mask(); p.es = es; p.us = us;
  p.sw = make_swar(p.eb);
  p.wc = WideConf{p.el, p.mx, p.eb, p.em, p.ub, p.um};
  const size_t smem = (size_t)WARPS * (us + 33u * es) * 4;
  WCU(cudaFuncSetAttribute(k_wide_round, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

  cudaEvent_t ev0, ev1;
  WCU(cudaEventCreate(&ev0));
  WCU(cudaEventCreate(&ev1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } evg{ev0, ev1};
  WCU(cudaEventRecord(ev0, S));
  unsigned long long launches = 0;
  if (gi.n_reach) {
    k_wide_mark_reach<<<(gi.n_reach + 255) / 256, 256, 0, S>>>(p, d_reach, gi.n_reach);
    launches++;
  }
  Ctr h{};
  auto fill_next = [&](uint32_t &size) -> geq_status {
    WCU(cudaMemsetAsync(&d_ctr->next_size, 0, 4, S));
    k_wide_fill<<<(mwords + 255) / 256, 256, 0, S>>>(p);
    launches++;
    WCU(cudaMemcpyAsync(&h, d_ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
    WCU(cudaStreamSynchronize(S));
    size = h.next_size;
    return GEQ_OK;
  };
  uint32_t fsize = 0;
  if (n && (st = fill_next(fsize))) return st;
  std::swap(d_front, d_next);
  p.front = d_front;
  p.next = d_next;
  uint64_t rounds = 0;
  const auto t_start = std::chrono::steady_clock::now();
  while (fsize) {
    rounds++;
    if (std::chrono::steady_clock::now() - t_start > std::chrono::seconds(600))
      return fail(GEQ_ERR_TIMEOUT, "no fixpoint after 600 s (%llu rounds)", (unsigned long long)rounds);
    // the round, repeated for positions whose antichain outgrew the scratch
    p.slots = nullptr;
    p.n_items = fsize;
    for (;;) {
      WCU(cudaMemsetAsync(&d_ctr->next_slot, 0, 4, S));
      WCU(cudaMemsetAsync(&d_ctr->n_ovf, 0, 4, S));
      WCU(cudaMemsetAsync(&d_ctr->arena_full, 0, 4, S));
      const uint32_t warps = std::min<uint32_t>(scratch_warps, std::max<uint32_t>(p.n_items, 1));
      p.n_warps = warps;
      k_wide_round<<<(warps + WARPS - 1) / WARPS, BLOCK_T, smem, S>>>(p);
      launches++;
      WCU(cudaGetLastError());
      WCU(cudaMemcpyAsync(&h, d_ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
      WCU(cudaStreamSynchronize(S));
      if (h.arena_full) {
        // compact the committed lists into a larger arena and run the round again
        std::vector<unsigned long long> hd(n), noff(n);
        WCU(cudaMemcpyAsync(hd.data(), d_desc, n * 8ull, cudaMemcpyDeviceToHost, S));
        WCU(cudaStreamSynchronize(S));
        unsigned long long live = 0;
        for (uint32_t v = 0; v < n; v++) {
          noff[v] = live;
          live += hd[v] & CNT_MASK;
        }
        const unsigned long long cap2 = std::max(2 * arena_cap, 4 * live + (1ull << 16));
        uint32_t *na;
        unsigned long long *d_noff;
        if ((st = B.get(na, cap2 * es)) || (st = B.get(d_noff, n))) return st;
        WCU(cudaMemcpyAsync(d_noff, noff.data(), n * 8ull, cudaMemcpyHostToDevice, S));
        k_wide_move<<<(n + 7) / 8, 256, 0, S>>>(d_desc, d_noff, n, d_arena, na, es);
        k_wide_redesc<<<(n + 255) / 256, 256, 0, S>>>(d_desc, d_noff, n);
        launches += 2;
        B.put(d_arena);
        B.put(d_noff);
        d_arena = na;
        arena_cap = cap2;
        p.arena = d_arena;
        p.arena_cap = arena_cap;
        WCU(cudaMemcpyAsync(&d_ctr->arena_top, &live, 8, cudaMemcpyHostToDevice, S));
        p.slots = nullptr;
        p.n_items = fsize;
        continue;
      }
      if (!h.n_ovf) break;
      // positions whose antichain did not fit: again with 8x the scratch
      // each, on as many warps as the memory allows
      scratch_words *= 8;
      if (scratch_words > (1ull << 31)) return fail(GEQ_ERR_OUT_OF_MEMORY, "antichain beyond 8 GB of warp scratch");
      B.put(d_scratch);
      scratch_warps = (uint32_t)std::max<unsigned long long>(
          1, std::min<unsigned long long>(max_warps, (4ull << 30) / (scratch_words * 4)));
      if ((st = B.get(d_scratch, scratch_words * scratch_warps))) return st;
      // the overflowed slots become the items (copied: the kernel appends to ovf)
      uint32_t *d_items;
      if ((st = B.get(d_items, h.n_ovf))) return st;
      WCU(cudaMemcpyAsync(d_items, d_ovf, h.n_ovf * 4ull, cudaMemcpyDeviceToDevice, S));
      p.scratch = d_scratch;
      p.scratch_words = scratch_words;
      p.slots = d_items;
      p.n_items = h.n_ovf;
    }
    k_wide_commit<<<(fsize + 255) / 256, 256, 0, S>>>(p, fsize);
    launches++;
    if ((st = fill_next(fsize))) return st;
    std::swap(d_front, d_next);
    p.front = d_front;
    p.next = d_next;
  }
  WCU(cudaEventRecord(ev1, S));
  // download: offsets and words of every list
  std::vector<unsigned long long> hd(n);
  if (n) WCU(cudaMemcpyAsync(hd.data(), d_desc, n * 8ull, cudaMemcpyDeviceToHost, S));
  WCU(cudaMemcpyAsync(&h, d_ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, S));
  WCU(cudaStreamSynchronize(S));
  std::vector<unsigned long long> noff(n);
  unsigned long long total = 0;
  for (uint32_t v = 0; v < n; v++) {
    noff[v] = total;
    total += hd[v] & CNT_MASK;
  }
  uint32_t *d_out = nullptr;
  unsigned long long *d_noff = nullptr;
  if ((st = B.get(d_out, total * es)) || (st = B.get(d_noff, n))) return st;
  if (n) {
    WCU(cudaMemcpyAsync(d_noff, noff.data(), n * 8ull, cudaMemcpyHostToDevice, S));
    k_wide_move<<<(n + 7) / 8, 256, 0, S>>>(d_desc, d_noff, n, d_arena, d_out, es);
    launches++;
  }
  const uint64_t ob = sol.offsets.size(), db = sol.data.size() / es;
  sol.n_vertices.push_back(n);
  sol.offsets_base.push_back(ob);
  sol.data_base.push_back(db);
  sol.offsets.resize(ob + n + 1);
  for (uint32_t v = 0; v < n; v++) sol.offsets[ob + v] = noff[v];
  sol.offsets[ob + n] = total;
  sol.data.resize((db + total) * es);
  if (total) WCU(cudaMemcpyAsync(sol.data.data() + db * es, d_out, total * es * 4, cudaMemcpyDeviceToHost, S));
  WCU(cudaStreamSynchronize(S));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0, ev1);
  sol.stats.rounds += rounds;
  sol.stats.positions_computed += h.positions;
  sol.stats.edges_relaxed += h.edges;
  sol.stats.algorithmic_bytes += h.bytes;
  sol.stats.kernel_launches += launches;
  sol.stats.device_ms += ms;
  (void)g_index;
  return GEQ_OK;
}

}  // namespace wide

bool wide_supported(const Conf &c, std::string *why) {
  if (c.energy_size() > wide::ES_MAX || c.update_size() > wide::US_MAX) {
    if (why)
      *why = "EnergyConf {" + std::to_string(c.elements) + ", " + std::to_string(c.max) + "} needs " +
             std::to_string(c.energy_size()) + " energy / " + std::to_string(c.update_size()) +
             " update words (the solver takes up to " + std::to_string(wide::ES_MAX) + " / " +
             std::to_string(wide::US_MAX) + ")";
    return false;
  }
  return c.elements >= 1;
}

geq_status solve_wide(Engine &e, int device, std::vector<GameInput> &in, geq_solution &sol) {
  if (in.empty()) return fail(GEQ_ERR_INVALID_INPUT, "no games");
  const Conf c(in[0].g.conf);
  std::string why;
  if (!wide_supported(c, &why)) return fail(GEQ_ERR_UNSUPPORTED, "%s", why.c_str());
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device) cudaSetDevice(device);
  struct Restore {
    int prev, dev;
    ~Restore() { if (prev != dev && prev >= 0) cudaSetDevice(prev); }
  } restore{prev, device};
  cudaStream_t S = (cudaStream_t)e.stream_handle();
  sol.energy_size = c.energy_size();
  for (uint32_t g = 0; g < in.size(); g++) {
    GameInput &gi = in[g];
    if (gi.std_reach) {
      gi.reach_storage = standard_reach_of(gi.g);
      gi.to_reach = gi.reach_storage.data();
      gi.n_reach = (uint32_t)gi.reach_storage.size();
      gi.std_reach = false;
    }
    const geq_status st = wide::solve_one_game(S, e.n_sms, gi, c, sol, g);
    if (st) return st;
  }
  return GEQ_OK;
}

}  // namespace geq
