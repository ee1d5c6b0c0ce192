// gbuild.cu - the device game builder (gbuild.cuh) and the device
// minimisation (refine.cuh) on the CUDA stream of a context:
// GameBuild::compare (src/gamebuild.rs:165-170) for a batch of (LTS, p, q)
// jobs, one breadth-first level per pass over the level kernels (all levels
// inside one CUDA graph WHILE node), results either copied back as one CSR
// game graph per job (geq_game_build_compare_batch) or handed to the solver
// on the device (build_and_upload, used by geq_compare_batch, the serving
// loop's queries and geq_equivalences); and
// TransitionSystem::signature_refinement of many systems at once
// (geq_lts_signature_refinement_batch).
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "gbuild.cuh"
#include "refine.cuh"
#include "geq_internal.h"
#include "lts.h"

namespace geq {
namespace gb {

constexpr int EACH_T = 256;
// blocks per SM of the level kernels' grids (grid-stride loops over the
// level's items; the count is only known on the device)
#ifndef GEQ_EACH_BLOCKS_PER_SM
#define GEQ_EACH_BLOCKS_PER_SM 16  // measured: 2 → 99 ms, 4 → 80.5, 8 → 74.4, 12 → 73.0, 16 → 72.3 per build of the batch
#endif
constexpr int SCAN_T = 256;
#ifndef GEQ_SCAN_ITEMS
#define GEQ_SCAN_ITEMS 8  // values per thread of a scan tile
#endif
constexpr int SCAN_ITEMS = GEQ_SCAN_ITEMS;
constexpr uint32_t SCAN_TILE = SCAN_T * SCAN_ITEMS;

template <class F>
__global__ void __launch_bounds__(EACH_T) k_each(uint32_t n, F f) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f(i);
}
// the same with the count read on the device; nothing while *go == 0
template <class F>
__global__ void __launch_bounds__(EACH_T) k_each_d(const unsigned long long *np, const unsigned long long *go, F f) {
  if (!*go) return;
  const uint32_t n = (uint32_t)*np;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f(i);
}

// exclusive scan of a block's values (one per thread); returns the block total
__device__ __forceinline__ unsigned long long block_scan(unsigned long long x, unsigned long long &total) {
  __shared__ unsigned long long ws[SCAN_T / 32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (uint32_t)o) inc += y;
  }
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    unsigned long long s = lane < SCAN_T / 32 ? ws[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    if (lane < SCAN_T / 32) ws[lane] = s;
  }
  __syncthreads();
  const unsigned long long before = (w ? ws[w - 1] : 0ull) + inc - x;
  total = ws[SCAN_T / 32 - 1];
  __syncthreads();
  return before;
}

// per tile of SCAN_TILE values: its sum
__global__ void __launch_bounds__(SCAN_T) k_scan_up(const uint32_t *in, uint32_t n, unsigned long long *part) {
  const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  unsigned long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++)
    if (base + k < n) s += in[base + k];
  unsigned long long total;
  block_scan(s, total);
  if (threadIdx.x == 0) part[blockIdx.x] = total;
}
// exclusive scan of the tile sums in one block; the grand total to *tot
__global__ void __launch_bounds__(SCAN_T) k_scan_mid(unsigned long long *part, uint32_t nb, unsigned long long *tot) {
  unsigned long long carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += SCAN_T) {
    const uint32_t i = b0 + threadIdx.x;
    const unsigned long long x = i < nb ? part[i] : 0ull;
    unsigned long long total;
    const unsigned long long e = block_scan(x, total);
    if (i < nb) part[i] = carry + e;
    carry += total;
  }
  if (threadIdx.x == 0) *tot = carry;
}
__global__ void __launch_bounds__(SCAN_T) k_scan_down(const uint32_t *in, uint32_t n, const unsigned long long *part,
                                                      uint32_t *out) {
  const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  unsigned long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < n ? in[base + k] : 0u;
    s += v[k];
  }
  unsigned long long total;
  unsigned long long e = block_scan(s, total) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++)
    if (base + k < n) {
      out[base + k] = (uint32_t)e;
      e += v[k];
    }
}

// Single-pass scans of up to three arrays, each with its item count read on
// the device (chained scan with decoupled look-back): block b scans tiles b,
// b + G, b + 2G, ... of SCAN_TILE values.  A tile publishes its sum at once,
// then looks back over the tiles before it -- one warp reading the status
// words of 32 tiles at a time, adding published sums until it meets a
// published inclusive prefix -- and publishes its own inclusive prefix.  The status words carry the scan's sequence number (bumped by the
// last block of every launch), so no clearing is needed between launches.
// The look-back waits are bounded: a tile that gives up sums its
// predecessors' inputs itself, so the result never depends on how the blocks
// were scheduled.
struct ScanR {
  const uint32_t *in[3];
  uint32_t *out[3];
  const unsigned long long *np[3];
  unsigned long long *tot[3];
};
struct LbCtl {
  uint32_t seq, done;
};
constexpr uint32_t LB_AGG = 1u, LB_INC = 2u;
constexpr uint32_t LB_SPIN_LIMIT = 1u << 16;
constexpr uint32_t LB_FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t ld_vol(const uint32_t *p) { return *(const volatile uint32_t *)p; }
__device__ __forceinline__ unsigned long long ld_vol(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

template <int R>
__global__ void __launch_bounds__(SCAN_T) k_lbscan(ScanR a, const unsigned long long *go, LbCtl *ctl, uint32_t *flag,
                                                   unsigned long long *agg, unsigned long long *inc, uint32_t tcap) {
  __shared__ uint32_t s_seq, s_gaveup;
  __shared__ unsigned long long s_prefix;
  const bool run = !go || *go;
  if (threadIdx.x == 0) s_seq = ld_vol(&ctl->seq) & 0x3FFFFFFFu;
  __syncthreads();
  const uint32_t tag = s_seq << 2;
#pragma unroll
  for (int r = 0; r < R && run; r++) {
    const uint32_t n = (uint32_t)*a.np[r];
    const uint32_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    uint32_t *fl = flag + (size_t)r * tcap;
    unsigned long long *ag = agg + (size_t)r * tcap, *ic = inc + (size_t)r * tcap;
    if (ntiles == 0 && blockIdx.x == 0 && threadIdx.x == 0) *a.tot[r] = 0ull;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const bool status = t < tcap;  // tiles beyond the status space take the direct path
      const uint32_t base = t * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
      uint32_t v[SCAN_ITEMS];
      unsigned long long s = 0;
#pragma unroll
      for (int k = 0; k < SCAN_ITEMS; k++) {
        v[k] = base + k < n ? a.in[r][base + k] : 0u;
        s += v[k];
      }
      unsigned long long total;
      unsigned long long e = block_scan(s, total);
      if (threadIdx.x < 32) {
        // warp 0 looks back 32 tiles at a time: lane k reads tile hi - k
        const uint32_t lane = threadIdx.x;
        unsigned long long prefix = 0;
        uint32_t gaveup = 0;
        if (!status) {
          gaveup = 1;
        } else if (t == 0) {
          if (lane == 0) {
            ic[0] = total;
            __threadfence();
            *(volatile uint32_t *)&fl[0] = tag | LB_INC;
          }
        } else {
          if (lane == 0) {
            ag[t] = total;
            __threadfence();
            *(volatile uint32_t *)&fl[t] = tag | LB_AGG;
          }
          long long hi = (long long)t - 1;
          uint32_t spins = 0;
          for (;;) {
            const long long j = hi - (long long)lane;
            const uint32_t f = j >= 0 ? ld_vol(&fl[j]) : 0u;
            const bool ready = j >= 0 && (f & ~3u) == tag && (f & 3u) != 0u;
            const uint32_t incm = __ballot_sync(LB_FULL, ready && (f & 3u) == LB_INC);
            const uint32_t waitm = __ballot_sync(LB_FULL, j >= 0 && !ready);
            // tiles hi .. the nearest inclusive prefix (or the whole window)
            // must all have published; tile 0 always publishes an inclusive one
            const uint32_t need = incm ? ((incm & (0u - incm)) << 1) - 1u : LB_FULL;
            if (waitm & need) {
              if (++spins > LB_SPIN_LIMIT) {
                gaveup = 1;
                break;
              }
              __nanosleep(64);
              continue;
            }
            __threadfence();
            const bool mine = ((need >> lane) & 1u) != 0u && j >= 0;
            unsigned long long x = 0;
            if (mine) x = ((f & 3u) == LB_INC) ? ld_vol(&ic[j]) : ld_vol(&ag[j]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(LB_FULL, x, o);
            prefix += x;
            if (incm) break;
            hi -= 32;
          }
        }
        if (lane == 0) {
          s_prefix = prefix;
          s_gaveup = gaveup;
        }
      }
      __syncthreads();
      if (s_gaveup) {
        // the block sums the inputs of every tile before this one itself
        unsigned long long part = 0;
        for (uint32_t i = threadIdx.x; i < t * SCAN_TILE; i += SCAN_T) part += a.in[r][i];
        unsigned long long all;
        block_scan(part, all);
        if (threadIdx.x == 0) s_prefix = all;
        __syncthreads();
      }
      const unsigned long long prefix = s_prefix;
      if (threadIdx.x == 0 && t > 0 && status) {
        ic[t] = prefix + total;
        __threadfence();
        *(volatile uint32_t *)&fl[t] = tag | LB_INC;
      }
      if (threadIdx.x == 0 && t + 1 == ntiles) *a.tot[r] = prefix + total;
      e += prefix;
#pragma unroll
      for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) {
          a.out[r][base + k] = (uint32_t)e;
          e += v[k];
        }
      __syncthreads();
    }
  }
  // the last block of the launch moves the sequence on
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->done, 1u) == gridDim.x - 1) {
      ctl->done = 0;
      ctl->seq = ctl->seq + 1u;
      __threadfence();
    }
  }
}

// ---- the warp path for attack positions with many q's ------------------------
// AttackPosition::successors (gamepos.rs:17-106) by one warp: each label's
// union Q' is a bitmap over the job's states in shared memory (its set bits in
// order are the sorted union), the observation moves and the enabledness
// splits are placed by ballots in the reference's order.  Same output as
// gen_one.
constexpr int GH_WARPS = 8;
#ifndef GEQ_BUILD_HEAVY_MIN
#define GEQ_BUILD_HEAVY_MIN 6  // attack positions with this many q's or more take the warp path; measured: 2 → 70.4 ms, 3 → 68.2, 4 → 66.6, 6 → 64.8, 8 → 64.7, 12 → 66.0 per build of the batch
#endif
#ifndef GEQ_GH_BLOCKS_PER_SM
#define GEQ_GH_BLOCKS_PER_SM 4  // k_gen_heavy blocks per SM (32 KB of shared memory each); measured: 2 → 72.5 ms, 4 → 67.6, 6 → 69.1 per build of the batch
#endif
constexpr uint32_t GH_BM_WORDS = 1024;  // jobs of up to 32768 states; larger ones: gen_one by lane 0
constexpr uint32_t FULLMASK = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ uint32_t warp_scan_incl(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULLMASK, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}

__device__ void gen_attack_warp(const View &v, uint32_t i, uint32_t *bm, uint32_t lane) {
  const Key x = v.nkey[F0(v) + i];
  const uint32_t j = v.sjob[x.p];
  const uint32_t sb = v.jsb[j], nw = (v.jsb[j + 1] - sb + 31) / 32;
  if (nw > GH_BM_WORDS) {
    if (lane == 0) gen_one(v, i);
    return;
  }
  const uint32_t s0 = v.off_s[i], ns = v.ub_s[i], c0 = v.off_c[i], nc = v.ub_c[i], e0 = v.off_e[i];
  const uint32_t nq = v.slen[x.a];
  const uint32_t *Q = v.sdata + v.sstart[x.a];
  uint32_t *el = v.celem + e0;
  uint32_t cnt = 0, cc = 0, ecur = 0;
  uint32_t k = v.soff[x.p];
  const uint32_t ke = v.soff[x.p + 1];
  while (k < ke) {
    const int32_t a = v.slab[k];
    uint32_t run_end = k + 1;
    while (run_end < ke && v.slab[run_end] == a) run_end++;
    for (uint32_t w = lane; w < nw; w += 32) bm[w] = 0u;
    __syncwarp();
    for (uint32_t t = lane; t < nq; t += 32) {
      const uint32_t q = Q[t];
      for (uint32_t u = label_lower(v, q, a); u < v.soff[q + 1] && v.slab[u] == a; u++) {
        const uint32_t s = v.stgt[u] - sb;
        atomicOr(&bm[s >> 5], 1u << (s & 31));
      }
    }
    __syncwarp();
    uint32_t len = 0;
    for (uint32_t w0 = 0; w0 < nw; w0 += 32) {
      const uint32_t w = w0 + lane;
      uint32_t bits = w < nw ? bm[w] : 0u;
      const uint32_t c = __popc(bits);
      const uint32_t incl = warp_scan_incl(c, lane);
      uint32_t o = ecur + len + incl - c;
      while (bits) {
        el[o++] = sb + w * 32 + (uint32_t)(__ffs(bits) - 1);
        bits &= bits - 1;
      }
      len += __shfl_sync(FULLMASK, incl, 31);
    }
    if (lane == 0) {
      v.cstart[c0 + cc] = e0 + ecur;
      v.clen[c0 + cc] = len;
    }
    const uint32_t qref = CAND | (c0 + cc);
    cc++;
    for (uint32_t kk = k; kk < run_end; kk += 32) {
      const uint32_t idx = kk + lane;
      bool keep = false;
      uint32_t p2 = 0;
      if (idx < run_end) {
        p2 = v.stgt[idx];
        const uint32_t s = p2 - sb;
        keep = ((bm[s >> 5] >> (s & 31)) & 1u) == 0u;
      }
      const uint32_t bal = __ballot_sync(FULLMASK, keep);
      if (keep) {
        const uint32_t pos = s0 + cnt + __popc(bal & lane_lt());
        v.succ[pos] = Key{K_ATTACK, p2, qref, 0};
        v.swt[pos] = W_OBS;
      }
      cnt += __popc(bal);
    }
    ecur += len;
    k = run_end;
    __syncwarp();
  }
  if (lane == 0) {
    v.succ[s0 + cnt] = Key{K_DEFEND, x.p, x.a, 0};
    v.swt[s0 + cnt] = W_CHAL;
  }
  cnt++;
  // enabledness splits: flags per q, then a stable partition per pair
  uint32_t *b0 = el + ecur, *fl = el + ecur + 3 * nq;
  uint32_t n1[3] = {0, 0, 0};
  for (uint32_t t0 = 0; t0 < nq; t0 += 32) {
    const uint32_t t = t0 + lane;
    uint32_t f = 0;
    if (t < nq) {
      bool sub, sup;
      compare_enabled(v, x.p, Q[t], sub, sup);
      f = (sub ? 1u : 0u) | (sup ? 2u : 0u) | ((sub && sup) ? 4u : 0u);
      fl[t] = f;
    }
#pragma unroll
    for (int pr = 0; pr < 3; pr++) n1[pr] += __popc(__ballot_sync(FULLMASK, t < nq && ((f >> pr) & 1u)));
  }
  uint32_t r0[3] = {0, 0, 0}, r1[3] = {0, 0, 0};
  for (uint32_t t0 = 0; t0 < nq; t0 += 32) {
    const uint32_t t = t0 + lane;
    const uint32_t f = t < nq ? fl[t] : 0u;
    const uint32_t q = t < nq ? Q[t] : 0u;
#pragma unroll
    for (int pr = 0; pr < 3; pr++) {
      const bool pass = ((f >> pr) & 1u) != 0u;
      const uint32_t bp = __ballot_sync(FULLMASK, t < nq && pass), bf = __ballot_sync(FULLMASK, t < nq && !pass);
      uint32_t *b = b0 + (uint32_t)pr * nq;
      if (t < nq) {
        if (pass) b[nq - n1[pr] + r1[pr] + __popc(bp & lane_lt())] = q;
        else b[r0[pr] + __popc(bf & lane_lt())] = q;
      }
      r0[pr] += __popc(bf);
      r1[pr] += __popc(bp);
    }
  }
  __syncwarp();
  uint32_t pushed[3];
  uint32_t np = 0;
  for (uint32_t pr = 0; pr < 3; pr++) {
    const uint32_t nqx = n1[pr], nqs = nq - nqx;
    if (nqs == 0 || nqx == 0) continue;
    bool dup = false;  // push_unique: an equal split was pushed already
    for (uint32_t o = 0; o < np && !dup; o++) {
      const uint32_t po = pushed[o];
      if (n1[po] != nqx) continue;
      bool diff = false;
      for (uint32_t t = lane; t < nq; t += 32) diff |= b0[po * nq + t] != b0[pr * nq + t];
      dup = !__any_sync(FULLMASK, diff);
    }
    if (dup) continue;
    if (lane == 0) {
      v.cstart[c0 + cc] = e0 + ecur + pr * nq;
      v.clen[c0 + cc] = nqs;
      v.cstart[c0 + cc + 1] = e0 + ecur + pr * nq + nqs;
      v.clen[c0 + cc + 1] = nqx;
      v.succ[s0 + cnt] = Key{K_DEFEND, x.p, CAND | (c0 + cc), CAND | (c0 + cc + 1)};
      v.swt[s0 + cnt] = W_CHAL;
    }
    cc += 2;
    cnt++;
    pushed[np++] = pr;
  }
  for (uint32_t t = cnt + lane; t < ns; t += 32) v.succ[s0 + t] = Key{K_NONE, 0, 0, 0};
  for (uint32_t t = cc + lane; t < nc; t += 32) v.clen[c0 + t] = UNSET;
  if (lane == 0) v.fcnt[i] = cnt;
}

// End of one level inside the graph's WHILE node: run the next level while
// the loop may go on, at most ctr[1] levels per graph launch (ctr[0] counts).
__global__ void k_level_cond(cudaGraphConditionalHandle h, const unsigned long long *go, uint32_t *ctr) {
  const uint32_t k = ++ctr[0];
  cudaGraphSetConditional(h, (*go != 0ull && k < ctr[1]) ? 1u : 0u);
}

__global__ void __launch_bounds__(GH_WARPS * 32) k_gen_heavy(View v, const unsigned long long *go) {
  __shared__ uint32_t bm_all[GH_WARPS][GH_BM_WORDS];
  if (go && !*go) return;
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nh = v.ctl->n_heavy;
  for (uint32_t h = blockIdx.x * GH_WARPS + wib; h < nh; h += gridDim.x * GH_WARPS)
    gen_attack_warp(v, v.hq[h], bm_all[wib], lane);
}

// Backend of the level loop: stream-ordered allocation, kernels and copies on
// the context's stream.
struct DevBackend {
  cudaStream_t s = nullptr;
  int n_sms = 148;
  cudaError_t err = cudaSuccess;
  unsigned long long *part = nullptr;
  uint32_t part_cap = 0;
  uint32_t launches = 0;
  // single-pass scans: sequence/arrival counters and per-tile status of up to
  // three arrays (lb_cap tiles each)
  LbCtl *lb_ctl = nullptr;
  uint32_t *lb_flag = nullptr;
  unsigned long long *lb_agg = nullptr, *lb_inc = nullptr;
  uint32_t lb_cap = 0;

  void note(cudaError_t e) {
    if (e != cudaSuccess && err == cudaSuccess) err = e;
  }
  bool ok() {
    note(cudaGetLastError());
    return err == cudaSuccess;
  }
  void *alloc(size_t b) {
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, b, s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return p;
  }
  void release(void *p) {
    if (p) note(cudaFreeAsync(p, s));
  }
  void fill(void *p, int v, size_t b) { note(cudaMemsetAsync(p, v, b, s)); }
  void copy(void *d, const void *src, size_t b) {
    if (b) note(cudaMemcpyAsync(d, src, b, cudaMemcpyDefault, s));
  }
  void fetch(void *h, const void *d, size_t b) {
    copy(h, d, b);
    note(cudaStreamSynchronize(s));
  }
  template <class F>
  void each(uint32_t n, const F &f) {
    if (!n) return;
    const uint32_t blocks = std::min<uint32_t>((n + EACH_T - 1) / EACH_T, (uint32_t)n_sms * 16);
    k_each<<<blocks, EACH_T, 0, s>>>(n, f);
    launches++;
  }
  void scan(const uint32_t *in, uint32_t *out, uint32_t n, unsigned long long *tot) {
    const uint32_t nb = std::max<uint32_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    if (nb > part_cap) {
      release(part);
      part_cap = std::max<uint32_t>(nb, 1024);
      part = (unsigned long long *)alloc((size_t)part_cap * 8);
      if (!part) {
        part_cap = 0;
        note(cudaErrorMemoryAllocation);
        return;
      }
    }
    k_scan_up<<<nb, SCAN_T, 0, s>>>(in, n, part);
    k_scan_mid<<<1, SCAN_T, 0, s>>>(part, nb, tot);
    k_scan_down<<<nb, SCAN_T, 0, s>>>(in, n, part, out);
    launches += 3;
  }
  void gen_heavy(const View &v, const unsigned long long *go) {
    if (v.heavy_min == 0xffffffffu) return;
    k_gen_heavy<<<(unsigned)n_sms * GEQ_GH_BLOCKS_PER_SM, GH_WARPS * 32, 0, s>>>(v, go);
    launches++;
  }
  // ---- device-counted launches (the level loop) ----
  uint32_t grid_for(uint32_t cap) const {
    return std::max<uint32_t>(
        1, std::min<uint32_t>((cap + EACH_T - 1) / EACH_T, (uint32_t)n_sms * GEQ_EACH_BLOCKS_PER_SM));
  }
  template <class F>
  void each_d(const unsigned long long *np, uint32_t cap, const unsigned long long *go, const F &f) {
    k_each_d<<<grid_for(cap), EACH_T, 0, s>>>(np, go, f);
    launches++;
  }
  uint32_t cnb() const { return (uint32_t)n_sms * 2; }
  // status space for scans of up to max_items values (called whenever the
  // level buffers are sized, before a level is recorded)
  void scan_capacity(uint64_t max_items) {
    const uint64_t tiles = (max_items + SCAN_TILE - 1) / SCAN_TILE + 1;
    if (lb_ctl && tiles <= lb_cap) return;
    const uint32_t cap = (uint32_t)std::max<uint64_t>(tiles * 2, 1024);
    release(lb_flag);
    release(lb_agg);
    release(lb_inc);
    lb_flag = (uint32_t *)alloc((size_t)3 * cap * 4);
    lb_agg = (unsigned long long *)alloc((size_t)3 * cap * 8);
    lb_inc = (unsigned long long *)alloc((size_t)3 * cap * 8);
    if (!lb_ctl) {
      lb_ctl = (LbCtl *)alloc(sizeof(LbCtl));
      if (lb_ctl) fill(lb_ctl, 0, sizeof(LbCtl));
    }
    if (!lb_flag || !lb_agg || !lb_inc || !lb_ctl) {
      lb_cap = 0;
      note(cudaErrorMemoryAllocation);
      return;
    }
    fill(lb_flag, 0, (size_t)3 * cap * 4);  // tag 0 with state 0: never ready
    lb_cap = cap;
  }
  template <int R>
  void lbscan(const ScanR &a, const unsigned long long *go) {
    if (!lb_cap) scan_capacity(0);
    k_lbscan<R><<<cnb(), SCAN_T, 0, s>>>(a, go, lb_ctl, lb_flag, lb_agg, lb_inc, lb_cap);
    launches++;
  }
  void scan_d(const uint32_t *in, uint32_t *out, const unsigned long long *np, unsigned long long *tot,
              const unsigned long long *go) {
    lbscan<1>(ScanR{{in, in, in}, {out, out, out}, {np, np, np}, {tot, tot, tot}}, go);
  }
  // two scans with their own counts in one launch
  void scan2_d(const uint32_t *i0, uint32_t *o0, const unsigned long long *np0, unsigned long long *t0,
               const uint32_t *i1, uint32_t *o1, const unsigned long long *np1, unsigned long long *t1,
               const unsigned long long *go) {
    lbscan<2>(ScanR{{i0, i1, i1}, {o0, o1, o1}, {np0, np1, np1}, {t0, t1, t1}}, go);
  }
  void scan3_d(const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, uint32_t *o0, uint32_t *o1, uint32_t *o2,
               const unsigned long long *np, unsigned long long *tot, const unsigned long long *go) {
    lbscan<3>(ScanR{{i0, i1, i2}, {o0, o1, o2}, {np, np, np}, {tot, tot + 1, tot + 2}}, go);
  }
  // ---- the level loop as a CUDA graph: a WHILE node whose body is one
  // recorded level followed by k_level_cond, so that one launch runs levels
  // until the loop stops (frontier empty, a stall) or the launch's limit ----
  cudaGraph_t graph = nullptr, body = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaGraphConditionalHandle cond = 0;
  uint32_t *d_loop = nullptr;  // [levels run in this launch, limit]
  uint32_t h_loop[2] = {0, 0};
  uint32_t graph_launches = 0, mark = 0;
  bool plain = false;  // levels as plain launches, one per host sync (profilers see every kernel)
  bool has_graph() const { return gexec != nullptr; }
  void begin_capture() {
    if (plain) return;  // the level that "capture" enqueues runs as it is
    if (!d_loop) d_loop = (uint32_t *)alloc(2 * sizeof(uint32_t));
    if (!d_loop) note(cudaErrorMemoryAllocation);
    mark = launches;
    note(cudaGraphCreate(&graph, 0));
    note(cudaGraphConditionalHandleCreate(&cond, graph, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    note(cudaGraphAddNode(&node, graph, nullptr, 0, &np));
    body = np.conditional.phGraph_out[0];
    note(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  }
  void end_capture(const unsigned long long *go) {
    if (plain) return;
    k_level_cond<<<1, 1, 0, s>>>(cond, go, d_loop);
    note(cudaStreamEndCapture(s, &body));
    graph_launches = launches - mark;
    launches = mark;
    if (err == cudaSuccess) note(cudaGraphInstantiate(&gexec, graph, 0));
  }
  // up to `limit` levels in one launch
  void run_graph(uint32_t limit) {
    if (!gexec) return;
    h_loop[0] = 0;
    h_loop[1] = limit;
    note(cudaMemcpyAsync(d_loop, h_loop, sizeof(h_loop), cudaMemcpyHostToDevice, s));
    note(cudaGraphLaunch(gexec, s));
  }
  // kernel launches of the levels that ran
  void note_levels(unsigned long long levels) { launches += (uint32_t)(levels * graph_launches); }
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);  // the WHILE node's body with it
    gexec = nullptr;
    graph = nullptr;
    body = nullptr;
  }
  ~DevBackend() {
    drop_graph();
    if (d_loop) cudaFreeAsync(d_loop, s);
    if (part) cudaFreeAsync(part, s);
    for (void *q : {(void *)lb_ctl, (void *)lb_flag, (void *)lb_agg, (void *)lb_inc})
      if (q) cudaFreeAsync(q, s);
  }
};

}  // namespace gb
}  // namespace geq

namespace geq {

// One device build: the LTSs of all jobs staged and uploaded as one id space,
// then the level loop.  The result arrays live until the Build object dies.
struct DeviceBuild {
  gb::DevBackend be;
  std::unique_ptr<gb::Builder<gb::DevBackend>> b;
  std::unique_ptr<rf::Refiner<gb::DevBackend>> rf;
  gb::Result r;
  char *din = nullptr;
  uint32_t *dstarts = nullptr;
  HostBuf stage;
  double upload_ms = 0, build_ms = 0, minimize_ms = 0;
  ~DeviceBuild() {
    b.reset();
    rf.reset();
    be.release(din);
    be.release(dstarts);
    cudaStreamSynchronize(be.s);
  }
};

static geq_status refine_status(int rc, gb::DevBackend &be) {
  if (!be.ok()) return fail(GEQ_ERR_CUDA, "device minimisation: %s", cudaGetErrorString(be.err));
  if (rc == 1) return fail(GEQ_ERR_OUT_OF_MEMORY, "device minimisation: out of device memory");
  if (rc == 3) return fail(GEQ_ERR_INTERNAL, "device minimisation: fingerprint collisions under four hash seeds");
  return GEQ_OK;
}

// Job j starts from Attack(p[t], {q[t]}) for t in start_off[j] .. start_off[j+1]-1
// (local process ids of L[j]), in that order.
// With `trivial` set, the LTSs are first minimised on the device (signature
// refinement, then the minimised systems written in place of the originals)
// and a one-start job whose two processes fall into one class gets no game
// (the bisimilar short cut of lib.rs:279-281): trivial[j] = 1.  With `stop`
// set, only the LTSs are staged (for the refinement entry point).
static geq_status device_build(Engine &eng, int device, uint32_t n_jobs, const Lts *const *L,
                               const uint32_t *start_off, const uint32_t *p, const uint32_t *q,
                               uint64_t max_positions, DeviceBuild &db, std::vector<uint8_t> *trivial = nullptr,
                               gb::Input *staged = nullptr) {
  using clk = std::chrono::steady_clock;
  std::vector<uint64_t> sb(n_jobs + 1, 0), tb(n_jobs + 1, 0);
  for (uint32_t j = 0; j < n_jobs; j++) {
    sb[j + 1] = sb[j] + L[j]->n;
    tb[j + 1] = tb[j] + L[j]->n_transitions();
  }
  const uint64_t NS = sb[n_jobs], MS = tb[n_jobs], T = start_off[n_jobs];
  if (NS >= (1ull << 31) || MS >= (1ull << 32) - 1 || T >= (1ull << 30))
    return fail(GEQ_ERR_INVALID_INPUT, "batch too large: %llu states, %llu transitions", (unsigned long long)NS,
                (unsigned long long)MS);
  const uint32_t max_pos = max_positions >= (1ull << 31) ? 0u : (uint32_t)max_positions;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return fail(GEQ_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  }
  // the builder allocates stream-ordered from the device's default pool; keep
  // freed blocks cached in this process instead of returning them at every
  // synchronisation
  static std::once_flag pool_once[64];
  if (device >= 0 && device < 64)
    std::call_once(pool_once[device], [device]() {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      cudaGetLastError();
    });
  gb::DevBackend &be = db.be;
  be.s = (cudaStream_t)eng.stream_handle();
  be.n_sms = eng.n_sms;
  // GEQ_TUNE_NO_GRAPH: levels as plain launches (ncu does not profile the
  // kernels of a graph with conditional nodes)
  be.plain = (eng.tuning.flags & GEQ_TUNE_NO_GRAPH) != 0;
  // stage the LTSs: soff | slab | stgt | sjob | p0 | q0
  const auto t0 = clk::now();
  const size_t o_soff = 0, o_slab = o_soff + (NS + 1) * 4, o_stgt = o_slab + MS * 4, o_sjob = o_stgt + MS * 4,
               o_p0 = o_sjob + NS * 4, o_q0 = o_p0 + (size_t)T * 4, o_jsb = o_q0 + (size_t)T * 4,
               bytes = o_jsb + ((size_t)n_jobs + 1) * 4;
  if (!db.stage.alloc(eng.host_pool(), bytes)) return fail(GEQ_ERR_OUT_OF_MEMORY, "staging %zu bytes", bytes);
  char *hs = (char *)db.stage.p;
  parallel_for(n_jobs, [&](uint32_t j) {
    const Lts &l = *L[j];
    uint32_t *soff = (uint32_t *)(hs + o_soff) + sb[j];
    int32_t *slab = (int32_t *)(hs + o_slab) + tb[j];
    uint32_t *stgt = (uint32_t *)(hs + o_stgt) + tb[j];
    uint32_t *sjob = (uint32_t *)(hs + o_sjob) + sb[j];
    for (uint32_t s = 0; s < l.n; s++) {
      soff[s] = (uint32_t)(tb[j] + l.off[s]);
      sjob[s] = j;
    }
    const uint64_t m = l.n_transitions();
    for (uint64_t k = 0; k < m; k++) {
      slab[k] = l.lab_[k];
      stgt[k] = (uint32_t)(sb[j] + l.tgt[k]);
    }
    for (uint32_t t = start_off[j]; t < start_off[j + 1]; t++) {
      ((uint32_t *)(hs + o_p0))[t] = (uint32_t)(sb[j] + p[t]);
      ((uint32_t *)(hs + o_q0))[t] = (uint32_t)(sb[j] + q[t]);
    }
    ((uint32_t *)(hs + o_jsb))[j] = (uint32_t)sb[j];
  });
  ((uint32_t *)(hs + o_soff))[NS] = (uint32_t)MS;
  ((uint32_t *)(hs + o_jsb))[n_jobs] = (uint32_t)NS;
  db.din = (char *)be.alloc(bytes);
  if (!db.din) return fail(GEQ_ERR_OUT_OF_MEMORY, "device input %zu bytes", bytes);
  be.copy(db.din, hs, bytes);
  gb::Input in;
  in.NS = (uint32_t)NS;
  in.MS = (uint32_t)MS;
  in.n_jobs = n_jobs;
  in.n_starts = (uint32_t)T;
  in.soff = (const uint32_t *)(db.din + o_soff);
  in.slab = (const int32_t *)(db.din + o_slab);
  in.stgt = (const uint32_t *)(db.din + o_stgt);
  in.sjob = (const uint32_t *)(db.din + o_sjob);
  in.p0 = (const uint32_t *)(db.din + o_p0);
  in.q0 = (const uint32_t *)(db.din + o_q0);
  in.jsb = (const uint32_t *)(db.din + o_jsb);
  in.max_pos = max_pos;
  // attack positions with at least this many q's take the warp path
  in.heavy_min = (eng.tuning.flags & GEQ_TUNE_BUILD_WARP_ALL) ? 1u : (uint32_t)GEQ_BUILD_HEAVY_MIN;
  if (staged) {
    *staged = in;
    db.upload_ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    return GEQ_OK;
  }
  gb::Input bin = in;
  if (trivial) {
    const auto tm = clk::now();
    db.rf.reset(new rf::Refiner<gb::DevBackend>(be));
    int rrc = db.rf->run(in);
    uint32_t *rp0 = nullptr, *rq0 = nullptr;
    if (rrc == 0) rrc = db.rf->reduce(in, bin, rp0, rq0);
    geq_status rst = refine_status(rrc, be);
    if (rst) return rst;
    // the bisimilar short cut, decided on the host from the mapped starts
    std::vector<uint32_t> mp((size_t)T), mq((size_t)T);
    be.copy(mp.data(), rp0, (size_t)T * 4);
    be.fetch(mq.data(), rq0, (size_t)T * 4);
    if (!be.ok()) return fail(GEQ_ERR_CUDA, "device minimisation: %s", cudaGetErrorString(be.err));
    trivial->assign(n_jobs, 0);
    std::vector<uint32_t> keep;
    keep.reserve(2 * (size_t)T);
    for (uint32_t j = 0; j < n_jobs; j++) {
      const uint32_t t0j = start_off[j], t1j = start_off[j + 1];
      if (t1j - t0j == 1 && mp[t0j] == mq[t0j]) {
        (*trivial)[j] = 1;
        continue;
      }
      for (uint32_t t = t0j; t < t1j; t++) keep.push_back(t);
    }
    const uint32_t K = (uint32_t)keep.size();
    std::vector<uint32_t> hst(2 * (size_t)K + 1);
    for (uint32_t k = 0; k < K; k++) {
      hst[k] = mp[keep[k]];
      hst[K + k] = mq[keep[k]];
    }
    db.dstarts = (uint32_t *)be.alloc(((size_t)2 * K + 1) * 4);
    if (!db.dstarts) return fail(GEQ_ERR_OUT_OF_MEMORY, "device start positions");
    be.copy(db.dstarts, hst.data(), ((size_t)2 * K + 1) * 4);
    bin.p0 = db.dstarts;
    bin.q0 = db.dstarts + K;
    bin.n_starts = K;
    be.fetch(hst.data(), db.dstarts, 4);  // the host copy above is done
    db.minimize_ms = std::chrono::duration<double, std::milli>(clk::now() - tm).count();
  }
  const auto t1 = clk::now();
  db.b.reset(new gb::Builder<gb::DevBackend>(be));
  // start from the capacities the previous build on this stream ended with
  static std::mutex hint_mu;
  static std::unordered_map<void *, gb::Builder<gb::DevBackend>::Caps> hints;
  {
    std::lock_guard<std::mutex> g(hint_mu);
    auto it = hints.find((void *)be.s);
    if (it != hints.end()) db.b->hint = it->second;
  }
  const int rc = db.b->run(bin, db.r);
  if (rc == 0) {
    std::lock_guard<std::mutex> g(hint_mu);
    hints[(void *)be.s] = db.b->used;
  }
  db.upload_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  db.build_ms = std::chrono::duration<double, std::milli>(clk::now() - t1).count();
  if (!be.ok()) return fail(GEQ_ERR_CUDA, "device game build: %s", cudaGetErrorString(be.err));
  if (rc == 1)
    return fail(GEQ_ERR_OUT_OF_MEMORY,
                "device game build: out of device memory (a request of %llu could not be met; %llu positions, "
                "%llu edges after %llu levels)",
                (unsigned long long)db.b->short_, (unsigned long long)db.b->reached_positions(),
                (unsigned long long)db.b->reached_edges(), (unsigned long long)db.b->reached_levels());
  if (rc == 2) return fail(GEQ_ERR_INVALID_INPUT, "device game build: game beyond 2^31 positions or 2^32 edges");
  if (rc == 3) return fail(GEQ_ERR_INTERNAL, "device game build: fingerprint collisions under four hash seeds");
  return GEQ_OK;
}

// GameBuild::compare of every job on the device, handed to the solver as an
// upload (the graphs never leave the device).  Jobs whose game exceeds
// max_positions (0 = no bound) fail the call with GEQ_ERR_OUT_OF_MEMORY --
// unless `over` is given: then over[j] marks them and they are uploaded as
// the part the builder numbered before it stopped expanding them (a well
// formed game whose unexpanded positions have no successors), whose lists
// the caller must discard.
geq_status build_and_upload(Engine &eng, int device, uint32_t n_jobs, const Lts *const *L, const uint32_t *start_off,
                            const uint32_t *p, const uint32_t *q, uint64_t max_positions, GamesPtr &out,
                            double *build_ms, std::vector<uint8_t> *trivial, std::vector<uint8_t> *over) {
  DeviceBuild db;
  geq_status st = device_build(eng, device, n_jobs, L, start_off, p, q, max_positions, db, trivial);
  if (st) return st;
  std::vector<uint32_t> jcount(n_jobs), jm(n_jobs), jover(n_jobs);
  db.be.copy(jcount.data(), db.r.jcount, (size_t)n_jobs * 4);
  db.be.copy(jover.data(), db.r.jover, (size_t)n_jobs * 4);
  db.be.fetch(jm.data(), db.r.jm, (size_t)n_jobs * 4);
  if (!db.be.ok()) return fail(GEQ_ERR_CUDA, "device game build: %s", cudaGetErrorString(db.be.err));
  if (over) over->assign(n_jobs, 0);
  for (uint32_t j = 0; j < n_jobs; j++) {
    if (!jover[j]) continue;
    if (!over)
      return fail(GEQ_ERR_OUT_OF_MEMORY, "job %u: game exceeds %llu positions", j, (unsigned long long)max_positions);
    (*over)[j] = 1;
  }
  if (build_ms) *build_ms = db.upload_ms + db.minimize_ms + db.build_ms;
  // jobs without positions (no start pairs, or the bisimilar short cut) add
  // nothing to the arrays: the games are the other jobs, in order
  std::vector<uint32_t> gn, gm;
  for (uint32_t j = 0; j < n_jobs; j++)
    if (jcount[j]) {
      gn.push_back(jcount[j]);
      gm.push_back(jm[j]);
    }
  if (gn.empty()) {
    out.reset();
    return GEQ_OK;
  }
  BuiltGames bg;
  bg.n_games = (uint32_t)gn.size();
  bg.n_nodes = gn.data();
  bg.n_edges = gm.data();
  bg.N = db.r.N;
  bg.M = db.r.M;
  bg.row_rel = db.r.rrel;
  bg.col = db.r.col;
  bg.wt = db.r.wt;
  bg.att = db.r.att;
  return eng.upload_built(bg, out);  // copies on the same stream before db's buffers are freed
}

}  // namespace geq

using namespace geq;

struct geq_game_batch {
  uint32_t n_jobs = 0;
  std::vector<uint32_t> node_base, edge_base, n_nodes, n_edges, n_starts;
  std::vector<uint8_t> over;
  HostBuf row, col, wt, att;
  uint64_t N = 0, M = 0;
  uint32_t levels = 0, launches = 0, attempts = 0;
  double upload_ms = 0, build_ms = 0, download_ms = 0;
};

static geq_status build_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts, const uint32_t *start_off,
                              const uint32_t *p, const uint32_t *q, uint64_t max_positions, geq_game_batch **out);

extern "C" geq_status geq_game_build_compare_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts,
                                                   const uint32_t *p, const uint32_t *q, uint64_t max_positions,
                                                   geq_game_batch **out) {
  if (!out || !lts || !p || !q) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  std::vector<uint32_t> start_off(n_jobs + 1);
  for (uint32_t j = 0; j <= n_jobs; j++) start_off[j] = j;
  return build_batch(ctx, n_jobs, lts, start_off.data(), p, q, max_positions, out);
}

extern "C" geq_status geq_game_build_starts_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts,
                                                  const uint32_t *start_off, const uint32_t *p, const uint32_t *q,
                                                  uint64_t max_positions, geq_game_batch **out) {
  if (!out || !lts || !start_off) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (n_jobs && start_off[0] != 0) return fail(GEQ_ERR_INVALID_INPUT, "start_off[0] must be 0");
  for (uint32_t j = 0; j < n_jobs; j++)
    if (start_off[j + 1] < start_off[j]) return fail(GEQ_ERR_INVALID_INPUT, "start_off must not decrease");
  if (n_jobs && start_off[n_jobs] && (!p || !q)) return fail(GEQ_ERR_INVALID_INPUT, "NULL start arrays");
  return build_batch(ctx, n_jobs, lts, start_off, p, q, max_positions, out);
}

static geq_status build_batch(geq_context *ctx, uint32_t n_jobs, const geq_lts *const *lts, const uint32_t *start_off,
                              const uint32_t *p, const uint32_t *q, uint64_t max_positions, geq_game_batch **out) {
  using clk = std::chrono::steady_clock;
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  *out = nullptr;
  if (n_jobs == 0) return fail(GEQ_ERR_INVALID_INPUT, "no jobs");
  std::vector<const Lts *> L(n_jobs);
  for (uint32_t j = 0; j < n_jobs; j++) {
    if (!lts[j]) return fail(GEQ_ERR_INVALID_INPUT, "job %u: LTS is NULL", j);
    L[j] = &lts[j]->l;
    for (uint32_t t = start_off[j]; t < start_off[j + 1]; t++)
      if (p[t] >= L[j]->n || q[t] >= L[j]->n) return fail(GEQ_ERR_INVALID_INPUT, "job %u: process out of range", j);
  }
  Engine &eng = *ctx->engine;
  std::unique_ptr<geq_game_batch> res(new geq_game_batch());
  res->n_jobs = n_jobs;
  res->n_starts.resize(n_jobs);
  for (uint32_t j = 0; j < n_jobs; j++) res->n_starts[j] = start_off[j + 1] - start_off[j];
  DeviceBuild db;
  geq_status st = device_build(eng, ctx->device, n_jobs, L.data(), start_off, p, q, max_positions, db);
  if (st) return st;
  // per-job CSR back to the host
  const auto t2 = clk::now();
  const gb::Result &r = db.r;
  gb::DevBackend &be = db.be;
  const uint32_t J = n_jobs;
  std::vector<uint32_t> jcount(J), jover(J), jbase(J);
  auto hp = eng.host_pool();
  if (!res->row.alloc(hp, ((size_t)r.N + J) * 4) || !res->col.alloc(hp, (size_t)r.M * 4) ||
      !res->wt.alloc(hp, (size_t)r.M * 4) || !res->att.alloc(hp, (size_t)r.N))
    return fail(GEQ_ERR_OUT_OF_MEMORY, "host result buffers");
  be.copy(res->row.p, r.row, ((size_t)r.N + J) * 4);
  be.copy(res->col.p, r.col, (size_t)r.M * 4);
  be.copy(res->wt.p, r.wt, (size_t)r.M * 4);
  be.copy(res->att.p, r.att, (size_t)r.N);
  be.copy(jcount.data(), r.jcount, (size_t)J * 4);
  be.copy(jover.data(), r.jover, (size_t)J * 4);
  be.fetch(jbase.data(), r.jbase, (size_t)J * 4);
  if (!be.ok()) return fail(GEQ_ERR_CUDA, "device game build: %s", cudaGetErrorString(be.err));
  res->node_base = jbase;
  res->n_nodes = jcount;
  res->edge_base.resize(J);
  res->n_edges.resize(J);
  res->over.resize(J);
  const uint32_t *row = (const uint32_t *)res->row.p;
  uint64_t eb = 0;
  for (uint32_t j = 0; j < J; j++) {
    res->edge_base[j] = (uint32_t)eb;
    res->n_edges[j] = row[(size_t)jbase[j] + j + jcount[j]];
    res->over[j] = jover[j] != 0;
    eb += res->n_edges[j];
  }
  res->N = r.N;
  res->M = r.M;
  res->levels = r.levels;
  res->attempts = r.attempts;
  res->launches = be.launches;
  res->upload_ms = db.upload_ms;
  res->build_ms = db.build_ms;
  res->download_ms = std::chrono::duration<double, std::milli>(clk::now() - t2).count();
  *out = res.release();
  return GEQ_OK;
}

extern "C" geq_status geq_lts_signature_refinement_batch(geq_context *ctx, uint32_t n_lts, const geq_lts *const *lts,
                                                         uint64_t *partitions, uint64_t *n_classes) {
  if (!ctx || !ctx->engine) return fail(GEQ_ERR_INVALID_INPUT, "context is NULL");
  if (!lts || !partitions || !n_classes) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (n_lts == 0) return fail(GEQ_ERR_INVALID_INPUT, "no systems");
  std::vector<const Lts *> L(n_lts);
  for (uint32_t j = 0; j < n_lts; j++) {
    if (!lts[j]) return fail(GEQ_ERR_INVALID_INPUT, "system %u is NULL", j);
    L[j] = &lts[j]->l;
  }
  std::vector<uint32_t> start_off(n_lts + 1, 0);
  DeviceBuild db;
  gb::Input in;
  geq_status st = device_build(*ctx->engine, ctx->device, n_lts, L.data(), start_off.data(), nullptr, nullptr, 0, db,
                               nullptr, &in);
  if (st) return st;
  db.rf.reset(new rf::Refiner<gb::DevBackend>(db.be));
  if ((st = refine_status(db.rf->run(in), db.be))) return st;
  std::vector<uint32_t> part(in.NS), cnt(n_lts);
  db.be.copy(part.data(), db.rf->partition(), (size_t)in.NS * 4);
  db.be.fetch(cnt.data(), db.rf->counts(), (size_t)n_lts * 4);
  if (!db.be.ok()) return fail(GEQ_ERR_CUDA, "device minimisation: %s", cudaGetErrorString(db.be.err));
  for (uint32_t i = 0; i < in.NS; i++) partitions[i] = part[i];
  for (uint32_t j = 0; j < n_lts; j++) n_classes[j] = cnt[j];
  return GEQ_OK;
}

extern "C" uint32_t geq_game_batch_n_jobs(const geq_game_batch *b) { return b ? b->n_jobs : 0; }

extern "C" geq_status geq_game_batch_graph(const geq_game_batch *b, uint32_t job, geq_game_graph *out) {
  if (!b || !out) return fail(GEQ_ERR_INVALID_INPUT, "NULL argument");
  if (job >= b->n_jobs) return fail(GEQ_ERR_INVALID_INPUT, "job %u out of range", job);
  if (b->over[job]) return fail(GEQ_ERR_OUT_OF_MEMORY, "job %u: game exceeds the position bound", job);
  out->conf = geq_energy_conf{6, 3};
  out->n_vertices = b->n_nodes[job];
  out->row_offsets = (const uint32_t *)b->row.p + (size_t)b->node_base[job] + job;
  out->column_indices = (const uint32_t *)b->col.p + b->edge_base[job];
  out->weights = (const uint32_t *)b->wt.p + b->edge_base[job];
  out->attacker_pos = (const uint8_t *)b->att.p + b->node_base[job];
  return GEQ_OK;
}

extern "C" void geq_game_batch_stats(const geq_game_batch *b, geq_game_batch_info *out) {
  if (!b || !out) return;
  out->positions = b->N;
  out->edges = b->M;
  out->levels = b->levels;
  out->kernel_launches = b->launches;
  out->attempts = b->attempts;
  out->upload_ms = b->upload_ms;
  out->build_ms = b->build_ms;
  out->download_ms = b->download_ms;
}

extern "C" uint32_t geq_game_batch_n_starting_points(const geq_game_batch *b, uint32_t job) {
  return b && job < b->n_jobs ? b->n_starts[job] : 0;
}

extern "C" void geq_game_batch_free(geq_game_batch *b) { delete b; }
