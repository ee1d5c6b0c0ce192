// gbuild.cuh - GameBuild::compare on the device (src/gamebuild.rs:139-266,
// successor rules of src/gamebuild/gamepos.rs:17-198), for many jobs at once.
//
// The reference numbers positions in the order a FIFO queue discovers them
// (gamebuild.rs:229-265).  That order is reproduced level by level: the
// positions of one breadth-first level are expanded together, their
// successors are written into slots laid out in (job, parent id, successor
// index) order, and a successor that is new gets the next position id of its
// job in the order of its first slot.  Since every level's positions are
// already in (job, local id) order, the ids equal the queue's.
//
// Process sets (the Q and Q* of the positions) are interned in a device hash
// table keyed by a 64-bit fingerprint of the sorted contents; positions in a
// second table keyed by a fingerprint of (kind, p, a, b).  Equal fingerprints
// are merged and then verified element by element against the stored
// representative: a fingerprint collision sets an error flag and the build
// restarts with another hash seed, so the result never depends on the hash.
//
// Everything per item is a functor over raw pointers; `Backend::each(n, f)`
// runs f(i) for i < n (a grid-stride kernel on the device).
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#define __align__(n) alignas(n)
#endif

namespace geq {
namespace gb {

constexpr uint32_t K_ATTACK = 0, K_CLAUSE = 1, K_DEFEND = 2, K_NONE = 3;
constexpr uint32_t CAND = 0x80000000u;  // a set reference that is a candidate of this level
constexpr uint32_t UNSET = 0xffffffffu;
enum : uint32_t { ERR_COLLISION = 1u, ERR_RANGE = 2u };

// Packed STANDARD updates of the game (gamepos.rs:21-22, :145-146, :183-184).
constexpr uint32_t W_OBS = 1u;                           // [-1]
constexpr uint32_t W_CHAL = 1u << 4;                     // [0, -1]
constexpr uint32_t W_REV = 4u;                           // [Min(3)]
constexpr uint32_t W_ANS = 4u << 12;                     // [0, 0, 0, Min(3)]
constexpr uint32_t W_CL1 = 5u;                           // [Min(4)]
constexpr uint32_t W_CL2 = 6u | (1u << 20);              // [Min(5), 0, 0, 0, 0, -1]

struct __align__(16) Key {
  uint32_t kind, p, a, b;
};
__host__ __device__ __forceinline__ bool key_eq(const Key &x, const Key &y) {
  return x.kind == y.kind && x.p == y.p && x.a == y.a && x.b == y.b;
}

// ---- atomics (sequential stand-ins when compiled for the host) -------------
__host__ __device__ __forceinline__ uint32_t at_add(uint32_t *a, uint32_t v) {
#ifdef __CUDA_ARCH__
  return atomicAdd(a, v);
#else
  uint32_t o = *a;
  *a = o + v;
  return o;
#endif
}
__host__ __device__ __forceinline__ void at_min(uint32_t *a, uint32_t v) {
#ifdef __CUDA_ARCH__
  atomicMin(a, v);
#else
  if (v < *a) *a = v;
#endif
}
__host__ __device__ __forceinline__ void at_or(uint32_t *a, uint32_t v) {
#ifdef __CUDA_ARCH__
  atomicOr(a, v);
#else
  *a |= v;
#endif
}
__host__ __device__ __forceinline__ unsigned long long at_cas(unsigned long long *a, unsigned long long cmp,
                                                              unsigned long long v) {
#ifdef __CUDA_ARCH__
  return atomicCAS(a, cmp, v);
#else
  unsigned long long o = *a;
  if (o == cmp) *a = v;
  return o;
#endif
}

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long h) {
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  h *= 0xc4ceb9fe1a85ec53ull;
  h ^= h >> 33;
  return h;
}
__host__ __device__ __forceinline__ unsigned long long set_hash(const uint32_t *v, uint32_t n,
                                                                unsigned long long seed) {
  unsigned long long h = mix64(seed ^ (0x51ed270b27a3f1d7ull + n));
  for (uint32_t i = 0; i < n; i++) h = mix64(h ^ (v[i] + 0x9e3779b97f4a7c15ull));
  return h ? h : 1ull;
}
__host__ __device__ __forceinline__ unsigned long long key_hash(const Key &k, unsigned long long seed) {
  unsigned long long h = mix64(seed ^ (((unsigned long long)k.kind << 32) | k.p));
  h = mix64(h ^ (((unsigned long long)k.a << 32) | k.b));
  return h ? h : 1ull;
}

// Counts of the level loop, kept on the device (Totals::t) so that levels
// run without the host: kernels take their item counts from here.
enum : int {
  T_NEW = 0,     // new positions of the level
  T_S = 1,       // successor slots (upper bound), set words, candidate sets: three in a row
  T_E = 2,
  T_C = 3,
  T_EDGE = 4,    // edges of the level
  T_N = 5,       // positions of all jobs (final)
  T_F0 = 6,      // first frontier position
  T_F = 7,       // frontier size
  T_NN = 8,      // positions so far
  T_NE = 9,      // edges so far
  T_GO = 10,     // 1 while levels may run
  T_STALL = 11,  // a level stopped for a buffer to grow
  T_DONE = 12,   // the frontier ran empty
  T_LEVELS = 13, // levels completed
  T_COUNT = 16
};

// Control block on the device.
struct Ctl {
  uint32_t err;
  uint32_t n_sets;     // interned sets
  uint32_t sdata_top;  // words of set contents
  uint32_t n_heavy;    // this level's attack positions for the warp path
};

// Every array of a build.  Rebuilt by the host whenever a buffer grows.
struct View {
  // LTS of all jobs in one id space (state ids global, rows sorted by label)
  const uint32_t *soff;  // NS + 1, global transition offsets
  const int32_t *slab;
  const uint32_t *stgt;
  const uint32_t *sjob;  // job of each state
  const uint32_t *jsb;   // n_jobs + 1: first state of each job
  // interned sets
  uint32_t *sdata, *sstart, *slen;
  uint32_t sdata_cap, sets_cap;
  unsigned long long *stab;  // fingerprints, 0 = free
  uint32_t *sval, *sclaim;   // set id or UNSET; smallest claiming candidate
  uint32_t smask;
  // positions, in discovery order (level by level)
  Key *nkey;
  uint32_t *nlocal, *nrow, *neoff;
  uint32_t nodes_cap;
  unsigned long long *ntab;
  uint32_t *nval, *nclaim;
  uint32_t nmask;
  // per job
  uint32_t *jcount, *jfirst, *jover;
  // level scratch: frontier positions t[T_F0] .. t[T_F0]+t[T_F]-1
  unsigned long long *t;            // Totals::t on the device
  uint32_t capF, capS, capE, capC;  // scratch capacities (the level gate checks them)
  uint32_t scap, ncap;              // hash table sizes
  uint32_t *ub_s, *ub_e, *ub_c;     // upper bounds: successor slots, set words, candidate sets
  uint32_t *off_s, *off_e, *off_c;  // their exclusive scans
  uint32_t *fcnt, *feoff;           // exact successor counts, their scan
  uint32_t *hq;                     // frontier indices taken by the warp path
  uint32_t heavy_min;               // |Q| from which an attack position takes the warp path
  Key *succ;
  uint32_t *swt, *sslot, *sres, *snew, *srank;
  uint32_t *celem, *cstart, *clen, *cslot, *cid;
  // edges in discovery order of their source
  uint32_t *ecol, *ewt;
  uint32_t edges_cap;
  // start positions: Attack(p0[t], {q0[t]}), job-major
  const uint32_t *p0, *q0;
  uint32_t n_jobs;
  uint32_t max_pos;  // 0 = unbounded
  Ctl *ctl;
  unsigned long long seed;
};

__host__ __device__ __forceinline__ uint32_t deg(const View &v, uint32_t s) { return v.soff[s + 1] - v.soff[s]; }
__host__ __device__ __forceinline__ uint32_t F0(const View &v) { return (uint32_t)v.t[T_F0]; }
__host__ __device__ __forceinline__ uint32_t NN(const View &v) { return (uint32_t)v.t[T_NN]; }
__host__ __device__ __forceinline__ uint32_t NE(const View &v) { return (uint32_t)v.t[T_NE]; }

// TransitionSystem::compare_enabled (gamebuild.rs:23-98): (enabled(p) ⊆
// enabled(q), enabled(p) ⊇ enabled(q)), rows being label-sorted.
__host__ __device__ inline void compare_enabled(const View &v, uint32_t p, uint32_t q, bool &subset, bool &superset) {
  subset = superset = true;
  if (p == q) return;
  uint32_t pp = v.soff[p], pm = v.soff[p + 1], qp = v.soff[q], qm = v.soff[q + 1];
  for (;;) {
    if (!(subset || superset)) break;
    if (pp == pm && qp == qm) break;
    if (pp == pm) { subset = false; break; }
    if (qp == qm) { superset = false; break; }
    const int32_t pa = v.slab[pp], qa = v.slab[qp];
    bool ap = false, aq = false;
    if (pa == qa) { ap = aq = true; }
    else if (pa < qa) { superset = false; ap = true; }
    else { subset = false; aq = true; }
    if (ap) { pp++; while (pp < pm && v.slab[pp] == pa) pp++; }
    if (aq) { qp++; while (qp < qm && v.slab[qp] == qa) qp++; }
  }
}

__host__ __device__ __forceinline__ uint32_t label_lower(const View &v, uint32_t q, int32_t a) {
  uint32_t lo = v.soff[q], hi = v.soff[q + 1];
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (v.slab[mid] < a) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// In-place sort of a short u32 array (insertion sort up to 32, heapsort above).
__host__ __device__ inline void sort_u32(uint32_t *a, uint32_t n) {
  if (n <= 32) {
    for (uint32_t i = 1; i < n; i++) {
      const uint32_t x = a[i];
      uint32_t j = i;
      while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; j--; }
      a[j] = x;
    }
    return;
  }
  auto sift = [&](uint32_t r, uint32_t end) {
    for (;;) {
      uint32_t c = 2 * r + 1;
      if (c >= end) return;
      if (c + 1 < end && a[c + 1] > a[c]) c++;
      if (a[r] >= a[c]) return;
      const uint32_t t = a[r]; a[r] = a[c]; a[c] = t;
      r = c;
    }
  };
  for (uint32_t r = n / 2; r-- > 0;) sift(r, n);
  for (uint32_t end = n - 1; end > 0; end--) {
    const uint32_t t = a[0]; a[0] = a[end]; a[end] = t;
    sift(0, end);
  }
}
__host__ __device__ __forceinline__ bool bsearch_u32(const uint32_t *a, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < n && a[lo] == x;
}

// ---- level 0: the start positions --------------------------------------------
struct StartF {
  View v;
  __host__ __device__ void operator()(uint32_t j) const {
    v.succ[j] = Key{K_ATTACK, v.p0[j], CAND | j, 0};
    v.swt[j] = 0;
    v.celem[j] = v.q0[j];
    v.cstart[j] = j;
    v.clen[j] = 1;
  }
};

// ---- per frontier position: upper bounds of its output ----------------------
struct CountF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    const Key x = v.nkey[F0(v) + i];
    uint32_t s = 0, e = 0, c = 0;
    if (!v.jover[v.sjob[x.p]]) {
      if (x.kind == K_ATTACK) {
        const uint32_t nq = v.slen[x.a];
        if (nq == 0) {
          s = 1;
        } else {
          const uint32_t d = deg(v, x.p);
          s = d + 4;
          c = d + 6;
          const uint32_t *Q = v.sdata + v.sstart[x.a];
          for (uint32_t k = 0; k < nq; k++) e += deg(v, Q[k]);
          e += 4 * nq;  // unions, three split pairs, one word of flags per q (warp path)
          if (nq >= v.heavy_min) v.hq[at_add(&v.ctl->n_heavy, 1u)] = i;
        }
      } else if (x.kind == K_CLAUSE) {
        s = 2; e = 2; c = 2;
      } else {
        s = v.slen[x.a] + (v.slen[x.b] != 0 ? 1u : 0u);
      }
    }
    v.ub_s[i] = s;
    v.ub_e[i] = e;
    v.ub_c[i] = c;
  }
};

// ---- per frontier position: its successors (Position::successors) ----------
__host__ __device__ inline void gen_one(const View &v, uint32_t i) {
  {
    const Key x = v.nkey[F0(v) + i];
    const uint32_t s0 = v.off_s[i], ns = v.ub_s[i];
    const uint32_t c0 = v.off_c[i], nc = v.ub_c[i];
    const uint32_t e0 = v.off_e[i];
    uint32_t cnt = 0, cc = 0, ecur = 0;
    auto push = [&](const Key &k, uint32_t w) {
      v.succ[s0 + cnt] = k;
      v.swt[s0 + cnt] = w;
      cnt++;
    };
    // a candidate set whose words are at celem[e0 + start .. + len)
    auto cand = [&](uint32_t start, uint32_t len) -> uint32_t {
      v.cstart[c0 + cc] = e0 + start;
      v.clen[c0 + cc] = len;
      return CAND | (c0 + cc++);
    };
    if (ns != 0) {
      if (x.kind == K_ATTACK) {  // AttackPosition::successors (gamepos.rs:17-106)
        const uint32_t nq = v.slen[x.a];
        if (nq == 0) {
          push(Key{K_DEFEND, x.p, 0, 0}, W_CHAL);
        } else {
          const uint32_t *Q = v.sdata + v.sstart[x.a];
          uint32_t *el = v.celem + e0;
          // observation moves: Q' = union of the a-successors of Q, per label run
          uint32_t k = v.soff[x.p];
          const uint32_t ke = v.soff[x.p + 1];
          while (k < ke) {
            const int32_t a = v.slab[k];
            uint32_t run_end = k;
            while (run_end < ke && v.slab[run_end] == a) run_end++;
            uint32_t len = 0;
            for (uint32_t t = 0; t < nq; t++) {
              const uint32_t q = Q[t];
              for (uint32_t u = label_lower(v, q, a); u < v.soff[q + 1] && v.slab[u] == a; u++)
                el[ecur + len++] = v.stgt[u];
            }
            sort_u32(el + ecur, len);
            uint32_t w = 0;
            for (uint32_t r = 0; r < len; r++)
              if (w == 0 || el[ecur + r] != el[ecur + w - 1]) el[ecur + w++] = el[ecur + r];
            const uint32_t qref = cand(ecur, w);
            for (; k < run_end; k++) {
              const uint32_t p2 = v.stgt[k];
              if (!bsearch_u32(el + ecur, w, p2)) push(Key{K_ATTACK, p2, qref, 0}, W_OBS);
            }
            ecur += w;
          }
          // conjunction challenges: Defend(p, Q, {}) and the enabledness splits
          push(Key{K_DEFEND, x.p, x.a, 0}, W_CHAL);
          // enabledness splits (gamepos.rs:60-104): pair pr (0 subset,
          // 1 superset, 2 equal) gets nq words; the q's whose enabledness
          // fails the test grow up from the start, the others down from the
          // end, and the latter are reversed into ascending order afterwards
          uint32_t *b0 = el + ecur;
          uint32_t sn[6] = {0, 0, 0, 0, 0, 0};
          for (uint32_t t = 0; t < nq; t++) {
            bool sub, sup;
            compare_enabled(v, x.p, Q[t], sub, sup);
            const bool fl[3] = {sub, sup, sub && sup};
            for (uint32_t pr = 0; pr < 3; pr++) {
              uint32_t *b = b0 + pr * nq;
              if (fl[pr]) b[nq - 1 - sn[2 * pr + 1]++] = Q[t];
              else b[sn[2 * pr]++] = Q[t];
            }
          }
          for (uint32_t pr = 0; pr < 3; pr++) {
            uint32_t *b = b0 + pr * nq;
            const uint32_t n1 = sn[2 * pr + 1];
            for (uint32_t l = 0; 2 * l + 1 < n1; l++) {
              const uint32_t t = b[nq - n1 + l];
              b[nq - n1 + l] = b[nq - 1 - l];
              b[nq - 1 - l] = t;
            }
          }
          uint32_t pushed[3];
          uint32_t np = 0;
          for (uint32_t pr = 0; pr < 3; pr++) {
            const uint32_t nqs = sn[2 * pr], nqx = sn[2 * pr + 1];
            if (nqs == 0 || nqx == 0) continue;
            const uint32_t *qs = b0 + pr * nq, *qx = b0 + pr * nq + (nq - nqx);
            bool dup = false;  // push_unique: an equal split was pushed already
            for (uint32_t o = 0; o < np && !dup; o++) {
              const uint32_t po = pushed[o];
              if (sn[2 * po] != nqs || sn[2 * po + 1] != nqx) continue;
              const uint32_t *os = b0 + po * nq, *ox = b0 + po * nq + (nq - nqx);
              bool same = true;
              for (uint32_t t = 0; t < nqs && same; t++) same = os[t] == qs[t];
              for (uint32_t t = 0; t < nqx && same; t++) same = ox[t] == qx[t];
              dup = same;
            }
            if (dup) continue;
            const uint32_t ra = cand(ecur + pr * nq, nqs);
            const uint32_t rb = cand(ecur + pr * nq + (nq - nqx), nqx);
            push(Key{K_DEFEND, x.p, ra, rb}, W_CHAL);
            pushed[np++] = pr;
          }
        }
      } else if (x.kind == K_CLAUSE) {  // SingletonPosition::successors (gamepos.rs:139-158)
        v.celem[e0] = x.a;
        v.celem[e0 + 1] = x.p;
        const uint32_t r1 = cand(0, 1), r2 = cand(1, 1);
        push(Key{K_ATTACK, x.p, r1, 0}, W_CL1);
        push(Key{K_ATTACK, x.a, r2, 0}, W_CL2);
      } else {  // DefendPosition::successors (gamepos.rs:179-198)
        const uint32_t nq = v.slen[x.a];
        const uint32_t *Q = v.sdata + v.sstart[x.a];
        for (uint32_t t = 0; t < nq; t++) push(Key{K_CLAUSE, x.p, Q[t], 0}, W_ANS);
        if (v.slen[x.b] != 0) push(Key{K_ATTACK, x.p, x.b, 0}, W_REV);
      }
    }
    for (uint32_t t = cnt; t < ns; t++) v.succ[s0 + t] = Key{K_NONE, 0, 0, 0};
    for (uint32_t t = cc; t < nc; t++) v.clen[c0 + t] = UNSET;
    v.fcnt[i] = cnt;
  }
}
// whether frontier position i was queued for the warp path by CountF
__host__ __device__ __forceinline__ bool is_heavy(const View &v, uint32_t i) {
  const Key x = v.nkey[F0(v) + i];
  if (x.kind != K_ATTACK || v.jover[v.sjob[x.p]]) return false;
  const uint32_t nq = v.slen[x.a];
  return nq != 0 && nq >= v.heavy_min;
}
struct GenF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    if (!is_heavy(v, i)) gen_one(v, i);
  }
};

// ---- set interning -------------------------------------------------------------
struct SetProbeF {
  View v;
  __host__ __device__ void operator()(uint32_t c) const {
    const uint32_t len = v.clen[c];
    if (len == UNSET) return;
    const unsigned long long h = set_hash(v.celem + v.cstart[c], len, v.seed);
    uint32_t s = (uint32_t)(h >> 20) & v.smask;
    for (uint32_t probes = 0;; probes++) {
      if (probes > v.smask) {  // cannot happen below half load; never spin
        at_or(&v.ctl->err, ERR_RANGE);
        v.clen[c] = UNSET;
        return;
      }
      const unsigned long long k = v.stab[s];
      if (k == h) break;
      if (k == 0) {
        const unsigned long long o = at_cas(&v.stab[s], 0ull, h);
        if (o == 0ull || o == h) break;
      }
      s = (s + 1) & v.smask;
    }
    v.cslot[c] = s;
    if (v.sval[s] == UNSET) at_min(&v.sclaim[s], c);
  }
};
// the first candidate of each new set stores it
struct SetNewF {
  View v;
  __host__ __device__ void operator()(uint32_t c) const {
    const uint32_t len = v.clen[c];
    if (len == UNSET) return;
    const uint32_t s = v.cslot[c];
    if (v.sval[s] != UNSET || v.sclaim[s] != c) return;
    const uint32_t id = at_add(&v.ctl->n_sets, 1u);
    const uint32_t off = at_add(&v.ctl->sdata_top, len);
    if (id >= v.sets_cap || (unsigned long long)off + len > v.sdata_cap) {
      at_or(&v.ctl->err, ERR_RANGE);
      return;
    }
    const uint32_t *src = v.celem + v.cstart[c];
    for (uint32_t t = 0; t < len; t++) v.sdata[off + t] = src[t];
    v.sstart[id] = off;
    v.slen[id] = len;
    v.sval[s] = id;
  }
};
// every candidate: its set id, verified against the stored contents
struct SetFillF {
  View v;
  __host__ __device__ void operator()(uint32_t c) const {
    const uint32_t len = v.clen[c];
    if (len == UNSET) return;
    const uint32_t id = v.sval[v.cslot[c]];
    bool ok = id < v.sets_cap && v.slen[id] == len;
    if (ok) {
      const uint32_t *a = v.celem + v.cstart[c], *b = v.sdata + v.sstart[id];
      for (uint32_t t = 0; t < len && ok; t++) ok = a[t] == b[t];
    }
    if (!ok) at_or(&v.ctl->err, ERR_COLLISION);
    v.cid[c] = ok ? id : 0u;
  }
};

// ---- position interning --------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t node_probe(const View &v, unsigned long long h) {
  uint32_t s = (uint32_t)(h >> 20) & v.nmask;
  for (uint32_t probes = 0;; probes++) {
    if (probes > v.nmask) {  // cannot happen below half load; never spin
      at_or(&v.ctl->err, ERR_RANGE);
      return UNSET;
    }
    const unsigned long long k = v.ntab[s];
    if (k == h) return s;
    if (k == 0) {
      const unsigned long long o = at_cas(&v.ntab[s], 0ull, h);
      if (o == 0ull || o == h) return s;
    }
    s = (s + 1) & v.nmask;
  }
}
struct SuccProbeF {
  View v;
  __host__ __device__ void operator()(uint32_t s) const {
    Key k = v.succ[s];
    if (k.kind == K_NONE) return;
    if (k.kind != K_CLAUSE) {
      if (k.a & CAND) k.a = v.cid[k.a & ~CAND];
      if (k.b & CAND) k.b = v.cid[k.b & ~CAND];
      v.succ[s] = k;
    }
    const uint32_t slot = node_probe(v, key_hash(k, v.seed));
    v.sslot[s] = slot;
    if (slot == UNSET) {
      v.succ[s].kind = K_NONE;
      return;
    }
    if (v.nval[slot] == UNSET) at_min(&v.nclaim[slot], s);
  }
};
struct SuccFlagF {
  View v;
  __host__ __device__ void operator()(uint32_t s) const {
    uint32_t f = 0;
    if (v.succ[s].kind != K_NONE) {
      const uint32_t slot = v.sslot[s];
      f = (v.nval[slot] == UNSET && v.nclaim[slot] == s) ? 1u : 0u;
    }
    v.snew[s] = f;
  }
};
struct SuccNewF {
  View v;
  __host__ __device__ void operator()(uint32_t s) const {
    if (!v.snew[s]) return;
    const uint32_t id = NN(v) + v.srank[s];
    if (id >= v.nodes_cap) {
      at_or(&v.ctl->err, ERR_RANGE);
      return;
    }
    v.nkey[id] = v.succ[s];
    v.nval[v.sslot[s]] = id;
  }
};
struct SuccFillF {
  View v;
  __host__ __device__ void operator()(uint32_t s) const {
    const Key k = v.succ[s];
    if (k.kind == K_NONE) return;
    const uint32_t id = v.nval[v.sslot[s]];
    const bool ok = id < v.nodes_cap && key_eq(v.nkey[id], k);
    if (!ok) at_or(&v.ctl->err, ERR_COLLISION);
    v.sres[s] = ok ? id : 0u;
  }
};

// ---- edges of the frontier ----------------------------------------------------
struct EdgeF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    const uint32_t g = F0(v) + i, n = v.fcnt[i];
    const unsigned long long e = (unsigned long long)NE(v) + v.feoff[i];
    v.nrow[g] = n;
    v.neoff[g] = (uint32_t)e;
    if (e + n > v.edges_cap) {
      at_or(&v.ctl->err, ERR_RANGE);
      return;
    }
    const uint32_t s0 = v.off_s[i];
    for (uint32_t t = 0; t < n; t++) {
      v.ecol[e + t] = v.sres[s0 + t];
      v.ewt[e + t] = v.swt[s0 + t];
    }
  }
};

// ---- job-local ids of the new positions (n_nodes .. n_nodes+cnt-1) ---------
// The new positions of a level are sorted by job, each job's in discovery order.
struct LocalAF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    const uint32_t g = NN(v) + i, j = v.sjob[v.nkey[g].p];
    if (i == 0 || v.sjob[v.nkey[g - 1].p] != j) v.jfirst[j] = g;
  }
};
struct LocalBF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    const uint32_t g = NN(v) + i, j = v.sjob[v.nkey[g].p];
    v.nlocal[g] = v.jcount[j] + (g - v.jfirst[j]);
  }
};
struct LocalCF {
  View v;
  __host__ __device__ void operator()(uint32_t i) const {
    const uint32_t cnt = (uint32_t)v.t[T_NEW];
    const uint32_t g = NN(v) + i, j = v.sjob[v.nkey[g].p];
    if (i + 1 == cnt || v.sjob[v.nkey[g + 1].p] != j) {
      v.jcount[j] = v.nlocal[g] + 1;
      if (v.max_pos && v.jcount[j] > v.max_pos) v.jover[j] = 1;
    }
  }
};

// ---- table growth ----------------------------------------------------------------
struct SetRehashF {
  View v;
  __host__ __device__ void operator()(uint32_t id) const {
    const unsigned long long h = set_hash(v.sdata + v.sstart[id], v.slen[id], v.seed);
    uint32_t s = (uint32_t)(h >> 20) & v.smask;
    for (uint32_t probes = 0; at_cas(&v.stab[s], 0ull, h) != 0ull; probes++) {
      if (probes > v.smask) {
        at_or(&v.ctl->err, ERR_RANGE);
        return;
      }
      s = (s + 1) & v.smask;
    }
    v.sval[s] = id;
  }
};
struct NodeRehashF {
  View v;
  __host__ __device__ void operator()(uint32_t g) const {
    const unsigned long long h = key_hash(v.nkey[g], v.seed);
    uint32_t s = (uint32_t)(h >> 20) & v.nmask;
    for (uint32_t probes = 0; at_cas(&v.ntab[s], 0ull, h) != 0ull; probes++) {
      if (probes > v.nmask) {
        at_or(&v.ctl->err, ERR_RANGE);
        return;
      }
      s = (s + 1) & v.nmask;
    }
    v.nval[s] = g;
  }
};

// ---- output: per-job CSR in local ids -----------------------------------------
struct Out {
  uint32_t *jbase;  // n_jobs + 1: first position of each job in the output order
  uint32_t *fperm;  // output position -> discovery index
  uint32_t *frl;    // row lengths in output order, then their exclusive scan
  uint32_t *frow;
  uint32_t *row;    // per job n_j + 1 offsets, jobs concatenated (N + n_jobs)
  uint32_t *rrel;   // the same without each job's last entry (N): the solver's input layout
  uint32_t *jm;     // edges per job
  uint32_t *col, *wt;
  uint8_t *att;
};
struct PermF {
  View v;
  Out o;
  __host__ __device__ void operator()(uint32_t g) const {
    const uint32_t f = o.jbase[v.sjob[v.nkey[g].p]] + v.nlocal[g];
    o.fperm[f] = g;
    o.frl[f] = v.nrow[g];
  }
};
struct RowsF {
  View v;
  Out o;
  __host__ __device__ void operator()(uint32_t f) const {
    const uint32_t g = o.fperm[f], j = v.sjob[v.nkey[g].p];
    const uint32_t eb = o.frow[o.jbase[j]];
    o.row[o.jbase[j] + j + v.nlocal[g]] = o.frow[f] - eb;
    o.rrel[f] = o.frow[f] - eb;
    o.att[f] = v.nkey[g].kind != K_DEFEND;
    const uint32_t n = v.nrow[g], src = v.neoff[g], dst = o.frow[f];
    for (uint32_t t = 0; t < n; t++) {
      o.col[dst + t] = v.nlocal[v.ecol[src + t]];
      o.wt[dst + t] = v.ewt[src + t];
    }
  }
};
struct RowEndF {
  View v;
  Out o;
  __host__ __device__ void operator()(uint32_t j) const {
    // a job without positions (no start pairs) has an empty graph
    const uint32_t last = o.jbase[j] + v.jcount[j];
    const uint32_t end = last < NN(v) ? o.frow[last] : NE(v);
    const uint32_t begin = v.jcount[j] ? o.frow[o.jbase[j]] : end;
    o.row[o.jbase[j] + j + v.jcount[j]] = end - begin;
    o.jm[j] = end - begin;
  }
};

// ---- level bookkeeping on the device (one thread each) ---------------------------
// Start of a level: done when the frontier is empty; a frontier beyond the
// scratch capacity stalls the loop until the host has grown the buffers.
__host__ __device__ inline void level_start(const View &v) {
  v.ctl->n_heavy = 0;
  if (v.t[T_F] == 0) {
    v.t[T_GO] = 0;
    v.t[T_DONE] = 1;
  } else if (v.t[T_F] > v.capF) {
    v.t[T_GO] = 0;
    v.t[T_STALL] = 1;
  }
}
struct LevelStartF {
  View v;
  __host__ __device__ void operator()(uint32_t) const {
    if (v.t[T_GO]) level_start(v);
  }
};
// After the bounds' scans and before anything persistent is written: every
// buffer and table must hold this level, else the level stalls (and is run
// again after the host grew them).
__host__ __device__ inline void level_gate(const View &v) {
  {
    const unsigned long long S = v.t[T_S], E = v.t[T_E], C = v.t[T_C], nn = v.t[T_NN], ne = v.t[T_NE];
    const unsigned long long ns = v.ctl->n_sets, top = v.ctl->sdata_top;
    const bool fits = S < (1ull << 31) && E < (1ull << 31) && C < (1ull << 31) && S <= v.capS && E <= v.capE &&
                      C <= v.capC && ns + C <= v.sets_cap && top + E <= v.sdata_cap && 2 * (ns + C) <= v.scap &&
                      nn + S <= v.nodes_cap && 2 * (nn + S) <= v.ncap && ne + S <= v.edges_cap;
    if (!fits) {
      v.t[T_GO] = 0;
      v.t[T_STALL] = 1;
    }
  }
}
struct LevelGateF {
  View v;
  __host__ __device__ void operator()(uint32_t) const {
    if (v.t[T_GO]) level_gate(v);
  }
};
__host__ __device__ inline void level_end(const View &v) {
  v.t[T_NN] += v.t[T_NEW];
  v.t[T_NE] += v.t[T_EDGE];
  v.t[T_F0] += v.t[T_F];
  v.t[T_F] = v.t[T_NEW];
  v.t[T_LEVELS] += 1;
}
struct LevelEndF {
  View v;
  __host__ __device__ void operator()(uint32_t) const {
    if (v.t[T_GO]) level_end(v);
  }
};

// ---- the level loop ------------------------------------------------------------
// Host-side driver over a backend B with
//   void *alloc(size_t); void release(void *); void fill(void *, int, size_t);
//   void copy(void *dst, const void *src, size_t);        (stream-ordered)
//   void fetch(void *host, const void *dev, size_t);      (waits)
//   template <class F> void each(uint32_t n, const F &);
//   void scan(const uint32_t *in, uint32_t *out, uint32_t n, unsigned long long *dev_total);
//   void gen_heavy(const View &, const unsigned long long *go);  (the positions CountF queued in v.hq)
//   each_d / scan_d / scan2_d / scan3_d: the same with the item count read on
//     the device (*n), doing nothing while *go == 0 (a stalled or finished
//     loop); scan2_d scans two arrays with their own counts;
//   void scan_capacity(uint64_t max_items): room for scans of that many items;
//   begin_capture / end_capture(go) / run_graph(limit) / note_levels /
//     has_graph / drop_graph: one level recorded once and run repeatedly
//     (on the device a CUDA graph WHILE node: up to `limit` levels per launch,
//     stopping as soon as *go == 0).
//   bool ok();                                             (no backend error so far)
struct Totals {
  Ctl ctl;
  unsigned long long t[T_COUNT];
};

// Inputs: all jobs' LTSs in one id space (states of job j contiguous).
struct Input {
  uint32_t NS = 0, MS = 0, n_jobs = 0;
  const uint32_t *soff = nullptr;  // NS + 1
  const int32_t *slab = nullptr;   // MS
  const uint32_t *stgt = nullptr;  // MS, global ids
  const uint32_t *sjob = nullptr;  // NS
  uint32_t n_starts = 0;                         // start positions, job-major
  const uint32_t *p0 = nullptr, *q0 = nullptr;  // n_starts, global ids
  const uint32_t *jsb = nullptr;                 // n_jobs + 1: first state of each job
  uint32_t max_pos = 0;
  uint32_t heavy_min = 0xffffffffu;              // |Q| from which the warp path takes an attack position
};
// Output, in backend memory until fetched: per job j, positions
// jbase[j] .. jbase[j]+jcount[j]-1 and row offsets at row[jbase[j]+j ..].
struct Result {
  uint32_t N = 0, M = 0, levels = 0, attempts = 0;
  uint32_t *row = nullptr, *rrel = nullptr, *col = nullptr, *wt = nullptr, *jcount = nullptr, *jover = nullptr,
           *jbase = nullptr, *jm = nullptr;
  uint8_t *att = nullptr;
};

template <class B>
class Builder {
 public:
  explicit Builder(B &be) : be_(be) {}
  ~Builder() { release_all(); }
  // 0 on success; 1 backend failure / out of memory; 2 sizes beyond u32; 3 repeated collisions
  int run(const Input &in, Result &out, unsigned long long seed = 0x243f6a8885a308d3ull) {
    for (uint32_t attempt = 0; attempt < 4; attempt++) {
      const int r = attempt_build(in, seed + 0x9e3779b97f4a7c15ull * attempt, out);
      out.attempts = attempt + 1;
      if (r != 3) return r;
      release_all();
    }
    return 3;
  }
  // Capacities to start from (a hint, e.g. those of the previous build on
  // the same stream: a serving loop's batches then rarely stall for buffers)
  // and those a successful build ended with.
  struct Caps {
    uint32_t F = 0, S = 0, E = 0, C = 0, sets = 0, sdata = 0, nodes = 0, edges = 0;
  };
  Caps hint, used;
  // device buffers of the result stay owned by the builder until it dies
  // After a failure: the request that could not be met (elements or bytes),
  // and the positions / edges / levels reached.
  uint64_t short_ = 0;
  uint64_t reached_positions() const { return h_tot_.t[T_NN]; }
  uint64_t reached_edges() const { return h_tot_.t[T_NE]; }
  uint64_t reached_levels() const { return h_tot_.t[T_LEVELS]; }

 private:
  B &be_;
  struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
  };
  std::vector<Buf> bufs_;
  bool exact_ = false;
  template <class T>
  T *get(size_t n) {
    const size_t b = (n ? n : 1) * sizeof(T);
    void *p = be_.alloc(b);
    if (p) bufs_.push_back(Buf{p, b});
    return (T *)p;
  }
  template <class T>
  void put(T *&p) {
    for (size_t i = 0; i < bufs_.size(); i++)
      if (bufs_[i].p == (void *)p) {
        be_.release(p);
        bufs_[i] = bufs_.back();
        bufs_.pop_back();
        break;
      }
    p = nullptr;
  }
  void release_all() {
    for (auto &b : bufs_) be_.release(b.p);
    bufs_.clear();
  }
  // grow array p (keeping `keep` elements) to at least `need` elements
  template <class T>
  bool grow(T *&p, uint32_t &cap, uint64_t need, uint64_t keep) {
    if (need <= cap) return true;
    // doubling: few stalls of the level loop (exact while capacities from a
    // hint are applied, so that hints do not grow from build to build)
    uint64_t nc = exact_ ? need : std::max<uint64_t>(2 * need, 1024);
    if (nc > 0xffffffffull) nc = need;
    if (nc > 0xffffffffull) {
      short_ = need;
      return false;
    }
    T *q = get<T>(nc);
    if (!q) {  // no room for headroom: exactly what is needed
      nc = need;
      q = get<T>(nc);
    }
    if (!q) {
      short_ = need * sizeof(T);
      return false;
    }
    if (p && keep) be_.copy(q, p, keep * sizeof(T));
    put(p);
    p = q;
    cap = (uint32_t)nc;
    return true;
  }

  View v_{};
  Totals *d_tot_ = nullptr;
  Totals h_tot_{};
  uint32_t capF_ = 0, capS_ = 0, capE_ = 0, capC_ = 0, capNew_ = 0;
  uint32_t capSets_ = 0, capSdata_ = 0, capNodes_ = 0, capEdges_ = 0;
  uint32_t scap_ = 0, ncap_ = 0;  // table sizes

  bool fetch_totals() {
    be_.fetch(&h_tot_, d_tot_, sizeof(Totals));
    return be_.ok();
  }
  bool ensure_frontier(uint32_t F) {
    uint32_t c;
    bool ok = true;
    uint32_t m_capF_ = 0xffffffffu;
    c = capF_; ok = ok && grow(v_.ub_s, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.ub_e, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.ub_c, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.off_s, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.off_e, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.off_c, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.fcnt, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.feoff, c, F, 0); m_capF_ = std::min(m_capF_, c);
    c = capF_; ok = ok && grow(v_.hq, c, F, 0); m_capF_ = std::min(m_capF_, c);
    capF_ = m_capF_;
    return ok;
  }
  bool ensure_level(uint32_t S, uint32_t E, uint32_t C) {
    bool ok = true;
    uint32_t c;
    uint32_t m_capS_ = 0xffffffffu;
    c = capS_; ok = ok && grow(v_.succ, c, S, 0); m_capS_ = std::min(m_capS_, c);
    c = capS_; ok = ok && grow(v_.swt, c, S, 0); m_capS_ = std::min(m_capS_, c);
    c = capS_; ok = ok && grow(v_.sslot, c, S, 0); m_capS_ = std::min(m_capS_, c);
    c = capS_; ok = ok && grow(v_.sres, c, S, 0); m_capS_ = std::min(m_capS_, c);
    c = capS_; ok = ok && grow(v_.snew, c, S, 0); m_capS_ = std::min(m_capS_, c);
    c = capS_; ok = ok && grow(v_.srank, c, S, 0); m_capS_ = std::min(m_capS_, c);
    capS_ = m_capS_;
    uint32_t m_capE_ = 0xffffffffu;
    c = capE_; ok = ok && grow(v_.celem, c, E, 0); m_capE_ = std::min(m_capE_, c);
    capE_ = m_capE_;
    uint32_t m_capC_ = 0xffffffffu;
    c = capC_; ok = ok && grow(v_.cstart, c, C, 0); m_capC_ = std::min(m_capC_, c);
    c = capC_; ok = ok && grow(v_.clen, c, C, 0); m_capC_ = std::min(m_capC_, c);
    c = capC_; ok = ok && grow(v_.cslot, c, C, 0); m_capC_ = std::min(m_capC_, c);
    c = capC_; ok = ok && grow(v_.cid, c, C, 0); m_capC_ = std::min(m_capC_, c);
    capC_ = m_capC_;
    return ok;
  }
  // set store and table for `extra` more sets of at most `words` words
  bool ensure_sets(uint32_t n_sets, uint32_t top, uint64_t extra, uint64_t words) {
    bool ok = true;
    uint32_t c;
    uint32_t m_capSdata_ = 0xffffffffu;
    c = capSdata_; ok = ok && grow(v_.sdata, c, top + words, top); m_capSdata_ = std::min(m_capSdata_, c);
    capSdata_ = m_capSdata_;
    uint32_t m_capSets_ = 0xffffffffu;
    c = capSets_; ok = ok && grow(v_.sstart, c, n_sets + extra, n_sets); m_capSets_ = std::min(m_capSets_, c);
    c = capSets_; ok = ok && grow(v_.slen, c, n_sets + extra, n_sets); m_capSets_ = std::min(m_capSets_, c);
    capSets_ = m_capSets_;
    if (!ok) return false;
    const uint64_t need = 2 * ((uint64_t)n_sets + extra);
    if (need <= scap_) return true;
    uint64_t cap = 1024;
    while (cap < 2 * need && cap < (1ull << 31)) cap <<= 1;  // load <= 1/4, at most 2^31 slots
    if (cap < need) {
      short_ = need;
      return false;
    }
    put(v_.stab); put(v_.sval); put(v_.sclaim);
    v_.stab = get<unsigned long long>(cap);
    v_.sval = get<uint32_t>(cap);
    v_.sclaim = get<uint32_t>(cap);
    if (!v_.stab || !v_.sval || !v_.sclaim) {
      short_ = cap * 16;
      return false;
    }
    be_.fill(v_.stab, 0, cap * 8);
    be_.fill(v_.sval, 0xff, cap * 4);
    be_.fill(v_.sclaim, 0xff, cap * 4);
    scap_ = (uint32_t)cap;
    sync_view();
    v_.smask = scap_ - 1;
    be_.each(n_sets, SetRehashF{v_});
    return true;
  }
  bool ensure_nodes(uint32_t n_nodes, uint64_t extra, uint32_t n_edges, uint64_t extra_edges) {
    bool ok = true;
    uint32_t c;
    uint32_t m_capNodes_ = 0xffffffffu;
    c = capNodes_; ok = ok && grow(v_.nkey, c, n_nodes + extra, n_nodes); m_capNodes_ = std::min(m_capNodes_, c);
    c = capNodes_; ok = ok && grow(v_.nlocal, c, n_nodes + extra, n_nodes); m_capNodes_ = std::min(m_capNodes_, c);
    c = capNodes_; ok = ok && grow(v_.nrow, c, n_nodes + extra, n_nodes); m_capNodes_ = std::min(m_capNodes_, c);
    c = capNodes_; ok = ok && grow(v_.neoff, c, n_nodes + extra, n_nodes); m_capNodes_ = std::min(m_capNodes_, c);
    capNodes_ = m_capNodes_;
    uint32_t m_capEdges_ = 0xffffffffu;
    c = capEdges_; ok = ok && grow(v_.ecol, c, (uint64_t)n_edges + extra_edges, n_edges); m_capEdges_ = std::min(m_capEdges_, c);
    c = capEdges_; ok = ok && grow(v_.ewt, c, (uint64_t)n_edges + extra_edges, n_edges); m_capEdges_ = std::min(m_capEdges_, c);
    capEdges_ = m_capEdges_;
    if (!ok) return false;
    const uint64_t need = 2 * ((uint64_t)n_nodes + extra);
    if (need <= ncap_) return true;
    uint64_t cap = 1024;
    while (cap < 2 * need && cap < (1ull << 31)) cap <<= 1;  // load <= 1/4, at most 2^31 slots
    if (cap < need) {
      short_ = need;
      return false;
    }
    put(v_.ntab); put(v_.nval); put(v_.nclaim);
    v_.ntab = get<unsigned long long>(cap);
    v_.nval = get<uint32_t>(cap);
    v_.nclaim = get<uint32_t>(cap);
    if (!v_.ntab || !v_.nval || !v_.nclaim) {
      short_ = cap * 16;
      return false;
    }
    be_.fill(v_.ntab, 0, cap * 8);
    be_.fill(v_.nval, 0xff, cap * 4);
    be_.fill(v_.nclaim, 0xff, cap * 4);
    ncap_ = (uint32_t)cap;
    sync_view();
    v_.nmask = ncap_ - 1;
    be_.each(n_nodes, NodeRehashF{v_});
    return true;
  }
  void sync_view() {
    v_.sdata_cap = capSdata_;
    v_.sets_cap = capSets_;
    v_.smask = scap_ ? scap_ - 1 : 0;
    v_.nodes_cap = capNodes_;
    v_.nmask = ncap_ ? ncap_ - 1 : 0;
    v_.edges_cap = capEdges_;
    v_.capF = capF_;
    v_.capS = capS_;
    v_.capE = capE_;
    v_.capC = capC_;
    v_.scap = scap_;
    v_.ncap = ncap_;
    v_.t = d_tot_ ? d_tot_->t : nullptr;
    be_.scan_capacity(std::max<uint64_t>(capF_, capS_));
  }
  const unsigned long long *tp(int k) const { return &d_tot_->t[k]; }
  // One breadth-first level, every count read on the device (no host sync):
  // bounds, gate, successors, interning, numbering, edges, local ids.
  void enqueue_level() {
    const unsigned long long *go = tp(T_GO);
    be_.each(1, LevelStartF{v_});
    be_.each_d(tp(T_F), capF_, go, CountF{v_});
    be_.scan3_d(v_.ub_s, v_.ub_e, v_.ub_c, v_.off_s, v_.off_e, v_.off_c, tp(T_F), &d_tot_->t[T_S], go);
    be_.each(1, LevelGateF{v_});
    be_.each_d(tp(T_F), capF_, go, GenF{v_});
    be_.gen_heavy(v_, go);
    be_.each_d(tp(T_C), capC_, go, SetProbeF{v_});
    be_.each_d(tp(T_C), capC_, go, SetNewF{v_});
    be_.each_d(tp(T_C), capC_, go, SetFillF{v_});
    be_.each_d(tp(T_S), capS_, go, SuccProbeF{v_});
    be_.each_d(tp(T_S), capS_, go, SuccFlagF{v_});
    be_.scan2_d(v_.snew, v_.srank, tp(T_S), &d_tot_->t[T_NEW], v_.fcnt, v_.feoff, tp(T_F), &d_tot_->t[T_EDGE], go);
    be_.each_d(tp(T_S), capS_, go, SuccNewF{v_});
    be_.each_d(tp(T_S), capS_, go, SuccFillF{v_});
    be_.each_d(tp(T_F), capF_, go, EdgeF{v_});
    be_.each_d(tp(T_NEW), capS_, go, LocalAF{v_});
    be_.each_d(tp(T_NEW), capS_, go, LocalBF{v_});
    be_.each_d(tp(T_NEW), capS_, go, LocalCF{v_});
    be_.each(1, LevelEndF{v_});
  }

  int attempt_build(const Input &in, unsigned long long seed, Result &out) {
    v_ = View{};
    capF_ = capS_ = capE_ = capC_ = capNew_ = capSets_ = capSdata_ = capNodes_ = capEdges_ = scap_ = ncap_ = 0;
    be_.drop_graph();
    v_.soff = in.soff;
    v_.slab = in.slab;
    v_.stgt = in.stgt;
    v_.sjob = in.sjob;
    v_.p0 = in.p0;
    v_.q0 = in.q0;
    v_.jsb = in.jsb;
    v_.heavy_min = in.heavy_min;
    v_.n_jobs = in.n_jobs;
    v_.max_pos = in.max_pos;
    v_.seed = seed;
    const uint32_t J = in.n_jobs;
    d_tot_ = get<Totals>(1);
    v_.jcount = get<uint32_t>(J);
    v_.jfirst = get<uint32_t>(J);
    v_.jover = get<uint32_t>(J);
    if (!d_tot_ || !v_.jcount || !v_.jfirst || !v_.jover) return 1;
    be_.fill(d_tot_, 0, sizeof(Totals));
    be_.fill(v_.jcount, 0, (size_t)J * 4);
    be_.fill(v_.jover, 0, (size_t)J * 4);
    v_.ctl = &d_tot_->ctl;
    // the empty set is set 0
    if (!ensure_sets(0, 0, (uint64_t)in.n_starts + 1, (uint64_t)in.n_starts + 1)) return 1;
    {
      const uint32_t zero = 0;
      Ctl c0{0, 1, 0, 0};
      be_.copy(v_.sstart, &zero, 4);
      be_.copy(v_.slen, &zero, 4);
      be_.copy(&d_tot_->ctl, &c0, sizeof(Ctl));
      sync_view();
      be_.each(1, SetRehashF{v_});
      be_.fetch(&h_tot_, d_tot_, sizeof(Totals));  // also keeps the host copies alive until done
    }
    // level 0: the start positions Attack(p0[t], {q0[t]}), numbered in order
    const uint32_t T = in.n_starts;
    if (!ensure_level(T, T, T) || !ensure_nodes(0, T, 0, 0)) return 1;
    sync_view();
    be_.each(T, StartF{v_});
    be_.each(T, SetProbeF{v_});
    be_.each(T, SetNewF{v_});
    be_.each(T, SetFillF{v_});
    be_.each(T, SuccProbeF{v_});
    be_.each(T, SuccFlagF{v_});
    be_.scan(v_.snew, v_.srank, T, &d_tot_->t[T_NEW]);
    if (!fetch_totals()) return 1;
    const uint32_t newN = (uint32_t)h_tot_.t[T_NEW];
    be_.each(T, SuccNewF{v_});
    be_.each(T, SuccFillF{v_});
    be_.each(newN, LocalAF{v_});
    be_.each(newN, LocalBF{v_});
    be_.each(newN, LocalCF{v_});
    // the level loop from here on runs on the device
    if (!fetch_totals()) return 1;
    h_tot_.t[T_NN] = newN;
    h_tot_.t[T_NE] = 0;
    h_tot_.t[T_F0] = 0;
    h_tot_.t[T_F] = newN;
    h_tot_.t[T_GO] = 1;
    h_tot_.t[T_STALL] = 0;
    h_tot_.t[T_DONE] = 0;
    h_tot_.t[T_LEVELS] = 0;
    be_.copy(d_tot_, &h_tot_, sizeof(Totals));
    // first guesses; the gate stalls a level that does not fit and the
    // buffers grow to its exact needs
    {
      const uint64_t guess = 8ull * newN + 4096;
      auto mx = [&](uint32_t h) { return (uint32_t)std::max<uint64_t>(guess, h); };
      const uint32_t n_sets = h_tot_.ctl.n_sets, top = h_tot_.ctl.sdata_top;
      exact_ = true;
      bool ok =
          ensure_frontier(std::max<uint32_t>(std::max<uint32_t>(newN, 4096), hint.F)) &&
          ensure_level(mx(hint.S), mx(hint.E), mx(hint.C)) &&
          ensure_sets(n_sets, top, std::max<uint64_t>(guess, hint.sets > n_sets ? hint.sets - n_sets : 0),
                      std::max<uint64_t>(guess, hint.sdata > top ? hint.sdata - top : 0)) &&
          ensure_nodes(newN, std::max<uint64_t>(guess, hint.nodes > newN ? hint.nodes - newN : 0), 0, mx(hint.edges));
      exact_ = false;
      if (!ok)  // the hint asked for more than the device has now: start small
        ok = ensure_frontier(std::max<uint32_t>(newN, 4096)) &&
             ensure_level((uint32_t)guess, (uint32_t)guess, (uint32_t)guess) &&
             ensure_sets(n_sets, top, guess, guess) && ensure_nodes(newN, guess, 0, guess);
      if (!ok) return 1;
      short_ = 0;
    }
    // levels per graph launch: the loop stops by itself when the frontier
    // runs empty or a level stalls; the limit only bounds one launch
    const uint32_t batch = 4096;
    unsigned long long last_stall = ~0ull;
    uint32_t same_stall = 0;
    for (;;) {
      sync_view();
      if (!be_.has_graph()) {
        be_.begin_capture();
        enqueue_level();
        be_.end_capture(tp(T_GO));
      }
      const unsigned long long levels_before = h_tot_.t[T_LEVELS];
      be_.run_graph(batch);  // up to `batch` levels, fewer when the loop stops
      if (!fetch_totals()) return 1;
      be_.note_levels(h_tot_.t[T_LEVELS] - levels_before + (h_tot_.t[T_STALL] ? 1 : 0));
      if (h_tot_.ctl.err & ERR_COLLISION) return 3;
      if (h_tot_.ctl.err) return 2;
      if (h_tot_.t[T_DONE]) break;
      if (!h_tot_.t[T_STALL]) {
        // no progress without a stall would be a defect (a recorded loop
        // always runs a level; plain mode runs one as it is "recorded")
        if (h_tot_.t[T_LEVELS] == levels_before && be_.has_graph()) return 2;
        continue;
      }
      // grow to the stalled level's needs (its bounds were counted, or the
      // frontier itself did not fit) and run it again; a level that stalls
      // again after its buffers grew would be a defect: give up
      if (h_tot_.t[T_LEVELS] == last_stall && ++same_stall > 2) return 2;
      if (h_tot_.t[T_LEVELS] != last_stall) same_stall = 0;
      last_stall = h_tot_.t[T_LEVELS];
      const unsigned long long F = h_tot_.t[T_F], S = h_tot_.t[T_S], E = h_tot_.t[T_E], C = h_tot_.t[T_C];
      const unsigned long long nn = h_tot_.t[T_NN], ne = h_tot_.t[T_NE];
      if (F >= (1ull << 31) || S >= (1ull << 31) || E >= (1ull << 31) || C >= (1ull << 31) ||
          (uint64_t)h_tot_.ctl.sdata_top + E >= (1ull << 32) || nn + S >= (1ull << 31) || ne + S >= (1ull << 32))
        return 2;
      if (!ensure_frontier((uint32_t)F) || !ensure_level((uint32_t)S, (uint32_t)E, (uint32_t)C)) return 1;
      if (!ensure_sets(h_tot_.ctl.n_sets, h_tot_.ctl.sdata_top, C, E)) return 1;
      if (!ensure_nodes((uint32_t)nn, S, (uint32_t)ne, S)) return 1;
      be_.drop_graph();
      h_tot_.t[T_GO] = 1;
      h_tot_.t[T_STALL] = 0;
      be_.copy(&d_tot_->t[T_GO], &h_tot_.t[T_GO], 2 * sizeof(unsigned long long));
    }
    be_.drop_graph();
    v_.t = d_tot_->t;
    const uint32_t levels = (uint32_t)h_tot_.t[T_LEVELS];
    if (!fetch_totals()) return 1;
    if (h_tot_.ctl.err & ERR_COLLISION) return 3;
    if (h_tot_.ctl.err) return 2;
    // per-job CSR in local ids
    const uint32_t N = (uint32_t)h_tot_.t[T_NN], M = (uint32_t)h_tot_.t[T_NE];
    Out o{};
    o.jbase = get<uint32_t>((size_t)J + 1);
    o.fperm = get<uint32_t>(N);
    o.frl = get<uint32_t>(N);
    o.frow = get<uint32_t>(N);
    o.row = get<uint32_t>((size_t)N + J);
    o.rrel = get<uint32_t>(N);
    o.jm = get<uint32_t>(J);
    o.col = get<uint32_t>(M);
    o.wt = get<uint32_t>(M);
    o.att = get<uint8_t>(N);
    if (!o.jbase || !o.fperm || !o.frl || !o.frow || !o.row || !o.rrel || !o.jm || !o.col || !o.wt || !o.att)
      return 1;
    sync_view();
    be_.scan(v_.jcount, o.jbase, J, &d_tot_->t[T_N]);
    be_.each(N, PermF{v_, o});
    be_.scan(o.frl, o.frow, N, &d_tot_->t[T_EDGE]);
    be_.each(N, RowsF{v_, o});
    be_.each(J, RowEndF{v_, o});
    if (!fetch_totals()) return 1;
    if (h_tot_.t[T_N] != N || h_tot_.t[T_EDGE] != M || h_tot_.ctl.err) return 2;
    used = Caps{capF_, capS_, capE_, capC_, capSets_, capSdata_, capNodes_, capEdges_};
    out.N = N;
    out.M = M;
    out.levels = levels;
    out.row = o.row;
    out.rrel = o.rrel;
    out.jm = o.jm;
    out.col = o.col;
    out.wt = o.wt;
    out.att = o.att;
    out.jcount = v_.jcount;
    out.jover = v_.jover;
    out.jbase = o.jbase;
    return 0;
  }
};

}  // namespace gb
}  // namespace geq
