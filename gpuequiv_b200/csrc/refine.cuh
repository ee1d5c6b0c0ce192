// refine.cuh - strong bisimulation minimisation on the device for many LTSs at
// once: TransitionSystem::signature_refinement (src/lib.rs:444-478) and
// bisimilar_minimize (src/lib.rs:413-432).
//
// One iteration for every state p of every job: the signature
// {(label, class of target)} sorted and deduplicated, a 64-bit fingerprint of
// (job, signature), a hash table whose slot is claimed by the smallest state
// (the first process of the class in process order, as the reference hands out
// ids), a check of every state's signature against its representative's (a
// fingerprint collision raises an error flag and the caller retries with
// another seed), and the new class id = rank of the representative among its
// job's representatives.  The loop ends when no job's class count changed in
// an iteration; extra iterations of a stable job reproduce its partition, so
// all jobs run together.
//
// The minimised systems are then written, still on the device, in the
// builder's input layout (gbuild.cuh Input): class c of job j is represented
// by its first process, whose transitions are copied with targets replaced by
// their classes.
#pragma once

#include "gbuild.cuh"

namespace geq {
namespace rf {

using gb::at_add;
using gb::at_cas;
using gb::at_min;
using gb::at_or;
using gb::mix64;
using gb::UNSET;

struct RView {
  const uint32_t *soff;  // NS + 1
  const int32_t *slab;
  const uint32_t *stgt;  // global ids
  const uint32_t *sjob;
  const uint32_t *jsb;   // J + 1
  uint32_t NS, J;
  const uint32_t *part;  // per state (global id): its class (job-local id) in the previous iteration
  uint32_t *npart;       // the same for this iteration
  unsigned long long *sig;  // per state at soff[p]: (label ^ 0x80000000) << 32 | class
  uint32_t *slen;
  unsigned long long *fp;   // fingerprint per state
  unsigned long long *tab;  // fingerprints, 0 = free
  uint32_t *claim;          // smallest state per slot
  uint32_t mask;
  uint32_t *slot, *rep, *isrep, *rank;
  uint32_t *cnt;            // classes per job (last iteration)
  uint32_t *flags;          // [0] changed in this iteration, [1] error
  unsigned long long *tot;  // number of representatives (scan total)
  unsigned long long seed;
};

__host__ __device__ inline void sort_u64(unsigned long long *a, uint32_t n) {
  if (n <= 32) {
    for (uint32_t i = 1; i < n; i++) {
      const unsigned long long x = a[i];
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
      const unsigned long long t = a[r]; a[r] = a[c]; a[c] = t;
      r = c;
    }
  };
  for (uint32_t r = n / 2; r-- > 0;) sift(r, n);
  for (uint32_t end = n - 1; end > 0; end--) {
    const unsigned long long t = a[0]; a[0] = a[end]; a[end] = t;
    sift(0, end);
  }
}

// signatures (lib.rs:467-477) and their fingerprints
struct SigF {
  RView v;
  __host__ __device__ void operator()(uint32_t p) const {
    const uint32_t b = v.soff[p], e = v.soff[p + 1], j = v.sjob[p];
    unsigned long long *s = v.sig + b;
    for (uint32_t k = b; k < e; k++)
      s[k - b] = ((unsigned long long)((uint32_t)v.slab[k] ^ 0x80000000u) << 32) | v.part[v.stgt[k]];
    sort_u64(s, e - b);
    uint32_t n = 0;
    for (uint32_t k = 0; k < e - b; k++)
      if (n == 0 || s[k] != s[n - 1]) s[n++] = s[k];
    v.slen[p] = n;
    unsigned long long h = mix64(v.seed ^ (((unsigned long long)j << 32) | n));
    for (uint32_t k = 0; k < n; k++) h = mix64(h ^ (s[k] + 0x9e3779b97f4a7c15ull));
    v.fp[p] = h ? h : 1ull;
  }
};
struct ProbeF {
  RView v;
  __host__ __device__ void operator()(uint32_t p) const {
    const unsigned long long h = v.fp[p];
    uint32_t s = (uint32_t)(h >> 20) & v.mask;
    for (uint32_t probes = 0;; probes++) {
      if (probes > v.mask) {  // cannot happen below half load; never spin
        at_or(&v.flags[1], 2u);
        v.slot[p] = UNSET;
        return;
      }
      const unsigned long long k = v.tab[s];
      if (k == h) break;
      if (k == 0) {
        const unsigned long long o = at_cas(&v.tab[s], 0ull, h);
        if (o == 0ull || o == h) break;
      }
      s = (s + 1) & v.mask;
    }
    v.slot[p] = s;
    at_min(&v.claim[s], p);
  }
};
// representative of each state, verified word by word
struct RepF {
  RView v;
  __host__ __device__ void operator()(uint32_t p) const {
    const uint32_t s = v.slot[p];
    const uint32_t r = s == UNSET ? p : v.claim[s];
    bool ok = s != UNSET && v.sjob[r] == v.sjob[p] && v.slen[r] == v.slen[p];
    if (ok) {
      const unsigned long long *a = v.sig + v.soff[p], *b = v.sig + v.soff[r];
      for (uint32_t k = 0; k < v.slen[p] && ok; k++) ok = a[k] == b[k];
    }
    if (!ok) at_or(&v.flags[1], 1u);
    v.rep[p] = ok ? r : p;
    v.isrep[p] = (ok ? r : p) == p ? 1u : 0u;
  }
};
__host__ __device__ __forceinline__ uint32_t rank_at(const RView &v, uint32_t s) {
  return s < v.NS ? v.rank[s] : (uint32_t)*v.tot;
}
// new class = rank of the representative among its job's representatives
struct AssignF {
  RView v;
  __host__ __device__ void operator()(uint32_t p) const {
    const uint32_t j = v.sjob[p];
    v.npart[p] = v.rank[v.rep[p]] - rank_at(v, v.jsb[j]);
  }
};
struct CountJobF {
  RView v;
  __host__ __device__ void operator()(uint32_t j) const {
    const uint32_t c = rank_at(v, v.jsb[j + 1]) - rank_at(v, v.jsb[j]);
    if (c != v.cnt[j]) {
      v.cnt[j] = c;
      at_or(&v.flags[0], 1u);
    }
  }
};

// ---- the minimised systems, in the builder's input layout ---------------------
// Inputs: the final partition (npart of the last iteration, job-local ids in
// part arrays indexed by global state), isrep/rank of that iteration.
struct Reduce {
  const uint32_t *cbase;  // J + 1: first reduced state of each job (scan of cnt)
  uint32_t *crep;         // reduced state -> its representative (original global id)
  uint32_t *rdeg;         // reduced state -> degree, then scanned into roff
  uint32_t *roff;         // NR + 1
  int32_t *rlab;
  uint32_t *rtgt;
  uint32_t *rjob;         // NR
  uint32_t NR, MR;
};
// the first process of each class represents it (lib.rs:418-421)
struct RepListF {
  RView v;
  Reduce r;
  __host__ __device__ void operator()(uint32_t p) const {
    if (!v.isrep[p]) return;
    const uint32_t j = v.sjob[p];
    const uint32_t c = v.rank[p] - rank_at(v, v.jsb[j]);
    const uint32_t x = r.cbase[j] + c;
    r.crep[x] = p;
    r.rdeg[x] = v.soff[p + 1] - v.soff[p];
    r.rjob[x] = j;
  }
};
// its transitions with targets mapped to classes (lib.rs:422-430)
struct RowsF {
  RView v;
  Reduce r;
  __host__ __device__ void operator()(uint32_t x) const {
    const uint32_t p = r.crep[x], j = r.rjob[x];
    const uint32_t b = v.soff[p], e = v.soff[p + 1], o = r.roff[x];
    for (uint32_t k = b; k < e; k++) {
      r.rlab[o + (k - b)] = v.slab[k];
      r.rtgt[o + (k - b)] = r.cbase[j] + v.part[v.stgt[k]];
    }
  }
};

struct OneF {
  uint32_t *a;
  __host__ __device__ void operator()(uint32_t i) const { a[i] = 1u; }
};
// start positions mapped to the minimised systems: p -> cbase[job] + class
struct MapStartsF {
  const uint32_t *part, *sjob, *cbase, *p0, *q0;
  uint32_t *rp0, *rq0;
  __host__ __device__ void operator()(uint32_t t) const {
    const uint32_t j = sjob[p0[t]];
    rp0[t] = cbase[j] + part[p0[t]];
    rq0[t] = cbase[j] + part[q0[t]];
  }
};

// Host driver over the same backend interface as gb::Builder.
template <class B>
class Refiner {
 public:
  explicit Refiner(B &be) : be_(be) {}
  ~Refiner() { release_all(); }
  // 0 ok; 1 out of memory / backend failure; 3 repeated fingerprint collisions
  int run(const gb::Input &in) {
    for (uint32_t attempt = 0; attempt < 4; attempt++) {
      const int r = attempt_run(in, 0x13198a2e03707344ull + 0x9e3779b97f4a7c15ull * attempt);
      if (r != 3) return r;
      release_all();
    }
    return 3;
  }
  uint32_t iterations = 0;
  const uint32_t *partition() const { return final_; }  // per state: job-local class
  const uint32_t *counts() const { return v_.cnt; }     // per job
  // The minimised systems in the builder's input layout (device arrays owned
  // by this object), with the start positions of `in` mapped onto them.
  int reduce(const gb::Input &in, gb::Input &out, uint32_t *&rp0, uint32_t *&rq0) {
    const uint32_t J = in.n_jobs, T = in.n_starts;
    Reduce r{};
    uint32_t *cbase = get<uint32_t>((size_t)J + 1);
    r.cbase = cbase;
    if (!cbase) return 1;
    be_.scan(v_.cnt, cbase, J, tot_ + 1);
    be_.fetch(htot_, tot_, sizeof(htot_));
    if (!be_.ok()) return 1;
    const uint32_t NR = (uint32_t)htot_[1];
    be_.copy(cbase + J, &NR, 4);
    r.NR = NR;
    r.crep = get<uint32_t>(NR);
    r.rdeg = get<uint32_t>(NR);
    r.roff = get<uint32_t>((size_t)NR + 1);
    r.rjob = get<uint32_t>(NR);
    rp0 = get<uint32_t>(T);
    rq0 = get<uint32_t>(T);
    if (!r.crep || !r.rdeg || !r.roff || !r.rjob || !rp0 || !rq0) return 1;
    RView v = v_;
    v.part = final_;
    v.isrep = final_isrep_;
    v.rank = final_rank_;
    be_.each(in.NS, RepListF{v, r});
    be_.scan(r.rdeg, r.roff, NR, tot_ + 2);
    be_.fetch(htot_, tot_, sizeof(htot_));
    if (!be_.ok()) return 1;
    const uint32_t MR = (uint32_t)htot_[2];
    be_.copy(r.roff + NR, &MR, 4);
    r.MR = MR;
    r.rlab = get<int32_t>(MR);
    r.rtgt = get<uint32_t>(MR);
    if (!r.rlab || !r.rtgt) return 1;
    be_.each(NR, RowsF{v, r});
    be_.each(T, MapStartsF{final_, in.sjob, cbase, in.p0, in.q0, rp0, rq0});
    out = in;
    out.NS = NR;
    out.MS = MR;
    out.soff = r.roff;
    out.slab = r.rlab;
    out.stgt = r.rtgt;
    out.sjob = r.rjob;
    out.jsb = cbase;
    out.p0 = rp0;
    out.q0 = rq0;
    be_.fetch(htot_, tot_, sizeof(htot_));  // the host copies above are done
    return be_.ok() ? 0 : 1;
  }

 private:
  B &be_;
  std::vector<void *> bufs_;
  RView v_{};
  unsigned long long *tot_ = nullptr;
  unsigned long long htot_[4] = {0, 0, 0, 0};
  uint32_t hflags_[2] = {0, 0};
  const uint32_t *final_ = nullptr;
  uint32_t *final_isrep_ = nullptr, *final_rank_ = nullptr;
  template <class T>
  T *get(size_t n) {
    void *p = be_.alloc((n ? n : 1) * sizeof(T));
    if (p) bufs_.push_back(p);
    return (T *)p;
  }
  void release_all() {
    for (void *p : bufs_) be_.release(p);
    bufs_.clear();
  }
  int attempt_run(const gb::Input &in, unsigned long long seed) {
    const uint32_t NS = in.NS, J = in.n_jobs;
    v_ = RView{};
    v_.soff = in.soff;
    v_.slab = in.slab;
    v_.stgt = in.stgt;
    v_.sjob = in.sjob;
    v_.jsb = in.jsb;
    v_.NS = NS;
    v_.J = J;
    v_.seed = seed;
    uint64_t cap = 1024;
    while (cap < 4 * (uint64_t)NS) cap <<= 1;
    if (cap > (1ull << 31)) return 1;
    v_.mask = (uint32_t)cap - 1;
    uint32_t *part0 = get<uint32_t>(NS), *part1 = get<uint32_t>(NS);
    uint32_t *isrep0 = get<uint32_t>(NS), *isrep1 = get<uint32_t>(NS);
    uint32_t *rank0 = get<uint32_t>(NS), *rank1 = get<uint32_t>(NS);
    v_.sig = get<unsigned long long>(in.MS);
    v_.slen = get<uint32_t>(NS);
    v_.fp = get<unsigned long long>(NS);
    v_.tab = get<unsigned long long>(cap);
    v_.claim = get<uint32_t>(cap);
    v_.slot = get<uint32_t>(NS);
    v_.rep = get<uint32_t>(NS);
    v_.cnt = get<uint32_t>(J);
    v_.flags = get<uint32_t>(2);
    tot_ = get<unsigned long long>(4);
    if (!part0 || !part1 || !isrep0 || !isrep1 || !rank0 || !rank1 || !v_.sig || !v_.slen || !v_.fp || !v_.tab ||
        !v_.claim || !v_.slot || !v_.rep || !v_.cnt || !v_.flags || !tot_)
      return 1;
    v_.tot = tot_;
    be_.fill(part0, 0, (size_t)NS * 4);
    be_.fill(v_.flags, 0, 8);
    be_.fill(tot_, 0, 32);
    be_.each(J, OneF{v_.cnt});  // the reference starts from one class (lib.rs:446-448)
    uint32_t *parts[2] = {part0, part1}, *isreps[2] = {isrep0, isrep1}, *ranks[2] = {rank0, rank1};
    uint32_t it = 0;
    const uint32_t max_it = NS + 2;  // every iteration but the last splits a class
    for (;;) {
      const uint32_t batch = 4;
      for (uint32_t k = 0; k < batch; k++, it++) {
        RView v = v_;
        v.part = parts[it & 1];
        v.npart = parts[(it + 1) & 1];
        v.isrep = isreps[it & 1];
        v.rank = ranks[it & 1];
        be_.fill(v.flags, 0, 4);
        be_.fill(v.tab, 0, cap * 8);
        be_.fill(v.claim, 0xff, cap * 4);
        be_.each(NS, SigF{v});
        be_.each(NS, ProbeF{v});
        be_.each(NS, RepF{v});
        be_.scan(v.isrep, v.rank, NS, tot_);
        be_.each(NS, AssignF{v});
        be_.each(J, CountJobF{v});
      }
      be_.fetch(hflags_, v_.flags, 8);
      if (!be_.ok()) return 1;
      if (hflags_[1] & 1u) return 3;
      if (hflags_[1]) return 1;
      if (!hflags_[0] || it > max_it) break;
    }
    iterations = it;
    final_ = parts[it & 1];
    final_isrep_ = isreps[(it - 1) & 1];
    final_rank_ = ranks[(it - 1) & 1];
    return 0;
  }
};

}  // namespace rf
}  // namespace geq
