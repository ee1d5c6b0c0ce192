// gbuild_host.cpp - test driver: the device game builder's level loop
// (gpuequiv_b200/csrc/gbuild.cuh) and the device minimisation
// (gpuequiv_b200/csrc/refine.cuh) run on the host through a sequential
// backend, against the host GameBuilder and Lts::minimize.  The functors are
// the ones the CUDA kernels run; this checks the algorithm (numbering,
// interning, capacity gate and regrowth, capacity hints, start sets,
// minimised systems) without a GPU.  Test infrastructure only.
//
//   gbuild_host build  <jobs> <max_states> <max_positions> <seed> <density> <labels> <heavy_min> <all>
//   gbuild_host refine <jobs> <max_states> <seed> <density> <labels>
// prints "bad <n> of <jobs>" and exits 1 on any mismatch.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "gamebuild.h"
#include "gbuild.cuh"
#include "lts.h"
#include "refine.cuh"

namespace geq {
void set_last_error(const std::string &msg) { std::fprintf(stderr, "%s\n", msg.c_str()); }
geq_status fail(geq_status st, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stderr, fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "\n");
  return st;
}
}  // namespace geq

using namespace geq;

// Every "launch" runs its items in order; a recorded level is run as it is
// recorded (one level per host iteration of the loop).
struct HostBackend {
  void *alloc(size_t b) { return std::calloc(1, b + 64); }
  void release(void *p) { std::free(p); }
  void fill(void *p, int v, size_t b) { std::memset(p, v, b); }
  void copy(void *d, const void *s, size_t b) { std::memmove(d, s, b); }
  void fetch(void *h, const void *d, size_t b) { std::memmove(h, d, b); }
  bool ok() { return true; }
  template <class F>
  void each(uint32_t n, const F &f) {
    for (uint32_t i = 0; i < n; i++) f(i);
  }
  template <class F>
  void each_d(const unsigned long long *np, uint32_t, const unsigned long long *go, const F &f) {
    if (!*go) return;
    const uint32_t n = (uint32_t)*np;
    for (uint32_t i = 0; i < n; i++) f(i);
  }
  void gen_heavy(const gb::View &v, const unsigned long long *go) {
    if (go && !*go) return;
    for (uint32_t h = 0; h < v.ctl->n_heavy; h++) gb::gen_one(v, v.hq[h]);
  }
  void scan(const uint32_t *in, uint32_t *out, uint32_t n, unsigned long long *tot) {
    unsigned long long s = 0;
    for (uint32_t i = 0; i < n; i++) {
      const uint32_t x = in[i];
      out[i] = (uint32_t)s;
      s += x;
    }
    *tot = s;
  }
  void scan_d(const uint32_t *in, uint32_t *out, const unsigned long long *np, unsigned long long *tot,
              const unsigned long long *go) {
    if (*go) scan(in, out, (uint32_t)*np, tot);
  }
  void scan2_d(const uint32_t *a, uint32_t *x, const unsigned long long *na, unsigned long long *ta,
               const uint32_t *b, uint32_t *y, const unsigned long long *nb, unsigned long long *tb,
               const unsigned long long *go) {
    if (!*go) return;
    scan(a, x, (uint32_t)*na, ta);
    scan(b, y, (uint32_t)*nb, tb);
  }
  void scan_capacity(uint64_t) {}
  void scan3_d(const uint32_t *a, const uint32_t *b, const uint32_t *c, uint32_t *x, uint32_t *y, uint32_t *z,
               const unsigned long long *np, unsigned long long *t, const unsigned long long *go) {
    if (!*go) return;
    const uint32_t n = (uint32_t)*np;
    scan(a, x, n, t);
    scan(b, y, n, t + 1);
    scan(c, z, n, t + 2);
  }
  bool has_graph() const { return false; }
  void begin_capture() {}
  void end_capture(const unsigned long long *) {}
  void run_graph(uint32_t) {}
  void note_levels(unsigned long long) {}
  void drop_graph() {}
};

struct Batch {
  std::vector<Lts> L;
  std::vector<uint32_t> P, Q;
  std::vector<uint64_t> sb, tb;
  std::vector<uint32_t> soff, stgt, sjob, jsb;
  std::vector<int32_t> slab;
};

static void make_batch(Batch &b, int njobs, int maxs, uint64_t seed, int dens, int labs) {
  std::mt19937_64 rng(seed);
  b.L.resize(njobs);
  b.P.resize(njobs);
  b.Q.resize(njobs);
  for (int j = 0; j < njobs; j++) {
    const uint32_t n = 1 + rng() % maxs, m = rng() % (dens * n + 1), nl = 1 + rng() % labs;
    std::vector<uint32_t> s(m), d(m);
    std::vector<int32_t> lab(m);
    for (uint32_t k = 0; k < m; k++) {
      s[k] = rng() % n;
      d[k] = rng() % n;
      lab[k] = (int32_t)(rng() % nl);
    }
    Lts::from_edges(m, s.data(), d.data(), lab.data(), b.L[j], n);
    b.P[j] = rng() % b.L[j].n;
    b.Q[j] = rng() % b.L[j].n;
  }
  b.sb.assign(njobs + 1, 0);
  b.tb.assign(njobs + 1, 0);
  for (int j = 0; j < njobs; j++) {
    b.sb[j + 1] = b.sb[j] + b.L[j].n;
    b.tb[j + 1] = b.tb[j] + b.L[j].n_transitions();
  }
  const uint32_t NS = (uint32_t)b.sb[njobs], MS = (uint32_t)b.tb[njobs];
  b.soff.assign(NS + 1, 0);
  b.stgt.assign(MS, 0);
  b.sjob.assign(NS, 0);
  b.slab.assign(MS, 0);
  b.jsb.assign(njobs + 1, 0);
  for (int j = 0; j <= njobs; j++) b.jsb[j] = (uint32_t)b.sb[j];
  for (int j = 0; j < njobs; j++) {
    for (uint32_t s = 0; s < b.L[j].n; s++) {
      b.soff[b.sb[j] + s] = (uint32_t)(b.tb[j] + b.L[j].off[s]);
      b.sjob[b.sb[j] + s] = j;
    }
    for (uint64_t k = 0; k < b.L[j].n_transitions(); k++) {
      b.slab[b.tb[j] + k] = b.L[j].lab_[k];
      b.stgt[b.tb[j] + k] = (uint32_t)(b.sb[j] + b.L[j].tgt[k]);
    }
  }
  b.soff[NS] = MS;
}

static gb::Input input_of(const Batch &b, const std::vector<uint32_t> &sp, const std::vector<uint32_t> &sq) {
  gb::Input in;
  in.NS = (uint32_t)b.soff.size() - 1;
  in.MS = (uint32_t)b.stgt.size();
  in.n_jobs = (uint32_t)b.L.size();
  in.soff = b.soff.data();
  in.slab = b.slab.data();
  in.stgt = b.stgt.data();
  in.sjob = b.sjob.data();
  in.jsb = b.jsb.data();
  in.p0 = sp.data();
  in.q0 = sq.data();
  in.n_starts = (uint32_t)sp.size();
  return in;
}

static int run_build(int argc, char **argv) {
  const int njobs = atoi(argv[2]), maxs = atoi(argv[3]);
  const uint32_t maxpos = (uint32_t)atoi(argv[4]);
  const uint64_t seed = strtoull(argv[5], nullptr, 10);
  const int dens = atoi(argv[6]), labs = atoi(argv[7]);
  const uint32_t heavy_min = (uint32_t)strtoul(argv[8], nullptr, 10);
  const bool all = atoi(argv[9]) != 0;
  Batch b;
  make_batch(b, njobs, maxs, seed, dens, labs);
  std::vector<uint32_t> sp, sq;
  for (int j = 0; j < njobs; j++) {
    if (all) {
      std::vector<uint32_t> procs(b.L[j].n);
      for (uint32_t i = 0; i < b.L[j].n; i++) procs[i] = i;
      std::vector<std::pair<uint32_t, uint32_t>> pr;
      GameBuilder::start_pairs(b.L[j], procs.data(), b.L[j].n, pr);
      for (auto &x : pr) {
        sp.push_back((uint32_t)(b.sb[j] + x.first));
        sq.push_back((uint32_t)(b.sb[j] + x.second));
      }
    } else {
      sp.push_back((uint32_t)(b.sb[j] + b.P[j]));
      sq.push_back((uint32_t)(b.sb[j] + b.Q[j]));
    }
  }
  gb::Input in = input_of(b, sp, sq);
  in.max_pos = maxpos;
  in.heavy_min = heavy_min;
  HostBackend be;
  // a first build, then one that starts from its capacities (the hint path)
  gb::Builder<HostBackend> b0(be);
  gb::Result r0;
  if (b0.run(in, r0) != 0) {
    std::printf("first build failed\n");
    return 1;
  }
  gb::Builder<HostBackend> bb(be);
  bb.hint = b0.used;
  gb::Result r;
  if (bb.run(in, r) != 0) {
    std::printf("hinted build failed\n");
    return 1;
  }
  int bad = 0;
  uint64_t eb = 0;
  for (int j = 0; j < njobs; j++) {
    GameBuilder g;
    g.max_positions = maxpos;
    if (all) {
      GameBuilder::compare_all(b.L[j], g);
    } else {
      g.new_node(PosKey{POS_ATTACK, b.P[j], g.sets.intern(&b.Q[j], 1), 0});
      g.build(b.L[j]);
    }
    const bool over = r.jover[j] != 0;
    const uint32_t n = r.jcount[j];
    const uint32_t *row = r.row + r.jbase[j] + j;
    const uint32_t m = row[n];
    bool ok = over == g.truncated;
    if (ok && !over) {
      ok = n == g.nodes.size() && m == g.col.size();
      for (uint32_t i = 0; ok && i <= n; i++) ok = row[i] == g.row[i];
      for (uint32_t i = 0; ok && i < m; i++) ok = r.col[eb + i] == g.col[i] && r.wt[eb + i] == g.wt[i];
      for (uint32_t i = 0; ok && i < n; i++) ok = r.att[r.jbase[j] + i] == g.attacker[i];
    }
    if (!ok) bad++;
    eb += m;
  }
  if (bb.used.nodes > b0.used.nodes || bb.used.S > b0.used.S || bb.used.edges > b0.used.edges) {
    std::printf("capacities grew from the hint\n");
    bad++;
  }
  std::printf("bad %d of %d (%u positions, %u edges, %u levels)\n", bad, njobs, r.N, r.M, r.levels);
  return bad != 0;
}

static int run_refine(int argc, char **argv) {
  const int njobs = atoi(argv[2]), maxs = atoi(argv[3]);
  const uint64_t seed = strtoull(argv[4], nullptr, 10);
  const int dens = atoi(argv[5]), labs = atoi(argv[6]);
  Batch b;
  make_batch(b, njobs, maxs, seed, dens, labs);
  std::vector<uint32_t> sp(njobs), sq(njobs);
  for (int j = 0; j < njobs; j++) {
    sp[j] = (uint32_t)(b.sb[j] + b.P[j]);
    sq[j] = (uint32_t)(b.sb[j] + b.Q[j]);
  }
  gb::Input in = input_of(b, sp, sq);
  HostBackend be;
  rf::Refiner<HostBackend> R(be);
  if (R.run(in) != 0) {
    std::printf("refinement failed\n");
    return 1;
  }
  gb::Input out;
  uint32_t *rp0 = nullptr, *rq0 = nullptr;
  if (R.reduce(in, out, rp0, rq0) != 0) {
    std::printf("reduce failed\n");
    return 1;
  }
  int bad = 0;
  for (int j = 0; j < njobs; j++) {
    std::vector<uint64_t> part;
    const uint64_t c = b.L[j].signature_refinement(part);
    bool ok = c == R.counts()[j];
    for (uint32_t s = 0; ok && s < b.L[j].n; s++) ok = part[s] == R.partition()[b.sb[j] + s];
    std::vector<uint64_t> mp;
    Lts red;
    b.L[j].minimize(mp, red);
    const uint32_t cb = out.jsb[j];
    ok = ok && red.n == out.jsb[j + 1] - cb;
    for (uint32_t x = 0; ok && x < red.n; x++) {
      ok = (out.soff[cb + x + 1] - out.soff[cb + x]) == (red.off[x + 1] - red.off[x]) && out.sjob[cb + x] == (uint32_t)j;
      for (uint64_t k = red.off[x]; ok && k < red.off[x + 1]; k++) {
        const uint32_t o = out.soff[cb + x] + (uint32_t)(k - red.off[x]);
        ok = out.slab[o] == red.lab_[k] && out.stgt[o] == cb + red.tgt[k];
      }
    }
    ok = ok && rp0[j] == cb + mp[b.P[j]] && rq0[j] == cb + mp[b.Q[j]];
    if (!ok) bad++;
  }
  std::printf("bad %d of %d (%u iterations)\n", bad, njobs, R.iterations);
  return bad != 0;
}

int main(int argc, char **argv) {
  if (argc >= 10 && !std::strcmp(argv[1], "build")) return run_build(argc, argv);
  if (argc >= 7 && !std::strcmp(argv[1], "refine")) return run_refine(argc, argv);
  std::fprintf(stderr, "usage: see the file header\n");
  return 2;
}
