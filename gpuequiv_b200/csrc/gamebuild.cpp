// gamebuild.cpp - the spectroscopy energy game of Bisping (2023) as built by
// GameBuild (src/gamebuild.rs:229-265) with the successor rules of
// src/gamebuild/gamepos.rs.  Positions are discovered breadth-first from the
// start positions and numbered in discovery order, so GameBuild::compare
// yields exactly the reference's node numbering and adjacency order.
#include "gamebuild.h"

#include <algorithm>
#include <unordered_map>

namespace geq {

static inline uint64_t mix64(uint64_t h) {
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  h *= 0xc4ceb9fe1a85ec53ull;
  h ^= h >> 33;
  return h;
}

SetPool::SetPool() {
  table.assign(1024, 0);
  intern(nullptr, 0);  // id 0: the empty set
}

void SetPool::grow() {
  std::vector<uint32_t> t(table.size() * 2, 0);
  const size_t mask = t.size() - 1;
  for (uint32_t id = 0; id < len.size(); id++) {
    size_t s = (size_t)hash[id] & mask;
    while (t[s]) s = (s + 1) & mask;
    t[s] = id + 1;
  }
  table.swap(t);
}

uint32_t SetPool::intern(const uint32_t *v, uint32_t n) {
  uint64_t h = 0x51ed270b27a3f1d7ull ^ n;
  for (uint32_t i = 0; i < n; i++) h = mix64(h ^ (v[i] + 0x9e3779b97f4a7c15ull));
  const size_t mask = table.size() - 1;
  size_t s = (size_t)h & mask;
  while (uint32_t t = table[s]) {
    uint32_t id = t - 1;
    if (hash[id] == h && len[id] == n && std::equal(v, v + n, data.data() + start[id])) return id;
    s = (s + 1) & mask;
  }
  uint32_t id = (uint32_t)len.size();
  start.push_back(data.size());
  len.push_back(n);
  hash.push_back(h);
  data.insert(data.end(), v, v + n);
  table[s] = id + 1;
  if (2 * len.size() > table.size()) grow();
  return id;
}

size_t GameBuilder::slot_of(const PosKey &k) const {
  uint64_t h = mix64(((uint64_t)k.kind << 32 | k.p) ^ mix64((uint64_t)k.a << 32 | k.b));
  return (size_t)h & (table.size() - 1);
}

void GameBuilder::grow() {
  std::vector<uint32_t> t(std::max<size_t>(table.size() * 2, 1024), 0);
  table.swap(t);
  const size_t mask = table.size() - 1;
  for (uint32_t id = 0; id < nodes.size(); id++) {
    size_t s = slot_of(nodes[id]);
    while (table[s]) s = (s + 1) & mask;
    table[s] = id + 1;
  }
}

// GameBuild::new_node (gamebuild.rs:255-265)
uint32_t GameBuilder::new_node(const PosKey &k) {
  if (2 * (nodes.size() + 1) > table.size()) grow();
  uint32_t id = (uint32_t)nodes.size();
  nodes.push_back(k);
  attacker.push_back(k.kind != POS_DEFEND);  // Position::is_attack (gamepos.rs:239-241)
  size_t s = slot_of(k);
  const size_t mask = table.size() - 1;
  while (table[s]) s = (s + 1) & mask;
  table[s] = id + 1;
  return id;
}

// node_map lookup or new_node (gamebuild.rs:247-248)
uint32_t GameBuilder::node_for(const PosKey &k) {
  if (table.empty()) grow();
  const size_t mask = table.size() - 1;
  size_t s = slot_of(k);
  while (uint32_t t = table[s]) {
    if (nodes[t - 1] == k) return t - 1;
    s = (s + 1) & mask;
  }
  return new_node(k);
}

namespace {

// Packed STANDARD updates used by the game (gamepos.rs:21-22, :145-146, :183-184).
struct Weights {
  uint32_t obs, chal, rev, ans, cl1, cl2;
  Weights() {
    auto code = [](int dim, uint32_t c) { return c << (4 * dim); };
    obs = code(0, 1);                   // [-1]
    chal = code(1, 1);                  // [0, -1]
    rev = code(0, 3 + 1);               // [Min(3)]
    ans = code(3, 3 + 1);               // [0, 0, 0, Min(3)]
    cl1 = code(0, 4 + 1);               // [Min(4)]
    cl2 = code(0, 5 + 1) | code(5, 1);  // [Min(5), 0, 0, 0, 0, -1]
  }
};

// TransitionSystem::compare_enabled (gamebuild.rs:23-98)
std::pair<bool, bool> compare_enabled(const Lts &l, uint32_t p, uint32_t q) {
  if (p == q) return {true, true};
  bool subset = true, superset = true;
  uint64_t pp = l.off[p], pm = l.off[p + 1], qp = l.off[q], qm = l.off[q + 1];
  for (;;) {
    if (!(subset || superset)) break;
    if (pp == pm && qp == qm) break;
    if (pp == pm) { subset = false; break; }
    if (qp == qm) { superset = false; break; }
    int32_t pa = l.lab_[pp], qa = l.lab_[qp];
    bool ap = false, aq = false;
    if (pa == qa) { ap = aq = true; }
    else if (pa < qa) { superset = false; ap = true; }
    else { subset = false; aq = true; }
    if (ap) { pp++; while (pp < pm && l.lab_[pp] == pa) pp++; }
    if (aq) { qp++; while (qp < qm && l.lab_[qp] == qa) qp++; }
  }
  return {subset, superset};
}

// First index of label `a` in the label-sorted row of q.
inline uint64_t label_lower(const Lts &l, uint32_t q, int32_t a) {
  uint64_t lo = l.off[q], hi = l.off[q + 1];
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (l.lab_[mid] < a) lo = mid + 1; else hi = mid;
  }
  return lo;
}

}  // namespace

void GameBuilder::build(const Lts &l) {
  static const Weights W;
  n_starting = (uint32_t)nodes.size();
  std::vector<PosKey> succ;
  std::vector<uint32_t> sw, qbuf, q_sub, qx_sub, q_sup, qx_sup, q_eq, qx_eq;
  row.clear();
  col.clear();
  wt.clear();
  for (size_t idx = 0; idx < nodes.size(); idx++) {
    if (max_positions && nodes.size() > max_positions) {
      truncated = true;
      break;
    }
    const PosKey x = nodes[idx];
    succ.clear();
    sw.clear();
    if (x.kind == POS_ATTACK) {  // AttackPosition::successors (gamepos.rs:17-106)
      const uint32_t nq = sets.size(x.a);
      if (nq == 0) {
        succ.push_back(PosKey{POS_DEFEND, x.p, 0, 0});
        sw.push_back(W.chal);
      } else {
        // observation moves; Q' depends only on the label, so it is computed
        // once per run of equal labels
        uint64_t k = l.off[x.p];
        const uint64_t ke = l.off[x.p + 1];
        while (k < ke) {
          const int32_t a = l.lab_[k];
          uint64_t run_end = k;
          while (run_end < ke && l.lab_[run_end] == a) run_end++;
          qbuf.clear();
          const uint32_t *Q = sets.ptr(x.a);
          for (uint32_t i = 0; i < nq; i++) {
            const uint32_t q = Q[i];
            for (uint64_t t = label_lower(l, q, a); t < l.off[q + 1] && l.lab_[t] == a; t++) qbuf.push_back(l.tgt[t]);
          }
          std::sort(qbuf.begin(), qbuf.end());
          qbuf.erase(std::unique(qbuf.begin(), qbuf.end()), qbuf.end());
          const uint32_t qid = sets.intern(qbuf.data(), (uint32_t)qbuf.size());
          for (; k < run_end; k++) {
            const uint32_t p2 = l.tgt[k];
            if (!std::binary_search(qbuf.begin(), qbuf.end(), p2)) {
              succ.push_back(PosKey{POS_ATTACK, p2, qid, 0});
              sw.push_back(W.obs);
            }
          }
        }
        // conjunction challenges
        const size_t cs = succ.size();
        succ.push_back(PosKey{POS_DEFEND, x.p, x.a, 0});
        q_sub.clear(); qx_sub.clear(); q_sup.clear(); qx_sup.clear(); q_eq.clear(); qx_eq.clear();
        const uint32_t *Q = sets.ptr(x.a);
        for (uint32_t i = 0; i < nq; i++) {
          const uint32_t q = Q[i];
          auto se = compare_enabled(l, x.p, q);
          (se.first ? qx_sub : q_sub).push_back(q);
          (se.second ? qx_sup : q_sup).push_back(q);
          ((se.first && se.second) ? qx_eq : q_eq).push_back(q);
        }
        auto push_unique = [&](const std::vector<uint32_t> &qs, const std::vector<uint32_t> &qxs, bool check) {
          PosKey c{POS_DEFEND, x.p, sets.intern(qs.data(), (uint32_t)qs.size()),
                   sets.intern(qxs.data(), (uint32_t)qxs.size())};
          if (check)
            for (size_t i = cs + 1; i < succ.size(); i++)
              if (succ[i] == c) return;
          succ.push_back(c);
        };
        if (!qx_sub.empty() && !q_sub.empty()) push_unique(q_sub, qx_sub, false);
        if (!qx_sup.empty() && !q_sup.empty()) push_unique(q_sup, qx_sup, true);
        if (!qx_eq.empty() && !q_eq.empty()) push_unique(q_eq, qx_eq, true);
        for (size_t i = cs; i < succ.size(); i++) sw.push_back(W.chal);
      }
    } else if (x.kind == POS_CLAUSE) {  // SingletonPosition::successors (gamepos.rs:139-158)
      const uint32_t qs = x.a, ps = x.p;
      succ.push_back(PosKey{POS_ATTACK, x.p, sets.intern(&qs, 1), 0});
      succ.push_back(PosKey{POS_ATTACK, x.a, sets.intern(&ps, 1), 0});
      sw.push_back(W.cl1);
      sw.push_back(W.cl2);
    } else {  // DefendPosition::successors (gamepos.rs:179-198)
      const uint32_t nq = sets.size(x.a);
      const uint32_t *Q = sets.ptr(x.a);
      for (uint32_t i = 0; i < nq; i++) {
        succ.push_back(PosKey{POS_CLAUSE, x.p, Q[i], 0});
        sw.push_back(W.ans);
      }
      if (sets.size(x.b) != 0) {
        succ.push_back(PosKey{POS_ATTACK, x.p, x.b, 0});
        sw.push_back(W.rev);
      }
    }
    row.push_back((uint32_t)col.size());
    for (size_t i = 0; i < succ.size(); i++) col.push_back(node_for(succ[i]));
    wt.insert(wt.end(), sw.begin(), sw.end());
  }
  row.push_back((uint32_t)col.size());
}

// GameBuild::compare (gamebuild.rs:165-170)
void GameBuilder::compare(const Lts &l, uint32_t p, uint32_t q, GameBuilder &out) {
  out.new_node(PosKey{POS_ATTACK, p, out.sets.intern(&q, 1), 0});
  out.build(l);
}

// Start pairs for every ordered pair inside each enabledness class
// (gamebuild.rs:104-133, :176-215).  Classes are visited in order of their
// first process.
void GameBuilder::start_pairs(const Lts &l, const uint32_t *procs, uint32_t n,
                              std::vector<std::pair<uint32_t, uint32_t>> &out) {
  std::unordered_map<uint32_t, uint32_t> class_of_set;  // label-set id -> class index
  SetPool labelsets;
  std::vector<std::vector<uint32_t>> classes;
  std::vector<uint32_t> en;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t p = procs[i];
    en.clear();
    for (uint64_t k = l.off[p]; k < l.off[p + 1]; k++) {
      uint32_t a = (uint32_t)l.lab_[k];
      if (en.empty() || en.back() != a) en.push_back(a);  // rows are label-sorted
    }
    const uint32_t sid = labelsets.intern(en.data(), (uint32_t)en.size());
    auto it = class_of_set.find(sid);
    if (it == class_of_set.end()) {
      class_of_set.emplace(sid, (uint32_t)classes.size());
      classes.push_back({p});
    } else {
      classes[it->second].push_back(p);
    }
  }
  out.clear();
  for (auto &c : classes)
    for (uint32_t p : c)
      for (uint32_t q : c)
        if (p != q) out.emplace_back(p, q);
}

void GameBuilder::compare_processes(const Lts &l, const uint32_t *procs, uint32_t n, GameBuilder &out) {
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  start_pairs(l, procs, n, pairs);
  for (auto &pq : pairs) out.new_node(PosKey{POS_ATTACK, pq.first, out.sets.intern(&pq.second, 1), 0});
  out.build(l);
}

void GameBuilder::compare_all(const Lts &l, GameBuilder &out) {
  std::vector<uint32_t> all(l.n);
  for (uint32_t p = 0; p < l.n; p++) all[p] = p;
  compare_processes(l, all.data(), l.n, out);
}

}  // namespace geq
