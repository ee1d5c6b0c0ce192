// gamebuild.h - spectroscopy game construction (src/gamebuild.rs,
// src/gamebuild/gamepos.rs) emitting the CSR game graph directly.
#pragma once
#include <cstdint>
#include <vector>

#include "geq_internal.h"
#include "lts.h"

namespace geq {

// Interned, sorted process sets; id 0 is the empty set.
struct SetPool {
  std::vector<uint32_t> data;
  std::vector<uint64_t> start;
  std::vector<uint32_t> len;
  std::vector<uint64_t> hash;
  std::vector<uint32_t> table;  // id + 1, 0 = free
  SetPool();
  uint32_t intern(const uint32_t *v, uint32_t n);
  const uint32_t *ptr(uint32_t id) const { return data.data() + start[id]; }
  uint32_t size(uint32_t id) const { return len[id]; }

 private:
  void grow();
};

enum : uint32_t { POS_ATTACK = 0, POS_CLAUSE = 1, POS_DEFEND = 2 };
// Attack(p, Q): a = id(Q), b = 0.  Clause(p, q): a = q, b = 0.
// Defend(p, Q, Q*): a = id(Q), b = id(Q*).
struct PosKey {
  uint32_t kind, p, a, b;
  bool operator==(const PosKey &o) const { return kind == o.kind && p == o.p && a == o.a && b == o.b; }
};

struct GameBuilder {
  SetPool sets;
  std::vector<PosKey> nodes;
  std::vector<uint32_t> table;  // node id + 1, 0 = free
  uint32_t n_starting = 0;
  uint64_t max_positions = 0;  // 0 = unbounded; build() stops once exceeded
  bool truncated = false;
  std::vector<uint32_t> row, col, wt;
  std::vector<uint8_t> attacker;

  uint32_t new_node(const PosKey &k);
  uint32_t node_for(const PosKey &k);
  void build(const Lts &l);
  static void compare(const Lts &l, uint32_t p, uint32_t q, GameBuilder &out);
  static void compare_all(const Lts &l, GameBuilder &out);
  static void compare_processes(const Lts &l, const uint32_t *procs, uint32_t n, GameBuilder &out);
  static void start_pairs(const Lts &l, const uint32_t *procs, uint32_t n,
                          std::vector<std::pair<uint32_t, uint32_t>> &out);

 private:
  void grow();
  size_t slot_of(const PosKey &k) const;
};

}  // namespace geq

struct geq_game_build {
  geq::GameBuilder b;
};
