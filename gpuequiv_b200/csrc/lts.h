// lts.h - labelled transition system in CSR form (src/lib.rs TransitionSystem).
#pragma once
#include <cstdint>
#include <vector>

#include "geq_internal.h"

namespace geq {

struct Lts {
  uint32_t n = 0;
  std::vector<uint64_t> off;  // n + 1
  std::vector<uint32_t> tgt;  // target process of each transition
  std::vector<int32_t> lab_;  // label of each transition (rows sorted by label)

  static geq_status from_edges(uint64_t m, const uint32_t *src, const uint32_t *dst, const int32_t *label,
                               Lts &out, uint32_t min_vertices = 0);
  static geq_status from_csv_file(const char *path, Lts &out);
  uint64_t signature_refinement(std::vector<uint64_t> &part) const;
  void minimize(std::vector<uint64_t> &mapping, Lts &out) const;
  uint64_t n_transitions() const { return tgt.size(); }

 private:
  void finish_from_buckets(uint32_t nv, const std::vector<uint32_t> &src, const std::vector<uint32_t> &dst,
                           const std::vector<int32_t> &lab);
};

}  // namespace geq

struct geq_lts {
  geq::Lts l;
};
