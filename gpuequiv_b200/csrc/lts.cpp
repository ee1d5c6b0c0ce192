// lts.cpp - TransitionSystem for the product library (src/lib.rs).
//
// The LTS is held in CSR form with every adjacency list sorted by label
// (stable, TransitionSystem::sort_labels, lib.rs:489-493), which is the
// order GameBuild iterates transitions in.
#include "lts.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>

namespace geq {

void Lts::finish_from_buckets(uint32_t nv, const std::vector<uint32_t> &src, const std::vector<uint32_t> &dst,
                              const std::vector<int32_t> &lab) {
  n = nv;
  const size_t m = src.size();
  off.assign((size_t)n + 1, 0);
  for (size_t i = 0; i < m; i++) off[src[i] + 1]++;
  for (uint32_t p = 0; p < n; p++) off[p + 1] += off[p];
  tgt.assign(m, 0);
  lab_.assign(m, 0);
  std::vector<uint64_t> fill(off.begin(), off.end() - 1);
  for (size_t i = 0; i < m; i++) {  // edge order is kept within a source
    uint64_t k = fill[src[i]]++;
    tgt[k] = dst[i];
    lab_[k] = lab[i];
  }
  // stable sort of every row by label
  std::vector<std::pair<int32_t, uint32_t>> tmp;
  for (uint32_t p = 0; p < n; p++) {
    uint64_t b = off[p], e = off[p + 1];
    if (e - b < 2) continue;
    bool sorted = true;
    for (uint64_t k = b + 1; k < e; k++)
      if (lab_[k] < lab_[k - 1]) { sorted = false; break; }
    if (sorted) continue;
    tmp.clear();
    for (uint64_t k = b; k < e; k++) tmp.emplace_back(lab_[k], tgt[k]);
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<int32_t, uint32_t> &a, const std::pair<int32_t, uint32_t> &c) { return a.first < c.first; });
    for (uint64_t k = b; k < e; k++) { lab_[k] = tmp[k - b].first; tgt[k] = tmp[k - b].second; }
  }
}

// FromIterator<Edge> (lib.rs:523-536): the vertex count is one more than the
// largest id mentioned by any edge.
geq_status Lts::from_edges(uint64_t m, const uint32_t *src, const uint32_t *dst, const int32_t *label, Lts &out,
                           uint32_t min_vertices) {
  uint64_t nv = min_vertices;
  for (uint64_t i = 0; i < m; i++) nv = std::max<uint64_t>(nv, (uint64_t)std::max(src[i], dst[i]) + 1);
  if (nv > 0xFFFFFFF0ull) return fail(GEQ_ERR_INVALID_INPUT, "process id too large");
  std::vector<uint32_t> s(src, src + m), d(dst, dst + m);
  std::vector<int32_t> l(label, label + m);
  out.finish_from_buckets((uint32_t)nv, s, d, l);
  return GEQ_OK;
}

// TransitionSystem::from_csv_lines (lib.rs:372-406).  Label "i" is 0 (tau);
// other labels are numbered 1, 2, ... in order of first appearance.
geq_status Lts::from_csv_file(const char *path, Lts &out) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(GEQ_ERR_IO, "cannot open %s", path);
  std::string buf;
  {
    char chunk[1 << 16];
    size_t r;
    while ((r = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.append(chunk, r);
    std::fclose(f);
  }
  std::unordered_map<std::string, int32_t> labels;
  labels.emplace("i", 0);
  int32_t max_label = 0;
  std::vector<uint32_t> src, dst;
  std::vector<int32_t> lab;
  uint64_t nv = 0;
  size_t pos = 0, line_no = 0;
  auto parse_uint = [](const char *b, const char *e, uint64_t lim, uint64_t &v) {
    if (b < e && *b == '+') b++;
    if (b >= e) return false;
    v = 0;
    for (; b < e; b++) {
      if (*b < '0' || *b > '9') return false;
      v = v * 10 + (uint64_t)(*b - '0');
      if (v > lim) return false;
    }
    return true;
  };
  while (pos < buf.size()) {
    size_t eol = buf.find('\n', pos);
    if (eol == std::string::npos) eol = buf.size();
    size_t end = eol;
    if (end > pos && buf[end - 1] == '\r') end--;
    line_no++;
    const char *b = buf.data() + pos, *e = buf.data() + end;
    const char *c1 = (const char *)std::memchr(b, ',', (size_t)(e - b));
    if (!c1) return fail(GEQ_ERR_PARSE, "line %zu: missing field", line_no);
    const char *c2 = (const char *)std::memchr(c1 + 1, ',', (size_t)(e - c1 - 1));
    if (!c2) return fail(GEQ_ERR_PARSE, "line %zu: missing field", line_no);
    uint64_t from, to;
    if (!parse_uint(b, c1, 0xFFFFFFEFull, from) || !parse_uint(c1 + 1, c2, 0xFFFFFFEFull, to))
      return fail(GEQ_ERR_PARSE, "line %zu: invalid process id", line_no);
    std::string label(c2 + 1, e);
    if (label.size() >= 2 && label.front() == '"' && label.back() == '"') label = label.substr(1, label.size() - 2);
    auto it = labels.find(label);
    int32_t ln;
    if (it != labels.end()) ln = it->second;
    else { ln = ++max_label; labels.emplace(std::move(label), ln); }
    src.push_back((uint32_t)from);
    dst.push_back((uint32_t)to);
    lab.push_back(ln);
    nv = std::max<uint64_t>(nv, std::max(from, to) + 1);
    pos = eol + 1;
  }
  out.finish_from_buckets((uint32_t)nv, src, dst, lab);
  return GEQ_OK;
}

namespace {
struct SigKey {
  uint64_t h;
  uint32_t start, len;
};
}  // namespace

// signatures + signature_refinement (lib.rs:444-478): partition ids are
// handed out in process order of each signature's first occurrence.
uint64_t Lts::signature_refinement(std::vector<uint64_t> &part) const {
  part.assign(n, 0);
  uint64_t prev = 0, cur = 1;
  std::vector<uint64_t> sig;  // (label << 32 | class) pairs, flat
  std::vector<uint32_t> sstart((size_t)n + 1);
  std::vector<uint64_t> newpart(n);
  std::vector<int64_t> table;
  std::vector<SigKey> keys;
  while (prev != cur) {
    prev = cur;
    sig.clear();
    for (uint32_t p = 0; p < n; p++) {
      sstart[p] = (uint32_t)sig.size();
      size_t b = sig.size();
      for (uint64_t k = off[p]; k < off[p + 1]; k++)
        sig.push_back(((uint64_t)(uint32_t)(lab_[k] ^ 0x80000000) << 32) | (uint64_t)part[tgt[k]]);
      std::sort(sig.begin() + b, sig.end());
      sig.erase(std::unique(sig.begin() + b, sig.end()), sig.end());
    }
    sstart[n] = (uint32_t)sig.size();
    size_t cap = 1;
    while (cap < 2 * (size_t)n + 2) cap <<= 1;
    table.assign(cap, -1);
    keys.clear();
    cur = 0;
    for (uint32_t p = 0; p < n; p++) {
      uint32_t b = sstart[p], len = sstart[p + 1] - b;
      uint64_t h = 0x9e3779b97f4a7c15ull ^ len;
      for (uint32_t i = 0; i < len; i++) {
        h ^= sig[b + i] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        h *= 0xff51afd7ed558ccdull;
      }
      size_t slot = (size_t)(h ^ (h >> 29)) & (cap - 1);
      for (;;) {
        int64_t t = table[slot];
        if (t < 0) {
          table[slot] = (int64_t)keys.size();
          keys.push_back(SigKey{h, b, len});
          newpart[p] = cur++;
          break;
        }
        const SigKey &k = keys[(size_t)t];
        if (k.h == h && k.len == len && std::equal(sig.begin() + k.start, sig.begin() + k.start + len, sig.begin() + b)) {
          newpart[p] = (uint64_t)t;
          break;
        }
        slot = (slot + 1) & (cap - 1);
      }
    }
    part.swap(newpart);
  }
  return cur;
}

// bisimilar_minimize (lib.rs:413-432): the first process of each class
// represents it; its transitions are redirected to the classes.
void Lts::minimize(std::vector<uint64_t> &mapping, Lts &out) const {
  uint64_t count = signature_refinement(mapping);
  std::vector<int64_t> rep(count, -1);
  for (uint32_t p = 0; p < n; p++)
    if (rep[mapping[p]] < 0) rep[mapping[p]] = p;
  out.n = (uint32_t)count;
  out.off.assign(count + 1, 0);
  for (uint64_t c = 0; c < count; c++) {
    uint32_t p = (uint32_t)rep[c];
    out.off[c + 1] = out.off[c] + (off[p + 1] - off[p]);
  }
  out.tgt.resize(out.off[count]);
  out.lab_.resize(out.off[count]);
  for (uint64_t c = 0; c < count; c++) {
    uint32_t p = (uint32_t)rep[c];
    uint64_t o = out.off[c];
    for (uint64_t k = off[p]; k < off[p + 1]; k++, o++) {
      out.tgt[o] = (uint32_t)mapping[tgt[k]];
      out.lab_[o] = lab_[k];
    }
  }
}

}  // namespace geq
