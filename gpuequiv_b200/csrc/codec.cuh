// codec.cuh - device arithmetic on energies.
//
// Energies cross the C ABI in the crate's packed layout (src/energy.rs:
// 143-179): element i in bits [i*b, i*b+b) of one u32.  Inside the kernels
// an energy is held as a thermometer code, in which the operations the
// shaders spell out field by field become single bitwise instructions:
//   a <= b field-wise     (shadergen.rs:55-73  IMPL_LESS_EQ)   <=>  (a & ~b) == 0
//   max(a, b) field-wise  (shadergen.rs:151-157 MAX_SUPREMUM)  <=>  a | b
//   inverse update        (shadergen.rs:103-128 UPDATE1 / UPDATE_MIN,
//                          attack_update.wgsl:45-61)          <=>  a few shifts/ORs
// The code of value v in 0..max is the v lowest bits of a max-bit field.
//
// CodecStd is specialised for EnergyConf::STANDARD = {6, 3} (the conf
// GameBuild uses, gamebuild.rs:152).  Its 24-bit code keeps the three
// thermometer bits of field i in "bit planes": bit 2i = (v >= 1),
// bit 2i+1 = (v >= 2), bit 12+2i = (v == 3).  Conversion from and to the
// packed 12-bit word is then a handful of mask operations.
//
// CodecGen handles every other conf whose energy and update fit one word and
// whose code fits 32 bits (elements * max <= 32); field i occupies bits
// [i*max, (i+1)*max).
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace geq {

struct CodecStd {
  static constexpr bool kBitmap = true;
  __host__ __device__ __forceinline__ uint32_t to_t(uint32_t p) const {
    uint32_t lo = p & 0x555u, hi = (p >> 1) & 0x555u;
    return (lo | hi) | (p & 0xAAAu) | ((lo & hi) << 12);
  }
  __host__ __device__ __forceinline__ uint32_t to_p(uint32_t t) const {
    uint32_t p0 = t & 0x555u, p1 = (t >> 1) & 0x555u, p2 = (t >> 12) & 0x555u;
    return (p0 ^ p1 ^ p2) | (p1 << 1);
  }
  // Inverse of the edge update u (4-bit codes: 0 Zero, 1 Decrement, k+2 =
  // Min into element k): all decrements first, then the merges in index
  // order, exactly as UPDATE1 followed by UPDATE_MIN.  An update is decoded
  // once per edge (prep) and applied to each energy of the successor's list
  // (apply): `lod` = plane-0 bits of the decremented fields, `mg` = the
  // merges as (2*source, 2*target) nibble pairs in index order.
  struct Upd {
    uint32_t lod, nm;
    unsigned long long mg;
  };
  __host__ __device__ __forceinline__ Upd prep(uint32_t u) const {
    Upd q{0u, 0u, 0ull};
    // fields whose code is 1: bit 4i of z, then moved to bit 2i
    const uint32_t x = u ^ 0x111111u;
    uint32_t z = ~(x | (x >> 1) | (x >> 2) | (x >> 3)) & 0x111111u;
    z = (z & ~0x101010u) | ((z & 0x101010u) >> 2);
    z = (z & ~0x000500u) | ((z & 0x000500u) >> 4);
    z = (z & ~0x050000u) | ((z & 0x050000u) >> 8);
    q.lod = z;
    // fields whose code is >= 2
    uint32_t m = ((u >> 1) | (u >> 2) | (u >> 3)) & 0x111111u;
    while (m) {
#ifdef __CUDA_ARCH__
      const uint32_t b = (uint32_t)__ffs((int)m) - 1u;
#else
      const uint32_t b = (uint32_t)__builtin_ctz(m);
#endif
      m &= m - 1u;
      const uint32_t i = b >> 2, tg = ((u >> b) & 15u) - 2u;
      if (tg < 6u) {
        q.mg |= (unsigned long long)((2u * i) | ((2u * tg) << 4)) << (8u * q.nm);
        q.nm++;
      }
    }
    return q;
  }
  __host__ __device__ __forceinline__ uint32_t apply(uint32_t t, const Upd &q) const {
    // v -> min(v+1, 3): plane 0 becomes 1, plane 1 takes plane 0, plane 2 takes plane 1.
    t = t | q.lod | ((t & q.lod) << 1) | ((t & (q.lod << 1)) << 11);
    for (uint32_t k = 0; k < q.nm; k++) {
      const uint32_t e = (uint32_t)(q.mg >> (8u * k));
      t |= ((t >> (e & 15u)) & 0x1003u) << ((e >> 4) & 15u);
    }
    return t;
  }
  __host__ __device__ __forceinline__ uint32_t upd(uint32_t t, uint32_t u) const { return apply(t, prep(u)); }
  // An edge's update as the round kernel reads it from its edge pairs: the
  // decoded form when the update has at most two merges (bits 0-11 `lod`,
  // 12-13 the merge count, 14-29 the merges), else the raw word with bit 31
  // set (decoded when read).  Every update GameBuild emits has at most one
  // merge.
  __host__ __device__ static uint32_t pack_edge(uint32_t u) {
    const Upd q = CodecStd{}.prep(u);
    if (q.nm > 2u) return 0x80000000u | u;
    return q.lod | (q.nm << 12) | ((uint32_t)q.mg << 14);
  }
  __host__ __device__ __forceinline__ Upd unpack_edge(uint32_t pw) const {
    if (pw >> 31) return prep(pw & 0x7FFFFFFFu);
    return Upd{pw & 0xFFFu, (pw >> 12) & 3u, (unsigned long long)((pw >> 14) & 0xFFFFu)};
  }
};

struct CodecGen {
  static constexpr bool kBitmap = false;
  uint32_t el, mx, eb, em, ub, um, fm;
  __host__ __device__ CodecGen(uint32_t elements, uint32_t max, uint32_t ebits, uint32_t emask,
                               uint32_t ubits, uint32_t umask)
      : el(elements), mx(max), eb(ebits), em(emask), ub(ubits), um(umask),
        fm((uint32_t)((1ull << max) - 1ull)) {}
  __host__ __device__ __forceinline__ uint32_t to_t(uint32_t p) const {
    uint32_t t = 0;
    for (uint32_t i = 0; i < el; i++) {
      uint32_t v = (p >> (i * eb)) & em;
      v = v < mx ? v : mx;  // inv_update clamps with min(., max)
      t |= (uint32_t)((1ull << v) - 1ull) << (i * mx);
    }
    return t;
  }
  __host__ __device__ __forceinline__ uint32_t to_p(uint32_t t) const {
    uint32_t p = 0;
    for (uint32_t i = 0; i < el; i++) {
      uint32_t f = (t >> (i * mx)) & fm;
#ifdef __CUDA_ARCH__
      uint32_t v = (uint32_t)__popc(f);
#else
      uint32_t v = (uint32_t)__builtin_popcount(f);
#endif
      p |= v << (i * eb);
    }
    return p;
  }
  using Upd = uint32_t;
  __host__ __device__ __forceinline__ Upd prep(uint32_t u) const { return u; }
  __host__ __device__ static uint32_t pack_edge(uint32_t u) { return u; }
  __host__ __device__ __forceinline__ Upd unpack_edge(uint32_t pw) const { return pw; }
  __host__ __device__ __forceinline__ uint32_t apply(uint32_t t, Upd u) const { return upd(t, u); }
  __host__ __device__ __forceinline__ uint32_t upd(uint32_t t, uint32_t u) const {
    if (u == 0) return t;
    for (uint32_t i = 0; i < el; i++) {
      if (((u >> (i * ub)) & um) == 1u) {
        uint32_t f = (t >> (i * mx)) & fm;
        f = ((f << 1) | 1u) & fm;
        t = (t & ~(fm << (i * mx))) | (f << (i * mx));
      }
    }
    for (uint32_t i = 0; i < el; i++) {
      uint32_t c = (u >> (i * ub)) & um;
      if (c >= 2u) {
        uint32_t tg = c - 2u;
        if (tg < el) t |= ((t >> (i * mx)) & fm) << (tg * mx);
      }
    }
    return t;
  }
};

__host__ __device__ __forceinline__ bool t_leq(uint32_t a, uint32_t b) { return (a & ~b) == 0u; }

}  // namespace geq
