// wide_arith.cuh - energy arithmetic of the multi-word solver (wide.cu) on
// the crate's packed layout, for any EnergyConf: the operations the shader
// preprocessor generates per conf (src/energygame/shadergen.rs:55-157).
// Host and device: the CPU tests run the same functions.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace geq {

// field widths of a conf (energy_bits and update_bits are powers of two, so
// no field straddles a word)
struct WideConf {
  uint32_t el, mx, eb, em, ub, um;
};

__host__ __device__ __forceinline__ uint32_t getf(const uint32_t *x, uint32_t i, uint32_t b, uint32_t m) {
  const uint32_t bit = i * b;
  return (x[bit >> 5] >> (bit & 31u)) & m;
}
__host__ __device__ __forceinline__ void setf(uint32_t *x, uint32_t i, uint32_t b, uint32_t m, uint32_t v) {
  const uint32_t bit = i * b, w = bit >> 5, s = bit & 31u;
  x[w] = (x[w] & ~(m << s)) | ((v & m) << s);
}

// Field-wise compare and max of one word by SWAR arithmetic: fields of k <= 16
// bits are split into even and odd fields, each in a 2k-bit slot whose bit k
// is a guard; (b | G) - a keeps the guard of a slot iff its b field >= its a
// field, with no borrow between slots.  32-bit fields compare directly.
struct Swar {
  uint32_t k, fm, g;  // field bits, even-field mask, guard bits
};
__host__ __device__ inline Swar make_swar(uint32_t k) {
  Swar s{k, 0u, 0u};
  if (k >= 32) return s;
  for (uint32_t slot = 0; slot < 32; slot += 2 * k) {
    s.fm |= ((1u << k) - 1u) << slot;
    s.g |= 1u << (slot + k);
  }
  return s;
}
// a <= b in every field (IMPL_LESS_EQ, shadergen.rs:55-73)
__host__ __device__ __forceinline__ bool swar_leq(uint32_t a, uint32_t b, const Swar &s) {
  if (s.k == 32u) return a <= b;
  const uint32_t ae = a & s.fm, be = b & s.fm, ao = (a >> s.k) & s.fm, bo = (b >> s.k) & s.fm;
  return ((((be | s.g) - ae) & s.g) == s.g) && ((((bo | s.g) - ao) & s.g) == s.g);
}
// field-wise max (MAX_SUPREMUM, shadergen.rs:151-157)
__host__ __device__ __forceinline__ uint32_t swar_max(uint32_t a, uint32_t b, const Swar &s) {
  if (s.k == 32u) return a > b ? a : b;
  const uint32_t f = (1u << s.k) - 1u;
  const uint32_t ae = a & s.fm, be = b & s.fm, ao = (a >> s.k) & s.fm, bo = (b >> s.k) & s.fm;
  const uint32_t me = ((((be | s.g) - ae) & s.g) >> s.k) * f;  // fields where b >= a
  const uint32_t mo = ((((bo | s.g) - ao) & s.g) >> s.k) * f;
  return ((be & me) | (ae & ~me)) | (((bo & mo) | (ao & ~mo)) << s.k);
}

// Inverse update of one energy in place (UPDATE1 then UPDATE_MIN,
// shadergen.rs:103-128, as inv_update in attack_update.wgsl:45-61): every
// field +1 in u32 arithmetic where the code is 1 (Decrement), then min with
// max; then, in index order, a field with code k+2 (Min into k) raises field
// k to its value.  u = the update words, null for the zero update (the
// clamp alone, applied to an attacker's own energies).
__host__ __device__ inline void wide_inv_update(const WideConf &c, uint32_t *x, const uint32_t *u) {
  for (uint32_t i = 0; i < c.el; i++) {
    const uint32_t code = u ? getf(u, i, c.ub, c.um) : 0u;
    const uint32_t f = getf(x, i, c.eb, c.em) + (code == 1u ? 1u : 0u);
    setf(x, i, c.eb, c.em, f < c.mx ? f : c.mx);
  }
  if (!u) return;
  for (uint32_t i = 0; i < c.el; i++) {
    const uint32_t code = getf(u, i, c.ub, c.um);
    if (code >= 2u && code - 2u < c.el) {
      const uint32_t t = code - 2u, a = getf(x, t, c.eb, c.em), b = getf(x, i, c.eb, c.em);
      if (b > a) setf(x, t, c.eb, c.em, b);
    }
  }
}

}  // namespace geq
