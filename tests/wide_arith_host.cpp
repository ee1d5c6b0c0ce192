// wide_arith_host.cpp - test support: the multi-word solver's energy
// arithmetic (gpuequiv_b200/csrc/wide_arith.cuh) compiled for the host as a
// small shared library, so that the CPU tests can compare it with the
// oracle on random energies and updates of many confs.  Test infrastructure.
#include <cstdint>

#include "geq_internal.h"
#include "wide_arith.cuh"

using namespace geq;

static WideConf conf_of(uint32_t el, uint32_t mx) {
  const Conf c(el, mx);
  return WideConf{el, mx, c.energy_bits(), c.energy_mask(), c.update_bits(), c.update_mask()};
}

extern "C" {
// field-wise a <= b over all words of two energies
int wa_leq(uint32_t el, uint32_t mx, const uint32_t *a, const uint32_t *b) {
  const Conf c(el, mx);
  const Swar s = make_swar(c.energy_bits());
  for (uint32_t w = 0; w < c.energy_size(); w++)
    if (!swar_leq(a[w], b[w], s)) return 0;
  return 1;
}
void wa_max(uint32_t el, uint32_t mx, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  const Conf c(el, mx);
  const Swar s = make_swar(c.energy_bits());
  for (uint32_t w = 0; w < c.energy_size(); w++) out[w] = swar_max(a[w], b[w], s);
}
void wa_inv_update(uint32_t el, uint32_t mx, const uint32_t *e, const uint32_t *u, uint32_t *out) {
  const Conf c(el, mx);
  for (uint32_t w = 0; w < c.energy_size(); w++) out[w] = e[w];
  wide_inv_update(conf_of(el, mx), out, u);
}
}
