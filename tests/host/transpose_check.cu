// Host-side check of the in-register bit transposes of
// gpz_b200/csrc/gpz_device.cuh against a bit-by-bit transpose: compiled with
// nvcc, runs on the CPU.
#include <cstdio>
#include <cstdint>
#include "gpz_device.cuh"

static uint64_t s = 0x2545F4914F6CDD1Dull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

// plane b bit k = bit b of value k
static void naive_planes(const uint32_t *v, uint32_t *p) {
  for (int b = 0; b < 32; ++b) {
    p[b] = 0;
    for (int k = 0; k < 32; ++k) p[b] |= ((v[k] >> b) & 1u) << k;
  }
}

int main() {
  long bad = 0, checks = 0;
  for (int it = 0; it < 20000; ++it) {
    const int width = 1 + it % 32;
    uint32_t v[32], p[32];
    for (int k = 0; k < 32; ++k) v[k] = width == 32 ? rnd() : rnd() & ((1u << width) - 1u);
    naive_planes(v, p);
    // values -> planes
    uint32_t a[32];
    for (int k = 0; k < 32; ++k) a[k] = v[k];
    gpzb::transpose32(a);
    for (int b = 0; b < 32; ++b) bad += a[b] != p[b];
    if (width <= 16) {
      for (int k = 0; k < 32; ++k) a[k] = v[k];
      gpzb::transpose_lo16(a);
      for (int b = 0; b < 16; ++b) bad += a[b] != p[b];
    } else {
      for (int k = 0; k < 32; ++k) a[k] = v[k];
      gpzb::transpose_hi16(a);
      for (int b = 16; b < 32; ++b) bad += a[b - 16] != p[b];
    }
    if (width <= 8) {
      for (int k = 0; k < 32; ++k) a[k] = v[k];
      gpzb::transpose_lo8(a);
      for (int b = 0; b < 8; ++b) bad += a[b] != p[b];
    }
    // planes -> values
    for (int b = 0; b < 32; ++b) a[b] = p[b];
    gpzb::transpose32(a);
    for (int k = 0; k < 32; ++k) bad += a[k] != v[k];
    if (width <= 16) {
      uint32_t h[16];
      for (int b = 0; b < 16; ++b) h[b] = p[b];
      gpzb::planes16_to_pairs(h);
      for (int k = 0; k < 32; ++k) bad += gpzb::pair_value(h, k) != v[k];
    }
    if (width <= 8) {
      uint32_t q[8];
      for (int b = 0; b < 8; ++b) q[b] = p[b];
      gpzb::planes8_to_quads(q);
      for (int k = 0; k < 32; ++k) bad += gpzb::quad_value(q, k) != v[k];
    }
    // stream byte order round trip, and the order itself
    const uint32_t w = rnd();
    bad += gpzb::from_msb_bytes(gpzb::to_msb_bytes(w)) != w;
    const uint32_t m = gpzb::to_msb_bytes(w);
    for (int k = 0; k < 32; ++k) bad += ((w >> k) & 1u) != ((m >> (8 * (k / 8) + 7 - k % 8)) & 1u);
    ++checks;
  }
  printf("checks=%ld bad=%ld\n", checks, bad);
  return bad != 0;
}
