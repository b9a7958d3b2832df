// Host-side check of the register sorting networks of
// gpz_b200/csrc/gpz_encode.cuh (odd-even merge sort of 32 values, merge of two
// sorted halves): compiled with nvcc, runs on the CPU.
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include "gpz_encode.cuh"

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

int main() {
  long bad = 0, checks = 0;
  // 0-1 principle: a comparator network sorts every input iff it sorts every 0/1 input
  for (uint64_t m = 0; m < (1ull << 32); m += 0x10001ull + (m >> 20)) {
    uint32_t a[32];
    for (int i = 0; i < 32; ++i) a[i] = (uint32_t)(m >> i) & 1u;
    gpzb::oem_sort32(a);
    for (int i = 1; i < 32; ++i) bad += a[i - 1] > a[i];
    ++checks;
  }
  for (int it = 0; it < 200000; ++it) {
    uint32_t a[32], b[32];
    const uint32_t range = it % 3 == 0 ? 4u : (it % 3 == 1 ? 1000u : 0xFFFFFFFFu);
    for (int i = 0; i < 32; ++i) b[i] = a[i] = range == 0xFFFFFFFFu ? rnd() : rnd() % range;
    gpzb::oem_sort32(a);
    std::sort(b, b + 32);
    for (int i = 0; i < 32; ++i) bad += a[i] != b[i];
    // two sorted halves
    uint32_t c[32];
    for (int i = 0; i < 32; ++i) c[i] = range == 0xFFFFFFFFu ? rnd() : rnd() % range;
    std::sort(c, c + 16);
    std::sort(c + 16, c + 32);
    uint32_t d[32];
    std::copy(c, c + 32, d);
    std::sort(d, d + 32);
    gpzb::merge_halves32(c);
    for (int i = 0; i < 32; ++i) bad += c[i] != d[i];
    ++checks;
  }
  printf("checks=%ld bad=%ld\n", checks, bad);
  return bad != 0;
}
