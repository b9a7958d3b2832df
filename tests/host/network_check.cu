// Host-side check of the register sorting networks of
// gpz_b200/csrc/gpz_encode.cuh: the odd-even merge sort of 32 values, and the
// comparator schedule of warp_sort1024_rows (32 lanes x 32 registers, the
// cross-lane stages emulated lane by lane): compiled with nvcc, runs on the
// CPU.
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include "gpz_encode.cuh"

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

// The comparators of warp_sort1024_rows on V[lane][j] (element 32 * lane + j).
static void sort1024_schedule(uint32_t (&V)[32][32]) {
  for (int l = 0; l < 32; ++l) gpzb::oem_sort32(V[l]);
  for (int lk = 6; lk <= 10; ++lk) {
    uint32_t W[32][32];
    const int m = (1 << (lk - 5)) - 1;
    for (int l = 0; l < 32; ++l) {
      const bool lo = ((l >> (lk - 6)) & 1) == 0;
      for (int j = 0; j < 32; ++j) {
        const uint32_t a = V[l ^ m][31 - j];
        W[l][j] = lo ? std::min(V[l][j], a) : std::max(V[l][j], a);
      }
    }
    std::copy(&W[0][0], &W[0][0] + 1024, &V[0][0]);
    for (int s = lk - 2; s >= 5; --s) {
      const int dl = 1 << (s - 5);
      for (int l = 0; l < 32; ++l) {
        const bool lo = (l & dl) == 0;
        for (int j = 0; j < 32; ++j) {
          const uint32_t a = V[l ^ dl][j];
          W[l][j] = lo ? std::min(V[l][j], a) : std::max(V[l][j], a);
        }
      }
      std::copy(&W[0][0], &W[0][0] + 1024, &V[0][0]);
    }
    for (int l = 0; l < 32; ++l)
      for (int d = 16; d >= 1; d >>= 1)
        for (int j = 0; j < 32; ++j)
          if ((j & d) == 0) {
            const uint32_t x = V[l][j], y = V[l][j | d];
            V[l][j] = std::min(x, y);
            V[l][j | d] = std::max(x, y);
          }
  }
}

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
    if (it % 50 == 0) {  // the whole warp's 1024 values
      uint32_t V[32][32], ref[1024];
      const uint32_t r2 = it % 150 == 0 ? 8u : 1u << 22;
      for (int i = 0; i < 1024; ++i) ref[i] = V[i / 32][i % 32] = rnd() % r2;
      sort1024_schedule(V);
      std::sort(ref, ref + 1024);
      for (int i = 0; i < 1024; ++i) bad += V[i / 32][i % 32] != ref[i];
    }
    ++checks;
  }
  printf("checks=%ld bad=%ld\n", checks, bad);
  return bad != 0;
}
