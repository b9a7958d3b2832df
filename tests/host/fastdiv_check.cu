// Host-side check of the exact divider used by the decompress kernel
// (gpz_b200/csrc/gpz_device.cuh, FastDiv): compiled with nvcc, runs on the CPU.
#include <cstdio>
#include <cstdint>
#include "gpz_device.cuh"

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

int main() {
  long bad = 0, checks = 0;
  uint32_t divs[] = {0u, 1u, 2u, 3u, 5u, 7u, 157u, 1024u, 1025u, 65535u, 65536u, 65537u, 2147483647u,
                     2147483648u, 2147483649u, 4294967294u, 4294967295u};
  auto check = [&](uint32_t d, uint32_t n) {
    gpzb::FastDiv f;
    f.init(d);
    uint32_t q = d ? n / d : 0xFFFFFFFFu, r = d ? n % d : n;
    ++checks;
    if (f.div(n) != q || f.mod(n) != r) {
      if (bad < 10) printf("mismatch d=%u n=%u got %u/%u want %u/%u\n", d, n, f.div(n), f.mod(n), q, r);
      ++bad;
    }
  };
  for (uint32_t d : divs) {
    for (uint32_t n : {0u, 1u, d, d - 1u, d + 1u, 2u * d, 4294967295u, 4294967294u, 2147483648u}) check(d, n);
    for (int i = 0; i < 20000; ++i) check(d, rnd());
  }
  for (int i = 0; i < 2000000; ++i) {
    uint32_t d = rnd() >> (rnd() % 32);
    check(d, rnd());
    check(d, rnd() >> (rnd() % 32));
  }
  // FastDiv31: n < 2^31, d >= 1
  auto check31 = [&](uint32_t d, uint32_t n) {
    gpzb::FastDiv31 f;
    f.init(d);
    ++checks;
    if (f.div2(n + n) != n / d) {
      if (bad < 20) printf("fd31 mismatch d=%u n=%u got %u want %u\n", d, n, f.div2(n + n), n / d);
      ++bad;
    }
  };
  for (uint32_t d : divs) {
    if (d == 0) continue;
    for (uint32_t n : {0u, 1u, d, d - 1u, d + 1u, 2u * d, 2u * d - 1u, 2147483647u, 2147483646u, 1073741824u})
      if (n < 2147483648u) check31(d, n);
    for (int i = 0; i < 20000; ++i) check31(d, rnd() >> 1);
  }
  for (int i = 0; i < 4000000; ++i) {
    const uint32_t d = rnd() >> (rnd() % 32);
    if (d == 0) continue;
    const uint32_t n = (rnd() >> 1) >> (rnd() % 31);
    check31(d, n);
    const uint32_t q = n / d;  // near multiples of d
    check31(d, q * d);
    if (q * d) check31(d, q * d - 1u);
  }
  printf("checks=%ld bad=%ld\n", checks, bad);
  return bad != 0;
}
