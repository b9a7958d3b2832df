// gpz_device.cuh -- device-side building blocks of the B200 GPZ codec.
//
// Layout and arithmetic follow the GPZ reference format (path:line citations
// refer to the reference project); the parallel decomposition is this
// library's own: one warp per 1024-point chunk in persistent grids, register
// sorting networks for the stable order by block id, in-register bit
// transposes for the bit planes, and a single-pass decoupled look-back scan
// that places each group's payloads directly in the output stream.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace gpzb {

constexpr int kChunk = 1024;        // points per chunk (ELEMS_PER_BLOCK, include/cudaCompress.cuh:9-11)
constexpr int kStageBytes = 9472;   // >= max payload: 31*128 + 11*128 + 31*128 + padding
constexpr uint32_t kSpinLimit = 1u << 22;  // bounded waits in the look-back scan
constexpr int kCtlBytes = 256;      // control block at the head of scratch

// Error codes (same values as include/gpz_b200.h).
constexpr int kOK = 0, kEINVAL = 1, kESEG = 2, kESTREAM = 3, kENOSPACE = 4, kETIMEOUT = 6;

// Control block in device scratch.  The first 24 bytes are gpz_result.
struct Control {
  unsigned long long stream_bytes;  // 0
  uint32_t seg;                     // 8
  uint32_t adjusted;                // 12
  int32_t status;                   // 16
  uint32_t id_overflow;             // 20
  uint32_t chunk_ctr;               // 24  persistent-grid work counter
  uint32_t abort;                   // 28  set when a bounded wait gives up
  uint32_t sample_done;             // 32  last-block detection for the sampling kernel
  uint32_t exit_ctr;                // 36  CTAs that left the persistent loop
  unsigned long long mm[6];         // 40  ordered min/max accumulators (min stored inverted)
  double out_eb;                    // 88  rel->abs result
  double out_mm[6];                 // 96  rel->abs min/max
  uint64_t G;                       // 144 chunks (decompress: from the header)
  double strict_eb;                 // 152 bound actually encoded in strict-bound mode
  uint32_t deferred;                // 160 decompress: chunks left to the general float64 pass
};
static_assert(sizeof(Control) <= kCtlBytes, "control block too large");

template <typename T> struct TT;
template <> struct TT<float> {
  using U = uint32_t;
  static constexpr uint32_t hdr = 24, meta = 36, pad = 3, bits = 32, u16_at = 28;
};
template <> struct TT<double> {
  using U = unsigned long long;
  static constexpr uint32_t hdr = 32, meta = 64, pad = 7, bits = 64, u16_at = 56;
};

// The last CTA of a persistent grid to leave rewinds the work counter, so a
// replay of the same launch (a profiler pass, a graph relaunch) starts over.
__device__ __forceinline__ void rewind_work_counter(Control *ctl) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->exit_ctr, 1u) == gridDim.x - 1) {
      atomicExch(&ctl->chunk_ctr, 0u);
      atomicExch(&ctl->exit_ctr, 0u);
    }
  }
}

__device__ __forceinline__ void set_status(Control *ctl, int code) {
  atomicCAS(reinterpret_cast<int *>(&ctl->status), 0, code);
}

// ---------------------------------------------------------------------------
// Ordered-integer views of floats: a < b  <=>  ord(a) < ord(b), with -0.0
// below +0.0, matching FMNMX on the GPU.  NaNs are filtered by the callers.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t f32_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}
__host__ __device__ __forceinline__ float bits_f32(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
__host__ __device__ __forceinline__ unsigned long long f64_bits(double f) {
  unsigned long long u;
  memcpy(&u, &f, 8);
  return u;
}
__host__ __device__ __forceinline__ double bits_f64(unsigned long long u) {
  double f;
  memcpy(&f, &u, 8);
  return f;
}
__host__ __device__ __forceinline__ uint32_t ord_of(float f) {
  const uint32_t u = f32_bits(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float from_ord(uint32_t o) {
  return bits_f32((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}
__host__ __device__ __forceinline__ unsigned long long ord_of(double f) {
  const unsigned long long u = f64_bits(f);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double from_ord(unsigned long long o) {
  return bits_f64((o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o);
}

// Warp-wide max of 32/64-bit unsigned values (REDUX on sm_80+).
__device__ __forceinline__ uint32_t warp_max(uint32_t v) { return __reduce_max_sync(0xFFFFFFFFu, v); }
__device__ __forceinline__ uint32_t warp_min(uint32_t v) { return __reduce_min_sync(0xFFFFFFFFu, v); }
__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
  uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, (uint32_t)(v >> 32));
  uint32_t lo = __reduce_max_sync(0xFFFFFFFFu, ((uint32_t)(v >> 32) == hi) ? (uint32_t)v : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

// Three-source float min / max (sm_100's min.f32 / max.f32 with three inputs):
// the same result as two two-input fminf / fmaxf, NaN sources ignored.
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return 32u - (uint32_t)__clz(v); }
__device__ __forceinline__ uint32_t bitlen64(unsigned long long v) { return 64u - (uint32_t)__clzll(v); }

// Section sizes (src/cudaWarpCompress.cu:324-328; Double :325-329).
__host__ __device__ __forceinline__ uint32_t section_bytes(uint32_t U, uint32_t nbits, uint32_t pad) {
  return ((((U + 7u) & ~7u) * nbits >> 3) + pad) & ~pad;
}
__host__ __device__ __forceinline__ uint32_t rel_section_bytes(uint32_t rbits, uint32_t pad) {
  return (((uint32_t)kChunk * rbits >> 3) + pad) & ~pad;
}

// Per-axis block counts, GPU arithmetic of the reference:
//   f32 (enc+dec):  static_cast<uint32_t>(ceilf(range / (2*seg*eb))) + 1     (:151-154, :831-834)
//   f64 3D enc:     static_cast<uint32_t>(ceil(...)) + 1 (u32 wrap)          (Double :151-154)
//   f64 2D enc:     static_cast<uint64_t>(ceil(...)) + 1                     (Double :525-526)
//   f64 dec:        static_cast<uint32_t>(ceil(...)) + 1                     (Double :835-838)
__device__ __forceinline__ unsigned long long block_num(float range, uint32_t seg, float eb, bool) {
  const float den = __fmul_rn(__uint2float_rn(2u * seg), eb);
  return (uint32_t)(__float2uint_rz(ceilf(__fdiv_rn(range, den))) + 1u);
}
__device__ __forceinline__ unsigned long long block_num(double range, uint32_t seg, double eb, bool wide) {
  const double den = __dmul_rn(__uint2double_rn(2u * seg), eb);
  const double c = ceil(__ddiv_rn(range, den));
  if (wide) return __double2ull_rz(c) + 1ull;
  return (unsigned long long)(uint32_t)(__double2uint_rz(c) + 1u);
}

// ---------------------------------------------------------------------------
// Swizzled index for 1024-entry u32 arrays that one thread per 32-element
// group reads with 16-byte loads: the 16-byte chunk index inside each group is
// XORed with the group number, so the 8 threads of a load phase hit 8
// different bank quads.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 0x1C); }

// Offset of the 16-byte quad m (0..7) of row `row` in the same layout: 8 lanes
// touching the same quad of their rows (or 8 quads of one row) hit 8
// different bank groups.
__device__ __forceinline__ uint32_t qoff(int row, int m) { return 32u * row + ((uint32_t)((m ^ row) & 7) << 2); }

// Loads the 32 values of group g (elements 32g..32g+31) from a swizzled array.
__device__ __forceinline__ void load_group(const uint32_t *arr, int g, uint32_t (&a)[32]) {
  const uint4 *p = reinterpret_cast<const uint4 *>(arr + 32 * g);
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const uint4 v = p[m ^ (g & 7)];
    a[4 * m + 0] = v.x;
    a[4 * m + 1] = v.y;
    a[4 * m + 2] = v.z;
    a[4 * m + 3] = v.w;
  }
}
__device__ __forceinline__ void store_group(uint32_t *arr, int g, const uint32_t (&a)[32]) {
  uint4 *p = reinterpret_cast<uint4 *>(arr + 32 * g);
#pragma unroll
  for (int m = 0; m < 8; ++m) p[m ^ (g & 7)] = make_uint4(a[4 * m], a[4 * m + 1], a[4 * m + 2], a[4 * m + 3]);
}

// ---------------------------------------------------------------------------
// In-register 32x32 bit transposes.  Input a[k] = value of element k; output
// rows are bit planes: row b bit k = bit b of element k.  A transpose swaps the
// five row-index bits with the five column-index bits one pair at a time; the
// pair swaps commute and each is its own inverse, so the same stages (in any
// order) also turn planes back into values.
// The 16- and 8-bit block swaps are byte permutes (PRMT); the 4/2/1-bit
// stages are masked XOR swaps.  Host-callable so they can be checked on a CPU.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
#ifdef __CUDA_ARCH__
  return __byte_perm(a, b, sel);
#else
  const unsigned long long x = ((unsigned long long)b << 32) | a;
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) r |= (uint32_t)((x >> (8 * ((sel >> (4 * i)) & 7u))) & 0xFFu) << (8 * i);
  return r;
#endif
}

template <int J>
__host__ __device__ __forceinline__ void bit_stage(uint32_t &lo, uint32_t &hi) {
  constexpr uint32_t m = J == 4 ? 0x0F0F0F0Fu : (J == 2 ? 0x33333333u : 0x55555555u);
  const uint32_t t = ((lo >> J) ^ hi) & m;
  lo ^= t << J;
  hi ^= t;
}

// The 4/2/1-bit stages over the first N words.
template <int N>
__host__ __device__ __forceinline__ void low_stages(uint32_t *a) {
#pragma unroll
  for (int q = 0; q < N; q += 8)
#pragma unroll
    for (int k = 0; k < 4; ++k) bit_stage<4>(a[q + k], a[q + k + 4]);
#pragma unroll
  for (int q = 0; q < N; q += 4)
#pragma unroll
    for (int k = 0; k < 2; ++k) bit_stage<2>(a[q + k], a[q + k + 2]);
#pragma unroll
  for (int q = 0; q < N; q += 2) bit_stage<1>(a[q], a[q + 1]);
}

// Byte-swap stage between words k and k+8 of each 16-word half.
template <int N>
__host__ __device__ __forceinline__ void byte_stage(uint32_t *a) {
#pragma unroll
  for (int q = 0; q < N; q += 16)
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t lo = prmt(a[q + k], a[q + k + 8], 0x6240);
      const uint32_t hi = prmt(a[q + k], a[q + k + 8], 0x7351);
      a[q + k] = lo;
      a[q + k + 8] = hi;
    }
}

// Full transpose: a[b] = plane b for b = 0..31 (and back).
__host__ __device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const uint32_t lo = prmt(a[k], a[k + 16], 0x5410);
    const uint32_t hi = prmt(a[k], a[k + 16], 0x7632);
    a[k] = lo;
    a[k + 16] = hi;
  }
  byte_stage<32>(a);
  low_stages<32>(a);
}

// Planes 0..15 only (values that need <= 16 bits): a[b] = plane b, b < 16.
__host__ __device__ __forceinline__ void transpose_lo16(uint32_t (&a)[32]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = prmt(a[k], a[k + 16], 0x5410);
  byte_stage<16>(a);
  low_stages<16>(a);
}

// Planes 16..31 only: a[b - 16] = plane b.
__host__ __device__ __forceinline__ void transpose_hi16(uint32_t (&a)[32]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = prmt(a[k], a[k + 16], 0x7632);
  byte_stage<16>(a);
  low_stages<16>(a);
}

// Planes 0..7 only (values that need <= 8 bits): a[b] = plane b, b < 8.
__host__ __device__ __forceinline__ void transpose_lo8(uint32_t (&a)[32]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = prmt(a[k], a[k + 16], 0x5410);
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = prmt(a[k], a[k + 8], 0x6240);
  low_stages<8>(a);
}

// Inverse of transpose_lo16 for values below 2^16: planes a[b], b < 16, become
// pairs a[k] = value k | value (k+16) << 16, k < 16.
__host__ __device__ __forceinline__ void planes16_to_pairs(uint32_t (&a)[16]) {
  low_stages<16>(a);
  byte_stage<16>(a);
}
__host__ __device__ __forceinline__ uint32_t pair_value(const uint32_t (&a)[16], int j) {
  return j < 16 ? (a[j] & 0xFFFFu) : (a[j - 16] >> 16);
}

// Inverse of transpose_lo8 for values below 2^8: planes a[b], b < 8, become
// quads a[k] = value k | value (k+8) << 8 | value (k+16) << 16 | value (k+24) << 24.
__host__ __device__ __forceinline__ void planes8_to_quads(uint32_t (&a)[8]) {
  low_stages<8>(a);
}
__host__ __device__ __forceinline__ uint32_t quad_value(const uint32_t (&a)[8], int j) {
  return (a[j & 7] >> (8 * (j >> 3))) & 0xFFu;
}

// A 32-bit plane word (bit t = element 32g+t) in the byte order of the
// delta / count sections: element k at bit 7-(k%8) of byte k/8
// (src/cudaWarpCompress.cu:366-378).
__host__ __device__ __forceinline__ uint32_t brev32(uint32_t w) {
#ifdef __CUDA_ARCH__
  return __brev(w);
#else
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i) r |= ((w >> i) & 1u) << (31 - i);
  return r;
#endif
}
__host__ __device__ __forceinline__ uint32_t to_msb_bytes(uint32_t w) { return prmt(brev32(w), 0, 0x0123); }
__host__ __device__ __forceinline__ uint32_t from_msb_bytes(uint32_t w) { return brev32(prmt(w, 0, 0x0123)); }

// ---------------------------------------------------------------------------
// Exact unsigned division by a per-chunk constant (round-up magic multiplier,
// Granlund & Montgomery 1994): q = (t + ((n - t) >> 1)) >> (l - 1),
// t = umulhi(m, n), l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1.
// d == 0 follows the GPU's integer division: quotient all ones, remainder n.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t clz32(uint32_t v) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__clz(v);
#else
  return v ? (uint32_t)__builtin_clz(v) : 32u;
#endif
}

struct FastDiv {
  uint32_t d, m, s;
  __host__ __device__ void init(uint32_t dv) {
    d = dv;
    m = 0;
    s = 0;
    if (dv <= 1) return;
    const uint32_t l = 32u - clz32(dv - 1u);
    m = (uint32_t)((((unsigned long long)1 << 32) * (((unsigned long long)1 << l) - dv)) / dv + 1ull);
    s = l - 1u;
  }
  __host__ __device__ uint32_t div(uint32_t n) const {
    if (d == 0) return 0xFFFFFFFFu;
    if (d == 1) return n;
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(m, n);
#else
    const uint32_t t = (uint32_t)(((unsigned long long)m * n) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> s;
  }
  __host__ __device__ uint32_t mod(uint32_t n) const { return d == 0 ? n : n - div(n) * d; }
};

// Exact division of n < 2^31 by d >= 1 in three instructions:
// q = umulhi(m, 2n) >> l, l = ceil(log2 d), m = ceil(2^(31+l) / d) < 2^32.
// Error bound: m = 2^(31+l)/d + e with 0 <= e < 1, so m*n / 2^(31+l) exceeds
// n/d by less than n / 2^(31+l) < 2^-l <= 1/d, which cannot carry past the
// next integer.  d > 2^31 quotients are all 0 (m = 0).
struct FastDiv31 {
  uint32_t d, m, l;
  __host__ __device__ void init(uint32_t dv) {
    d = dv;
    const uint32_t lg = dv <= 1 ? 0u : 32u - clz32(dv - 1u);
    if (dv == 0 || lg >= 32) { m = 0; l = 0; return; }
    const unsigned long long num = 1ull << (31 + lg);
    m = (uint32_t)((num + dv - 1) / dv);
    l = lg;
  }
  // n2 = 2n with n < 2^31
  __host__ __device__ __forceinline__ uint32_t div2(uint32_t n2) const {
#ifdef __CUDA_ARCH__
    return __umulhi(m, n2) >> l;
#else
    return (uint32_t)(((unsigned long long)m * n2) >> 32) >> l;
#endif
  }
};

// Relaxed GPU-scope accesses for the look-back words.
__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *(const volatile uint32_t *)p; }

}  // namespace gpzb
