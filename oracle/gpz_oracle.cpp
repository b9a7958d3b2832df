// gpz_oracle.cpp -- CPU restatement of GPZ's particle compress/decompress.
//
// TEST INFRASTRUCTURE ONLY (parity checker + timed CPU baseline).  Nothing
// in gpz_b200/ links or calls this code.
//
// Build: g++ -O3 -fopenmp -ffp-contract=off -std=c++17 (no -march=native),
// so host float arithmetic matches the reference's host code bit for bit and
// the GPU-side float arithmetic is spelled out with explicit fma calls.
//
// Citations are path:line inside the GPZ reference project.

#include "gpz_oracle.h"

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <string>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kChunk = 1024;  // ELEMS_PER_BLOCK, include/cudaCompress.cuh:9-11

// ---------------------------------------------------------------------------
// GPU arithmetic semantics the reference kernels rely on.
// ---------------------------------------------------------------------------

// static_cast<uint32_t>(float) on the GPU is cvt.rzi.u32.f32: truncation with
// saturation (negative and NaN -> 0, >= 2^32 -> UINT32_MAX).
inline uint32_t cvt_u32(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967296.0f) return 0xFFFFFFFFu;
  return static_cast<uint32_t>(v);
}
inline uint32_t cvt_u32(double v) {
  if (!(v > 0.0)) return 0u;
  if (v >= 4294967296.0) return 0xFFFFFFFFu;
  return static_cast<uint32_t>(v);
}
inline uint64_t cvt_u64(double v) {
  if (!(v > 0.0)) return 0u;
  if (v >= 18446744073709551616.0) return UINT64_MAX;
  return static_cast<uint64_t>(v);
}
inline uint64_t cvt_u64(float v) { return cvt_u64(static_cast<double>(v)); }

// fminf / fmaxf as the GPU evaluates them (FMNMX): a NaN operand is ignored
// and -0.0 orders below +0.0.
template <typename T>
inline T gmin(T a, T b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  if (a == b) return std::signbit(a) ? a : b;
  return a < b ? a : b;
}
template <typename T>
inline T gmax(T a, T b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  if (a == b) return std::signbit(a) ? b : a;
  return a > b ? a : b;
}

inline uint32_t bitlen32(uint32_t v) { return v ? 32u - (uint32_t)__builtin_clz(v) : 0u; }
inline uint32_t bitlen64(uint64_t v) { return v ? 64u - (uint32_t)__builtin_clzll(v) : 0u; }
inline uint32_t ffs_shift(uint32_t seg) { return (uint32_t)__builtin_ffs((int)seg) - 1u; }
// shr.u32 clamps shift counts >= 32 to 32 (result 0).
inline uint32_t shr32(uint32_t v, uint32_t s) { return s >= 32 ? 0u : (v >> s); }
inline uint64_t shr64(uint64_t v, uint32_t s) { return s >= 64 ? 0u : (v >> s); }

inline void put_u16(uint8_t *p, uint16_t v) { memcpy(p, &v, 2); }
inline void put_u32(uint8_t *p, uint32_t v) { memcpy(p, &v, 4); }
inline void put_u64(uint8_t *p, uint64_t v) { memcpy(p, &v, 8); }
inline uint16_t get_u16(const uint8_t *p) { uint16_t v; memcpy(&v, p, 2); return v; }
inline uint32_t get_u32(const uint8_t *p) { uint32_t v; memcpy(&v, p, 4); return v; }
inline uint64_t get_u64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }

// ---------------------------------------------------------------------------
// Per-type layout constants.
//   f32: header 24 B (src/cudaWarpCompress.cu:1673-1679), meta 36 B (:20),
//        sections padded to 4 B (:324-328).
//   f64: header 32 B (src/cudaWarpCompressDouble.cu:1672-1680), meta 64 B
//        (:20), sections padded to 8 B (:325-329).
// ---------------------------------------------------------------------------
template <typename T> struct Lay;
template <> struct Lay<float> {
  static constexpr uint32_t hdr = 24, meta = 36, pad = 3, bits = 32, u16_at = 28;
};
template <> struct Lay<double> {
  static constexpr uint32_t hdr = 32, meta = 64, pad = 7, bits = 64, u16_at = 56;
};

inline uint32_t section_bytes(uint32_t U, uint32_t nbits, uint32_t pad) {
  // (((((U + 7) & ~7U) * bits) >> 3) + pad) & ~pad   (src/cudaWarpCompress.cu:324-327)
  return ((((U + 7u) & ~7u) * nbits >> 3) + pad) & ~pad;
}
inline uint32_t rel_bytes(uint32_t rbits, uint32_t pad) {
  return (((kChunk * rbits) >> 3) + pad) & ~pad;  // :328
}

// Per-chunk block-count along one axis.
//   f32:      static_cast<uint32_t>(ceilf(range / (2*seg*eb))) + 1   (:151-154)
//   f64 3D:   static_cast<uint32_t>(ceil (range / (2*seg*eb))) + 1   (Double :151-154)
//   f64 2D:   static_cast<uint64_t>(ceil (range / (2*seg*eb))) + 1   (Double :525-526)
//   f64 dec:  static_cast<uint32_t>(ceil (...)) + 1, both dims       (Double :835-838, :1046-1049)
inline uint64_t block_num(float range, uint32_t seg, float eb, bool /*wide*/) {
  float den = static_cast<float>(2u * seg) * eb;
  return (uint32_t)(cvt_u32(std::ceil(range / den)) + 1u);
}
inline uint64_t block_num(double range, uint32_t seg, double eb, bool wide) {
  double den = static_cast<double>(2u * seg) * eb;
  double c = std::ceil(range / den);
  if (wide) return cvt_u64(c) + 1u;
  return (uint64_t)(uint32_t)(cvt_u32(c) + 1u);
}

// fma with the operand type.
inline float tfma(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double tfma(double a, double b, double c) { return std::fma(a, b, c); }

// The reference reconstructs with `min + ((q << 1) | 1) * eb`, which nvcc
// contracts into one fused multiply-add (--fmad=true is nvcc's default).
int g_decode_fma = 1;

// ---------------------------------------------------------------------------
// Chunk encoder.
// ---------------------------------------------------------------------------
template <typename T>
struct ChunkEnc {
  T mn[3], mx[3];
  uint32_t nvalid = 0;
  uint64_t first_id = 0;
  uint32_t dbits = 0, cbits = 0, rbits = 0, U = 0;
  uint32_t dbytes = 0, cbytes = 0, rbytes = 0;
  uint32_t delta[kChunk], count[kChunk];
  uint32_t rel_sorted[kChunk];
  uint16_t perm[kChunk];  // sorted slot -> local point index
  uint32_t payload() const { return dbytes + cbytes + rbytes; }
};

// Stable LSD radix sort of composite keys (block_id << 10 | r), 8-bit digits.
inline void sort_composite(uint64_t *a, uint64_t *tmp, uint32_t n, uint32_t nbits) {
  for (uint32_t sh = 0; sh < nbits; sh += 8) {
    uint32_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (uint32_t i = 0; i < n; ++i) cnt[((a[i] >> sh) & 0xFF) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (uint32_t i = 0; i < n; ++i) tmp[cnt[(a[i] >> sh) & 0xFF]++] = a[i];
    memcpy(a, tmp, sizeof(uint64_t) * n);
  }
}

// runCompressKernel / runCompressKernel2D: src/cudaWarpCompress.cu:58-435,
// 437-796; float64 twins src/cudaWarpCompressDouble.cu:57-437, 439-799.
template <typename T>
void encode_chunk(const T *x, const T *y, const T *z, uint32_t nvalid,
                  uint32_t dim, T eb, uint32_t seg, ChunkEnc<T> &e) {
  using Q = typename std::conditional<sizeof(T) == 4, uint32_t, uint64_t>::type;
  const bool is64 = sizeof(T) == 8;
  e.nvalid = nvalid;
  // min/max over valid points (:104-139)
  T lo = is64 ? (T)DBL_MAX : (T)FLT_MAX;
  for (int a = 0; a < 3; ++a) { e.mn[a] = lo; e.mx[a] = -lo; }
  for (uint32_t p = 0; p < nvalid; ++p) {
    e.mn[0] = gmin(e.mn[0], x[p]); e.mx[0] = gmax(e.mx[0], x[p]);
    e.mn[1] = gmin(e.mn[1], y[p]); e.mx[1] = gmax(e.mx[1], y[p]);
    if (dim == 3) { e.mn[2] = gmin(e.mn[2], z[p]); e.mx[2] = gmax(e.mx[2], z[p]); }
  }
  if (dim == 2) { e.mn[2] = 0; e.mx[2] = 0; }  // meta z = 0 (:518,521)

  const T inv = (T)1 / ((T)2 * eb);  // :141 (IEEE division)
  const uint64_t bnx = block_num(e.mx[0] - e.mn[0], seg, eb, is64 && dim == 2);
  const uint64_t bny = (dim == 3) ? block_num(e.mx[1] - e.mn[1], seg, eb, false) : 0;
  const uint32_t sh = ffs_shift(seg);  // :157
  const uint32_t msk = seg - 1u;       // :166
  const T nx = -e.mn[0] * inv, ny = -e.mn[1] * inv, nz = -e.mn[2] * inv;

  uint64_t comp[kChunk], tmp[kChunk];
  uint32_t rel_by_p[kChunk];
  uint32_t rmax_bits = 0;
  uint64_t cmax = 0;
  for (uint32_t p = 0; p < nvalid; ++p) {
    uint64_t key;
    uint32_t rel;
    if (!is64) {
      uint32_t qx = cvt_u32((float)tfma(x[p], inv, nx));
      uint32_t qy = cvt_u32((float)tfma(y[p], inv, ny));
      uint32_t bx = (uint32_t)bnx, by = (uint32_t)bny;
      if (dim == 3) {
        uint32_t qz = cvt_u32((float)tfma(z[p], inv, nz));
        key = ((qx >> sh) + (qy >> sh) * bx + (qz >> sh) * bx * by) & 0x7FFFFFFFu;  // :187-189
        rel = ((qx & msk) + (qy & msk) * seg + (qz & msk) * seg * seg) & 0x7FFFFFFFu;  // :191-193
      } else {
        key = ((qx >> sh) + (qy >> sh) * bx) & 0x7FFFFFFFu;  // :550-551
        rel = ((qx & msk) + (qy & msk) * seg) & 0x7FFFFFFFu;  // :553-554
      }
    } else {
      Q qx = cvt_u64((double)tfma(x[p], inv, nx));  // Double :179-184
      Q qy = cvt_u64((double)tfma(y[p], inv, ny));
      Q m = (Q)msk, s = (Q)seg;
      if (dim == 3) {
        Q qz = cvt_u64((double)tfma(z[p], inv, nz));
        key = ((qx >> sh) + (qy >> sh) * bnx + (qz >> sh) * bnx * bny) & 0x7FFFFFFFull;
        rel = (uint32_t)(((qx & m) + (qy & m) * s + (qz & m) * s * s) & 0x7FFFFFFFull);
      } else {
        key = ((qx >> sh) + (qy >> sh) * bnx) & 0x7FFFFFFFull;
        rel = (uint32_t)(((qx & m) + (qy & m) * s) & 0x7FFFFFFFull);
      }
    }
    // Rank of point p in the reference's cub::BlockRadixSort input: the
    // kernel loads point 32*i + lane into register i of `lane` (:103-118)
    // and BlockRadixSort ranks items in blocked order lane*32 + i.
    uint32_t r = (p & 31u) * 32u + (p >> 5);
    comp[p] = (key << 10) | r;
    cmax = std::max(cmax, comp[p]);
    rel_by_p[p] = rel;
    rmax_bits = std::max(rmax_bits, bitlen32(rel));
  }
  // Stable sort by block id (:212-218); invalid tail keys (UINT_MAX) sort
  // after every valid key, so only valid points are sorted here.
  sort_composite(comp, tmp, nvalid, bitlen64(cmax));

  uint32_t keys_s[kChunk];
  for (uint32_t i = 0; i < nvalid; ++i) {
    uint32_t r = (uint32_t)(comp[i] & 1023u);
    uint32_t p = ((r & 31u) << 5) | (r >> 5);
    keys_s[i] = (uint32_t)(comp[i] >> 10);
    e.rel_sorted[i] = rel_by_p[p];
    e.perm[i] = (uint16_t)p;
  }
  for (uint32_t i = nvalid; i < kChunk; ++i) e.rel_sorted[i] = 0xFFFFFFFFu;  // :197
  // Invalid slots count as 1 bit (:200-201).
  e.rbits = nvalid < kChunk ? std::max(rmax_bits, 1u) : rmax_bits;

  // Runs of equal ids: unique count, counts, deltas (:222-311).
  uint32_t U = 0, dbits = 0, cbits = 0;
  uint32_t start = 0;
  for (uint32_t i = 0; i < nvalid; ++i) {
    if (i == 0 || keys_s[i] != keys_s[i - 1]) {
      if (i > 0) {
        e.count[U - 1] = i - start;
        cbits = std::max(cbits, bitlen32(i - start));
      }
      uint32_t d = (i == 0) ? 0u : keys_s[i] - keys_s[i - 1];
      e.delta[U] = d;
      dbits = std::max(dbits, bitlen32(d));
      start = i;
      ++U;
    }
  }
  e.count[U - 1] = nvalid - start;
  cbits = std::max(cbits, bitlen32(nvalid - start));
  e.U = U; e.dbits = dbits; e.cbits = cbits;
  e.first_id = keys_s[0];  // outlier = first sorted id (:321)
  e.dbytes = section_bytes(U, dbits, Lay<T>::pad);
  e.cbytes = section_bytes(U, cbits, Lay<T>::pad);
  e.rbytes = rel_bytes(e.rbits, Lay<T>::pad);
}

// Byte-granular bit planes, MSB plane first, element k at bit 7-(k%8) of
// byte k/8 (:357-408).
inline void put_planes_bytes(uint8_t *dst, const uint32_t *v, uint32_t n, uint32_t nbits) {
  const uint32_t bpp = (n + 7u) >> 3;
  for (uint32_t pi = 0; pi < nbits; ++pi) {
    const uint32_t bit = nbits - 1u - pi;
    uint8_t *pl = dst + (size_t)pi * bpp;
    for (uint32_t k = 0; k < n; ++k)
      if ((v[k] >> bit) & 1u) pl[k >> 3] |= (uint8_t)(0x80u >> (k & 7u));
  }
}
// Relative-position planes: 32 little-endian words per plane, word w bit t
// = sorted element 32w+t (:411-434).
inline void put_planes_words(uint8_t *dst, const uint32_t *v, uint32_t nbits) {
  for (uint32_t pi = 0; pi < nbits; ++pi) {
    const uint32_t bit = nbits - 1u - pi;
    for (uint32_t w = 0; w < 32; ++w) {
      uint32_t word = 0;
      for (uint32_t t = 0; t < 32; ++t) word |= ((v[32 * w + t] >> bit) & 1u) << t;
      put_u32(dst + (size_t)pi * 128 + 4 * w, word);
    }
  }
}

template <typename T>
void write_meta(uint8_t *m, const ChunkEnc<T> &e) {
  // meta record (:332-344 / Double :333-345)
  T mm[6] = {e.mn[0], e.mn[1], e.mn[2], e.mx[0], e.mx[1], e.mx[2]};
  memcpy(m, mm, sizeof(mm));
  if (sizeof(T) == 4) put_u32(m + 24, (uint32_t)e.first_id);
  else put_u64(m + 48, e.first_id);
  uint8_t *u = m + Lay<T>::u16_at;
  put_u16(u + 0, (uint16_t)e.dbits);
  put_u16(u + 2, (uint16_t)e.cbits);
  put_u16(u + 4, (uint16_t)e.rbits);
  put_u16(u + 6, (uint16_t)e.U);
}

template <typename T>
void write_payload(uint8_t *dst, const ChunkEnc<T> &e) {
  memset(dst, 0, e.payload());
  put_planes_bytes(dst, e.delta, e.U, e.dbits);
  put_planes_bytes(dst + e.dbytes, e.count, e.U, e.cbits);
  put_planes_words(dst + e.dbytes + e.cbytes, e.rel_sorted, e.rbits);
}

inline int set_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

template <typename T>
void write_header(uint8_t *out, uint32_t dim, uint64_t n, T eb, uint32_t seg) {
  // f32: src/cudaWarpCompress.cu:1674-1678; f64: src/cudaWarpCompressDouble.cu:1672-1680
  memset(out, 0, Lay<T>::hdr);
  put_u32(out, dim);
  put_u64(out + 4, n);
  put_u32(out + 12, Lay<T>::bits);
  memcpy(out + 16, &eb, sizeof(T));
  put_u32(out + 16 + sizeof(T), seg);
  if (sizeof(T) == 8) put_u32(out + 28, 32u);
}

template <typename T>
int compress_impl(const T *x, const T *y, const T *z, uint64_t n, uint32_t dim,
                  T eb, uint32_t seg, uint8_t *out, uint64_t *out_bytes, int nthreads) {
  if (!x || !y || (dim == 3 && !z) || !out || !out_bytes) return GPZO_EINVAL;
  if (n == 0 || (dim != 2 && dim != 3) || seg == 0) return GPZO_EINVAL;
  const uint64_t G = (n + kChunk - 1) / kChunk;
  const uint64_t meta_base = Lay<T>::hdr + 8 * G;
  const uint64_t pay_base = meta_base + (uint64_t)Lay<T>::meta * G;
  write_header<T>(out, dim, n, eb, seg);
  const int nt = set_threads(nthreads);
  std::vector<std::vector<uint8_t>> bufs(nt);
  std::vector<uint64_t> tot(nt + 1, 0);
  std::vector<uint32_t> sizes(G);
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    const uint64_t c0 = G * tid / nt, c1 = G * (tid + 1) / nt;
    std::vector<uint8_t> &buf = bufs[tid];
    buf.reserve((size_t)((c1 - c0) * 4200));
    ChunkEnc<T> *e = new ChunkEnc<T>;
    for (uint64_t c = c0; c < c1; ++c) {
      const uint64_t b = c * kChunk;
      const uint32_t nv = (uint32_t)std::min<uint64_t>(kChunk, n - b);
      encode_chunk<T>(x + b, y + b, dim == 3 ? z + b : nullptr, nv, dim, eb, seg, *e);
      write_meta<T>(out + meta_base + c * Lay<T>::meta, *e);
      const size_t at = buf.size();
      buf.resize(at + e->payload());
      write_payload<T>(buf.data() + at, *e);
      sizes[c] = e->payload();
    }
    delete e;
    tot[tid + 1] = buf.size();
  }
  for (int t = 0; t < nt; ++t) tot[t + 1] += tot[t];
  // Offsets = exclusive scan of payload sizes (cub::DeviceScan::ExclusiveSum, :1660-1666).
  uint64_t acc = 0;
  for (uint64_t c = 0; c < G; ++c) { put_u64(out + Lay<T>::hdr + 8 * c, acc); acc += sizes[c]; }
#pragma omp parallel for num_threads(nt) schedule(static, 1)
  for (int t = 0; t < nt; ++t)
    if (!bufs[t].empty()) memcpy(out + pay_base + tot[t], bufs[t].data(), bufs[t].size());
  *out_bytes = pay_base + acc;  // :1702
  return GPZO_OK;
}

// ---------------------------------------------------------------------------
// Decoder.
// ---------------------------------------------------------------------------
struct Hdr {
  uint32_t dim = 0, bits = 0, seg = 0;
  uint64_t n = 0, G = 0;
  double eb = 0;
  float eb32 = 0;
  uint32_t hdr = 0, meta = 0, pad = 0;
};

int parse(const uint8_t *s, uint64_t bytes, Hdr &h) {
  if (!s || bytes < 24) return GPZO_ESTREAM;
  h.dim = get_u32(s);
  h.n = get_u64(s + 4);
  h.bits = get_u32(s + 12);
  if (h.bits == 32) {
    memcpy(&h.eb32, s + 16, 4);
    h.eb = h.eb32;
    h.seg = get_u32(s + 20);
    h.hdr = 24; h.meta = 36; h.pad = 3;
  } else if (h.bits == 64) {
    if (bytes < 32) return GPZO_ESTREAM;
    memcpy(&h.eb, s + 16, 8);
    h.seg = get_u32(s + 24);
    h.hdr = 32; h.meta = 64; h.pad = 7;
  } else {
    return GPZO_ESTREAM;
  }
  if ((h.dim != 2 && h.dim != 3) || h.n == 0 || h.seg == 0) return GPZO_ESTREAM;
  h.G = (h.n + kChunk - 1) / kChunk;
  if (h.G > (bytes - h.hdr) / (8ull + h.meta)) return GPZO_ESTREAM;
  return GPZO_OK;
}

inline void get_planes_bytes(const uint8_t *src, uint32_t *v, uint32_t n, uint32_t nbits) {
  const uint32_t bpp = (n + 7u) >> 3;
  for (uint32_t k = 0; k < n; ++k) v[k] = 0;
  for (uint32_t pi = 0; pi < nbits; ++pi) {
    const uint32_t bit = nbits - 1u - pi;
    const uint8_t *pl = src + (size_t)pi * bpp;
    for (uint32_t k = 0; k < n; ++k) v[k] |= (uint32_t)((pl[k >> 3] >> (7u - (k & 7u))) & 1u) << bit;
  }
}

// runDecompressKernel[2D]: src/cudaWarpCompress.cu:798-1214; Double :801-1217.
template <typename T>
int decode_chunk(const uint8_t *s, uint64_t bytes, const Hdr &h, uint64_t c,
                 T *x, T *y, T *z) {
  using Q = typename std::conditional<sizeof(T) == 4, uint32_t, uint64_t>::type;
  const bool is64 = sizeof(T) == 8;
  const uint64_t meta_base = h.hdr + 8 * h.G;
  const uint64_t pay_base = meta_base + (uint64_t)h.meta * h.G;
  const uint8_t *m = s + meta_base + c * h.meta;
  T mm[6];
  memcpy(mm, m, sizeof(mm));
  const uint64_t first = is64 ? get_u64(m + 48) : get_u32(m + 24);
  const uint8_t *u = m + (is64 ? 56 : 28);
  const uint32_t dbits = get_u16(u), cbits = get_u16(u + 2), rbits = get_u16(u + 4), U = get_u16(u + 6);
  const uint32_t nvalid = (uint32_t)std::min<uint64_t>(kChunk, h.n - c * kChunk);
  if (U == 0 || U > nvalid || dbits > 32 || cbits > 32 || rbits > 32) return GPZO_ESTREAM;
  const uint32_t db = section_bytes(U, dbits, h.pad), cb = section_bytes(U, cbits, h.pad);
  const uint32_t rb = rel_bytes(rbits, h.pad);
  const uint64_t off = get_u64(s + h.hdr + 8 * c);
  if (off > bytes - pay_base || (uint64_t)db + cb + rb > bytes - pay_base - off) return GPZO_ESTREAM;
  const uint8_t *p = s + pay_base + off;

  uint32_t delta[kChunk], cnt[kChunk], rel[kChunk];
  get_planes_bytes(p, delta, U, dbits);
  get_planes_bytes(p + db, cnt, U, cbits);
  for (uint32_t i = 0; i < kChunk; ++i) rel[i] = 0;
  for (uint32_t pi = 0; pi < rbits; ++pi) {
    const uint32_t bit = rbits - 1u - pi;
    for (uint32_t w = 0; w < 32; ++w) {
      uint32_t word = get_u32(p + db + cb + (size_t)pi * 128 + 4 * w);
      for (uint32_t t = 0; t < 32; ++t) rel[32 * w + t] |= ((word >> t) & 1u) << bit;
    }
  }
  // ids: inclusive prefix of deltas seeded with the first id (:930-934);
  // the reference keeps ids in the key type (u32 / u64).
  Q ids[kChunk];
  ids[0] = (Q)first;
  for (uint32_t k = 1; k < U; ++k) ids[k] = (Q)(ids[k - 1] + (Q)delta[k]);
  uint64_t total = 0;
  for (uint32_t k = 0; k < U; ++k) total += cnt[k];
  if (total != nvalid) return GPZO_ESTREAM;

  T eb = is64 ? (T)h.eb : (T)h.eb32;
  const uint32_t seg = h.seg;
  uint64_t bnx, bny;
  if (!is64) {
    bnx = block_num((float)(mm[3] - mm[0]), seg, (float)eb, false);
    bny = block_num((float)(mm[4] - mm[1]), seg, (float)eb, false);
  } else {
    bnx = block_num((double)(mm[3] - mm[0]), seg, (double)eb, false);
    bny = block_num((double)(mm[4] - mm[1]), seg, (double)eb, false);
  }
  const uint32_t sh = ffs_shift(seg), msk = seg - 1u;
  const uint64_t base = c * kChunk;
  uint32_t pos = 0;
  for (uint32_t k = 0; k < U; ++k) {
    for (uint32_t j = 0; j < cnt[k]; ++j, ++pos) {
      const Q id = ids[k];
      const uint32_t rp = rel[pos];
      T vx, vy, vz = 0;
      if (!is64) {
        const uint32_t bx32 = (uint32_t)bnx, by32 = (uint32_t)bny;
        const uint32_t id32 = (uint32_t)id;
        // Unsigned division by zero on the GPU yields all ones, remainder = dividend.
        auto dv = [](uint32_t a, uint32_t b) { return b ? a / b : 0xFFFFFFFFu; };
        auto md = [](uint32_t a, uint32_t b) { return b ? a % b : a; };
        const uint32_t bx = md(id32, bx32);                       // :988
        const uint32_t by = md(dv(id32, bx32), by32);             // :989
        const uint32_t rx = rp & msk, ry = (rp >> sh) & msk;      // :992-993
        const uint32_t qx = bx * seg + rx, qy = by * seg + ry;    // :996-997
        const float fx = (float)((qx << 1) | 1u), fy = (float)((qy << 1) | 1u);
        const float e32 = (float)eb;
        vx = (T)(g_decode_fma ? std::fmaf(fx, e32, (float)mm[0]) : (float)mm[0] + fx * e32);
        vy = (T)(g_decode_fma ? std::fmaf(fy, e32, (float)mm[1]) : (float)mm[1] + fy * e32);
        if (h.dim == 3) {
          const uint32_t bz = dv(id32, bx32 * by32);              // :990
          const uint32_t rz = shr32(rp, sh * 2);                  // :994
          const uint32_t qz = bz * seg + rz;
          const float fz = (float)((qz << 1) | 1u);
          vz = (T)(g_decode_fma ? std::fmaf(fz, e32, (float)mm[2]) : (float)mm[2] + fz * e32);
        }
      } else {
        auto dv = [](uint64_t a, uint64_t b) { return b ? a / b : UINT64_MAX; };
        auto md = [](uint64_t a, uint64_t b) { return b ? a % b : a; };
        const uint64_t id64 = (uint64_t)id;
        const uint64_t bx = md(id64, bnx), by = md(dv(id64, bnx), bny);
        const uint64_t m64 = msk, s64 = seg;
        const uint64_t r64 = rp;
        const uint64_t rx = r64 & m64, ry = (r64 >> sh) & m64;
        const uint64_t qx = bx * s64 + rx, qy = by * s64 + ry;
        const double fx = (double)((qx << 1) | 1u), fy = (double)((qy << 1) | 1u);
        const double e64 = (double)eb;
        vx = (T)(g_decode_fma ? std::fma(fx, e64, (double)mm[0]) : (double)mm[0] + fx * e64);
        vy = (T)(g_decode_fma ? std::fma(fy, e64, (double)mm[1]) : (double)mm[1] + fy * e64);
        if (h.dim == 3) {
          const uint64_t bz = dv(id64, bnx * bny);
          const uint64_t rz = shr64(r64, sh * 2);
          const uint64_t qz = bz * s64 + rz;
          const double fz = (double)((qz << 1) | 1u);
          vz = (T)(g_decode_fma ? std::fma(fz, e64, (double)mm[2]) : (double)mm[2] + fz * e64);
        }
      }
      x[base + pos] = vx;
      y[base + pos] = vy;
      if (h.dim == 3 && z) z[base + pos] = vz;
    }
  }
  return GPZO_OK;
}

template <typename T>
int decompress_impl(const uint8_t *s, uint64_t bytes, T *x, T *y, T *z,
                    uint64_t cap, int nthreads) {
  Hdr h;
  int rc = parse(s, bytes, h);
  if (rc) return rc;
  if (h.bits != Lay<T>::bits) return GPZO_EINVAL;
  if (!x || !y || (h.dim == 3 && !z) || cap < h.n) return GPZO_EINVAL;
  const int nt = set_threads(nthreads);
  int err = GPZO_OK;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
  for (int64_t c = 0; c < (int64_t)h.G; ++c) {
    int r = decode_chunk<T>(s, bytes, h, (uint64_t)c, x, y, z);
    if (r) {
#pragma omp critical
      err = r;
    }
  }
  return err;
}

// ---------------------------------------------------------------------------
// computeSegSize.
// ---------------------------------------------------------------------------
// sampleMinMaxXYZKernel + reduceMinMax (src/cudaWarpCompress.cu:1216-1418):
// 1024 samples of 256 consecutive points at stride max((N-256)/1024, 1).
// Sample blocks whose window passes N return without writing (:1230); the
// reduction then reads the scratch slot, which the CLI has zero-filled
// (src/main.cpp:318), so a skipped block contributes 0.0 to min and max.
template <typename T>
void sample_minmax(const T *x, const T *y, const T *z, uint64_t n, uint32_t dim, T out[6]) {
  const int L = 256, B = 1024;
  const uint64_t stride = std::max<uint64_t>((n - (uint64_t)L) / (uint64_t)B, 1ull);
  const bool is64 = sizeof(T) == 8;
  T mnx = is64 ? (T)DBL_MAX : (T)FLT_MAX;
  T mx_init = -mnx;
  T v[6] = {mnx, mx_init, mnx, mx_init, mnx, mx_init};
  for (int b = 0; b < B; ++b) {
    const uint64_t st = (uint64_t)b * stride;
    if (st + (uint64_t)L > n) {
      for (int k = 0; k < 6; ++k) v[k] = (k & 1) ? gmax(v[k], (T)0) : gmin(v[k], (T)0);
      continue;
    }
    for (int t = 0; t < L; ++t) {
      v[0] = gmin(v[0], x[st + t]); v[1] = gmax(v[1], x[st + t]);
      v[2] = gmin(v[2], y[st + t]); v[3] = gmax(v[3], y[st + t]);
      if (dim == 3) { v[4] = gmin(v[4], z[st + t]); v[5] = gmax(v[5], z[st + t]); }
    }
  }
  if (dim == 2) { v[4] = 0; v[5] = 0; }  // :1484-1485
  for (int k = 0; k < 6; ++k) out[k] = v[k];
}

// Host arithmetic of computeSegSize (:1488-1554); f64 twin (Double :1488-1553).
int seg_decide_f32(const float mm[6], uint32_t dim, uint32_t seg_in, int rel_mode,
                   float rel_eb, float eb, int safe31, uint32_t *seg_out, int *adjusted) {
  float dx = mm[1] - mm[0], dy = mm[3] - mm[2], dz = mm[5] - mm[4];
  float mean = (dx + dy + dz) / 3.0f;
  float var;
  if (dim == 3) var = ((dx - mean) * (dx - mean) + (dy - mean) * (dy - mean) + (dz - mean) * (dz - mean)) / 3.0f;
  else var = ((dx - mean) * (dx - mean) + (dy - mean) * (dy - mean) + (dz - mean) * (dz - mean)) / 2.0f;
  float sd = std::sqrt(var);
  float ratio = sd / mean;
  float max_range = std::fmax(std::fmax(dx, dy), dz);
  uint32_t seg = seg_in;
  if (seg == 0 && rel_mode) {
    if (ratio < 0.1f) seg = ((double)rel_eb <= 1e-4) ? 32u : 2u;
    else seg = ((double)rel_eb <= 1e-4) ? 4u : 1u;
  }
  if (seg == 0) return GPZO_EINVAL;  // abs mode without a segment size: the reference shifts by -1 (UB)
  const uint64_t limit = safe31 ? 0x7FFFFFFFull : 0xFFFFFFFFull;
  auto total = [&](uint32_t s) {
    uint64_t mb = cvt_u64(std::ceil(max_range / ((float)(2u * s) * eb))) + 1u;
    return dim == 3 ? mb * mb * mb : mb * mb;
  };
  int adj = 0;
  if (total(seg) > limit) {
    uint32_t t = seg;
    for (int i = 0; i < 11; ++i) {
      t *= 2u;
      if (total(t) <= limit) break;
    }
    if (t > 1024u) return GPZO_ESEG;  // :1547-1550 exit(1)
    seg = t;
    adj = 1;
  }
  *seg_out = seg;
  *adjusted = adj;
  return GPZO_OK;
}

int seg_decide_f64(const double mm[6], uint32_t dim, uint32_t seg_in, int rel_mode,
                   double rel_eb, double eb, int safe31, uint32_t *seg_out, int *adjusted) {
  double dx = mm[1] - mm[0], dy = mm[3] - mm[2], dz = mm[5] - mm[4];
  double mean = (dx + dy + dz) / 3.0;
  // The double path divides by 3 for 2D as well (Double :1500-1503).
  double var = ((dx - mean) * (dx - mean) + (dy - mean) * (dy - mean) + (dz - mean) * (dz - mean)) / 3.0;
  double sd = std::sqrt(var);
  double ratio = sd / mean;
  double max_range = std::fmax(std::fmax(dx, dy), dz);
  (void)dim;
  uint32_t seg = seg_in;
  if (seg == 0 && rel_mode) {
    if (ratio < 0.1f) seg = (rel_eb <= 1e-4) ? 32u : 2u;
    else seg = (rel_eb <= 1e-4) ? 4u : 1u;
  }
  if (seg == 0) return GPZO_EINVAL;
  int adj = 0;
  // The reference's guard compares against UINT64_MAX and never fires
  // (Double :1532); only the 31-bit extension mode adjusts here.
  if (safe31) {
    auto total = [&](uint32_t s) {
      uint64_t mb = cvt_u64(std::ceil(max_range / ((double)(2u * s) * eb))) + 1u;
      return dim == 3 ? mb * mb * mb : mb * mb;
    };
    if (total(seg) > 0x7FFFFFFFull) {
      uint32_t t = seg;
      for (int i = 0; i < 11; ++i) {
        t *= 2u;
        if (total(t) <= 0x7FFFFFFFull) break;
      }
      if (t > 1024u) return GPZO_ESEG;
      seg = t;
      adj = 1;
    }
  }
  *seg_out = seg;
  *adjusted = adj;
  return GPZO_OK;
}

// ---------------------------------------------------------------------------
// Generators.
// ---------------------------------------------------------------------------
inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline double u01(uint64_t seed, uint64_t idx) {
  return (double)(mix64(seed * 0x9E3779B97F4A7C15ull + idx * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull) >> 11) *
         (1.0 / 9007199254740992.0);
}
inline double gauss(uint64_t seed, uint64_t idx) {
  double a = 1.0 - u01(seed, 2 * idx), b = u01(seed, 2 * idx + 1);
  return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
}

template <typename T>
void generate(int kind, uint64_t n, uint32_t dim, double lo, double hi, uint64_t seed,
              T *x, T *y, T *z) {
  T *ax[3] = {x, y, z};
  if (kind == 0) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
      for (uint32_t a = 0; a < dim; ++a) ax[a][i] = (T)(lo + (hi - lo) * u01(seed + a, (uint64_t)i));
    return;
  }
  if (kind == 1) {
    // 70 % of points in Gaussian clusters (uniform centres, sigma log-uniform
    // in [0.5, 10] scaled by box/1000, Pareto(1.5) populations), 30 % uniform.
    const double box = hi - lo, sc = box / 1000.0;
    const uint64_t K = std::max<uint64_t>(1, std::min<uint64_t>(20000, n / 7187));
    std::vector<double> cen(3 * K), sig(K), cdf(K);
    double acc = 0;
    for (uint64_t k = 0; k < K; ++k) {
      for (int a = 0; a < 3; ++a) cen[3 * k + a] = lo + box * u01(seed ^ 0xC3, 3 * k + a);
      sig[k] = sc * 0.5 * std::pow(20.0, u01(seed ^ 0x51, k));
      acc += std::pow(1.0 - u01(seed ^ 0x9A, k), -1.0 / 1.5);  // Pareto(1.5) weight
      cdf[k] = acc;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      const uint64_t ui = (uint64_t)i;
      if (u01(seed ^ 0x11, ui) < 0.7) {
        const double pick = u01(seed ^ 0x22, ui) * acc;
        uint64_t k = (uint64_t)(std::lower_bound(cdf.begin(), cdf.end(), pick) - cdf.begin());
        if (k >= K) k = K - 1;
        for (uint32_t a = 0; a < dim; ++a) {
          double v = cen[3 * k + a] + sig[k] * gauss(seed ^ (0x33 + a), ui);
          v = std::min(std::max(v, lo), hi);
          ax[a][i] = (T)v;
        }
      } else {
        for (uint32_t a = 0; a < dim; ++a) ax[a][i] = (T)(lo + box * u01(seed ^ (0x44 + a), ui));
      }
    }
    return;
  }
  // Lattice with jitter: FCC (3D, 4 sites per unit cell) or square (2D),
  // spacing 1, visited through an affine permutation of the site index.
  const double sigma = hi;
  uint64_t cells;
  if (dim == 3) {
    cells = (uint64_t)std::ceil(std::cbrt((double)n / 4.0));
    while (cells * cells * cells * 4 < n) ++cells;
  } else {
    cells = (uint64_t)std::ceil(std::sqrt((double)n));
    while (cells * cells < n) ++cells;
  }
  uint64_t a = (uint64_t)(0.6180339887 * (double)n) | 1ull;
  auto gcd = [](uint64_t p, uint64_t q) { while (q) { uint64_t t = p % q; p = q; q = t; } return p; };
  while (gcd(a, n) != 1) a += 2;
  const uint64_t b = n / 3;
  static const double fcc[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t j = (uint64_t)(((unsigned __int128)a * (uint64_t)i + b) % n);
    double p[3];
    if (dim == 3) {
      const uint64_t cell = j / 4, site = j % 4;
      p[0] = (double)(cell % cells) + fcc[site][0];
      p[1] = (double)((cell / cells) % cells) + fcc[site][1];
      p[2] = (double)(cell / (cells * cells)) + fcc[site][2];
    } else {
      p[0] = (double)(j % cells);
      p[1] = (double)(j / cells);
      p[2] = 0;
    }
    for (uint32_t d = 0; d < dim; ++d) ax[d][i] = (T)(lo + p[d] + sigma * gauss(seed ^ (0x55 + d), (uint64_t)i));
  }
}

template <typename T>
int perm_impl(const T *x, const T *y, const T *z, uint64_t n, uint32_t dim, T eb,
                     uint32_t seg, uint64_t *perm) {
  if (!x || !y || (dim == 3 && !z) || !perm || n == 0 || seg == 0) return GPZO_EINVAL;
  const uint64_t G = (n + kChunk - 1) / kChunk;
  int rc = GPZO_OK;
#pragma omp parallel
  {
    ChunkEnc<T> *e = new ChunkEnc<T>;
#pragma omp for schedule(dynamic, 64)
    for (int64_t c = 0; c < (int64_t)G; ++c) {
      const uint64_t b = (uint64_t)c * kChunk;
      const uint32_t nv = (uint32_t)std::min<uint64_t>(kChunk, n - b);
      encode_chunk<T>(x + b, y + b, dim == 3 ? z + b : nullptr, nv, dim, eb, seg, *e);
      for (uint32_t j = 0; j < nv; ++j) perm[b + j] = b + e->perm[j];
    }
    delete e;
  }
  return rc;
}

}  // namespace

extern "C" {

uint64_t gpzo_stream_bound(uint64_t n, uint32_t dim, uint32_t float_bits) {
  (void)dim;
  const uint64_t G = (n + kChunk - 1) / kChunk;
  const uint64_t hdr = float_bits == 64 ? 32 : 24, meta = float_bits == 64 ? 64 : 36;
  // delta <= 31 planes, counts <= 11 planes, rel <= 31 planes of 128 B, + padding
  return hdr + G * (8 + meta + 31 * 128 + 11 * 128 + 31 * 128 + 16);
}

float gpzo_rel_to_abs_f32(const float *x, const float *y, const float *z, uint64_t n, float rel) {
  // findMinimumValues<float> (include/utils.cuh:44-65): std::min / std::max keep
  // the current value on ties; start from float limits.
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint64_t i = 0; i < n; ++i) {
    const float v[3] = {x[i], y[i], z ? z[i] : 0.0f};
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], v[a]);
      mx[a] = std::max(mx[a], v[a]);
    }
  }
  // convertRelEb<float> (src/main.cpp:35-55), rel already cast to float (:254)
  float xr = mx[0] - mn[0], yr = mx[1] - mn[1], zr = mx[2] - mn[2];
  float r = std::fmax(std::fmax(xr, yr), zr);
  return r * rel;
}

double gpzo_rel_to_abs_f64(const double *x, const double *y, const double *z, uint64_t n, double rel) {
  // findMinimumValues<double> starts from float limits (include/utils.cuh:48-53).
  double mn[3], mx[3];
  for (int a = 0; a < 3; ++a) { mn[a] = (double)FLT_MAX; mx[a] = (double)(-FLT_MAX); }
  for (uint64_t i = 0; i < n; ++i) {
    const double v[3] = {x[i], y[i], z ? z[i] : 0.0};
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], v[a]);
      mx[a] = std::max(mx[a], v[a]);
    }
  }
  double xr = mx[0] - mn[0], yr = mx[1] - mn[1], zr = mx[2] - mn[2];
  double r = std::fmax(std::fmax(xr, yr), zr);
  return r * rel;
}

int gpzo_seg_size_f32(const float *x, const float *y, const float *z, uint64_t n, uint32_t dim,
                      uint32_t seg_in, int rel_mode, float rel_eb, float eb, int safe31,
                      uint32_t *seg_out, int *adjusted) {
  if (!x || !y || (dim == 3 && !z) || !seg_out || !adjusted || n == 0) return GPZO_EINVAL;
  float mm[6];
  sample_minmax<float>(x, y, z, n, dim, mm);
  return seg_decide_f32(mm, dim, seg_in, rel_mode, rel_eb, eb, safe31, seg_out, adjusted);
}

int gpzo_seg_size_f64(const double *x, const double *y, const double *z, uint64_t n, uint32_t dim,
                      uint32_t seg_in, int rel_mode, double rel_eb, double eb, int safe31,
                      uint32_t *seg_out, int *adjusted) {
  if (!x || !y || (dim == 3 && !z) || !seg_out || !adjusted || n == 0) return GPZO_EINVAL;
  double mm[6];
  sample_minmax<double>(x, y, z, n, dim, mm);
  return seg_decide_f64(mm, dim, seg_in, rel_mode, rel_eb, eb, safe31, seg_out, adjusted);
}

int gpzo_compress_f32(const float *x, const float *y, const float *z, uint64_t n, uint32_t dim,
                      float eb, uint32_t seg, uint8_t *out, uint64_t *out_bytes, int nthreads) {
  return compress_impl<float>(x, y, z, n, dim, eb, seg, out, out_bytes, nthreads);
}
int gpzo_compress_f64(const double *x, const double *y, const double *z, uint64_t n, uint32_t dim,
                      double eb, uint32_t seg, uint8_t *out, uint64_t *out_bytes, int nthreads) {
  return compress_impl<double>(x, y, z, n, dim, eb, seg, out, out_bytes, nthreads);
}
int gpzo_decompress_f32(const uint8_t *s, uint64_t bytes, float *x, float *y, float *z,
                        uint64_t cap, int nthreads) {
  return decompress_impl<float>(s, bytes, x, y, z, cap, nthreads);
}
int gpzo_decompress_f64(const uint8_t *s, uint64_t bytes, double *x, double *y, double *z,
                        uint64_t cap, int nthreads) {
  return decompress_impl<double>(s, bytes, x, y, z, cap, nthreads);
}

int gpzo_parse_header(const uint8_t *s, uint64_t bytes, uint32_t *dim, uint64_t *n,
                      uint32_t *float_bits, double *eb, uint32_t *seg) {
  Hdr h;
  int rc = parse(s, bytes, h);
  if (rc) return rc;
  if (dim) *dim = h.dim;
  if (n) *n = h.n;
  if (float_bits) *float_bits = h.bits;
  if (eb) *eb = h.eb;
  if (seg) *seg = h.seg;
  return GPZO_OK;
}

int gpzo_permutation_f32(const float *x, const float *y, const float *z, uint64_t n, uint32_t dim,
                         float eb, uint32_t seg, uint64_t *perm) {
  return perm_impl<float>(x, y, z, n, dim, eb, seg, perm);
}
int gpzo_permutation_f64(const double *x, const double *y, const double *z, uint64_t n,
                         uint32_t dim, double eb, uint32_t seg, uint64_t *perm) {
  return perm_impl<double>(x, y, z, n, dim, eb, seg, perm);
}

int gpzo_padding_mask(const uint8_t *s, uint64_t bytes, uint8_t *mask) {
  Hdr h;
  int rc = parse(s, bytes, h);
  if (rc) return rc;
  memset(mask, 0, bytes);
  const uint64_t meta_base = h.hdr + 8 * h.G;
  const uint64_t pay_base = meta_base + (uint64_t)h.meta * h.G;
  const uint32_t u16_at = h.bits == 64 ? 56 : 28;
  for (uint64_t c = 0; c < h.G; ++c) {
    const uint8_t *m = s + meta_base + c * h.meta + u16_at;
    const uint32_t dbits = get_u16(m), cbits = get_u16(m + 2), U = get_u16(m + 6);
    const uint32_t bpp = (U + 7) >> 3;
    const uint32_t db = section_bytes(U, dbits, h.pad), cb = section_bytes(U, cbits, h.pad);
    const uint64_t off = get_u64(s + h.hdr + 8 * c);
    const uint64_t p = pay_base + off;
    if (p + db + cb > bytes) return GPZO_ESTREAM;
    for (uint64_t i = p + (uint64_t)dbits * bpp; i < p + db; ++i) mask[i] = 1;
    for (uint64_t i = p + db + (uint64_t)cbits * bpp; i < p + db + cb; ++i) mask[i] = 1;
  }
  return GPZO_OK;
}

void gpzo_generate_f32(int kind, uint64_t n, uint32_t dim, double lo, double hi, uint64_t seed,
                       float *x, float *y, float *z) {
  generate<float>(kind, n, dim, lo, hi, seed, x, y, z);
}
void gpzo_generate_f64(int kind, uint64_t n, uint32_t dim, double lo, double hi, uint64_t seed,
                       double *x, double *y, double *z) {
  generate<double>(kind, n, dim, lo, hi, seed, x, y, z);
}

// Switch for pinning the reconstruction arithmetic against reference output
// (1 = fused multiply-add, 0 = separate multiply and add).
void gpzo_set_decode_fma(int on) { g_decode_fma = on ? 1 : 0; }

}  // extern "C"
