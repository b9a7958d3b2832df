// gpz_kernels.cuh -- sm_100a kernels of the B200 GPZ codec.
//
//   seg_sample_kernel   computeSegSize (reference src/cudaWarpCompress.cu:1424-1557)
//   rel_to_abs_kernel   findMinimumValues + convertRelEb (include/utils.cuh:44-65,
//                       src/main.cpp:35-55), on the device
//   compress_kernel     runCompressKernel[2D] + CUB scan + header/meta assembly +
//                       runCompactKernel (src/cudaWarpCompress.cu:32-796, 1620-1702)
//                       fused into one persistent, single-pass kernel
//   (decompress_kernel: gpz_decode.cuh)
//
// float64 twins: src/cudaWarpCompressDouble.cu (same line ranges +/- 3).
#pragma once

#include <cfloat>
#include "gpz_device.cuh"

namespace gpzb {

// ===========================================================================
// Automatic segment size (computeSegSize).
// ===========================================================================
// Host arithmetic of computeSegSize (src/cudaWarpCompress.cu:1488-1554),
// evaluated on the device with explicitly rounded operations so no
// contraction can differ from the reference's host build.
__device__ void seg_decide(const float mm[6], uint32_t dim, uint32_t seg_in, int rel_mode,
                           float rel_eb, float eb, int safe31, Control *ctl) {
  const float dx = __fsub_rn(mm[3], mm[0]), dy = __fsub_rn(mm[4], mm[1]), dz = __fsub_rn(mm[5], mm[2]);
  const float mean = __fdiv_rn(__fadd_rn(__fadd_rn(dx, dy), dz), 3.0f);
  const float ex = __fsub_rn(dx, mean), ey = __fsub_rn(dy, mean), ez = __fsub_rn(dz, mean);
  float var = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
  var = __fdiv_rn(var, dim == 3 ? 3.0f : 2.0f);  // the float 2D path divides by 2 (:1503)
  const float ratio = __fdiv_rn(__fsqrt_rn(var), mean);
  const float maxr = fmaxf(fmaxf(dx, dy), dz);
  uint32_t seg = seg_in;
  if (seg == 0 && rel_mode) {
    if (ratio < 0.1f) seg = ((double)rel_eb <= 1e-4) ? 32u : 2u;
    else seg = ((double)rel_eb <= 1e-4) ? 4u : 1u;
  }
  if (seg == 0) { set_status(ctl, kEINVAL); return; }
  const unsigned long long limit = safe31 ? 0x7FFFFFFFull : 0xFFFFFFFFull;
  auto total = [&](uint32_t s) {
    const unsigned long long mb =
        __float2ull_rz(ceilf(__fdiv_rn(maxr, __fmul_rn(__uint2float_rn(2u * s), eb)))) + 1ull;
    return dim == 3 ? mb * mb * mb : mb * mb;
  };
  uint32_t adj = 0;
  if (total(seg) > limit) {
    uint32_t t = seg;
    for (int i = 0; i < 11; ++i) {
      t *= 2u;
      if (total(t) <= limit) break;
    }
    if (t > 1024u) { set_status(ctl, kESEG); return; }
    seg = t;
    adj = 1;
  }
  ctl->seg = seg;
  ctl->adjusted = adj;
}

// Double twin (src/cudaWarpCompressDouble.cu:1488-1553): variance divides by 3
// for 2D too, and the reference's overflow guard compares with UINT64_MAX and
// never fires; only the 31-bit extension adjusts.
__device__ void seg_decide(const double mm[6], uint32_t dim, uint32_t seg_in, int rel_mode,
                           double rel_eb, double eb, int safe31, Control *ctl) {
  const double dx = __dsub_rn(mm[3], mm[0]), dy = __dsub_rn(mm[4], mm[1]), dz = __dsub_rn(mm[5], mm[2]);
  const double mean = __ddiv_rn(__dadd_rn(__dadd_rn(dx, dy), dz), 3.0);
  const double ex = __dsub_rn(dx, mean), ey = __dsub_rn(dy, mean), ez = __dsub_rn(dz, mean);
  double var = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
  var = __ddiv_rn(var, 3.0);
  const double ratio = __ddiv_rn(__dsqrt_rn(var), mean);
  const double maxr = fmax(fmax(dx, dy), dz);
  uint32_t seg = seg_in;
  if (seg == 0 && rel_mode) {
    if (ratio < (double)0.1f) seg = (rel_eb <= 1e-4) ? 32u : 2u;
    else seg = (rel_eb <= 1e-4) ? 4u : 1u;
  }
  if (seg == 0) { set_status(ctl, kEINVAL); return; }
  uint32_t adj = 0;
  if (safe31) {
    auto total = [&](uint32_t s) {
      const unsigned long long mb =
          __double2ull_rz(ceil(__ddiv_rn(maxr, __dmul_rn(__uint2double_rn(2u * s), eb)))) + 1ull;
      return dim == 3 ? mb * mb * mb : mb * mb;
    };
    if (total(seg) > 0x7FFFFFFFull) {
      uint32_t t = seg;
      for (int i = 0; i < 11; ++i) {
        t *= 2u;
        if (total(t) <= 0x7FFFFFFFull) break;
      }
      if (t > 1024u) { set_status(ctl, kESEG); return; }
      seg = t;
      adj = 1;
    }
  }
  ctl->seg = seg;
  ctl->adjusted = adj;
}

template <typename T>
__device__ __forceinline__ void fold_minmax(T v, typename TT<T>::U &mn_inv, typename TT<T>::U &mx) {
  if (v == v) {
    const typename TT<T>::U o = ord_of(v);
    mn_inv = max(mn_inv, (typename TT<T>::U)~o);
    mx = max(mx, o);
  }
}

// sampleMinMaxXYZKernel[2D] + reduceMinMax[2D] (src/cudaWarpCompress.cu:1216-1418):
// 1024 windows of 256 consecutive points at stride max((N-256)/1024, 1).
// A window that would run past N is skipped by the reference and its
// min/max slot keeps the zero-filled scratch value, so it contributes 0.0.
// Launch: 128 blocks x 256 threads, 8 windows per block.  The last block to
// finish applies the host decision rules (seg_decide).
template <typename T>
__global__ void __launch_bounds__(256) seg_sample_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                         const T *__restrict__ z, uint64_t n, uint32_t dim,
                                                         uint32_t seg_in, int rel_mode, T rel_eb, T eb,
                                                         int safe31, Control *ctl) {
  using U = typename TT<T>::U;
  __shared__ U red[6][8];
  __shared__ int last;
  const unsigned long long L = 256, B = 1024;
  const unsigned long long stride = max((n - L) / B, 1ull);
  U acc[6] = {0, 0, 0, 0, 0, 0};  // [min_inv, max] per axis
  const T *X[3] = {x, y, z};
  for (int w = 0; w < 8; ++w) {
    const unsigned long long win = (unsigned long long)blockIdx.x * 8 + w;
    const unsigned long long st = win * stride;
    if (st + L > n) {
      for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>((T)0, acc[2 * d], acc[2 * d + 1]);
      continue;
    }
    for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>(X[d][st + threadIdx.x], acc[2 * d], acc[2 * d + 1]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const U v = warp_max(acc[k]);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 2 * dim) {
    U v = 0;
    for (int w = 0; w < 8; ++w) v = max(v, red[threadIdx.x][w]);
    atomicMax(&ctl->mm[threadIdx.x], (unsigned long long)v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&ctl->sample_done, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    T mm[6];
    for (uint32_t d = 0; d < 3; ++d) {
      if (d < dim) {
        const U mi = (U)(~(U)((volatile unsigned long long *)ctl->mm)[2 * d]);
        const U ma = (U)((volatile unsigned long long *)ctl->mm)[2 * d + 1];
        mm[d] = from_ord(mi);
        mm[3 + d] = from_ord(ma);
      } else {
        mm[d] = 0;
        mm[3 + d] = 0;
      }
    }
    seg_decide(mm, dim, seg_in, rel_mode, rel_eb, eb, safe31, ctl);
  }
}

// findMinimumValues<T> + convertRelEb<T> on the device.  The host scan starts
// from float limits (include/utils.cuh:48-53) and ignores NaNs; 2D data has
// z == 0 (utils.cuh:141).
template <typename T>
__global__ void __launch_bounds__(256) rel_to_abs_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                         const T *__restrict__ z, uint64_t n, uint32_t dim,
                                                         T rel, Control *ctl) {
  using U = typename TT<T>::U;
  __shared__ U red[6][8];
  __shared__ int last;
  U acc[6];
  // min starts at FLT_MAX and max at -FLT_MAX, as on the host
  for (int d = 0; d < 3; ++d) {
    acc[2 * d] = (U)~ord_of((T)FLT_MAX);
    acc[2 * d + 1] = ord_of((T)(-FLT_MAX));
  }
  const T *X[3] = {x, y, z};
  const unsigned long long step = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step)
    for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>(X[d][i], acc[2 * d], acc[2 * d + 1]);
  if (dim == 2) fold_minmax<T>((T)0, acc[4], acc[5]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const U v = warp_max(acc[k]);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    U v = 0;
    for (int w = 0; w < 8; ++w) v = max(v, red[threadIdx.x][w]);
    atomicMax(&ctl->mm[threadIdx.x], (unsigned long long)v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&ctl->sample_done, 1u) == gridDim.x - 1);
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    T mn[3], mx[3];
    for (int d = 0; d < 3; ++d) {
      mn[d] = from_ord((U)~(U)((volatile unsigned long long *)ctl->mm)[2 * d]);
      mx[d] = from_ord((U)((volatile unsigned long long *)ctl->mm)[2 * d + 1]);
      ctl->out_mm[d] = (double)mn[d];
      ctl->out_mm[3 + d] = (double)mx[d];
    }
    T r;
    if (sizeof(T) == 4) {
      const float xr = __fsub_rn((float)mx[0], (float)mn[0]), yr = __fsub_rn((float)mx[1], (float)mn[1]);
      const float zr = __fsub_rn((float)mx[2], (float)mn[2]);
      r = (T)__fmul_rn(fmaxf(fmaxf(xr, yr), zr), (float)rel);
    } else {
      const double xr = __dsub_rn((double)mx[0], (double)mn[0]), yr = __dsub_rn((double)mx[1], (double)mn[1]);
      const double zr = __dsub_rn((double)mx[2], (double)mn[2]);
      r = (T)__dmul_rn(fmax(fmax(xr, yr), zr), (double)rel);
    }
    ctl->out_eb = (double)r;
  }
}

// ===========================================================================
// Compress.
// ===========================================================================
template <typename T>
struct CArgs {
  const T *x, *y, *z;
  uint8_t *out;
  unsigned long long out_cap;
  Control *ctl;
  unsigned long long *look;  // one look-back word per chunk
  unsigned long long n, G;
  T eb;
  uint32_t dim;
  int vec_ok;  // x, y, z all 16-byte aligned
};

template <typename T>
struct __align__(16) CSmem {
  uint32_t hist[kBuckets / 2 + 16];      // packed 16-bit bucket counts -> starts; later run starts
  unsigned long long tmp[kChunk];        // composites; later delta words [0,1024) + count words [1024,2048)
  uint32_t sortedK[kChunk];
  uint32_t sortedRel[kChunk];            // swizzled
  uint16_t big[kChunk / kSmallBucket + 8];  // buckets ranked by a warp sort
  uint32_t nbig, nwork;
  // payload staging, two chunks in flight; stage[cur] doubles as ranking
  // scratch (relative position by sort rank, work items) until it is packed
  uint32_t stage[2][kStageBytes / 4 + 4];
  uint32_t pmeta[2][16];                 // meta record of the staged chunk
  unsigned long long pchunk[2];          // chunk id of the staged chunk (~0 = none)
  uint32_t ppay[2];                      // payload bytes of the staged chunk
  typename TT<T>::U wmm[6][kWarps];      // per-warp ordered min/max
  uint32_t wk[3][kWarps];                // per-warp key min / key max / rel max
  uint32_t ws1[kWarps];                  // per-warp scan totals / maxima
  uint32_t ws3[kWarps], ws4[kWarps], ws5[kWarps];
  T mm[6];
  unsigned long long bn[2];
  unsigned long long excl;
  uint32_t chunk;
};

constexpr unsigned long long kFlagAgg = 1ull << 62, kFlagInc = 2ull << 62, kValMask = (1ull << 62) - 1;

// Decoupled look-back over the chunk sizes.  A chunk publishes its own
// payload size (aggregate) as soon as it knows it; placing it later
// (resolve_prefix, one CTA iteration afterwards) sums the aggregates of its
// predecessors back to the nearest published inclusive prefix, then
// publishes its own inclusive prefix.
__device__ __forceinline__ void publish_aggregate(unsigned long long *look, unsigned long long c,
                                                  unsigned long long agg) {
  st_relaxed(&look[c], (c == 0 ? kFlagInc : kFlagAgg) | agg);
}

// Warp-collective.  Returns false when a bounded wait gave up or another CTA
// aborted (the kernel then stops taking chunks and reports GPZ_ETIMEOUT).
__device__ bool resolve_prefix(unsigned long long *look, unsigned long long c, unsigned long long agg,
                               Control *ctl, unsigned long long &excl_out) {
  const int lane = threadIdx.x & 31;
  if (c == 0) {
    excl_out = 0;
    return true;
  }
  unsigned long long excl = 0;
  long long top = (long long)c - 1;
  uint32_t spins = 0, backoff = 32;
  while (true) {
    const long long idx = top - lane;
    const unsigned long long v = idx >= 0 ? ld_relaxed(&look[idx]) : kFlagInc;
    const uint32_t fl = (uint32_t)(v >> 62);
    const uint32_t mInc = __ballot_sync(0xFFFFFFFFu, fl == 2u);
    const uint32_t mNone = __ballot_sync(0xFFFFFFFFu, fl == 0u);
    const uint32_t need = mInc ? (((mInc & (0u - mInc)) << 1) - 1u) : 0xFFFFFFFFu;
    if (mNone & need) {
      if (++spins > kSpinLimit || ld_volatile(&ctl->abort)) {
        if (lane == 0) {
          atomicExch(&ctl->abort, 1u);
          set_status(ctl, kETIMEOUT);
        }
        return false;
      }
      __nanosleep(backoff);
      backoff = min(backoff * 2, 256u);
      continue;
    }
    unsigned long long add = ((need >> lane) & 1u) ? (v & kValMask) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xFFFFFFFFu, add, o);
    excl += add;
    if (mInc) break;
    top -= 32;
  }
  if (lane == 0) st_relaxed(&look[c], kFlagInc | (excl + agg));
  excl_out = excl;
  return true;
}

// Ascending in-place sort of a[0..n) by one warp: a bitonic network in the
// variant whose compare-exchanges all put the minimum at the lower index (the
// first step of each merge compares mirrored positions), so the array is
// virtually padded with +inf up to a power of two and any exchange that
// touches the padding is skipped.  Used for large ranking buckets.
__device__ void warp_bitonic_u64(unsigned long long *a, int n) {
  const int lane = threadIdx.x & 31;
  int P = 2;
  while (P < n) P <<= 1;
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < (P >> 1); q += 32) {
        const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));
        const int p = (j == (k >> 1)) ? (i ^ (k - 1)) : (i + j);
        if (p < n) {
          const unsigned long long x = a[i], y = a[p];
          if (y < x) {
            a[i] = y;
            a[p] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Writes the plane words of one 32-element group into the staging buffer.
// Byte sections (deltas, counts): plane pi occupies bytes [pi*bpp, (pi+1)*bpp)
// of the section, MSB plane first (src/cudaWarpCompress.cu:357-408).
__device__ __forceinline__ void put_byte_word(uint8_t *stage8, uint32_t sec_off, uint32_t bpp, uint32_t pi,
                                              int g, uint32_t word) {
  const uint32_t w = to_msb_bytes(word);
  const uint32_t base = sec_off + pi * bpp + 4u * g;
  const uint32_t room = bpp - 4u * g;  // > 0 for every group that holds elements
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if ((uint32_t)j < room) stage8[base + j] = (uint8_t)(w >> (8 * j));
}

template <typename T>
__device__ void pack_unit(CSmem<T> &s, uint32_t *stage, int unit, uint32_t U, uint32_t dbits, uint32_t cbits,
                          uint32_t rbits, uint32_t dbytes, uint32_t cbytes) {
  const uint32_t ng = (U + 31u) >> 5;
  const uint32_t hd = dbits ? (dbits > 16 ? 2u : 1u) * ng : 0u;
  const uint32_t hc = cbits ? (cbits > 16 ? 2u : 1u) * ng : 0u;
  const uint32_t hr = rbits ? (rbits > 16 ? 64u : 32u) : 0u;
  uint32_t u = (uint32_t)unit;
  int sec;
  uint32_t nb;
  const uint32_t *src;
  if (u < hd) { sec = 0; nb = dbits; src = reinterpret_cast<const uint32_t *>(s.tmp); }
  else if ((u -= hd) < hc) { sec = 1; nb = cbits; src = reinterpret_cast<const uint32_t *>(s.tmp) + kChunk; }
  else if ((u -= hc) < hr) { sec = 2; nb = rbits; src = s.sortedRel; }
  else return;
  const uint32_t groups = sec == 2 ? 32u : ng;
  const int g = (int)(u % groups);
  const int half = (int)(u / groups);
  uint32_t a[32];
  load_group(src, g, a);
  uint32_t b0, cnt;
  if (nb <= 8) { transpose_lo8(a); b0 = 0; cnt = nb; }
  else if (half == 0) { transpose_lo16(a); b0 = 0; cnt = min(nb, 16u); }
  else { transpose_hi16(a); b0 = 16; cnt = nb - 16; }
  uint8_t *stage8 = reinterpret_cast<uint8_t *>(stage);
  const uint32_t bpp = (U + 7u) >> 3;
  const uint32_t sec_off = sec == 0 ? 0u : dbytes;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if ((uint32_t)k < cnt) {
      const uint32_t b = b0 + k;
      const uint32_t pi = nb - 1u - b;
      if (sec == 2) stage[((dbytes + cbytes) >> 2) + pi * 32u + g] = a[k];
      else put_byte_word(stage8, sec_off, bpp, pi, g, a[k]);
    }
  }
}

// Places the chunk staged in slot `sl` (warp 0): resolves its stream offset,
// writes its offset-table entry (:1679), meta record and -- for chunk 0 -- the
// header (:1674-1678; Double :1672-1680).  The staged copy-out follows after
// the next CTA barrier.
template <typename T>
__device__ void place_staged(CSmem<T> &s, int sl, const CArgs<T> &a, unsigned long long G,
                             unsigned long long pay_base, uint32_t seg, Control *ctl) {
  using Tr = TT<T>;
  constexpr bool is64 = sizeof(T) == 8;
  const int lane = threadIdx.x & 31;
  const unsigned long long c = s.pchunk[sl];
  if (c == ~0ull) return;
  const uint32_t payload = s.ppay[sl];
  unsigned long long excl = 0;
  const bool ok = resolve_prefix(a.look, c, payload, ctl, excl);
  if (lane == 0) s.excl = ok ? excl : ~0ull;
  if (!ok) return;
  if (lane == 0) reinterpret_cast<unsigned long long *>(a.out + Tr::hdr)[c] = excl;
  uint8_t *meta = a.out + Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * c;
  if (!is64) {
    if (lane < 9) reinterpret_cast<uint32_t *>(meta)[lane] = s.pmeta[sl][lane];
  } else {
    if (lane < 8)
      reinterpret_cast<unsigned long long *>(meta)[lane] =
          (unsigned long long)s.pmeta[sl][2 * lane] | ((unsigned long long)s.pmeta[sl][2 * lane + 1] << 32);
  }
  if (c == 0) {
    uint32_t *h = reinterpret_cast<uint32_t *>(a.out);
    if (lane == 0) h[0] = a.dim;
    if (lane == 1) h[1] = (uint32_t)a.n;
    if (lane == 2) h[2] = (uint32_t)(a.n >> 32);
    if (lane == 3) h[3] = Tr::bits;
    if (!is64) {
      if (lane == 4) h[4] = __float_as_uint((float)a.eb);
      if (lane == 5) h[5] = seg;
    } else {
      if (lane == 4)
        reinterpret_cast<unsigned long long *>(a.out)[2] = (unsigned long long)__double_as_longlong((double)a.eb);
      if (lane == 6) h[6] = seg;
      if (lane == 7) h[7] = 32u;
    }
  }
  if (c == G - 1 && lane == 0) ctl->stream_bytes = pay_base + excl + payload;
}

// All threads: copies the staged payload of slot `sl` to its stream offset.
template <typename T>
__device__ void copy_out_staged(CSmem<T> &s, int sl, const CArgs<T> &a, unsigned long long pay_base) {
  const unsigned long long c = s.pchunk[sl];
  if (c == ~0ull) return;
  const unsigned long long excl = s.excl;
  const uint32_t payload = s.ppay[sl];
  if (excl != ~0ull) {
    if (pay_base + excl + payload > a.out_cap) {
      if (threadIdx.x == 0) set_status(a.ctl, kENOSPACE);
    } else {
      uint32_t *dst = reinterpret_cast<uint32_t *>(a.out + pay_base + excl);
      for (uint32_t w = threadIdx.x; w < payload / 4u; w += kThreads) dst[w] = s.stage[sl][w];
    }
  }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(kThreads, kCompressMinBlocks) compress_kernel(const CArgs<T> a) {
  using Tr = TT<T>;
  using U = typename Tr::U;
  constexpr bool is64 = sizeof(T) == 8;
  __shared__ CSmem<T> s;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  Control *ctl = a.ctl;
  if (ld_volatile(reinterpret_cast<const uint32_t *>(&ctl->status)) != 0) return;
  const uint32_t seg = ctl->seg;
  const uint32_t sh = (uint32_t)__ffs((int)seg) - 1u, msk = seg - 1u;
  const T eb = a.eb;
  const T inv = is64 ? (T)__ddiv_rn(1.0, __dmul_rn(2.0, (double)eb)) : (T)__fdiv_rn(1.0f, __fmul_rn(2.0f, (float)eb));
  constexpr uint32_t dim = DIM;
  const unsigned long long G = a.G, n = a.n;
  const unsigned long long pay_base = Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * G;
  const T *const X[3] = {a.x, a.y, a.z};

  if (t == 0) {
    s.chunk = atomicAdd(&ctl->chunk_ctr, 1u);
    s.pchunk[0] = s.pchunk[1] = ~0ull;
  }
  __syncthreads();
  // Iteration k computes chunk c_k into stage[k & 1] and places chunk c_{k-1}
  // (look-back + copy-out), so no CTA waits on its neighbours' sizes.
  uint32_t it = 0;
  for (;; ++it) {
    const unsigned long long c = s.chunk;
    const int cur = (int)(it & 1u), prv = cur ^ 1;
    if (c >= G) break;
    const unsigned long long base = c * kChunk;
    const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, n - base);

    // ---- load, chunk min/max (:104-139) ----
    T v[3][4] = {};
    if (nvalid == (uint32_t)kChunk && a.vec_ok) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        if (!is64) {
          const float4 q = reinterpret_cast<const float4 *>(X[d] + base)[t];
          v[d][0] = (T)q.x; v[d][1] = (T)q.y; v[d][2] = (T)q.z; v[d][3] = (T)q.w;
        } else {
          const double2 q0 = reinterpret_cast<const double2 *>(X[d] + base)[2 * t];
          const double2 q1 = reinterpret_cast<const double2 *>(X[d] + base)[2 * t + 1];
          v[d][0] = (T)q0.x; v[d][1] = (T)q0.y; v[d][2] = (T)q1.x; v[d][3] = (T)q1.y;
        }
      }
    } else {
#pragma unroll
      for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const uint32_t p = 4 * t + e;
          v[d][e] = p < nvalid ? X[d][base + p] : (T)0;
        }
    }
    {
      // fminf / fmaxf ignore NaN and order -0.0 below +0.0, as the reference's
      // warp reductions do (:122-139); one ordered-int transform per axis for REDUX
      const T lim = is64 ? (T)DBL_MAX : (T)FLT_MAX;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        T mn = lim, mxv = -lim;
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (4u * t + e < nvalid) { mn = fmin(mn, v[d][e]); mxv = fmax(mxv, v[d][e]); }
        const U a0 = warp_max((U)~ord_of(mn)), a1 = warp_max(ord_of(mxv));
        if (lane == 0) { s.wmm[2 * d][warp] = a0; s.wmm[2 * d + 1][warp] = a1; }
      }
    }
    __syncthreads();  // B1
    if (t < 3) {
      if ((uint32_t)t < dim) {
        U a0 = 0, a1 = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) { a0 = max(a0, s.wmm[2 * t][w]); a1 = max(a1, s.wmm[2 * t + 1][w]); }
        const T mn = from_ord((U)~a0), mxv = from_ord(a1);
        s.mm[t] = mn;
        s.mm[3 + t] = mxv;
        const T range = is64 ? (T)__dsub_rn((double)mxv, (double)mn) : (T)__fsub_rn((float)mxv, (float)mn);
        if (t == 0) s.bn[0] = block_num(range, seg, eb, is64 && dim == 2);
        if (t == 1) s.bn[1] = block_num(range, seg, eb, false);
      } else {
        s.mm[2] = (T)0;  // 2D meta carries z = 0 (:518, :521)
        s.mm[5] = (T)0;
      }
    }
    for (int i = t; i < kBuckets / 2 + 1; i += kThreads) s.hist[i] = 0;
    __syncthreads();  // B2

    // ---- quantize, block id, relative position (:141-205) ----
    uint32_t key[4], rel[4], r[4];
    uint32_t kmin = 0xFFFFFFFFu, kmax = 0u, rmax = 0u;
    {
      T nmn[3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        nmn[d] = is64 ? (T)__dmul_rn(-(double)s.mm[d], (double)inv) : (T)__fmul_rn(-(float)s.mm[d], (float)inv);
      const unsigned long long bnx = s.bn[0], bny = s.bn[1];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t p = 4 * t + e;
        r[e] = (p & 31u) * 32u + (p >> 5);
        if (!is64) {
          const uint32_t bx = (uint32_t)bnx, bxy = (uint32_t)bnx * (uint32_t)bny;
          const uint32_t qx = __float2uint_rz(__fmaf_rn((float)v[0][e], (float)inv, (float)nmn[0]));
          const uint32_t qy = __float2uint_rz(__fmaf_rn((float)v[1][e], (float)inv, (float)nmn[1]));
          if (dim == 3) {
            const uint32_t qz = __float2uint_rz(__fmaf_rn((float)v[2][e], (float)inv, (float)nmn[2]));
            key[e] = ((qx >> sh) + (qy >> sh) * bx + (qz >> sh) * bxy) & 0x7FFFFFFFu;
            rel[e] = ((qx & msk) + (qy & msk) * seg + (qz & msk) * (seg * seg)) & 0x7FFFFFFFu;
          } else {
            key[e] = ((qx >> sh) + (qy >> sh) * bx) & 0x7FFFFFFFu;
            rel[e] = ((qx & msk) + (qy & msk) * seg) & 0x7FFFFFFFu;
          }
        } else {
          // All arithmetic below is mod 2^32 of the reference's u64 expression,
          // which is exact because the result is masked to 31 bits.
          const unsigned long long qx = __double2ull_rz(__fma_rn((double)v[0][e], (double)inv, (double)nmn[0]));
          const unsigned long long qy = __double2ull_rz(__fma_rn((double)v[1][e], (double)inv, (double)nmn[1]));
          const uint32_t bx = (uint32_t)bnx;
          if (dim == 3) {
            const unsigned long long qz = __double2ull_rz(__fma_rn((double)v[2][e], (double)inv, (double)nmn[2]));
            const uint32_t bxy = (uint32_t)(bnx * bny);
            key[e] = ((uint32_t)(qx >> sh) + (uint32_t)(qy >> sh) * bx + (uint32_t)(qz >> sh) * bxy) & 0x7FFFFFFFu;
            rel[e] = ((uint32_t)(qx & msk) + (uint32_t)(qy & msk) * seg + (uint32_t)(qz & msk) * seg * seg) &
                     0x7FFFFFFFu;
          } else {
            key[e] = ((uint32_t)(qx >> sh) + (uint32_t)(qy >> sh) * bx) & 0x7FFFFFFFu;
            rel[e] = ((uint32_t)(qx & msk) + (uint32_t)(qy & msk) * seg) & 0x7FFFFFFFu;
          }
        }
        if (p < nvalid) {
          kmin = min(kmin, key[e]);
          kmax = max(kmax, key[e]);
          rmax = max(rmax, rel[e]);
        }
      }
      if (t == 0) {
        // block-id overflow check on the chunk's largest quantized corner
        unsigned long long qm[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          qm[d] = is64 ? __double2ull_rz(__fma_rn((double)s.mm[3 + d], (double)inv, (double)nmn[d]))
                       : (unsigned long long)__float2uint_rz(__fmaf_rn((float)s.mm[3 + d], (float)inv, (float)nmn[d]));
        const unsigned long long bound = (qm[0] >> sh) + (qm[1] >> sh) * bnx + (dim == 3 ? (qm[2] >> sh) * bnx * bny : 0ull);
        if (bound > 0x7FFFFFFFull) ctl->id_overflow = 1u;
      }
    }
    {
      const uint32_t a0 = warp_min(kmin), a1 = warp_max(kmax), a2 = warp_max(rmax);
      if (lane == 0) { s.wk[0][warp] = a0; s.wk[1][warp] = a1; s.wk[2][warp] = a2; }
    }
    __syncthreads();  // B3
    kmin = warp_min(lane < kWarps ? s.wk[0][lane & 7] : 0xFFFFFFFFu);
    kmax = warp_max(lane < kWarps ? s.wk[1][lane & 7] : 0u);
    rmax = warp_max(lane < kWarps ? s.wk[2][lane & 7] : 0u);
    const uint32_t rbits = max(bitlen(rmax), nvalid < (uint32_t)kChunk ? 1u : 0u);  // :200-201

    // ---- ranking: bucket the unique composite (block id, rank) ----
    const unsigned long long cmax = ((unsigned long long)(kmax - kmin) << 10) | 1023ull;
    const uint32_t shb = (uint32_t)max(0, (int)bitlen64(cmax) - kBucketBits);
    unsigned long long C[4];
    uint32_t bk[4], slot[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool valid = 4u * t + e < nvalid;
      C[e] = ((unsigned long long)(key[e] - kmin) << 10) | r[e];
      bk[e] = valid ? (uint32_t)(C[e] >> shb) : 0u;  // < kBuckets for every valid point
      if (valid) {
        const uint32_t h = 16u * (bk[e] & 1u);
        slot[e] = (atomicAdd(&s.hist[bk[e] >> 1], 1u << h) >> h) & 0xFFFFu;
      }
    }
    __syncthreads();  // B4
    // exclusive scan of the bucket counts (16-bit, two per word); thread t owns
    // buckets 16t..16t+15
    {
      constexpr int BPT = kBuckets / kThreads;
      const uint4 h0 = reinterpret_cast<const uint4 *>(s.hist)[2 * t];
      const uint4 h1 = reinterpret_cast<const uint4 *>(s.hist)[2 * t + 1];
      const uint32_t w[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
      uint32_t tot = 0;
      uint32_t o[8];
      uint32_t bigmask = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t c0 = w[q] & 0xFFFFu, c1 = w[q] >> 16;
        o[q] = tot | ((tot + c0) << 16);
        tot += c0 + c1;
        bigmask |= (c0 > (uint32_t)kSmallBucket ? 1u : 0u) << (2 * q);
        bigmask |= (c1 > (uint32_t)kSmallBucket ? 1u : 0u) << (2 * q + 1);
      }
      uint32_t inc = tot;
#pragma unroll
      for (int q = 1; q < 32; q <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, q);
        if (lane >= q) inc += v;
      }
      if (lane == 31) s.ws1[warp] = inc;
      if (t == 0) { s.nbig = 0; s.nwork = 0; }
      __syncthreads();  // B5
      const uint32_t base = __reduce_add_sync(0xFFFFFFFFu, lane < warp ? s.ws1[lane & 7] : 0u) + inc - tot;
      const uint32_t b2 = base | (base << 16);
#pragma unroll
      for (int q = 0; q < 8; ++q) o[q] += b2;
      reinterpret_cast<uint4 *>(s.hist)[2 * t] = make_uint4(o[0], o[1], o[2], o[3]);
      reinterpret_cast<uint4 *>(s.hist)[2 * t + 1] = make_uint4(o[4], o[5], o[6], o[7]);
      if (t == kThreads - 1) s.hist[kBuckets / 2] = base + tot;
      while (bigmask) {
        const int q = __ffs(bigmask) - 1;
        bigmask &= bigmask - 1;
        s.big[atomicAdd(&s.nbig, 1u)] = (uint16_t)(BPT * t + q);
      }
    }
    __syncthreads();  // B6
    const uint16_t *const bstart = reinterpret_cast<const uint16_t *>(s.hist);  // start of bucket b; b+1 = end
    uint32_t *const relR = s.stage[cur];             // relative position by sort rank r
    uint32_t *const work = s.stage[cur] + kChunk;    // own slot | start << 11 | len << 22
    // scatter into bucket slices; a point alone in its bucket is placed at
    // once, points of 2..16-point buckets become work items
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      uint32_t item = 0;
      bool is_work = false;
      if (4u * t + e < nvalid) {
        const uint32_t st = bstart[bk[e]], len = bstart[bk[e] + 1] - st;
        if (len == 1) {
          s.sortedK[st] = key[e];
          s.sortedRel[swz(st)] = rel[e];
        } else {
          s.tmp[st + slot[e]] = C[e];
          relR[r[e]] = rel[e];
          is_work = len <= (uint32_t)kSmallBucket;
          item = (st + slot[e]) | (st << 11) | (len << 22);
        }
      }
      // warp-aggregated append to the work list
      const uint32_t m = __ballot_sync(0xFFFFFFFFu, is_work);
      uint32_t at = 0;
      if (lane == 0 && m) at = atomicAdd(&s.nwork, (uint32_t)__popc(m));
      at = __shfl_sync(0xFFFFFFFFu, at, 0);
      if (is_work) work[at + __popc(m & ((1u << lane) - 1u))] = item;
    }
    __syncthreads();  // B7
    // work items: rank = number of smaller composites in the bucket
    for (uint32_t i = t; i < s.nwork; i += kThreads) {
      const uint32_t wi = work[i];
      const uint32_t own = wi & 0x7FFu, st = (wi >> 11) & 0x7FFu, len = wi >> 22;
      const unsigned long long cv = s.tmp[own];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < len; ++j) rank += (s.tmp[st + j] < cv) ? 1u : 0u;
      const uint32_t pos = st + rank;
      s.sortedK[pos] = kmin + (uint32_t)(cv >> 10);
      s.sortedRel[swz(pos)] = relR[cv & 1023u];
    }
    // large buckets: one warp sorts each slice in place
    for (uint32_t bi = warp; bi < s.nbig; bi += kWarps) {
      const uint32_t b = s.big[bi];
      const uint32_t st = bstart[b], n_b = bstart[b + 1] - st;
      warp_bitonic_u64(s.tmp + st, (int)n_b);
      for (uint32_t i = lane; i < n_b; i += 32) {
        const unsigned long long cv = s.tmp[st + i];
        s.sortedK[st + i] = kmin + (uint32_t)(cv >> 10);
        s.sortedRel[swz(st + i)] = relR[cv & 1023u];
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint32_t pos = 4 * t + e;
      if (pos >= nvalid) s.sortedRel[swz(pos)] = 0xFFFFFFFFu;  // invalid slots (:197)
    }
    __syncthreads();  // B8

    // ---- runs: unique ids, deltas, counts (:222-311) ----
    uint32_t* const runStart = s.hist;
    uint32_t* const deltaA = reinterpret_cast<uint32_t *>(s.tmp);
    uint32_t* const countA = deltaA + kChunk;
    uint32_t Ucnt, dbits, cbits;
    {
      const uint4 k4 = reinterpret_cast<const uint4 *>(s.sortedK)[t];
      const uint32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
      const uint32_t prev = t > 0 ? s.sortedK[4 * t - 1] : 0u;
      uint32_t f = 0, dm = 0, cnt = 0;
      uint32_t dl[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t pos = 4 * t + e;
        const uint32_t pk = e ? kk[e - 1] : prev;
        const bool fl = pos < nvalid && (pos == 0 || kk[e] != pk);
        dl[e] = pos == 0 ? 0u : kk[e] - pk;
        if (fl) { f |= 1u << e; ++cnt; dm = max(dm, bitlen(dl[e])); }
      }
      uint32_t inc = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t q = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += q;
      }
      const uint32_t wd = warp_max(dm);
      if (lane == 31) { s.ws3[warp] = inc; s.ws4[warp] = wd; }
      __syncthreads();  // B9
      const uint32_t w3 = lane < kWarps ? s.ws3[lane & 7] : 0u;
      const uint32_t pre = __reduce_add_sync(0xFFFFFFFFu, lane < warp ? w3 : 0u);
      Ucnt = __reduce_add_sync(0xFFFFFFFFu, w3);
      dbits = warp_max(lane < kWarps ? s.ws4[lane & 7] : 0u);
      uint32_t u = pre + inc - cnt;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (f & (1u << e)) {
          runStart[u] = 4 * t + e;
          deltaA[swz(u)] = dl[e];
          ++u;
        }
      if (t == 0) runStart[Ucnt] = nvalid;
    }
    __syncthreads();  // B10
    {
      uint32_t cm = 0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t u = 4 * t + e;
        if (u < Ucnt) {
          const uint32_t cv = runStart[u + 1] - runStart[u];
          countA[swz(u)] = cv;
          cm = max(cm, bitlen(cv));
        } else {
          countA[swz(u)] = 0u;
          deltaA[swz(u)] = 0u;
        }
      }
      cm = warp_max(cm);
      if (lane == 0) s.ws5[warp] = cm;
    }
    __syncthreads();  // B11
    cbits = warp_max(lane < kWarps ? s.ws5[lane & 7] : 0u);

    const uint32_t dbytes = section_bytes(Ucnt, dbits, Tr::pad);
    const uint32_t cbytes = section_bytes(Ucnt, cbits, Tr::pad);
    const uint32_t rbytes = rel_section_bytes(rbits, Tr::pad);
    const uint32_t payload = dbytes + cbytes + rbytes;

    // ---- publish this chunk's size; place the previous chunk while the other
    //      warps pack this one's bit planes ----
    if (warp == 0) {
      if (lane == 0) publish_aggregate(a.look, c, payload);
      place_staged<T>(s, prv, a, G, pay_base, seg, ctl);
    } else {
      pack_unit<T>(s, s.stage[cur], t - 32, Ucnt, dbits, cbits, rbits, dbytes, cbytes);
      if (t == kThreads - 1) {
        // section padding is zero (the reference leaves it unwritten)
        uint8_t *stage8 = reinterpret_cast<uint8_t *>(s.stage[cur]);
        const uint32_t bpp = (Ucnt + 7u) >> 3;
        for (uint32_t i = dbits * bpp; i < dbytes; ++i) stage8[i] = 0;
        for (uint32_t i = dbytes + cbits * bpp; i < dbytes + cbytes; ++i) stage8[i] = 0;
        // meta record (:332-344 / Double :333-345) for placement next iteration
        uint32_t *m = s.pmeta[cur];
        if (!is64) {
#pragma unroll
          for (int k = 0; k < 6; ++k) m[k] = __float_as_uint((float)s.mm[k]);
          m[6] = s.sortedK[0];
          m[7] = dbits | (cbits << 16);
          m[8] = rbits | (Ucnt << 16);
        } else {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const unsigned long long b = (unsigned long long)__double_as_longlong((double)s.mm[k]);
            m[2 * k] = (uint32_t)b;
            m[2 * k + 1] = (uint32_t)(b >> 32);
          }
          m[12] = s.sortedK[0];
          m[13] = 0;
          m[14] = dbits | (cbits << 16);
          m[15] = rbits | (Ucnt << 16);
        }
        s.pchunk[cur] = c;
        s.ppay[cur] = payload;
      }
      if (t == kThreads - 2) s.chunk = ld_volatile(&ctl->abort) ? 0xFFFFFFFFu : atomicAdd(&ctl->chunk_ctr, 1u);
    }
    __syncthreads();  // B12 (also publishes the next chunk id)
    copy_out_staged<T>(s, prv, a, pay_base);
  }
  // drain: the chunk computed in the last iteration is still staged
  if (it > 0) {
    const int sl = (int)((it - 1u) & 1u);
    if (warp == 0) place_staged<T>(s, sl, a, G, pay_base, seg, ctl);
    __syncthreads();
    copy_out_staged<T>(s, sl, a, pay_base);
  }
  rewind_work_counter(ctl);
}

}  // namespace gpzb
