// gpz_encode.cuh -- compress kernel of the B200 GPZ codec.
//
//   compress_kernel   runCompressKernel[2D] + CUB scan + header/meta assembly
//                     + runCompactKernel (reference src/cudaWarpCompress.cu:32-796,
//                     1620-1702; float64 twin src/cudaWarpCompressDouble.cu)
//                     fused into one persistent, single-pass kernel.
//
// One warp encodes one 1024-point chunk.  Lane l holds the 32 points whose
// stable rank r(p) = (p % 32) * 32 + p / 32 (the reference's sort order for
// equal block ids) is 32l..32l+31, so the composite (block id, r) is unique
// and a point's register index is its rank within the lane.  The warp:
//   1. loads and quantizes one axis at a time (block id in registers, the
//      relative position accumulated in a shared row per lane);
//   2. ranks the composites (block id - kmin) << 10 | r through 2048 buckets
//      on their top bits (shared-atomic counts, placement by bucket start +
//      arrival slot, multi-point buckets put in order afterwards) when they
//      span 21 bits or more; a data-independent warp sort of the 1024 values
//      (odd-even merge sort of each lane's 32, then bitonic merges across
//      lanes on the transposed matrix) ranks narrower ones and the 32-bit
//      chunks the buckets decline;
//   3. finds the runs of equal ids (unique ids, deltas, counts) and compacts
//      them through shared memory so lane l holds runs 32l..32l+31;
//   4. reports its payload size, then transposes deltas, counts and relative
//      positions into bit planes in registers and assembles the payload in
//      its shared region.
// The 8 warps of a CTA take 8 consecutive chunks (a group) together, with
// three CTA barriers per group: B0 before the next group is claimed, B1 once
// every payload size is known (warp 0 then publishes the group's aggregate),
// B2 once warp 0, after building its own planes, has resolved the group's
// stream offset (one decoupled look-back per group); each warp then copies
// its payload out while the next chunk's loads are in flight.
#pragma once

#include <cfloat>
#include <type_traits>
#include "gpz_kernels.cuh"

namespace gpzb {

#ifndef GPZ_ENC_MIN_CTAS
#define GPZ_ENC_MIN_CTAS 2                // resident CTAs per SM the register budget is sized for
#endif
#ifndef GPZ_ENC_WARPS
#define GPZ_ENC_WARPS 8
#endif
#ifndef GPZ_ENC_WARPS_F64_3D
#define GPZ_ENC_WARPS_F64_3D 6
#endif
constexpr int kEncWarps = GPZ_ENC_WARPS;  // chunks (warps) per CTA
constexpr int kEncBucketBits = 11;        // ranking buckets per chunk: 2048
constexpr int kEncSmall = 16;             // buckets of this many points or more are sorted by the whole warp
constexpr uint32_t kEncBucketBackoff = 8; // chunks ranked by the warp sort alone after a declined one
constexpr int kEncWords = 3 * kChunk;     // per-warp shared words (12 KB)
static_assert(kStageBytes <= kEncWords * 4, "payload staging must fit the warp region");

// Chunks (warps) per CTA of compress_kernel<T, DIM>: float64 3D streams use
// 6 (about 170 registers a thread, where 8 warps spill: FCC 200M 4.6 -> 4.1
// ms), the others 8 (6 measured slower for float32 and float64 2D).
template <typename T, int DIM>
constexpr int enc_warps() { return (sizeof(T) == 8 && DIM == 3) ? GPZ_ENC_WARPS_F64_3D : kEncWarps; }

// Per-CTA state of the group of W consecutive chunks a CTA encodes.
template <int W>
struct EncGroupT {
  uint32_t sz[W];            // payload bytes of each warp's chunk
  unsigned long long goff;   // stream offset of the group (~0: look-back gave up)
  unsigned long long next;   // first chunk of the next group
};

template <int W = kEncWarps>
constexpr size_t enc_smem_bytes() { return (size_t)W * kEncWords * 4; }

// Index of bucket-count word w, position / run u, ... in a swizzled 1024-word
// array (rows of 32 words, 16-byte quads XORed by the row).
__device__ __forceinline__ uint32_t sx(uint32_t i) { return (uint32_t)swz((int)i); }

// Ascending in-place bitonic sort of the n = hi - lo values a[sx(lo..hi)) by
// one warp (variant whose exchanges all put the minimum at the lower index,
// virtually padded with +inf up to a power of two).
static __device__ void warp_bitonic_u32(uint32_t *a, uint32_t lo, uint32_t n, int lane) {
  uint32_t P = 2;
  while (P < n) P <<= 1;
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t q = lane; q < (P >> 1); q += 32) {
        const uint32_t i = ((q & ~(j - 1)) << 1) | (q & (j - 1));
        const uint32_t p = (j == (k >> 1)) ? (i ^ (k - 1)) : (i + j);
        if (p < n) {
          const uint32_t x = a[sx(lo + i)], y = a[sx(lo + p)];
          if (y < x) {
            a[sx(lo + i)] = y;
            a[sx(lo + p)] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Batcher's odd-even merge sort network on 32 registers (191 exchanges).
__host__ __device__ __forceinline__ void oem_sort32(uint32_t (&a)[32]) {
#pragma unroll
  for (int p = 1; p < 32; p <<= 1)
#pragma unroll
    for (int k = p; k >= 1; k >>= 1)
#pragma unroll
      for (int j = k % p; j + k < 32; j += 2 * k)
#pragma unroll
        for (int i = 0; i < k; ++i)
          if (i + j + k < 32 && (i + j) / (2 * p) == (i + j + k) / (2 * p)) {
            const uint32_t x = a[i + j], y = a[i + j + k];
            a[i + j] = x < y ? x : y;
            a[i + j + k] = x < y ? y : x;
          }
}

__device__ __forceinline__ void cas_up(uint32_t &x, uint32_t &y) {
  const uint32_t lo = min(x, y);
  y = max(x, y);
  x = lo;
}

// Row <-> column transposes of the warp's 32x32 value matrix through a
// 1024-word swizzled scratch (row l = lane l's registers).  Column reads and
// writes touch one row per instruction, so all 32 banks; c[t] is the lane's
// column offset inside rows with (row & 7) == t.
__device__ __forceinline__ void column_offsets(uint32_t (&c)[8], int lane) {
#pragma unroll
  for (int t = 0; t < 8; ++t) c[t] = ((uint32_t)(((lane >> 2) ^ t) & 7) << 2) + (lane & 3);
}
__device__ __forceinline__ void rows_to_columns(uint32_t (&v)[32], uint32_t *tsm, const uint32_t (&c)[8], int lane) {
#pragma unroll
  for (int m = 0; m < 8; ++m)
    *reinterpret_cast<uint4 *>(tsm + qoff(lane, m)) = make_uint4(v[4 * m], v[4 * m + 1], v[4 * m + 2], v[4 * m + 3]);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = tsm[32 * j + c[j & 7]];
}
__device__ __forceinline__ void columns_to_rows(uint32_t (&v)[32], uint32_t *tsm, const uint32_t (&c)[8], int lane) {
#pragma unroll
  for (int j = 0; j < 32; ++j) tsm[32 * j + c[j & 7]] = v[j];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const uint4 t = *reinterpret_cast<const uint4 *>(tsm + qoff(lane, m));
    v[4 * m] = t.x; v[4 * m + 1] = t.y; v[4 * m + 2] = t.z; v[4 * m + 3] = t.w;
  }
}


// Ascending sort of the warp's 1024 values held in the swizzled rows `rows`
// (lane l: elements 32l..32l+31), in place; tsm is a second 1024-word scratch.  Bitonic sort in the variant whose comparators
// all keep the minimum at the lower index: each merge of size k first pairs
// mirrored elements (i, i ^ (k-1)), then (i, i + d) for d = k/4 .. 1.  Lanes
// first sort their rows (odd-even merge network).  For k >= 64 the stages of
// distance >= 32 run on the transposed matrix (lane L holding elements
// 32j + L), where distance-d pairs are registers j, j + d/32 and the mirrored
// pairs are register j ^ (k/32 - 1) of lane 31 - L.
static __device__ __noinline__ void warp_sort1024_rows(uint32_t *rows, uint32_t *tsm, int lane) {
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  uint32_t v[32];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const uint4 t = *reinterpret_cast<const uint4 *>(rows + qoff(lane, m));
    v[4 * m] = t.x; v[4 * m + 1] = t.y; v[4 * m + 2] = t.z; v[4 * m + 3] = t.w;
  }
  uint32_t c[8];
  column_offsets(c, lane);
  oem_sort32(v);
#pragma unroll
  for (int lk = 6; lk <= 10; ++lk) {
    rows_to_columns(v, tsm, c, lane);
    {
      const int mk = (1 << (lk - 5)) - 1, hb = 1 << (lk - 6);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if ((j & hb) == 0) {
          const int jj = j ^ mk;
          const uint32_t pj = __shfl_xor_sync(FULL, v[jj], 31), pjj = __shfl_xor_sync(FULL, v[j], 31);
          v[j] = min(v[j], pj);
          v[jj] = max(v[jj], pjj);
        }
    }
#pragma unroll
    for (int s = lk - 2; s >= 5; --s) {
      const int dj = 1 << (s - 5);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if ((j & dj) == 0) cas_up(v[j], v[j | dj]);
    }
    columns_to_rows(v, tsm, c, lane);
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1)
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if ((j & d) == 0) cas_up(v[j], v[j | d]);
  }
#pragma unroll
  for (int m = 0; m < 8; ++m)
    *reinterpret_cast<uint4 *>(rows + qoff(lane, m)) = make_uint4(v[4 * m], v[4 * m + 1], v[4 * m + 2], v[4 * m + 3]);
}

// Start of bucket b (b = 2048 gives the number of ranked points).
__device__ __forceinline__ uint32_t bucket_start(const uint32_t *hist, uint32_t b, uint32_t total) {
  if (b >= (1u << kEncBucketBits)) return total;
  return (hist[sx(b >> 1)] >> ((b & 1u) << 4)) & 0xFFFFu;
}

// Writes one 32-element plane word of a delta / count section into the
// staged payload: bytes 4*lane.. of the plane, MSB-first bit order
// (src/cudaWarpCompress.cu:357-408), only the bytes the plane has.
__device__ __forceinline__ void put_plane_bytes(uint8_t *stage8, uint32_t pos, uint32_t bpp, uint32_t word,
                                                int lane) {
  const int room = (int)bpp - 4 * lane;
  if (room <= 0) return;
  const uint32_t w = to_msb_bytes(word);
  uint8_t *d = stage8 + pos + 4u * lane;
  d[0] = (uint8_t)w;
  if (room > 1) d[1] = (uint8_t)(w >> 8);
  if (room > 2) d[2] = (uint8_t)(w >> 16);
  if (room > 3) d[3] = (uint8_t)(w >> 24);
}

// Bit planes of this lane's 32 values (v: value of element j) into the staged
// payload: byte planes at pos0 + pi*bpp (bpp != 0) or 32-word planes at word
// pos0/4 + 32*pi + lane (bpp == 0), MSB plane first.  v is clobbered.
__device__ __forceinline__ void put_planes(uint32_t *stage, uint32_t pos0, uint32_t nb, uint32_t bpp,
                                           uint32_t (&v)[32], int lane) {
  uint8_t *stage8 = reinterpret_cast<uint8_t *>(stage);
  auto put = [&](uint32_t b, uint32_t w) {
    const uint32_t pi = nb - 1u - b;
    if (bpp) put_plane_bytes(stage8, pos0 + pi * bpp, bpp, w, lane);
    else stage[(pos0 >> 2) + 32u * pi + lane] = w;
  };
  if (nb <= 8) {
    transpose_lo8(v);
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if ((uint32_t)b < nb) put(b, v[b]);
  } else if (nb <= 16) {
    transpose_lo16(v);
#pragma unroll
    for (int b = 0; b < 16; ++b)
      if ((uint32_t)b < nb) put(b, v[b]);
  } else {
    transpose32(v);
#pragma unroll
    for (int b = 0; b < 32; ++b)
      if ((uint32_t)b < nb) put(b, v[b]);
  }
}

// Ranks the chunk's composites (block id - kmin) << 10 | r through buckets
// on their top bits: shared-atomic counts (the old count is the point's
// arrival slot), an exclusive scan to bucket starts, placement at bucket
// start + slot, then the order inside the buckets by odd-even transposition
// steps on the lanes' registers once the positions are loaded in order.
// cbits is the composites' width.
//  * kNarrow (21 <= cbits <= 32): 1024 buckets with a 32-bit counter each
//    (the fewest instructions per point); S holds whole composites, so neighbours of
//    different buckets are already in order and the steps compare values
//    alone.  A chunk with a bucket of 16 or more points is declined (the
//    data-independent warp sort ranks it instead): false is returned before
//    the placement, with S unchanged.
//  * wide (cbits > 32): 2048 buckets, two 16-bit counters a word (S keeps
//    the bits below the bucket, and they must fit 32 bits); the bucket of
//    every position is scattered beside it, and the steps compare within a
//    bucket only; buckets of 16 or more points are sorted by the warp's
//    bitonic network in S first.
// On entry S's row l holds lane l's block ids; after a true return S's row l
// holds the sorted block ids of positions 32l..32l+31 and the first 16 words
// of hist's row l the ranks r of positions j, j+16 as 16-bit pairs.
template <bool kNarrow>
static __device__ __noinline__ bool rank_buckets(uint32_t *sw, uint32_t kmin, uint32_t cbits, uint32_t nvalid,
                                                 int lane) {
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  uint32_t *const S = sw, *const hist = sw + kChunk;
  const bool full = nvalid == (uint32_t)kChunk;
  uint32_t key[32], rp[16];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const uint4 t = *reinterpret_cast<const uint4 *>(S + qoff(lane, m));
    key[4 * m] = t.x; key[4 * m + 1] = t.y; key[4 * m + 2] = t.z; key[4 * m + 3] = t.w;
  }
#pragma unroll
  for (int m = 0; m < 8; ++m) *reinterpret_cast<uint4 *>(hist + qoff(lane, m)) = make_uint4(0u, 0u, 0u, 0u);
  __syncwarp();
  // narrow: 1024 buckets on the top 10 bits, one 32-bit counter each, S
  // keeps the whole composite; wide: 2048 buckets on the top 11 bits, two
  // 16-bit counters a word, S keeps the bits below the bucket
  const uint32_t shb = cbits - kEncBucketBits, lowb = shb - 10u;
  uint32_t bs[32];  // narrow: counter word << 10 | arrival slot; wide: bucket << 10 | arrival
                    // slot, then position << 11 | bucket
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const uint32_t koff = key[j] - kmin;
    bs[j] = 0;
    if constexpr (kNarrow) {
      key[j] = (koff << 10) | (32u * lane + j);
      if (full || 32u * j + lane < nvalid) {
        const uint32_t w = sx(key[j] >> (shb + 1u));
        bs[j] = (w << 10) | atomicAdd(&hist[w], 1u);
      }
    } else {
      const uint32_t b = koff >> lowb;
      key[j] = ((koff & ((1u << lowb) - 1u)) << 10) | (32u * lane + j);
      if (full || 32u * j + lane < nvalid) {
        const uint32_t h = (b & 1u) << 4;
        const uint32_t old = atomicAdd(&hist[sx(b >> 1)], 1u << h);
        bs[j] = (b << 10) | ((old >> h) & 0x3FFu);
      }
    }
  }
  __syncwarp();
  // exclusive scan of the bucket counts; lane l owns counter words
  // 32l..32l+31 (buckets 32l.. narrow, 64l.. wide)
  uint32_t bigw = 0;  // bit k: a bucket of count word k holds 16 or more points
  uint32_t rounds;    // transposition rounds the small buckets need
  {
    // two passes over the lane's row (the counts, then the starts), so that
    // only one quad of it is held beside key and bs
    uint32_t tot = 0, mx2 = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(hist + qoff(lane, m));
      const uint32_t w4[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if constexpr (kNarrow) {
          if (w4[e] >= (uint32_t)kEncSmall) bigw |= 1u << (4 * m + e);
          tot += w4[e];
          mx2 = max(mx2, w4[e]);
        } else {
          if (w4[e] & 0xFFF0FFF0u) bigw |= 1u << (4 * m + e);
          tot += (w4[e] & 0xFFFFu) + (w4[e] >> 16);
          mx2 = __vmaxu2(mx2, w4[e]);
        }
      }
    }
    if (kNarrow && __any_sync(FULL, bigw != 0u)) return false;
    // a bucket of n points is in order after n alternating odd / even steps
    // (whichever comes first), ceil(n / 2) rounds of the pair; buckets of 16
    // or more are sorted already, so 8 rounds cover the rest
    rounds = min((warp_max(max(mx2 & 0xFFFFu, mx2 >> 16)) + 1u) >> 1, (uint32_t)kEncSmall / 2u);
    uint32_t inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += t;
    }
    uint32_t run = inc - tot;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      uint4 *const q4 = reinterpret_cast<uint4 *>(hist + qoff(lane, m));
      const uint4 t = *q4;
      uint32_t w4[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if constexpr (kNarrow) {
          const uint32_t c0 = w4[e];
          w4[e] = run;
          run += c0;
        } else {
          const uint32_t c0 = w4[e] & 0xFFFFu, c1 = w4[e] >> 16;
          w4[e] = run | ((run + c0) << 16);
          run += c0 + c1;
        }
      }
      *q4 = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
  }
  __syncwarp();
  // place: bucket start + arrival slot; every point now lies inside its
  // bucket's range of S, and the buckets are in order
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (full || 32u * j + lane < nvalid) {
      if constexpr (kNarrow) {
        S[sx(hist[bs[j] >> 10] + (bs[j] & 0x3FFu))] = key[j];
      } else {
        const uint32_t b = bs[j] >> 10;
        const uint32_t pos = ((hist[sx(b >> 1)] >> ((b & 1u) << 4)) & 0xFFFFu) + (bs[j] & 0x3FFu);
        S[sx(pos)] = key[j];
        bs[j] = (pos << 11) | b;
      }
    }
  }
  __syncwarp();
  // buckets of 16 or more points (wide composites only; narrow chunks with
  // one were declined): the whole warp sorts each one
  while (!kNarrow && __any_sync(FULL, bigw != 0)) {
    const int src = __ffs((int)__ballot_sync(FULL, bigw != 0)) - 1;
    const int k = __ffs((int)__shfl_sync(FULL, bigw, src)) - 1;
    if (lane == src) bigw &= bigw - 1;
#pragma unroll 1
    for (uint32_t b = 64u * src + 2 * k; b < 64u * src + 2 * k + 2; ++b) {
      const uint32_t st = bucket_start(hist, b, nvalid), en = bucket_start(hist, b + 1, nvalid);
      if (en - st >= (uint32_t)kEncSmall) warp_bitonic_u32(S, st, en - st, lane);
    }
  }
  __syncwarp();
  if constexpr (!kNarrow) {
    // the bucket of every position (the bucket starts are done with; a sort
    // inside a big bucket keeps its positions' bucket)
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (full || 32u * j + lane < nvalid) hist[sx(bs[j] >> 11)] = bs[j] & 0x7FFu;
    __syncwarp();
  }

  // sorted order: this lane's positions 32l..32l+31
  {
    uint32_t bpos[32];  // wide: the bucket of each position
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(S + qoff(lane, m));
      key[4 * m] = t.x; key[4 * m + 1] = t.y; key[4 * m + 2] = t.z; key[4 * m + 3] = t.w;
      if constexpr (!kNarrow) {
        const uint4 u = *reinterpret_cast<const uint4 *>(hist + qoff(lane, m));
        bpos[4 * m] = u.x; bpos[4 * m + 1] = u.y; bpos[4 * m + 2] = u.z; bpos[4 * m + 3] = u.w;
      }
    }
    // positions past the chunk's end (stale words; the caller gives them the
    // last id) take the largest value (narrow) or distinct out-of-range
    // buckets (wide), so no step moves them
    if (!full) {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (32u * lane + j >= nvalid) {
          if constexpr (kNarrow) key[j] = 0xFFFFFFFFu;
          else bpos[j] = 0x80000000u | (32u * lane + j);
        }
    }
    // order inside the buckets of 2..15 points (they arrive in slot order;
    // the big ones are sorted): odd-even transposition steps between
    // neighbouring positions of one bucket, `rounds` pairs of steps
#pragma unroll 1
    for (uint32_t it = 0; it < rounds; ++it) {
#pragma unroll
      for (int j = 0; j < 32; j += 2) {
        const bool x = (kNarrow || bpos[j] == bpos[j + 1]) && key[j] > key[j + 1];
        const uint32_t lo = x ? key[j + 1] : key[j], hi = x ? key[j] : key[j + 1];
        key[j] = lo; key[j + 1] = hi;
      }
      const uint32_t nk = __shfl_down_sync(FULL, key[0], 1), pk = __shfl_up_sync(FULL, key[31], 1);
      const uint32_t nb = kNarrow ? 0u : __shfl_down_sync(FULL, bpos[0], 1);
      const uint32_t pb = kNarrow ? 0u : __shfl_up_sync(FULL, bpos[31], 1);
#pragma unroll
      for (int j = 1; j < 31; j += 2) {
        const bool x = (kNarrow || bpos[j] == bpos[j + 1]) && key[j] > key[j + 1];
        const uint32_t lo = x ? key[j + 1] : key[j], hi = x ? key[j] : key[j + 1];
        key[j] = lo; key[j + 1] = hi;
      }
      // the pair across lanes: positions 32l+31 and 32(l+1); both lanes
      // decide on the same two values
      const bool xr = lane < 31 && (kNarrow || nb == bpos[31]) && key[31] > nk;
      const bool xl = lane > 0 && (kNarrow || pb == bpos[0]) && pk > key[0];
      if (xr) key[31] = nk;
      if (xl) key[0] = pk;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) rp[k] = (key[k] & 1023u) | ((key[k + 16] & 1023u) << 16);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if constexpr (kNarrow) key[j] = kmin + (key[j] >> 10);
      else key[j] = kmin + ((bpos[j] << lowb) | (key[j] >> 10));
    }
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < 8; ++m)
    *reinterpret_cast<uint4 *>(S + qoff(lane, m)) = make_uint4(key[4 * m], key[4 * m + 1], key[4 * m + 2], key[4 * m + 3]);
#pragma unroll
  for (int m = 0; m < 4; ++m)
    *reinterpret_cast<uint4 *>(hist + qoff(lane, m)) = make_uint4(rp[4 * m], rp[4 * m + 1], rp[4 * m + 2], rp[4 * m + 3]);
  __syncwarp();
  return true;
}

// A quantized chunk between the two encode phases: its 31-bit block ids
// (element j of lane l is point 32j + l), their range, the relative-position
// bit width and this lane's word of the meta record's min/max part.
struct ChunkQ {
  uint32_t key[32];
  uint32_t kmin, kmax, rbits, mword;
};

// The points of one chunk, loaded ahead of encoding: float streams keep all
// axes in registers (element j of lane l is point 32j + l of the chunk), so a
// chunk costs one round of loads and the next chunk's loads overlap the
// current one's placement.  Double streams load one axis at a time.
//
// The slots past the end of a short last chunk hold a copy of the chunk's
// first point: they leave the chunk's min / max, id range and largest
// relative position unchanged, so the encoder's per-point loops need no
// validity test and only the ranking and the relative-position section treat
// those slots specially.
template <typename T, int DIM>
struct ChunkPoints {
  static constexpr bool kAhead = sizeof(T) == 4;
  T v[kAhead ? DIM : 1][32];
  __device__ __forceinline__ void load(const CArgs<T> &a, unsigned long long c, int lane) {
    if constexpr (kAhead) {
      c = c < a.G ? c : a.G - 1;  // past the end: reload the last chunk (unused)
      const unsigned long long base = c * kChunk;
      const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, a.n - base);
      const T *const X[3] = {a.x, a.y, a.z};
      if (nvalid == (uint32_t)kChunk) {
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
          for (int j = 0; j < 32; ++j) v[d][j] = X[d][base + 32u * j + lane];
      } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const uint32_t p = 32u * j + lane;
            v[d][j] = X[d][base + (p < nvalid ? p : 0u)];
          }
      }
    } else {
      // Double streams keep no points in registers: lane d asks for axis d
      // of the chunk in L2 (one bulk prefetch of its valid, 16-byte aligned
      // span), so that the quantize phase's loads hit L2.
      if (lane < DIM && c < a.G) {
        const unsigned long long base = c * kChunk;
        const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, a.n - base);
        const T *p = (lane == 0 ? a.x : (lane == 1 ? a.y : a.z)) + base;
        const uint32_t bytes = (nvalid * (uint32_t)sizeof(T)) & ~15u;
        if (bytes != 0u && (reinterpret_cast<uintptr_t>(p) & 15u) == 0u)
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
      }
    }
  }
};

// First phase of encoding chunk c: min/max, quantization, block ids (into q)
// and relative positions (into the warp's third 4 KB, by rank r); double
// streams also stage each axis in the region's first 8 KB.
template <typename T, int DIM>
__device__ __forceinline__ void encode_quantize(const CArgs<T> &a, unsigned long long c, uint32_t *sw,
                                                uint32_t seg, uint32_t sh, uint32_t msk, T eb, T inv,
                                                ChunkPoints<T, DIM> &pts, ChunkQ &q, int lane) {
  using Tr = TT<T>;
  using UO = typename Tr::U;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  const unsigned long long n = a.n;
  const unsigned long long base = c * kChunk;
  const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, n - base);
  const bool full = nvalid == (uint32_t)kChunk;
  uint32_t *const relR = sw + 2 * kChunk;
  const T *const X[3] = {a.x, a.y, a.z};

  // ---- 1. quantize one axis at a time (:104-205) ----
  uint32_t (&key)[32] = q.key;
  T mm[6];
  unsigned long long bnx = 0, bny = 0, bound = 0;
  uint32_t rmax = 0;
  // Double streams stage each axis in the warp's first 8 KB (free while a
  // chunk is quantized: the previous payload has been copied out), element j
  // of lane l at word pair 32j + l, so the min/max and quantize passes read
  // it back without holding 32 doubles in registers.
  T *const stash = reinterpret_cast<T *>(sw);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    if constexpr (!ChunkPoints<T, DIM>::kAhead) {
      const T *src = X[d] + base;
      if (d > 0) __syncwarp();  // the previous axis has been read
      if (full && a.vec_ok) {
        // a full chunk of 16-byte aligned axes: 16-byte asynchronous copies,
        // 16 per lane, all in flight at once, no registers
        const uint32_t s0 = (uint32_t)__cvta_generic_to_shared(stash) + 16u * lane;
        const char *g0 = reinterpret_cast<const char *>(src) + 16u * lane;
#pragma unroll
        for (int i = 0; i < 16; ++i)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s0 + 512u * i), "l"(g0 + 512u * i) : "memory");
        asm volatile("cp.async.wait_all;" ::: "memory");
      } else {
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
          const uint32_t p = 32u * j + lane;
          stash[p] = (full || p < nvalid) ? src[p] : src[0];  // past the end: the first point
        }
      }
      __syncwarp();
    }
    auto vv_of = [&](int j) -> T {
      if constexpr (ChunkPoints<T, DIM>::kAhead) return pts.v[d][j];
      else return stash[32u * j + lane];
    };
    // fmin / fmax ignore NaN and order -0.0 below +0.0, as the reference's
    // warp reductions do (:122-139); slots past the end repeat a point
    const T lim = is64 ? (T)DBL_MAX : (T)FLT_MAX;
    T mn = lim, mx = -lim;
    if constexpr (!is64) {
#pragma unroll
      for (int j = 0; j < 32; j += 2) {
        mn = fmin3f(mn, vv_of(j), vv_of(j + 1));
        mx = fmax3f(mx, vv_of(j), vv_of(j + 1));
      }
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) { mn = fmin(mn, vv_of(j)); mx = fmax(mx, vv_of(j)); }
    }
    mn = from_ord((UO)~warp_max((UO)~ord_of(mn)));
    mx = from_ord(warp_max(ord_of(mx)));
    mm[d] = mn;
    mm[3 + d] = mx;
    const T range = is64 ? (T)__dsub_rn((double)mx, (double)mn) : (T)__fsub_rn((float)mx, (float)mn);
    if (d == 0) bnx = block_num(range, seg, eb, is64 && DIM == 2);
    if (d == 1) bny = block_num(range, seg, eb, false);
    const T nmn = is64 ? (T)__dmul_rn(-(double)mn, (double)inv) : (T)__fmul_rn(-(float)mn, (float)inv);
    // id_overflow: the chunk's largest quantized corner (u64 arithmetic)
    const unsigned long long qm = is64 ? __double2ull_rz(__fma_rn((double)mx, (double)inv, (double)nmn))
                                       : (unsigned long long)__float2uint_rz(__fmaf_rn((float)mx, (float)inv, (float)nmn));
    bound += (qm >> sh) * (d == 0 ? 1ull : (d == 1 ? bnx : bnx * bny));
    // block id (mod 2^32, masked to 31 bits at the end) and relative position
    const uint32_t kmul = d == 0 ? 1u : (d == 1 ? (uint32_t)bnx : (uint32_t)(bnx * bny));
    const uint32_t rmul = d == 0 ? 1u : (d == 1 ? seg : seg * seg);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      uint32_t rq[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = 4 * m + e;
        uint32_t kq, r;
        if constexpr (!is64) {
          const uint32_t q = __float2uint_rz(__fmaf_rn((float)vv_of(j), (float)inv, (float)nmn));
          kq = q >> sh;
          r = q & msk;
        } else {
          const unsigned long long q = __double2ull_rz(__fma_rn((double)vv_of(j), (double)inv, (double)nmn));
          kq = (uint32_t)(q >> sh);
          r = (uint32_t)(q & msk);
        }
        key[j] = d == 0 ? kq : key[j] + kq * kmul;
        rq[e] = r * rmul;
      }
      uint4 *row = reinterpret_cast<uint4 *>(relR + qoff(lane, m));
      if (d > 0) {
        const uint4 o = *row;
        rq[0] += o.x; rq[1] += o.y; rq[2] += o.z; rq[3] += o.w;
      }
      if (d == DIM - 1) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          rq[e] &= 0x7FFFFFFFu;
          rmax = max(rmax, rq[e]);
        }
      }
      *row = make_uint4(rq[0], rq[1], rq[2], rq[3]);
    }
  }
  if (DIM == 2) { mm[2] = (T)0; mm[5] = (T)0; }  // 2D meta carries z = 0 (:518, :521)
  // this lane's word of the meta record's min/max part (:332-344 / Double
  // :333-345), taken now so the six values need no registers later
  uint32_t mword = 0;
  {
    T mv = mm[0];
#pragma unroll
    for (int k = 1; k < 6; ++k)
      if ((is64 ? (lane >> 1) : lane) == k) mv = mm[k];
    if (!is64) {
      mword = __float_as_uint((float)mv);
    } else {
      const unsigned long long b = (unsigned long long)__double_as_longlong((double)mv);
      mword = (lane & 1) ? (uint32_t)(b >> 32) : (uint32_t)b;
    }
  }
  if (lane == 0 && bound > 0x7FFFFFFFull) a.ctl->id_overflow = 1u;
  uint32_t kmin = FULL, kmax = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    key[j] &= 0x7FFFFFFFu;
    kmin = min(kmin, key[j]);
    kmax = max(kmax, key[j]);
  }
  q.kmin = warp_min(kmin);
  q.kmax = warp_max(kmax);
  rmax = warp_max(rmax);
  q.rbits = max(bitlen(rmax), nvalid < (uint32_t)kChunk ? 1u : 0u);  // :200-201
  q.mword = mword;
}

// Ranks, runs and bit planes of a quantized chunk (encode_quantize left its
// ids in q and its relative positions in the warp's third 4 KB); stages the
// payload in the warp's region, returns its bytes and leaves the meta record
// in meta_word (word k of the record in lane k).
template <typename T, int DIM, class OnSize>
__device__ __forceinline__ uint32_t encode_pack(const CArgs<T> &a, unsigned long long c, uint32_t *sw, ChunkQ &q,
                                                uint32_t &meta_word, int lane, uint32_t &rank_skip,
                                                OnSize &&on_size) {
  using Tr = TT<T>;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  const unsigned long long base = c * kChunk;
  const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, a.n - base);
  const bool full = nvalid == (uint32_t)kChunk;
  // per-warp words: [0,1024) ranked composites -> run starts -> staged payload;
  // [1024,2048) bucket counts -> deltas -> staged payload; [2048,3072)
  // relative positions by rank r (staged payload only past 8 KB, after use)
  uint32_t *const S = sw, *const hist = sw + kChunk, *const relR = sw + 2 * kChunk;
  uint32_t (&key)[32] = q.key;
  const uint32_t kmin = q.kmin, kmax = q.kmax, rbits = q.rbits, mword = q.mword;

  // ---- 2. rank the composites (block id - kmin) << 10 | r ----
  const unsigned long long cmax = ((unsigned long long)(kmax - kmin) << 10) | 1023ull;
  const uint32_t cbits_all = bitlen64(cmax);
  uint32_t rp[16];  // rank r of positions j and j+16 (16-bit pairs)
  // Buckets rank every chunk whose composites are wider than 32 bits, and
  // the 32-bit ones of at least 21 bits unless they have a bucket of 16 or
  // more points (then the chunk is declined and the warp sorts its next
  // kEncBucketBackoff chunks directly); the data-independent warp sort ranks
  // the rest.  Both give the same order.
  bool ranked = false;
  if (cbits_all > 32u || (cbits_all >= 21u && rank_skip == 0u)) {
    // block ids in and results out through S and hist rows
#pragma unroll
    for (int m = 0; m < 8; ++m)
      *reinterpret_cast<uint4 *>(S + qoff(lane, m)) = make_uint4(key[4 * m], key[4 * m + 1], key[4 * m + 2], key[4 * m + 3]);
    ranked = cbits_all > 32u ? rank_buckets<false>(sw, kmin, cbits_all, nvalid, lane)
                             : rank_buckets<true>(sw, kmin, cbits_all, nvalid, lane);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(S + qoff(lane, m));
      key[4 * m] = t.x; key[4 * m + 1] = t.y; key[4 * m + 2] = t.z; key[4 * m + 3] = t.w;
    }
    if (ranked) {
      if (!full) {  // positions past the end carry the last id: they start no run
#pragma unroll
        for (int j = 0; j < 32; ++j) key[j] = 32u * lane + j < nvalid ? key[j] : kmax;
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const uint4 t = *reinterpret_cast<const uint4 *>(hist + qoff(lane, m));
        rp[4 * m] = t.x; rp[4 * m + 1] = t.y; rp[4 * m + 2] = t.z; rp[4 * m + 3] = t.w;
      }
    } else {
      rank_skip = kEncBucketBackoff;
      __syncwarp();  // S is read back before the warp sort writes it
    }
  } else if (rank_skip != 0u) {
    --rank_skip;
  }
  if (!ranked) {
    // 32-bit composites: one data-independent warp sort.  Slots past the
    // chunk's end (point 32j + lane >= nvalid) take the largest
    // composite, (kmax - kmin) << 10 | 1023: no point of a short chunk has
    // r = 1023, so they sort last, and they carry the last id kmax, so they
    // start no run.
#pragma unroll
    for (int j = 0; j < 32; ++j)
      key[j] = (full || 32u * j + lane < nvalid) ? (((key[j] - kmin) << 10) | (32u * lane + j)) : (uint32_t)cmax;
#pragma unroll
    for (int m = 0; m < 8; ++m)
      *reinterpret_cast<uint4 *>(S + qoff(lane, m)) = make_uint4(key[4 * m], key[4 * m + 1], key[4 * m + 2], key[4 * m + 3]);
    warp_sort1024_rows(S, hist, lane);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(S + qoff(lane, m));
      key[4 * m] = t.x; key[4 * m + 1] = t.y; key[4 * m + 2] = t.z; key[4 * m + 3] = t.w;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) rp[k] = (key[k] & 1023u) | ((key[k + 16] & 1023u) << 16);
#pragma unroll
    for (int j = 0; j < 32; ++j) key[j] = kmin + (key[j] >> 10);
  }
  __syncwarp();  // ranking scratch is done with

  // ---- 3. runs: unique ids, deltas, counts (:222-311) ----
  uint32_t *const runStart = sw, *const deltaA = sw + kChunk;
  uint32_t U, dbits, cbits, first;
  {
    // ids ascend, so a run starts where the id differs from its predecessor,
    // and the widest delta is the bit length of all deltas ORed together;
    // position 0 starts the first run with delta 0.  Positions past the end
    // repeat kmax and start no run.
    const uint32_t prevk = __shfl_up_sync(FULL, key[31], 1);
    const uint32_t pk0 = lane == 0 ? key[0] : prevk;
    uint32_t fm = lane == 0 ? 1u : 0u, dm = 0;
    if constexpr (!is64) {
      uint32_t dor = 0;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const uint32_t dlt = key[j] - (j ? key[j - 1] : pk0);
        dor |= dlt;
        if (dlt != 0u) fm |= 1u << j;
      }
      dm = bitlen(dor);
    } else {  // the same result; this form keeps the double kernels' registers lower
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const uint32_t dlt = key[j] - (j ? key[j - 1] : pk0);
        if (dlt != 0u) {
          fm |= 1u << j;
          dm = max(dm, bitlen(dlt));
        }
      }
    }
    const uint32_t cnt = __popc(fm);
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += t;
    }
    U = __shfl_sync(FULL, inc, 31);
    dbits = warp_max(dm);
    first = __shfl_sync(FULL, key[0], 0);
    uint32_t u = inc - cnt;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if ((fm >> j) & 1u) {
        runStart[sx(u)] = 32u * lane + j;
        deltaA[sx(u)] = key[j] - (j ? key[j - 1] : pk0);
        ++u;
      }
    }
  }
  __syncwarp();
  // this lane's runs 32l..32l+31: deltas, and counts as 16-bit pairs
  uint32_t dl[32], cp[16];
  {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(runStart + qoff(lane, m));
      const uint4 q = *reinterpret_cast<const uint4 *>(deltaA + qoff(lane, m));
      key[4 * m] = t.x; key[4 * m + 1] = t.y; key[4 * m + 2] = t.z; key[4 * m + 3] = t.w;
      dl[4 * m] = q.x; dl[4 * m + 1] = q.y; dl[4 * m + 2] = q.z; dl[4 * m + 3] = q.w;
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const bool live = 32u * lane + j < U;
      key[j] = live ? key[j] : nvalid;
      dl[j] = live ? dl[j] : 0u;
    }
    const uint32_t nx = __shfl_down_sync(FULL, key[0], 1);
    uint32_t cm = 0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint32_t e = j < 31 ? key[j + 1] : (lane < 31 ? nx : nvalid);
      key[j] = e - key[j];  // run length (0 past the last run)
      cm = max(cm, key[j]);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) cp[k] = key[k] | (key[k + 16] << 16);
    cbits = bitlen(warp_max(cm));
  }
  __syncwarp();  // run rows read: the region becomes the payload staging

  // ---- 4. bit planes -> staged payload (:313-411) ----
  const uint32_t db = section_bytes(U, dbits, Tr::pad), cb = section_bytes(U, cbits, Tr::pad);
  const uint32_t rb = rel_section_bytes(rbits, Tr::pad);
  on_size(db + cb + rb);  // the payload size is known before its planes are built
  const uint32_t bpp = (U + 7u) >> 3;
  uint32_t *const stage = sw;
  put_planes(stage, 0u, dbits, bpp, dl, lane);
#pragma unroll
  for (int k = 0; k < 16; ++k) { dl[k] = cp[k] & 0xFFFFu; dl[k + 16] = cp[k] >> 16; }
  put_planes(stage, db, cbits, bpp, dl, lane);
  // delta + count sections end below 8 KB: the rank rows are still intact
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const uint32_t r = (rp[j & 15] >> (16 * (j >> 4))) & 1023u;
    dl[j] = relR[sx(r)];
  }
  if (!full) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (32u * lane + j >= nvalid) dl[j] = 0xFFFFFFFFu;  // slots past the end (:197)
  }
  __syncwarp();
  put_planes(stage, db + cb, rbits, 0u, dl, lane);
  {
    // section padding is zero (the reference leaves it unwritten)
    uint8_t *stage8 = reinterpret_cast<uint8_t *>(stage);
    const uint32_t p0 = dbits * bpp + lane, p1 = db + cbits * bpp + lane;
    if (p0 < db) stage8[p0] = 0;
    if (p1 < db + cb) stage8[p1] = 0;
  }

  // meta record (:332-344 / Double :333-345)
  {
    uint32_t w = 0;
    if (!is64) {
      if (lane < 6) w = mword;
      if (lane == 6) w = first;
      if (lane == 7) w = dbits | (cbits << 16);
      if (lane == 8) w = rbits | (U << 16);
    } else {
      if (lane < 12) w = mword;
      if (lane == 12) w = first;
      if (lane == 13) w = 0;
      if (lane == 14) w = dbits | (cbits << 16);
      if (lane == 15) w = rbits | (U << 16);
    }
    meta_word = w;
  }
  return db + cb + rb;
}

// Encodes chunk c into the warp's region `sw`; returns the payload bytes and
// leaves the meta record in meta_word (word k of the record in lane k).
// on_size(bytes) runs (warp-wide) as soon as the payload size is known, before
// the bit planes are built.  rank_skip is the warp's count of chunks still to
// rank by the warp sort without trying the buckets first.
template <typename T, int DIM, class OnSize>
__device__ __forceinline__ uint32_t encode_chunk(const CArgs<T> &a, unsigned long long c, uint32_t *sw,
                                                 uint32_t seg, uint32_t sh, uint32_t msk, T eb, T inv,
                                                 ChunkPoints<T, DIM> &pts, uint32_t &meta_word, int lane,
                                                 uint32_t &rank_skip, OnSize &&on_size) {
  ChunkQ q;
  encode_quantize<T, DIM>(a, c, sw, seg, sh, msk, eb, inv, pts, q, lane);
  return encode_pack<T, DIM>(a, c, sw, q, meta_word, lane, rank_skip, on_size);
}

// Copies a staged payload (whole words) to its place in the stream: four
// independent shared loads per lane before their global stores, so the loads'
// latency is paid once per 512 bytes rather than per 128.
__device__ __forceinline__ void copy_payload(uint32_t *dst, const uint32_t *sw, uint32_t payload, int lane) {
  const uint32_t nw = payload / 4u;
  for (uint32_t w = lane; w < nw; w += 128) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    if (w < nw) t0 = sw[w];
    if (w + 32 < nw) t1 = sw[w + 32];
    if (w + 64 < nw) t2 = sw[w + 64];
    if (w + 96 < nw) t3 = sw[w + 96];
    if (w < nw) dst[w] = t0;
    if (w + 32 < nw) dst[w + 32] = t1;
    if (w + 64 < nw) dst[w + 64] = t2;
    if (w + 96 < nw) dst[w + 96] = t3;
  }
}

// Writes a placed chunk: its offset-table entry (:1679), meta record, payload,
// and for chunk 0 the header (:1674-1678; Double :1672-1680).
template <typename T>
__device__ __forceinline__ void place_chunk(const CArgs<T> &a, unsigned long long c, unsigned long long G,
                                            unsigned long long pay_base, unsigned long long off, uint32_t payload,
                                            uint32_t meta_word, uint32_t seg, T eb, const uint32_t *sw, int lane) {
  using Tr = TT<T>;
  constexpr bool is64 = sizeof(T) == 8;
  if (lane == 0) reinterpret_cast<unsigned long long *>(a.out + Tr::hdr)[c] = off;
  uint8_t *meta = a.out + Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * c;
  if (lane < (int)(Tr::meta / 4)) reinterpret_cast<uint32_t *>(meta)[lane] = meta_word;
  if (c == 0) {
    uint32_t *h = reinterpret_cast<uint32_t *>(a.out);
    if (lane == 0) h[0] = a.dim;
    if (lane == 1) h[1] = (uint32_t)a.n;
    if (lane == 2) h[2] = (uint32_t)(a.n >> 32);
    if (lane == 3) h[3] = Tr::bits;
    if (!is64) {
      if (lane == 4) h[4] = __float_as_uint((float)eb);
      if (lane == 5) h[5] = seg;
    } else {
      if (lane == 4) h[4] = (uint32_t)__double_as_longlong((double)eb);
      if (lane == 5) h[5] = (uint32_t)((unsigned long long)__double_as_longlong((double)eb) >> 32);
      if (lane == 6) h[6] = seg;
      if (lane == 7) h[7] = 32u;
    }
  }
  if (pay_base + off + payload > a.out_cap) {
    if (lane == 0) set_status(a.ctl, kENOSPACE);
  } else {
    copy_payload(reinterpret_cast<uint32_t *>(a.out + pay_base + off), sw, payload, lane);
  }
  if (c == G - 1 && lane == 0) a.ctl->stream_bytes = pay_base + off + payload;
}

// Persistent compress kernel: every CTA encodes groups of W consecutive
// chunks, one chunk per warp.  Per group: the warps quantize,
// rank and find the runs of their chunks; their payload sizes are then known
// (barrier B1) and warp 0 publishes the group's aggregate, so that later
// groups' look-backs can pass it while the warps build their bit planes;
// warp 0 then resolves the group's stream offset (decoupled look-back) and
// after barrier B2 every warp copies its staged payload out.
template <typename T, int DIM, int W = enc_warps<T, DIM>()>
__global__ void __launch_bounds__(32 * W, GPZ_ENC_MIN_CTAS) compress_kernel(const CArgs<T> a) {
  using Tr = TT<T>;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(16) uint32_t enc_smem[];
  __shared__ EncGroupT<W> eg;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *const sw = enc_smem + warp * kEncWords;
  Control *ctl = a.ctl;
  if (ld_volatile(reinterpret_cast<const uint32_t *>(&ctl->status)) != 0) return;
  const uint32_t seg = ctl->seg;
  const uint32_t sh = (uint32_t)__ffs((int)seg) - 1u, msk = seg - 1u;
  const T eb = a.eb_dev ? (T)*a.eb_dev : a.eb;
  const T inv = is64 ? (T)__ddiv_rn(1.0, __dmul_rn(2.0, (double)eb)) : (T)__fdiv_rn(1.0f, __fmul_rn(2.0f, (float)eb));
  const unsigned long long G = a.G;
  const unsigned long long pay_base = Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * G;

  if (threadIdx.x == 0) eg.next = atomicAdd(&ctl->chunk_ctr, (uint32_t)W);
  __syncthreads();
  ChunkPoints<T, DIM> pts;
  pts.load(a, eg.next + warp, lane);
  uint32_t rank_skip = 0;
  for (;;) {
    const unsigned long long gbase = eg.next;
    if (gbase >= G) break;
    __syncthreads();  // B0: everyone has the group before it is replaced
    if (threadIdx.x == 0) eg.next = ld_volatile(&ctl->abort) ? G : atomicAdd(&ctl->chunk_ctr, (uint32_t)W);
    const unsigned long long c = gbase + warp;
    const unsigned long long gid = gbase / W;
    uint32_t total = 0;
    auto on_size = [&](uint32_t bytes) {
      if (lane == 0) eg.sz[warp] = bytes;
      __syncthreads();  // B1: the group's sizes are known
      if (warp == 0) {
        const uint32_t s = lane < W ? eg.sz[lane] : 0u;
        total = __reduce_add_sync(FULL, s);
        if (lane == 0) publish_aggregate(a.look, gid, total);
      }
    };
    uint32_t payload = 0, meta_word = 0;
    if (c < G) payload = encode_chunk<T, DIM>(a, c, sw, seg, sh, msk, eb, inv, pts, meta_word, lane, rank_skip, on_size);
    else on_size(0u);
    if (warp == 0) {
      // resolved only now: the predecessors have had this group's plane
      // building to publish, so the look-back rarely waits
      unsigned long long excl = 0;
      const bool ok = resolve_prefix(a.look, gid, total, ctl, excl);
      if (lane == 0) eg.goff = ok ? excl : ~0ull;
    }
    pts.load(a, eg.next + warp, lane);  // in flight during the copy-out
    __syncthreads();  // B2: the group's stream offset is known
    const unsigned long long goff = eg.goff;
    if (c < G && goff != ~0ull) {
      unsigned long long off = goff;
      for (int w = 0; w < warp; ++w) off += eg.sz[w];
      place_chunk<T>(a, c, G, pay_base, off, payload, meta_word, seg, eb, sw, lane);
    }
  }
  rewind_work_counter(ctl);
}

}  // namespace gpzb
