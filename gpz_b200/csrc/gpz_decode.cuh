// gpz_decode.cuh -- decompress kernel of the B200 GPZ codec.
//
//   decompress_kernel   runDecompressKernel[2D] (reference
//                       src/cudaWarpCompress.cu:798-1214; float64 twin
//                       src/cudaWarpCompressDouble.cu, same ranges +/- 3)
//
// One warp decodes one 1024-point chunk.  Lane l owns unit l of every section
// -- elements 32l..32l+31 of the delta and count planes, positions
// 32l..32l+31 of the relative-position planes and of the output -- so every
// plane word is one coalesced 32-bit load per lane, straight from the stream
// into registers, transposed there.  The only cross-lane step is the run
// expansion: each run writes its id at its start position in a per-warp map
// and an inclusive max-scan over positions hands every position the id of its
// run (ids never decrease along a chunk).  Output rows are staged in shared
// memory so every global store is a 512-byte coalesced row segment.  Warps
// take chunks c = w, w + W, ... of a grid that fits the GPU; warps never wait
// for each other.
#pragma once

#include "gpz_device.cuh"

namespace gpzb {

template <typename T>
struct DArgs {
  const uint8_t *s;
  unsigned long long bytes;
  T *x, *y, *z;
  unsigned long long cap;
  Control *ctl;
  int vec_ok;
};

// Per-warp shared memory, in 32-bit words.
//   A   run map: id (fast path) or run index at every run start
//   TL  id table (low words) of the general path
//   TH  id table high words (float64 streams)
//   P   per-position id (fast path: then running quotients) or run index
//   R   per-position relative position word
//   C   staged output rows
// Float32 decoder CTAs: 8 warps x 2 per SM (16 warps, 128 registers, 192 KB
// of shared memory); 4 x 4 measured 2.7 % slower on the 143.7M-point
// snapshot, 6 x 3 (112 registers) and 2 x 8 slower still.
#ifndef GPZ_DEC_MIN_CTAS_F32
#define GPZ_DEC_MIN_CTAS_F32 2  // resident float32 decoder CTAs per SM the register budget is sized for
#endif
#ifndef GPZ_DEC_WARPS_F32
#define GPZ_DEC_WARPS_F32 8     // float32 decoder warps per CTA
#endif
template <typename T> struct DecCfg;
template <> struct DecCfg<float> {
  static constexpr int warps = GPZ_DEC_WARPS_F32, min_ctas = GPZ_DEC_MIN_CTAS_F32;
  static constexpr int A = 0, P = 0, TL = kChunk, TH = kChunk, R = kChunk, C = 2 * kChunk, words = 3 * kChunk;
};
template <> struct DecCfg<double> {
  static constexpr int warps = 2, min_ctas = 8;
  static constexpr int A = 0, TL = kChunk, TH = 2 * kChunk, P = 3 * kChunk, R = 4 * kChunk, C = 5 * kChunk,
                       words = 6 * kChunk;
};
template <typename T>
constexpr size_t dec_smem_bytes() { return (size_t)DecCfg<T>::warps * DecCfg<T>::words * 4; }

// Float64 streams whose chunks have ordinary geometry (block counts whose
// product fits 32 bits; ids are below 2^31 in every valid stream) need no
// 64-bit id tables: they decode in the float layout, 12 KB per warp, twice
// the warps per SM of the general layout.  A chunk with wider geometry is
// left to a second pass in the general layout.
struct DecCfgF64Fast {
  static constexpr int warps = 4, min_ctas = 4;
  static constexpr int A = 0, P = 0, TL = kChunk, TH = kChunk, R = kChunk, C = 2 * kChunk, words = 3 * kChunk;
};
template <class Cfg>
constexpr size_t dec_smem_bytes_of() { return (size_t)Cfg::warps * Cfg::words * 4; }

// Which chunks a decompress pass decodes.
constexpr int kPassAll = 0;      // every chunk (general layout)
constexpr int kPassFast = 1;     // chunks of ordinary geometry; the others are flagged in ctl->deferred
constexpr int kPassGeneral = 2;  // only the chunks kPassFast left (general layout)

// ---------------------------------------------------------------------------
// Bit planes.  Delta and count planes are ceil(U/8) bytes each, MSB plane
// first, element k at bit 7-(k%8) of byte k/8 (src/cudaWarpCompress.cu:366-378);
// relative-position planes are 32 little-endian words each.
// ---------------------------------------------------------------------------

// Aligned word under this lane of the byte plane starting at byte `pos`; no
// read reaches past the section's last word `endw`.
__device__ __forceinline__ uint32_t bplane_lo(const uint32_t *__restrict__ pw, uint32_t pos, uint32_t endw,
                                              int lane) {
  const uint32_t ai = (pos >> 2) + (uint32_t)lane;
  return ai < endw ? __ldg(pw + ai) : 0u;
}

// Bytes 4*lane..4*lane+3 of the plane as a word in element order (bit t =
// element 32*lane + t), masked to the lane's valid elements `vm`.  The
// unaligned window takes its upper part from the next lane's aligned word;
// lane 31 loads its own when the plane is longer than 124 bytes.
__device__ __forceinline__ uint32_t bplane_word(uint32_t lo, const uint32_t *__restrict__ pw, uint32_t pos,
                                                uint32_t bpp, uint32_t endw, uint32_t vm, int lane) {
  uint32_t hi = __shfl_down_sync(0xFFFFFFFFu, lo, 1);
  if (bpp > 124u) {
    const uint32_t a32 = (pos >> 2) + 32u;
    if (lane == 31) hi = a32 < endw ? __ldg(pw + a32) : 0u;
  }
  return from_msb_bytes(__funnelshift_r(lo, hi, (pos & 3u) << 3)) & vm;
}

// Plane words of one section loaded ahead of use (when it has at most CAP
// planes): w[b] = the aligned word of value bit b's plane.
template <int CAP, bool BYTES>
struct PlaneWords {
  uint32_t w[CAP];
  __device__ __forceinline__ void load(const uint32_t *__restrict__ pw, uint32_t pos0, uint32_t nb, uint32_t bpp,
                                       uint32_t endw, int lane) {
    const bool pre = nb <= (uint32_t)CAP;
#pragma unroll
    for (int b = 0; b < CAP; ++b) {
      w[b] = 0u;
      if (pre && (uint32_t)b < nb) {
        const uint32_t pi = nb - 1u - b;
        w[b] = BYTES ? bplane_lo(pw, pos0 + pi * bpp, endw, lane) : __ldg(pw + (pos0 >> 2) + 32u * pi + lane);
      }
    }
  }
};

// This lane's transposed section words: N = 8 gives quads (value k | k+8 <<
// 8 | k+16 << 16 | k+24 << 24), N = 16 pairs (value k | k+16 << 16), N = 32
// values.  Requires nb <= N; planes come from `raw` when N <= CAP.  `orw`
// collects the OR of the (masked) plane words.
template <int N, int CAP, bool BYTES>
__device__ __forceinline__ void section_words(uint32_t (&q)[N], const PlaneWords<CAP, BYTES> &raw,
                                              const uint32_t *__restrict__ pw, uint32_t pos0, uint32_t nb,
                                              uint32_t bpp, uint32_t endw, uint32_t vm, int lane, uint32_t &orw) {
#pragma unroll
  for (int b = 0; b < N; ++b) {
    uint32_t w = 0u;
    if ((uint32_t)b < nb) {
      const uint32_t pi = nb - 1u - b;
      const uint32_t pos = pos0 + pi * bpp;
      uint32_t lo;
      if constexpr (N <= CAP) lo = raw.w[b < CAP ? b : 0];
      else lo = BYTES ? bplane_lo(pw, pos, endw, lane) : __ldg(pw + (pos0 >> 2) + 32u * pi + lane);
      w = BYTES ? bplane_word(lo, pw, pos, bpp, endw, vm, lane) : lo;
    }
    q[b] = w;
    orw |= w;
  }
  if constexpr (N == 8) planes8_to_quads(q);
  else if constexpr (N == 16) planes16_to_pairs(q);
  else transpose32(q);
}

template <int N>
__device__ __forceinline__ uint32_t word_value(const uint32_t (&q)[N], int j) {
  if constexpr (N == 8) return (q[j & 7] >> (8 * (j >> 3))) & 0xFFu;
  else if constexpr (N == 16) return j < 16 ? (q[j] & 0xFFFFu) : (q[j - 16] >> 16);
  else return q[j];
}

// ---------------------------------------------------------------------------
// Reconstruction (src/cudaWarpCompress.cu:971-1007): q = block*seg + rel,
// value = fma(2q+1, eb, min), block coordinates from the run id
//   x = id % bnx,  y = (id / bnx) % bny,  z = id / (bnx*bny)   (u32 for float
// streams, u64 for double streams).
// ---------------------------------------------------------------------------
struct ChunkGeom {
  uint32_t bnx, bny, seg, sh, msk;
  FastDiv31 gx, gy;         // fast path: ids < 2^31, bnx*bny < 2^32
  FastDiv fx, fy, fxy;      // general float path: any 32-bit id
  unsigned long long bnx64, bny64;
  bool wide;                // float64: a block count or their product needs 64 bits
};

template <int D>
__device__ __forceinline__ uint32_t rel_coord(uint32_t rp, const ChunkGeom &g) {
  if constexpr (D == 0) return rp & g.msk;
  if constexpr (D == 1) return (rp >> g.sh) & g.msk;
  return (2u * g.sh >= 32u) ? 0u : (rp >> (2u * g.sh));
}

template <typename T>
__device__ __forceinline__ uint32_t value_bits(unsigned long long b, uint32_t rel, uint32_t seg, T eb, T mn,
                                               uint32_t &hi) {
  if constexpr (sizeof(T) == 4) {
    const uint32_t q = (uint32_t)b * seg + rel;
    hi = 0u;
    return __float_as_uint(__fmaf_rn(__uint2float_rn((q << 1) | 1u), (float)eb, (float)mn));
  } else {
    const unsigned long long q = b * (unsigned long long)seg + rel;
    const unsigned long long v =
        (unsigned long long)__double_as_longlong(__fma_rn(__ull2double_rn((q << 1) | 1ull), (double)eb, (double)mn));
    hi = (uint32_t)(v >> 32);
    return (uint32_t)v;
  }
}

// Coalesced copy of the staged rows to `dst`: step k writes rows 4k..4k+3,
// 8 lanes per 128-byte row (float: whole rows; double: half-rows `half`).
template <typename T>
__device__ __forceinline__ void copy_out_rows(const uint32_t *stage, T *dst, int lane, uint32_t half,
                                              uint32_t nvalid, bool full) {
  constexpr int EPQ = 16 / (int)sizeof(T);
#pragma unroll 2  // partly rolled: the smaller instruction footprint measured faster
  for (int k = 0; k < 8; ++k) {
    const int row = 4 * k + (lane >> 3), qd = lane & 7;
    const uint4 w = *reinterpret_cast<const uint4 *>(stage + qoff(row, qd));
    const uint32_t p0 = 32u * row + 16u * half + (uint32_t)(EPQ * qd);
    if (full) {
      *reinterpret_cast<uint4 *>(dst + p0) = w;
    } else {
      const uint32_t ww[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int e = 0; e < EPQ; ++e) {
        if (p0 + e < nvalid) {
          if constexpr (sizeof(T) == 4) dst[p0 + e] = (T)__uint_as_float(ww[e]);
          else dst[p0 + e] = (T)__hiloint2double((int)ww[2 * e + 1], (int)ww[2 * e]);
        }
      }
    }
  }
}

// One axis.  MODE 0: P holds ids (axis 0), then id/bnx (axis 1), then
// id/(bnx*bny) (axis 2), each axis leaving the next quotient in place.
// MODE 1: P holds 32-bit ids, general dividers.  MODE 2 (double streams): P
// holds run indices, 64-bit ids come from the id table.
template <typename T, int D, int MODE, bool KEEP, class Cfg>
__device__ __forceinline__ void reconstruct_axis(uint32_t *sw, const ChunkGeom &g, T eb, T mn, T *dst, int lane,
                                                 uint32_t nvalid, bool full) {
  constexpr bool is64 = sizeof(T) == 8;
  constexpr int H = is64 ? 2 : 1;  // staged (half-)rows per axis
  uint32_t *P = sw + Cfg::P;
  const uint32_t *R = sw + Cfg::R, *TL = sw + Cfg::TL, *TH = sw + Cfg::TH;
  uint32_t *C = sw + Cfg::C;
#pragma unroll 1
  for (int h = 0; h < H; ++h) {
#pragma unroll 1  // rolled: a smaller instruction footprint beats the extra overlap
    for (int m = 0; m < 8 / H; ++m) {
      const int mq = h * (8 / H) + m;
      const uint4 p4 = *reinterpret_cast<const uint4 *>(P + qoff(lane, mq));
      const uint4 r4 = *reinterpret_cast<const uint4 *>(R + qoff(lane, mq));
      const uint32_t pp[4] = {p4.x, p4.y, p4.z, p4.w}, rr[4] = {r4.x, r4.y, r4.z, r4.w};
      uint32_t lo[4], hi[4], nq[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        unsigned long long b;
        if constexpr (MODE == 0) {
          const uint32_t n = pp[e];
          if constexpr (D == 2) {
            b = n;
          } else {
            const uint32_t qn = (D == 0 ? g.gx : g.gy).div2(n + n);
            nq[e] = qn;
            b = n - qn * (D == 0 ? g.bnx : g.bny);
          }
        } else if constexpr (MODE == 1) {
          const uint32_t id = pp[e];
          b = D == 0 ? g.fx.mod(id) : (D == 1 ? g.fy.mod(g.fx.div(id)) : g.fxy.div(id));
        } else {
          const int r = swz((int)pp[e]);
          const unsigned long long id = TL[r] | ((unsigned long long)TH[r] << 32);
          if (!g.wide && (id >> 32) == 0) {
            const uint32_t i32 = (uint32_t)id;
            b = D == 0 ? g.fx.mod(i32) : (D == 1 ? g.fy.mod(g.fx.div(i32)) : g.fxy.div(i32));
          } else {
            const unsigned long long dx = g.bnx64, dy = g.bny64, dxy = g.bnx64 * g.bny64;
            if (D == 0) b = dx ? id % dx : id;
            else if (D == 1) { const unsigned long long q1 = dx ? id / dx : ~0ull; b = dy ? q1 % dy : q1; }
            else b = dxy ? id / dxy : ~0ull;
          }
        }
        lo[e] = value_bits<T>(b, rel_coord<D>(rr[e], g), g.seg, eb, mn, hi[e]);
      }
      if constexpr (MODE == 0 && D < 2 && KEEP)
        *reinterpret_cast<uint4 *>(P + qoff(lane, mq)) = make_uint4(nq[0], nq[1], nq[2], nq[3]);
      if constexpr (!is64) {
        *reinterpret_cast<uint4 *>(C + qoff(lane, m)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      } else {
        *reinterpret_cast<uint4 *>(C + qoff(lane, 2 * m)) = make_uint4(lo[0], hi[0], lo[1], hi[1]);
        *reinterpret_cast<uint4 *>(C + qoff(lane, 2 * m + 1)) = make_uint4(lo[2], hi[2], lo[3], hi[3]);
      }
    }
    __syncwarp();
    copy_out_rows<T>(C, dst, lane, (uint32_t)h, nvalid, full);
    __syncwarp();
  }
}

template <typename T, int DIM, int MODE, class Cfg>
__device__ __forceinline__ void reconstruct(uint32_t *sw, const ChunkGeom &g, T eb, const T (&mm)[6], T *const (&Y)[3],
                                            unsigned long long base, int lane, uint32_t nvalid, bool full) {
  reconstruct_axis<T, 0, MODE, true, Cfg>(sw, g, eb, mm[0], Y[0] + base, lane, nvalid, full);
  reconstruct_axis<T, 1, MODE, DIM == 3, Cfg>(sw, g, eb, mm[1], Y[1] + base, lane, nvalid, full);
  if constexpr (DIM == 3) reconstruct_axis<T, 2, MODE, false, Cfg>(sw, g, eb, mm[2], Y[2] + base, lane, nvalid, full);
}

template <typename T>
__device__ __forceinline__ uint32_t dec_meta_word(const uint8_t *s, unsigned long long G, unsigned long long c,
                                                  int lane) {
  using Tr = TT<T>;
  constexpr int MW = Tr::meta / 4;
  if (lane < MW) return reinterpret_cast<const uint32_t *>(s + Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * c)[lane];
  if (lane < MW + 2) return reinterpret_cast<const uint32_t *>(s + Tr::hdr + 8ull * c)[lane - MW];
  return 0u;
}

// Deltas -> run ids -> run map (and id table on the general path).  Called
// with the section words of width N; P16 holds the run starts as 16-bit pairs.
template <typename T, int N, class Cfg>
__device__ __forceinline__ void scatter_runs(const uint32_t (&q)[N], const uint32_t (&P16)[16], uint32_t *sw,
                                             typename TT<T>::U id, uint32_t nl, bool fast, int lane) {
  uint32_t *A = sw + Cfg::A, *TL = sw + Cfg::TL, *TH = sw + Cfg::TH;
  if (fast) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      id += word_value<N>(q, j);
      const uint32_t st = j < 16 ? (P16[j] & 0xFFFFu) : (P16[j - 16] >> 16);
      if ((uint32_t)j < nl) A[swz((int)st)] = (uint32_t)id;
    }
  } else {
    uint32_t lo4[4], hi4[4];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      id += word_value<N>(q, j);
      const uint32_t st = j < 16 ? (P16[j] & 0xFFFFu) : (P16[j - 16] >> 16);
      if ((uint32_t)j < nl) A[swz((int)st)] = 32u * lane + j;
      lo4[j & 3] = (uint32_t)id;
      hi4[j & 3] = (uint32_t)((unsigned long long)id >> 32);
      if ((j & 3) == 3) {
        *reinterpret_cast<uint4 *>(TL + qoff(lane, j >> 2)) = make_uint4(lo4[0], lo4[1], lo4[2], lo4[3]);
        if constexpr (sizeof(T) == 8)
          *reinterpret_cast<uint4 *>(TH + qoff(lane, j >> 2)) = make_uint4(hi4[0], hi4[1], hi4[2], hi4[3]);
      }
    }
  }
}

// One chunk of a stream: c its index, n/G/pay_base/eb/seg from the validated
// header, mwc the lanes' words of its meta record (dec_meta_word).  A record
// or payload that fails validation sets GPZ_ESTREAM and writes nothing.
template <typename T, int DIM, class Cfg = DecCfg<T>, int PASS = kPassAll>
__device__ __forceinline__ void decode_chunk(const DArgs<T> &a, unsigned long long c, unsigned long long n,
                                             unsigned long long G, unsigned long long pay_base, T eb, uint32_t seg,
                                             ChunkGeom &g, uint32_t mwc, uint32_t *sw, int lane) {
  using Tr = TT<T>;
  using Acc = typename TT<T>::U;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  Control *ctl = a.ctl;
  T *const Y[3] = {a.x, a.y, a.z};
  const unsigned long long base = c * kChunk;
  const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, n - base);

  // ---- chunk record: min/max, first id, bit widths, U, payload offset ----
  T mm[6];
  unsigned long long first, off;
  uint32_t dbits, cbits, rbits, U;
  if (!is64) {
#pragma unroll
    for (int k = 0; k < 6; ++k) mm[k] = (T)__uint_as_float(__shfl_sync(FULL, mwc, k));
    first = __shfl_sync(FULL, mwc, 6);
    const uint32_t w7 = __shfl_sync(FULL, mwc, 7), w8 = __shfl_sync(FULL, mwc, 8);
    dbits = w7 & 0xFFFFu; cbits = w7 >> 16; rbits = w8 & 0xFFFFu; U = w8 >> 16;
    off = __shfl_sync(FULL, mwc, 9) | ((unsigned long long)__shfl_sync(FULL, mwc, 10) << 32);
  } else {
#pragma unroll
    for (int k = 0; k < 6; ++k)
      mm[k] = (T)__hiloint2double((int)__shfl_sync(FULL, mwc, 2 * k + 1), (int)__shfl_sync(FULL, mwc, 2 * k));
    first = __shfl_sync(FULL, mwc, 12) | ((unsigned long long)__shfl_sync(FULL, mwc, 13) << 32);
    const uint32_t w14 = __shfl_sync(FULL, mwc, 14), w15 = __shfl_sync(FULL, mwc, 15);
    dbits = w14 & 0xFFFFu; cbits = w14 >> 16; rbits = w15 & 0xFFFFu; U = w15 >> 16;
    off = __shfl_sync(FULL, mwc, 16) | ((unsigned long long)__shfl_sync(FULL, mwc, 17) << 32);
  }
  const uint32_t db = section_bytes(U, dbits, Tr::pad), cb = section_bytes(U, cbits, Tr::pad);
  const uint32_t rb = rel_section_bytes(rbits, Tr::pad);
  const unsigned long long pl = (unsigned long long)db + cb + rb;
  const bool ok = U >= 1 && U <= nvalid && dbits <= 32 && cbits <= 32 && rbits <= 32 && (off & (Tr::pad)) == 0 &&
                  pl <= (unsigned long long)kStageBytes && pay_base <= a.bytes && off <= a.bytes - pay_base &&
                  pl <= a.bytes - pay_base - off;
  if (!ok) {
    if (lane == 0) set_status(ctl, kESTREAM);
    return;
  }
  const uint32_t *pw = reinterpret_cast<const uint32_t *>(a.s + pay_base + off);
  const uint32_t bpp = (U + 7u) >> 3;
  const uint32_t endd = db >> 2, endc = (db + cb) >> 2;  // section end words

  // all plane words of the usual section widths in flight at once
  PlaneWords<8, true> rawc;
  PlaneWords<16, true> rawd;
  PlaneWords<16, false> rawr;
  rawc.load(pw, db, cbits, bpp, endc, lane);
  rawd.load(pw, 0u, dbits, bpp, endd, lane);
  rawr.load(pw, db + cb, rbits, 0u, 0u, lane);

  // valid elements of this lane's unit; delta 0 is replaced by the first id
  const int nl_i = min(max((int)U - 32 * lane, 0), 32);
  const uint32_t nl = (uint32_t)nl_i;
  const uint32_t vm = nl >= 32u ? FULL : ((1u << nl) - 1u);
  const uint32_t vmd = lane == 0 ? (vm & ~1u) : vm;

  // block counts (:831-837 / Double :835-838); lanes 0..2 build the three
  // dividers at once
  const T rx = is64 ? (T)__dsub_rn((double)mm[3], (double)mm[0]) : (T)__fsub_rn((float)mm[3], (float)mm[0]);
  const T ry = is64 ? (T)__dsub_rn((double)mm[4], (double)mm[1]) : (T)__fsub_rn((float)mm[4], (float)mm[1]);
  const unsigned long long bnx = block_num(rx, seg, eb, false), bny = block_num(ry, seg, eb, false);
  g.bnx = (uint32_t)bnx;
  g.bny = (uint32_t)bny;
  g.bnx64 = bnx;
  g.bny64 = bny;
  g.wide = is64 && ((bnx >> 32) != 0 || (bny >> 32) != 0 || ((bnx * bny) >> 32) != 0);
  if constexpr (PASS != kPassAll) {
    const bool general_geom = g.wide || bnx == 0 || bny == 0 || bnx * bny >= (1ull << 32);
    if constexpr (PASS == kPassFast) {
      if (general_geom) {  // left to the general pass
        if (lane == 0) atomicExch(&ctl->deferred, 1u);
        return;
      }
    } else {
      if (!general_geom) return;  // decoded by the fast pass
    }
  }
  const uint32_t my_div = lane == 0 ? (uint32_t)bnx : (lane == 1 ? (uint32_t)bny : (uint32_t)(bnx * bny));
  {
    FastDiv31 d31;
    d31.init(my_div);
    g.gx.d = __shfl_sync(FULL, d31.d, 0); g.gx.m = __shfl_sync(FULL, d31.m, 0); g.gx.l = __shfl_sync(FULL, d31.l, 0);
    g.gy.d = __shfl_sync(FULL, d31.d, 1); g.gy.m = __shfl_sync(FULL, d31.m, 1); g.gy.l = __shfl_sync(FULL, d31.l, 1);
  }
  uint32_t *const A = sw + Cfg::A;
#pragma unroll
  for (int m = 0; m < 8; ++m) *reinterpret_cast<uint4 *>(A + qoff(lane, m)) = make_uint4(0u, 0u, 0u, 0u);  // swizzled: no bank conflicts

  // ---- counts -> run starts as 16-bit pairs P16[k] = st_k | st_{k+16} << 16 ----
  uint32_t P16[16];
  bool bad = false;
  {
    uint32_t orw = 0;
    if (cbits <= 8u) {
      uint32_t q[8];
      section_words<8>(q, rawc, pw, db, cbits, bpp, endc, vm, lane, orw);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        P16[k] = prmt(q[k], 0u, 0x4240);
        P16[k + 8] = prmt(q[k], 0u, 0x4341);
      }
    } else if (cbits <= 16u) {
      uint32_t q[16];
      section_words<16>(q, rawc, pw, db, cbits, bpp, endc, vm, lane, orw);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        bad |= (q[k] & 0xFFFFu) > (uint32_t)kChunk || (q[k] >> 16) > (uint32_t)kChunk;
        P16[k] = q[k];
      }
    } else {
      uint32_t q[32];
      section_words<32>(q, rawc, pw, db, cbits, bpp, endc, vm, lane, orw);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        bad |= q[k] > (uint32_t)kChunk || q[k + 16] > (uint32_t)kChunk;
        P16[k] = (q[k] & 0xFFFFu) | (q[k + 16] << 16);
      }
    }
    // every run holds 1..1024 points (8-bit counts cannot exceed 1024)
    bad |= (orw & vm) != vm;  // a zero count
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t v = P16[k];
      P16[k] = run;
      run += v;
    }
    const uint32_t s_lo = run & 0xFFFFu, loc = s_lo + (run >> 16);
    uint32_t inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += t;
    }
    if (__any_sync(FULL, bad) || __shfl_sync(FULL, inc, 31) != nvalid) {
      if (lane == 0) set_status(ctl, kESTREAM);
      return;
    }
    const uint32_t cbase = inc - loc, add = cbase | ((cbase + s_lo) << 16);
#pragma unroll
    for (int k = 0; k < 16; ++k) P16[k] += add;
  }
  __syncwarp();  // run map rows cleared

  // ---- deltas -> ids: id[0] = first, id[u] = id[u-1] + delta[u] (:930-938) ----
  bool fast = false, bail = false;
  {
    auto run_ids = [&](auto &q) {
      constexpr int N = sizeof(q) / sizeof(uint32_t);
      Acc loc = 0;
      if constexpr (N == 8) {
        uint32_t t = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) t = __dp4a(q[k], 0x01010101u, t);
        loc = t;
      } else if constexpr (N == 16) {
        uint32_t t = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) t = __dp2a_lo(q[k], 0x0101u, t);
        loc = t;
      } else {
#pragma unroll
        for (int k = 0; k < 32; ++k) loc += (Acc)q[k];
      }
      Acc inc = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const Acc t = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += t;
      }
      // the last id bounds them all (ids never decrease).  In a valid stream
      // every prefix of the deltas is an id difference below 2^31, so the
      // 32-bit sums of float streams cannot wrap; float64 streams sum in 64
      // bits.  (A corrupt stream can only yield wrong coordinates here, no
      // access depends on the ids.)
      const unsigned long long total = (unsigned long long)__shfl_sync(FULL, inc, 31);
      fast = first + total < (1ull << 31) && !g.wide && bnx != 0 && bny != 0 && bnx * bny < (1ull << 32);
      if constexpr (PASS == kPassFast) {
        // the fast layout has no id tables: ids of 2^31 or more (which no
        // valid stream holds, ids are masked to 31 bits) are rejected
        if (!fast) {
          bail = true;
          return;
        }
      }
      scatter_runs<T, N, Cfg>(q, P16, sw, (Acc)first + (inc - loc), nl, fast, lane);
    };
    uint32_t orw = 0;
    if (dbits <= 8u) {
      uint32_t q[8];
      section_words<8>(q, rawd, pw, 0u, dbits, bpp, endd, vmd, lane, orw);
      run_ids(q);
    } else if (dbits <= 16u) {
      uint32_t q[16];
      section_words<16>(q, rawd, pw, 0u, dbits, bpp, endd, vmd, lane, orw);
      run_ids(q);
    } else {
      uint32_t q[32];
      section_words<32>(q, rawd, pw, 0u, dbits, bpp, endd, vmd, lane, orw);
      run_ids(q);
    }
  }
  if (bail) {
    if (lane == 0) set_status(ctl, kESTREAM);
    return;
  }
  __syncwarp();

  // ---- every position's id (or run): inclusive max-scan of the run map ----
  {
    uint32_t v[32];
    uint32_t mx = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint4 t = *reinterpret_cast<const uint4 *>(A + qoff(lane, m));
      mx = max(mx, t.x); v[4 * m] = mx;
      mx = max(mx, t.y); v[4 * m + 1] = mx;
      mx = max(mx, t.z); v[4 * m + 2] = mx;
      mx = max(mx, t.w); v[4 * m + 3] = mx;
    }
    uint32_t inc = mx;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc = max(inc, t);
    }
    uint32_t pre = __shfl_up_sync(FULL, inc, 1);
    if (lane == 0) pre = 0;
    uint32_t *const P = sw + Cfg::P;
    const uint32_t *const TL = sw + Cfg::TL;
    const bool gather = !is64 && !fast;  // float general path: run index -> 32-bit id
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      uint32_t o[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t r = max(v[4 * m + e], pre);
        o[e] = gather ? TL[swz((int)r)] : r;
      }
      *reinterpret_cast<uint4 *>(P + qoff(lane, m)) = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
  __syncwarp();  // the float id table becomes the relative-position rows

  // ---- relative positions of this lane's 32 positions ----
  {
    uint32_t *const R = sw + Cfg::R;
    uint32_t orw = 0;
    auto put = [&](auto &q) {
      constexpr int N = sizeof(q) / sizeof(uint32_t);
#pragma unroll
      for (int m = 0; m < 8; ++m)
        *reinterpret_cast<uint4 *>(R + qoff(lane, m)) =
            make_uint4(word_value<N>(q, 4 * m), word_value<N>(q, 4 * m + 1), word_value<N>(q, 4 * m + 2),
                       word_value<N>(q, 4 * m + 3));
    };
    if (rbits <= 8u) {
      uint32_t q[8];
      section_words<8>(q, rawr, pw, db + cb, rbits, 0u, 0u, FULL, lane, orw);
      put(q);
    } else if (rbits <= 16u) {
      uint32_t q[16];
      section_words<16>(q, rawr, pw, db + cb, rbits, 0u, 0u, FULL, lane, orw);
      put(q);
    } else {
      uint32_t q[32];
      section_words<32>(q, rawr, pw, db + cb, rbits, 0u, 0u, FULL, lane, orw);
      put(q);
    }
  }

  // ---- reconstruct ----
  const bool full = nvalid == (uint32_t)kChunk && a.vec_ok;
  if (fast) {
    reconstruct<T, DIM, 0, Cfg>(sw, g, eb, mm, Y, base, lane, nvalid, full);
  } else {
    FastDiv f;
    f.init(my_div);
    g.fx.d = __shfl_sync(FULL, f.d, 0); g.fx.m = __shfl_sync(FULL, f.m, 0); g.fx.s = __shfl_sync(FULL, f.s, 0);
    g.fy.d = __shfl_sync(FULL, f.d, 1); g.fy.m = __shfl_sync(FULL, f.m, 1); g.fy.s = __shfl_sync(FULL, f.s, 1);
    g.fxy.d = __shfl_sync(FULL, f.d, 2); g.fxy.m = __shfl_sync(FULL, f.m, 2); g.fxy.s = __shfl_sync(FULL, f.s, 2);
    if constexpr (PASS != kPassFast) {
      if constexpr (!is64) reconstruct<T, DIM, 1, Cfg>(sw, g, eb, mm, Y, base, lane, nvalid, full);
      else reconstruct<T, DIM, 2, Cfg>(sw, g, eb, mm, Y, base, lane, nvalid, full);
    }
  }
}

// Persistent decompress kernel.  Float streams: one pass (PASS kPassAll) in
// the float layout.  Float64 streams: the fast pass in the 12 KB layout, then
// the general pass, which returns at once unless the fast pass left chunks.
template <typename T, int DIM, class Cfg = DecCfg<T>, int PASS = kPassAll>
__global__ void __launch_bounds__(32 * Cfg::warps, Cfg::min_ctas) decompress_kernel(const DArgs<T> a) {
  using Tr = TT<T>;
  constexpr int W = Cfg::warps;
  extern __shared__ __align__(16) uint32_t dec_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *const sw = dec_smem + warp * Cfg::words;
  Control *ctl = a.ctl;
  if (PASS == kPassGeneral && ld_volatile(&ctl->deferred) == 0u) return;
  // ---- header (:1801-1828) ----
  if (a.bytes < Tr::hdr) { if (threadIdx.x == 0) set_status(ctl, kESTREAM); return; }
  const uint32_t dim = *reinterpret_cast<const uint32_t *>(a.s);
  unsigned long long n;
  memcpy(&n, a.s + 4, 8);
  const uint32_t bits = *reinterpret_cast<const uint32_t *>(a.s + 12);
  T eb;
  memcpy(&eb, a.s + 16, sizeof(T));
  const uint32_t seg = *reinterpret_cast<const uint32_t *>(a.s + 16 + sizeof(T));
  const unsigned long long G = (n + kChunk - 1) / kChunk;
  if (bits != Tr::bits || dim != (uint32_t)DIM || n == 0 || seg == 0 ||
      G > (a.bytes - Tr::hdr) / (8ull + Tr::meta)) {
    if (threadIdx.x == 0) set_status(ctl, kESTREAM);
    return;
  }
  if (n > a.cap) { if (threadIdx.x == 0) set_status(ctl, kENOSPACE); return; }
  const unsigned long long pay_base = Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * G;
  const unsigned long long nwarps = (unsigned long long)gridDim.x * W;
  ChunkGeom g;
  g.seg = seg;
  g.sh = (uint32_t)__ffs((int)seg) - 1u;
  g.msk = seg - 1u;

  unsigned long long c = (unsigned long long)blockIdx.x * W + warp;
  uint32_t mw = c < G ? dec_meta_word<T>(a.s, G, c, lane) : 0u;
  for (; c < G; c += nwarps) {
    const uint32_t mwc = mw;
    if (c + nwarps < G) mw = dec_meta_word<T>(a.s, G, c + nwarps, lane);  // next record, in flight meanwhile
    decode_chunk<T, DIM, Cfg, PASS>(a, c, n, G, pay_base, eb, seg, g, mwc, sw, lane);
  }
}

}  // namespace gpzb
