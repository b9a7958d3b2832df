// gpz_batch.cuh -- batched compress: many snapshots of one (float type,
// dimension) class in one persistent launch.
//
// The reference compresses one snapshot per call (CompressorManager::compressWarp,
// src/CompressorManager.cpp:12-16), so a workload of many small snapshots is
// dominated by per-call launches, syncs and an almost idle GPU.  Here every
// snapshot keeps its own stream, control block and look-back words; the
// groups of 8 chunks of all snapshots of a class form one global work list
// (snapshot after snapshot, so each snapshot's groups are claimed in order),
// and one persistent kernel per class claims them.  A snapshot's stream is
// byte-identical to the one gpz_compress writes for it: the per-chunk
// encoder, the placement and the header/meta writes are the same code.
#pragma once

#include "gpz_kernels.cuh"
#include "gpz_encode.cuh"
#include "gpz_decode.cuh"

namespace gpzb {

constexpr uint32_t kBatchSegFixed = 1u;  // the segment size is given (no sampling)
constexpr uint32_t kBatchSafe31 = 2u;    // GPZ_FLAG_SAFE31 rules for the automatic segment size
constexpr uint32_t kBatchRelDev = 4u;    // absolute bound computed on the device from rel_eb
constexpr int kBatchLocalBits = 40;      // map entry: item << 40 | group within the item

// One snapshot of a batch.  `a` is what the single-stream kernel gets as its
// parameter; a.eb is rewritten on the device when kBatchRelDev is set.
template <typename T>
struct BItem {
  CArgs<T> a;
  Control *rctl;     // control block of the device rel->abs reduction
  T rel_eb;
  uint32_t seg_in;
  int32_t rel_mode;
  uint32_t flags;
};

// computeSegSize for every snapshot of the class (blockIdx.y = snapshot, 128
// blocks each), or the given segment size.
template <typename T>
__global__ void __launch_bounds__(256) batch_sample_kernel(const BItem<T> *items) {
  const BItem<T> &it = items[blockIdx.y];
  if (it.flags & kBatchSegFixed) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      it.a.ctl->seg = it.seg_in;
      it.a.ctl->adjusted = 0;
    }
    return;
  }
  seg_sample_block<T>(it.a.x, it.a.y, it.a.z, it.a.n, it.a.dim, it.seg_in, it.rel_mode, it.rel_eb, it.a.eb,
                      (it.flags & kBatchSafe31) ? 1 : 0, it.a.ctl, blockIdx.x, gridDim.x);
}

template <int W>
struct BatchGroup {
  uint32_t sz[W];             // payload bytes of each warp's chunk
  unsigned long long goff;    // stream offset of the group (~0: look-back gave up)
  unsigned long long next;    // next global group
  unsigned long long nmap;    // its map entry
};

// The compress loop of compress_kernel over a work list of many snapshots:
// map[g] = snapshot << 40 | group of global group g.  The arguments of the
// current and the next group's snapshot live in shared memory (double
// buffered: the next group's points are loaded before the current group's
// copy-out).  A snapshot whose segment size could not be chosen (sampling
// error, status set) is skipped as a whole.  Groups of W chunks, as in
// compress_kernel<T, DIM>.
template <typename T, int DIM, int W = enc_warps<T, DIM>()>
__global__ void __launch_bounds__(32 * W, GPZ_ENC_MIN_CTAS)
    compress_batch_kernel(const BItem<T> *__restrict__ items, const unsigned long long *__restrict__ map,
                          unsigned long long total, unsigned long long *claim) {
  using Tr = TT<T>;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  constexpr unsigned long long kLocal = (1ull << kBatchLocalBits) - 1;
  extern __shared__ __align__(16) uint32_t enc_smem[];
  __shared__ BatchGroup<W> eg;
  __shared__ CArgs<T> args[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *const sw = enc_smem + warp * kEncWords;
  auto claim_next = [&](int slot) {  // thread 0
    const unsigned long long g = atomicAdd(claim, 1ull);
    eg.next = g;
    // past the end: the first snapshot's first group stands in, so the
    // prefetch below needs no condition (its loads are never used)
    const unsigned long long m = g < total ? map[g] : 0ull;
    eg.nmap = m;
    args[slot] = items[m >> kBatchLocalBits].a;
  };
  if (threadIdx.x == 0) claim_next(0);
  __syncthreads();
  ChunkPoints<T, DIM> pts;
  pts.load(args[0], (eg.nmap & kLocal) * W + warp, lane);
  int slot = 0;
  uint32_t rank_skip = 0;
  for (;;) {
    const unsigned long long g = eg.next;
    if (g >= total) break;
    const unsigned long long m = eg.nmap;
    __syncthreads();  // B0: everyone has the group before it is replaced
    if (threadIdx.x == 0) claim_next(slot ^ 1);
    const CArgs<T> &a = args[slot];
    Control *ctl = a.ctl;
    const unsigned long long G = a.G;
    const unsigned long long gid = m & kLocal, gbase = gid * W;
    const uint32_t seg = ctl->seg;  // 0: the snapshot's sampling failed
    const bool live = seg != 0;
    const uint32_t sh = live ? (uint32_t)__ffs((int)seg) - 1u : 0u, msk = seg - 1u;
    const T eb = a.eb;
    const T inv = is64 ? (T)__ddiv_rn(1.0, __dmul_rn(2.0, (double)eb)) : (T)__fdiv_rn(1.0f, __fmul_rn(2.0f, (float)eb));
    const unsigned long long pay_base = Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * G;
    const unsigned long long c = gbase + warp;
    uint32_t tot = 0;
    auto on_size = [&](uint32_t bytes) {
      if (lane == 0) eg.sz[warp] = bytes;
      __syncthreads();  // B1: the group's sizes are known (and the next group's snapshot)
      if (live && warp == 0) {
        const uint32_t s = lane < W ? eg.sz[lane] : 0u;
        tot = __reduce_add_sync(FULL, s);
        if (lane == 0) publish_aggregate(a.look, gid, tot);
      }
    };
    uint32_t payload = 0, meta_word = 0;
    if (live && c < G) payload = encode_chunk<T, DIM>(a, c, sw, seg, sh, msk, eb, inv, pts, meta_word, lane, rank_skip, on_size);
    else on_size(0u);
    if (live && warp == 0) {
      unsigned long long excl = 0;
      const bool ok = resolve_prefix(a.look, gid, tot, ctl, excl);
      if (lane == 0) eg.goff = ok ? excl : ~0ull;
    }
    pts.load(args[slot ^ 1], (eg.nmap & kLocal) * W + warp, lane);  // in flight during the copy-out
    __syncthreads();  // B2: the group's stream offset is known
    const unsigned long long goff = eg.goff;
    if (live && c < G && goff != ~0ull) {
      unsigned long long off = goff;
      for (int w = 0; w < warp; ++w) off += eg.sz[w];
      place_chunk<T>(a, c, G, pay_base, off, payload, meta_word, seg, eb, sw, lane);
    }
    slot ^= 1;
  }
}

// ---------------------------------------------------------------------------
// Batched decompress.
// ---------------------------------------------------------------------------

// One stream of a decompress batch; n is the point count the caller read
// from the stream's header (the work map is built from it); G, pay_base, eb,
// seg and ok come from the device-side header check.
template <typename T>
struct DItem {
  DArgs<T> a;
  unsigned long long n, G, pay_base;
  T eb;
  uint32_t seg;
  int32_t ok;
};

// The header checks of decompress_kernel, once per stream (one thread each).
template <typename T, int DIM>
__global__ void dbatch_header_kernel(DItem<T> *items, uint32_t K) {
  using Tr = TT<T>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  DItem<T> &it = items[k];
  it.ok = 0;
  Control *ctl = it.a.ctl;
  if (it.a.bytes < Tr::hdr) { set_status(ctl, kESTREAM); return; }
  const uint8_t *s = it.a.s;
  const uint32_t dim = *reinterpret_cast<const uint32_t *>(s);
  unsigned long long n;
  memcpy(&n, s + 4, 8);
  const uint32_t bits = *reinterpret_cast<const uint32_t *>(s + 12);
  T eb;
  memcpy(&eb, s + 16, sizeof(T));
  const uint32_t seg = *reinterpret_cast<const uint32_t *>(s + 16 + sizeof(T));
  const unsigned long long G = (n + kChunk - 1) / kChunk;
  if (bits != Tr::bits || dim != (uint32_t)DIM || n == 0 || n != it.n || seg == 0 ||
      G > (it.a.bytes - Tr::hdr) / (8ull + Tr::meta)) {
    set_status(ctl, kESTREAM);
    return;
  }
  if (n > it.a.cap) { set_status(ctl, kENOSPACE); return; }
  it.G = G;
  it.pay_base = Tr::hdr + 8ull * G + (unsigned long long)Tr::meta * G;
  it.eb = eb;
  it.seg = seg;
  it.ok = 1;
}

// decompress_kernel over the chunks of many streams: warps stride over the
// global chunk list, cmap[c] = stream << 40 | chunk within the stream.  The
// passes are decompress_kernel's: float64 classes run the fast pass in the
// 12 KB layout, then the general pass, which skips every stream whose fast
// pass left no chunk.
template <typename T, int DIM, class Cfg = DecCfg<T>, int PASS = kPassAll>
__global__ void __launch_bounds__(32 * Cfg::warps, Cfg::min_ctas)
    decompress_batch_kernel(const DItem<T> *__restrict__ items, const unsigned long long *__restrict__ cmap,
                            unsigned long long total) {
  constexpr int W = Cfg::warps;
  constexpr unsigned long long kLocal = (1ull << kBatchLocalBits) - 1;
  extern __shared__ __align__(16) uint32_t dec_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *const sw = dec_smem + warp * Cfg::words;
  const unsigned long long nwarps = (unsigned long long)gridDim.x * W;
  for (unsigned long long gc = (unsigned long long)blockIdx.x * W + warp; gc < total; gc += nwarps) {
    const unsigned long long m = cmap[gc];
    const DItem<T> &it = items[m >> kBatchLocalBits];
    if (!it.ok) continue;
    if (PASS == kPassGeneral && ld_volatile(&it.a.ctl->deferred) == 0u) continue;
    const DArgs<T> a = it.a;
    const unsigned long long c = m & kLocal, G = it.G;
    const uint32_t seg = it.seg;
    ChunkGeom g;
    g.seg = seg;
    g.sh = (uint32_t)__ffs((int)seg) - 1u;
    g.msk = seg - 1u;
    const uint32_t mwc = dec_meta_word<T>(a.s, G, c, lane);
    decode_chunk<T, DIM, Cfg, PASS>(a, c, it.n, G, it.pay_base, it.eb, seg, g, mwc, sw, lane);
  }
}

}  // namespace gpzb
