// gpz_batchapi.cu -- C ABI of the batched compress (include/gpz_b200.h,
// gpz_batch_*): plan creation, graph capture, launch and results.
//
// Device memory of a batch (one allocation):
//   [controls: 256 B per snapshot][rel controls: 256 B per snapshot]
//   [look-back words: one per 8-chunk group of every snapshot][claim counters]
//     -- zeroed at the start of every launch (a memset node of the graph)
//   [per class: item descriptors (BItem<T>), group map, rel-block map]
// Classes are (float, 2D), (float, 3D), (double, 2D), (double, 3D); the graph
// runs them one after another: rel->abs (when any of its snapshots asks for
// it), sampling, persistent compress.

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "gpz_b200.h"
#include "gpz_batch.cuh"

using namespace gpzb;

namespace {

constexpr uint64_t kRelPointsPerBlock = 1u << 16;  // points per rel->abs block of a snapshot
constexpr uint32_t kRelMaxBlocks = 256;

inline uint64_t align256(uint64_t v) { return (v + 255u) & ~255ull; }

int class_of(uint32_t bits, uint32_t dim) { return (bits == 64 ? 2 : 0) + (dim == 3 ? 1 : 0); }

struct ClassPlan {
  std::vector<uint32_t> items;  // batch indices, in work-list order
  uint64_t groups = 0;          // 8-chunk groups of all its snapshots
  uint64_t rel_blocks = 0;      // rel->abs blocks (snapshots with GPZ_FLAG_REL_ON_DEVICE)
  uint64_t table_off = 0, map_off = 0, rmap_off = 0;
  int grid = 0;
};

template <typename T>
void fill_item(BItem<T> &bi, const gpz_batch_item &it, uint8_t *dev, uint64_t ctl_off, uint64_t rctl_off,
               uint64_t look_off) {
  memset(&bi, 0, sizeof(bi));
  bi.a.x = static_cast<const T *>(it.d_x);
  bi.a.y = static_cast<const T *>(it.d_y);
  bi.a.z = static_cast<const T *>(it.dim == 3 ? it.d_z : it.d_y);
  bi.a.out = static_cast<uint8_t *>(it.d_out);
  bi.a.out_cap = it.out_capacity;
  bi.a.ctl = reinterpret_cast<Control *>(dev + ctl_off);
  bi.a.look = reinterpret_cast<unsigned long long *>(dev + look_off);
  bi.a.n = it.n;
  bi.a.G = (it.n + kChunk - 1) / kChunk;
  bi.a.eb = (T)it.eb;
  bi.a.dim = it.dim;
  auto al = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  bi.a.vec_ok = al(it.d_x) && al(it.d_y) && (it.dim == 2 || al(it.d_z));
  bi.rctl = reinterpret_cast<Control *>(dev + rctl_off);
  bi.rel_eb = (T)it.rel_eb;
  bi.seg_in = it.seg_size;
  bi.rel_mode = it.rel_mode;
  bi.flags = ((it.flags & GPZ_FLAG_SEG_FIXED) ? kBatchSegFixed : 0u) | ((it.flags & GPZ_FLAG_SAFE31) ? kBatchSafe31 : 0u) |
             ((it.flags & GPZ_FLAG_REL_ON_DEVICE) ? kBatchRelDev : 0u);
}

// findMinimumValues + convertRelEb for the GPZ_FLAG_REL_ON_DEVICE snapshots
// of a class, sized to each snapshot: rmap[block] = snapshot << 40 |
// blocks of the snapshot << 20 | block within the snapshot.  The result is
// exactly gpz_rel_to_abs's (min and max do not depend on the partition) and
// goes to the snapshot's descriptor, where sampling and compress read it.
template <typename T>
__global__ void __launch_bounds__(256) batch_rel_mapped_kernel(BItem<T> *items, const unsigned long long *rmap) {
  const unsigned long long e = rmap[blockIdx.x];
  BItem<T> &it = items[e >> 40];
  const unsigned nb = (unsigned)((e >> 20) & 0xFFFFFu), b = (unsigned)(e & 0xFFFFFu);
  rel_to_abs_block<T>(it.a.x, it.a.y, it.a.z, it.a.n, it.a.dim, it.rel_eb, it.rctl, &it.a.eb, b, nb);
}

int num_sms_now() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

template <typename T, int DIM>
int compress_grid(uint64_t groups) {
  auto k = compress_batch_kernel<T, DIM>;
  const size_t smem = enc_smem_bytes();
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 32 * kEncWarps, smem) != cudaSuccess || occ < 1) occ = 1;
  return (int)std::min<uint64_t>(groups, (uint64_t)num_sms_now() * occ);
}

template <typename T, int DIM>
void enqueue_class(const ClassPlan &cp, uint8_t *dev, uint64_t claim_off, cudaStream_t st) {
  BItem<T> *tab = reinterpret_cast<BItem<T> *>(dev + cp.table_off);
  const unsigned long long *map = reinterpret_cast<const unsigned long long *>(dev + cp.map_off);
  if (cp.rel_blocks)
    batch_rel_mapped_kernel<T><<<(unsigned)cp.rel_blocks, 256, 0, st>>>(
        tab, reinterpret_cast<const unsigned long long *>(dev + cp.rmap_off));
  batch_sample_kernel<T><<<dim3(128, (unsigned)cp.items.size()), 256, 0, st>>>(tab);
  compress_batch_kernel<T, DIM><<<cp.grid, 32 * kEncWarps, enc_smem_bytes(), st>>>(
      tab, map, cp.groups, reinterpret_cast<unsigned long long *>(dev + claim_off));
}

}  // namespace

struct gpz_batch {
  int device = 0;
  uint32_t count = 0;
  uint8_t *mem = nullptr;
  uint64_t bytes = 0, zero_bytes = 0;
  std::vector<gpz_batch_item> items;
  cudaGraphExec_t exec = nullptr;
};

extern "C" {

int gpz_batch_create(const gpz_batch_item *items, uint32_t count, gpz_batch **batch, uint32_t *bad_item) {
  if (!batch || !items || count == 0) return GPZ_EINVAL;
  *batch = nullptr;
  for (uint32_t i = 0; i < count; ++i) {
    const gpz_batch_item &it = items[i];
    const uint64_t G = (it.n + kChunk - 1) / kChunk;
    const uint64_t hdr = it.float_bits == 64 ? 32 : 24, meta = it.float_bits == 64 ? 64 : 36;
    const bool ok = (it.float_bits == 32 || it.float_bits == 64) && (it.dim == 2 || it.dim == 3) && it.n >= 1 &&
                    it.d_x && it.d_y && (it.dim == 2 || it.d_z) && it.d_out &&
                    it.out_capacity >= hdr + G * (8 + meta) && !((it.flags & GPZ_FLAG_SEG_FIXED) && it.seg_size == 0) &&
                    (it.flags & ~(GPZ_FLAG_SAFE31 | GPZ_FLAG_SEG_FIXED | GPZ_FLAG_REL_ON_DEVICE)) == 0;
    if (!ok) {
      if (bad_item) *bad_item = i;
      return GPZ_EINVAL;
    }
  }
  gpz_batch *b = new (std::nothrow) gpz_batch;
  if (!b) return GPZ_ECUDA;
  b->count = count;
  b->items.assign(items, items + count);
  cudaGetDevice(&b->device);

  // ---- layout
  ClassPlan cls[4];
  std::vector<uint64_t> look_off(count);
  uint64_t off = 2ull * count * kCtlBytes;
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t G = (items[i].n + kChunk - 1) / kChunk, groups = (G + kEncWarps - 1) / kEncWarps;
    look_off[i] = off;
    off += 8 * groups;
    ClassPlan &cp = cls[class_of(items[i].float_bits, items[i].dim)];
    cp.items.push_back(i);
    cp.groups += groups;
    if (items[i].flags & GPZ_FLAG_REL_ON_DEVICE)
      cp.rel_blocks += std::min<uint64_t>(kRelMaxBlocks, std::max<uint64_t>(1, items[i].n / kRelPointsPerBlock));
  }
  const uint64_t claim_off = align256(off);
  b->zero_bytes = claim_off + 4 * 8;
  off = align256(b->zero_bytes);
  for (int c = 0; c < 4; ++c) {
    if (cls[c].items.empty()) continue;
    const uint64_t isz = c < 2 ? sizeof(BItem<float>) : sizeof(BItem<double>);
    cls[c].table_off = off;
    off = align256(off + isz * cls[c].items.size());
    cls[c].map_off = off;
    off = align256(off + 8 * cls[c].groups);
    cls[c].rmap_off = off;
    off = align256(off + 8 * cls[c].rel_blocks);
  }
  b->bytes = off;
  if (cudaMalloc(&b->mem, b->bytes) != cudaSuccess) {
    delete b;
    return GPZ_ECUDA;
  }

  // ---- descriptors and maps (host-built, uploaded once)
  std::vector<uint8_t> host(b->bytes - b->zero_bytes);
  auto H = [&](uint64_t dev_off) { return host.data() + (dev_off - b->zero_bytes); };
  for (int c = 0; c < 4; ++c) {
    ClassPlan &cp = cls[c];
    if (cp.items.empty()) continue;
    uint64_t g = 0, rb = 0;
    for (size_t k = 0; k < cp.items.size(); ++k) {
      const uint32_t i = cp.items[k];
      const gpz_batch_item &it = items[i];
      if (c < 2) fill_item<float>(reinterpret_cast<BItem<float> *>(H(cp.table_off))[k], it, b->mem,
                                  (uint64_t)i * kCtlBytes, (uint64_t)(count + i) * kCtlBytes, look_off[i]);
      else fill_item<double>(reinterpret_cast<BItem<double> *>(H(cp.table_off))[k], it, b->mem,
                             (uint64_t)i * kCtlBytes, (uint64_t)(count + i) * kCtlBytes, look_off[i]);
      const uint64_t G = (it.n + kChunk - 1) / kChunk, groups = (G + kEncWarps - 1) / kEncWarps;
      unsigned long long *map = reinterpret_cast<unsigned long long *>(H(cp.map_off));
      for (uint64_t q = 0; q < groups; ++q) map[g++] = ((unsigned long long)k << kBatchLocalBits) | q;
      if (it.flags & GPZ_FLAG_REL_ON_DEVICE) {
        const uint64_t nb = std::min<uint64_t>(kRelMaxBlocks, std::max<uint64_t>(1, it.n / kRelPointsPerBlock));
        unsigned long long *rmap = reinterpret_cast<unsigned long long *>(H(cp.rmap_off));
        for (uint64_t q = 0; q < nb; ++q) rmap[rb++] = ((unsigned long long)k << 40) | (nb << 20) | q;
      }
    }
    switch (c) {
      case 0: cp.grid = compress_grid<float, 2>(cp.groups); break;
      case 1: cp.grid = compress_grid<float, 3>(cp.groups); break;
      case 2: cp.grid = compress_grid<double, 2>(cp.groups); break;
      default: cp.grid = compress_grid<double, 3>(cp.groups); break;
    }
    if (cp.grid < 1) {
      cudaFree(b->mem);
      delete b;
      return GPZ_ECUDA;
    }
  }
  if (cudaMemcpy(b->mem + b->zero_bytes, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(b->mem);
    delete b;
    return GPZ_ECUDA;
  }

  // ---- graph: memset, then one branch per class
  cudaStream_t s0 = nullptr;
  cudaGraph_t graph = nullptr;
  bool okc = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking) == cudaSuccess;
  if (okc) okc = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (okc) {
    // The classes run one after another: two different compress kernels
    // resident on one SM thrash its instruction cache (each is a few hundred
    // KB of unrolled code), which costs far more than the overlap gains.
    cudaMemsetAsync(b->mem, 0, b->zero_bytes, s0);
    for (int c = 0; c < 4; ++c) {
      if (cls[c].items.empty()) continue;
      const uint64_t claim = claim_off + 8ull * c;
      switch (c) {
        case 0: enqueue_class<float, 2>(cls[c], b->mem, claim, s0); break;
        case 1: enqueue_class<float, 3>(cls[c], b->mem, claim, s0); break;
        case 2: enqueue_class<double, 2>(cls[c], b->mem, claim, s0); break;
        default: enqueue_class<double, 3>(cls[c], b->mem, claim, s0); break;
      }
    }
    okc = cudaStreamEndCapture(s0, &graph) == cudaSuccess && graph;
  }
  if (okc) okc = cudaGraphInstantiate(&b->exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (s0) cudaStreamDestroy(s0);
  if (!okc) {
    cudaGetLastError();
    cudaFree(b->mem);
    delete b;
    return GPZ_ECUDA;
  }
  *batch = b;
  return GPZ_OK;
}

int gpz_batch_launch(gpz_batch *b, void *stream) {
  if (!b || !b->exec) return GPZ_EINVAL;
  return cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
}

int gpz_batch_results(gpz_batch *b, gpz_result *results, double *h_eb, void *stream) {
  if (!b || !results) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<Control> h(2ull * b->count);
  static_assert(sizeof(Control) <= kCtlBytes, "control block");
  for (uint32_t i = 0; i < 2 * b->count; ++i)
    if (cudaMemcpyAsync(&h[i], b->mem + (uint64_t)i * kCtlBytes, sizeof(Control), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      return GPZ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GPZ_ECUDA;
  for (uint32_t i = 0; i < b->count; ++i) {
    const Control &c = h[i];
    results[i].stream_bytes = c.stream_bytes;
    results[i].seg_size = c.seg;
    results[i].adjusted = c.adjusted;
    results[i].status = c.status;
    results[i].id_overflow = c.id_overflow;
    if (h_eb) {
      const gpz_batch_item &it = b->items[i];
      if (it.flags & GPZ_FLAG_REL_ON_DEVICE) h_eb[i] = h[b->count + i].out_eb;
      else h_eb[i] = it.float_bits == 32 ? (double)(float)it.eb : it.eb;
    }
  }
  return GPZ_OK;
}

uint64_t gpz_batch_device_bytes(const gpz_batch *b) { return b ? b->bytes : 0; }

int gpz_batch_destroy(gpz_batch *b) {
  if (!b) return GPZ_EINVAL;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->mem) cudaFree(b->mem);
  delete b;
  return GPZ_OK;
}

}  // extern "C"

// ===========================================================================
// Batched decompress.
// ===========================================================================
namespace {

template <typename T, int DIM>
int dec_grid(uint64_t chunks) {
  auto k = decompress_batch_kernel<T, DIM>;
  constexpr size_t smem = dec_smem_bytes<T>();
  constexpr int W = DecCfg<T>::warps;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 32 * W, smem) != cudaSuccess || occ < 1) occ = 1;
  return (int)std::min<uint64_t>((chunks + W - 1) / W, (uint64_t)num_sms_now() * occ);
}

struct DClass {
  std::vector<uint32_t> items;
  uint64_t chunks = 0, table_off = 0, map_off = 0;
  int grid = 0;
};

template <typename T, int DIM>
void enqueue_dclass(const DClass &cp, uint8_t *dev, cudaStream_t st) {
  DItem<T> *tab = reinterpret_cast<DItem<T> *>(dev + cp.table_off);
  const uint32_t K = (uint32_t)cp.items.size();
  dbatch_header_kernel<T, DIM><<<(K + 127) / 128, 128, 0, st>>>(tab, K);
  decompress_batch_kernel<T, DIM><<<cp.grid, 32 * DecCfg<T>::warps, dec_smem_bytes<T>(), st>>>(
      tab, reinterpret_cast<const unsigned long long *>(dev + cp.map_off), cp.chunks);
}

template <typename T>
void fill_ditem(DItem<T> &d, const gpz_dbatch_item &it, Control *ctl) {
  memset(&d, 0, sizeof(d));
  d.a.s = static_cast<const uint8_t *>(it.d_stream);
  d.a.bytes = it.stream_bytes;
  d.a.x = static_cast<T *>(it.d_x);
  d.a.y = static_cast<T *>(it.d_y);
  d.a.z = static_cast<T *>(it.dim == 3 ? it.d_z : it.d_y);
  d.a.cap = it.out_capacity;
  d.a.ctl = ctl;
  auto al = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  d.a.vec_ok = al(it.d_x) && al(it.d_y) && (it.dim == 2 || al(it.d_z));
  d.n = it.n;
}

}  // namespace

struct gpz_dbatch {
  uint32_t count = 0;
  uint8_t *mem = nullptr;
  uint64_t bytes = 0, zero_bytes = 0;
  cudaGraphExec_t exec = nullptr;
};

extern "C" {

int gpz_dbatch_create(const gpz_dbatch_item *items, uint32_t count, gpz_dbatch **batch, uint32_t *bad_item) {
  if (!batch || !items || count == 0) return GPZ_EINVAL;
  *batch = nullptr;
  for (uint32_t i = 0; i < count; ++i) {
    const gpz_dbatch_item &it = items[i];
    const bool ok = (it.float_bits == 32 || it.float_bits == 64) && (it.dim == 2 || it.dim == 3) && it.n >= 1 &&
                    it.d_stream && ((uintptr_t)it.d_stream & 7u) == 0 && it.d_x && it.d_y &&
                    (it.dim == 2 || it.d_z) && it.out_capacity >= it.n;
    if (!ok) {
      if (bad_item) *bad_item = i;
      return GPZ_EINVAL;
    }
  }
  gpz_dbatch *b = new (std::nothrow) gpz_dbatch;
  if (!b) return GPZ_ECUDA;
  b->count = count;
  DClass cls[4];
  for (uint32_t i = 0; i < count; ++i) {
    DClass &cp = cls[class_of(items[i].float_bits, items[i].dim)];
    cp.items.push_back(i);
    cp.chunks += (items[i].n + kChunk - 1) / kChunk;
  }
  b->zero_bytes = (uint64_t)count * kCtlBytes;
  uint64_t off = align256(b->zero_bytes);
  for (int c = 0; c < 4; ++c) {
    if (cls[c].items.empty()) continue;
    const uint64_t isz = c < 2 ? sizeof(DItem<float>) : sizeof(DItem<double>);
    cls[c].table_off = off;
    off = align256(off + isz * cls[c].items.size());
    cls[c].map_off = off;
    off = align256(off + 8 * cls[c].chunks);
  }
  b->bytes = off;
  if (cudaMalloc(&b->mem, b->bytes) != cudaSuccess) {
    delete b;
    return GPZ_ECUDA;
  }
  std::vector<uint8_t> host(b->bytes - b->zero_bytes);
  auto H = [&](uint64_t dev_off) { return host.data() + (dev_off - b->zero_bytes); };
  for (int c = 0; c < 4; ++c) {
    DClass &cp = cls[c];
    if (cp.items.empty()) continue;
    uint64_t q = 0;
    for (size_t k = 0; k < cp.items.size(); ++k) {
      const uint32_t i = cp.items[k];
      Control *ctl = reinterpret_cast<Control *>(b->mem + (uint64_t)i * kCtlBytes);
      if (c < 2) fill_ditem<float>(reinterpret_cast<DItem<float> *>(H(cp.table_off))[k], items[i], ctl);
      else fill_ditem<double>(reinterpret_cast<DItem<double> *>(H(cp.table_off))[k], items[i], ctl);
      const uint64_t G = (items[i].n + kChunk - 1) / kChunk;
      unsigned long long *map = reinterpret_cast<unsigned long long *>(H(cp.map_off));
      for (uint64_t ch = 0; ch < G; ++ch) map[q++] = ((unsigned long long)k << kBatchLocalBits) | ch;
    }
    switch (c) {
      case 0: cp.grid = dec_grid<float, 2>(cp.chunks); break;
      case 1: cp.grid = dec_grid<float, 3>(cp.chunks); break;
      case 2: cp.grid = dec_grid<double, 2>(cp.chunks); break;
      default: cp.grid = dec_grid<double, 3>(cp.chunks); break;
    }
    if (cp.grid < 1) {
      cudaFree(b->mem);
      delete b;
      return GPZ_ECUDA;
    }
  }
  if (cudaMemcpy(b->mem + b->zero_bytes, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(b->mem);
    delete b;
    return GPZ_ECUDA;
  }
  cudaStream_t s0 = nullptr;
  cudaGraph_t graph = nullptr;
  bool okc = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking) == cudaSuccess;
  if (okc) okc = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (okc) {
    cudaMemsetAsync(b->mem, 0, b->zero_bytes, s0);
    for (int c = 0; c < 4; ++c) {  // one class after another, as in the compress graph
      if (cls[c].items.empty()) continue;
      switch (c) {
        case 0: enqueue_dclass<float, 2>(cls[c], b->mem, s0); break;
        case 1: enqueue_dclass<float, 3>(cls[c], b->mem, s0); break;
        case 2: enqueue_dclass<double, 2>(cls[c], b->mem, s0); break;
        default: enqueue_dclass<double, 3>(cls[c], b->mem, s0); break;
      }
    }
    okc = cudaStreamEndCapture(s0, &graph) == cudaSuccess && graph;
  }
  if (okc) okc = cudaGraphInstantiate(&b->exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (s0) cudaStreamDestroy(s0);
  if (!okc) {
    cudaGetLastError();
    cudaFree(b->mem);
    delete b;
    return GPZ_ECUDA;
  }
  *batch = b;
  return GPZ_OK;
}

int gpz_dbatch_launch(gpz_dbatch *b, void *stream) {
  if (!b || !b->exec) return GPZ_EINVAL;
  return cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
}

int gpz_dbatch_results(gpz_dbatch *b, gpz_result *results, void *stream) {
  if (!b || !results) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<Control> h(b->count);
  for (uint32_t i = 0; i < b->count; ++i)
    if (cudaMemcpyAsync(&h[i], b->mem + (uint64_t)i * kCtlBytes, sizeof(Control), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      return GPZ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GPZ_ECUDA;
  for (uint32_t i = 0; i < b->count; ++i) {
    memset(&results[i], 0, sizeof(gpz_result));
    results[i].status = h[i].status;
  }
  return GPZ_OK;
}

int gpz_dbatch_destroy(gpz_dbatch *b) {
  if (!b) return GPZ_EINVAL;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->mem) cudaFree(b->mem);
  delete b;
  return GPZ_OK;
}

}  // extern "C"
