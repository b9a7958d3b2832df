// gpz_batchapi.cu -- batched compress / decompress: workspace layout, table
// building and kernel launches (gpz_batch_host.h), and the plan API of
// include/gpz_b200.h (gpz_batch_*, gpz_dbatch_*), which captures them in a
// CUDA graph.
//
// Classes are (float, 2D), (float, 3D), (double, 2D), (double, 3D); a batch
// runs them one after another: (compress) rel->abs when any of its snapshots
// asks for it, sampling, one persistent compress kernel; (decompress) a header
// check per stream, one persistent decompress kernel.  Two different codec
// kernels resident on one SM thrash its instruction cache (each is a few
// hundred KB of unrolled code), which costs far more than overlapping the
// classes would gain.

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "gpz_b200.h"
#include "gpz_batch.cuh"
#include "gpz_batch_host.h"
#include "gpz_launch.h"

using namespace gpzb;

namespace {

constexpr uint64_t kRelPointsPerBlock = 1u << 13;  // points per rel->abs block of a snapshot
constexpr uint64_t kRelMaxBlocks = 1024;

inline uint64_t align256(uint64_t v) { return (v + 255u) & ~255ull; }
inline uint64_t chunks_of(uint64_t n) { return (n + kChunk - 1) / kChunk; }
inline uint64_t rel_blocks_of(uint64_t n) { return std::min(kRelMaxBlocks, std::max<uint64_t>(1, n / kRelPointsPerBlock)); }
int class_of(uint32_t bits, uint32_t dim) { return (bits == 64 ? 2 : 0) + (dim == 3 ? 1 : 0); }
// chunks per group of a class's compress kernel (enc_warps of its float type and dimension)
constexpr int class_warps(int c) {
  return c == 0 ? enc_warps<float, 2>() : c == 1 ? enc_warps<float, 3>() : c == 2 ? enc_warps<double, 2>() : enc_warps<double, 3>();
}
inline uint64_t groups_of(uint64_t n, int c) { return (chunks_of(n) + class_warps(c) - 1) / class_warps(c); }

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
  bi.a.G = chunks_of(it.n);
  bi.a.eb = (T)it.eb;
  bi.a.eb_dev = nullptr;
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

// Grids of the batched persistent kernels on the current device (-1 when the
// kernel's shared-memory attribute cannot be raised there).
template <typename T, int DIM>
int compress_grid(uint64_t groups) {
  constexpr int W = enc_warps<T, DIM>();
  const int o = resident_ctas(compress_batch_kernel<T, DIM>, 32 * W, enc_smem_bytes<W>());
  return o ? (int)std::min<uint64_t>(groups, (uint64_t)current_sms() * o) : -1;
}

template <typename T, int DIM, class Cfg = DecCfg<T>, int PASS = kPassAll>
int dec_grid(uint64_t chunks) {
  constexpr int W = Cfg::warps;
  const int o = resident_ctas(decompress_batch_kernel<T, DIM, Cfg, PASS>, 32 * W, dec_smem_bytes_of<Cfg>());
  return o ? (int)std::min<uint64_t>((chunks + W - 1) / W, (uint64_t)current_sms() * o) : -1;
}

template <typename T, int DIM>
void enqueue_class(const gpzb_host::ClassPlan &cp, uint8_t *dev, uint64_t claim_off, cudaStream_t st) {
  BItem<T> *tab = reinterpret_cast<BItem<T> *>(dev + cp.table_off);
  if (cp.rel_blocks)
    batch_rel_mapped_kernel<T><<<(unsigned)cp.rel_blocks, 256, 0, st>>>(
        tab, reinterpret_cast<const unsigned long long *>(dev + cp.rmap_off));
  batch_sample_kernel<T><<<dim3(128, (unsigned)cp.items.size()), 256, 0, st>>>(tab);
  constexpr int W = enc_warps<T, DIM>();
  compress_batch_kernel<T, DIM><<<cp.grid, 32 * W, enc_smem_bytes<W>(), st>>>(
      tab, reinterpret_cast<const unsigned long long *>(dev + cp.map_off), cp.work,
      reinterpret_cast<unsigned long long *>(dev + claim_off));
}

template <typename T, int DIM>
void enqueue_dclass(const gpzb_host::ClassPlan &cp, uint8_t *dev, cudaStream_t st) {
  DItem<T> *tab = reinterpret_cast<DItem<T> *>(dev + cp.table_off);
  const uint32_t K = (uint32_t)cp.items.size();
  dbatch_header_kernel<T, DIM><<<(K + 127) / 128, 128, 0, st>>>(tab, K);
  const auto *map = reinterpret_cast<const unsigned long long *>(dev + cp.map_off);
  if constexpr (sizeof(T) == 4) {
    decompress_batch_kernel<T, DIM><<<cp.grid, 32 * DecCfg<T>::warps, dec_smem_bytes<T>(), st>>>(tab, map, cp.work);
  } else {
    decompress_batch_kernel<T, DIM, DecCfgF64Fast, kPassFast>
        <<<cp.grid, 32 * DecCfgF64Fast::warps, dec_smem_bytes_of<DecCfgF64Fast>(), st>>>(tab, map, cp.work);
    decompress_batch_kernel<T, DIM, DecCfg<T>, kPassGeneral>
        <<<cp.grid2, 32 * DecCfg<T>::warps, dec_smem_bytes<T>(), st>>>(tab, map, cp.work);
  }
}

}  // namespace

// ===========================================================================
// Workspace layout, tables, launches.
// ===========================================================================
namespace gpzb_host {

bool compress_item_ok(const gpz_batch_item &it) {
  const uint64_t hdr = it.float_bits == 64 ? 32 : 24, meta = it.float_bits == 64 ? 64 : 36;
  return (it.float_bits == 32 || it.float_bits == 64) && (it.dim == 2 || it.dim == 3) && it.n >= 1 && it.d_x &&
         it.d_y && (it.dim == 2 || it.d_z) && it.d_out && it.out_capacity >= hdr + chunks_of(it.n) * (8 + meta) &&
         !((it.flags & GPZ_FLAG_SEG_FIXED) && it.seg_size == 0) &&
         (it.flags & ~(GPZ_FLAG_SAFE31 | GPZ_FLAG_SEG_FIXED | GPZ_FLAG_REL_ON_DEVICE)) == 0;
}

bool decompress_item_ok(const gpz_dbatch_item &it) {
  return (it.float_bits == 32 || it.float_bits == 64) && (it.dim == 2 || it.dim == 3) && it.n >= 1 && it.d_stream &&
         ((uintptr_t)it.d_stream & 7u) == 0 && it.d_x && it.d_y && (it.dim == 2 || it.d_z) && it.out_capacity >= it.n;
}

bool compress_layout(const gpz_batch_item *items, uint32_t count, Layout &L) {
  L = Layout();
  L.count = count;
  L.look_off.resize(count);
  uint64_t off = 2ull * count * kCtlBytes;
  for (uint32_t i = 0; i < count; ++i) {
    L.look_off[i] = off;
    const int c = class_of(items[i].float_bits, items[i].dim);
    off += 8 * groups_of(items[i].n, c);
    ClassPlan &cp = L.cls[c];
    cp.items.push_back(i);
    cp.work += groups_of(items[i].n, c);
    if (items[i].flags & GPZ_FLAG_REL_ON_DEVICE) cp.rel_blocks += rel_blocks_of(items[i].n);
  }
  L.claim_off = align256(off);
  L.zero_bytes = L.claim_off + 4 * 8;
  off = align256(L.zero_bytes);
  for (int c = 0; c < 4; ++c) {
    ClassPlan &cp = L.cls[c];
    if (cp.items.empty()) continue;
    cp.table_off = off;
    off = align256(off + (c < 2 ? sizeof(BItem<float>) : sizeof(BItem<double>)) * cp.items.size());
    cp.map_off = off;
    off = align256(off + 8 * cp.work);
    cp.rmap_off = off;
    off = align256(off + 8 * cp.rel_blocks);
    switch (c) {
      case 0: cp.grid = compress_grid<float, 2>(cp.work); break;
      case 1: cp.grid = compress_grid<float, 3>(cp.work); break;
      case 2: cp.grid = compress_grid<double, 2>(cp.work); break;
      default: cp.grid = compress_grid<double, 3>(cp.work); break;
    }
    if (cp.grid < 1) return false;
  }
  L.bytes = off;
  return true;
}

bool decompress_layout(const gpz_dbatch_item *items, uint32_t count, Layout &L) {
  L = Layout();
  L.count = count;
  for (uint32_t i = 0; i < count; ++i) {
    ClassPlan &cp = L.cls[class_of(items[i].float_bits, items[i].dim)];
    cp.items.push_back(i);
    cp.work += chunks_of(items[i].n);
  }
  L.zero_bytes = (uint64_t)count * kCtlBytes;
  uint64_t off = align256(L.zero_bytes);
  for (int c = 0; c < 4; ++c) {
    ClassPlan &cp = L.cls[c];
    if (cp.items.empty()) continue;
    cp.table_off = off;
    off = align256(off + (c < 2 ? sizeof(DItem<float>) : sizeof(DItem<double>)) * cp.items.size());
    cp.map_off = off;
    off = align256(off + 8 * cp.work);
    switch (c) {
      case 0: cp.grid = dec_grid<float, 2>(cp.work); break;
      case 1: cp.grid = dec_grid<float, 3>(cp.work); break;
      case 2:
        cp.grid = dec_grid<double, 2, DecCfgF64Fast, kPassFast>(cp.work);
        cp.grid2 = dec_grid<double, 2, DecCfg<double>, kPassGeneral>(cp.work);
        break;
      default:
        cp.grid = dec_grid<double, 3, DecCfgF64Fast, kPassFast>(cp.work);
        cp.grid2 = dec_grid<double, 3, DecCfg<double>, kPassGeneral>(cp.work);
        break;
    }
    if (cp.grid < 1 || (c >= 2 && cp.grid2 < 1)) return false;
  }
  L.bytes = off;
  return true;
}

void compress_tables(const gpz_batch_item *items, const Layout &L, uint8_t *dev, uint8_t *image) {
  auto H = [&](uint64_t dev_off) { return image + (dev_off - L.zero_bytes); };
  for (int c = 0; c < 4; ++c) {
    const ClassPlan &cp = L.cls[c];
    if (cp.items.empty()) continue;
    uint64_t g = 0, rb = 0;
    unsigned long long *map = reinterpret_cast<unsigned long long *>(H(cp.map_off));
    unsigned long long *rmap = reinterpret_cast<unsigned long long *>(H(cp.rmap_off));
    for (size_t k = 0; k < cp.items.size(); ++k) {
      const uint32_t i = cp.items[k];
      const gpz_batch_item &it = items[i];
      if (c < 2) fill_item<float>(reinterpret_cast<BItem<float> *>(H(cp.table_off))[k], it, dev, ctl_off(i),
                                  ctl_off(L.count + i), L.look_off[i]);
      else fill_item<double>(reinterpret_cast<BItem<double> *>(H(cp.table_off))[k], it, dev, ctl_off(i),
                             ctl_off(L.count + i), L.look_off[i]);
      const uint64_t groups = groups_of(it.n, c);
      for (uint64_t q = 0; q < groups; ++q) map[g++] = ((unsigned long long)k << kBatchLocalBits) | q;
      if (it.flags & GPZ_FLAG_REL_ON_DEVICE) {
        const uint64_t nb = rel_blocks_of(it.n);
        for (uint64_t q = 0; q < nb; ++q) rmap[rb++] = ((unsigned long long)k << 40) | (nb << 20) | q;
      }
    }
  }
}

void decompress_tables(const gpz_dbatch_item *items, const Layout &L, uint8_t *dev, uint8_t *image) {
  auto H = [&](uint64_t dev_off) { return image + (dev_off - L.zero_bytes); };
  for (int c = 0; c < 4; ++c) {
    const ClassPlan &cp = L.cls[c];
    if (cp.items.empty()) continue;
    uint64_t q = 0;
    unsigned long long *map = reinterpret_cast<unsigned long long *>(H(cp.map_off));
    for (size_t k = 0; k < cp.items.size(); ++k) {
      const uint32_t i = cp.items[k];
      Control *ctl = reinterpret_cast<Control *>(dev + ctl_off(i));
      if (c < 2) fill_ditem<float>(reinterpret_cast<DItem<float> *>(H(cp.table_off))[k], items[i], ctl);
      else fill_ditem<double>(reinterpret_cast<DItem<double> *>(H(cp.table_off))[k], items[i], ctl);
      const uint64_t G = chunks_of(items[i].n);
      for (uint64_t ch = 0; ch < G; ++ch) map[q++] = ((unsigned long long)k << kBatchLocalBits) | ch;
    }
  }
}

void compress_enqueue(const Layout &L, uint8_t *dev, cudaStream_t st) {
  cudaMemsetAsync(dev, 0, L.zero_bytes, st);
  for (int c = 0; c < 4; ++c) {
    if (L.cls[c].items.empty()) continue;
    const uint64_t claim = L.claim_off + 8ull * c;
    switch (c) {
      case 0: enqueue_class<float, 2>(L.cls[c], dev, claim, st); break;
      case 1: enqueue_class<float, 3>(L.cls[c], dev, claim, st); break;
      case 2: enqueue_class<double, 2>(L.cls[c], dev, claim, st); break;
      default: enqueue_class<double, 3>(L.cls[c], dev, claim, st); break;
    }
  }
}

void decompress_enqueue(const Layout &L, uint8_t *dev, cudaStream_t st) {
  cudaMemsetAsync(dev, 0, L.zero_bytes, st);
  for (int c = 0; c < 4; ++c) {
    if (L.cls[c].items.empty()) continue;
    switch (c) {
      case 0: enqueue_dclass<float, 2>(L.cls[c], dev, st); break;
      case 1: enqueue_dclass<float, 3>(L.cls[c], dev, st); break;
      case 2: enqueue_dclass<double, 2>(L.cls[c], dev, st); break;
      default: enqueue_dclass<double, 3>(L.cls[c], dev, st); break;
    }
  }
}

}  // namespace gpzb_host

// ===========================================================================
// Plans: the workspace allocated once, the launches captured in a graph.
// ===========================================================================
namespace {

struct Plan {
  uint32_t count = 0;
  uint8_t *mem = nullptr;
  uint64_t bytes = 0;
  cudaGraphExec_t exec = nullptr;
  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (mem) cudaFree(mem);
  }
};

// Allocates the workspace, uploads the table image built by `tables` and
// captures `enqueue` into the plan's graph.
template <typename Tables, typename Enq>
int make_plan(Plan &p, const gpzb_host::Layout &L, Tables tables, Enq enqueue) {
  p.count = L.count;
  p.bytes = L.bytes;
  if (cudaMalloc(&p.mem, p.bytes) != cudaSuccess) {
    p.mem = nullptr;
    return GPZ_ECUDA;
  }
  std::vector<uint8_t> image(L.bytes - L.zero_bytes);
  tables(p.mem, image.data());
  if (cudaMemcpy(p.mem + L.zero_bytes, image.data(), image.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return GPZ_ECUDA;
  cudaStream_t s0 = nullptr;
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    enqueue(p.mem, s0);
    ok = cudaStreamEndCapture(s0, &graph) == cudaSuccess && graph;
  }
  if (ok) ok = cudaGraphInstantiate(&p.exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (s0) cudaStreamDestroy(s0);
  if (!ok) cudaGetLastError();
  return ok ? GPZ_OK : GPZ_ECUDA;
}

int read_controls(const uint8_t *dev, uint32_t blocks, std::vector<Control> &h, cudaStream_t st) {
  h.resize(blocks);
  for (uint32_t i = 0; i < blocks; ++i)
    if (cudaMemcpyAsync(&h[i], dev + gpzb_host::ctl_off(i), sizeof(Control), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      return GPZ_ECUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
}

}  // namespace

struct gpz_batch {
  Plan plan;
  std::vector<gpz_batch_item> items;
};

struct gpz_dbatch {
  Plan plan;
};

extern "C" {

int gpz_batch_create(const gpz_batch_item *items, uint32_t count, gpz_batch **batch, uint32_t *bad_item) {
  if (!batch || !items || count == 0) return GPZ_EINVAL;
  *batch = nullptr;
  for (uint32_t i = 0; i < count; ++i)
    if (!gpzb_host::compress_item_ok(items[i])) {
      if (bad_item) *bad_item = i;
      return GPZ_EINVAL;
    }
  gpzb_host::Layout L;
  if (!gpzb_host::compress_layout(items, count, L)) return GPZ_ECUDA;
  gpz_batch *b = new (std::nothrow) gpz_batch;
  if (!b) return GPZ_ECUDA;
  b->items.assign(items, items + count);
  const int rc = make_plan(
      b->plan, L, [&](uint8_t *dev, uint8_t *image) { gpzb_host::compress_tables(items, L, dev, image); },
      [&](uint8_t *dev, cudaStream_t s) { gpzb_host::compress_enqueue(L, dev, s); });
  if (rc != GPZ_OK) {
    delete b;
    return rc;
  }
  *batch = b;
  return GPZ_OK;
}

int gpz_batch_launch(gpz_batch *b, void *stream) {
  if (!b || !b->plan.exec) return GPZ_EINVAL;
  return cudaGraphLaunch(b->plan.exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
}

int gpz_batch_results(gpz_batch *b, gpz_result *results, double *h_eb, void *stream) {
  if (!b || !results) return GPZ_EINVAL;
  const uint32_t n = b->plan.count;
  std::vector<Control> h;
  const int rc = read_controls(b->plan.mem, 2 * n, h, static_cast<cudaStream_t>(stream));
  if (rc != GPZ_OK) return rc;
  for (uint32_t i = 0; i < n; ++i) {
    const Control &c = h[i];
    results[i].stream_bytes = c.stream_bytes;
    results[i].seg_size = c.seg;
    results[i].adjusted = c.adjusted;
    results[i].status = c.status;
    results[i].id_overflow = c.id_overflow;
    if (h_eb) {
      const gpz_batch_item &it = b->items[i];
      if (it.flags & GPZ_FLAG_REL_ON_DEVICE) h_eb[i] = h[n + i].out_eb;
      else h_eb[i] = it.float_bits == 32 ? (double)(float)it.eb : it.eb;
    }
  }
  return GPZ_OK;
}

uint64_t gpz_batch_device_bytes(const gpz_batch *b) { return b ? b->plan.bytes : 0; }

int gpz_batch_destroy(gpz_batch *b) {
  if (!b) return GPZ_EINVAL;
  delete b;
  return GPZ_OK;
}

int gpz_dbatch_create(const gpz_dbatch_item *items, uint32_t count, gpz_dbatch **batch, uint32_t *bad_item) {
  if (!batch || !items || count == 0) return GPZ_EINVAL;
  *batch = nullptr;
  for (uint32_t i = 0; i < count; ++i)
    if (!gpzb_host::decompress_item_ok(items[i])) {
      if (bad_item) *bad_item = i;
      return GPZ_EINVAL;
    }
  gpzb_host::Layout L;
  if (!gpzb_host::decompress_layout(items, count, L)) return GPZ_ECUDA;
  gpz_dbatch *b = new (std::nothrow) gpz_dbatch;
  if (!b) return GPZ_ECUDA;
  const int rc = make_plan(
      b->plan, L, [&](uint8_t *dev, uint8_t *image) { gpzb_host::decompress_tables(items, L, dev, image); },
      [&](uint8_t *dev, cudaStream_t s) { gpzb_host::decompress_enqueue(L, dev, s); });
  if (rc != GPZ_OK) {
    delete b;
    return rc;
  }
  *batch = b;
  return GPZ_OK;
}

int gpz_dbatch_launch(gpz_dbatch *b, void *stream) {
  if (!b || !b->plan.exec) return GPZ_EINVAL;
  return cudaGraphLaunch(b->plan.exec, static_cast<cudaStream_t>(stream)) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
}

int gpz_dbatch_results(gpz_dbatch *b, gpz_result *results, void *stream) {
  if (!b || !results) return GPZ_EINVAL;
  std::vector<Control> h;
  const int rc = read_controls(b->plan.mem, b->plan.count, h, static_cast<cudaStream_t>(stream));
  if (rc != GPZ_OK) return rc;
  for (uint32_t i = 0; i < b->plan.count; ++i) {
    memset(&results[i], 0, sizeof(gpz_result));
    results[i].status = h[i].status;
  }
  return GPZ_OK;
}

int gpz_dbatch_destroy(gpz_dbatch *b) {
  if (!b) return GPZ_EINVAL;
  delete b;
  return GPZ_OK;
}

}  // extern "C"
