// gpz_serve.cu -- the request server of include/gpz_b200.h (gpz_server_*):
// admission by device-memory budget, continuous batching over several CUDA
// streams, completion tracking.
//
// One worker thread owns the GPU side.  Each pass it
//   1. retires finished batches (their completion event has fired; the
//      control blocks were copied to pinned memory by the same stream),
//   2. fills every idle stream with a new batch: queued requests in arrival
//      order, each admitted only once its output fits in the arena (the head
//      of the queue waits for memory rather than being overtaken),
//   3. sleeps until a submit or, while batches run, for a short poll interval.
// A batch is the batched compress / decompress of gpz_batchapi.cu launched
// directly (no graph): the descriptor image is built in the stream's pinned
// buffer and copied into the stream's workspace in the arena.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "gpz_b200.h"
#include "gpz_batch_host.h"
#include "gpz_device.cuh"

using gpzb::Control;
using gpzb::kCtlBytes;

namespace {

using Clock = std::chrono::steady_clock;
constexpr uint64_t kAlign = 256;
inline uint64_t up(uint64_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

// First-fit allocator over one device allocation (offsets, 256-byte aligned).
class Arena {
 public:
  uint8_t *base = nullptr;
  uint64_t size = 0;

  bool init(uint64_t bytes) {
    size = bytes & ~(kAlign - 1);
    if (cudaMalloc(&base, size) != cudaSuccess) {
      base = nullptr;
      return false;
    }
    free_[0] = size;
    return true;
  }
  void destroy() {
    if (base) cudaFree(base);
    base = nullptr;
  }
  // offset, or -1 when no free range is large enough
  int64_t alloc(uint64_t bytes) {
    bytes = up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const uint64_t off = it->first, rest = it->second - bytes;
      free_.erase(it);
      if (rest) free_[off + bytes] = rest;
      return (int64_t)off;
    }
    return -1;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = up(bytes);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  uint64_t free_bytes() const {
    uint64_t s = 0;
    for (const auto &kv : free_) s += kv.second;
    return s;
  }

 private:
  std::map<uint64_t, uint64_t> free_;
};

struct Req {
  gpz_request r{};
  int64_t out_off = -1;
  uint64_t out_bytes = 0;
  Clock::time_point t_submit, t_launch;
  bool done = false;
  gpz_completion c{};
};

struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  uint64_t ws_off = 0;
  uint8_t *image = nullptr;   // pinned: descriptor images
  uint8_t *ctl_h = nullptr;   // pinned: control blocks copied back
  bool busy = false;
  std::vector<uint64_t> comp, dec;  // tickets of the batch, compress and decompress
};

// Decompress outputs: x, y, z, each starting at a multiple of 256 bytes.
uint64_t axis_stride(const gpz_request &r) { return up(r.n * (r.float_bits / 8)); }

uint64_t out_bytes_of(const gpz_request &r) {
  if (r.op == GPZ_OP_COMPRESS) return gpz_stream_bound(r.n, r.dim, r.float_bits);
  return (uint64_t)r.dim * axis_stride(r);
}

gpz_batch_item compress_item(const gpz_request &r, void *d_out, uint64_t cap) {
  gpz_batch_item it;
  memset(&it, 0, sizeof(it));
  it.float_bits = r.float_bits;
  it.dim = r.dim;
  it.n = r.n;
  it.d_x = r.d_x;
  it.d_y = r.d_y;
  it.d_z = r.d_z;
  it.d_out = d_out;
  it.out_capacity = cap;
  it.eb = r.eb;
  it.rel_eb = r.rel_eb;
  it.rel_mode = r.rel_mode;
  it.seg_size = r.seg_size;
  it.flags = r.flags;
  return it;
}

gpz_dbatch_item decompress_item(const gpz_request &r, uint8_t *d_out) {
  gpz_dbatch_item it;
  memset(&it, 0, sizeof(it));
  const uint64_t axis = axis_stride(r);
  it.d_stream = r.d_stream;
  it.stream_bytes = r.stream_bytes;
  it.float_bits = r.float_bits;
  it.dim = r.dim;
  it.n = r.n;
  it.d_x = d_out;
  it.d_y = d_out ? d_out + axis : nullptr;
  it.d_z = d_out && r.dim == 3 ? d_out + 2 * axis : nullptr;
  it.out_capacity = r.n;
  return it;
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct gpz_server {
  gpz_server_config cfg{};
  int device = 0;
  Arena arena;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, Req> reqs;
  uint64_t next_ticket = 1, submitted = 0, completed = 0, batches = 0;
  uint64_t gen = 0;  // bumped by submit, release and stop: the worker's wake-up reasons
  cudaEvent_t last = nullptr;  // completion event of the most recently launched batch
  bool stop = false;
  std::thread worker;

  // ---- worker side (called with mu held) ----
  void retire(Slot &s) {
    const cudaError_t q = cudaEventQuery(s.done);
    if (q == cudaErrorNotReady) return;
    const Clock::time_point now = Clock::now();
    const uint32_t nc = (uint32_t)s.comp.size();
    for (uint32_t i = 0; i < nc; ++i) {
      Req &q2 = reqs[s.comp[i]];
      const Control &c = *reinterpret_cast<const Control *>(s.ctl_h + gpzb_host::ctl_off(i));
      const Control &rc = *reinterpret_cast<const Control *>(s.ctl_h + gpzb_host::ctl_off(nc + i));
      q2.c.status = q == cudaSuccess ? c.status : GPZ_ECUDA;
      q2.c.seg_size = c.seg;
      q2.c.stream_bytes = c.stream_bytes;
      q2.c.eb = (q2.r.flags & GPZ_FLAG_REL_ON_DEVICE) ? rc.out_eb
                                                      : (q2.r.float_bits == 32 ? (double)(float)q2.r.eb : q2.r.eb);
    }
    const uint8_t *dctl = s.ctl_h + gpzb_host::ctl_off(2 * nc);
    for (uint32_t i = 0; i < s.dec.size(); ++i) {
      Req &q2 = reqs[s.dec[i]];
      const Control &c = *reinterpret_cast<const Control *>(dctl + gpzb_host::ctl_off(i));
      q2.c.status = q == cudaSuccess ? c.status : GPZ_ECUDA;
    }
    for (const auto *v : {&s.comp, &s.dec})
      for (uint64_t t : *v) {
        Req &q2 = reqs[t];
        q2.c.queue_ms = ms_between(q2.t_submit, q2.t_launch);
        q2.c.total_ms = ms_between(q2.t_submit, now);
        q2.c.batch_size = (uint32_t)(s.comp.size() + s.dec.size());
        q2.done = true;
        ++completed;
      }
    if (q != cudaSuccess) cudaGetLastError();
    s.comp.clear();
    s.dec.clear();
    s.busy = false;
    cv_done.notify_all();
  }

  // Takes queued requests for slot s while their outputs fit; returns false
  // when nothing could be started.
  bool launch(Slot &s) {
    std::vector<uint64_t> chosen;
    while (!pending.empty() && chosen.size() < cfg.max_batch) {
      Req &q = reqs[pending.front()];
      if (q.out_off < 0) {
        q.out_off = arena.alloc(q.out_bytes);
        if (q.out_off < 0) break;  // the head waits for memory
      }
      chosen.push_back(pending.front());
      pending.pop_front();
    }
    if (chosen.empty()) return false;
    // descriptors; drop requests from the tail until the workspace holds them
    std::vector<gpz_batch_item> ci;
    std::vector<gpz_dbatch_item> di;
    gpzb_host::Layout Lc, Ld;
    for (;;) {
      ci.clear();
      di.clear();
      s.comp.clear();
      s.dec.clear();
      for (uint64_t t : chosen) {
        Req &q = reqs[t];
        uint8_t *out = arena.base + q.out_off;
        if (q.r.op == GPZ_OP_COMPRESS) {
          ci.push_back(compress_item(q.r, out, q.out_bytes));
          s.comp.push_back(t);
        } else {
          di.push_back(decompress_item(q.r, out));
          s.dec.push_back(t);
        }
      }
      bool ok = true;
      if (!ci.empty()) ok &= gpzb_host::compress_layout(ci.data(), (uint32_t)ci.size(), Lc);
      if (!di.empty()) ok &= gpzb_host::decompress_layout(di.data(), (uint32_t)di.size(), Ld);
      const uint64_t need = (ci.empty() ? 0 : up(Lc.bytes)) + (di.empty() ? 0 : Ld.bytes);
      if (ok && need <= cfg.workspace_bytes) break;
      if (!ok || chosen.size() == 1) {  // cannot run: fail it
        Req &q = reqs[chosen.back()];
        q.c.status = ok ? GPZ_ENOSPACE : GPZ_ECUDA;
        q.t_launch = Clock::now();
        q.c.total_ms = ms_between(q.t_submit, q.t_launch);
        q.done = true;
        ++completed;
        cv_done.notify_all();
      } else {
        pending.push_front(chosen.back());
      }
      chosen.pop_back();
      if (chosen.empty()) {
        s.comp.clear();
        s.dec.clear();
        return false;
      }
    }
    // without GPZ_SERVER_OVERLAP the GPU runs batches in launch order; with
    // it, batches on different slots run at once, each persistent grid sized
    // to its slot's share of the SMs, so concurrent batches split the GPU
    // instead of competing for residency with full-occupancy grids
    if (!(cfg.flags & GPZ_SERVER_OVERLAP) && last) cudaStreamWaitEvent(s.st, last, 0);
    if ((cfg.flags & GPZ_SERVER_OVERLAP) && cfg.streams > 1) {
      for (int c = 0; c < 4; ++c) {
        if (!ci.empty() && Lc.cls[c].grid > 0)
          Lc.cls[c].grid = std::max(1, (int)((Lc.cls[c].grid + cfg.streams - 1) / cfg.streams));
        if (!di.empty() && Ld.cls[c].grid > 0)
          Ld.cls[c].grid = std::max(1, (int)((Ld.cls[c].grid + cfg.streams - 1) / cfg.streams));
        if (!di.empty() && Ld.cls[c].grid2 > 0)
          Ld.cls[c].grid2 = std::max(1, (int)((Ld.cls[c].grid2 + cfg.streams - 1) / cfg.streams));
      }
    }
    uint8_t *ws = arena.base + s.ws_off;
    uint8_t *wsd = ws + (ci.empty() ? 0 : up(Lc.bytes));
    uint8_t *img = s.image;
    const Clock::time_point now = Clock::now();
    for (uint64_t t : chosen) reqs[t].t_launch = now;
    // every enqueue is checked: a batch whose upload, launch or status
    // read-back could not be queued is failed as a whole (GPZ_ECUDA) instead
    // of being retired later with stale status bytes
    bool queued = true;
    auto ck = [&](cudaError_t e) { queued &= e == cudaSuccess; };
    if (!ci.empty()) {
      gpzb_host::compress_tables(ci.data(), Lc, ws, img);
      ck(cudaMemcpyAsync(ws + Lc.zero_bytes, img, Lc.bytes - Lc.zero_bytes, cudaMemcpyHostToDevice, s.st));
      if (queued) gpzb_host::compress_enqueue(Lc, ws, s.st);
      ck(cudaGetLastError());
      img += up(Lc.bytes - Lc.zero_bytes);
    }
    if (queued && !di.empty()) {
      gpzb_host::decompress_tables(di.data(), Ld, wsd, img);
      ck(cudaMemcpyAsync(wsd + Ld.zero_bytes, img, Ld.bytes - Ld.zero_bytes, cudaMemcpyHostToDevice, s.st));
      if (queued) gpzb_host::decompress_enqueue(Ld, wsd, s.st);
      ck(cudaGetLastError());
    }
    const uint64_t nc = ci.size();
    if (queued && nc) ck(cudaMemcpyAsync(s.ctl_h, ws, 2 * nc * kCtlBytes, cudaMemcpyDeviceToHost, s.st));
    if (queued && !di.empty())
      ck(cudaMemcpyAsync(s.ctl_h + 2 * nc * kCtlBytes, wsd, di.size() * kCtlBytes, cudaMemcpyDeviceToHost, s.st));
    if (queued) ck(cudaEventRecord(s.done, s.st));
    if (!queued) {
      // wait out whatever part of the batch did get queued (its kernels use
      // the slot's workspace), then complete its requests with the error
      cudaStreamSynchronize(s.st);
      cudaGetLastError();
      const Clock::time_point t_end = Clock::now();
      for (uint64_t t : chosen) {
        Req &q = reqs[t];
        q.c.status = GPZ_ECUDA;
        q.c.queue_ms = ms_between(q.t_submit, q.t_launch);
        q.c.total_ms = ms_between(q.t_submit, t_end);
        q.c.batch_size = (uint32_t)chosen.size();
        q.done = true;
        ++completed;
      }
      s.comp.clear();
      s.dec.clear();
      cv_done.notify_all();
      return true;
    }
    last = s.done;
    s.busy = true;
    ++batches;
    return true;
  }

  void run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      const uint64_t seen = gen;
      bool any_busy = false;
      for (Slot &s : slots)
        if (s.busy) retire(s);
      for (Slot &s : slots) {
        if (!s.busy && !pending.empty()) launch(s);
        any_busy |= s.busy;
      }
      if (stop && pending.empty() && !any_busy) break;
      // batches in flight: poll their events; idle: sleep until a submit,
      // a release (the queue head may fit now) or stop
      if (any_busy) cv_work.wait_for(lk, std::chrono::microseconds(20));
      else cv_work.wait(lk, [&] { return gen != seen; });
    }
  }
};

extern "C" {

int gpz_server_create(const gpz_server_config *cfg, gpz_server **server) {
  if (!cfg || !server || cfg->streams == 0 || cfg->max_batch == 0 || cfg->hbm_budget == 0 ||
      (cfg->flags & ~GPZ_SERVER_OVERLAP) != 0)
    return GPZ_EINVAL;
  *server = nullptr;
  gpz_server *s = new (std::nothrow) gpz_server;
  if (!s) return GPZ_ECUDA;
  s->cfg = *cfg;
  if (s->cfg.workspace_bytes == 0) s->cfg.workspace_bytes = 64ull << 20;
  s->cfg.workspace_bytes = up(s->cfg.workspace_bytes);
  if (s->cfg.workspace_bytes * s->cfg.streams >= cfg->hbm_budget) {
    delete s;
    return GPZ_EINVAL;
  }
  cudaGetDevice(&s->device);
  if (!s->arena.init(cfg->hbm_budget)) {
    delete s;
    return GPZ_ECUDA;
  }
  s->slots.resize(s->cfg.streams);
  bool ok = true;
  for (Slot &sl : s->slots) {
    const int64_t off = s->arena.alloc(s->cfg.workspace_bytes);
    ok &= off >= 0;
    sl.ws_off = (uint64_t)std::max<int64_t>(off, 0);
    ok &= cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) == cudaSuccess;
    ok &= cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess;
    ok &= cudaHostAlloc(reinterpret_cast<void **>(&sl.image), s->cfg.workspace_bytes, cudaHostAllocDefault) ==
          cudaSuccess;
    ok &= cudaHostAlloc(reinterpret_cast<void **>(&sl.ctl_h), 3ull * s->cfg.max_batch * kCtlBytes,
                        cudaHostAllocDefault) == cudaSuccess;
  }
  if (!ok) {
    gpz_server_destroy(s);
    return GPZ_ECUDA;
  }
  s->worker = std::thread([s] { s->run(); });
  *server = s;
  return GPZ_OK;
}

int gpz_server_submit(gpz_server *s, const gpz_request *req, uint64_t *ticket) {
  if (!s || !req || !ticket) return GPZ_EINVAL;
  const gpz_request &r = *req;
  bool ok;
  if (r.op == GPZ_OP_COMPRESS) {
    const gpz_batch_item it = compress_item(r, reinterpret_cast<void *>(kAlign), out_bytes_of(r));
    ok = r.n >= 1 && gpzb_host::compress_item_ok(it);
  } else if (r.op == GPZ_OP_DECOMPRESS) {
    const gpz_dbatch_item it = decompress_item(r, reinterpret_cast<uint8_t *>(kAlign));
    ok = gpzb_host::decompress_item_ok(it);
  } else {
    ok = false;
  }
  if (!ok) return GPZ_EINVAL;
  const uint64_t bytes = out_bytes_of(r);
  if (up(bytes) > s->arena.size - s->cfg.workspace_bytes * s->cfg.streams) return GPZ_ENOSPACE;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t t = s->next_ticket++;
    Req &q = s->reqs[t];
    q.r = r;
    q.out_bytes = bytes;
    q.t_submit = Clock::now();
    s->pending.push_back(t);
    ++s->submitted;
    ++s->gen;
    *ticket = t;
  }
  s->cv_work.notify_one();
  return GPZ_OK;
}

int gpz_server_wait(gpz_server *s, uint64_t ticket, gpz_completion *out, uint32_t timeout_ms) {
  if (!s) return GPZ_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return GPZ_EINVAL;
  auto ready = [&] { return s->reqs[ticket].done; };
  if (timeout_ms == 0) s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return GPZ_ETIMEOUT;
  Req &q = s->reqs[ticket];
  q.c.d_out = q.out_off >= 0 ? s->arena.base + q.out_off : nullptr;
  if (out) *out = q.c;
  return GPZ_OK;
}

int gpz_server_release(gpz_server *s, uint64_t ticket) {
  if (!s) return GPZ_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || !it->second.done) return GPZ_EINVAL;
    if (it->second.out_off >= 0) s->arena.release((uint64_t)it->second.out_off, it->second.out_bytes);
    s->reqs.erase(it);
    ++s->gen;
  }
  s->cv_work.notify_one();  // memory freed: the head of the queue may fit now
  return GPZ_OK;
}

int gpz_server_stats_get(gpz_server *s, gpz_server_stats *st) {
  if (!s || !st) return GPZ_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->batches = s->batches;
  st->arena_bytes = s->arena.size;
  st->arena_free_bytes = s->arena.free_bytes();
  st->queued = (uint32_t)s->pending.size();
  for (const Slot &sl : s->slots) st->in_flight += sl.busy ? 1u : 0u;
  return GPZ_OK;
}

int gpz_server_destroy(gpz_server *s) {
  if (!s) return GPZ_EINVAL;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
      ++s->gen;
    }
    s->cv_work.notify_all();
    s->worker.join();
  }
  for (Slot &sl : s->slots) {
    if (sl.st) cudaStreamSynchronize(sl.st);
    if (sl.st) cudaStreamDestroy(sl.st);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.image) cudaFreeHost(sl.image);
    if (sl.ctl_h) cudaFreeHost(sl.ctl_h);
  }
  s->arena.destroy();
  delete s;
  return GPZ_OK;
}

}  // extern "C"
