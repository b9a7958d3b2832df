// gpz_capi.cu -- C ABI of the B200 GPZ codec (declared in include/gpz_b200.h).
//
// Host orchestration replacing CudaWarpCompress::compressImpl /
// decompressImpl (reference src/cudaWarpCompress.cu:1573-1856 and the double
// twin): no allocation, no host synchronisation and no small memcpys inside
// the call -- one memset of the scratch control block, the sampling kernel
// that resolves the segment size on the device, and one persistent
// compress kernel that writes the finished stream.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <nvtx3/nvToolsExt.h>

#include "gpz_b200.h"
#include "gpz_launch.h"
#include "gpz_kernels.cuh"
#include "gpz_encode.cuh"
#include "gpz_decode.cuh"

using namespace gpzb;

namespace {

int num_sms() { return current_sms(); }

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? GPZ_OK : GPZ_ECUDA; }

// NVTX range for the duration of a scope, with the names the reference's
// codec pushes (src/cudaWarpCompress.cu:1577, 1626, 1747, 1817), so profiler
// timelines of either codec line up.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

inline uint64_t chunks(uint64_t n) { return (n + kChunk - 1) / kChunk; }

// Control-block head (the gpz_result fields) into device-addressable pinned
// host memory, one word per lane.
__global__ void result_post_kernel(const gpz_result *src, gpz_result *dst) {
  constexpr int W = (int)(sizeof(gpz_result) / 4);
  static_assert(sizeof(gpz_result) % 4 == 0, "word copy");
  if ((int)threadIdx.x < W)
    reinterpret_cast<volatile uint32_t *>(dst)[threadIdx.x] = reinterpret_cast<const volatile uint32_t *>(src)[threadIdx.x];
}

template <typename T>
int compress_t(const gpz_params *p, const void *d_x, const void *d_y, const void *d_z, void *d_out,
               uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes, cudaStream_t st) {
  using Tr = TT<T>;
  NvtxRange range("compress");
  const uint64_t G = chunks(p->n);
  if (out_capacity < Tr::hdr + G * (8ull + Tr::meta)) return GPZ_ENOSPACE;
  if (scratch_bytes < gpz_compress_scratch_bytes(p->n)) return GPZ_ENOSPACE;
  Control *ctl = static_cast<Control *>(d_scratch);
  unsigned long long *look = reinterpret_cast<unsigned long long *>(static_cast<uint8_t *>(d_scratch) + kCtlBytes);
  cudaError_t e = cudaMemsetAsync(d_scratch, 0, kCtlBytes + 8ull * G, st);
  if (e != cudaSuccess) return GPZ_ECUDA;
  const T eb = (T)p->eb;
  const T rel = (T)p->rel_eb;
  const T *x = static_cast<const T *>(d_x), *y = static_cast<const T *>(d_y), *z = static_cast<const T *>(d_z);
  // strict-bound mode: the bound actually encoded is shrunk on the device by
  // the reconstruction's worst rounding over the snapshot's magnitude range
  const bool strict = (p->flags & GPZ_FLAG_STRICT_BOUND) != 0;
  const double *eb_dev = strict ? &ctl->strict_eb : nullptr;
  if (strict)
    strict_bound_kernel<T><<<num_sms() * 4, 256, 0, st>>>(x, y, p->dim == 3 ? z : y, p->n, p->dim, eb, ctl);
  if (p->flags & GPZ_FLAG_SEG_FIXED) {
    if (p->seg_size == 0) return GPZ_EINVAL;
    set_seg_kernel<<<1, 1, 0, st>>>(ctl, p->seg_size);
  } else {
    const int safe31 = (p->flags & (GPZ_FLAG_SAFE31 | GPZ_FLAG_STRICT_BOUND)) ? 1 : 0;
    seg_sample_kernel<T><<<128, 256, 0, st>>>(x, y, p->dim == 3 ? z : y, p->n, p->dim, p->seg_size, p->rel_mode, rel,
                                              eb, safe31, ctl, eb_dev);
  }
  CArgs<T> a;
  a.x = x; a.y = y; a.z = p->dim == 3 ? z : y;
  a.out = static_cast<uint8_t *>(d_out);
  a.out_cap = out_capacity;
  a.ctl = ctl;
  a.look = look;
  a.n = p->n;
  a.G = G;
  a.eb = eb;
  a.eb_dev = eb_dev;
  a.dim = p->dim;
  a.vec_ok = aligned16(d_x) && aligned16(d_y) && (p->dim == 2 || aligned16(d_z));
  // persistent grid: one CTA per W chunks in flight (W = enc_warps<T, DIM>)
  NvtxRange krange("run compress kernel");
  auto launch = [&](auto kernel, auto w) -> bool {
    constexpr int W = decltype(w)::value;
    constexpr size_t smem = enc_smem_bytes<W>();
    const int occ = resident_ctas(kernel, 32 * W, smem);
    if (occ == 0) return false;
    const uint64_t grid = std::min<uint64_t>((G + W - 1) / W, (uint64_t)num_sms() * occ);
    kernel<<<(unsigned)grid, 32 * W, smem, st>>>(a);
    return true;
  };
  using W3 = std::integral_constant<int, enc_warps<T, 3>()>;
  using W2 = std::integral_constant<int, enc_warps<T, 2>()>;
  if (!(p->dim == 3 ? launch(compress_kernel<T, 3>, W3{}) : launch(compress_kernel<T, 2>, W2{}))) return GPZ_ECUDA;
  return cuda_status(cudaGetLastError());
}

template <typename T>
int decompress_t(const void *d_stream, uint64_t stream_bytes, uint32_t dim, void *d_x, void *d_y, void *d_z,
                 uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes, cudaStream_t st) {
  NvtxRange range("decompress");
  if (scratch_bytes < gpz_decompress_scratch_bytes()) return GPZ_ENOSPACE;
  if (((uintptr_t)d_stream & 7u) != 0) return GPZ_EINVAL;
  Control *ctl = static_cast<Control *>(d_scratch);
  cudaError_t e = cudaMemsetAsync(d_scratch, 0, kCtlBytes, st);
  if (e != cudaSuccess) return GPZ_ECUDA;
  DArgs<T> a;
  a.s = static_cast<const uint8_t *>(d_stream);
  a.bytes = stream_bytes;
  a.x = static_cast<T *>(d_x);
  a.y = static_cast<T *>(d_y);
  a.z = dim == 3 ? static_cast<T *>(d_z) : static_cast<T *>(d_y);
  a.cap = out_capacity;
  a.ctl = ctl;
  a.vec_ok = aligned16(d_x) && aligned16(d_y) && (dim == 2 || aligned16(d_z));
  // The chunk count lives in the device header: one warp per chunk in a grid
  // of at most one full wave, each warp striding over the chunks.
  NvtxRange krange("run decompress kernel");
  auto launch = [&](auto kernel, auto cfg) -> bool {
    using Cfg = decltype(cfg);
    constexpr int W = Cfg::warps;
    constexpr size_t smem = dec_smem_bytes_of<Cfg>();
    const uint64_t bound_ctas = (stream_bytes / (8ull + TT<T>::meta) + W) / W;
    const int occ = resident_ctas(kernel, 32 * W, smem);
    if (occ == 0) return false;
    const uint64_t grid = std::min<uint64_t>((uint64_t)num_sms() * occ, bound_ctas);
    kernel<<<(unsigned)grid, 32 * W, smem, st>>>(a);
    return true;
  };
  if constexpr (sizeof(T) == 4) {
    if (!(dim == 3 ? launch(decompress_kernel<T, 3>, DecCfg<T>{}) : launch(decompress_kernel<T, 2>, DecCfg<T>{})))
      return GPZ_ECUDA;
  } else {
    // fast pass in the 12 KB layout, then the general pass for the chunks it
    // left (it returns at once when there are none)
    bool ok = dim == 3 ? launch(decompress_kernel<T, 3, DecCfgF64Fast, kPassFast>, DecCfgF64Fast{})
                       : launch(decompress_kernel<T, 2, DecCfgF64Fast, kPassFast>, DecCfgF64Fast{});
    ok = ok && (dim == 3 ? launch(decompress_kernel<T, 3, DecCfg<T>, kPassGeneral>, DecCfg<T>{})
                         : launch(decompress_kernel<T, 2, DecCfg<T>, kPassGeneral>, DecCfg<T>{}));
    if (!ok) return GPZ_ECUDA;
  }
  return cuda_status(cudaGetLastError());
}

}  // namespace

// AoS <-> SoA for the file path (reference host loops load_file_to_soa_xyz /
// write_xyz_to_aos_file, include/utils.cuh:83-180).
template <typename T, int DIM>
__global__ void __launch_bounds__(256) aos_to_soa_kernel(const T *__restrict__ aos, T *__restrict__ x,
                                                         T *__restrict__ y, T *__restrict__ z, uint64_t n) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
    const T *p = aos + DIM * i;
    x[i] = p[0];
    y[i] = p[1];
    z[i] = DIM == 3 ? p[2] : (T)0;
  }
}
template <typename T, int DIM>
__global__ void __launch_bounds__(256) soa_to_aos_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                         const T *__restrict__ z, T *__restrict__ aos, uint64_t n) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
    T *p = aos + DIM * i;
    p[0] = x[i];
    p[1] = y[i];
    if (DIM == 3) p[2] = z[i];
  }
}

template <typename T>
int aos_soa(bool to_soa, uint32_t dim, uint64_t n, const void *aos, const void *x, const void *y, const void *z,
            cudaStream_t st) {
  if (n == 0) return GPZ_OK;
  const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)num_sms() * 8);
  T *X = (T *)x, *Y = (T *)y, *Z = (T *)z, *A = (T *)aos;
  if (to_soa) {
    if (dim == 3) aos_to_soa_kernel<T, 3><<<grid, 256, 0, st>>>(A, X, Y, Z, n);
    else aos_to_soa_kernel<T, 2><<<grid, 256, 0, st>>>(A, X, Y, Z, n);
  } else {
    if (dim == 3) soa_to_aos_kernel<T, 3><<<grid, 256, 0, st>>>(X, Y, Z, A, n);
    else soa_to_aos_kernel<T, 2><<<grid, 256, 0, st>>>(X, Y, Z, A, n);
  }
  return cuda_status(cudaGetLastError());
}

extern "C" {

const char *gpz_version(void) { return "gpz_b200 0.1 (sm_100a)"; }

uint64_t gpz_stream_bound(uint64_t n, uint32_t dim, uint32_t float_bits) {
  (void)dim;
  const uint64_t G = chunks(n);
  const uint64_t hdr = float_bits == 64 ? 32 : 24, meta = float_bits == 64 ? 64 : 36;
  return hdr + G * (8 + meta + 31 * 128 + 11 * 128 + 31 * 128 + 16);
}

uint64_t gpz_compress_scratch_bytes(uint64_t n) { return (uint64_t)kCtlBytes + 8ull * chunks(n); }

uint64_t gpz_decompress_scratch_bytes(void) { return (uint64_t)kCtlBytes; }

int gpz_compress_async(const gpz_params *p, const void *d_x, const void *d_y, const void *d_z, void *d_out,
                       uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes, void *stream) {
  if (!p || !d_x || !d_y || !d_out || !d_scratch) return GPZ_EINVAL;
  if (p->dim != 2 && p->dim != 3) return GPZ_EINVAL;
  if (p->dim == 3 && !d_z) return GPZ_EINVAL;
  if (p->float_bits != 32 && p->float_bits != 64) return GPZ_EINVAL;
  if (p->n == 0 || chunks(p->n) >= (1ull << 31)) return GPZ_EINVAL;
  // abs mode without a segment size: the reference shifts by __ffs(0)-1 (UB)
  if (p->seg_size == 0 && !p->rel_mode) return GPZ_EINVAL;
  if (((uintptr_t)d_out & 7u) != 0 || ((uintptr_t)d_scratch & 15u) != 0) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->float_bits == 32 ? compress_t<float>(p, d_x, d_y, d_z, d_out, out_capacity, d_scratch, scratch_bytes, st)
                             : compress_t<double>(p, d_x, d_y, d_z, d_out, out_capacity, d_scratch, scratch_bytes, st);
}

int gpz_result_get(const void *d_scratch, gpz_result *result, void *stream) {
  if (!d_scratch) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  gpz_result r;
  memset(&r, 0, sizeof(r));
  cudaError_t e = cudaMemcpyAsync(&r, d_scratch, sizeof(gpz_result), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return GPZ_ECUDA;
  if (result) *result = r;
  return r.status;
}

int gpz_result_post(const void *d_scratch, gpz_result *h_result, void *stream) {
  if (!d_scratch || !h_result) return GPZ_EINVAL;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, h_result) != cudaSuccess) {
    cudaGetLastError();  // clear the (non-sticky) error the query leaves behind
    return GPZ_EINVAL;
  }
  if (at.type != cudaMemoryTypeHost || at.devicePointer == nullptr) return GPZ_EINVAL;
  result_post_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const gpz_result *>(d_scratch), static_cast<gpz_result *>(at.devicePointer));
  return cuda_status(cudaGetLastError());
}

int gpz_compress(const gpz_params *p, const void *d_x, const void *d_y, const void *d_z, void *d_out,
                 uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes, gpz_result *result, void *stream) {
  int rc = gpz_compress_async(p, d_x, d_y, d_z, d_out, out_capacity, d_scratch, scratch_bytes, stream);
  if (rc) return rc;
  return gpz_result_get(d_scratch, result, stream);
}

int gpz_decompress_async(const void *d_stream, uint64_t stream_bytes, uint32_t float_bits, uint32_t dim, void *d_x,
                         void *d_y, void *d_z, uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes,
                         void *stream) {
  if (!d_stream || !d_x || !d_y || !d_scratch) return GPZ_EINVAL;
  if (float_bits != 32 && float_bits != 64) return GPZ_EINVAL;
  if (dim != 2 && dim != 3) return GPZ_EINVAL;
  if (dim == 3 && !d_z) return GPZ_EINVAL;
  if (((uintptr_t)d_scratch & 15u) != 0) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return float_bits == 32
             ? decompress_t<float>(d_stream, stream_bytes, dim, d_x, d_y, d_z, out_capacity, d_scratch, scratch_bytes,
                                   st)
             : decompress_t<double>(d_stream, stream_bytes, dim, d_x, d_y, d_z, out_capacity, d_scratch,
                                    scratch_bytes, st);
}

int gpz_decompress(const void *d_stream, uint64_t stream_bytes, uint32_t float_bits, uint32_t dim, void *d_x,
                   void *d_y, void *d_z, uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes,
                   gpz_result *result, void *stream) {
  int rc = gpz_decompress_async(d_stream, stream_bytes, float_bits, dim, d_x, d_y, d_z, out_capacity, d_scratch,
                                scratch_bytes, stream);
  if (rc) return rc;
  return gpz_result_get(d_scratch, result, stream);
}

int gpz_parse_header(const void *h_stream, uint64_t bytes, uint32_t *dim, uint64_t *n, uint32_t *float_bits,
                     double *eb, uint32_t *seg_size) {
  // CompressorManager::decompressLoadParas (src/CompressorManager.cpp:24-34):
  // dim @0, N @4, float_bits @12; eb @16; seg @20 (f32) / @24 (f64).
  if (!h_stream || bytes < 24) return GPZ_ESTREAM;
  const uint8_t *s = static_cast<const uint8_t *>(h_stream);
  uint32_t d, b, sg;
  uint64_t nn;
  memcpy(&d, s, 4);
  memcpy(&nn, s + 4, 8);
  memcpy(&b, s + 12, 4);
  double e;
  if (b == 32) {
    float f;
    memcpy(&f, s + 16, 4);
    e = f;
    memcpy(&sg, s + 20, 4);
  } else if (b == 64) {
    if (bytes < 32) return GPZ_ESTREAM;
    memcpy(&e, s + 16, 8);
    memcpy(&sg, s + 24, 4);
  } else {
    return GPZ_ESTREAM;
  }
  if ((d != 2 && d != 3) || nn == 0) return GPZ_ESTREAM;
  if (dim) *dim = d;
  if (n) *n = nn;
  if (float_bits) *float_bits = b;
  if (eb) *eb = e;
  if (seg_size) *seg_size = sg;
  return GPZ_OK;
}

int gpz_rel_to_abs(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y,
                   const void *d_z, double rel, void *d_scratch, uint64_t scratch_bytes, double *h_eb,
                   double *h_minmax6, void *stream) {
  if (!d_x || !d_y || (dim == 3 && !d_z) || !d_scratch || n == 0) return GPZ_EINVAL;
  if ((dim != 2 && dim != 3) || (float_bits != 32 && float_bits != 64)) return GPZ_EINVAL;
  if (scratch_bytes < (uint64_t)kCtlBytes) return GPZ_ENOSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Control *ctl = static_cast<Control *>(d_scratch);
  if (cudaMemsetAsync(d_scratch, 0, kCtlBytes, st) != cudaSuccess) return GPZ_ECUDA;
  const int grid = num_sms() * 4;
  if (float_bits == 32)
    rel_to_abs_kernel<float><<<grid, 256, 0, st>>>(static_cast<const float *>(d_x), static_cast<const float *>(d_y),
                                                   static_cast<const float *>(dim == 3 ? d_z : d_y), n, dim,
                                                   (float)rel, ctl);
  else
    rel_to_abs_kernel<double><<<grid, 256, 0, st>>>(static_cast<const double *>(d_x),
                                                    static_cast<const double *>(d_y),
                                                    static_cast<const double *>(dim == 3 ? d_z : d_y), n, dim, rel,
                                                    ctl);
  if (cudaGetLastError() != cudaSuccess) return GPZ_ECUDA;
  Control h;
  if (cudaMemcpyAsync(&h, d_scratch, sizeof(Control), cudaMemcpyDeviceToHost, st) != cudaSuccess) return GPZ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GPZ_ECUDA;
  if (h_eb) *h_eb = h.out_eb;
  if (h_minmax6)
    for (int k = 0; k < 6; ++k) h_minmax6[k] = h.out_mm[k];
  return GPZ_OK;
}

int gpz_aos_to_soa(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_aos, void *d_x, void *d_y, void *d_z,
                   void *stream) {
  if ((float_bits != 32 && float_bits != 64) || (dim != 2 && dim != 3) || (n && (!d_aos || !d_x || !d_y || !d_z)))
    return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return float_bits == 32 ? aos_soa<float>(true, dim, n, d_aos, d_x, d_y, d_z, st)
                          : aos_soa<double>(true, dim, n, d_aos, d_x, d_y, d_z, st);
}

int gpz_soa_to_aos(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y, const void *d_z,
                   void *d_aos, void *stream) {
  if ((float_bits != 32 && float_bits != 64) || (dim != 2 && dim != 3) ||
      (n && (!d_aos || !d_x || !d_y || (dim == 3 && !d_z))))
    return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return float_bits == 32 ? aos_soa<float>(false, dim, n, d_aos, d_x, d_y, d_z, st)
                          : aos_soa<double>(false, dim, n, d_aos, d_x, d_y, d_z, st);
}

int gpz_sample_minmax(uint32_t float_bits, uint32_t dim, uint64_t n, uint64_t begin, uint64_t count, const void *d_x,
                      const void *d_y, const void *d_z, void *d_scratch, uint64_t scratch_bytes, uint64_t *h_acc6,
                      void *stream) {
  if ((float_bits != 32 && float_bits != 64) || (dim != 2 && dim != 3) || !d_scratch || !h_acc6 || n == 0 ||
      begin > n || count > n - begin || (count && (!d_x || !d_y || (dim == 3 && !d_z))))
    return GPZ_EINVAL;
  if (scratch_bytes < kCtlBytes) return GPZ_ENOSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Control *ctl = static_cast<Control *>(d_scratch);
  if (cudaMemsetAsync(d_scratch, 0, kCtlBytes, st) != cudaSuccess) return GPZ_ECUDA;
  if (float_bits == 32) {
    const float *x = (const float *)d_x, *y = (const float *)d_y, *z = (const float *)d_z;
    seg_sample_shard_kernel<float><<<128, 256, 0, st>>>(x, y, dim == 3 ? z : y, n, begin, count, dim, ctl);
  } else {
    const double *x = (const double *)d_x, *y = (const double *)d_y, *z = (const double *)d_z;
    seg_sample_shard_kernel<double><<<128, 256, 0, st>>>(x, y, dim == 3 ? z : y, n, begin, count, dim, ctl);
  }
  if (cudaGetLastError() != cudaSuccess) return GPZ_ECUDA;
  if (cudaMemcpyAsync(h_acc6, &ctl->mm[0], 6 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return GPZ_ECUDA;
  return cuda_status(cudaStreamSynchronize(st));
}

int gpz_decide_seg(uint32_t float_bits, uint32_t dim, const uint64_t *acc6, uint32_t seg_in, int32_t rel_mode,
                   double rel_eb, double eb, uint32_t flags, uint32_t *seg, uint32_t *adjusted) {
  if ((float_bits != 32 && float_bits != 64) || (dim != 2 && dim != 3) || !acc6 || !seg || !adjusted)
    return GPZ_EINVAL;
  SegDecision sd;
  const int safe31 = (flags & GPZ_FLAG_SAFE31) ? 1 : 0;
  if (float_bits == 32) {
    float mm[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t d = 0; d < dim; ++d) {
      mm[d] = from_ord((uint32_t)~(uint32_t)acc6[2 * d]);
      mm[3 + d] = from_ord((uint32_t)acc6[2 * d + 1]);
    }
    sd = decide_seg<float>(mm, dim, seg_in, rel_mode, (float)rel_eb, (float)eb, safe31);
  } else {
    double mm[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t d = 0; d < dim; ++d) {
      mm[d] = from_ord((unsigned long long)~acc6[2 * d]);
      mm[3 + d] = from_ord((unsigned long long)acc6[2 * d + 1]);
    }
    sd = decide_seg<double>(mm, dim, seg_in, rel_mode, rel_eb, eb, safe31);
  }
  if (sd.status != kOK) return sd.status;
  *seg = sd.seg;
  *adjusted = sd.adjusted;
  return GPZ_OK;
}

int gpz_strict_bound(uint32_t float_bits, double eb, double max_abs, double max_range, double *eb_strict) {
  if ((float_bits != 32 && float_bits != 64) || !eb_strict || !(eb > 0.0) || !(max_abs >= 0.0) ||
      !(max_range >= 0.0))
    return GPZ_EINVAL;
  const double e = float_bits == 32 ? (double)strict_bound<float>((float)eb, max_abs, max_range)
                                    : strict_bound<double>(eb, max_abs, max_range);
  if (!(e > 0.0)) return GPZ_EINVAL;
  *eb_strict = e;
  return GPZ_OK;
}

int gpz_rel_abs_from_minmax(uint32_t float_bits, const double *minmax6, double rel, double *eb) {
  if ((float_bits != 32 && float_bits != 64) || !minmax6 || !eb) return GPZ_EINVAL;
  if (float_bits == 32) {
    // convertRelEb<float> (src/main.cpp:35-55), as rel_to_abs_kernel evaluates it
    const float xr = (float)minmax6[3] - (float)minmax6[0], yr = (float)minmax6[4] - (float)minmax6[1];
    const float zr = (float)minmax6[5] - (float)minmax6[2];
    *eb = (double)(fmaxf(fmaxf(xr, yr), zr) * (float)rel);
  } else {
    const double xr = minmax6[3] - minmax6[0], yr = minmax6[4] - minmax6[1], zr = minmax6[5] - minmax6[2];
    *eb = fmax(fmax(xr, yr), zr) * rel;
  }
  return GPZ_OK;
}

int gpz_stream_size(const void *d_stream, uint64_t cap, uint64_t *bytes, void *stream) {
  if (!d_stream || !bytes) return GPZ_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint8_t *s = static_cast<const uint8_t *>(d_stream);
  auto fetch = [&](void *dst, uint64_t off, uint64_t len) -> int {
    if (off > cap || len > cap - off) return GPZ_ESTREAM;
    if (cudaMemcpyAsync(dst, s + off, len, cudaMemcpyDeviceToHost, st) != cudaSuccess) return GPZ_ECUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? GPZ_OK : GPZ_ECUDA;
  };
  uint8_t h[32] = {0};
  int rc = fetch(h, 0, 24);
  if (rc != GPZ_OK) return rc;
  uint32_t bits = 0;
  uint64_t n = 0;
  memcpy(&n, h + 4, 8);
  memcpy(&bits, h + 12, 4);
  if ((bits != 32 && bits != 64) || n == 0) return GPZ_ESTREAM;
  const uint64_t hdr = bits == 32 ? TT<float>::hdr : TT<double>::hdr;
  const uint64_t meta = bits == 32 ? TT<float>::meta : TT<double>::meta;
  const uint32_t pad = bits == 32 ? TT<float>::pad : TT<double>::pad;
  const uint64_t G = chunks(n);
  if (G > (UINT64_MAX - hdr) / (8 + meta)) return GPZ_ESTREAM;
  const uint64_t pay_base = hdr + G * (8 + meta);
  uint64_t off = 0;
  uint8_t m[64] = {0};
  if ((rc = fetch(&off, hdr + 8 * (G - 1), 8)) != GPZ_OK) return rc;
  if ((rc = fetch(m, hdr + 8 * G + meta * (G - 1), meta)) != GPZ_OK) return rc;
  uint32_t dbits, cbits, rbits, U;
  if (bits == 32) {
    uint16_t f[4];
    memcpy(f, m + TT<float>::u16_at, 8);
    dbits = f[0]; cbits = f[1]; rbits = f[2]; U = f[3];
  } else {
    uint16_t f[4];
    memcpy(f, m + TT<double>::u16_at, 8);
    dbits = f[0]; cbits = f[1]; rbits = f[2]; U = f[3];
  }
  if (dbits > 32 || cbits > 32 || rbits > 32) return GPZ_ESTREAM;
  const uint64_t pl = (uint64_t)section_bytes(U, dbits, pad) + section_bytes(U, cbits, pad) + rel_section_bytes(rbits, pad);
  if (off > UINT64_MAX - pay_base - pl || pay_base + off + pl > cap) return GPZ_ESTREAM;
  *bytes = pay_base + off + pl;
  return GPZ_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free compress.
//
// Some callers cannot allocate device memory themselves: a codec plugin hosted
// by an application that owns the whole device-memory budget and only hands
// out the input and output buffers, or a latency-critical path where the
// implicit device synchronisation of cudaMalloc is not acceptable.  For them
// gpz_compress_noalloc takes its scratch (control block + one look-back word
// per 1024-point chunk) from a fixed array compiled into this library instead
// of from the caller.
// ===========================================================================
namespace {

constexpr uint64_t kNoAllocScratchBytes = 4ull << 20;  // 4 MiB per GPU, held from load to exit
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
void *g_noalloc_ptr[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name only stands for a host-side shadow, so it is never handed
// to a kernel; the address comes from cudaGetSymbolAddress, once per device,
// with that device current.
int noalloc_scratch(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return GPZ_ECUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return GPZ_ECUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return GPZ_ECUDA;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return GPZ_OK;
}

}  // namespace

extern "C" {

uint64_t gpz_compress_noalloc_max_points(void) {
  return ((kNoAllocScratchBytes - (uint64_t)kCtlBytes) / 8ull) * (uint64_t)kChunk;
}

int gpz_compress_noalloc(const gpz_params *params, const void *d_x, const void *d_y, const void *d_z, void *d_out,
                         uint64_t out_capacity, gpz_result *result, void *stream) {
  if (!params) return GPZ_EINVAL;
  if (params->n > gpz_compress_noalloc_max_points()) return GPZ_ELIMIT;
  void *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  // gpz_compress_async clears the control block and the look-back words it
  // uses, so the previous call's leftovers in the shared array do not matter.
  rc = gpz_compress_async(params, d_x, d_y, d_z, d_out, out_capacity, scratch, kNoAllocScratchBytes, stream);
  if (rc) return rc;
  return gpz_result_get(scratch, result, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Check of the bounded wait of the placement look-back: group 1 waits on a
// group 0 that never publishes its size (its look-back word stays zero, as if
// the CTA holding it had stopped), so the wait runs out after `polls` polls.
// ---------------------------------------------------------------------------
namespace {
__global__ void lookback_timeout_kernel(unsigned long long *look, Control *ctl, uint32_t polls) {
  unsigned long long excl = 0;
  const bool ok = resolve_prefix(look, 1ull, 0ull, ctl, excl, polls);
  if (threadIdx.x == 0) ctl->stream_bytes = ok ? 1ull : 0ull;
}
}  // namespace

extern "C" int gpz_selftest_lookback_timeout(uint32_t polls, void *d_scratch, uint64_t scratch_bytes, int32_t *status,
                                             void *stream) {
  if (!d_scratch || !status || polls == 0 || polls > kSpinLimit) return GPZ_EINVAL;
  if (scratch_bytes < kCtlBytes + 16) return GPZ_ENOSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Control *ctl = static_cast<Control *>(d_scratch);
  unsigned long long *look = reinterpret_cast<unsigned long long *>(static_cast<uint8_t *>(d_scratch) + kCtlBytes);
  if (cudaMemsetAsync(d_scratch, 0, kCtlBytes + 16, st) != cudaSuccess) return GPZ_ECUDA;
  lookback_timeout_kernel<<<1, 32, 0, st>>>(look, ctl, polls);
  if (cudaGetLastError() != cudaSuccess) return GPZ_ECUDA;
  Control h;
  if (cudaMemcpyAsync(&h, d_scratch, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return GPZ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GPZ_ECUDA;
  *status = h.status;
  return GPZ_OK;
}
