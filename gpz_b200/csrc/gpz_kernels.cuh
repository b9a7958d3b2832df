// gpz_kernels.cuh -- sm_100a kernels of the B200 GPZ codec.
//
//   seg_sample_kernel   computeSegSize (reference src/cudaWarpCompress.cu:1424-1557)
//   rel_to_abs_kernel   findMinimumValues + convertRelEb (include/utils.cuh:44-65,
//                       src/main.cpp:35-55), on the device
//   (compress_kernel: gpz_encode.cuh; decompress_kernel: gpz_decode.cuh)
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

}  // namespace gpzb
