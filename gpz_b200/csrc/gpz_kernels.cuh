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
// Correctly rounded scalar operations, the same on the device and on the host
// (the host build uses plain IEEE operations with contraction off).
template <typename T> struct Rn;
template <> struct Rn<float> {
  __host__ __device__ static float add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
  }
  __host__ __device__ static float sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
  }
  __host__ __device__ static float mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
  }
  __host__ __device__ static float div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
  }
  __host__ __device__ static float sqrt(float a) {
#ifdef __CUDA_ARCH__
    return __fsqrt_rn(a);
#else
    return sqrtf(a);
#endif
  }
  __host__ __device__ static float from_u32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __uint2float_rn(v);
#else
    return (float)v;
#endif
  }
  // truncation with saturation (cvt.rzi.sat.u64), NaN -> 0
  __host__ __device__ static unsigned long long to_u64_rz(float v) {
#ifdef __CUDA_ARCH__
    return __float2ull_rz(v);
#else
    if (!(v > 0.0f)) return 0ull;
    if (v >= 18446744073709551616.0f) return ~0ull;
    return (unsigned long long)v;
#endif
  }
};
template <> struct Rn<double> {
  __host__ __device__ static double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
  }
  __host__ __device__ static double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
  }
  __host__ __device__ static double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
  }
  __host__ __device__ static double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
  }
  __host__ __device__ static double sqrt(double a) {
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(a);
#else
    return ::sqrt(a);
#endif
  }
  __host__ __device__ static double from_u32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __uint2double_rn(v);
#else
    return (double)v;
#endif
  }
  __host__ __device__ static unsigned long long to_u64_rz(double v) {
#ifdef __CUDA_ARCH__
    return __double2ull_rz(v);
#else
    if (!(v > 0.0)) return 0ull;
    if (v >= 18446744073709551616.0) return ~0ull;
    return (unsigned long long)v;
#endif
  }
};

// Outcome of the automatic segment-size rules.
struct SegDecision {
  int status;         // kOK, kEINVAL (no segment size in abs mode) or kESEG
  uint32_t seg, adjusted;
};

// Host arithmetic of computeSegSize (src/cudaWarpCompress.cu:1488-1554; double
// twin src/cudaWarpCompressDouble.cu:1488-1553) on the sampled per-axis
// min/max mm = (x, y, z minima, x, y, z maxima).  float: the 2D variance
// divides by 2 (:1503) and seg doubles (<= 11 times) while the block count
// would exceed UINT32_MAX; double: variance divides by 3 and the reference's
// guard compares with UINT64_MAX and never fires.  With safe31 both double
// until every id fits 31 bits.  Evaluated the same on the device (sampling
// kernel) and on the host (sharded compress).
template <typename T>
__host__ __device__ SegDecision decide_seg(const T mm[6], uint32_t dim, uint32_t seg_in, int rel_mode, T rel_eb, T eb,
                                           int safe31) {
  using R = Rn<T>;
  constexpr bool is64 = sizeof(T) == 8;
  const T dx = R::sub(mm[3], mm[0]), dy = R::sub(mm[4], mm[1]), dz = R::sub(mm[5], mm[2]);
  const T mean = R::div(R::add(R::add(dx, dy), dz), (T)3);
  const T ex = R::sub(dx, mean), ey = R::sub(dy, mean), ez = R::sub(dz, mean);
  T var = R::add(R::add(R::mul(ex, ex), R::mul(ey, ey)), R::mul(ez, ez));
  var = R::div(var, (!is64 && dim == 2) ? (T)2 : (T)3);
  const T ratio = R::div(R::sqrt(var), mean);
  const T maxr3 = is64 ? (T)fmax(fmax((double)dx, (double)dy), (double)dz) : (T)fmaxf(fmaxf((float)dx, (float)dy), (float)dz);
  uint32_t seg = seg_in;
  if (seg == 0 && rel_mode) {
    if (ratio < (T)0.1f) seg = ((double)rel_eb <= 1e-4) ? 32u : 2u;
    else seg = ((double)rel_eb <= 1e-4) ? 4u : 1u;
  }
  if (seg == 0) return {kEINVAL, 0u, 0u};
  const bool guard = !is64 || safe31;
  if (!guard) return {kOK, seg, 0u};
  const unsigned long long limit = safe31 ? 0x7FFFFFFFull : 0xFFFFFFFFull;
  auto total = [&](uint32_t s) {
    const T q = R::div(maxr3, R::mul(R::from_u32(2u * s), eb));
    const T c = is64 ? (T)::ceil((double)q) : (T)::ceilf((float)q);
    const unsigned long long mb = R::to_u64_rz(c) + 1ull;
    return dim == 3 ? mb * mb * mb : mb * mb;
  };
  if (total(seg) <= limit) return {kOK, seg, 0u};
  uint32_t t = seg;
  for (int i = 0; i < 11; ++i) {
    t *= 2u;
    if (total(t) <= limit) break;
  }
  if (t > 1024u) return {kESEG, 0u, 0u};
  return {kOK, t, 1u};
}

template <typename T>
__device__ __forceinline__ void fold_minmax(T v, typename TT<T>::U &mn_inv, typename TT<T>::U &mx) {
  if (v == v) {
    const typename TT<T>::U o = ord_of(v);
    mn_inv = max(mn_inv, (typename TT<T>::U)~o);
    mx = max(mx, o);
  }
}

// Strict-bound mode (an extension; the reference holds eb only up to the
// rounding of its reconstruction, which its verifier hides with a 1.01*eb
// slack, src/utils.cu:28).  For a snapshot whose coordinates satisfy |x| <= M
// and whose per-axis ranges are at most R, every finite point reconstructs
// within eb when the stream is encoded with
//   eb' = eb - u * (3 R + 2 M + 4 eb),   u = 2^-24 (float) / 2^-53 (double),
// rounded down.  With t = (x - m) / (2 eb') (m the chunk minimum, 0 <= x - m
// <= R), inv = fl(1/(2 eb')) = (1 + d1) / (2 eb'), nmn = fl(-m inv) and
// qf = fl(x inv + nmn), |qf - t| <= u (2 t + |m| inv) + O(u^2): truncation
// leaves x within eb' + u (2R + M) of the center m + (2q+1) eb' of its bin.
// The decoder's fused multiply-add rounds the center once, by at most
// u (M + eb'), and its conversion of 2q+1 (<= R/eb' + 1) to T by at most
// u (R + eb') eb'/eb' when 2q+1 needs more than the mantissa:
//   |x - v| <= eb' + u (3R + 2M + 2 eb') + O(u^2) < eb.
// Returns 0 when no positive eb' exists.
template <typename T>
__host__ __device__ inline T strict_bound(T eb, double max_abs, double max_range) {
  const double u = sizeof(T) == 4 ? 5.9604644775390625e-08 : 1.1102230246251565e-16;
  const double e = (double)eb - u * (3.0 * max_range + 2.0 * max_abs + 4.0 * (double)eb);
  if (!(e > 0.0)) return (T)0;
  T r = (T)e;
  if ((double)r > e) r = sizeof(T) == 4 ? (T)nextafterf((float)r, 0.0f) : (T)nextafter((double)r, 0.0);
  return r;
}

// The strict bound of a snapshot (strict_bound above with its largest
// coordinate magnitude and largest per-axis range, NaNs ignored), into
// ctl->strict_eb; kEINVAL in ctl->status when there is none.  Grid-stride;
// the last block decides.
template <typename T>
__global__ void __launch_bounds__(256) strict_bound_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                           const T *__restrict__ z, uint64_t n, uint32_t dim, T eb,
                                                           Control *ctl) {
  using U = typename TT<T>::U;
  __shared__ U red[6][8];
  __shared__ int last;
  U acc[6] = {0, 0, 0, 0, 0, 0};  // [min_inv, max] per axis
  const T *X[3] = {x, y, z};
  const unsigned long long step = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step)
    for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>(X[d][i], acc[2 * d], acc[2 * d + 1]);
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
    double M = 0.0, R = 0.0;
    for (uint32_t d = 0; d < dim; ++d) {
      const U mi = (U)~(U)((volatile unsigned long long *)ctl->mm)[2 * d];
      const U ma = (U)((volatile unsigned long long *)ctl->mm)[2 * d + 1];
      if (ma == 0) continue;  // no finite value on this axis
      const double lo = (double)from_ord(mi), hi = (double)from_ord(ma);
      M = fmax(M, fmax(fabs(lo), fabs(hi)));
      R = fmax(R, hi - lo);
    }
    const T e = strict_bound<T>(eb, M, R);
    if (!(e > (T)0)) set_status(ctl, kEINVAL);
    ctl->strict_eb = (double)e;
    // the sampling kernel that follows reuses these accumulators
    for (int k = 0; k < 6; ++k) ctl->mm[k] = 0;
    ctl->sample_done = 0;
  }
}

// sampleMinMaxXYZKernel[2D] + reduceMinMax[2D] (src/cudaWarpCompress.cu:1216-1418):
// 1024 windows of 256 consecutive points at stride max((N-256)/1024, 1).
// A window that would run past N is skipped by the reference and its
// min/max slot keeps the zero-filled scratch value, so it contributes 0.0.
// Launch: 128 blocks x 256 threads, 8 windows per block.  The last block to
// finish applies the host decision rules (decide_seg).
// One block's share (8 windows) of the sampling; `block` of `nblocks`
// (128 blocks cover the 1024 windows).
template <typename T>
__device__ __forceinline__ void seg_sample_block(const T *__restrict__ x, const T *__restrict__ y,
                                                 const T *__restrict__ z, uint64_t n, uint32_t dim, uint32_t seg_in,
                                                 int rel_mode, T rel_eb, T eb, int safe31, Control *ctl,
                                                 unsigned block, unsigned nblocks, const double *eb_dev = nullptr) {
  using U = typename TT<T>::U;
  __shared__ U red[6][8];
  __shared__ int last;
  const unsigned long long L = 256, B = 1024;
  const unsigned long long stride = max((n - L) / B, 1ull);
  U acc[6] = {0, 0, 0, 0, 0, 0};  // [min_inv, max] per axis
  const T *X[3] = {x, y, z};
  for (int w = 0; w < 8; ++w) {
    const unsigned long long win = (unsigned long long)block * 8 + w;
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
  if (threadIdx.x == 0) last = (atomicAdd(&ctl->sample_done, 1u) == nblocks - 1);
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
    const T ebv = eb_dev ? (T)*(const volatile double *)eb_dev : eb;
    const SegDecision sd = decide_seg<T>(mm, dim, seg_in, rel_mode, rel_eb, ebv, safe31);
    if (sd.status != kOK) set_status(ctl, sd.status);
    else {
      ctl->seg = sd.seg;
      ctl->adjusted = sd.adjusted;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) seg_sample_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                         const T *__restrict__ z, uint64_t n, uint32_t dim,
                                                         uint32_t seg_in, int rel_mode, T rel_eb, T eb,
                                                         int safe31, Control *ctl, const double *eb_dev) {
  if (eb_dev && ld_volatile(reinterpret_cast<const uint32_t *>(&ctl->status)) != 0) return;
  seg_sample_block<T>(x, y, z, n, dim, seg_in, rel_mode, rel_eb, eb, safe31, ctl, blockIdx.x, gridDim.x, eb_dev);
}

// The sampling windows of computeSegSize restricted to one shard
// [begin, begin + count) of a larger array (pointers start at `begin`): folds
// the shard's share of every window into ctl->mm (windows past n contribute
// 0.0, as in seg_sample_kernel).  Combining the shards' accumulators with an
// unsigned max gives exactly the whole array's.
template <typename T>
__global__ void __launch_bounds__(256) seg_sample_shard_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                               const T *__restrict__ z, uint64_t n, uint64_t begin,
                                                               uint64_t count, uint32_t dim, Control *ctl) {
  using U = typename TT<T>::U;
  __shared__ U red[6][8];
  const unsigned long long L = 256, B = 1024;
  const unsigned long long stride = max((n - L) / B, 1ull);
  U acc[6] = {0, 0, 0, 0, 0, 0};
  const T *X[3] = {x, y, z};
  for (int w = 0; w < 8; ++w) {
    const unsigned long long win = (unsigned long long)blockIdx.x * 8 + w;
    const unsigned long long st = win * stride;
    if (st + L > n) {
      for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>((T)0, acc[2 * d], acc[2 * d + 1]);
      continue;
    }
    const unsigned long long p = st + threadIdx.x;
    if (p >= begin && p - begin < count)
      for (uint32_t d = 0; d < dim; ++d) fold_minmax<T>(X[d][p - begin], acc[2 * d], acc[2 * d + 1]);
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
}

// The segment size chosen by the caller is used as is (sharded compress).
static __global__ void set_seg_kernel(Control *ctl, uint32_t seg) {
  ctl->seg = seg;
  ctl->adjusted = 0;
}

// findMinimumValues<T> + convertRelEb<T> on the device.  The host scan starts
// from float limits (include/utils.cuh:48-53) and ignores NaNs; 2D data has
// z == 0 (utils.cuh:141).
// One block (`block` of `nblocks`) of the grid-stride min/max; the last block
// to finish converts, stores the bound in ctl->out_eb and, when eb_out is
// given, in *eb_out.
template <typename T>
__device__ __forceinline__ void rel_to_abs_block(const T *__restrict__ x, const T *__restrict__ y,
                                                 const T *__restrict__ z, uint64_t n, uint32_t dim, T rel,
                                                 Control *ctl, T *eb_out, unsigned block, unsigned nblocks) {
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
  const unsigned long long step = (unsigned long long)nblocks * blockDim.x;
  for (unsigned long long i = (unsigned long long)block * blockDim.x + threadIdx.x; i < n; i += step)
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
  if (threadIdx.x == 0) last = (atomicAdd(&ctl->sample_done, 1u) == nblocks - 1);
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
    if (eb_out) *eb_out = r;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) rel_to_abs_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                         const T *__restrict__ z, uint64_t n, uint32_t dim,
                                                         T rel, Control *ctl) {
  rel_to_abs_block<T>(x, y, z, n, dim, rel, ctl, nullptr, blockIdx.x, gridDim.x);
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
  const double *eb_dev;  // when set, the bound is read here on the device (strict-bound mode)
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

// Warp-collective.  Returns false when a bounded wait (`limit` polls of a
// predecessor that has published nothing) gave up or another CTA aborted (the
// kernel then stops taking chunks and reports GPZ_ETIMEOUT).
static __device__ bool resolve_prefix(unsigned long long *look, unsigned long long c, unsigned long long agg,
                                      Control *ctl, unsigned long long &excl_out, uint32_t limit = kSpinLimit) {
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
      if (++spins > limit || ld_volatile(&ctl->abort)) {
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
