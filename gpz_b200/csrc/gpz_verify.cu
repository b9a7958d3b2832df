// gpz_verify.cu -- per-point verification of a reconstruction against the
// original points (gpz_verify of include/gpz_b200.h).
//
// The reference verifier (src/utils.cu:17-217) sorts every axis of both
// arrays and compares the sorted sequences: it never pairs a reconstructed
// point with its original, because the decoder emits points in the stream's
// order (sorted by block within each chunk).  Here the pairing is recovered
// exactly: for each 1024-point chunk the kernel recomputes what the encoder
// sorted -- the composite (block id - min block id) << 10 | r, r being the
// point's rank in the encoder's input order -- and sorts it, so sorted
// position s of the chunk holds the composite of the point the decoder wrote
// at s.  Every point is then checked against the bound, and per axis the
// maximum error and the squared-error sum (for MSE / PSNR) are accumulated.
// The quantization arithmetic is the compress kernel's (gpz_encode.cuh step
// 1) so the block ids are the encoder's bit for bit.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "gpz_b200.h"
#include "gpz_kernels.cuh"
#include "gpz_launch.h"

using namespace gpzb;

namespace {

struct VerifyAcc {
  unsigned long long over;      // points with some axis off by more than eb
  unsigned long long over_tol;  // ... by more than 1.01 * eb (the reference verifier's tolerance)
  unsigned long long max_err[3];  // ordered keys of the largest |error| per axis (non-negative floats)
  double sq[3];                 // squared-error sums
  unsigned long long mm[6];     // ordered min (inverted) / max of the originals, per axis
};

constexpr int kVerifyWarps = 8;

template <typename T, int DIM>
__global__ void __launch_bounds__(32 * kVerifyWarps) verify_kernel(const T *__restrict__ x, const T *__restrict__ y,
                                                                   const T *__restrict__ z, const T *__restrict__ rx,
                                                                   const T *__restrict__ ry, const T *__restrict__ rz,
                                                                   unsigned long long n, T eb, uint32_t seg,
                                                                   T bound, VerifyAcc *acc) {
  using UO = typename TT<T>::U;
  constexpr bool is64 = sizeof(T) == 8;
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(16) unsigned long long vsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long *const C = vsm + warp * kChunk;
  const T *X[3] = {x, y, z};
  const T *R[3] = {rx, ry, rz};
  const uint32_t sh = (uint32_t)__ffs((int)seg) - 1u, msk = seg - 1u;
  (void)msk;
  const T inv = is64 ? (T)__ddiv_rn(1.0, __dmul_rn(2.0, (double)eb)) : (T)__fdiv_rn(1.0f, __fmul_rn(2.0f, (float)eb));
  const unsigned long long G = (n + kChunk - 1) / kChunk;
  unsigned long long over = 0, over_tol = 0;
  const T tol = (T)1.01f * bound;
  T emax[3] = {0, 0, 0};
  double sq[3] = {0.0, 0.0, 0.0};
  UO gmn[3] = {0, 0, 0}, gmx[3] = {0, 0, 0};
  for (unsigned long long c = (unsigned long long)blockIdx.x * kVerifyWarps + warp; c < G;
       c += (unsigned long long)gridDim.x * kVerifyWarps) {
    const unsigned long long base = c * kChunk;
    const uint32_t nvalid = (uint32_t)min((unsigned long long)kChunk, n - base);
    // ---- block ids exactly as encode_chunk computes them ----
    uint32_t key[32];
    unsigned long long bnx = 0, bny = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      T v[32];
      const T lim = is64 ? (T)DBL_MAX : (T)FLT_MAX;
      T mn = lim, mx = -lim;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const uint32_t p = 32u * j + lane;
        v[j] = p < nvalid ? X[d][base + p] : (T)0;
        if (p < nvalid) { mn = fmin(mn, v[j]); mx = fmax(mx, v[j]); }
      }
      mn = from_ord((UO)~warp_max((UO)~ord_of(mn)));
      mx = from_ord(warp_max(ord_of(mx)));
      gmn[d] = max(gmn[d], (UO)~ord_of(mn));
      gmx[d] = max(gmx[d], ord_of(mx));
      const T range = is64 ? (T)__dsub_rn((double)mx, (double)mn) : (T)__fsub_rn((float)mx, (float)mn);
      if (d == 0) bnx = block_num(range, seg, eb, is64 && DIM == 2);
      if (d == 1) bny = block_num(range, seg, eb, false);
      const T nmn = is64 ? (T)__dmul_rn(-(double)mn, (double)inv) : (T)__fmul_rn(-(float)mn, (float)inv);
      const uint32_t kmul = d == 0 ? 1u : (d == 1 ? (uint32_t)bnx : (uint32_t)(bnx * bny));
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        uint32_t kq;
        if constexpr (!is64) {
          kq = __float2uint_rz(__fmaf_rn((float)v[j], (float)inv, (float)nmn)) >> sh;
        } else {
          kq = (uint32_t)(__double2ull_rz(__fma_rn((double)v[j], (double)inv, (double)nmn)) >> sh);
        }
        key[j] = d == 0 ? kq : key[j] + kq * kmul;
      }
    }
    uint32_t kmin = FULL;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      key[j] &= 0x7FFFFFFFu;
      if (32u * j + lane < nvalid) kmin = min(kmin, key[j]);
    }
    kmin = warp_min(kmin);
    // composites: point p = 32j + lane has rank r = 32 lane + j
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint32_t r = 32u * lane + j;
      C[r] = 32u * j + lane < nvalid ? ((unsigned long long)(key[j] - kmin) << 10) | r : ~0ull;
    }
    __syncwarp();
    // ---- ascending bitonic sort of the 1024 composites in shared memory ----
    for (uint32_t k = 2; k <= (uint32_t)kChunk; k <<= 1) {
      for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
        for (uint32_t q = lane; q < (uint32_t)kChunk / 2; q += 32) {
          const uint32_t i = ((q & ~(jj - 1)) << 1) | (q & (jj - 1));
          const uint32_t p = i + jj;
          const bool up = (i & k) == 0;
          const unsigned long long a = C[i], b = C[p];
          if ((a > b) == up) {
            C[i] = b;
            C[p] = a;
          }
        }
        __syncwarp();
      }
    }
    // ---- sorted position s holds the point the decoder wrote at s ----
#pragma unroll 4
    for (int j = 0; j < 32; ++j) {
      const uint32_t s = 32u * j + lane;
      if (s >= nvalid) continue;
      const uint32_t r = (uint32_t)(C[s] & 1023u);
      const uint32_t p = (r & 31u) * 32u + (r >> 5);
      bool off = false, off_tol = false;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const T o = X[d][base + p], rec = R[d][base + s];
        const T e = o > rec ? o - rec : rec - o;
        off |= !(e <= bound);
        off_tol |= !(e <= tol);
        emax[d] = fmax(emax[d], e);
        sq[d] += (double)e * (double)e;
      }
      over += off ? 1ull : 0ull;
      over_tol += off_tol ? 1ull : 0ull;
    }
    __syncwarp();
  }
  // ---- warp, then global accumulation ----
  over = __reduce_add_sync(FULL, (uint32_t)over);
  over_tol = __reduce_add_sync(FULL, (uint32_t)over_tol);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const UO em = warp_max(ord_of(emax[d]));
    double s = sq[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    const UO a = warp_max(gmn[d]), b = warp_max(gmx[d]);
    if (lane == 0) {
      atomicMax(&acc->max_err[d], (unsigned long long)em);
      atomicAdd(&acc->sq[d], s);
      atomicMax(&acc->mm[2 * d], (unsigned long long)a);
      atomicMax(&acc->mm[2 * d + 1], (unsigned long long)b);
    }
  }
  if (lane == 0) {
    atomicAdd(&acc->over, over);
    atomicAdd(&acc->over_tol, over_tol);
  }
}

template <typename T>
double unord(unsigned long long o) {
  if constexpr (sizeof(T) == 4) return (double)from_ord((uint32_t)o);
  else return from_ord(o);
}

template <typename T>
int verify_t(uint32_t dim, uint64_t n, const void *dx, const void *dy, const void *dz, const void *rx, const void *ry,
             const void *rz, double eb, uint32_t seg, double bound, void *d_scratch, gpz_verify_result *out,
             cudaStream_t st) {
  VerifyAcc *acc = static_cast<VerifyAcc *>(d_scratch);
  if (cudaMemsetAsync(acc, 0, sizeof(VerifyAcc), st) != cudaSuccess) return GPZ_ECUDA;
  const size_t smem = (size_t)kVerifyWarps * kChunk * 8;
  const T *x = (const T *)dx, *y = (const T *)dy, *z = (const T *)(dim == 3 ? dz : dy);
  const T *a = (const T *)rx, *b = (const T *)ry, *c = (const T *)(dim == 3 ? rz : ry);
  const int sms = current_sms();
  const uint64_t G = (n + kChunk - 1) / kChunk;
  auto launch = [&](auto kernel) -> bool {
    const int occ = resident_ctas(kernel, 32 * kVerifyWarps, smem);
    if (occ == 0) return false;
    const uint64_t grid = std::min<uint64_t>((G + kVerifyWarps - 1) / kVerifyWarps, (uint64_t)sms * occ);
    kernel<<<(unsigned)grid, 32 * kVerifyWarps, smem, st>>>(x, y, z, a, b, c, n, (T)eb, seg, (T)bound, acc);
    return true;
  };
  if (!(dim == 3 ? launch(verify_kernel<T, 3>) : launch(verify_kernel<T, 2>))) return GPZ_ECUDA;
  if (cudaGetLastError() != cudaSuccess) return GPZ_ECUDA;
  VerifyAcc h;
  if (cudaMemcpyAsync(&h, acc, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return GPZ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return GPZ_ECUDA;
  memset(out, 0, sizeof(*out));
  out->points = n;
  out->over_bound = h.over;
  out->over_bound_tol = h.over_tol;
  double nrm = 0.0;
  for (uint32_t d = 0; d < dim; ++d) {
    using UO = typename TT<T>::U;
    out->max_abs_err[d] = unord<T>(h.max_err[d]);
    out->mse[d] = h.sq[d] / (double)n;
    const double mn = unord<T>((UO) ~(UO)h.mm[2 * d]), mx = unord<T>(h.mm[2 * d + 1]);
    out->value_range[d] = mx - mn;
    out->psnr[d] = 20.0 * log10(mx - mn) - 10.0 * log10(out->mse[d]);
    const double r = pow(10.0, out->psnr[d] / -20.0);
    nrm += r * r;
  }
  const double rms = sqrt(nrm / dim);
  out->psnr_combined = rms > 0.0 ? -20.0 * log10(rms) : INFINITY;
  return GPZ_OK;
}

}  // namespace

extern "C" {

uint64_t gpz_verify_scratch_bytes(void) { return 256; }

int gpz_verify_bound(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y, const void *d_z,
                     const void *d_rx, const void *d_ry, const void *d_rz, double eb, uint32_t seg_size, double bound,
                     void *d_scratch, uint64_t scratch_bytes, gpz_verify_result *result, void *stream) {
  if ((float_bits != 32 && float_bits != 64) || (dim != 2 && dim != 3) || n == 0 || !d_x || !d_y ||
      (dim == 3 && !d_z) || !d_rx || !d_ry || (dim == 3 && !d_rz) || seg_size == 0 || !(eb > 0.0) ||
      !(bound > 0.0) || !d_scratch || !result)
    return GPZ_EINVAL;
  if (scratch_bytes < sizeof(VerifyAcc)) return GPZ_ENOSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return float_bits == 32
             ? verify_t<float>(dim, n, d_x, d_y, d_z, d_rx, d_ry, d_rz, eb, seg_size, bound, d_scratch, result, st)
             : verify_t<double>(dim, n, d_x, d_y, d_z, d_rx, d_ry, d_rz, eb, seg_size, bound, d_scratch, result, st);
}

int gpz_verify(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y, const void *d_z,
               const void *d_rx, const void *d_ry, const void *d_rz, double eb, uint32_t seg_size, void *d_scratch,
               uint64_t scratch_bytes, gpz_verify_result *result, void *stream) {
  return gpz_verify_bound(float_bits, dim, n, d_x, d_y, d_z, d_rx, d_ry, d_rz, eb, seg_size, eb, d_scratch,
                          scratch_bytes, result, stream);
}

}  // extern "C"
