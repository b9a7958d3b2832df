// gpz_launch.h -- per-device launch facts of the codec's persistent kernels.
//
// Grid sizes depend on the SM count and on how many CTAs of a kernel fit on
// one SM, and kernels that use more than 48 KB of dynamic shared memory need
// cudaFuncAttributeMaxDynamicSharedMemorySize raised first.  That attribute
// is set on the CURRENT device only, so both facts are cached per device
// ordinal: a process that drives several GPUs raises the attribute once on
// each of them.  The caches are guarded by a mutex, so calls from several host
// threads (the request server's worker and its callers) are safe.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace gpzb {

// SM count of the current device (148, a B200's, if the query fails).
int current_sms();

// CTAs of `func` (launched with `threads` threads and `smem` bytes of dynamic
// shared memory) resident per SM on the current device, after raising its
// dynamic shared-memory limit there.  0 when the attribute cannot be set.
int resident_ctas_fn(const void *func, int threads, size_t smem);

template <typename K>
inline int resident_ctas(K kernel, int threads, size_t smem) {
  return resident_ctas_fn(reinterpret_cast<const void *>(kernel), threads, smem);
}

}  // namespace gpzb
