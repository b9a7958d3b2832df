// gpz_launch.cu -- per-device caches of SM counts and kernel residency.
#include "gpz_launch.h"

#include <mutex>

namespace gpzb {
namespace {

constexpr int kMaxDevices = 64;
constexpr int kMaxKernels = 48;

struct KernelFacts {
  const void *func;
  int threads;
  size_t smem;
  int ctas;
};

struct DeviceFacts {
  int sms = 0;
  int nk = 0;
  KernelFacts k[kMaxKernels];
};

DeviceFacts g_dev[kMaxDevices];
std::mutex g_mu;

int query_sms(int dev) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 148;
  return sms;
}

int query_ctas(const void *func, int threads, size_t smem) {
  if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int ctas = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, func, threads, smem) != cudaSuccess || ctas < 1) ctas = 1;
  return ctas;
}

}  // namespace

int current_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 0 || dev >= kMaxDevices) return query_sms(dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_dev[dev].sms == 0) g_dev[dev].sms = query_sms(dev);
  return g_dev[dev].sms;
}

int resident_ctas_fn(const void *func, int threads, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (dev < 0 || dev >= kMaxDevices) return query_ctas(func, threads, smem);
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceFacts &d = g_dev[dev];
  for (int i = 0; i < d.nk; ++i)
    if (d.k[i].func == func && d.k[i].threads == threads && d.k[i].smem == smem) return d.k[i].ctas;
  const int ctas = query_ctas(func, threads, smem);
  if (ctas > 0 && d.nk < kMaxKernels) d.k[d.nk++] = KernelFacts{func, threads, smem, ctas};
  return ctas;
}

}  // namespace gpzb
