// ref_harness.cu -- drives the GPZ reference's own codec classes, compiled
// from the reference sources by oracle/Makefile (target `ref`), to produce
// golden streams / reconstructions and reference timings.
//
// TEST INFRASTRUCTURE ONLY.  Not part of the product and never built from
// or shipped in the repository's own sources.
//
// Why a harness instead of the reference CLI: the CLI sizes its scratch as
// 4*N*sizeof(T) and its output as 3*N*sizeof(T) (src/main.cpp:283-295), which
// is too small for short inputs (one 12 KiB scratch slot per 1024-point chunk,
// src/cudaWarpCompress.cu:353).  Here both buffers are sized from the format's
// worst case and zero-filled before each call, as the CLI does between runs
// (src/main.cpp:318-319).
//
// The reference decoder writes one element past b_buff_block_id when a chunk
// has 1024 unique blocks (src/cudaWarpCompress.cu:932, :1144); `decompress`
// therefore refuses such streams instead of running them.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include <cuda_runtime.h>

#include "CompressorManager.h"
#include "cudaWarpCompress.cuh"
#include "cudaWarpCompressDouble.cuh"

#define CK(x)                                                                      \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                           \
      return 2;                                                                    \
    }                                                                              \
  } while (0)

static std::vector<unsigned char> read_file(const char *path) {
  std::vector<unsigned char> v;
  FILE *f = fopen(path, "rb");
  if (!f) return v;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  rewind(f);
  v.resize((size_t)n);
  if (n > 0 && fread(v.data(), 1, (size_t)n, f) != (size_t)n) v.clear();
  fclose(f);
  return v;
}

static bool write_file(const char *path, const void *p, size_t n) {
  FILE *f = fopen(path, "wb");
  if (!f) return false;
  bool ok = fwrite(p, 1, n, f) == n;
  fclose(f);
  return ok;
}

// compress <soa_file> <n> <dim> <bits> <eb> <rel_eb> <mode> <seg> <out_stream> <reps>
template <typename T>
static int do_compress(char **a) {
  const char *soa = a[0];
  const uint64_t n = strtoull(a[1], nullptr, 10);
  const uint32_t dim = (uint32_t)atoi(a[2]);
  const uint32_t bits = (uint32_t)atoi(a[3]);
  const double eb = strtod(a[4], nullptr), rel = strtod(a[5], nullptr);
  const std::string mode = a[6];
  const uint32_t seg = (uint32_t)strtoul(a[7], nullptr, 10);
  const char *out = a[8];
  const int reps = std::max(1, atoi(a[9]));
  std::vector<unsigned char> in = read_file(soa);
  if (in.size() != 3 * n * sizeof(T)) {
    fprintf(stderr, "input size %zu != 3*n*sizeof(T)\n", in.size());
    return 1;
  }
  const uint64_t G = (n + 1023) / 1024;
  const uint64_t meta = bits == 64 ? 64 : 36, slot = bits == 64 ? 24576 : 12288;
  const uint64_t hdr = bits == 64 ? 32 : 24;
  const uint64_t xyz_bytes = std::max<uint64_t>(3 * n * sizeof(T), hdr + G * (8 + meta + slot));
  const uint64_t scratch_bytes = std::max<uint64_t>(4 * n * sizeof(T), G * (meta + slot) + 65536);
  ICudaCompressor *comp;
  if (bits == 32) {
    CudaConfig cfg(seg, false, dim, n, mode, (float)eb, (float)rel, bits);
    comp = new CudaWarpCompress(cfg);
  } else {
    CudaConfig cfg(seg, false, dim, n, mode, eb, rel, bits);
    comp = new CudaWarpCompressDouble(cfg);
  }
  CompressorManager mgr;
  void *d_xyz = nullptr;
  unsigned char *d_scratch = nullptr;
  CK(cudaMalloc(&d_xyz, xyz_bytes));
  CK(cudaMalloc(&d_scratch, scratch_bytes));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  uint64_t comp_size = 0;
  std::vector<float> ms;
  for (int r = 0; r < reps; ++r) {
    CK(cudaMemset(d_scratch, 0, scratch_bytes));
    CK(cudaMemset(d_xyz, 0, xyz_bytes));
    CK(cudaMemcpy(d_xyz, in.data(), in.size(), cudaMemcpyHostToDevice));
    CK(cudaDeviceSynchronize());
    CK(cudaEventRecord(e0));
    mgr.compressWarp(d_xyz, d_scratch, &comp_size, "none", comp);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    ms.push_back(t);
  }
  CK(cudaGetLastError());
  std::vector<unsigned char> s(comp_size);
  CK(cudaMemcpy(s.data(), d_xyz, comp_size, cudaMemcpyDeviceToHost));
  if (!write_file(out, s.data(), s.size())) return 1;
  const CudaConfig &cf = comp->getConfig();
  printf("{\"op\": \"compress\", \"n\": %llu, \"dim\": %u, \"bits\": %u, \"seg\": %u, \"adjusted\": %s, "
         "\"bytes\": %llu, \"ms\": [",
         (unsigned long long)n, dim, bits, cf.seg_size, cf.adjusted_seg ? "true" : "false",
         (unsigned long long)comp_size);
  for (size_t i = 0; i < ms.size(); ++i) printf("%s%.6f", i ? ", " : "", ms[i]);
  printf("]}\n");
  cudaFree(d_xyz);
  cudaFree(d_scratch);
  delete comp;
  return 0;
}

// decompress <stream> <out_soa> <reps>
template <typename T>
static int do_decompress(const std::vector<unsigned char> &s, const char *out, int reps) {
  uint32_t dim = 0, bits = 0;
  uint64_t n = 0;
  memcpy(&dim, s.data(), 4);
  memcpy(&n, s.data() + 4, 8);
  memcpy(&bits, s.data() + 12, 4);
  const uint64_t G = (n + 1023) / 1024;
  const uint64_t hdr = bits == 64 ? 32 : 24, meta = bits == 64 ? 64 : 36, u16_at = bits == 64 ? 56 : 28;
  if (s.size() < hdr + G * (8 + meta)) {
    fprintf(stderr, "stream too short\n");
    return 1;
  }
  for (uint64_t c = 0; c < G; ++c) {
    uint16_t U;
    memcpy(&U, s.data() + hdr + 8 * G + c * meta + u16_at + 6, 2);
    if (U >= 1024) {
      printf("{\"op\": \"decompress\", \"refused\": \"chunk %llu has 1024 unique blocks\"}\n",
             (unsigned long long)c);
      return 3;
    }
  }
  const uint64_t one = n * sizeof(T);
  unsigned char *d_s = nullptr;
  void *d_o[3] = {nullptr, nullptr, nullptr};
  CK(cudaMalloc(&d_s, std::max<uint64_t>(s.size(), 2 * one)));
  for (int k = 0; k < 3; ++k) CK(cudaMalloc(&d_o[k], one));
  ICudaCompressor *dec = bits == 32 ? (ICudaCompressor *)new CudaWarpCompress()
                                    : (ICudaCompressor *)new CudaWarpCompressDouble();
  CompressorManager mgr;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  std::vector<float> ms;
  for (int r = 0; r < reps; ++r) {
    for (int k = 0; k < 3; ++k) CK(cudaMemset(d_o[k], 0, one));
    CK(cudaMemcpy(d_s, s.data(), s.size(), cudaMemcpyHostToDevice));
    CK(cudaDeviceSynchronize());
    CK(cudaEventRecord(e0));
    mgr.decompressWarp(d_o[0], d_o[1], d_o[2], d_s, dec, "none");
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    ms.push_back(t);
  }
  CK(cudaGetLastError());
  std::vector<unsigned char> h(3 * one);
  for (int k = 0; k < 3; ++k) CK(cudaMemcpy(h.data() + k * one, d_o[k], one, cudaMemcpyDeviceToHost));
  if (!write_file(out, h.data(), h.size())) return 1;
  printf("{\"op\": \"decompress\", \"n\": %llu, \"dim\": %u, \"bits\": %u, \"ms\": [",
         (unsigned long long)n, dim, bits);
  for (size_t i = 0; i < ms.size(); ++i) printf("%s%.6f", i ? ", " : "", ms[i]);
  printf("]}\n");
  cudaFree(d_s);
  for (int k = 0; k < 3; ++k) cudaFree(d_o[k]);
  delete dec;
  return 0;
}

int main(int argc, char **argv) {
  if (argc >= 12 && !strcmp(argv[1], "compress")) {
    return atoi(argv[5]) == 64 ? do_compress<double>(argv + 2) : do_compress<float>(argv + 2);
  }
  if (argc >= 5 && !strcmp(argv[1], "decompress")) {
    std::vector<unsigned char> s = read_file(argv[2]);
    if (s.size() < 24) {
      fprintf(stderr, "cannot read stream\n");
      return 1;
    }
    uint32_t bits;
    memcpy(&bits, s.data() + 12, 4);
    const int reps = std::max(1, atoi(argv[4]));
    return bits == 64 ? do_decompress<double>(s, argv[3], reps) : do_decompress<float>(s, argv[3], reps);
  }
  fprintf(stderr,
          "usage: %s compress <soa> <n> <dim> <bits> <eb> <rel_eb> <mode> <seg> <out> <reps>\n"
          "       %s decompress <stream> <out_soa> <reps>\n",
          argv[0], argv[0]);
  return 1;
}
