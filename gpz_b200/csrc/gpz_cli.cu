// gpz_cli.cu -- the `gpz` command line tool on the B200 library.
//
// Same flags, validation, messages and printed results as the reference CLI
// (src/main.cpp:59-561), so scripts written for it run unchanged:
//   gpz -x -i <aos file> -o <stream> -n <N> -m rel|abs -e <bound> -f 32|64 [-p 2|3] [-s seg] [-t none]
//   gpz -d -o <stream> -r <aos out> [-v <original aos>]
// Differences: the AoS<->SoA file transposition and the rel->abs bound run on
// the GPU (the reference loops on the host, include/utils.cuh:44-180), and a
// failing codec call ends the program with status 1 and a message (the
// reference exits inside the library).  Verification (-v) follows the
// reference's: each axis of the decoded and original points is sorted, then
// points off by more than 1.01*eb are counted and the MSE / PSNR reported
// (src/utils.cu:17-217).

#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include <chrono>

#include <getopt.h>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/sort.h>
#include <thrust/transform_reduce.h>
#include <thrust/iterator/counting_iterator.h>

#include "gpz_b200.h"
#include "../../include/gpz/CompressorManager.h"

namespace {

void print_usage(const char *prog) {
  std::cerr << "\nUsage:\n"
            << "  " << prog
            << " -x -i <input_file> -o <output_file> -n <num_points> -e <error_bound> -s <segment_size> -m <error_mode> [-t <nvcomp_type>]\n"
            << "      Compress mode:\n"
            << "        -x               Enable compression mode\n"
            << "        -i <file>        Input file to compress (required)\n"
            << "        -o <file>        Output compressed file (required)\n"
            << "        -p <dim>         [Optional]Number of dimensions (only support 2 or 3) (default: 3)\n"
            << "        -n <num>         Number of points (required)\n"
            << "        -m <string>      Error mode (e.g., rel, abs) (required)\n"
            << "        -f <int>         Float bits (32 or 64)\n"
            << "        -e <float>       Error bound (required)\n"
            << "        -s <int>         [Optional] Segment size\n"
            << "        -t <string>      [Optional] nvcomp compression type (e.g., none, lz4)\n"
            << "\n"
            << "  " << prog
            << " -d -i <input_file> -o <output_file> [-r <recontracted_file>] [-v <original_file>] [-t <nvcomp_type> -n <num_points> -e <error_bound> -f <float_bits>]\n"
            << "      Decompress mode:\n"
            << "        -d               Enable decompression mode\n"
            << "        -o <file>        Output decompressed file (required)\n"
            << "        -r <file>        Output recontracted (refitted) file\n"
            << "        -v <file>        [Optional] Verification mode, compares output to original file\n"
            << "        -t <string>      [Optional] nvcomp type; if set, requires -n, -e, and -f\n"
            << "        -n <num>         [Required if -t used] Number of points\n"
            << "        -e <float>       [Required if -t used] Error bound\n"
            << "        -f <int>         [Required if -t used] Float bits (32 or 64)\n"
            << "        -p <dim>         [Optional] Number of dimensions (default: 3)\n"
            << "\n"
            << "  Extension (not in the reference):\n"
            << "        -B               [Optional, compress] Hold the error bound for every point (strict-bound mode)\n"
            << std::endl;
}

void cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void gpz_ok(int rc, const char *what) {
  if (rc != GPZ_OK) throw std::runtime_error(std::string(what) + " failed with status " + std::to_string(rc));
}

// Whole file into pinned host memory.
std::vector<unsigned char> read_file(const char *path, uint64_t *size) {
  FILE *f = fopen(path, "rb");
  if (!f) throw std::runtime_error(std::string("Failed to open input file ") + path);
  fseek(f, 0, SEEK_END);
  const long long sz = ftell(f);
  rewind(f);
  std::vector<unsigned char> buf((size_t)sz);
  if (sz > 0 && fread(buf.data(), 1, (size_t)sz, f) != (size_t)sz) {
    fclose(f);
    throw std::runtime_error(std::string("Failed to read ") + path);
  }
  fclose(f);
  *size = (uint64_t)sz;
  return buf;
}

void write_file(const char *path, const void *data, uint64_t bytes) {
  FILE *f = fopen(path, "wb");
  if (!f) throw std::runtime_error(std::string("Failed to open file for writing: ") + path);
  if (bytes && fwrite(data, 1, (size_t)bytes, f) != (size_t)bytes) {
    fclose(f);
    throw std::runtime_error(std::string("Failed to write ") + path);
  }
  fclose(f);
}

struct Pinned {
  void *p = nullptr;
  explicit Pinned(uint64_t bytes) { cuda_ok(cudaMallocHost(&p, bytes ? bytes : 1), "cudaMallocHost"); }
  ~Pinned() { cudaFreeHost(p); }
};
struct Device {
  void *p = nullptr;
  explicit Device(uint64_t bytes) { cuda_ok(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~Device() { cudaFree(p); }
};

// AoS file -> device SoA (x[N] y[N] z[N], z = 0 for 2D), as
// load_file_to_soa_xyz<T> (include/utils.cuh:83-144) with the transposition on
// the GPU.  `aos` keeps the pinned file contents for reloads.
template <typename T>
void check_points_file(const char *path, uint64_t n, uint32_t dim) {
  FILE *f = fopen(path, "rb");
  if (!f) throw std::runtime_error("Failed to open input file");
  fseek(f, 0, SEEK_END);
  const uint64_t file_size = (uint64_t)ftell(f);
  fclose(f);
  if (file_size % (dim * sizeof(T)) != 0) throw std::runtime_error("File size is not aligned to expected T struct");
  if (file_size / (dim * sizeof(T)) != n) throw std::runtime_error("File size does not match expected number of points");
}

template <typename T>
void load_points(const char *path, uint64_t n, uint32_t dim, Pinned &aos) {
  FILE *f = fopen(path, "rb");
  if (!f) throw std::runtime_error("Failed to open input file");
  fseek(f, 0, SEEK_END);
  const uint64_t file_size = (uint64_t)ftell(f);
  rewind(f);
  const uint64_t point_size = dim * sizeof(T);
  if (file_size % point_size != 0) {
    fclose(f);
    throw std::runtime_error("File size is not aligned to expected T struct");
  }
  if (file_size / point_size != n) {
    fclose(f);
    throw std::runtime_error("File size does not match expected number of points");
  }
  if (fread(aos.p, point_size, n, f) != n) {
    fclose(f);
    throw std::runtime_error(dim == 3 ? "Failed to read complete 3D data" : "Failed to read complete 2D data");
  }
  fclose(f);
}

template <typename T>
void upload_soa(const Pinned &aos, Device &d_aos, void *d_xyz, uint64_t n, uint32_t dim) {
  cuda_ok(cudaMemcpy(d_aos.p, aos.p, n * dim * sizeof(T), cudaMemcpyHostToDevice), "upload");
  T *x = static_cast<T *>(d_xyz);
  gpz_ok(gpz_aos_to_soa(sizeof(T) * 8, dim, n, d_aos.p, x, x + n, x + 2 * n, nullptr), "gpz_aos_to_soa");
}

void print_compression_result(uint64_t comp_size, uint64_t original_bytes, double g_bytes, float ms,
                              const CudaConfig &cfg) {
  printf("Segment size: %d\n", cfg.seg_size);
  printf("Adjusted Seg: %s\n", cfg.adjusted_seg ? "true" : "false");
  printf("PCompression size (MB): %f\n", comp_size / 1024.0 / 1024.0);
  printf("PCompression ratio: %f\n", (original_bytes * 1.0 / comp_size));
  printf("PCompression_CUDA throughput (GB/s): %f\n", (original_bytes / g_bytes) / (ms / 1000.0));
  printf("PCompression_CUDA execution time (ms): %f\n", ms);
}

// The reference prints this with sizeof(float) for either width (src/main.cpp:17).
void print_decompression_result(uint64_t n, double ms, uint32_t dim) {
  printf("Decompression_CUDA throughput (GB/s): %f\n", (n * dim * sizeof(float) / 1024 / 1024 / 1024.0) / (ms / 1000.0));
  printf("Decompression_CUDA execution time (ms): %f\n", ms);
}

// Per-axis check of the reference verifier (src/utils.cu:47-128): both axes
// sorted, points off by more than 1.01*eb counted, MSE and PSNR.
template <typename T>
std::pair<uint32_t, double> verify_axis(const T *d_dec, const T *d_ref, uint64_t n, T eb, T mn, T mx,
                                        const char *label) {
  thrust::device_vector<T> dec(d_dec, d_dec + n), ref(d_ref, d_ref + n);
  thrust::sort(dec.begin(), dec.end());
  thrust::sort(ref.begin(), ref.end());
  const T *a = thrust::raw_pointer_cast(dec.data()), *b = thrust::raw_pointer_cast(ref.data());
  const uint64_t count = thrust::transform_reduce(
      thrust::device, thrust::counting_iterator<uint64_t>(0), thrust::counting_iterator<uint64_t>(n),
      [a, b, eb] __device__(uint64_t i) -> uint64_t {
        const T diff = a[i] - b[i];
        return (diff < 0 ? -diff : diff) > (T)1.01f * eb ? 1ull : 0ull;
      },
      0ull, thrust::plus<uint64_t>());
  const double sum = thrust::transform_reduce(
      thrust::device, thrust::counting_iterator<uint64_t>(0), thrust::counting_iterator<uint64_t>(n),
      [a, b] __device__(uint64_t i) -> double {
        const T diff = a[i] - b[i];
        return (double)(diff * diff);
      },
      0.0, thrust::plus<double>());
  const double mse = sum / n;
  const double psnr = 20.0 * log10(mx - mn) - 10.0 * log10(mse);
  printf("[%s] Error count = %u / %zu\n", label, (uint32_t)count, (size_t)n);
  printf("[%s] MSE = %e\n", label, mse);
  printf("[%s] PSNR = %.4f dB\n", label, psnr);
  return {(uint32_t)count, psnr};
}

double combine_psnr(const std::vector<double> &psnr_list) {
  if (psnr_list.empty()) return std::numeric_limits<double>::infinity();
  double sum_sq = 0.0;
  for (double p : psnr_list) {
    const double nrmse = std::pow(10.0, p / -20.0);
    sum_sq += nrmse * nrmse;
  }
  const double rms = std::sqrt(sum_sq / psnr_list.size());
  return rms > 0.0 ? -20.0 * std::log10(rms) : std::numeric_limits<double>::infinity();
}

template <typename T>
void verify(const T *d_dec, const char *original, uint64_t n, uint32_t dim, double eb) {
  check_points_file<T>(original, n, dim);
  Pinned aos(n * dim * sizeof(T));
  load_points<T>(original, n, dim, aos);
  Device d_aos(n * dim * sizeof(T)), d_ref(3 * n * sizeof(T)), scratch(gpz_compress_scratch_bytes(0));
  upload_soa<T>(aos, d_aos, d_ref.p, n, dim);
  const T *ref = static_cast<const T *>(d_ref.p);
  // findMinimumValues<T> (include/utils.cuh:44-65) through the rel->abs kernel
  double eb_unused = 0.0, mm[6];
  gpz_ok(gpz_rel_to_abs(sizeof(T) * 8, dim, n, ref, ref + n, ref + 2 * n, 1.0, scratch.p,
                        gpz_compress_scratch_bytes(0), &eb_unused, mm, nullptr),
         "gpz_rel_to_abs");
  printf("verify by CUDA...\n");
  const T e = (T)eb;
  auto [cx, px] = verify_axis<T>(d_dec, ref, n, e, (T)mm[0], (T)mm[3], "X");
  auto [cy, py] = verify_axis<T>(d_dec + n, ref + n, n, e, (T)mm[1], (T)mm[4], "Y");
  std::vector<double> psnrs = {px, py};
  uint64_t total = (uint64_t)cx + cy;
  if (dim == 3) {
    auto [cz, pz] = verify_axis<T>(d_dec + 2 * n, ref + 2 * n, n, e, (T)mm[2], (T)mm[5], "Z");
    psnrs = {px, py, pz};
    total += cz;
  }
  printf("Error Count: %zu\n", (size_t)total);
  printf("PSNR: %f\n", combine_psnr(psnrs));
}

// -B (an extension): strict-bound mode through the C ABI
// (GPZ_FLAG_STRICT_BOUND): the stream holds the stated bound for every
// finite point; its header carries the shrunk bound actually encoded.
template <typename T>
int run_compress_strict(const Pinned &aos, const Device &d_aos, const Device &d_xyz, const char *out, uint64_t n,
                        uint32_t dim, const std::string &mode, double bound, double input_bound, uint32_t seg) {
  gpz_params p;
  memset(&p, 0, sizeof(p));
  p.float_bits = sizeof(T) * 8;
  p.dim = dim;
  p.n = n;
  p.eb = bound;
  p.rel_eb = input_bound;
  p.rel_mode = mode == "rel" ? 1 : 0;
  p.seg_size = seg;
  p.flags = GPZ_FLAG_STRICT_BOUND;
  const uint64_t cap = gpz_stream_bound(n, dim, p.float_bits), scr_bytes = gpz_compress_scratch_bytes(n);
  Device d_out(cap), scr(scr_bytes);
  const T *x = static_cast<const T *>(d_xyz.p);
  gpz_result r;
  for (int i = 0; i < 5; ++i)  // warm up, as the reference CLI does (src/main.cpp:300-321)
    gpz_ok(gpz_compress(&p, x, x + n, x + 2 * n, d_out.p, cap, scr.p, scr_bytes, &r, nullptr), "gpz_compress");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  gpz_ok(gpz_compress_async(&p, x, x + n, x + 2 * n, d_out.p, cap, scr.p, scr_bytes, nullptr), "gpz_compress_async");
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  gpz_ok(gpz_result_get(scr.p, &r, nullptr), "gpz_result_get");
  Pinned h_stream(r.stream_bytes);
  cuda_ok(cudaMemcpy(h_stream.p, d_out.p, r.stream_bytes, cudaMemcpyDeviceToHost), "download");
  double eb_enc = 0.0;
  uint32_t d2, b2, s2;
  uint64_t n2;
  gpz_ok(gpz_parse_header(h_stream.p, r.stream_bytes, &d2, &n2, &b2, &eb_enc, &s2), "gpz_parse_header");
  printf("Strict bound: encoded with eb %.10g (stated %.10g)\n", eb_enc, (double)(T)bound);
  write_file(out, h_stream.p, r.stream_bytes);
  CudaConfig cfg(r.seg_size, r.adjusted != 0, dim, n, mode, (float)bound, (float)input_bound, p.float_bits);
  print_compression_result(r.stream_bytes, n * dim * sizeof(T), 1024.0 * 1024.0 * 1024.0, ms, cfg);
  (void)aos;
  (void)d_aos;
  return 0;
}

template <typename T>
int run_compress(const char *in, const char *out, uint64_t n, uint32_t dim, const std::string &mode, double bound,
                 uint32_t seg, const std::string &nvcomp_type, bool strict) {
  const uint64_t aos_bytes = n * dim * sizeof(T), xyz_bytes = 3 * n * sizeof(T);
  check_points_file<T>(in, n, dim);
  Pinned aos(aos_bytes);
  load_points<T>(in, n, dim, aos);
  printf("Successfully read %ld points, %.03f MB from %s\n", (long)n, n * dim * sizeof(T) / 1024.0 / 1024.0, in);
  Device d_aos(aos_bytes), d_xyz(xyz_bytes), d_comp(4 * n * sizeof(T));
  upload_soa<T>(aos, d_aos, d_xyz.p, n, dim);
  const double input_bound = bound;
  if (mode == "rel") {
    // findMinimumValues + convertRelEb (include/utils.cuh:44-65, src/main.cpp:35-55)
    Device scratch(gpz_compress_scratch_bytes(0));
    const T *x = static_cast<const T *>(d_xyz.p);
    double mm[6];
    gpz_ok(gpz_rel_to_abs(sizeof(T) * 8, dim, n, x, x + n, x + 2 * n, bound, scratch.p,
                          gpz_compress_scratch_bytes(0), &bound, mm, nullptr),
           "gpz_rel_to_abs");
    const T m[6] = {(T)mm[0], (T)mm[1], (T)mm[2], (T)mm[3], (T)mm[4], (T)mm[5]};
    printf("min_max_values: %.10g %.10g %.10g %.10g %.10g %.10g\n", (double)m[0], (double)m[1], (double)m[2],
           (double)m[3], (double)m[4], (double)m[5]);
    const T range = std::fmax(std::fmax(m[3] - m[0], m[4] - m[1]), m[5] - m[2]);
    printf("Max Range is: %.10g\n", (double)range);
    printf("Abs Error bound: %.10g\n", (double)(T)bound);
  }
  if (strict) return run_compress_strict<T>(aos, d_aos, d_xyz, out, n, dim, mode, bound, input_bound, seg);
  ICudaCompressor *codec;
  if (sizeof(T) == 4)
    codec = new CudaWarpCompress(CudaConfig(seg, false, dim, n, mode, (float)bound, (float)input_bound, 32u));
  else
    codec = new CudaWarpCompressDouble(CudaConfig(seg, false, dim, n, mode, bound, input_bound, 64u));
  CompressorManager mgr;
  uint64_t comp_size = 0;
  for (int i = 0; i < 5; ++i) {  // warm up (src/main.cpp:300-321)
    uint64_t dummy = 0;
    upload_soa<T>(aos, d_aos, d_xyz.p, n, dim);
    mgr.compressWarp(d_xyz.p, static_cast<unsigned char *>(d_comp.p), &dummy, nvcomp_type, codec);
  }
  upload_soa<T>(aos, d_aos, d_xyz.p, n, dim);
  cuda_ok(cudaDeviceSynchronize(), "sync");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  mgr.compressWarp(d_xyz.p, static_cast<unsigned char *>(d_comp.p), &comp_size, nvcomp_type, codec);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  Pinned h_stream(comp_size);
  cuda_ok(cudaMemcpy(h_stream.p, d_xyz.p, comp_size, cudaMemcpyDeviceToHost), "download");
  write_file(out, h_stream.p, comp_size);
  print_compression_result(comp_size, n * dim * sizeof(T), 1024.0 * 1024.0 * 1024.0, ms, codec->getConfig());
  delete codec;
  return 0;
}

template <typename T>
int run_decompress(const std::vector<unsigned char> &h_stream, uint64_t data_size, uint64_t n, uint32_t dim,
                   double preload_ms, const char *out, const char *original, const std::string &nvcomp_type) {
  const uint64_t one = n * sizeof(T);
  Device d_stream(std::max<uint64_t>(data_size, 2 * one)), d_out(3 * one), d_aos(dim * one);
  ICudaCompressor *codec;
  if (sizeof(T) == 4) codec = new CudaWarpCompress();
  else codec = new CudaWarpCompressDouble();
  CompressorManager mgr;
  T *x = static_cast<T *>(d_out.p);
  for (int i = 0; i < 5; ++i) {  // warm up (src/main.cpp:437-451)
    cuda_ok(cudaMemcpy(d_stream.p, h_stream.data(), data_size, cudaMemcpyHostToDevice), "upload");
    mgr.decompressWarp(x, x + n, x + 2 * n, static_cast<unsigned char *>(d_stream.p), codec, nvcomp_type);
  }
  cuda_ok(cudaMemcpy(d_stream.p, h_stream.data(), data_size, cudaMemcpyHostToDevice), "upload");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  mgr.decompressWarp(x, x + n, x + 2 * n, static_cast<unsigned char *>(d_stream.p), codec, nvcomp_type);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  // SoA -> AoS on the GPU, then one copy (write_xyz_to_aos_file, include/utils.cuh:146-176)
  gpz_ok(gpz_soa_to_aos(sizeof(T) * 8, dim, n, x, x + n, x + 2 * n, d_aos.p, nullptr), "gpz_soa_to_aos");
  Pinned h_aos(dim * one);
  cuda_ok(cudaMemcpy(h_aos.p, d_aos.p, dim * one, cudaMemcpyDeviceToHost), "download");
  write_file(out, h_aos.p, dim * one);
  print_decompression_result(n, preload_ms + ms, dim);
  if (original && *original) {
    double eb = 0.0;
    if (sizeof(T) == 4) {
      float f;
      memcpy(&f, h_stream.data() + 16, 4);
      eb = f;
    } else {
      memcpy(&eb, h_stream.data() + 16, 8);
    }
    printf("Verification error bound: %.10g\n", eb);
    verify<T>(x, original, n, dim, eb);
  }
  delete codec;
  return 0;
}

}  // namespace

int main(int argc, char *argv[]) {
  const char *filename = nullptr, *output_filename = nullptr, *recon_filename = nullptr, *original_filename = nullptr;
  uint64_t num_points = 0;
  uint32_t float_bits = 0, dim = 3, segment_size = 0;
  double error_bound = 0.0;
  std::string err_mode, nvcomp_type = "none";
  bool compress_mode = false, decompress_mode = false, verification_mode = false, strict = false;
  int opt;
  try {
    while ((opt = getopt(argc, argv, "xdi:o:p:n:e:s:m:f:t:r:v:hB")) != -1) {
      switch (opt) {
        case 'x': compress_mode = true; break;
        case 'd': decompress_mode = true; break;
        case 'i': filename = optarg; break;
        case 'o': output_filename = optarg; break;
        case 'p': dim = (uint32_t)std::stoul(optarg); break;
        case 'n': num_points = std::stoull(optarg); break;
        case 'e': error_bound = std::stod(optarg); break;
        case 's': segment_size = (uint32_t)std::stoul(optarg); break;
        case 'm': err_mode = optarg; break;
        case 'f': float_bits = (uint32_t)std::stoul(optarg); break;
        case 't': nvcomp_type = optarg; break;
        case 'r': recon_filename = optarg; break;
        case 'v': verification_mode = true; original_filename = optarg; break;
        case 'B': strict = true; break;
        case 'h':
        default: print_usage(argv[0]); return 1;
      }
    }
  } catch (const std::exception &) {
    print_usage(argv[0]);
    return 1;
  }
  if (compress_mode && decompress_mode) {
    std::cerr << "Error: Cannot specify both -x (compress) and -d (decompress)\n";
    return 1;
  }
  if (!compress_mode && !decompress_mode) {
    std::cerr << "Error: Must specify either -x (compress) or -d (decompress)\n";
    print_usage(argv[0]);
    return 1;
  }
  if (compress_mode) {
    if (!filename || !output_filename || num_points == 0 || err_mode.empty()) {
      std::cerr << "Error: Missing required arguments for compression\n";
      print_usage(argv[0]);
      return 1;
    }
    if (dim != 2 && dim != 3) {
      std::cerr << "Error: Dimension must be 2 or 3\n";
      print_usage(argv[0]);
      return 1;
    }
    if (float_bits != 32 && float_bits != 64) {
      std::cerr << "Error: Float bits must be 32 or 64\n";
      print_usage(argv[0]);
      return 1;
    }
    if (nvcomp_type != "none" && !nvcomp_type.empty()) {
      std::cerr << "Error: -t option requires nvcomp support. Rebuild with -DNVCOMP_DIR=<path> to enable.\n";
      return 1;
    }
  }
  if (decompress_mode) {
    if (!recon_filename || !output_filename) {
      std::cerr << "Error: -i and -o are required for decompression\n";
      print_usage(argv[0]);
      return 1;
    }
    if (verification_mode && !original_filename) {
      std::cerr << "Error: -v requires an original file name\n";
      print_usage(argv[0]);
      return 1;
    }
    if (nvcomp_type != "none" && !nvcomp_type.empty()) {
      std::cerr << "Error: -t option requires nvcomp support. Rebuild with -DNVCOMP_DIR=<path> to enable.\n";
      return 1;
    }
  }
  try {
    if (compress_mode) {
      return float_bits == 32
                 ? run_compress<float>(filename, output_filename, num_points, dim, err_mode, error_bound, segment_size,
                                       nvcomp_type, strict)
                 : run_compress<double>(filename, output_filename, num_points, dim, err_mode, error_bound,
                                        segment_size, nvcomp_type, strict);
    }
    // decompress: -o is the compressed input, -r the reconstructed output (src/main.cpp:378-390)
    uint64_t data_size = 0;
    std::vector<unsigned char> h_stream = read_file(output_filename, &data_size);
    printf("Compressed file loaded, data size %f MB\n", data_size / 1024.0 / 1024.0);
    const auto t0 = std::chrono::steady_clock::now();
    uint32_t sdim = 0, sbits = 0;
    uint64_t n = 0;
    if (data_size < 24) throw std::runtime_error("compressed file too short");
    CompressorManager mgr;
    mgr.decompressLoadParas(&sdim, &n, &sbits, nvcomp_type, num_points, dim, float_bits, h_stream.data());
    printf("Decompressed num points: %zu\n", (size_t)n);
    const double preload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (sbits == 32)
      return run_decompress<float>(h_stream, data_size, n, sdim, preload_ms, recon_filename, original_filename,
                                   nvcomp_type);
    if (sbits == 64)
      return run_decompress<double>(h_stream, data_size, n, sdim, preload_ms, recon_filename, original_filename,
                                    nvcomp_type);
    throw std::runtime_error("compressed file has an unknown float width");
  } catch (const std::exception &e) {
    std::cerr << "Error: " << e.what() << "\n";
    return 1;
  }
}
