// gpz_plugin.cu -- the reference's C++ codec classes (CudaWarpCompress,
// CudaWarpCompressDouble, CompressorManager; include/gpz/) on top of the C ABI
// of include/gpz_b200.h.
//
// Reference behaviour kept: synchronous calls on the legacy default stream;
// compress reads SoA x[N] y[N] z[N] from d_xyz and overwrites d_xyz with the
// stream (src/cudaWarpCompress.cu:1669, read back at src/main.cpp:348), uses
// comp_data (>= 4*N*sizeof(T) bytes, src/main.cpp:289-291) as its working
// buffer, and records the chosen segment size in the object's CudaConfig
// (src/cudaWarpCompress.cu:1513-1554).  Changed: failures throw
// std::runtime_error instead of calling exit().

#include <cstring>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "gpz_b200.h"
#include "../../include/gpz/CompressorManager.h"

namespace {

const char *status_name(int rc) {
  switch (rc) {
    case GPZ_OK: return "ok";
    case GPZ_EINVAL: return "invalid argument";
    case GPZ_ESEG: return "automatic segment size would exceed 1024";
    case GPZ_ESTREAM: return "malformed compressed stream";
    case GPZ_ENOSPACE: return "buffer too small";
    case GPZ_ECUDA: return "CUDA runtime error";
    case GPZ_ETIMEOUT: return "device-side wait timed out";
    case GPZ_ENOTSUP: return "not supported in this build";
    case GPZ_ELIMIT: return "input too large";
    default: return "unknown error";
  }
}

void check(int rc, const char *what) {
  if (rc != GPZ_OK) throw std::runtime_error(std::string(what) + ": " + status_name(rc));
}

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void check_codec_type(const std::string &type) {
  // nvcomp back-ends (src/cudaWarpCompress.cu:1603-1617) are not built
  if (!type.empty() && type != "none") check(GPZ_ENOTSUP, ("compression type " + type).c_str());
}

template <typename T>
void compress_inplace(CudaConfig &cfg, void *d_xyz, unsigned char *comp_data, uint64_t *comp_data_size,
                      const std::string &comp_type) {
  check_codec_type(comp_type);
  if (!d_xyz || !comp_data || !comp_data_size) check(GPZ_EINVAL, "compress");
  constexpr bool is32 = sizeof(T) == 4;
  const uint64_t n = cfg.coordinate_num;
  gpz_params p;
  memset(&p, 0, sizeof(p));
  p.float_bits = is32 ? 32 : 64;
  p.dim = cfg.dim;
  p.n = n;
  p.eb = is32 ? (double)cfg.eb : cfg.eb_dbl;
  p.rel_eb = is32 ? (double)cfg.rel_eb : cfg.rel_eb_dbl;
  p.rel_mode = cfg.error_mode == "rel" ? 1 : 0;
  p.seg_size = cfg.seg_size;
  const T *x = static_cast<const T *>(d_xyz);
  // The stream goes to the head of comp_data and the scratch control block to
  // its tail; tiny inputs whose 4*N*sizeof(T) bytes cannot hold both use a
  // temporary allocation instead.
  const uint64_t work = 4ull * n * sizeof(T);
  const uint64_t need = gpz_compress_scratch_bytes(n);
  const uint64_t bound = gpz_stream_bound(n, p.dim, p.float_bits);
  uint8_t *out = comp_data, *scratch = nullptr, *tmp = nullptr;
  uint64_t out_cap = 0;
  if (work >= bound + need + 256) {
    scratch = comp_data + ((work - need) & ~255ull);
    out_cap = (uint64_t)(scratch - comp_data);
  } else {
    check_cuda(cudaMalloc(&tmp, bound + need + 256), "compress: temporary buffer");
    out = tmp;
    scratch = tmp + ((bound + 255) & ~255ull);
    out_cap = bound;
  }
  gpz_result r;
  const int rc = gpz_compress(&p, x, x + n, x + 2 * n, out, out_cap, scratch, need, &r, nullptr);
  if (rc == GPZ_OK) {
    check_cuda(cudaMemcpy(d_xyz, out, r.stream_bytes, cudaMemcpyDeviceToDevice), "compress: stream copy");
    *comp_data_size = r.stream_bytes;
    cfg.seg_size = r.seg_size;
    cfg.adjusted_seg = r.adjusted != 0;
  }
  if (tmp) cudaFree(tmp);
  check(rc, "compress");
}

template <typename T>
void decompress_into(CudaConfig &cfg, void **d_small, void *x, void *y, void *z, unsigned char *d_stream,
                     const std::string &nvcomp_type) {
  check_codec_type(nvcomp_type);
  if (!x || !y || !d_stream) check(GPZ_EINVAL, "decompress");
  uint8_t h[32];
  check_cuda(cudaMemcpy(h, d_stream, sizeof(h), cudaMemcpyDeviceToHost), "decompress: header");
  uint32_t dim = 0, bits = 0, seg = 0;
  uint64_t n = 0;
  double eb = 0.0;
  check(gpz_parse_header(h, sizeof(h), &dim, &n, &bits, &eb, &seg), "decompress: header");
  if (bits != sizeof(T) * 8) check(GPZ_EINVAL, "decompress: stream float width differs from the codec's");
  if (dim == 3 && !z) check(GPZ_EINVAL, "decompress");
  // The caller passes no size (include/ICudaCompressor.cuh:13-14): the
  // stream's own size fields bound it, everything else is validated on the device.
  uint64_t bytes = 0;
  check(gpz_stream_size(d_stream, UINT64_MAX, &bytes, nullptr), "decompress: stream size");
  if (!*d_small) check_cuda(cudaMalloc(d_small, gpz_decompress_scratch_bytes()), "decompress: scratch");
  gpz_result r;
  check(gpz_decompress(d_stream, bytes, bits, dim, x, y, z, n, *d_small, gpz_decompress_scratch_bytes(), &r,
                       nullptr),
        "decompress");
  cfg.dim = dim;
  cfg.coordinate_num = n;
  cfg.seg_size = seg;
  cfg.float_bits = bits;
  if (bits == 32) cfg.eb = (float)eb;
  else cfg.eb_dbl = eb;
}

}  // namespace

CudaWarpCompress::CudaWarpCompress(CudaConfig cuda_config_) : cuda_config(std::move(cuda_config_)) {}
CudaWarpCompress::CudaWarpCompress() { cuda_config.float_bits = 32; }
CudaWarpCompress::~CudaWarpCompress() {
  if (d_small_) cudaFree(d_small_);
}
void CudaWarpCompress::compress(void *d_xyz, unsigned char *comp_data, uint64_t *comp_data_size,
                                const std::string &comp_type) {
  compress_inplace<float>(cuda_config, d_xyz, comp_data, comp_data_size, comp_type);
}
void CudaWarpCompress::decompress(void *x, void *y, void *z, unsigned char *d_compressed_data,
                                  const std::string &nvcomp_type) {
  decompress_into<float>(cuda_config, &d_small_, x, y, z, d_compressed_data, nvcomp_type);
}

CudaWarpCompressDouble::CudaWarpCompressDouble(CudaConfig cuda_config_) : cuda_config(std::move(cuda_config_)) {}
CudaWarpCompressDouble::CudaWarpCompressDouble() { cuda_config.float_bits = 64; }
CudaWarpCompressDouble::~CudaWarpCompressDouble() {
  if (d_small_) cudaFree(d_small_);
}
void CudaWarpCompressDouble::compress(void *d_xyz, unsigned char *comp_data, uint64_t *comp_data_size,
                                      const std::string &comp_type) {
  compress_inplace<double>(cuda_config, d_xyz, comp_data, comp_data_size, comp_type);
}
void CudaWarpCompressDouble::decompress(void *x, void *y, void *z, unsigned char *d_compressed_data,
                                        const std::string &nvcomp_type) {
  decompress_into<double>(cuda_config, &d_small_, x, y, z, d_compressed_data, nvcomp_type);
}

CompressorManager::CompressorManager() = default;
CompressorManager::~CompressorManager() = default;

void CompressorManager::compressWarp(void *d_xyz, unsigned char *d_comp_data, uint64_t *comp_size,
                                     std::string nvcomp_type, ICudaCompressor *compressor) {
  compressor->compress(d_xyz, d_comp_data, comp_size, nvcomp_type);
}

void CompressorManager::decompressWarp(void *d_dec_data_x, void *d_dec_data_y, void *d_dec_data_z,
                                       unsigned char *d_compressed_data, ICudaCompressor *decompressor,
                                       const std::string &nvcomp_type) {
  decompressor->decompress(d_dec_data_x, d_dec_data_y, d_dec_data_z, d_compressed_data, nvcomp_type);
}

void CompressorManager::decompressLoadParas(uint32_t *dim, uint64_t *numPoints, uint32_t *float_bits,
                                            const std::string &nvcomp_type, uint64_t nvcomp_num, uint32_t nvcomp_dim,
                                            uint32_t float_bits_num, unsigned char *h_compressed_data) {
  if (!nvcomp_type.empty() && nvcomp_type != "none") {
    *dim = nvcomp_dim;
    *float_bits = float_bits_num;
    *numPoints = nvcomp_num;
    return;
  }
  // header fields: u32 dim @0, u64 N @4, u32 float bits @12
  memcpy(dim, h_compressed_data, 4);
  memcpy(numPoints, h_compressed_data + 4, 8);
  memcpy(float_bits, h_compressed_data + 12, 4);
}
