// CompressorManager.h -- dispatch helper of the GPZ reference
// (include/CompressorManager.h:16-25, src/CompressorManager.cpp), same
// signatures.
#ifndef GPZ_B200_COMPRESSOR_MANAGER_H
#define GPZ_B200_COMPRESSOR_MANAGER_H

#include <cstdint>
#include <string>
#include "cudaCompress.cuh"
#include "cudaWarpCompress.cuh"
#include "cudaWarpCompressDouble.cuh"

class CompressorManager {
 public:
  CompressorManager();
  ~CompressorManager();

  void compressWarp(void *d_xyz, unsigned char *d_comp_data, uint64_t *comp_size, std::string nvcomp_type,
                    ICudaCompressor *compressor);

  // Reads dim, point count and float width from the host copy of a stream's
  // header; with an nvcomp type the caller's values are taken instead.
  void decompressLoadParas(uint32_t *dim, uint64_t *numPoints, uint32_t *float_bits, const std::string &nvcomp_type,
                           uint64_t nvcomp_num, uint32_t nvcomp_dim, uint32_t float_bits_num,
                           unsigned char *h_compressed_data);

  void decompressWarp(void *d_dec_data_x, void *d_dec_data_y, void *d_dec_data_z, unsigned char *d_compressed_data,
                      ICudaCompressor *decompressor, const std::string &nvcomp_type);
};

#endif
