// ICudaCompressor.cuh -- the codec interface of the GPZ reference
// (include/ICudaCompressor.cuh:6-17), same signatures.
//
//   compress(d_xyz, comp_data, comp_data_size, comp_type)
//     d_xyz      device SoA input x[N] y[N] z[N] (3*N values of the stream's
//                float type, also for 2D); overwritten with the compressed stream
//     comp_data  device scratch of at least 4*N*sizeof(T) bytes
//     comp_data_size  receives the stream size in bytes
//     comp_type  "none" (or empty); other values are nvcomp back-ends, not built
//   decompress(x, y, z, d_compressed_data, nvcomp_type)
//     x, y, z    device SoA outputs of N values each (z unused for 2D)
//     d_compressed_data  device copy of the stream
//
// The reference reports failures with exit(); the B200 classes throw
// std::runtime_error instead (the gpz CLI turns that into exit status 1).
#ifndef GPZ_B200_ICUDA_COMPRESSOR_H
#define GPZ_B200_ICUDA_COMPRESSOR_H

#include <cstdint>
#include <string>
#include "cudaCompress.cuh"

class ICudaCompressor {
 public:
  virtual ~ICudaCompressor() = default;
  virtual void compress(void *d_xyz, unsigned char *comp_data, uint64_t *comp_data_size,
                        const std::string &comp_type) = 0;
  virtual void decompress(void *decData_x, void *decData_y, void *decData_z, unsigned char *d_compressed_data,
                          const std::string &nvcomp_type) = 0;
  virtual const CudaConfig &getConfig() const = 0;
};

#endif
