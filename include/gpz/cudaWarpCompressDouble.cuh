// cudaWarpCompressDouble.cuh -- the double codec class of the GPZ reference (include/cudaWarpCompressDouble.cuh:11-39),
// same public interface, implemented on the B200 library (include/gpz_b200.h).
// Synchronous on the legacy default stream, like the reference; compress
// records the chosen segment size in the object's CudaConfig.
#ifndef GPZ_B200_CUDAWARPCOMPRESSDOUBLE_H
#define GPZ_B200_CUDAWARPCOMPRESSDOUBLE_H

#include "ICudaCompressor.cuh"

class CudaWarpCompressDouble : public ICudaCompressor {
 public:
  explicit CudaWarpCompressDouble(CudaConfig cuda_config);
  CudaWarpCompressDouble();
  ~CudaWarpCompressDouble() override;

  void compress(void *d_xyz, unsigned char *comp_data, uint64_t *comp_data_size,
                const std::string &comp_type) override;
  void decompress(void *decData_x, void *decData_y, void *decData_z, unsigned char *d_compressed_data,
                  const std::string &nvcomp_type) override;
  const CudaConfig &getConfig() const override { return cuda_config; }

 private:
  CudaConfig cuda_config;
  void *d_small_ = nullptr;  // decompress scratch (control block), allocated on first use
};

#endif
