// cudaCompress.cuh -- CudaConfig, as declared by the GPZ reference
// (include/cudaCompress.cuh:16-40): same fields, constructors and meaning, so
// code written against the reference compiles unchanged.  Implemented by the
// B200 library (gpz_b200/csrc/gpz_plugin.cu) on top of include/gpz_b200.h.
#ifndef GPZ_B200_CUDA_COMPRESS_H
#define GPZ_B200_CUDA_COMPRESS_H

#include <cstdint>
#include <string>
#include <utility>

// Points per compressed chunk (the stream format's chunk size).
const int ELEMS_PER_BLOCK = 1024;

class CudaConfig {
 public:
  uint32_t seg_size;        // 0 = choose automatically (rel mode); set by compress
  bool adjusted_seg;        // set by compress when the segment size was doubled
  uint32_t dim;             // 2 or 3
  uint64_t coordinate_num;  // number of points
  float eb;                 // absolute error bound (float streams)
  float rel_eb;             // relative bound as given (float streams; auto-seg rule only)
  double eb_dbl;            // absolute error bound (double streams)
  double rel_eb_dbl;        // relative bound as given (double streams)
  std::string error_mode;   // "rel" or "abs"
  uint32_t float_bits;      // 32 or 64

  CudaConfig()
      : seg_size(0), adjusted_seg(false), dim(3), coordinate_num(0), eb(0.0f), rel_eb(0.0f), eb_dbl(0.0),
        rel_eb_dbl(0.0), float_bits(32) {}

  CudaConfig(uint32_t seg_size_, bool adjusted_seg_, uint32_t dim_, uint64_t coordinate_num_, std::string error_mode_,
             float eb_, float rel_eb_, uint32_t float_bits_)
      : seg_size(seg_size_), adjusted_seg(adjusted_seg_), dim(dim_), coordinate_num(coordinate_num_), eb(eb_),
        rel_eb(rel_eb_), eb_dbl(0.0), rel_eb_dbl(0.0), error_mode(std::move(error_mode_)), float_bits(float_bits_) {}

  CudaConfig(uint32_t seg_size_, bool adjusted_seg_, uint32_t dim_, uint64_t coordinate_num_, std::string error_mode_,
             double eb_, double rel_eb_, uint32_t float_bits_)
      : seg_size(seg_size_), adjusted_seg(adjusted_seg_), dim(dim_), coordinate_num(coordinate_num_), eb(0.0f),
        rel_eb(0.0f), eb_dbl(eb_), rel_eb_dbl(rel_eb_), error_mode(std::move(error_mode_)), float_bits(float_bits_) {}
};

#endif
