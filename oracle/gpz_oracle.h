/*
 * gpz_oracle.h -- CPU restatement of GPZ's compress / decompress path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA implementation in gpz_b200/ and the timed CPU baseline; the product
 * never links, loads or calls it.  Every function cites the reference
 * source (path:line within the GPZ project) whose arithmetic it restates.
 *
 * Parity is pinned against byte streams produced by the reference's own
 * CUDA build (oracle/ref_harness.cu, fixtures under tests/golden/).
 */
#ifndef GPZ_ORACLE_H
#define GPZ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (shared meaning with include/gpz_b200.h). */
#define GPZO_OK 0
#define GPZO_EINVAL 1
#define GPZO_ESEG 2       /* auto segment size exceeded 1024 (reference exits) */
#define GPZO_ESTREAM 3    /* malformed / truncated stream */
#define GPZO_ENOMEM 4

/* Upper bound of the compressed stream size for N points (any data). */
uint64_t gpzo_stream_bound(uint64_t n, uint32_t dim, uint32_t float_bits);

/* Relative -> absolute error bound exactly as the CLI computes it on the host
 * (findMinimumValues<T>, include/utils.cuh:44-65; convertRelEb<T>,
 * src/main.cpp:35-55 with the casts at src/main.cpp:254,263).
 * z may be NULL for 2D data (the CLI fills z with zeros, utils.cuh:141). */
float gpzo_rel_to_abs_f32(const float *x, const float *y, const float *z,
                          uint64_t n, float rel);
double gpzo_rel_to_abs_f64(const double *x, const double *y, const double *z,
                           uint64_t n, double rel);

/* computeSegSize (src/cudaWarpCompress.cu:1424-1557 / double twin
 * src/cudaWarpCompressDouble.cu:1426-1555).  seg_in is the configured
 * segment size (0 = auto); rel_mode is error_mode=="rel".  On return
 * *seg_out / *adjusted hold the mutated CudaConfig fields.  safe31 != 0
 * selects the extension mode that also doubles seg until every block id
 * fits in 31 bits (not in the reference; off for parity).  Returns
 * GPZO_ESEG where the reference calls exit(1). */
int gpzo_seg_size_f32(const float *x, const float *y, const float *z,
                      uint64_t n, uint32_t dim, uint32_t seg_in, int rel_mode,
                      float rel_eb, float eb, int safe31,
                      uint32_t *seg_out, int *adjusted);
int gpzo_seg_size_f64(const double *x, const double *y, const double *z,
                      uint64_t n, uint32_t dim, uint32_t seg_in, int rel_mode,
                      double rel_eb, double eb, int safe31,
                      uint32_t *seg_out, int *adjusted);

/* Full compress of SoA input into a GPZ stream (header, offset table,
 * meta records, payload) with an already-resolved segment size.
 * Restates runCompressKernel[2D] (src/cudaWarpCompress.cu:58-796),
 * the CUB exclusive scan + header assembly + compaction
 * (src/cudaWarpCompress.cu:1620-1702) and the float64 twins.
 * Padding bytes between sections are written as zero.
 * out must hold gpzo_stream_bound() bytes.  nthreads <= 0 = OpenMP default. */
int gpzo_compress_f32(const float *x, const float *y, const float *z,
                      uint64_t n, uint32_t dim, float eb, uint32_t seg,
                      uint8_t *out, uint64_t *out_bytes, int nthreads);
int gpzo_compress_f64(const double *x, const double *y, const double *z,
                      uint64_t n, uint32_t dim, double eb, uint32_t seg,
                      uint8_t *out, uint64_t *out_bytes, int nthreads);

/* Decompress a GPZ stream into SoA output (points in sorted order within
 * each 1024-point chunk).  Restates runDecompressKernel[2D]
 * (src/cudaWarpCompress.cu:798-1214) and decompressImpl (:1743-1856),
 * without the reference's out-of-bounds write at unique_num==1024.
 * z may be NULL for 2D streams. */
int gpzo_decompress_f32(const uint8_t *stream, uint64_t bytes,
                        float *x, float *y, float *z, uint64_t cap_points,
                        int nthreads);
int gpzo_decompress_f64(const uint8_t *stream, uint64_t bytes,
                        double *x, double *y, double *z, uint64_t cap_points,
                        int nthreads);

/* Header parse (CompressorManager::decompressLoadParas,
 * src/CompressorManager.cpp:24-34, plus eb / seg at :16/:20 or :16/:24). */
int gpzo_parse_header(const uint8_t *stream, uint64_t bytes, uint32_t *dim,
                      uint64_t *n, uint32_t *float_bits, double *eb,
                      uint32_t *seg);

/* Per-point order: perm[j] = input index of the point that decompresses to
 * output slot j (stable sort by block id within each chunk, tie order of
 * the reference's cub::BlockRadixSort over its striped load).  For tests. */
int gpzo_permutation_f32(const float *x, const float *y, const float *z,
                         uint64_t n, uint32_t dim, float eb, uint32_t seg,
                         uint64_t *perm);
int gpzo_permutation_f64(const double *x, const double *y, const double *z,
                         uint64_t n, uint32_t dim, double eb, uint32_t seg,
                         uint64_t *perm);

/* Padding mask: mask[i] = 1 where stream byte i is section padding that
 * the reference never writes (its value there is stale scratch). */
int gpzo_padding_mask(const uint8_t *stream, uint64_t bytes, uint8_t *mask);

/* Deterministic synthetic generators (splitmix64 based), shared by the
 * reference harness and the tests.  kind: 0 = uniform box [lo, hi)^dim,
 * 1 = Gaussian clusters + uniform background, shuffled (lo..hi box),
 * 2 = lattice with Gaussian jitter (FCC for dim 3, square for dim 2),
 *     spacing 1, jitter sigma = hi, random permutation.
 * For dim 2 z is left untouched (may be NULL). */
void gpzo_generate_f32(int kind, uint64_t n, uint32_t dim, double lo,
                       double hi, uint64_t seed, float *x, float *y, float *z);
void gpzo_generate_f64(int kind, uint64_t n, uint32_t dim, double lo,
                       double hi, uint64_t seed, double *x, double *y,
                       double *z);

#ifdef __cplusplus
}
#endif

#endif
