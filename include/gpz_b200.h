/*
 * gpz_b200.h -- C ABI of the B200-native GPZ particle compressor.
 *
 * Plain C: pointers, sizes and status codes only.  Device pointers are CUDA
 * global-memory addresses on the current device; `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Every entry point returns
 * GPZ_OK (0) or one of the GPZ_E* codes below and never exits the process.
 *
 * The compressed stream is byte-compatible with the GPZ reference format:
 * header, per-chunk offset table, per-chunk meta records and bit-plane
 * payloads for 1024-point chunks (reference src/cudaWarpCompress.cu:1668-1702,
 * src/cudaWarpCompressDouble.cu:1670-1702).
 *
 * Each entry point names the reference interface it replaces (path:line in
 * the GPZ project).  The C++ drop-in classes with the reference's own names
 * (ICudaCompressor, CudaWarpCompress, CudaWarpCompressDouble,
 * CompressorManager, CudaConfig) are declared in include/gpz/ and sit on top
 * of this ABI.
 */
#ifndef GPZ_B200_H
#define GPZ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define GPZ_OK 0
#define GPZ_EINVAL 1      /* bad argument (null pointer, dim, float_bits, seg 0 in abs mode ...) */
#define GPZ_ESEG 2        /* auto segment size would exceed 1024 (reference: exit(1),
                             src/cudaWarpCompress.cu:1547-1550) */
#define GPZ_ESTREAM 3     /* malformed or truncated compressed stream */
#define GPZ_ENOSPACE 4    /* output or scratch buffer too small */
#define GPZ_ECUDA 5       /* a CUDA runtime call failed */
#define GPZ_ETIMEOUT 6    /* a bounded device-side wait gave up (kernel returned early) */
#define GPZ_ENOTSUP 7     /* feature not compiled in (e.g. nvcomp back-ends) */
#define GPZ_ELIMIT 8      /* input larger than the fixed scratch of gpz_compress_noalloc */

/* ---- parameters ------------------------------------------------------------
 * Mirrors CudaConfig (reference include/cudaCompress.cuh:16-40). */
typedef struct gpz_params {
  uint32_t float_bits; /* 32 or 64 (CudaConfig::float_bits) */
  uint32_t dim;        /* 2 or 3 (CudaConfig::dim) */
  uint64_t n;          /* number of points (CudaConfig::coordinate_num) */
  double eb;           /* absolute error bound; rounded to float when float_bits == 32
                          (CudaConfig::eb / eb_dbl) */
  double rel_eb;       /* relative bound as given by the user; only read by the automatic
                          segment-size rule (CudaConfig::rel_eb / rel_eb_dbl) */
  int32_t rel_mode;    /* 1 when error_mode == "rel" (CudaConfig::error_mode) */
  uint32_t seg_size;   /* 0 = automatic (CudaConfig::seg_size) */
  uint32_t flags;      /* GPZ_FLAG_* */
  uint32_t reserved;
} gpz_params;

/* Extension (not in the reference): also double the segment size until every
 * block id fits in 31 bits, so the reference's 0x7FFFFFFF mask
 * (src/cudaWarpCompress.cu:187-189) never truncates an id.  Streams stay in
 * the reference format but differ from the reference's bytes when it fires. */
#define GPZ_FLAG_SAFE31 1u

/* Extension (not in the reference): use seg_size exactly as given -- no
 * sampling, no automatic choice, no doubling.  Used by the sharded compress,
 * where every shard must encode with the segment size decided once for the
 * whole array (gpz_sample_minmax + gpz_decide_seg); seg_size must not be 0. */
#define GPZ_FLAG_SEG_FIXED 2u

/* Extension (not in the reference): hold the stated bound for every finite
 * point.  The reference reconstructs v = min + (2q+1)*eb in the float type
 * (src/cudaWarpCompress.cu:971-1007), so its rounding can put a point a few
 * ulps past eb; its verifier hides that with a 1.01*eb slack
 * (src/utils.cu:28).  With this flag the codec finds the snapshot's largest
 * coordinate magnitude M and largest per-axis range R on the device and
 * encodes with
 *   eb' = eb - u*(3*R + 2*M + 4*eb)   (u = 2^-24 for float, 2^-53 for double),
 * rounded down, which bounds every rounding of quantization and
 * reconstruction (gpz_strict_bound computes the same value on the host).
 * The header carries eb'; the stream stays in the reference format (any GPZ
 * decoder reads it) but its bytes differ from the reference's.  Implies
 * GPZ_FLAG_SAFE31.  GPZ_EINVAL (device status) when eb' would not be
 * positive.  Costs one extra pass over the input.  gpz_compress and
 * gpz_compress_async only (the batched and served forms ignore it). */
#define GPZ_FLAG_STRICT_BOUND 8u

/* Result of a compress / decompress call, read back from device scratch. */
typedef struct gpz_result {
  uint64_t stream_bytes; /* compressed size (compress) */
  uint32_t seg_size;     /* resolved segment size (CudaConfig::seg_size after the call) */
  uint32_t adjusted;     /* CudaConfig::adjusted_seg after the call */
  int32_t status;        /* GPZ_OK or device-side error */
  uint32_t id_overflow;  /* 1 if some block id exceeded 31 bits and was masked (reference quirk) */
} gpz_result;

/* ---- sizes ------------------------------------------------------------------ */

/* Worst-case compressed size for n points (any data). */
uint64_t gpz_stream_bound(uint64_t n, uint32_t dim, uint32_t float_bits);

/* Device scratch needed by gpz_compress_async for n points (control block
 * plus one 8-byte look-back word per 1024-point chunk).  Replaces the
 * caller-provided 4*N*sizeof(T) scratch of ICudaCompressor::compress
 * (reference include/ICudaCompressor.cuh:10-11, src/main.cpp:289-291). */
uint64_t gpz_compress_scratch_bytes(uint64_t n);

/* Device scratch needed by gpz_decompress_async. */
uint64_t gpz_decompress_scratch_bytes(void);

/* ---- compress ----------------------------------------------------------------
 * Replaces CudaWarpCompress::compress / CudaWarpCompressDouble::compress
 * (reference include/cudaWarpCompress.cuh:21-22, src/cudaWarpCompress.cu:1559-1741;
 * src/cudaWarpCompressDouble.cu:1557-1741), reached through
 * CompressorManager::compressWarp (src/CompressorManager.cpp:12-16).
 *
 * d_x, d_y, d_z: SoA coordinates (n values of float or double each; d_z is
 * ignored for dim == 2).  d_out receives the complete stream (header, offset
 * table, meta, payload); out_capacity is its size in bytes.  The inputs are
 * not modified (the reference overwrites its input with the stream; the C++
 * drop-in class keeps that behaviour).
 *
 * Enqueues everything on `stream` and returns without synchronising; host
 * argument errors are returned immediately.  Device-side results (size,
 * chosen segment size, status) land in the scratch control block and are
 * read with gpz_result_get(). */
int gpz_compress_async(const gpz_params *params, const void *d_x, const void *d_y,
                       const void *d_z, void *d_out, uint64_t out_capacity,
                       void *d_scratch, uint64_t scratch_bytes, void *stream);

/* Synchronous form: gpz_compress_async + gpz_result_get.  `result` may be NULL. */
int gpz_compress(const gpz_params *params, const void *d_x, const void *d_y, const void *d_z,
                 void *d_out, uint64_t out_capacity, void *d_scratch, uint64_t scratch_bytes,
                 gpz_result *result, void *stream);

/* ---- decompress ----------------------------------------------------------------
 * Replaces CudaWarpCompress::decompress / CudaWarpCompressDouble::decompress
 * (reference include/cudaWarpCompress.cuh:24-25, src/cudaWarpCompress.cu:1743-1856),
 * reached through CompressorManager::decompressWarp (src/CompressorManager.cpp:18-22).
 *
 * d_stream: the compressed stream on the device, stream_bytes long.
 * float_bits and dim must match the stream header (the caller reads them from
 * its host copy with gpz_parse_header, as decompressLoadParas does).  Outputs are SoA,
 * out_capacity points each; points come out in the stream's order (sorted by
 * block within each 1024-point chunk), as in the reference.  d_z is ignored
 * for 2D streams.  Header and every chunk record are validated on the device;
 * a bad chunk sets GPZ_ESTREAM and is not written. */
int gpz_decompress_async(const void *d_stream, uint64_t stream_bytes, uint32_t float_bits,
                         uint32_t dim, void *d_x, void *d_y, void *d_z, uint64_t out_capacity,
                         void *d_scratch, uint64_t scratch_bytes, void *stream);

int gpz_decompress(const void *d_stream, uint64_t stream_bytes, uint32_t float_bits, uint32_t dim,
                   void *d_x, void *d_y, void *d_z, uint64_t out_capacity, void *d_scratch,
                   uint64_t scratch_bytes, gpz_result *result, void *stream);

/* Reads the control block written by the last call that used d_scratch
 * (synchronises `stream`). */
int gpz_result_get(const void *d_scratch, gpz_result *result, void *stream);

/* Enqueues on `stream` a copy of the control block into `h_result`, which must
 * be pinned host memory the device can address (cudaHostAlloc / cudaMallocHost,
 * or registered with cudaHostRegister).  A one-thread kernel writes it, so the
 * copy does not wait behind other transfers on the copy engines; the caller
 * reads `h_result` once an event recorded after this call has completed.
 * Returns GPZ_EINVAL for pageable or device memory.  No reference counterpart:
 * the reference reads its sizes with blocking cudaMemcpy
 * (src/cudaWarpCompress.cu:1692-1702). */
int gpz_result_post(const void *d_scratch, gpz_result *h_result, void *stream);

/* ---- helpers -------------------------------------------------------------------- */

/* Host-side header parse of a stream held in host memory.
 * Replaces CompressorManager::decompressLoadParas (src/CompressorManager.cpp:24-34). */
int gpz_parse_header(const void *h_stream, uint64_t bytes, uint32_t *dim, uint64_t *n,
                     uint32_t *float_bits, double *eb, uint32_t *seg_size);

/* Relative -> absolute error bound, computed on the device from the SoA input
 * with the same arithmetic the reference CLI uses on the host
 * (findMinimumValues<T>, include/utils.cuh:44-65; convertRelEb<T>,
 * src/main.cpp:35-55).  For float_bits == 32 `rel` is rounded to float first
 * (src/main.cpp:254).  Writes the absolute bound and the six min/max values
 * (x_min, y_min, z_min, x_max, y_max, z_max; z = 0 for 2D) to host memory.
 * Synchronises `stream`.  Needs gpz_compress_scratch_bytes(0) bytes of scratch. */
int gpz_rel_to_abs(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x,
                   const void *d_y, const void *d_z, double rel, void *d_scratch,
                   uint64_t scratch_bytes, double *h_eb, double *h_minmax6, void *stream);

/* The bound GPZ_FLAG_STRICT_BOUND encodes with, for a snapshot whose largest
 * coordinate magnitude is max_abs and whose largest per-axis range
 * (max - min) is max_range.  No counterpart in the reference.  GPZ_EINVAL
 * when it would not be positive. */
int gpz_strict_bound(uint32_t float_bits, double eb, double max_abs, double max_range, double *eb_strict);

/* ---- allocation-free compress -------------------------------------------------
 * No counterpart in the reference (whose compress allocates with cudaMalloc on
 * every call, src/cudaWarpCompress.cu:1631-1663).
 *
 * For callers that cannot allocate device memory themselves -- a codec plugin
 * inside an application that owns the device-memory budget and only lends it
 * the input and output buffers, or a latency-critical path that cannot take
 * cudaMalloc's implicit device synchronisation.  Same as gpz_compress, but
 * the scratch is a 4 MiB array compiled into the library (one copy per GPU
 * that loads it, kept until the process exits), so the caller passes only
 * inputs, output and stream, and nothing is allocated.
 *
 * Limit: n <= gpz_compress_noalloc_max_points() (536,838,144 points);
 * larger inputs return GPZ_ELIMIT before anything is launched.
 * The first call on each device also looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture
 * begins.  Every call, the first included, waits for `stream` to finish,
 * because it reads the result back to the host.
 * All calls share the one array: calls that overlap on the GPU (different
 * streams, or different host threads on the same device) race and must be
 * serialised by the caller. */
uint64_t gpz_compress_noalloc_max_points(void);
int gpz_compress_noalloc(const gpz_params *params, const void *d_x, const void *d_y,
                         const void *d_z, void *d_out, uint64_t out_capacity,
                         gpz_result *result, void *stream);

/* ---- file I/O helpers -----------------------------------------------------------
 * AoS <-> SoA on the device, for the CLI's file path (the reference does this
 * with host loops, load_file_to_soa_xyz / write_xyz_to_aos_file,
 * include/utils.cuh:83-180).  d_aos holds n points of `dim` interleaved
 * values (x, y[, z]); gpz_aos_to_soa writes zeros to d_z for dim == 2, as the
 * reference loader does; gpz_soa_to_aos ignores d_z for dim == 2.
 * Enqueued on `stream`, not synchronised. */
int gpz_aos_to_soa(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_aos, void *d_x,
                   void *d_y, void *d_z, void *stream);
int gpz_soa_to_aos(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y,
                   const void *d_z, void *d_aos, void *stream);

/* ---- sharded compress ------------------------------------------------------------
 * One array compressed as shards on several GPUs (chunk-aligned ranges, each
 * encoded as an ordinary stream with the common bound and segment size and
 * stitched by offset).  No counterpart in the reference, which runs on one GPU;
 * these split its computeSegSize (src/cudaWarpCompress.cu:1424-1557) and
 * convertRelEb (src/main.cpp:35-55) into a per-shard part and a host part so
 * the shards agree bit for bit with a single-GPU run.
 *
 * gpz_sample_minmax: the shard [begin, begin + count) of an n-point array
 * (d_x.. point at element `begin`) folds its share of computeSegSize's sample
 * windows into six ordered accumulators (x min, x max, y min, y max, z min,
 * z max, as order-preserving unsigned keys with the minima complemented);
 * combining the shards' accumulators with an unsigned max gives the whole
 * array's.  Synchronises `stream`; needs gpz_decompress_scratch_bytes() of
 * scratch.
 * gpz_decide_seg: the segment-size rules on combined accumulators (host only).
 * gpz_rel_abs_from_minmax: relative -> absolute bound from the combined
 * per-axis minima and maxima of gpz_rel_to_abs (host only). */
int gpz_sample_minmax(uint32_t float_bits, uint32_t dim, uint64_t n, uint64_t begin, uint64_t count,
                      const void *d_x, const void *d_y, const void *d_z, void *d_scratch,
                      uint64_t scratch_bytes, uint64_t *h_acc6, void *stream);
int gpz_decide_seg(uint32_t float_bits, uint32_t dim, const uint64_t *acc6, uint32_t seg_in,
                   int32_t rel_mode, double rel_eb, double eb, uint32_t flags, uint32_t *seg,
                   uint32_t *adjusted);
int gpz_rel_abs_from_minmax(uint32_t float_bits, const double *minmax6, double rel, double *eb);

/* Total size in bytes of a compressed stream held on the device, from its
 * header, last offset-table entry and last meta record (three small copies;
 * synchronises `stream`).  `cap` is the number of bytes readable at
 * d_stream; GPZ_ESTREAM if the stream does not fit in it.  No counterpart in
 * the reference, whose decompress takes no size (ICudaCompressor::decompress,
 * include/ICudaCompressor.cuh:13-14); the C++ drop-in uses it to bound the
 * stream it validates. */
int gpz_stream_size(const void *d_stream, uint64_t cap, uint64_t *bytes, void *stream);

/* ---- batched compress -------------------------------------------------------------
 * No counterpart in the reference, which compresses one snapshot per call
 * (CompressorManager::compressWarp, src/CompressorManager.cpp:12-16; each call
 * samples, launches and synchronises on its own).  A batch compresses many
 * snapshots of mixed size, float width and dimension with one CUDA graph:
 * device rel->abs bounds, segment-size sampling and one persistent compress
 * kernel per (float width, dimension) class whose work list holds the 8-chunk
 * groups of all its snapshots.  Every snapshot's stream is byte-identical to
 * what gpz_compress writes for the same parameters.
 *
 * A batch is a plan bound to the buffers named in its items (like an FFT
 * plan): gpz_batch_create validates the items, allocates the batch's device
 * memory (descriptors, work maps, one control block and look-back words per
 * snapshot) and captures the graph; gpz_batch_launch replays it on a stream
 * (the inputs may change between launches, the pointers and sizes may not);
 * gpz_batch_results synchronises the stream and reads every snapshot's result.
 * Launches of one batch must not overlap on the GPU. */
typedef struct gpz_batch_item {
  uint32_t float_bits;   /* 32 or 64 */
  uint32_t dim;          /* 2 or 3 */
  uint64_t n;            /* points, >= 1 */
  const void *d_x;       /* SoA device arrays; d_z is ignored for dim == 2 */
  const void *d_y;
  const void *d_z;
  void *d_out;           /* the snapshot's stream */
  uint64_t out_capacity; /* bytes at d_out */
  double eb;             /* absolute bound (ignored with GPZ_FLAG_REL_ON_DEVICE) */
  double rel_eb;         /* relative bound: segment-size rules; with GPZ_FLAG_REL_ON_DEVICE also the bound */
  int32_t rel_mode;      /* 1: the "rel" error mode of the segment-size rules */
  uint32_t seg_size;     /* 0: automatic; see GPZ_FLAG_SEG_FIXED */
  uint32_t flags;        /* GPZ_FLAG_SAFE31 | GPZ_FLAG_SEG_FIXED | GPZ_FLAG_REL_ON_DEVICE */
  uint32_t reserved;     /* 0 */
} gpz_batch_item;

/* Batch item flag: the absolute bound is computed on the device from rel_eb
 * exactly as gpz_rel_to_abs computes it. */
#define GPZ_FLAG_REL_ON_DEVICE 4u

typedef struct gpz_batch gpz_batch;

/* GPZ_EINVAL names no item; *bad_item (may be NULL) receives the index of the
 * first invalid item. */
int gpz_batch_create(const gpz_batch_item *items, uint32_t count, gpz_batch **batch, uint32_t *bad_item);
int gpz_batch_launch(gpz_batch *batch, void *stream);
/* results[count]; h_eb (may be NULL) receives each snapshot's absolute bound. */
int gpz_batch_results(gpz_batch *batch, gpz_result *results, double *h_eb, void *stream);
/* Device memory the batch holds (bytes). */
uint64_t gpz_batch_device_bytes(const gpz_batch *batch);
int gpz_batch_destroy(gpz_batch *batch);

/* ---- batched decompress ------------------------------------------------------------
 * No counterpart in the reference (one stream per CompressorManager::decompressWarp
 * call, src/CompressorManager.cpp:18-22).  Many streams of mixed float width
 * and dimension decoded by one CUDA graph: a header check per stream, then one
 * persistent decompress kernel per class whose warps stride over the chunks of
 * all its streams.  Each stream's output equals gpz_decompress's.  Same plan
 * model as gpz_batch: bound to the buffers at creation, launched any number of
 * times, launches must not overlap. */
typedef struct gpz_dbatch_item {
  const void *d_stream;  /* the stream on the device */
  uint64_t stream_bytes;
  uint32_t float_bits;   /* from the stream header (gpz_parse_header on a host copy) */
  uint32_t dim;
  uint64_t n;            /* points, from the stream header; checked on the device */
  void *d_x;             /* SoA outputs, out_capacity points each; d_z ignored for 2D */
  void *d_y;
  void *d_z;
  uint64_t out_capacity;
} gpz_dbatch_item;

typedef struct gpz_dbatch gpz_dbatch;

int gpz_dbatch_create(const gpz_dbatch_item *items, uint32_t count, gpz_dbatch **batch, uint32_t *bad_item);
int gpz_dbatch_launch(gpz_dbatch *batch, void *stream);
int gpz_dbatch_results(gpz_dbatch *batch, gpz_result *results, void *stream);
int gpz_dbatch_destroy(gpz_dbatch *batch);

/* ---- request server --------------------------------------------------------------
 * No counterpart in the reference (a command line tool: one file, one call).
 * A server admits compress / decompress requests as they arrive and runs them
 * in batches on several CUDA streams (continuous batching): whenever a stream
 * is free, every queued request whose output fits in the device-memory budget
 * joins the next batch, so requests that arrive while others run are started
 * as soon as a stream and memory free up; their preparation and upload
 * overlap the running batch, and with GPZ_SERVER_OVERLAP their kernels too.
 * All device memory -- request outputs and batch workspaces -- comes from one
 * arena of hbm_budget bytes allocated at creation; serving allocates nothing.
 * Outputs stay in the arena (device resident) until the caller releases them.
 * Each request's output equals the single-call API's (gpz_compress with the
 * same parameters, gpz_decompress). */
#define GPZ_OP_COMPRESS 1u
#define GPZ_OP_DECOMPRESS 2u

typedef struct gpz_server_config {
  uint64_t hbm_budget;      /* bytes of device memory for outputs and workspaces */
  uint32_t streams;         /* batches in flight at once, >= 1 */
  uint32_t max_batch;       /* requests per batch, >= 1 */
  uint64_t workspace_bytes; /* per stream: batch descriptors and control blocks (0: 64 MiB) */
  uint32_t flags;           /* GPZ_SERVER_OVERLAP */
  uint32_t reserved;        /* 0 */
} gpz_server_config;

/* Server flag: batches on different streams run concurrently on the GPU.
 * Without it the GPU runs the batches one after another (each waits for the
 * previous one's completion event) and the streams only let the server
 * prepare and queue the next batches while one runs: two different codec
 * kernels resident on one SM thrash its instruction cache, so concurrent
 * batches are usually slower. */
#define GPZ_SERVER_OVERLAP 1u

typedef struct gpz_request {
  uint32_t op;              /* GPZ_OP_COMPRESS or GPZ_OP_DECOMPRESS */
  uint32_t float_bits;      /* compress: the input's; decompress: from the stream header */
  uint32_t dim;
  uint32_t flags;           /* compress: GPZ_FLAG_SAFE31 | GPZ_FLAG_SEG_FIXED | GPZ_FLAG_REL_ON_DEVICE */
  uint64_t n;               /* points (decompress: from the stream header) */
  const void *d_x;          /* compress input; must stay valid until the request completes */
  const void *d_y;
  const void *d_z;
  const void *d_stream;     /* decompress input; must stay valid until the request completes */
  uint64_t stream_bytes;
  double eb;                /* as in gpz_batch_item */
  double rel_eb;
  int32_t rel_mode;
  uint32_t seg_size;
} gpz_request;

typedef struct gpz_completion {
  int32_t status;           /* GPZ_OK or the request's error */
  uint32_t seg_size;        /* compress: the segment size used */
  uint64_t stream_bytes;    /* compress: stream size */
  void *d_out;              /* compress: the stream; decompress: x, y, z, n values each, every axis
                               starting at a multiple of 256 bytes (stride: n * sizeof(T) rounded up to 256) */
  double eb;                /* compress: the absolute bound used */
  double queue_ms;          /* submit -> launch of its batch */
  double total_ms;          /* submit -> completion seen by the server */
  uint32_t batch_size;      /* requests in its batch */
  uint32_t reserved;
} gpz_completion;

typedef struct gpz_server_stats {
  uint64_t submitted, completed, batches, arena_bytes, arena_free_bytes;
  uint32_t queued, in_flight;
} gpz_server_stats;

typedef struct gpz_server gpz_server;

int gpz_server_create(const gpz_server_config *cfg, gpz_server **server);
/* Never blocks.  GPZ_EINVAL for a malformed request, GPZ_ENOSPACE when its
 * output could never fit in the arena. */
int gpz_server_submit(gpz_server *server, const gpz_request *req, uint64_t *ticket);
/* Blocks until the request completes (GPZ_ETIMEOUT after timeout_ms; 0 waits
 * without limit). */
int gpz_server_wait(gpz_server *server, uint64_t ticket, gpz_completion *out, uint32_t timeout_ms);
/* Returns a completed request's output memory to the arena.  Requests are
 * admitted in arrival order, so a caller that keeps outputs must release them
 * for later requests to start once the arena is full. */
int gpz_server_release(gpz_server *server, uint64_t ticket);
int gpz_server_stats_get(gpz_server *server, gpz_server_stats *stats);
/* Finishes the work in flight, then frees everything. */
int gpz_server_destroy(gpz_server *server);

/* ---- verification -------------------------------------------------------------------
 * Replaces the reference's verifier (src/utils.cu:17-217, used by the CLI's
 * -v), which sorts every axis of the original and of the reconstruction and
 * compares the sorted sequences, so it never pairs a point with its own
 * reconstruction.  gpz_verify recovers the exact pairing on the device: per
 * 1024-point chunk it recomputes the encoder's sort of the points by block
 * (from the originals, eb and seg_size, as found in the stream header), so
 * reconstructed point s of the chunk is compared with the original the
 * encoder placed at s.  Inputs: the original SoA arrays and the
 * reconstruction in stream order (gpz_decompress's output).  Synchronises
 * `stream`; needs gpz_verify_scratch_bytes() of scratch. */
typedef struct gpz_verify_result {
  uint64_t points;
  uint64_t over_bound;      /* points with some axis |reconstruction - original| > eb */
  uint64_t over_bound_tol;  /* ... > 1.01 * eb (the reference verifier's tolerance) */
  double max_abs_err[3];
  double mse[3];
  double value_range[3];    /* max - min of the originals */
  double psnr[3];           /* 20 log10(range) - 10 log10(mse), per axis */
  double psnr_combined;     /* from the per-axis normalised RMS errors, as the reference CLI combines them */
} gpz_verify_result;

uint64_t gpz_verify_scratch_bytes(void);
int gpz_verify(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y, const void *d_z,
               const void *d_rx, const void *d_ry, const void *d_rz, double eb, uint32_t seg_size, void *d_scratch,
               uint64_t scratch_bytes, gpz_verify_result *result, void *stream);

/* gpz_verify with the pairing and the check apart: `eb` and seg_size are the
 * stream's (its header), `bound` the error bound the points are checked
 * against (over_bound counts errors above bound, over_bound_tol above
 * 1.01*bound).  For streams encoded in strict-bound mode, whose header
 * carries a bound below the stated one.  No counterpart in the reference. */
int gpz_verify_bound(uint32_t float_bits, uint32_t dim, uint64_t n, const void *d_x, const void *d_y,
                     const void *d_z, const void *d_rx, const void *d_ry, const void *d_rz, double eb,
                     uint32_t seg_size, double bound, void *d_scratch, uint64_t scratch_bytes,
                     gpz_verify_result *result, void *stream);

/* ---- self-test of the bounded waits ---------------------------------------------
 * No counterpart in the reference (its placement is a separate CUB scan, with
 * no waiting between blocks).  The compress kernels place chunks with a
 * decoupled look-back whose every wait is bounded: after a limited number of
 * polls of a predecessor that has published nothing, the kernel sets
 * GPZ_ETIMEOUT and returns, so a stuck predecessor cannot hang the GPU.  This
 * runs that wait against a predecessor that never publishes, with `polls`
 * (1 .. 4,194,304) as the limit, and returns the status the kernel recorded
 * (GPZ_ETIMEOUT when the wait ran out).  Needs gpz_compress_scratch_bytes(2048)
 * of scratch; synchronises `stream`. */
int gpz_selftest_lookback_timeout(uint32_t polls, void *d_scratch, uint64_t scratch_bytes, int32_t *status,
                                  void *stream);

/* Library version string. */
const char *gpz_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GPZ_B200_H */
