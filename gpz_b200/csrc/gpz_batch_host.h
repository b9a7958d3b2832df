// gpz_batch_host.h -- host side of the batched kernels, shared by the batch
// plans (gpz_batchapi.cu) and the request server (gpz_serve.cu).
//
// A batch runs in a workspace of device memory laid out by *_layout:
//   [0, zero_bytes)      control blocks, look-back words, work counters;
//                        cleared by *_enqueue before the kernels run
//   [zero_bytes, bytes)  descriptors and work maps, built on the host by
//                        *_tables into a host image of that range
// *_enqueue clears the first range and launches the class kernels on a
// stream; it allocates nothing, so it runs inside a graph capture (the batch
// plans) or directly (the server, which uploads the table image itself).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "gpz_b200.h"

namespace gpzb_host {

struct ClassPlan {
  std::vector<uint32_t> items;  // item indices, in work-list order
  uint64_t work = 0;            // compress: 8-chunk groups; decompress: chunks
  uint64_t rel_blocks = 0;      // compress: rel->abs blocks of GPZ_FLAG_REL_ON_DEVICE items
  uint64_t table_off = 0, map_off = 0, rmap_off = 0;
  int grid = 0;   // persistent grid (float64 decompress: of the fast pass)
  int grid2 = 0;  // float64 decompress: grid of the general pass
};

struct Layout {
  ClassPlan cls[4];                // (float, 2D), (float, 3D), (double, 2D), (double, 3D)
  std::vector<uint64_t> look_off;  // compress: each item's look-back words
  uint64_t claim_off = 0, zero_bytes = 0, bytes = 0;
  uint32_t count = 0;
};

// Argument checks (no CUDA call).
bool compress_item_ok(const gpz_batch_item &it);
bool decompress_item_ok(const gpz_dbatch_item &it);

// Offsets of everything in the workspace and the persistent grids
// (false: a CUDA attribute query failed).
bool compress_layout(const gpz_batch_item *items, uint32_t count, Layout &L);
bool decompress_layout(const gpz_dbatch_item *items, uint32_t count, Layout &L);

// Host image of [zero_bytes, bytes) for a workspace at device address `dev`.
void compress_tables(const gpz_batch_item *items, const Layout &L, uint8_t *dev, uint8_t *image);
void decompress_tables(const gpz_dbatch_item *items, const Layout &L, uint8_t *dev, uint8_t *image);

// Clears the control range and launches the class kernels on `st`.
void compress_enqueue(const Layout &L, uint8_t *dev, cudaStream_t st);
void decompress_enqueue(const Layout &L, uint8_t *dev, cudaStream_t st);

// Item i's control block (compress: also its rel->abs block at count + i).
inline uint64_t ctl_off(uint32_t i) { return (uint64_t)i * 256u; }

}  // namespace gpzb_host
