// batch_launch.hpp -- descriptors of the persistent batched-thumbnail kernel.
//
// A batch is many thumbnail plans (one per image) executed by a few
// persistent launches that walk a device work list.  Every stage of every
// image plan becomes a BatchStage; its work is split into items (shrink: band
// of output rows x column chunk; fused reduce: output tile; affine / pixel:
// output row).  Stages are grouped by level (shrink, then the stage after it,
// ...) and each level runs as one launch of its shrink items and one of its
// other items, so a stage's input is complete when its launch starts.  The
// dependency fields (dep, dep_items, counters) support a bounded in-kernel
// wait for lists that mix levels; the level launches leave them unused.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "affine_launch.hpp"
#include "launch.hpp"

namespace viprs {

enum : int32_t { kBatchShrink = 1, kBatchReduce2D = 2, kBatchPixel = 3, kBatchAffine = 4,
                 kBatchReduceH = 5, kBatchReduceV = 6 };

struct BatchStage {
    int32_t type = 0;
    int32_t image = 0;
    int32_t in_src = 0;    // the input plane is the image's source buffer
    int32_t out_dst = 0;   // the output plane is the image's destination buffer
    int32_t n_items = 0;
    int32_t dep = -1;      // stage whose completion this stage waits for
    int32_t dep_items = 0; // that stage's item count
    // shrink items: chunk layout over the output columns, output rows per item
    int32_t lo = 0, hi = 0, chunk_cols = 1, n_chunks = 1, rows_per_item = 1;
    // reduce h/v items: samples per item
    int32_t per_item = 256;
    ShrinkArgs sh;
    Reduce2DArgs r2;
    PixelArgs px;
    AffineArgs af;
    ReduceArgs rd;
};

struct WorkItem {
    int32_t stage;
    int32_t index;
};

struct BatchArgs {
    const BatchStage* stages = nullptr;
    const WorkItem* items = nullptr;
    int32_t n_items = 0;
    int32_t* counters = nullptr;  // one per stage, zeroed before each launch
    int32_t* cursor = nullptr;    // work-list cursor, zeroed before each launch
    int32_t* err = nullptr;       // first error (timeout) seen by any block
    const uint64_t* srcs = nullptr;  // device array: source pointer of each image
    const uint64_t* dsts = nullptr;  // device array: destination pointer of each image
    uint32_t ring_stage_bytes = 0;   // bytes of one stage buffer of a shrink warp
    int32_t ring_slots = 0;          // unused by the warp shrink
    uint32_t work_bytes = 0;         // shared memory of the other item kinds
    uint32_t smem_bytes = 0;         // control block + stage copy + ring + work
};

namespace launch {
// Variants of the tile kernel: fused-reduce tiles of 3- or 4-band images only.
constexpr int kBatchTile3 = 13, kBatchTile4 = 14;
// Launch the persistent kernel on `grid` blocks: the shrink variant for
// images of `ring_bands` bands (1..4: independent warps, each with its own
// stage buffers of a.ring_stage_bytes), the tile variant for every other item
// kind (0), or a tile variant specialised to kBatchTile3 / kBatchTile4.
cudaError_t batch(const BatchArgs& a, int grid, int ring_bands, cudaStream_t s);
// Largest resident block count per SM for `smem` bytes of shared memory.
int batch_blocks_per_sm(size_t smem, int ring_bands);
// Shared memory of the other item kinds' variant ahead of its work region:
// control block and the queued stage copies.
size_t batch_ctl_bytes();
// Shared memory of a shrink launch whose warps have stage buffers of
// `stage_bytes` (a stage descriptor and the buffers per warp).
size_t batch_warp_smem_bytes(uint32_t stage_bytes);
}  // namespace launch

}  // namespace viprs
