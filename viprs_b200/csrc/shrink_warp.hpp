// shrink_warp.hpp -- host planning of the independent-warp u8 shrink
// (shrink_warp.cuh).
#pragma once

#include <cstdint>

#include "launch.hpp"

namespace viprs {
namespace launch {

constexpr int kWarpStagesHost = 4;   // source rows in flight per warp (== dev::kWarpStages)
constexpr int kWarpBlockThreads = 256;

// Warp geometry of a u8 ShrinkH+ShrinkV stage (a->fh, fv, bands, out, in,
// premul_in set): output pixels per warp (a->nxf: 32, 16 or 8, fewest lanes
// per box whose source row segment fits `stage_budget` bytes), the stage
// buffer size (a->row_cap), output rows per work item (a->rows_per_item,
// about `item_bytes` of source per item, fewer when that would leave fewer
// than `min_items` items) and the lane rotation of the premultiplied box walk
// (a->rot_shift).  Returns false when no geometry fits the budget.
bool shrink_warp_setup(ShrinkArgs* a, uint32_t stage_budget, int64_t item_bytes, int64_t min_items);

// Work items of a stage set up by shrink_warp_setup.
int64_t shrink_warp_items(const ShrinkArgs& a);

}  // namespace launch
}  // namespace viprs
