// chain.hpp -- internal representation of an executable builder chain (a
// plan): its planes, its fused stages and their device tables.  Shared by
// the C ABI (capi.cpp) and the batched executor (batch_plan.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "affine_launch.hpp"
#include "launch.hpp"
#include "plan.hpp"
#include "viprs_b200.h"

namespace viprs {

enum class StageType { Shrink, ReduceH, ReduceV, Reduce2D, Pixel, Affine };

struct Stage {
    StageType type;
    int in_plane = 0;   // index into planes; 0 = source
    int out_plane = 0;  // index into planes; last = destination
    ShrinkArgs sh;
    ReduceArgs rd;
    PixelArgs px;
    AffineArgs af;
    Reduce2DArgs r2;
    // offsets of this stage's tables inside the plan table buffer
    size_t starts_off = 0, phases_off = 0, coeffs_off = 0;
    size_t starts2_off = 0, phases2_off = 0, coeffs2_off = 0;
    // affine: per-axis weight tables at coeffs_off (columns) / coeffs2_off (rows)
    bool axis_weights = false;
};

struct PlaneInfo {
    Region r;
    size_t offset = 0;  // workspace offset (intermediates)
    int64_t pitch = 0;
};

}  // namespace viprs

struct viprs_plan {
    int device = 0;
    uint32_t in_w = 0, in_h = 0, bands = 0;
    int32_t fmt = 0;
    uint32_t out_w = 0, out_h = 0;
    int64_t in_pitch = 0, out_pitch = 0;
    std::vector<viprs::PlaneInfo> planes;
    std::vector<viprs::Stage> stages;
    std::vector<uint8_t> host_tables;
    uint8_t* d_tables = nullptr;
    uint8_t* d_work = nullptr;
    size_t work_bytes = 0;
    bool stream_ordered_alloc = false;
    cudaStream_t alloc_stream = nullptr;
    // execute_host staging
    uint8_t* d_in = nullptr;
    uint8_t* d_out = nullptr;
    // device error word inside d_tables (a bounded wait that gave up records
    // VIPRS_ERR_TIMEOUT there); read and cleared by viprs_plan_status
    size_t err_off = 0;
    int32_t* d_err = nullptr;
};


namespace viprs {

// Build a plan for `chain` on an image of (w, h, bands, format) and allocate
// its tables and workspace (cudaMalloc); status 0 on success.
// The builder chain of a C-ABI node list (PipelineBuilder node by node).
int32_t nodes_to_chain(const viprs_node* nodes, int32_t n_nodes, int32_t demand_override, Chain* out);

int create_chain_plan(uint32_t w, uint32_t h, uint32_t bands, int32_t format, const Chain& chain,
                      viprs_plan** out);
// Enqueue stages [first, first + count) (count < 0: all) on `s`.
int execute_plan(viprs_plan* p, const void* src, void* dst, cudaStream_t s, int first = 0, int count = -1);
void free_plan(viprs_plan* p);
PlaneArg plane_in_arg(const viprs_plan* p, int idx, const uint8_t* src);
OutPlaneArg plane_out_arg(const viprs_plan* p, int idx, uint8_t* dst);
int32_t cuda_status(cudaError_t e);
// Host-side plan of a one-node chain (no device memory touched); status 0 on success.
int plan_single_node(const viprs_image* in, const viprs_image* out, const PlanNode& node, viprs_plan* p);

}  // namespace viprs
