// affine_launch.hpp -- argument blocks of the affine / mapim kernels and the
// host helpers that plan an affine stage.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"
#include "plan.hpp"

namespace viprs {

// Affine (resample/affine.rs, affine/core.rs, affine/interpolation.rs).
struct AffineArgs {
    PlaneArg in;
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kU8;
    double m[4] = {1, 0, 0, 1};  // backward matrix: x_in = a x + b y + tx
    double tx = 0, ty = 0;
    int32_t kernel = 1;
    int32_t extend = 2;
    double background = 0.0;
    int32_t premultiplied = 0;
    uint32_t src_w = 0, src_h = 0;      // with_source_bounds(0, 0, src_w, src_h)
    uint32_t total_w = 0, total_h = 0;  // Affine output_w / output_h
    uint32_t tile_w = 128, tile_h = 128;
    int64_t tile_off_x = 0, tile_off_y = 0;  // tile grid origin in affine output coords
    uint32_t final_w = 0, final_h = 0;       // pipeline output the tile grid covers
    int32_t fast = 0;        // axis-aligned fast path: 0 none, 1 nearest, 2 bilinear, 3 bicubic
    int32_t separable = 0;   // b == c == 0: positions from per-axis tables
    const double* xs = nullptr;  // per output column x_in (separable general path)
    const double* ys = nullptr;  // per output row y_in
    // separable general path, kernels other than nearest / bilinear: the
    // kAxisTaps point-sampling weights of each output column (wx) and row (wy),
    // taps floor(x) - (support - 1) onwards, zero past the kernel's taps
    const double* wx = nullptr;
    const double* wy = nullptr;
    int32_t unpremul_out = 0;
    int32_t group = 1;       // consecutive output pixels per thread (set by the launcher)
};

// MapImOp (resample/mapim.rs).
struct MapimArgs {
    PlaneArg src;
    PlaneArg index;  // 2-band coordinates of index_fmt (u8, u16 or f32), read as f64
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kF32;
    int32_t index_fmt = kF32;
    int32_t kernel = 1;
    int32_t extend_copy = 0;
    int32_t alpha = 0;  // 2/4 bands, not premultiplied: the alpha-premultiplying sampler
    double background = 0.0;
    uint32_t src_w = 0, src_h = 0;
};

namespace launch {
// output pixels per thread of the affine kernels for an npx-pixel output
int affine_group(int64_t npx);
cudaError_t affine(const AffineArgs& a, cudaStream_t s);
cudaError_t mapim(const MapimArgs& a, cudaStream_t s);
}  // namespace launch

// Host planning of an affine stage.
bool affine_kernel_supported(Kernel k);
Region affine_required_region(const PlanNode& n, uint32_t in_w, uint32_t in_h, const Region& out);
Demand default_demand(const Chain& chain);
// Fills everything but the planes and the device table pointers; `tables`
// receives the per-axis position tables (xs then ys) when the walk is separable.
int affine_stage_setup(const PlanNode& n, uint32_t in_w, uint32_t in_h, uint32_t bands, int32_t fmt,
                       int32_t demand_override, Demand chain_demand, uint32_t final_w, uint32_t final_h,
                       int64_t tile_off_x, int64_t tile_off_y, AffineArgs* a);
// Per-axis positions of viprs's incremental walk (affine/core.rs:1593-1632)
// for a diagonal matrix over the tile grid in `a`.
void affine_axis_tables(const AffineArgs& a, double* xs, double* ys);
// Per-axis weights of the separable sampler for positions xs / ys (kAxisTaps
// per output column into wx, per output row into wy); the kernel reads them
// instead of evaluating InterpolationKernel::interpolate per pixel and band.
constexpr int kAxisTaps = 6;
bool affine_weight_tables_apply(const AffineArgs& a);
void affine_weight_tables(const AffineArgs& a, const double* xs, const double* ys, double* wx, double* wy);

}  // namespace viprs
