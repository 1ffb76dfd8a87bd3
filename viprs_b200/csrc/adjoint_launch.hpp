// adjoint_launch.hpp -- argument blocks of the adjoint (backward) kernels.
//
// These have no viprs counterpart: viprs's resample ops are forward only.
// Each adjoint is the exact transpose of the forward operator as this
// library evaluates it (same tables, same positions, same extend rules).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "affine_launch.hpp"
#include "launch.hpp"

namespace viprs {

// Transpose of one separable reduce pass over f32, as a gather: every input
// sample sums the output samples whose taps read it.  For input index i the
// outputs are [lo[i], hi[i]] (lo > hi: none) and the weight of output o is
// wt[i * wstride + (o - lo[i])]: the forward coefficient of that tap, or at a
// clamped edge the sum of the taps that clamp_axis folds onto it.
struct ReduceAdjArgs {
    const float* g_out = nullptr;  // gradient wrt the pass output
    float* g_in = nullptr;         // gradient wrt the pass input (overwritten)
    int32_t horizontal = 1;
    int32_t out_w = 0, out_h = 0;  // pass output size
    int32_t in_w = 0, in_h = 0;    // pass input size (the folded axis)
    int32_t bands = 1;
    const int32_t* lo = nullptr;   // per input index
    const int32_t* hi = nullptr;
    const float* wt = nullptr;     // per input index, wstride weights
    int32_t wstride = 1;
    // H pass of an H-then-V chain: input row r gathers mid row r - mid_y0, and
    // the edge rows also gather the virtual mid rows that the source read
    // clamps onto them
    int32_t fold_rows = 0;
    int32_t mid_y0 = 0;            // origin of the mid rows (may be negative)
};

// Gradient of the bilinear affine (forward: Affine::process_region with
// viprs's per-tile position walk) wrt its input image and its matrix.
struct AffineGradArgs {
    AffineArgs fwd;            // forward arguments (in = the forward input, out = shape only)
    const float* g_out = nullptr;
    float* g_in = nullptr;                 // atomic mode (may be null)
    unsigned long long* g_fixed = nullptr; // deterministic mode: fixed-point accumulator
    double fixed_scale = 0.0;
    double* partial = nullptr;             // per block: d/d(m0, m1, m2, m3, tx, ty)
};

struct MapimGradArgs {
    MapimArgs fwd;
    const float* g_out = nullptr;
    float* g_src = nullptr;
    unsigned long long* g_fixed = nullptr;
    double fixed_scale = 0.0;
    float* g_index = nullptr;  // (h, w, 2) gradient wrt the coordinates (may be null)
};

namespace launch {
cudaError_t reduce_adjoint(const ReduceAdjArgs& a, cudaStream_t s);
// blocks of affine_grad for an out_w x out_h output (one partial row each)
int affine_grad_blocks(int32_t out_w, int32_t out_h);
cudaError_t affine_grad(const AffineGradArgs& a, int blocks, cudaStream_t s);
cudaError_t mapim_grad(const MapimGradArgs& a, cudaStream_t s);
// fixed-point accumulator -> f32 (deterministic scatter), n values
cudaError_t fixed_to_f32(const unsigned long long* acc, float* out, int64_t n, double inv_scale, cudaStream_t s);
// sum `blocks` rows of 6 partials into out[6] in a fixed order
cudaError_t sum_partials(const double* partial, int blocks, double* out, cudaStream_t s);
}  // namespace launch

}  // namespace viprs
