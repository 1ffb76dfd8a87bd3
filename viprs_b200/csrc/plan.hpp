// plan.hpp -- host-side planning of the resample path (C++ mirror of viprs's
// L0/L1 planning code).  Everything here runs on the CPU in f64 with the
// same operation order as viprs, so that the device kernels only perform
// integer or float multiply-adds over tables computed here.
//
//   InterpolationKernel weights ... viprs-core/src/kernel.rs:50-214
//   ReduceKernel tables ........... viprs-ops-spatial/src/resample/reduce_common.rs:128-316
//   ReduceConfig regions .......... viprs-core/src/resample.rs:74-215
//   Thumbnail planner ............. resample/thumbnail.rs:204-524
//   Resize planner ................ resample/resize.rs:163-348
//   forward -> backward affine .... viprs-runtime/src/pipeline/builder/resample.rs:25-60
//
// This translation unit must be compiled with -ffp-contract=off: a product
// or sum is fused only where std::fma is written, which is where viprs calls
// `mul_add`.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace viprs {

enum class Kernel : int32_t {
    Nearest = 0, Bilinear = 1, Bicubic = 2, Quadratic = 3, Nohalo = 4, Lbb = 5,
    Vsqbs = 6, CatmullRom = 7, Lanczos2 = 8, Lanczos3 = 9
};
enum class Format : int32_t { U8 = 0, U16 = 1, F32 = 2 };
enum class Extend : int32_t { Black = 0, White = 1, Background = 2, Copy = 3, Repeat = 4, Mirror = 5 };
enum class Demand : int32_t { Any = 0, ThinStrip = 1, FatStrip = 2, SmallTile = 3, FullImage = 4, OneLine = 5 };

inline size_t format_size(Format f) { return f == Format::U8 ? 1 : (f == Format::U16 ? 2 : 4); }

struct Region {
    int64_t x = 0, y = 0, w = 0, h = 0;
};

double kernel_weight(Kernel k, double x);
double kernel_support(Kernel k);
void kernel_affine_padding(Kernel k, int32_t* left, int32_t* right);
bool reduce_kernel_is_separable(Kernel k);

// Rust `f64 as i64`: truncation toward zero, saturating; NaN -> 0.
int64_t f64_to_i64(double v);
uint32_t f64_to_u32(double v);

constexpr int kPhases = 64;
constexpr int kMaxTaps = 2000;

// ReduceKernel (reduce_common.rs:86-316)
struct ReduceKernel {
    double factor = 1.0;
    int32_t taps = 1;
    int64_t pad_before = 0;
    double offset = 0.0;
    std::vector<double> coeffs_f64;   // 65 * taps
    std::vector<int16_t> coeffs_i16;  // 65 * taps

    // status: 0 ok, otherwise a viprs_status code
    int init(double factor, Kernel kernel);
    void bind_input_len(uint32_t input_len);
    double source_position(double index) const;
    void plan(double pos, int64_t* start, int32_t* phase) const;
    // ReduceKernel::required_input_region_h/_v for one axis (offset applied)
    void required_axis(int64_t out_origin, int64_t out_len, int64_t* in_origin, int64_t* in_len) const;
    // ReduceConfig::required_input_region_h/_v for one axis (no offset, clamped at 0)
    void config_required_axis(int64_t out_origin, int64_t out_len, int64_t* in_origin, int64_t* in_len) const;
    // Largest sum over phases of |coefficient|, for accumulator range checks.
    int64_t max_abs_i16_sum() const;
};

uint32_t reduce_output_len(double factor, uint32_t input_len);

// Thumbnail / resize plans.
enum class NodeKind : int32_t {
    Premultiply = 1, ShrinkH = 2, ShrinkV = 3, ReduceH = 4, ReduceV = 5, Affine = 6,
    ExtractArea = 7, Unpremultiply = 8, Zoom = 9, Reduce = 10, Shrink = 11
};

struct PlanNode {
    NodeKind kind = NodeKind::ShrinkH;
    uint32_t ufactor = 1;     // shrink factor (h for Shrink)
    uint32_t vufactor = 1;    // Shrink v factor
    bool ceil = false;
    double factor = 1.0;      // reduce factor (h for Reduce)
    double vfactor = 1.0;     // Reduce v factor
    Kernel kernel = Kernel::Lanczos3;
    double m[4] = {1, 0, 0, 1};  // backward matrix
    double tx = 0, ty = 0;
    uint32_t out_w = 0, out_h = 0;
    Extend extend = Extend::Background;
    double background = 0.0;
    bool premultiplied = false;
    Demand demand = Demand::ThinStrip;
    uint32_t ex = 0, ey = 0, ew = 0, eh = 0;
    uint32_t zx = 1, zy = 1;
};

enum class ThumbTarget : int32_t { FitBox = 0, ForceExact = 1, Width = 2, Height = 3 };

struct ThumbnailPlan {
    std::vector<PlanNode> nodes;
    uint32_t output_width = 0, output_height = 0;
    uint32_t shrink_factor = 0;  // shrink-on-load hint (0 = none)
};

// Thumbnail::into_pipeline_nodes[_without_shrink_hint]
ThumbnailPlan thumbnail_plan(ThumbTarget target, uint32_t tw, uint32_t th, Kernel kernel, bool crop,
                             uint32_t in_w, uint32_t in_h, uint32_t bands, bool allow_shrink_hint);

struct ResizePlan {
    std::vector<PlanNode> nodes;
    uint32_t output_width = 0, output_height = 0;
};
ResizePlan resize_plan(double hscale, double vscale, Kernel kernel, double gap, uint32_t in_w, uint32_t in_h);

// PipelineBuilder::thumbnail / ::resize materialisation into a node chain
// plus the demand-hint override the builder sets.
struct Chain {
    std::vector<PlanNode> nodes;
    uint32_t out_w = 0, out_h = 0;
    int32_t demand_override = -1;  // -1: max over nodes
};
int builder_thumbnail_chain(uint32_t w, uint32_t h, uint32_t bands, ThumbTarget target, uint32_t tw,
                            uint32_t th, Kernel kernel, bool crop, Chain* out);
int builder_resize_chain(uint32_t w, uint32_t h, uint32_t bands, double hscale, double vscale,
                         Kernel kernel, Chain* out);

// SimilarityOp::new_auto_canvas (resample/similarity.rs:47-81, 178-232) as the
// Affine node PipelineBuilder::similarity runs (builder/resample.rs:595-626):
// backward matrix, canvas translation and size, Background(0), SmallTile.
PlanNode similarity_node(double scale, double angle, Kernel kernel, uint32_t in_w, uint32_t in_h);

// forward_affine_to_backward (builder/resample.rs:25-60); status 0 ok.
int forward_affine_to_backward(const double fwd[4], double tx, double ty, double bwd[4], double* btx,
                               double* bty);

// Output dims of one node.
int node_output_dims(const PlanNode& n, uint32_t in_w, uint32_t in_h, uint32_t* ow, uint32_t* oh);

// Tile geometry of the reference scheduler for a demand hint
// (demand.rs:41-83, planning.rs:550-596).
void tile_geometry(Demand hint, uint32_t w, uint32_t h, uint32_t* tw, uint32_t* th);

}  // namespace viprs
