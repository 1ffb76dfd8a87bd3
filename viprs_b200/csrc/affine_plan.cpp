// affine_plan.cpp -- host planning of affine stages (compiled with
// -ffp-contract=off, like plan.cpp).
//
//   Affine::required_input_region ... resample/affine/core.rs:1517-1560
//   fast-path selection ............. affine/core.rs:112-189, 1057-1095
//   incremental position walk ....... affine/core.rs:1593-1632
//   tile grid ....................... viprs-core/src/op/demand.rs:41-83
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "affine_launch.hpp"
#include "interp_weights.hpp"
#include "viprs_b200.h"

namespace viprs {

bool affine_kernel_supported(Kernel k) {
    // Nohalo, LBB and VSQBS are nonlinear 2-D interpolators outside this path.
    return !(k == Kernel::Nohalo || k == Kernel::Lbb || k == Kernel::Vsqbs) && int(k) >= 0 && int(k) <= 9;
}

static void map_to_input(const double* m, double tx, double ty, double x, double y, double* ox, double* oy) {
    *ox = std::fma(m[1], y, m[0] * x) + tx;
    *oy = std::fma(m[3], y, m[2] * x) + ty;
}

static void axis_bounds(int64_t start, int64_t end, int64_t bs, int64_t blen, int64_t* o, int64_t* len) {
    if (blen == 0) { *o = bs; *len = 0; return; }
    const int64_t be = bs + blen - 1;
    const int64_t cs = std::max(start, bs), ce = std::min(end, be);
    if (ce < cs) { *o = end < bs ? bs : be + 1; *len = 0; return; }
    *o = cs; *len = ce - cs + 1;
}

Region affine_required_region(const PlanNode& n, uint32_t in_w, uint32_t in_h, const Region& out) {
    const double ox0 = double(out.x), oy0 = double(out.y);
    const double ox1 = double(out.x) + double(std::max<int64_t>(out.w - 1, 0));
    const double oy1 = double(out.y) + double(std::max<int64_t>(out.h - 1, 0));
    double cx[4], cy[4];
    map_to_input(n.m, n.tx, n.ty, ox0, oy0, &cx[0], &cy[0]);
    map_to_input(n.m, n.tx, n.ty, ox1, oy0, &cx[1], &cy[1]);
    map_to_input(n.m, n.tx, n.ty, ox0, oy1, &cx[2], &cy[2]);
    map_to_input(n.m, n.tx, n.ty, ox1, oy1, &cx[3], &cy[3]);
    const double mnx = std::min(std::min(std::min(cx[0], cx[1]), cx[2]), cx[3]);
    const double mxx = std::max(std::max(std::max(cx[0], cx[1]), cx[2]), cx[3]);
    const double mny = std::min(std::min(std::min(cy[0], cy[1]), cy[2]), cy[3]);
    const double mxy = std::max(std::max(std::max(cy[0], cy[1]), cy[2]), cy[3]);
    int32_t lp, rp;
    kernel_affine_padding(n.kernel, &lp, &rp);
    Region r;
    if (in_w == 0 || in_h == 0) return r;
    axis_bounds(f64_to_i64(std::floor(mnx)) - lp, f64_to_i64(std::floor(mxx)) + rp, 0, in_w, &r.x, &r.w);
    axis_bounds(f64_to_i64(std::floor(mny)) - lp, f64_to_i64(std::floor(mxy)) + rp, 0, in_h, &r.y, &r.h);
    return r;
}

Demand default_demand(const Chain& chain) {
    int32_t h = int32_t(Demand::Any);
    for (const auto& n : chain.nodes) h = std::max(h, int32_t(n.demand));
    return Demand(h);
}

int affine_stage_setup(const PlanNode& n, uint32_t in_w, uint32_t in_h, uint32_t bands, int32_t fmt,
                       int32_t demand_override, Demand chain_demand, uint32_t final_w, uint32_t final_h,
                       int64_t tile_off_x, int64_t tile_off_y, AffineArgs* a) {
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(n.m[i])) return VIPRS_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(n.tx) || !std::isfinite(n.ty)) return VIPRS_ERR_INVALID_ARGUMENT;
    // Affine::try_new (affine/interpolation.rs:13-40)
    const double det = std::fma(n.m[1], -n.m[2], n.m[0] * n.m[3]);
    if (std::fabs(det) <= DBL_EPSILON) return VIPRS_ERR_DEGENERATE_AFFINE;
    if (!affine_kernel_supported(n.kernel)) return VIPRS_ERR_INVALID_KERNEL;
    for (int i = 0; i < 4; ++i) a->m[i] = n.m[i];
    a->tx = n.tx; a->ty = n.ty;
    a->bands = int32_t(bands); a->fmt = fmt;
    a->kernel = int32_t(n.kernel);
    a->extend = int32_t(n.extend);
    a->background = n.background;
    a->premultiplied = n.premultiplied ? 1 : 0;
    a->src_w = in_w; a->src_h = in_h;
    a->total_w = n.out_w; a->total_h = n.out_h;
    const Demand hint = demand_override >= 0 ? Demand(demand_override) : chain_demand;
    uint32_t tw, th;
    tile_geometry(hint, final_w, final_h, &tw, &th);
    if (n.ew > 0 && n.eh > 0) { tw = n.ew; th = n.eh; }  // explicit grid from the caller
    a->tile_w = std::max(tw, 1u); a->tile_h = std::max(th, 1u);
    a->tile_off_x = tile_off_x; a->tile_off_y = tile_off_y;
    a->final_w = final_w; a->final_h = final_h;
    a->fast = 0;
    if (std::fabs(n.m[1]) <= DBL_EPSILON && std::fabs(n.m[2]) <= DBL_EPSILON) {
        if (n.kernel == Kernel::Nearest) a->fast = 1;
        else if (n.kernel == Kernel::Bilinear) a->fast = 2;
        else if (n.kernel == Kernel::Bicubic) a->fast = 3;
    }
    const bool constant_fill = n.extend == Extend::Black || n.extend == Extend::White || n.extend == Extend::Background;
    if (!constant_fill || (bands == 4 && !n.premultiplied)) a->fast = 0;
    a->separable = (n.m[1] == 0.0 && n.m[2] == 0.0) ? 1 : 0;
    return VIPRS_OK;
}

static int64_t tile_origin(int64_t v, int64_t off, int64_t t) {
    const int64_t d = v - off;
    const int64_t q = d >= 0 ? d / t : -((-d + t - 1) / t);
    return off + q * t;
}

void affine_axis_tables(const AffineArgs& a, double* xs, double* ys) {
    const double* m = a.m;
    for (uint32_t X = 0; X < a.total_w; ++X) {
        const int64_t X0 = tile_origin(X, a.tile_off_x, a.tile_w);
        double x = std::fma(m[1], 0.0, m[0] * double(X0)) + a.tx;
        for (int64_t c = X0; c < int64_t(X); ++c) x += m[0];
        xs[X] = x;
    }
    for (uint32_t Y = 0; Y < a.total_h; ++Y) {
        const int64_t Y0 = tile_origin(Y, a.tile_off_y, a.tile_h);
        double y = std::fma(m[3], double(Y0), m[2] * 0.0) + a.ty;
        for (int64_t r = Y0; r < int64_t(Y); ++r) y += m[3];
        ys[Y] = y;
    }
}

bool affine_weight_tables_apply(const AffineArgs& a) {
    return a.separable && !a.fast && a.kernel != 0 && a.kernel != 1;
}

void affine_weight_tables(const AffineArgs& a, const double* xs, const double* ys, double* wx, double* wy) {
    const int nt = separable_taps(a.kernel), support = nt / 2;
    auto axis = [&](const double* pos, uint32_t n, double* w) {
        for (uint32_t i = 0; i < n; ++i) {
            const double p = pos[i];
            if (!std::isfinite(p)) {  // the kernel fills such pixels without weights
                for (int t = 0; t < kAxisTaps; ++t) w[size_t(i) * kAxisTaps + t] = 0.0;
                continue;
            }
            const int64_t t0 = int64_t(std::floor(p)) - (support - 1);
            for (int t = 0; t < kAxisTaps; ++t)
                w[size_t(i) * kAxisTaps + t] = t < nt ? kernel_w(a.kernel, std::fabs(double(t0 + t) - p)) : 0.0;
        }
    };
    axis(xs, a.total_w, wx);
    axis(ys, a.total_h, wy);
}

}  // namespace viprs
