// plan.cpp -- host planning for the resample path.  See plan.hpp for the
// viprs files each function follows.  Compiled with -ffp-contract=off.
#include "plan.hpp"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>

#include "viprs_b200.h"

namespace viprs {

static constexpr double kEps = DBL_EPSILON;
static constexpr double kPi = 3.141592653589793;
static constexpr double kThumbEps = 1e-9;

int64_t f64_to_i64(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return static_cast<int64_t>(v);
}

uint32_t f64_to_u32(double v) {
    if (v != v || v <= 0.0) return 0;
    if (v >= 4294967295.0) return 4294967295u;
    return static_cast<uint32_t>(v);
}

// kernel.rs:50-61 (libvips bicubic, a = -0.5)
static double bicubic_weight(double x) {
    x = std::fabs(x);
    if (x < 1.0) return std::fma(2.5 * x, -x, 1.5 * x * x * x) + 1.0;
    if (x < 2.0) return std::fma(4.0, -x, std::fma(2.5 * x, x, -0.5 * x * x * x)) + 2.0;
    return 0.0;
}

// kernel.rs:133-214
double kernel_weight(Kernel k, double x) {
    switch (k) {
    case Kernel::Nearest: return std::fabs(x) < 0.5 ? 1.0 : 0.0;
    case Kernel::Bilinear: x = std::fabs(x); return x < 1.0 ? 1.0 - x : 0.0;
    case Kernel::Bicubic:
    case Kernel::CatmullRom:
    case Kernel::Lbb: return bicubic_weight(x);
    case Kernel::Quadratic:
        x = std::fabs(x);
        if (x < 0.5) return std::fma(2.0 * x, -x, 1.0);
        if (x < 1.5) return std::fma(2.5, -x, x * x) + 1.5;
        return 0.0;
    case Kernel::Nohalo:
        x = std::fabs(x);
        if (x < kEps) return 1.0;
        if (x < 2.5) {
            const double px = kPi * x;
            return (std::sin(px) / px) * (0.5 * (1.0 + std::cos(px / 2.5)));
        }
        return 0.0;
    case Kernel::Vsqbs:
        x = std::fabs(x);
        if (x < 0.5) return std::fma(x, -x, 0.75);
        if (x < 1.5) { const double e = x - 1.5; return 0.5 * e * e; }
        return 0.0;
    case Kernel::Lanczos2:
        x = std::fabs(x);
        if (x < kEps) return 1.0;
        if (x < 2.0) { const double p = kPi * x; return 2.0 * std::sin(p) * std::sin(p / 2.0) / (p * p); }
        return 0.0;
    case Kernel::Lanczos3:
        x = std::fabs(x);
        if (x < kEps) return 1.0;
        if (x < 3.0) { const double p = kPi * x; return 3.0 * std::sin(p) * std::sin(p / 3.0) / (p * p); }
        return 0.0;
    }
    return 0.0;
}

double kernel_support(Kernel k) {
    switch (k) {
    case Kernel::Nearest: return 0.5;
    case Kernel::Bilinear: return 1.0;
    case Kernel::Quadratic: return 1.5;
    case Kernel::Nohalo: return 2.5;
    case Kernel::Lanczos3: return 3.0;
    default: return 2.0;
    }
}

void kernel_affine_padding(Kernel k, int32_t* left, int32_t* right) {
    int32_t size = 4, off = 1;
    if (k == Kernel::Nearest) { size = 1; off = 0; }
    else if (k == Kernel::Bilinear) { size = 2; off = 0; }
    else if (k == Kernel::Nohalo || k == Kernel::Lanczos3) { size = 6; off = 2; }
    *left = off;
    *right = size - off - 1;
}

// validate_reduce_kernel (reduce_common.rs:93-124)
bool reduce_kernel_is_separable(Kernel k) {
    return !(k == Kernel::Lbb || k == Kernel::Vsqbs || k == Kernel::Nohalo);
}

// tap_count (reduce_common.rs:257-277)
static int32_t tap_count(Kernel k, double factor) {
    if (std::fabs(factor - 1.0) < kEps) return 1;
    if (k == Kernel::Nearest) return 1;
    const double r = std::round(kernel_support(k) * factor);
    if (!std::isfinite(r) || r < 0.0 || r > double((kMaxTaps - 1) / 2)) return -1;
    const int64_t taps = static_cast<int64_t>(r) * 2 + 1;
    return taps <= kMaxTaps ? static_cast<int32_t>(taps) : -1;
}

uint32_t reduce_output_len(double factor, uint32_t input_len) {
    if (input_len == 0) return 0;
    return f64_to_u32(std::round(double(input_len) / factor));
}

int ReduceKernel::init(double f, Kernel kernel) {
    if (!std::isfinite(f) || f < 1.0) return VIPRS_ERR_INVALID_ARGUMENT;
    if (!reduce_kernel_is_separable(kernel)) return VIPRS_ERR_INVALID_KERNEL;
    const int32_t t = tap_count(kernel, f);
    if (t < 0) return VIPRS_ERR_TOO_MANY_TAPS;
    factor = f;
    taps = t;
    pad_before = static_cast<int64_t>(std::ceil(double(t) / 2.0)) - 1;
    offset = 0.0;
    coeffs_f64.assign(size_t(t) * (kPhases + 1), 0.0);
    coeffs_i16.assign(size_t(t) * (kPhases + 1), 0);
    // build_coefficients + quantize_coefficients (reduce_common.rs:279-316)
    for (int p = 0; p <= kPhases; ++p) {
        double* row = &coeffs_f64[size_t(p) * t];
        if (kernel == Kernel::Nearest) {
            row[0] = 1.0;
        } else {
            const double half = double(p) / double(kPhases) + double(t) / 2.0 - 1.0;
            const double scale = 1.0 / f;
            double sum = 0.0;
            for (int32_t i = 0; i < t; ++i) {
                const double distance = (double(i) - half) * scale;
                const double w = kernel_weight(kernel, std::fabs(distance));
                row[i] = w;
                sum += w;
            }
            if (sum > 0.0)
                for (int32_t i = 0; i < t; ++i) row[i] /= sum;
        }
        for (int32_t i = 0; i < t; ++i)
            coeffs_i16[size_t(p) * t + i] = static_cast<int16_t>(f64_to_i64(row[i] * 4096.0));
    }
    return VIPRS_OK;
}

// bind_input_len (reduce_common.rs:166-175)
void ReduceKernel::bind_input_len(uint32_t input_len) {
    if (input_len == 0 || std::fabs(factor - 1.0) < kEps) { offset = 0.0; return; }
    const uint32_t out_len = reduce_output_len(factor, input_len);
    const double extra = std::fma(double(out_len), factor, -double(input_len));
    offset = (1.0 + extra) / 2.0 - 1.0;  // f64::midpoint(1.0, extra) - 1.0
}

double ReduceKernel::source_position(double index) const {
    return std::fma(index + 0.5, factor, -0.5) - offset;
}

// plan_for_source_position (reduce_common.rs:128-135)
void ReduceKernel::plan(double pos, int64_t* start, int32_t* phase) const {
    const double fl = std::floor(pos);
    double ph = std::round(std::fma(pos - fl, double(kPhases), 0.0));
    ph = std::min(std::max(ph, 0.0), double(kPhases));
    *phase = static_cast<int32_t>(ph);
    *start = f64_to_i64(fl) - pad_before;
}

void ReduceKernel::required_axis(int64_t o, int64_t len, int64_t* io, int64_t* il) const {
    if (len <= 0) { *io = o; *il = 0; return; }
    const int64_t first = f64_to_i64(std::floor(source_position(double(o))));
    const int64_t last = f64_to_i64(std::floor(source_position(double(o + len - 1))));
    *io = first - pad_before;
    *il = (last - pad_before + taps - 1) - *io + 1;
}

void ReduceKernel::config_required_axis(int64_t o, int64_t len, int64_t* io, int64_t* il) const {
    if (len <= 0) { *io = o; *il = 0; return; }
    const int64_t first = f64_to_i64(std::floor(std::fma(double(o) + 0.5, factor, -0.5)));
    const int64_t last = f64_to_i64(std::floor(std::fma(double(o + len - 1) + 0.5, factor, -0.5)));
    const int64_t s = first - pad_before, e = last - pad_before + taps - 1;
    if (e < 0) { *io = 0; *il = 0; return; }
    int64_t cs = std::min<int64_t>(std::max<int64_t>(s, 0), INT32_MAX);
    int64_t ce = std::min<int64_t>(std::max(e, cs), INT32_MAX);
    *io = cs;
    *il = ce - cs + 1;
}

int64_t ReduceKernel::max_abs_i16_sum() const {
    int64_t best = 0;
    for (int p = 0; p <= kPhases; ++p) {
        int64_t s = 0;
        for (int32_t i = 0; i < taps; ++i) s += std::abs(int64_t(coeffs_i16[size_t(p) * taps + i]));
        best = std::max(best, s);
    }
    return best;
}

// ------------------------------------------------------------------ thumbnail
static Kernel affine_kernel_for_resize(Kernel k) {
    return k == Kernel::Nearest ? Kernel::Nearest : (k == Kernel::Bilinear ? Kernel::Bilinear : Kernel::Bicubic);
}

static void target_dimensions(ThumbTarget t, uint32_t tw, uint32_t th, uint32_t iw, uint32_t ih,
                              uint32_t* ow, uint32_t* oh) {
    *ow = 1; *oh = 1;
    switch (t) {
    case ThumbTarget::FitBox: {
        const double hs = double(std::max(tw, 1u)) / double(iw);
        const double vs = double(std::max(th, 1u)) / double(ih);
        const double s = std::min(std::min(hs, vs), 1.0);
        *ow = f64_to_u32(std::max(std::round(double(iw) * s), 1.0));
        *oh = f64_to_u32(std::max(std::round(double(ih) * s), 1.0));
        return;
    }
    case ThumbTarget::ForceExact: *ow = std::max(tw, 1u); *oh = std::max(th, 1u); return;
    case ThumbTarget::Width: {
        const uint32_t w = std::min(std::max(tw, 1u), iw);
        *ow = w;
        *oh = f64_to_u32(std::max(std::round((double(ih) * double(w)) / double(iw)), 1.0));
        return;
    }
    case ThumbTarget::Height: {
        const uint32_t h = std::min(std::max(th, 1u), ih);
        *oh = h;
        *ow = f64_to_u32(std::max(std::round((double(iw) * double(h)) / double(ih)), 1.0));
        return;
    }
    }
}

static uint32_t choose_integer_shrink(uint32_t input_len, uint32_t target_len, double total) {
    if (total <= 1.0 + kThumbEps) return 1;
    uint32_t f = f64_to_u32(std::max(std::floor(total), 1.0));
    while (f > 1) {
        const uint32_t after = input_len / f;
        const double residual = total / double(f);
        const uint32_t ar = residual > 1.0 + kThumbEps ? f64_to_u32(std::max(std::round(double(after) / residual), 1.0)) : after;
        if (ar >= target_len) break;
        --f;
    }
    return f;
}

static uint32_t shrink_on_load_factor(double s) {
    if (s >= 16.0) return 16;
    if (s >= 8.0) return 4;
    if (s >= 4.0) return 2;
    return 0;
}

static PlanNode make_affine_node(double isx, double isy, Kernel kernel, uint32_t ow, uint32_t oh) {
    PlanNode a;
    a.kind = NodeKind::Affine;
    a.m[0] = isx; a.m[1] = 0.0; a.m[2] = 0.0; a.m[3] = isy;
    a.tx = kernel == Kernel::Nearest ? 0.0 : 0.5 * (1.0 - isx);
    a.ty = kernel == Kernel::Nearest ? 0.0 : 0.5 * (1.0 - isy);
    a.out_w = ow; a.out_h = oh;
    a.kernel = affine_kernel_for_resize(kernel);
    return a;
}

ThumbnailPlan thumbnail_plan(ThumbTarget target, uint32_t tw, uint32_t th, Kernel kernel, bool crop,
                             uint32_t in_w, uint32_t in_h, uint32_t bands, bool allow_shrink_hint) {
    ThumbnailPlan plan;
    if (in_w == 0 || in_h == 0) return plan;
    const bool allow_up = target == ThumbTarget::ForceExact;
    const bool single = in_w == 1 && in_h == 1;
    uint32_t t_w = 1, t_h = 1;
    if (crop && (target == ThumbTarget::FitBox || target == ThumbTarget::ForceExact)) {
        t_w = std::max(tw, 1u); t_h = std::max(th, 1u);
    } else {
        target_dimensions(target, tw, th, in_w, in_h, &t_w, &t_h);
    }
    if (allow_up && !single) { t_w = std::max(t_w, 1u); t_h = std::max(t_h, 1u); }
    else { t_w = std::max(std::min(t_w, in_w), 1u); t_h = std::max(std::min(t_h, in_h), 1u); }
    const bool has_alpha = bands == 2 || bands == 4;
    uint32_t g_w = t_w, g_h = t_h;
    if (crop) {
        const double hs = double(std::max(t_w, 1u)) / double(in_w), vs = double(std::max(t_h, 1u)) / double(in_h);
        const double cover = std::max(hs, vs);
        g_w = f64_to_u32(std::max(std::round(double(in_w) * cover), double(t_w)));
        g_h = f64_to_u32(std::max(std::round(double(in_h) * cover), double(t_h)));
    }
    if (allow_up && !single) { g_w = std::max(g_w, 1u); g_h = std::max(g_h, 1u); }
    else { g_w = std::max(std::min(g_w, in_w), 1u); g_h = std::max(std::min(g_h, in_h), 1u); }

    std::vector<PlanNode> geo;
    if (in_w == 1 || in_h == 1) {
        if (single) { t_w = 1; t_h = 1; }
        if (t_w != in_w || t_h != in_h)
            geo.push_back(make_affine_node(double(in_w) / double(t_w), double(in_h) / double(t_h), kernel, t_w, t_h));
    } else {
        double hshrink = double(in_w) / double(g_w), vshrink = double(in_h) / double(g_h);
        const uint32_t sol = allow_shrink_hint ? shrink_on_load_factor(std::min(hshrink, vshrink)) : 0;
        const uint32_t ew = sol ? std::max(in_w / sol, 1u) : in_w;
        const uint32_t eh = sol ? std::max(in_h / sol, 1u) : in_h;
        plan.shrink_factor = sol;
        hshrink = double(ew) / double(g_w);
        vshrink = double(eh) / double(g_h);
        const uint32_t ihs = choose_integer_shrink(ew, g_w, hshrink);
        const uint32_t ivs = choose_integer_shrink(eh, g_h, vshrink);
        const uint32_t asw = ew / std::max(ihs, 1u), ash = eh / std::max(ivs, 1u);
        const double rh = hshrink > 1.0 ? hshrink / double(ihs) : 1.0;
        const double rv = vshrink > 1.0 ? vshrink / double(ivs) : 1.0;
        const uint32_t arw = rh > 1.0 + kThumbEps ? f64_to_u32(std::max(std::round(double(asw) / rh), 1.0)) : asw;
        const uint32_t arh = rv > 1.0 + kThumbEps ? f64_to_u32(std::max(std::round(double(ash) / rv), 1.0)) : ash;
        PlanNode n;
        if (ihs > 1) { n = PlanNode(); n.kind = NodeKind::ShrinkH; n.ufactor = ihs; geo.push_back(n); }
        if (ivs > 1) { n = PlanNode(); n.kind = NodeKind::ShrinkV; n.ufactor = ivs; geo.push_back(n); }
        if (rh > 1.0 + kThumbEps) { n = PlanNode(); n.kind = NodeKind::ReduceH; n.factor = rh; n.kernel = kernel; geo.push_back(n); }
        if (rv > 1.0 + kThumbEps) { n = PlanNode(); n.kind = NodeKind::ReduceV; n.factor = rv; n.kernel = kernel; geo.push_back(n); }
        const double asx = double(g_w) / double(arw), asy = double(g_h) / double(arh);
        if (std::fabs(asx - 1.0) > kThumbEps || std::fabs(asy - 1.0) > kThumbEps)
            geo.push_back(make_affine_node(1.0 / asx, 1.0 / asy, kernel, g_w, g_h));
        if (crop && (g_w != t_w || g_h != t_h)) {
            n = PlanNode();
            n.kind = NodeKind::ExtractArea;
            n.ex = (g_w - t_w) / 2; n.ey = (g_h - t_h) / 2; n.ew = t_w; n.eh = t_h;
            geo.push_back(n);
        }
    }
    // wrap_geometry_nodes (thumbnail.rs:438-456)
    if (has_alpha && !geo.empty()) { PlanNode p; p.kind = NodeKind::Premultiply; plan.nodes.push_back(p); }
    for (auto& g : geo) plan.nodes.push_back(g);
    if (has_alpha && !geo.empty()) { PlanNode p; p.kind = NodeKind::Unpremultiply; plan.nodes.push_back(p); }
    plan.output_width = t_w;
    plan.output_height = t_h;
    return plan;
}

// ------------------------------------------------------------------ resize
static uint32_t scaled_len(uint32_t in, double s) { return f64_to_u32(std::max(std::round(double(in) * s), 1.0)); }
static uint32_t pre_shrink_factor(uint32_t in, uint32_t t, Kernel k, double gap) {
    if (t == 0 || in <= t || k == Kernel::Nearest) return 1;
    return f64_to_u32(std::max(std::floor(double(in) / double(t) / gap), 1.0));
}
static double affine_offset(double s, Kernel k) { return k == Kernel::Nearest ? 0.0 : 0.5 * (1.0 - 1.0 / s); }

ResizePlan resize_plan(double hscale, double vscale, Kernel kernel, double gap, uint32_t in_w, uint32_t in_h) {
    ResizePlan p;
    if (!(std::isfinite(hscale) && hscale > 0.0)) hscale = 1.0;
    if (!(std::isfinite(vscale) && vscale > 0.0)) vscale = 1.0;
    if (!(std::isfinite(gap) && gap >= 1.0)) gap = 2.0;
    if (in_w == 0 || in_h == 0) return p;
    const uint32_t t_w = scaled_len(in_w, hscale), t_h = scaled_len(in_h, vscale);
    const Kernel k = kernel == Kernel::Nohalo ? Kernel::Bicubic : kernel;
    p.output_width = t_w;
    p.output_height = t_h;
    auto affine = [&](double sx, double sy) {
        PlanNode n;
        n.kind = NodeKind::Affine;
        n.m[0] = 1.0 / sx; n.m[3] = 1.0 / sy;
        n.tx = affine_offset(sx, k); n.ty = affine_offset(sy, k);
        n.out_w = t_w; n.out_h = t_h; n.kernel = k;
        return n;
    };
    if (k == Kernel::Lbb) {
        if (t_w != in_w || t_h != in_h)
            p.nodes.push_back(affine(double(t_w) / double(in_w), double(t_h) / double(in_h)));
        return p;
    }
    uint32_t cw = in_w, ch = in_h;
    const uint32_t hs = t_w < cw ? pre_shrink_factor(cw, t_w, k, gap) : 1;
    const uint32_t vs = t_h < ch ? pre_shrink_factor(ch, t_h, k, gap) : 1;
    PlanNode n;
    if (vs > 1) { n = PlanNode(); n.kind = NodeKind::ShrinkV; n.ufactor = vs; p.nodes.push_back(n); ch /= vs; }
    if (hs > 1) { n = PlanNode(); n.kind = NodeKind::ShrinkH; n.ufactor = hs; p.nodes.push_back(n); cw /= hs; }
    if (t_h < ch) { n = PlanNode(); n.kind = NodeKind::ReduceV; n.factor = double(ch) / double(t_h); n.kernel = k; p.nodes.push_back(n); ch = t_h; }
    if (t_w < cw) { n = PlanNode(); n.kind = NodeKind::ReduceH; n.factor = double(cw) / double(t_w); n.kernel = k; p.nodes.push_back(n); cw = t_w; }
    const bool can_zoom = k != Kernel::Vsqbs;
    const uint32_t zx = can_zoom && t_w > cw ? t_w / cw : 1, zy = can_zoom && t_h > ch ? t_h / ch : 1;
    if (zx > 1 || zy > 1) {
        n = PlanNode(); n.kind = NodeKind::Zoom; n.zx = zx; n.zy = zy; p.nodes.push_back(n);
        cw *= zx; ch *= zy;
    }
    const double asx = double(t_w) / double(cw), asy = double(t_h) / double(ch);
    if (std::fabs(asx - 1.0) > kThumbEps || std::fabs(asy - 1.0) > kThumbEps) p.nodes.push_back(affine(asx, asy));
    return p;
}

// ------------------------------------------------------------------ builder
int node_output_dims(const PlanNode& n, uint32_t iw, uint32_t ih, uint32_t* ow, uint32_t* oh) {
    switch (n.kind) {
    case NodeKind::ShrinkH:
        if (n.ufactor == 0) return VIPRS_ERR_INVALID_ARGUMENT;
        *ow = n.ceil ? (iw + n.ufactor - 1) / n.ufactor : iw / n.ufactor; *oh = ih; return VIPRS_OK;
    case NodeKind::ShrinkV:
        if (n.ufactor == 0) return VIPRS_ERR_INVALID_ARGUMENT;
        *ow = iw; *oh = n.ceil ? (ih + n.ufactor - 1) / n.ufactor : ih / n.ufactor; return VIPRS_OK;
    case NodeKind::Shrink:
        if (n.ufactor == 0 || n.vufactor == 0) return VIPRS_ERR_INVALID_ARGUMENT;
        *ow = iw / n.ufactor; *oh = ih / n.vufactor; return VIPRS_OK;
    case NodeKind::ReduceH: *ow = reduce_output_len(n.factor, iw); *oh = ih; return VIPRS_OK;
    case NodeKind::ReduceV: *ow = iw; *oh = reduce_output_len(n.factor, ih); return VIPRS_OK;
    case NodeKind::Reduce: *ow = reduce_output_len(n.factor, iw); *oh = reduce_output_len(n.vfactor, ih); return VIPRS_OK;
    case NodeKind::Affine: *ow = n.out_w; *oh = n.out_h; return VIPRS_OK;
    case NodeKind::ExtractArea:
        if (uint64_t(n.ex) + n.ew > iw || uint64_t(n.ey) + n.eh > ih) return VIPRS_ERR_INVALID_ARGUMENT;
        *ow = n.ew; *oh = n.eh; return VIPRS_OK;
    case NodeKind::Zoom:
        // PipelineBuilder::zoom rejects a zero factor (builder/geometry.rs:618-624)
        if (n.zx == 0 || n.zy == 0) return VIPRS_ERR_INVALID_ARGUMENT;
        if (uint64_t(iw) * n.zx > 0xFFFFFFFFull || uint64_t(ih) * n.zy > 0xFFFFFFFFull) return VIPRS_ERR_INVALID_ARGUMENT;
        *ow = iw * n.zx; *oh = ih * n.zy; return VIPRS_OK;
    default: *ow = iw; *oh = ih; return VIPRS_OK;
    }
}

int builder_thumbnail_chain(uint32_t w, uint32_t h, uint32_t bands, ThumbTarget target, uint32_t tw,
                            uint32_t th, Kernel kernel, bool crop, Chain* out) {
    if (bands == 0) return VIPRS_ERR_INVALID_ARGUMENT;  // Thumbnail::validate_input
    ThumbnailPlan plan = thumbnail_plan(target, tw, th, kernel, crop, w, h, bands, true);
    // an in-memory source declines shrink-on-load (viprs-ports/src/source.rs:257-259),
    // so the builder re-plans without the hint (builder/resample.rs:878-906)
    if (plan.shrink_factor) plan = thumbnail_plan(target, tw, th, kernel, crop, w, h, bands, false);
    const bool large = w > 512 || h > 512;
    out->nodes.clear();
    out->out_w = plan.output_width;
    out->out_h = plan.output_height;
    out->demand_override = large ? int32_t(Demand::ThinStrip) : -1;
    if (plan.nodes.empty()) {
        // builder.affine(identity, 0, 0, out_w, out_h, Nearest): Background(0), SmallTile
        PlanNode a;
        a.kind = NodeKind::Affine;
        a.kernel = Kernel::Nearest;
        a.out_w = plan.output_width; a.out_h = plan.output_height;
        a.extend = Extend::Background; a.background = 0.0;
        a.demand = Demand::SmallTile;
        out->nodes.push_back(a);
        return VIPRS_OK;
    }
    for (PlanNode n : plan.nodes) {
        n.demand = Demand::ThinStrip;
        if (n.kind == NodeKind::Affine) {
            n.extend = Extend::Copy;
            n.demand = large ? Demand::ThinStrip : Demand::SmallTile;
        }
        out->nodes.push_back(n);
    }
    return VIPRS_OK;
}

int builder_resize_chain(uint32_t w, uint32_t h, uint32_t bands, double hscale, double vscale,
                         Kernel kernel, Chain* out) {
    if (bands == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    ResizePlan plan = resize_plan(hscale, vscale, kernel, 2.0, w, h);
    out->nodes.clear();
    out->out_w = plan.output_width;
    out->out_h = plan.output_height;
    out->demand_override = -1;
    for (PlanNode n : plan.nodes) {
        n.demand = Demand::ThinStrip;
        if (n.kind == NodeKind::Affine) { n.extend = Extend::Copy; n.demand = Demand::SmallTile; }
        if (n.kind == NodeKind::Zoom) n.demand = Demand::FatStrip;  // ZoomBridge's hint
        out->nodes.push_back(n);
    }
    return VIPRS_OK;
}

// round_vips (resample/similarity.rs:223-230): half away from zero, then
// Rust's saturating `as i32`.
static int32_t round_vips(double v) {
    const double r = v > 0.0 ? v + 0.5 : v - 0.5;
    if (!(r == r)) return 0;
    if (r >= 2147483647.0) return INT32_MAX;
    if (r <= -2147483648.0) return INT32_MIN;
    return int32_t(r);
}

PlanNode similarity_node(double scale, double angle, Kernel kernel, uint32_t in_w, uint32_t in_h) {
    const double s = std::isfinite(scale) && scale > 0.0 ? scale : 1.0;  // safe_scale (:178-185)
    const double rad = angle * (kPi / 180.0);                            // f64::to_radians
    const double c = std::cos(rad), sn = std::sin(rad);
    // auto_canvas (:191-221) of the forward matrix
    const double a = s * c, b = s * -sn, cc = s * sn, d = s * c;
    int32_t left = 0, top = 0, cw = 0, ch = 0;
    if (in_w != 0 && in_h != 0) {
        const double W = double(in_w), H = double(in_h);
        const double x2 = a * W, y2 = cc * W, x3 = b * H, y3 = d * H;
        const double x4 = std::fma(b, H, a * W), y4 = std::fma(d, H, cc * W);
        const double l = std::fmin(std::fmin(std::fmin(0.0, x2), x3), x4);
        const double r = std::fmax(std::fmax(std::fmax(0.0, x2), x3), x4);
        const double t = std::fmin(std::fmin(std::fmin(0.0, y2), y3), y4);
        const double bt = std::fmax(std::fmax(std::fmax(0.0, y2), y3), y4);
        left = round_vips(l);
        top = round_vips(t);
        cw = std::max(round_vips(r - l), 0);
        ch = std::max(round_vips(bt - t), 0);
    }
    PlanNode n;
    n.kind = NodeKind::Affine;
    // inverse_similarity_matrix (:187-189), translation of the canvas origin (:66-67)
    n.m[0] = c / s; n.m[1] = sn / s; n.m[2] = -sn / s; n.m[3] = c / s;
    n.tx = std::fma(n.m[1], double(top), n.m[0] * double(left));
    n.ty = std::fma(n.m[3], double(top), n.m[2] * double(left));
    n.out_w = uint32_t(cw); n.out_h = uint32_t(ch);
    n.kernel = kernel;
    n.extend = Extend::Background;  // Affine::new's Background(0)
    n.background = 0.0;
    n.demand = Demand::SmallTile;   // SimilarityBridge's hint
    return n;
}

int forward_affine_to_backward(const double f[4], double tx, double ty, double b[4], double* btx, double* bty) {
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(f[i])) return VIPRS_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(tx) || !std::isfinite(ty)) return VIPRS_ERR_INVALID_ARGUMENT;
    const double det = std::fma(f[0], f[3], -f[1] * f[2]);
    if (std::fabs(det) <= kEps) return VIPRS_ERR_DEGENERATE_AFFINE;
    const double inv = 1.0 / det;
    b[0] = f[3] * inv; b[1] = -f[1] * inv; b[2] = -f[2] * inv; b[3] = f[0] * inv;
    *btx = -std::fma(b[1], ty, b[0] * tx);
    *bty = -std::fma(b[3], ty, b[2] * tx);
    return VIPRS_OK;
}

void tile_geometry(Demand hint, uint32_t w, uint32_t h, uint32_t* tw, uint32_t* th) {
    *tw = hint == Demand::SmallTile ? 128 : w;
    uint32_t t;
    switch (hint) {
    case Demand::SmallTile: t = 128; break;
    case Demand::ThinStrip: t = w > 10000 ? 1 : 16; break;
    case Demand::FullImage: t = h; break;
    case Demand::OneLine: t = 1; break;
    default: t = h <= 1024 ? 256 : (h >= 4096 ? 64 : 16); break;
    }
    *th = std::max(std::min(t, h), 1u);
    if (*tw == 0) *tw = 1;
}

}  // namespace viprs
