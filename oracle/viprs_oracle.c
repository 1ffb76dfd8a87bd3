/*
 * viprs_oracle.c -- CPU restatement of viprs 0.1.5's resample hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the bench's
 * CPU-baseline leg load this library to check or time the CUDA path.  The
 * product never links or calls it.
 *
 * Build: gcc -O2 -fPIC -shared -ffp-contract=off -fno-fast-math -pthread
 * (oracle/build_oracle.py).  -ffp-contract=off matters: viprs fuses a
 * multiply-add only where it calls `mul_add`, and this file calls fma() at
 * exactly those places.
 *
 * Semantics restated (file:line in the viprs tree):
 *   kernel weights ............ crates/viprs-core/src/kernel.rs:50-214
 *   ReduceKernel .............. crates/viprs-ops-spatial/src/resample/reduce_common.rs:128-316
 *   fixed-point rounding ...... resample/sample_conv.rs:24-33, viprs-core shared_ops/sample_conv.rs
 *   ReduceH / ReduceV ......... resample/reduceh.rs:100-163, reducev.rs:99-162,
 *                               reduce_simd.rs:48-144 (scalar), :2421-2888 (x86 AVX2 order)
 *   ReduceOp .................. resample/reduce.rs:37-264
 *   ShrinkH / ShrinkV ......... resample/shrinkh.rs:44-128,255-874, shrinkv.rs:153-537
 *   Premultiply/Unpremultiply . structural/premultiply.rs:84-121, structural/unpremultiply.rs:76-113
 *   Affine .................... resample/affine/core.rs, affine/interpolation.rs:43-137
 *   MapIm ..................... resample/mapim.rs:290-420, 1043-1274
 *   Thumbnail / Resize plans .. resample/thumbnail.rs:204-524, resample/resize.rs:163-348
 *   Builder materialisation ... viprs-runtime/src/pipeline/builder/resample.rs:25-60,637-711,871-979
 *   Tile geometry ............. viprs-core/src/op/demand.rs:41-83,
 *                               viprs-runtime/src/scheduler/rayon_scheduler/planning.rs:550-596
 *   Region propagation ........ rayon_scheduler/execute.rs:389-480 (required regions are
 *                               propagated unclipped; only the source read edge-replicates,
 *                               viprs-runtime/src/sources/memory.rs:186-215)
 */
#include "viprs_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define OR_PHASES 64
#define OR_MAX_TAPS 2000
#define OR_MAX_TAP_RADIUS ((OR_MAX_TAPS - 1) / 2)
#define OR_EPS DBL_EPSILON
#define OR_PI 3.141592653589793
#define THUMB_EPS 1e-9

typedef struct { int64_t x, y, w, h; } reg_t;

static inline int64_t f2i(double v) {
    /* Rust `f64 as i64`: truncation toward zero, saturating, NaN -> 0. */
    if (v != v) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}
static inline uint32_t f2u32(double v) {
    if (v != v || v <= 0.0) return 0;
    if (v >= 4294967295.0) return 4294967295u;
    return (uint32_t)v;
}
static inline double clampd(double v, double lo, double hi) {
    /* Rust f64::clamp: NaN stays NaN */
    if (v < lo) return lo;
    if (v > hi) return hi;
    return v;
}
static inline int64_t clampi(int64_t v, int64_t lo, int64_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

/* ------------------------------------------------------------------ */
/* kernel.rs:133-214                                                   */
/* ------------------------------------------------------------------ */
static double bicubic_w(double x) {
    x = fabs(x);
    if (x < 1.0) return fma(2.5 * x, -x, 1.5 * x * x * x) + 1.0;
    if (x < 2.0) return fma(4.0, -x, fma(2.5 * x, x, -0.5 * x * x * x)) + 2.0;
    return 0.0;
}

double or_kernel_weight(int32_t k, double x) {
    switch (k) {
    case OR_K_NEAREST: return fabs(x) < 0.5 ? 1.0 : 0.0;
    case OR_K_BILINEAR: x = fabs(x); return x < 1.0 ? 1.0 - x : 0.0;
    case OR_K_BICUBIC:
    case OR_K_CATMULLROM:
    case OR_K_LBB: return bicubic_w(x);
    case OR_K_QUADRATIC:
        x = fabs(x);
        if (x < 0.5) return fma(2.0 * x, -x, 1.0);
        if (x < 1.5) return fma(2.5, -x, x * x) + 1.5;
        return 0.0;
    case OR_K_NOHALO: {
        x = fabs(x);
        if (x < OR_EPS) return 1.0;
        if (x < 2.5) {
            double pi_x = OR_PI * x;
            double sinc = sin(pi_x) / pi_x;
            double window = 0.5 * (1.0 + cos(pi_x / 2.5));
            return sinc * window;
        }
        return 0.0;
    }
    case OR_K_VSQBS:
        x = fabs(x);
        if (x < 0.5) return fma(x, -x, 0.75);
        if (x < 1.5) { double e = x - 1.5; return 0.5 * e * e; }
        return 0.0;
    case OR_K_LANCZOS2: {
        x = fabs(x);
        if (x < OR_EPS) return 1.0;
        if (x < 2.0) { double p = OR_PI * x; return 2.0 * sin(p) * sin(p / 2.0) / (p * p); }
        return 0.0;
    }
    case OR_K_LANCZOS3: {
        x = fabs(x);
        if (x < OR_EPS) return 1.0;
        if (x < 3.0) { double p = OR_PI * x; return 3.0 * sin(p) * sin(p / 3.0) / (p * p); }
        return 0.0;
    }
    default: return 0.0;
    }
}

double or_kernel_support(int32_t k) {
    switch (k) {
    case OR_K_NEAREST: return 0.5;
    case OR_K_BILINEAR: return 1.0;
    case OR_K_QUADRATIC: return 1.5;
    case OR_K_NOHALO: return 2.5;
    case OR_K_LANCZOS3: return 3.0;
    default: return 2.0;
    }
}

/* affine_padding (kernel.rs:79-115) */
static void kernel_padding(int32_t k, int32_t *left, int32_t *right) {
    int32_t size, off;
    switch (k) {
    case OR_K_NEAREST: size = 1; off = 0; break;
    case OR_K_BILINEAR: size = 2; off = 0; break;
    case OR_K_NOHALO: case OR_K_LANCZOS3: size = 6; off = 2; break;
    default: size = 4; off = 1; break;
    }
    *left = off; *right = size - off - 1;
}

/* ------------------------------------------------------------------ */
/* ReduceKernel (reduce_common.rs:128-316)                             */
/* ------------------------------------------------------------------ */
typedef struct {
    double factor;
    int32_t taps;
    int64_t pad_before;
    double offset;
    double *c64;
    int16_t *c16;
} rk_t;

static int32_t tap_count(int32_t kernel, double factor) {
    if (fabs(factor - 1.0) < OR_EPS) return 1;
    if (kernel == OR_K_NEAREST) return 1;
    double r = round(or_kernel_support(kernel) * factor);
    if (!isfinite(r) || r < 0.0 || r > (double)OR_MAX_TAP_RADIUS) return -1;
    int64_t taps = (int64_t)r * 2 + 1;
    return taps <= OR_MAX_TAPS ? (int32_t)taps : -1;
}

static void build_coefficients(int32_t kernel, int32_t taps, double factor, double phase,
                               double *out) {
    if (kernel == OR_K_NEAREST) { out[0] = 1.0; return; }
    double half = phase + (double)taps / 2.0 - 1.0;
    double scale = 1.0 / factor;
    double sum = 0.0;
    for (int32_t t = 0; t < taps; t++) {
        double distance = ((double)t - half) * scale;
        double w = or_kernel_weight(kernel, fabs(distance));
        out[t] = w;
        sum += w;
    }
    if (sum > 0.0)
        for (int32_t t = 0; t < taps; t++) out[t] /= sum;
}

static uint32_t reduce_output_len(double factor, uint32_t input_len) {
    /* ReduceConfig::output_len (viprs-core/src/resample.rs:92-98) */
    if (input_len == 0) return 0;
    return f2u32(round((double)input_len / factor));
}

static int validate_reduce_kernel(int32_t k) {
    return !(k == OR_K_LBB || k == OR_K_VSQBS || k == OR_K_NOHALO);
}

static int32_t rk_init(rk_t *rk, double factor, int32_t kernel) {
    memset(rk, 0, sizeof(*rk));
    if (!isfinite(factor) || factor < 1.0) return OR_EINVAL;
    if (!validate_reduce_kernel(kernel)) return OR_EINVAL;
    int32_t taps = tap_count(kernel, factor);
    if (taps < 0) return OR_ETAPS;
    rk->factor = factor;
    rk->taps = taps;
    rk->pad_before = (int64_t)ceil((double)taps / 2.0) - 1;
    rk->offset = 0.0;
    rk->c64 = (double *)malloc(sizeof(double) * (size_t)taps * (OR_PHASES + 1));
    rk->c16 = (int16_t *)malloc(sizeof(int16_t) * (size_t)taps * (OR_PHASES + 1));
    if (!rk->c64 || !rk->c16) { free(rk->c64); free(rk->c16); return OR_ENOMEM; }
    for (int p = 0; p <= OR_PHASES; p++) {
        double *row = rk->c64 + (size_t)p * taps;
        build_coefficients(kernel, taps, factor, (double)p / (double)OR_PHASES, row);
        for (int32_t t = 0; t < taps; t++)
            rk->c16[(size_t)p * taps + t] = (int16_t)f2i(row[t] * 4096.0);
    }
    return OR_OK;
}

static void rk_free(rk_t *rk) { free(rk->c64); free(rk->c16); rk->c64 = NULL; rk->c16 = NULL; }

static void rk_bind(rk_t *rk, uint32_t input_len) {
    if (input_len == 0 || fabs(rk->factor - 1.0) < OR_EPS) { rk->offset = 0.0; return; }
    uint32_t out_len = reduce_output_len(rk->factor, input_len);
    double extra = fma((double)out_len, rk->factor, -(double)input_len);
    /* f64::midpoint(1.0, extra) for finite, moderate values is (a + b) / 2 */
    rk->offset = (1.0 + extra) / 2.0 - 1.0;
}

static inline double rk_pos(const rk_t *rk, double index) {
    return fma(index + 0.5, rk->factor, -0.5) - rk->offset;
}

static inline void rk_plan(const rk_t *rk, double pos, int64_t *start, int32_t *phase) {
    double fl = floor(pos);
    double ph = round(fma(pos - fl, (double)OR_PHASES, 0.0));
    ph = clampd(ph, 0.0, (double)OR_PHASES);
    *phase = (int32_t)ph;
    *start = f2i(fl) - rk->pad_before;
}

int32_t or_reduce_tables(double factor, int32_t kernel, uint32_t input_len, int32_t bind,
                         int32_t *taps, int64_t *pad_before, double *offset,
                         double *coeffs_f64, int16_t *coeffs_i16) {
    rk_t rk;
    int32_t st = rk_init(&rk, factor, kernel);
    if (st) return st;
    if (bind) rk_bind(&rk, input_len);
    if (taps) *taps = rk.taps;
    if (pad_before) *pad_before = rk.pad_before;
    if (offset) *offset = rk.offset;
    size_t n = (size_t)rk.taps * (OR_PHASES + 1);
    if (coeffs_f64) memcpy(coeffs_f64, rk.c64, n * sizeof(double));
    if (coeffs_i16) memcpy(coeffs_i16, rk.c16, n * sizeof(int16_t));
    rk_free(&rk);
    return OR_OK;
}

void or_reduce_plan(double factor, int32_t kernel, uint32_t input_len, int32_t bind,
                    double index, int64_t *start, int32_t *phase, double *position) {
    rk_t rk;
    if (rk_init(&rk, factor, kernel)) { *start = 0; *phase = 0; *position = 0; return; }
    if (bind) rk_bind(&rk, input_len);
    double p = rk_pos(&rk, index);
    rk_plan(&rk, p, start, phase);
    *position = p;
    rk_free(&rk);
}

/* fixed-point to sample (resample/sample_conv.rs:24-33) */
static inline int64_t fixed_round(int64_t v) { return (v + 2048) >> 12; }
static inline uint8_t fixed_u8(int64_t v) { return (uint8_t)clampi(fixed_round(v), 0, 255); }
static inline uint16_t fixed_u16(int64_t v) { return (uint16_t)clampi(fixed_round(v), 0, 65535); }

/* FromF64 (viprs-core/src/shared_ops/sample_conv.rs): clamp then round */
static inline uint8_t from_f64_u8(double v) {
    v = clampd(v, 0.0, 255.0);
    return (uint8_t)f2u32(round(v));
}
static inline uint16_t from_f64_u16(double v) {
    v = clampd(v, 0.0, 65535.0);
    return (uint16_t)f2u32(round(v));
}

/* ------------------------------------------------------------------ */
/* tiles                                                               */
/* ------------------------------------------------------------------ */
typedef struct {
    reg_t r;
    int32_t bands;
    int32_t fmt;
    void *data;
} tile_t;

static inline size_t fmt_size(int32_t fmt) { return fmt == OR_U8 ? 1 : (fmt == OR_U16 ? 2 : 4); }

static inline double tget(const tile_t *t, size_t idx) {
    switch (t->fmt) {
    case OR_U8: return (double)((const uint8_t *)t->data)[idx];
    case OR_U16: return (double)((const uint16_t *)t->data)[idx];
    default: return (double)((const float *)t->data)[idx];
    }
}
static inline void tset_f64(tile_t *t, size_t idx, double v) {
    switch (t->fmt) {
    case OR_U8: ((uint8_t *)t->data)[idx] = from_f64_u8(v); break;
    case OR_U16: ((uint16_t *)t->data)[idx] = from_f64_u16(v); break;
    default: ((float *)t->data)[idx] = (float)v; break;
    }
}

static int tile_alloc(tile_t *t, reg_t r, int32_t bands, int32_t fmt) {
    t->r = r; t->bands = bands; t->fmt = fmt;
    size_t n = (size_t)(r.w > 0 ? r.w : 0) * (size_t)(r.h > 0 ? r.h : 0) * (size_t)bands *
               fmt_size(fmt);
    t->data = calloc(n ? n : 1, 1);
    return t->data ? 0 : -1;
}

static inline size_t clamp_axis(int64_t abs, int64_t origin, int64_t len) {
    /* reduce_common.rs:318-322 */
    int64_t rel = abs - origin;
    int64_t hi = len > 0 ? len - 1 : 0;
    return (size_t)clampi(rel, 0, hi);
}

/* ------------------------------------------------------------------ */
/* node runtime                                                        */
/* ------------------------------------------------------------------ */
typedef struct {
    or_node n;
    uint32_t in_w, in_h, out_w, out_h;
    int32_t bands, fmt;
    rk_t rk, rk2; /* reduce tables (REDUCE uses rk for h, rk2 for v) */
    /* affine fast path tables */
    int32_t fast; /* 0 none, 1 nearest, 2 bilinear, 3 bicubic */
    int64_t *xs, *ys;
    double *xw, *yw;
} node_rt;

/* ---------------- shrink ---------------- */
static void shrinkh_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const size_t f = nd->n.ufactor, bands = (size_t)in->bands;
    const size_t in_stride = (size_t)in->r.w, out_w = (size_t)out->r.w, out_h = (size_t)out->r.h;
    if (in->fmt == OR_U8) {
        const uint8_t *src = (const uint8_t *)in->data;
        uint8_t *dst = (uint8_t *)out->data;
        const uint64_t amend = f / 2;
        const uint64_t mult = ((uint64_t)1 << 32) / (((uint64_t)1 << 8) * f);
        for (size_t y = 0; y < out_h; y++) {
            const uint8_t *row = src + y * in_stride * bands;
            uint8_t *orow = dst + y * out_w * bands;
            for (size_t x = 0; x < out_w; x++) {
                const uint8_t *px = row + x * f * bands;
                for (size_t b = 0; b < bands; b++) {
                    uint64_t sum = 0;
                    for (size_t k = 0; k < f; k++) sum += px[k * bands + b];
                    uint8_t v;
                    if (f == 1) v = px[b];
                    else if (f == 2) v = (uint8_t)((sum + 1) >> 1);
                    else if (f == 5 && (bands == 1 || bands == 3 || bands == 4))
                        v = (uint8_t)((sum + 2) / 5);
                    else v = (uint8_t)(((sum + amend) * mult) >> 24);
                    orow[x * bands + b] = v;
                }
            }
        }
        return;
    }
    const double inv = 1.0 / (double)f;
    for (size_t y = 0; y < out_h; y++)
        for (size_t x = 0; x < out_w; x++)
            for (size_t b = 0; b < bands; b++) {
                double sum = 0.0;
                for (size_t k = 0; k < f; k++)
                    sum += tget(in, (y * in_stride + x * f + k) * bands + b);
                double v = sum * inv;
                size_t o = (y * out_w + x) * bands + b;
                if (out->fmt == OR_U16) {
                    double r = clampd(round(v), 0.0, 65535.0);
                    ((uint16_t *)out->data)[o] = (uint16_t)f2u32(r);
                } else {
                    ((float *)out->data)[o] = (float)v;
                }
            }
}

static void shrinkv_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const size_t f = nd->n.ufactor, bands = (size_t)in->bands;
    const size_t out_w = (size_t)out->r.w, out_h = (size_t)out->r.h;
    const size_t row_len = out_w * bands;
    if (in->fmt == OR_U8) {
        const uint8_t *src = (const uint8_t *)in->data;
        uint8_t *dst = (uint8_t *)out->data;
        const uint64_t amend = f / 2;
        const uint64_t mult = (uint32_t)(((uint64_t)1 << 32) / (((uint64_t)1 << 8) * f));
        for (size_t y = 0; y < out_h; y++)
            for (size_t i = 0; i < row_len; i++) {
                uint8_t v;
                if (f == 1) v = src[y * row_len + i];
                else if (f == 2)
                    v = (uint8_t)(((uint32_t)src[(2 * y) * row_len + i] +
                                   src[(2 * y + 1) * row_len + i] + 1) >> 1);
                else {
                    uint64_t sum = amend;
                    for (size_t k = 0; k < f; k++) sum += src[(y * f + k) * row_len + i];
                    v = (uint8_t)((sum * mult) >> 24);
                }
                dst[y * row_len + i] = v;
            }
        return;
    }
    const double inv = 1.0 / (double)f;
    for (size_t y = 0; y < out_h; y++)
        for (size_t i = 0; i < row_len; i++) {
            double sum = 0.0;
            for (size_t k = 0; k < f; k++) sum += tget(in, (y * f + k) * row_len + i);
            double v = sum * inv;
            size_t o = y * row_len + i;
            if (out->fmt == OR_U16) {
                double r = clampd(round(v), 0.0, 65535.0);
                ((uint16_t *)out->data)[o] = (uint16_t)f2u32(r);
            } else {
                ((float *)out->data)[o] = (float)v;
            }
        }
}

/* ---------------- reduce ---------------- */
static void reduceh_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const rk_t *rk = &nd->rk;
    const size_t bands = (size_t)in->bands, out_w = (size_t)out->r.w, out_h = (size_t)out->r.h;
    const size_t in_w = (size_t)in->r.w;
    const int32_t taps = rk->taps;
    int64_t *starts = (int64_t *)malloc(sizeof(int64_t) * (out_w ? out_w : 1));
    int32_t *phases = (int32_t *)malloc(sizeof(int32_t) * (out_w ? out_w : 1));
    if (in->fmt == OR_U8) {
        /* reduceh.rs:102-130: positions accumulated by `+= factor` from the tile's x */
        double sx = rk_pos(rk, (double)out->r.x);
        for (size_t x = 0; x < out_w; x++) {
            rk_plan(rk, sx, &starts[x], &phases[x]);
            sx += rk->factor;
        }
    } else {
        for (size_t x = 0; x < out_w; x++) {
            double sx = rk_pos(rk, (double)out->r.x + (double)x);
            rk_plan(rk, sx, &starts[x], &phases[x]);
        }
    }
    for (size_t y = 0; y < out_h; y++)
        for (size_t x = 0; x < out_w; x++) {
            const int64_t s = starts[x];
            const int16_t *c16 = rk->c16 + (size_t)phases[x] * taps;
            const double *c64 = rk->c64 + (size_t)phases[x] * taps;
            for (size_t b = 0; b < bands; b++) {
                size_t o = (y * out_w + x) * bands + b;
                if (in->fmt == OR_U8 || in->fmt == OR_U16) {
                    int64_t acc = 0;
                    for (int32_t t = 0; t < taps; t++) {
                        size_t tx = clamp_axis(s + t, in->r.x, in->r.w);
                        acc += (int64_t)c16[t] * (int64_t)tget(in, (y * in_w + tx) * bands + b);
                    }
                    if (in->fmt == OR_U8) ((uint8_t *)out->data)[o] = fixed_u8(acc);
                    else ((uint16_t *)out->data)[o] = fixed_u16(acc);
                } else if (bands == 1) {
                    /* reduce_h_f32_avx2_pixel (reduce_simd.rs:2621-2694) */
                    double acc = 0.0;
                    int32_t t = 0;
                    for (; t + 4 <= taps; t += 4) {
                        double p[4];
                        for (int l = 0; l < 4; l++) {
                            size_t tx = clamp_axis(s + t + l, in->r.x, in->r.w);
                            p[l] = tget(in, (y * in_w + tx)) * c64[t + l];
                        }
                        double lanes = -0.0;
                        for (int l = 0; l < 4; l++) lanes += p[l];
                        acc += lanes;
                    }
                    for (; t < taps; t++) {
                        size_t tx = clamp_axis(s + t, in->r.x, in->r.w);
                        acc = fma(tget(in, (y * in_w + tx)), c64[t], acc);
                    }
                    ((float *)out->data)[o] = (float)acc;
                } else {
                    /* reduce_h_scalar (reduce_simd.rs:48-90) */
                    double acc = 0.0;
                    for (int32_t t = 0; t < taps; t++) {
                        size_t tx = clamp_axis(s + t, in->r.x, in->r.w);
                        acc = fma(tget(in, (y * in_w + tx) * bands + b), c64[t], acc);
                    }
                    ((float *)out->data)[o] = (float)acc;
                }
            }
        }
    free(starts);
    free(phases);
}

static void reducev_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const rk_t *rk = &nd->rk;
    const size_t bands = (size_t)in->bands, out_w = (size_t)out->r.w, out_h = (size_t)out->r.h;
    const size_t row_stride = (size_t)in->r.w * bands, row_len = out_w * bands;
    const size_t vector_len = row_len / 4 * 4; /* AVX2_F32_LANES */
    const int32_t taps = rk->taps;
    for (size_t y = 0; y < out_h; y++) {
        /* x86 AVX2 kernels recompute the position per row (reduce_simd.rs:2716-2717) */
        double sy = rk_pos(rk, (double)out->r.y + (double)y);
        int64_t s;
        int32_t ph;
        rk_plan(rk, sy, &s, &ph);
        const int16_t *c16 = rk->c16 + (size_t)ph * taps;
        const double *c64 = rk->c64 + (size_t)ph * taps;
        for (size_t i = 0; i < row_len; i++) {
            size_t o = y * row_len + i;
            if (in->fmt == OR_U8 || in->fmt == OR_U16) {
                int64_t acc = 0;
                for (int32_t t = 0; t < taps; t++) {
                    size_t ty = clamp_axis(s + t, in->r.y, in->r.h);
                    acc += (int64_t)c16[t] * (int64_t)tget(in, ty * row_stride + i);
                }
                if (in->fmt == OR_U8) ((uint8_t *)out->data)[o] = fixed_u8(acc);
                else ((uint16_t *)out->data)[o] = fixed_u16(acc);
            } else {
                double acc = 0.0;
                for (int32_t t = 0; t < taps; t++) {
                    size_t ty = clamp_axis(s + t, in->r.y, in->r.h);
                    double v = tget(in, ty * row_stride + i);
                    if (i < vector_len) acc += v * c64[t]; /* _mm256_mul_pd then add */
                    else acc = fma(v, c64[t], acc);
                }
                ((float *)out->data)[o] = (float)acc;
            }
        }
    }
}

/* ReduceConfig-based regions (viprs-core/src/resample.rs:74-215) used by ReduceOp */
static void cfg_axis_bounds(int64_t start, int64_t end, int64_t *o, int64_t *len) {
    if (end < 0) { *o = 0; *len = 0; return; }
    int64_t cs = start < 0 ? 0 : start;
    if (cs > INT32_MAX) cs = INT32_MAX;
    int64_t ce = end < cs ? cs : end;
    if (ce > INT32_MAX) ce = INT32_MAX;
    *o = cs; *len = ce - cs + 1;
}
static reg_t cfg_region_h(const rk_t *rk, reg_t out) {
    if (out.w == 0) { reg_t r = {out.x, out.y, 0, out.h}; return r; }
    int64_t first = f2i(floor(fma((double)out.x + 0.5, rk->factor, -0.5)));
    int64_t last = f2i(floor(fma((double)(out.x + out.w - 1) + 0.5, rk->factor, -0.5)));
    int64_t s = first - rk->pad_before, e = last - rk->pad_before + rk->taps - 1;
    reg_t r = {0, out.y, 0, out.h};
    cfg_axis_bounds(s, e, &r.x, &r.w);
    return r;
}
static reg_t cfg_region_v(const rk_t *rk, reg_t out) {
    if (out.h == 0) { reg_t r = {out.x, out.y, out.w, 0}; return r; }
    int64_t first = f2i(floor(fma((double)out.y + 0.5, rk->factor, -0.5)));
    int64_t last = f2i(floor(fma((double)(out.y + out.h - 1) + 0.5, rk->factor, -0.5)));
    int64_t s = first - rk->pad_before, e = last - rk->pad_before + rk->taps - 1;
    reg_t r = {out.x, 0, out.w, 0};
    cfg_axis_bounds(s, e, &r.y, &r.h);
    return r;
}

/* ReduceOp::process_region (reduce.rs:103-251): f64 path for every format */
static void reduce_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const rk_t *hr = &nd->rk, *vr = &nd->rk2;
    const size_t bands = (size_t)in->bands;
    reg_t ir = cfg_region_v(vr, out->r);
    tile_t mid;
    if (tile_alloc(&mid, ir, in->bands, in->fmt)) return;
    const size_t mw = (size_t)mid.r.w, mh = (size_t)mid.r.h, in_w = (size_t)in->r.w;
    for (size_t y = 0; y < mh; y++)
        for (size_t x = 0; x < mw; x++) {
            double sx = rk_pos(hr, (double)mid.r.x + (double)x);
            int64_t s; int32_t ph;
            rk_plan(hr, sx, &s, &ph);
            const double *w = hr->c64 + (size_t)ph * hr->taps;
            for (size_t b = 0; b < bands; b++) {
                double acc = 0.0;
                for (int32_t t = 0; t < hr->taps; t++) {
                    size_t tx = clamp_axis(s + t, in->r.x, in->r.w);
                    acc = fma(tget(in, (y * in_w + tx) * bands + b), w[t], acc);
                }
                tset_f64(&mid, (y * mw + x) * bands + b, acc);
            }
        }
    const size_t ow = (size_t)out->r.w, oh = (size_t)out->r.h;
    for (size_t y = 0; y < oh; y++) {
        double sy = rk_pos(vr, (double)out->r.y + (double)y);
        int64_t s; int32_t ph;
        rk_plan(vr, sy, &s, &ph);
        const double *w = vr->c64 + (size_t)ph * vr->taps;
        for (size_t x = 0; x < ow; x++)
            for (size_t b = 0; b < bands; b++) {
                double acc = 0.0;
                for (int32_t t = 0; t < vr->taps; t++) {
                    size_t ty = clamp_axis(s + t, mid.r.y, mid.r.h);
                    acc = fma(tget(&mid, (ty * mw + x) * bands + b), w[t], acc);
                }
                tset_f64(out, (y * ow + x) * bands + b, acc);
            }
    }
    free(mid.data);
}

/* ---------------- zoom ---------------- */
/* Zoom::process_region (structural/zoom.rs:44-149): output pixel (x, y)
   repeats input pixel (x / xfac, y / yfac) in image coordinates; every tile
   shape gives the same pixels. */
static void zoom_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    const int64_t zx = nd->n.ufactor, zy = nd->n.ceil_mode;
    const size_t px = (size_t)in->bands * fmt_size(in->fmt);
    for (int64_t yy = 0; yy < out->r.h; yy++) {
        const int64_t sy = (out->r.y + yy) / zy - in->r.y;
        for (int64_t xx = 0; xx < out->r.w; xx++) {
            const int64_t sx = (out->r.x + xx) / zx - in->r.x;
            memcpy((uint8_t *)out->data + ((size_t)yy * (size_t)out->r.w + (size_t)xx) * px,
                   (const uint8_t *)in->data + ((size_t)sy * (size_t)in->r.w + (size_t)sx) * px, px);
        }
    }
}

/* ---------------- premultiply / unpremultiply (u8) ---------------- */
static void premultiply_process(const tile_t *in, tile_t *out) {
    const size_t bands = (size_t)in->bands, n = (size_t)in->r.w * (size_t)in->r.h;
    const size_t ab = bands - 1;
    if (in->fmt == OR_U8) {
        const uint8_t *s = (const uint8_t *)in->data;
        uint8_t *d = (uint8_t *)out->data;
        for (size_t p = 0; p < n; p++) {
            double alpha = clampd((double)s[p * bands + ab], 0.0, 255.0);
            double na = alpha / 255.0;
            for (size_t b = 0; b < ab; b++)
                d[p * bands + b] = (uint8_t)f2u32(clampd(round((double)s[p * bands + b] * na), 0.0, 255.0));
            d[p * bands + ab] = s[p * bands + ab];
        }
    } else {
        memcpy(out->data, in->data, n * bands * fmt_size(in->fmt));
    }
}

static void unpremultiply_process(const tile_t *in, tile_t *out) {
    const size_t bands = (size_t)in->bands, n = (size_t)in->r.w * (size_t)in->r.h;
    const size_t ab = bands - 1;
    if (in->fmt == OR_U8) {
        const uint8_t *s = (const uint8_t *)in->data;
        uint8_t *d = (uint8_t *)out->data;
        for (size_t p = 0; p < n; p++) {
            double alpha = (double)s[p * bands + ab];
            for (size_t b = 0; b < ab; b++) {
                if (alpha == 0.0) d[p * bands + b] = 0;
                else d[p * bands + b] = (uint8_t)f2u32(clampd(round(((double)s[p * bands + b] * 255.0) / alpha), 0.0, 255.0));
            }
            d[p * bands + ab] = s[p * bands + ab];
        }
    } else if (in->fmt == OR_F32) {
        const float *s = (const float *)in->data;
        float *d = (float *)out->data;
        for (size_t p = 0; p < n; p++) {
            float alpha = s[p * bands + ab];
            for (size_t b = 0; b < ab; b++) {
                if (alpha > 0.0f) {
                    float inv = 1.0f / alpha;
                    float v = s[p * bands + b] * inv;
                    d[p * bands + b] = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
                } else d[p * bands + b] = 0.0f;
            }
            d[p * bands + ab] = alpha;
        }
    } else {
        memcpy(out->data, in->data, n * bands * fmt_size(in->fmt));
    }
}

/* ---------------- affine (affine/core.rs, affine/interpolation.rs) ---------------- */
typedef struct {
    const node_rt *nd;
    const tile_t *in;
    reg_t bounds;
    int32_t bands;
} aff_ctx;

static double aff_white(int32_t fmt) {
    return fmt == OR_F32 ? 1.0 : (fmt == OR_U16 ? 65535.0 : 255.0);
}
static double aff_fill(const aff_ctx *c) {
    switch (c->nd->n.extend) {
    case OR_EXT_WHITE: return aff_white(c->in->fmt);
    case OR_EXT_BACKGROUND: return c->nd->n.background;
    default: return 0.0;
    }
}
static int aff_constant_fill(int32_t ext) {
    return ext == OR_EXT_BLACK || ext == OR_EXT_WHITE || ext == OR_EXT_BACKGROUND;
}
static int resolve_coord(int64_t coord, int64_t origin, int64_t size, int32_t ext, int64_t *res) {
    if (size <= 0) return 0;
    int64_t rel = coord - origin;
    if (rel >= 0 && rel < size) { *res = coord; return 1; }
    switch (ext) {
    case OR_EXT_COPY: *res = clampi(rel, 0, size - 1) + origin; return 1;
    case OR_EXT_REPEAT: { int64_t m = rel % size; if (m < 0) m += size; *res = m + origin; return 1; }
    case OR_EXT_MIRROR: {
        int64_t p = size * 2, w = rel % p;
        if (w < 0) w += p;
        *res = (w < size ? w : p - 1 - w) + origin;
        return 1;
    }
    default: return 0;
    }
}
static double aff_sample_band(const aff_ctx *c, int64_t ix, int64_t iy, int32_t band) {
    int64_t rx, ry;
    const tile_t *in = c->in;
    if (!resolve_coord(ix, c->bounds.x, c->bounds.w, c->nd->n.extend, &rx) ||
        !resolve_coord(iy, c->bounds.y, c->bounds.h, c->nd->n.extend, &ry))
        return aff_fill(c);
    int64_t tx = rx - in->r.x, ty = ry - in->r.y;
    if ((uint64_t)tx >= (uint64_t)in->r.w || (uint64_t)ty >= (uint64_t)in->r.h) return aff_fill(c);
    return tget(in, ((size_t)ty * (size_t)in->r.w + (size_t)tx) * (size_t)in->bands + (size_t)band);
}
static double aff_alpha_max(int32_t fmt) {
    return fmt == OR_F32 ? 1.0 : (fmt == OR_U16 ? 65535.0 : 255.0);
}
static double aff_sample_band_pm(const aff_ctx *c, int64_t ix, int64_t iy, int32_t band,
                                 int32_t ab, double amax) {
    double v = aff_sample_band(c, ix, iy, band);
    if (band == ab) return v;
    return v * (aff_sample_band(c, ix, iy, ab) / amax);
}
static inline double bilinear_mix(double p00, double p01, double p10, double p11, double fx,
                                  double fy) {
    double top = fma(p01, fx, p00 * (1.0 - fx));
    double bottom = fma(p11, fx, p10 * (1.0 - fx));
    return top * (1.0 - fy) + bottom * fy;
}
/* pm: 0 plain sample_at, 1 premultiplied sampler */
static double aff_sample_at(const aff_ctx *c, double x_in, double y_in, int32_t band, int pm,
                            int32_t ab, double amax) {
    if (!isfinite(x_in) || !isfinite(y_in)) return aff_fill(c);
    int32_t k = c->nd->n.kernel;
#define SB(ix, iy) (pm ? aff_sample_band_pm(c, (ix), (iy), band, ab, amax) : aff_sample_band(c, (ix), (iy), band))
    if (k == OR_K_NEAREST) return SB(f2i(x_in), f2i(y_in));
    if (k == OR_K_BILINEAR) {
        int64_t x0 = f2i(x_in), y0 = f2i(y_in);
        double fx = x_in - (double)x0, fy = y_in - (double)y0;
        return bilinear_mix(SB(x0, y0), SB(x0 + 1, y0), SB(x0, y0 + 1), SB(x0 + 1, y0 + 1), fx, fy);
    }
    int64_t support = (k == OR_K_LANCZOS3) ? 3 : 2;
    int64_t cx = f2i(floor(x_in)), cy = f2i(floor(y_in));
    double acc = 0.0, wsum = 0.0;
    for (int64_t ky = -(support - 1); ky <= support; ky++) {
        int64_t iy = cy + ky;
        double wy = or_kernel_weight(k, fabs((double)iy - y_in));
        if (wy != 0.0) {
            for (int64_t kx = -(support - 1); kx <= support; kx++) {
                int64_t ix = cx + kx;
                double wx = or_kernel_weight(k, fabs((double)ix - x_in));
                if (wx != 0.0) {
                    double w = wx * wy;
                    wsum += w;
                    acc = fma(SB(ix, iy), w, acc);
                }
            }
        }
    }
#undef SB
    return wsum > 0.0 ? acc / wsum : aff_fill(c);
}

static void aff_store(tile_t *out, size_t idx, double v) { tset_f64(out, idx, v); }

static void aff_sample_pixel(const aff_ctx *c, double x_in, double y_in, tile_t *out, size_t base) {
    const int32_t bands = c->in->bands;
    const int should_pm = !c->nd->n.premultiplied && bands == 4;
    if (should_pm) {
        if (!isfinite(x_in) || !isfinite(y_in)) {
            for (int32_t b = 0; b < bands; b++) aff_store(out, base + b, aff_fill(c));
            return;
        }
        int32_t ab = bands - 1;
        double amax = aff_alpha_max(c->in->fmt);
        double alpha = clampd(aff_sample_at(c, x_in, y_in, ab, 1, ab, amax), 0.0, amax);
        double na = alpha / amax;
        for (int32_t b = 0; b < ab; b++) {
            double p = aff_sample_at(c, x_in, y_in, b, 1, ab, amax);
            aff_store(out, base + b, na > 0.0 ? p / na : 0.0);
        }
        aff_store(out, base + ab, alpha);
        return;
    }
    if (!isfinite(x_in) || !isfinite(y_in)) {
        for (int32_t b = 0; b < bands; b++) aff_store(out, base + b, aff_fill(c));
        return;
    }
    if (c->nd->n.kernel == OR_K_NEAREST) {
        int64_t ix = f2i(x_in), iy = f2i(y_in), rx, ry;
        const tile_t *in = c->in;
        int ok = resolve_coord(ix, c->bounds.x, c->bounds.w, c->nd->n.extend, &rx) &&
                 resolve_coord(iy, c->bounds.y, c->bounds.h, c->nd->n.extend, &ry);
        int64_t tx = ok ? rx - in->r.x : -1, ty = ok ? ry - in->r.y : -1;
        if (!ok || (uint64_t)tx >= (uint64_t)in->r.w || (uint64_t)ty >= (uint64_t)in->r.h) {
            for (int32_t b = 0; b < bands; b++) aff_store(out, base + b, aff_fill(c));
            return;
        }
        size_t sb = ((size_t)ty * (size_t)in->r.w + (size_t)tx) * (size_t)bands;
        for (int32_t b = 0; b < bands; b++) aff_store(out, base + b, tget(in, sb + b));
        return;
    }
    for (int32_t b = 0; b < bands; b++) aff_store(out, base + b, aff_sample_at(c, x_in, y_in, b, 0, 0, 1.0));
}

static void affine_build_fast(node_rt *nd) {
    nd->fast = 0;
    const double *m = nd->n.m;
    if (fabs(m[1]) > OR_EPS || fabs(m[2]) > OR_EPS) return;
    uint32_t ow = nd->n.out_w, oh = nd->n.out_h;
    int32_t k = nd->n.kernel;
    if (k != OR_K_NEAREST && k != OR_K_BILINEAR && k != OR_K_BICUBIC) return;
    int nw = k == OR_K_NEAREST ? 0 : (k == OR_K_BILINEAR ? 2 : 4);
    nd->xs = (int64_t *)calloc(ow + 1, sizeof(int64_t));
    nd->ys = (int64_t *)calloc(oh + 1, sizeof(int64_t));
    nd->xw = (double *)calloc((size_t)(ow + 1) * (nw ? nw : 1), sizeof(double));
    nd->yw = (double *)calloc((size_t)(oh + 1) * (nw ? nw : 1), sizeof(double));
    for (int axis = 0; axis < 2; axis++) {
        uint32_t len = axis ? oh : ow;
        double scale = axis ? m[3] : m[0], off = axis ? nd->n.ty : nd->n.tx;
        int64_t *st = axis ? nd->ys : nd->xs;
        double *w = axis ? nd->yw : nd->xw;
        for (uint32_t i = 0; i < len; i++) {
            double coord = fma(scale, (double)i, off);
            if (k == OR_K_NEAREST) st[i] = f2i(coord);
            else if (k == OR_K_BILINEAR) {
                int64_t s = f2i(coord);
                double frac = coord - (double)s;
                st[i] = s; w[i * 2] = 1.0 - frac; w[i * 2 + 1] = frac;
            } else {
                int64_t s = f2i(floor(coord)) - 1;
                double ws[4], sum = -0.0;
                for (int t = 0; t < 4; t++) ws[t] = or_kernel_weight(OR_K_BICUBIC, fabs((double)(s + t) - coord));
                for (int t = 0; t < 4; t++) sum += ws[t];
                if (sum > 0.0) for (int t = 0; t < 4; t++) ws[t] /= sum;
                st[i] = s;
                for (int t = 0; t < 4; t++) w[i * 4 + t] = ws[t];
            }
        }
    }
    nd->fast = k == OR_K_NEAREST ? 1 : (k == OR_K_BILINEAR ? 2 : 3);
}

static int affine_fast_process(const node_rt *nd, const aff_ctx *c, tile_t *out) {
    const tile_t *in = c->in;
    if (!aff_constant_fill(nd->n.extend)) return 0;
    if (!nd->n.premultiplied && in->bands == 4) return 0;
    if (out->r.x < 0 || out->r.y < 0) return 0;
    if (out->r.x + out->r.w > nd->n.out_w || out->r.y + out->r.h > nd->n.out_h) return 0;
    if (!nd->fast) return 0;
    const int64_t L = c->bounds.x, T = c->bounds.y, R = L + c->bounds.w, B = T + c->bounds.h;
    const size_t bands = (size_t)in->bands, ow = (size_t)out->r.w, oh = (size_t)out->r.h;
    const size_t stride = (size_t)in->r.w * bands;
    for (size_t yl = 0; yl < oh; yl++) {
        size_t yi = (size_t)out->r.y + yl;
        for (size_t xl = 0; xl < ow; xl++) {
            size_t xi = (size_t)out->r.x + xl;
            size_t ob = (yl * ow + xl) * bands;
            if (nd->fast == 1) {
                int64_t yc = nd->ys[yi], xc = nd->xs[xi];
                if (yc < T || yc >= B || xc < L || xc >= R) {
                    for (size_t b = 0; b < bands; b++) aff_store(out, ob + b, aff_fill(c));
                    continue;
                }
                size_t sb = (size_t)(yc - in->r.y) * stride + (size_t)(xc - in->r.x) * bands;
                for (size_t b = 0; b < bands; b++) aff_store(out, ob + b, tget(in, sb + b));
            } else if (nd->fast == 2) {
                int64_t ys = nd->ys[yi], xs = nd->xs[xi];
                double wy0 = nd->yw[yi * 2], wy1 = nd->yw[yi * 2 + 1];
                double wx0 = nd->xw[xi * 2], wx1 = nd->xw[xi * 2 + 1];
                if (ys < T || ys + 1 >= B || xs < L || xs + 1 >= R) {
                    aff_sample_pixel(c, (double)xs + wx1, (double)ys + wy1, out, ob);
                    continue;
                }
                size_t top = (size_t)(ys - in->r.y) * stride, bot = top + stride;
                size_t ib = (size_t)(xs - in->r.x) * bands;
                for (size_t b = 0; b < bands; b++) {
                    double p00 = tget(in, top + ib + b), p01 = tget(in, top + ib + bands + b);
                    double p10 = tget(in, bot + ib + b), p11 = tget(in, bot + ib + bands + b);
                    double tv = fma(p01, wx1, p00 * wx0), bv = fma(p11, wx1, p10 * wx0);
                    aff_store(out, ob + b, fma(bv, wy1, tv * wy0));
                }
            } else {
                int64_t ys = nd->ys[yi], xs = nd->xs[xi];
                if (ys < T || ys + 3 >= B || xs < L || xs + 3 >= R) {
                    double x_in = fma(nd->n.m[0], (double)xi, nd->n.tx);
                    double y_in = fma(nd->n.m[3], (double)yi, nd->n.ty);
                    if (in->fmt == OR_U8) {
                        for (size_t b = 0; b < bands; b++) {
                            double v = aff_sample_at(c, x_in, y_in, (int32_t)b, 0, 0, 1.0);
                            ((uint8_t *)out->data)[ob + b] = (uint8_t)f2u32(clampd(round(v), 0.0, 255.0));
                        }
                    } else {
                        aff_sample_pixel(c, x_in, y_in, out, ob);
                    }
                    continue;
                }
                const double *wx = nd->xw + xi * 4, *wy = nd->yw + yi * 4;
                size_t ib = (size_t)(xs - in->r.x) * bands;
                for (size_t b = 0; b < bands; b++) {
                    double acc = 0.0;
                    for (int r = 0; r < 4; r++) {
                        size_t rb = (size_t)(ys - in->r.y + r) * stride + ib;
                        double ra = fma(tget(in, rb + bands * 3 + b), wx[3],
                                    fma(tget(in, rb + bands * 2 + b), wx[2],
                                    fma(tget(in, rb + bands + b), wx[1], tget(in, rb + b) * wx[0])));
                        acc = fma(ra, wy[r], acc);
                    }
                    if (in->fmt == OR_U8)
                        ((uint8_t *)out->data)[ob + b] = (uint8_t)f2u32(clampd(round(acc), 0.0, 255.0));
                    else aff_store(out, ob + b, acc);
                }
            }
        }
    }
    return 1;
}

static void affine_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    aff_ctx c;
    c.nd = nd; c.in = in; c.bands = in->bands;
    reg_t b = {0, 0, nd->in_w, nd->in_h}; /* with_source_bounds(0, 0, in_w, in_h) */
    c.bounds = b;
    if (affine_fast_process(nd, &c, out)) return;
    const double *m = nd->n.m;
    const size_t bands = (size_t)in->bands, ow = (size_t)out->r.w, oh = (size_t)out->r.h;
    double row_x = fma(m[1], (double)out->r.y, m[0] * (double)out->r.x) + nd->n.tx;
    double row_y = fma(m[3], (double)out->r.y, m[2] * (double)out->r.x) + nd->n.ty;
    for (size_t yl = 0; yl < oh; yl++) {
        double x_in = row_x, y_in = row_y;
        for (size_t xl = 0; xl < ow; xl++) {
            aff_sample_pixel(&c, x_in, y_in, out, (yl * ow + xl) * bands);
            x_in += m[0];
            y_in += m[2];
        }
        row_x += m[1];
        row_y += m[3];
    }
}

static void aff_map(const double *m, double tx, double ty, double x, double y, double *ox, double *oy) {
    *ox = fma(m[1], y, m[0] * x) + tx;
    *oy = fma(m[3], y, m[2] * x) + ty;
}

static void aff_axis(int64_t start, int64_t end, int64_t bs, int64_t blen, int64_t *o, int64_t *len) {
    if (blen == 0) { *o = bs; *len = 0; return; }
    int64_t be = bs + blen - 1;
    int64_t cs = start > bs ? start : bs, ce = end < be ? end : be;
    if (ce < cs) { *o = end < bs ? bs : be + 1; *len = 0; return; }
    *o = cs; *len = ce - cs + 1;
}

static reg_t affine_region(const node_rt *nd, reg_t out) {
    const double *m = nd->n.m;
    double ox0 = (double)out.x, oy0 = (double)out.y;
    double ox1 = (double)out.x + (double)(out.w > 0 ? out.w - 1 : 0);
    double oy1 = (double)out.y + (double)(out.h > 0 ? out.h - 1 : 0);
    double cx[4], cy[4];
    aff_map(m, nd->n.tx, nd->n.ty, ox0, oy0, &cx[0], &cy[0]);
    aff_map(m, nd->n.tx, nd->n.ty, ox1, oy0, &cx[1], &cy[1]);
    aff_map(m, nd->n.tx, nd->n.ty, ox0, oy1, &cx[2], &cy[2]);
    aff_map(m, nd->n.tx, nd->n.ty, ox1, oy1, &cx[3], &cy[3]);
    double mnx = fmin(fmin(fmin(cx[0], cx[1]), cx[2]), cx[3]), mxx = fmax(fmax(fmax(cx[0], cx[1]), cx[2]), cx[3]);
    double mny = fmin(fmin(fmin(cy[0], cy[1]), cy[2]), cy[3]), mxy = fmax(fmax(fmax(cy[0], cy[1]), cy[2]), cy[3]);
    int32_t lp, rp;
    kernel_padding(nd->n.kernel, &lp, &rp);
    reg_t r;
    if (nd->in_w == 0 || nd->in_h == 0) { r.x = 0; r.y = 0; r.w = 0; r.h = 0; return r; }
    aff_axis(f2i(floor(mnx)) - lp, f2i(floor(mxx)) + rp, 0, nd->in_w, &r.x, &r.w);
    aff_axis(f2i(floor(mny)) - lp, f2i(floor(mxy)) + rp, 0, nd->in_h, &r.y, &r.h);
    return r;
}

/* ------------------------------------------------------------------ */
/* node setup, regions, dims                                           */
/* ------------------------------------------------------------------ */
static int32_t node_out_dims(const or_node *n, uint32_t iw, uint32_t ih, uint32_t *ow, uint32_t *oh) {
    switch (n->kind) {
    case OR_OP_SHRINKH:
        if (n->ufactor == 0) return OR_EINVAL;
        *ow = n->ceil_mode ? (iw + n->ufactor - 1) / n->ufactor : iw / n->ufactor; *oh = ih; return OR_OK;
    case OR_OP_SHRINKV:
        if (n->ufactor == 0) return OR_EINVAL;
        *ow = iw; *oh = n->ceil_mode ? (ih + n->ufactor - 1) / n->ufactor : ih / n->ufactor; return OR_OK;
    case OR_OP_SHRINK:
        if (n->ufactor == 0 || n->ceil_mode <= 0) return OR_EINVAL;
        /* ufactor = h factor, ceil_mode field reused as v factor for SHRINK */
        *ow = iw / n->ufactor; *oh = ih / (uint32_t)n->ceil_mode; return OR_OK;
    case OR_OP_REDUCEH: *ow = reduce_output_len(n->factor, iw); *oh = ih; return OR_OK;
    case OR_OP_REDUCEV: *ow = iw; *oh = reduce_output_len(n->factor, ih); return OR_OK;
    case OR_OP_REDUCE: *ow = reduce_output_len(n->factor, iw); *oh = reduce_output_len(n->vfactor, ih); return OR_OK;
    case OR_OP_AFFINE: *ow = n->out_w; *oh = n->out_h; return OR_OK;
    case OR_OP_EXTRACT: *ow = n->ew; *oh = n->eh; return OR_OK;
    case OR_OP_ZOOM:
        /* ZoomBridge::output_width/height (conversion/zoom.rs:108-115); a zero
           factor is a build error (builder/geometry.rs:618-624) */
        if (n->ufactor == 0 || n->ceil_mode <= 0) return OR_EINVAL;
        if ((uint64_t)iw * n->ufactor > 0xFFFFFFFFull || (uint64_t)ih * (uint32_t)n->ceil_mode > 0xFFFFFFFFull)
            return OR_EINVAL;
        *ow = iw * n->ufactor; *oh = ih * (uint32_t)n->ceil_mode; return OR_OK;
    default: *ow = iw; *oh = ih; return OR_OK;
    }
}

int32_t or_pipeline_dims(const or_node *nodes, int32_t n, uint32_t w, uint32_t h,
                         uint32_t *out_w, uint32_t *out_h) {
    for (int32_t i = 0; i < n; i++) {
        int32_t st = node_out_dims(&nodes[i], w, h, &w, &h);
        if (st) return st;
    }
    *out_w = w; *out_h = h;
    return OR_OK;
}

static reg_t node_required(const node_rt *nd, reg_t out) {
    reg_t r = out;
    switch (nd->n.kind) {
    case OR_OP_SHRINKH: r.x = out.x * (int64_t)nd->n.ufactor; r.w = out.w * (int64_t)nd->n.ufactor; break;
    case OR_OP_SHRINKV: r.y = out.y * (int64_t)nd->n.ufactor; r.h = out.h * (int64_t)nd->n.ufactor; break;
    case OR_OP_SHRINK:
        r.y = out.y * (int64_t)nd->n.ceil_mode; r.h = out.h * (int64_t)nd->n.ceil_mode;
        r.x = out.x * (int64_t)nd->n.ufactor; r.w = out.w * (int64_t)nd->n.ufactor; break;
    case OR_OP_REDUCEH: {
        if (out.w == 0) { r.w = 0; break; }
        int64_t first = f2i(floor(rk_pos(&nd->rk, (double)out.x)));
        int64_t last = f2i(floor(rk_pos(&nd->rk, (double)(out.x + out.w - 1))));
        r.x = first - nd->rk.pad_before;
        r.w = (last - nd->rk.pad_before + nd->rk.taps - 1) - r.x + 1;
        break;
    }
    case OR_OP_REDUCEV: {
        if (out.h == 0) { r.h = 0; break; }
        int64_t first = f2i(floor(rk_pos(&nd->rk, (double)out.y)));
        int64_t last = f2i(floor(rk_pos(&nd->rk, (double)(out.y + out.h - 1))));
        r.y = first - nd->rk.pad_before;
        r.h = (last - nd->rk.pad_before + nd->rk.taps - 1) - r.y + 1;
        break;
    }
    case OR_OP_REDUCE: r = cfg_region_h(&nd->rk, cfg_region_v(&nd->rk2, out)); break;
    case OR_OP_AFFINE: r = affine_region(nd, out); break;
    case OR_OP_EXTRACT: r.x = out.x + nd->n.ex; r.y = out.y + nd->n.ey; break;
    case OR_OP_ZOOM: {
        /* Zoom::required_input_region (structural/zoom.rs:343-349) */
        const int64_t zx = nd->n.ufactor, zy = nd->n.ceil_mode;
        if (out.w > 0) { r.x = out.x / zx; r.w = (out.x + out.w - 1) / zx - r.x + 1; }
        if (out.h > 0) { r.y = out.y / zy; r.h = (out.y + out.h - 1) / zy - r.y + 1; }
        break;
    }
    default: break;
    }
    return r;
}

static void node_process(const node_rt *nd, const tile_t *in, tile_t *out) {
    switch (nd->n.kind) {
    case OR_OP_SHRINKH: shrinkh_process(nd, in, out); break;
    case OR_OP_SHRINKV: shrinkv_process(nd, in, out); break;
    case OR_OP_SHRINK: {
        /* Shrink = ShrinkH into an intermediate, then ShrinkV (shrink.rs:179-223);
           the u8 2x2 special case computes the same values. */
        node_rt hn = *nd, vn = *nd;
        hn.n.ufactor = nd->n.ufactor;
        vn.n.ufactor = (uint32_t)nd->n.ceil_mode;
        reg_t mid_r = {out->r.x, out->r.y * nd->n.ceil_mode, out->r.w, out->r.h * nd->n.ceil_mode};
        tile_t mid;
        if (tile_alloc(&mid, mid_r, in->bands, in->fmt)) return;
        shrinkh_process(&hn, in, &mid);
        shrinkv_process(&vn, &mid, out);
        free(mid.data);
        break;
    }
    case OR_OP_REDUCEH: reduceh_process(nd, in, out); break;
    case OR_OP_REDUCEV: reducev_process(nd, in, out); break;
    case OR_OP_REDUCE: reduce_process(nd, in, out); break;
    case OR_OP_PREMULTIPLY: premultiply_process(in, out); break;
    case OR_OP_UNPREMULTIPLY: unpremultiply_process(in, out); break;
    case OR_OP_AFFINE: affine_process(nd, in, out); break;
    case OR_OP_EXTRACT: memcpy(out->data, in->data, (size_t)out->r.w * out->r.h * out->bands * fmt_size(out->fmt)); break;
    case OR_OP_ZOOM: zoom_process(nd, in, out); break;
    default: break;
    }
}

static int32_t node_setup(node_rt *nd, const or_node *n, uint32_t iw, uint32_t ih, int32_t bands,
                          int32_t fmt) {
    memset(nd, 0, sizeof(*nd));
    nd->n = *n; nd->in_w = iw; nd->in_h = ih; nd->bands = bands; nd->fmt = fmt;
    int32_t st = node_out_dims(n, iw, ih, &nd->out_w, &nd->out_h);
    if (st) return st;
    switch (n->kind) {
    case OR_OP_REDUCEH:
        st = rk_init(&nd->rk, n->factor, n->kernel);
        if (st) return st;
        rk_bind(&nd->rk, iw);
        break;
    case OR_OP_REDUCEV:
        st = rk_init(&nd->rk, n->factor, n->kernel);
        if (st) return st;
        rk_bind(&nd->rk, ih);
        break;
    case OR_OP_REDUCE:
        st = rk_init(&nd->rk, n->factor, n->kernel);
        if (st) return st;
        st = rk_init(&nd->rk2, n->vfactor, n->kernel);
        if (st) return st;
        break; /* ReduceOp never binds the input length (reduce.rs:51-67) */
    case OR_OP_PREMULTIPLY:
    case OR_OP_UNPREMULTIPLY:
        if (bands < 2) return OR_EINVAL;
        break;
    case OR_OP_AFFINE:
        if (n->kernel == OR_K_NOHALO || n->kernel == OR_K_LBB || n->kernel == OR_K_VSQBS) return OR_EFORMAT;
        affine_build_fast(nd);
        break;
    default: break;
    }
    return OR_OK;
}

static void node_free(node_rt *nd) {
    rk_free(&nd->rk); rk_free(&nd->rk2);
    free(nd->xs); free(nd->ys); free(nd->xw); free(nd->yw);
}

/* MemorySource::read_region (viprs-runtime/src/sources/memory.rs:186-215): edge replication */
static void source_read(const void *src, uint32_t w, uint32_t h, int32_t bands, int32_t fmt,
                        tile_t *t) {
    const size_t es = fmt_size(fmt), px = (size_t)bands * es;
    for (int64_t yy = 0; yy < t->r.h; yy++) {
        int64_t sy = clampi(t->r.y + yy, 0, (int64_t)h - 1);
        for (int64_t xx = 0; xx < t->r.w; xx++) {
            int64_t sx = clampi(t->r.x + xx, 0, (int64_t)w - 1);
            memcpy((uint8_t *)t->data + ((size_t)yy * (size_t)t->r.w + (size_t)xx) * px,
                   (const uint8_t *)src + ((size_t)sy * w + (size_t)sx) * px, px);
        }
    }
}

/* tile geometry (demand.rs:41-83, planning.rs:550-596) */
static void tile_geometry(int32_t hint, uint32_t W, uint32_t H, uint32_t *tw, uint32_t *th) {
    *tw = hint == OR_DH_SMALLTILE ? 128 : W;
    uint32_t t;
    switch (hint) {
    case OR_DH_SMALLTILE: t = 128; break;
    case OR_DH_THIN: t = W > 10000 ? 1 : 16; break;
    case OR_DH_FULL: t = H; break;
    case OR_DH_ONELINE: t = 1; break;
    default: t = H <= 1024 ? 256 : (H >= 4096 ? 64 : 16); break;
    }
    if (t > H) t = H;
    if (t < 1) t = 1;
    *th = t;
}

typedef struct {
    const void *src; uint32_t w, h; int32_t bands, fmt;
    node_rt *nodes; int32_t n;
    void *dst; uint32_t ow, oh, tw, th;
    int64_t ntiles; int64_t next; pthread_mutex_t mu;
    int32_t err;
} run_ctx;

static int32_t run_tile(run_ctx *rc, reg_t tile) {
    int32_t n = rc->n;
    reg_t *outr = (reg_t *)malloc(sizeof(reg_t) * (size_t)(n + 1));
    outr[n] = tile; /* outr[i+1] is the output region of node i; outr[0] = source read */
    for (int32_t i = n - 1; i >= 0; i--) {
        if (rc->nodes[i].n.kind == OR_OP_PREMULTIPLY || rc->nodes[i].n.kind == OR_OP_UNPREMULTIPLY)
            outr[i] = outr[i + 1];
        else outr[i] = node_required(&rc->nodes[i], outr[i + 1]);
    }
    tile_t cur;
    if (tile_alloc(&cur, outr[0], rc->bands, rc->fmt)) { free(outr); return OR_ENOMEM; }
    source_read(rc->src, rc->w, rc->h, rc->bands, rc->fmt, &cur);
    for (int32_t i = 0; i < n; i++) {
        tile_t nxt;
        if (tile_alloc(&nxt, outr[i + 1], rc->bands, rc->fmt)) { free(cur.data); free(outr); return OR_ENOMEM; }
        node_process(&rc->nodes[i], &cur, &nxt);
        free(cur.data);
        cur = nxt;
    }
    const size_t px = (size_t)rc->bands * fmt_size(rc->fmt);
    for (int64_t yy = 0; yy < tile.h; yy++)
        memcpy((uint8_t *)rc->dst + (((size_t)(tile.y + yy)) * rc->ow + (size_t)tile.x) * px,
               (uint8_t *)cur.data + (size_t)yy * (size_t)tile.w * px, (size_t)tile.w * px);
    free(cur.data);
    free(outr);
    return OR_OK;
}

static void *run_worker(void *arg) {
    run_ctx *rc = (run_ctx *)arg;
    const int64_t cols = (rc->ow + rc->tw - 1) / rc->tw;
    for (;;) {
        pthread_mutex_lock(&rc->mu);
        int64_t t = rc->next++;
        pthread_mutex_unlock(&rc->mu);
        if (t >= rc->ntiles) break;
        int64_t ty = t / cols, tx = t % cols;
        reg_t tile = {tx * rc->tw, ty * rc->th, rc->tw, rc->th};
        if (tile.x + tile.w > rc->ow) tile.w = rc->ow - tile.x;
        if (tile.y + tile.h > rc->oh) tile.h = rc->oh - tile.y;
        int32_t st = run_tile(rc, tile);
        if (st) rc->err = st;
    }
    return NULL;
}

static int32_t default_hint(const or_node *nodes, int32_t n) {
    int32_t h = OR_DH_ANY;
    for (int32_t i = 0; i < n; i++) if (nodes[i].demand_hint > h) h = nodes[i].demand_hint;
    return h;
}

int32_t or_pipeline_run(const void *src, uint32_t w, uint32_t h, uint32_t bands, int32_t fmt,
                        const or_node *nodes, int32_t n, int32_t demand_override, int32_t threads,
                        void *dst, uint32_t out_w, uint32_t out_h) {
    if (!src || !dst || bands == 0) return OR_EINVAL;
    if (fmt != OR_U8 && fmt != OR_U16 && fmt != OR_F32) return OR_EFORMAT;
    node_rt *rt = (node_rt *)calloc((size_t)(n > 0 ? n : 1), sizeof(node_rt));
    uint32_t cw = w, ch = h;
    int32_t st = OR_OK;
    for (int32_t i = 0; i < n && !st; i++) {
        st = node_setup(&rt[i], &nodes[i], cw, ch, (int32_t)bands, fmt);
        cw = rt[i].out_w; ch = rt[i].out_h;
    }
    if (!st && (cw != out_w || ch != out_h)) st = OR_EINVAL;
    if (!st && out_w > 0 && out_h > 0) {
        run_ctx rc;
        memset(&rc, 0, sizeof(rc));
        rc.src = src; rc.w = w; rc.h = h; rc.bands = (int32_t)bands; rc.fmt = fmt;
        rc.nodes = rt; rc.n = n; rc.dst = dst; rc.ow = out_w; rc.oh = out_h;
        int32_t hint = demand_override >= 0 ? demand_override : default_hint(nodes, n);
        tile_geometry(hint, out_w, out_h, &rc.tw, &rc.th);
        rc.ntiles = (int64_t)((out_w + rc.tw - 1) / rc.tw) * ((out_h + rc.th - 1) / rc.th);
        pthread_mutex_init(&rc.mu, NULL);
        int32_t nt = threads > 0 ? threads : 1;
        if (nt > 256) nt = 256;
        pthread_t th[256];
        for (int32_t i = 1; i < nt; i++) pthread_create(&th[i], NULL, run_worker, &rc);
        run_worker(&rc);
        for (int32_t i = 1; i < nt; i++) pthread_join(th[i], NULL);
        pthread_mutex_destroy(&rc.mu);
        st = rc.err;
    }
    for (int32_t i = 0; i < n; i++) node_free(&rt[i]);
    free(rt);
    return st;
}

/* ------------------------------------------------------------------ */
/* thumbnail planner (thumbnail.rs:204-524)                            */
/* ------------------------------------------------------------------ */
static int32_t affine_kernel_for_resize(int32_t k) {
    return k == OR_K_NEAREST ? OR_K_NEAREST : (k == OR_K_BILINEAR ? OR_K_BILINEAR : OR_K_BICUBIC);
}

static void target_dimensions(int32_t target, uint32_t tw, uint32_t th, uint32_t iw, uint32_t ih,
                              uint32_t *ow, uint32_t *oh) {
    switch (target) {
    case OR_TT_FITBOX: {
        double hs = (double)(tw > 1 ? tw : 1) / (double)iw;
        double vs = (double)(th > 1 ? th : 1) / (double)ih;
        double s = fmin(fmin(hs, vs), 1.0);
        *ow = f2u32(fmax(round((double)iw * s), 1.0));
        *oh = f2u32(fmax(round((double)ih * s), 1.0));
        break;
    }
    case OR_TT_FORCE: *ow = tw > 1 ? tw : 1; *oh = th > 1 ? th : 1; break;
    case OR_TT_WIDTH: {
        uint32_t w = tw > 1 ? tw : 1;
        if (w > iw) w = iw;
        *ow = w;
        *oh = f2u32(fmax(round(((double)ih * (double)w) / (double)iw), 1.0));
        break;
    }
    default: {
        uint32_t hh = th > 1 ? th : 1;
        if (hh > ih) hh = ih;
        *oh = hh;
        *ow = f2u32(fmax(round(((double)iw * (double)hh) / (double)ih), 1.0));
        break;
    }
    }
}

static uint32_t choose_integer_shrink(uint32_t input_len, uint32_t target_len, double total) {
    if (total <= 1.0 + THUMB_EPS) return 1;
    uint32_t f = f2u32(fmax(floor(total), 1.0));
    while (f > 1) {
        uint32_t after = input_len / f;
        double residual = total / (double)f;
        uint32_t ar = residual > 1.0 + THUMB_EPS ? f2u32(fmax(round((double)after / residual), 1.0)) : after;
        if (ar >= target_len) break;
        f -= 1;
    }
    return f;
}

static uint32_t shrink_on_load_factor(double s) {
    if (s >= 16.0) return 16;
    if (s >= 8.0) return 4;
    if (s >= 4.0) return 2;
    return 0;
}

static int32_t push_node(or_plan_node *nodes, int32_t max, int32_t *cnt, or_plan_node nd) {
    if (*cnt >= max) return OR_EINVAL;
    nodes[(*cnt)++] = nd;
    return OR_OK;
}

int32_t or_thumbnail_plan(int32_t target, uint32_t tw, uint32_t th, int32_t kernel, int32_t crop,
                          uint32_t in_w, uint32_t in_h, uint32_t bands, int32_t allow_shrink_hint,
                          or_plan_node *nodes, int32_t max_nodes, int32_t *n_nodes,
                          uint32_t *out_w, uint32_t *out_h, uint32_t *shrink_on_load) {
    *n_nodes = 0; *shrink_on_load = 0;
    if (bands == 0) return OR_EINVAL;
    if (in_w == 0 || in_h == 0) { *out_w = 0; *out_h = 0; return OR_OK; }
    or_plan_node geo[8];
    int32_t ng = 0;
    const int allow_up = target == OR_TT_FORCE;
    const int single = in_w == 1 && in_h == 1;
    uint32_t t_w, t_h;
    if (crop && (target == OR_TT_FITBOX || target == OR_TT_FORCE)) { t_w = tw > 1 ? tw : 1; t_h = th > 1 ? th : 1; }
    else target_dimensions(target, tw, th, in_w, in_h, &t_w, &t_h);
    if (allow_up && !single) { if (t_w < 1) t_w = 1; if (t_h < 1) t_h = 1; }
    else { if (t_w > in_w) t_w = in_w; if (t_w < 1) t_w = 1; if (t_h > in_h) t_h = in_h; if (t_h < 1) t_h = 1; }
    const int has_alpha = bands == 2 || bands == 4;
    uint32_t g_w, g_h;
    if (crop) {
        double hs = (double)(t_w > 1 ? t_w : 1) / (double)in_w, vs = (double)(t_h > 1 ? t_h : 1) / (double)in_h;
        double cover = fmax(hs, vs);
        g_w = f2u32(fmax(round((double)in_w * cover), (double)t_w));
        g_h = f2u32(fmax(round((double)in_h * cover), (double)t_h));
    } else { g_w = t_w; g_h = t_h; }
    if (allow_up && !single) { if (g_w < 1) g_w = 1; if (g_h < 1) g_h = 1; }
    else { if (g_w > in_w) g_w = in_w; if (g_w < 1) g_w = 1; if (g_h > in_h) g_h = in_h; if (g_h < 1) g_h = 1; }

    if (in_w == 1 || in_h == 1) {
        if (single) { t_w = 1; t_h = 1; }
        if (t_w != in_w || t_h != in_h) {
            double isx = (double)in_w / (double)t_w, isy = (double)in_h / (double)t_h;
            or_plan_node a; memset(&a, 0, sizeof(a));
            a.kind = OR_TN_AFFINE;
            a.m[0] = isx; a.m[3] = isy;
            a.tx = kernel == OR_K_NEAREST ? 0.0 : 0.5 * (1.0 - isx);
            a.ty = kernel == OR_K_NEAREST ? 0.0 : 0.5 * (1.0 - isy);
            a.out_w = t_w; a.out_h = t_h; a.kernel = affine_kernel_for_resize(kernel);
            geo[ng++] = a;
        }
    } else {
        double hshrink = (double)in_w / (double)g_w, vshrink = (double)in_h / (double)g_h;
        uint32_t sol = allow_shrink_hint ? shrink_on_load_factor(fmin(hshrink, vshrink)) : 0;
        uint32_t ew = sol ? (in_w / sol > 1 ? in_w / sol : 1) : in_w;
        uint32_t eh = sol ? (in_h / sol > 1 ? in_h / sol : 1) : in_h;
        *shrink_on_load = sol;
        hshrink = (double)ew / (double)g_w;
        vshrink = (double)eh / (double)g_h;
        uint32_t ih_ = choose_integer_shrink(ew, g_w, hshrink);
        uint32_t iv_ = choose_integer_shrink(eh, g_h, vshrink);
        uint32_t asw = ew / (ih_ > 1 ? ih_ : 1), ash = eh / (iv_ > 1 ? iv_ : 1);
        double rh = hshrink > 1.0 ? hshrink / (double)ih_ : 1.0;
        double rv = vshrink > 1.0 ? vshrink / (double)iv_ : 1.0;
        uint32_t arw = rh > 1.0 + THUMB_EPS ? f2u32(fmax(round((double)asw / rh), 1.0)) : asw;
        uint32_t arh = rv > 1.0 + THUMB_EPS ? f2u32(fmax(round((double)ash / rv), 1.0)) : ash;
        or_plan_node nd;
        if (ih_ > 1) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_SHRINKH; nd.ufactor = ih_; geo[ng++] = nd; }
        if (iv_ > 1) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_SHRINKV; nd.ufactor = iv_; geo[ng++] = nd; }
        if (rh > 1.0 + THUMB_EPS) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_REDUCEH; nd.factor = rh; nd.kernel = kernel; geo[ng++] = nd; }
        if (rv > 1.0 + THUMB_EPS) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_REDUCEV; nd.factor = rv; nd.kernel = kernel; geo[ng++] = nd; }
        double asx = (double)g_w / (double)arw, asy = (double)g_h / (double)arh;
        if (fabs(asx - 1.0) > THUMB_EPS || fabs(asy - 1.0) > THUMB_EPS) {
            double isx = 1.0 / asx, isy = 1.0 / asy;
            memset(&nd, 0, sizeof(nd));
            nd.kind = OR_TN_AFFINE;
            nd.m[0] = isx; nd.m[3] = isy;
            nd.tx = kernel == OR_K_NEAREST ? 0.0 : 0.5 * (1.0 - isx);
            nd.ty = kernel == OR_K_NEAREST ? 0.0 : 0.5 * (1.0 - isy);
            nd.out_w = g_w; nd.out_h = g_h; nd.kernel = affine_kernel_for_resize(kernel);
            geo[ng++] = nd;
        }
        if (crop && (g_w != t_w || g_h != t_h)) {
            memset(&nd, 0, sizeof(nd));
            nd.kind = OR_TN_EXTRACT;
            nd.ex = (g_w - t_w) / 2; nd.ey = (g_h - t_h) / 2; nd.ew = t_w; nd.eh = t_h;
            geo[ng++] = nd;
        }
    }
    /* wrap_geometry_nodes (thumbnail.rs:438-456) */
    int32_t cnt = 0, st = OR_OK;
    or_plan_node pm; memset(&pm, 0, sizeof(pm));
    if (has_alpha && ng > 0) { pm.kind = OR_TN_PREMULTIPLY; st |= push_node(nodes, max_nodes, &cnt, pm); }
    for (int32_t i = 0; i < ng; i++) st |= push_node(nodes, max_nodes, &cnt, geo[i]);
    if (has_alpha && ng > 0) { pm.kind = OR_TN_UNPREMULTIPLY; st |= push_node(nodes, max_nodes, &cnt, pm); }
    *n_nodes = cnt; *out_w = t_w; *out_h = t_h;
    return st;
}

/* ------------------------------------------------------------------ */
/* resize planner (resize.rs:163-348)                                  */
/* ------------------------------------------------------------------ */
static uint32_t scaled_len(uint32_t in, double s) { return f2u32(fmax(round((double)in * s), 1.0)); }
static uint32_t pre_shrink(uint32_t in, uint32_t t, int32_t k, double gap) {
    if (t == 0 || in <= t || k == OR_K_NEAREST) return 1;
    return f2u32(fmax(floor((double)in / (double)t / gap), 1.0));
}
static double affine_offset(double s, int32_t k) { return k == OR_K_NEAREST ? 0.0 : 0.5 * (1.0 - 1.0 / s); }

int32_t or_resize_plan(double hscale, double vscale, int32_t kernel, double gap, uint32_t in_w,
                       uint32_t in_h, or_plan_node *nodes, int32_t max_nodes, int32_t *n_nodes,
                       uint32_t *out_w, uint32_t *out_h) {
    *n_nodes = 0;
    if (!(isfinite(hscale) && hscale > 0.0)) hscale = 1.0;
    if (!(isfinite(vscale) && vscale > 0.0)) vscale = 1.0;
    if (!(isfinite(gap) && gap >= 1.0)) gap = 2.0;
    if (in_w == 0 || in_h == 0) { *out_w = 0; *out_h = 0; return OR_OK; }
    uint32_t t_w = scaled_len(in_w, hscale), t_h = scaled_len(in_h, vscale);
    int32_t k = kernel == OR_K_NOHALO ? OR_K_BICUBIC : kernel;
    int32_t cnt = 0, st = OR_OK;
    or_plan_node nd;
    *out_w = t_w; *out_h = t_h;
    if (k == OR_K_LBB) {
        if (t_w != in_w || t_h != in_h) {
            double sx = (double)t_w / (double)in_w, sy = (double)t_h / (double)in_h;
            memset(&nd, 0, sizeof(nd));
            nd.kind = OR_TN_AFFINE; nd.m[0] = 1.0 / sx; nd.m[3] = 1.0 / sy;
            nd.tx = affine_offset(sx, k); nd.ty = affine_offset(sy, k);
            nd.out_w = t_w; nd.out_h = t_h; nd.kernel = k;
            st |= push_node(nodes, max_nodes, &cnt, nd);
        }
        *n_nodes = cnt;
        return st;
    }
    uint32_t cw = in_w, chh = in_h;
    uint32_t hsf = t_w < cw ? pre_shrink(cw, t_w, k, gap) : 1;
    uint32_t vsf = t_h < chh ? pre_shrink(chh, t_h, k, gap) : 1;
    if (vsf > 1) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_SHRINKV; nd.ufactor = vsf; st |= push_node(nodes, max_nodes, &cnt, nd); chh /= vsf; }
    if (hsf > 1) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_SHRINKH; nd.ufactor = hsf; st |= push_node(nodes, max_nodes, &cnt, nd); cw /= hsf; }
    if (t_h < chh) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_REDUCEV; nd.factor = (double)chh / (double)t_h; nd.kernel = k; st |= push_node(nodes, max_nodes, &cnt, nd); chh = t_h; }
    if (t_w < cw) { memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_REDUCEH; nd.factor = (double)cw / (double)t_w; nd.kernel = k; st |= push_node(nodes, max_nodes, &cnt, nd); cw = t_w; }
    int can_zoom = k != OR_K_VSQBS;
    uint32_t zx = can_zoom && t_w > cw ? t_w / cw : 1, zy = can_zoom && t_h > chh ? t_h / chh : 1;
    if (zx > 1 || zy > 1) {
        memset(&nd, 0, sizeof(nd)); nd.kind = OR_TN_ZOOM; nd.zx = zx; nd.zy = zy;
        st |= push_node(nodes, max_nodes, &cnt, nd);
        cw *= zx; chh *= zy;
    }
    double asx = (double)t_w / (double)cw, asy = (double)t_h / (double)chh;
    if (fabs(asx - 1.0) > THUMB_EPS || fabs(asy - 1.0) > THUMB_EPS) {
        memset(&nd, 0, sizeof(nd));
        nd.kind = OR_TN_AFFINE; nd.m[0] = 1.0 / asx; nd.m[3] = 1.0 / asy;
        nd.tx = affine_offset(asx, k); nd.ty = affine_offset(asy, k);
        nd.out_w = t_w; nd.out_h = t_h; nd.kernel = k;
        st |= push_node(nodes, max_nodes, &cnt, nd);
    }
    *n_nodes = cnt;
    return st;
}

/* ------------------------------------------------------------------ */
/* builder materialisation                                             */
/* ------------------------------------------------------------------ */
static int32_t materialise(const or_plan_node *pn, int32_t np, int32_t thumb_large, int32_t is_thumb,
                           or_node *out, int32_t *n_out) {
    int32_t n = 0;
    for (int32_t i = 0; i < np; i++) {
        or_node nd; memset(&nd, 0, sizeof(nd));
        nd.demand_hint = OR_DH_THIN;
        switch (pn[i].kind) {
        case OR_TN_PREMULTIPLY: nd.kind = OR_OP_PREMULTIPLY; break;
        case OR_TN_UNPREMULTIPLY: nd.kind = OR_OP_UNPREMULTIPLY; break;
        case OR_TN_SHRINKH: nd.kind = OR_OP_SHRINKH; nd.ufactor = pn[i].ufactor; break;
        case OR_TN_SHRINKV: nd.kind = OR_OP_SHRINKV; nd.ufactor = pn[i].ufactor; break;
        case OR_TN_REDUCEH: nd.kind = OR_OP_REDUCEH; nd.factor = pn[i].factor; nd.kernel = pn[i].kernel; break;
        case OR_TN_REDUCEV: nd.kind = OR_OP_REDUCEV; nd.factor = pn[i].factor; nd.kernel = pn[i].kernel; break;
        case OR_TN_AFFINE:
            nd.kind = OR_OP_AFFINE;
            memcpy(nd.m, pn[i].m, sizeof(nd.m));
            nd.tx = pn[i].tx; nd.ty = pn[i].ty; nd.out_w = pn[i].out_w; nd.out_h = pn[i].out_h;
            nd.kernel = pn[i].kernel; nd.extend = OR_EXT_COPY;
            nd.demand_hint = (is_thumb && thumb_large) ? OR_DH_THIN : OR_DH_SMALLTILE;
            break;
        case OR_TN_EXTRACT:
            nd.kind = OR_OP_EXTRACT; nd.ex = pn[i].ex; nd.ey = pn[i].ey; nd.ew = pn[i].ew; nd.eh = pn[i].eh;
            break;
        case OR_TN_ZOOM:
            /* PipelineBuilder::zoom (builder/geometry.rs:618-643); ZoomBridge's hint is FatStrip */
            nd.kind = OR_OP_ZOOM; nd.ufactor = pn[i].zx; nd.ceil_mode = (int32_t)pn[i].zy;
            nd.demand_hint = OR_DH_FAT;
            break;
        default: return OR_EFORMAT;
        }
        out[n++] = nd;
    }
    *n_out = n;
    return OR_OK;
}

static int32_t thumb_nodes(uint32_t w, uint32_t h, uint32_t bands, int32_t target, uint32_t tw,
                           uint32_t th, int32_t kernel, int32_t crop, or_node *nodes, int32_t *n,
                           uint32_t *ow, uint32_t *oh, int32_t *override) {
    or_plan_node pn[16];
    int32_t np;
    uint32_t sol;
    int32_t st = or_thumbnail_plan(target, tw, th, kernel, crop, w, h, bands, 1, pn, 16, &np, ow, oh, &sol);
    if (st) return st;
    /* MemorySource declines shrink-on-load (viprs-ports/src/source.rs:257-259) */
    if (sol) {
        st = or_thumbnail_plan(target, tw, th, kernel, crop, w, h, bands, 0, pn, 16, &np, ow, oh, &sol);
        if (st) return st;
    }
    int32_t large = w > 512 || h > 512;
    *override = large ? OR_DH_THIN : -1;
    if (np == 0) {
        /* builder.affine(identity, 0, 0, out_w, out_h, Nearest) with Background(0) */
        or_node nd; memset(&nd, 0, sizeof(nd));
        nd.kind = OR_OP_AFFINE; nd.m[0] = 1.0; nd.m[3] = 1.0; nd.out_w = *ow; nd.out_h = *oh;
        nd.kernel = OR_K_NEAREST; nd.extend = OR_EXT_BACKGROUND; nd.background = 0.0;
        nd.demand_hint = OR_DH_SMALLTILE;
        nodes[0] = nd; *n = 1;
        return OR_OK;
    }
    return materialise(pn, np, large, 1, nodes, n);
}

int32_t or_thumbnail_dims(uint32_t w, uint32_t h, uint32_t bands, int32_t target, uint32_t tw,
                          uint32_t th, int32_t kernel, int32_t crop, uint32_t *out_w, uint32_t *out_h) {
    or_node nodes[16]; int32_t n, ov;
    return thumb_nodes(w, h, bands, target, tw, th, kernel, crop, nodes, &n, out_w, out_h, &ov);
}

int32_t or_thumbnail_run(const void *src, uint32_t w, uint32_t h, uint32_t bands, int32_t fmt,
                         int32_t target, uint32_t tw, uint32_t th, int32_t kernel, int32_t crop,
                         int32_t threads, void *dst, uint32_t *out_w, uint32_t *out_h) {
    or_node nodes[16]; int32_t n, ov;
    int32_t st = thumb_nodes(w, h, bands, target, tw, th, kernel, crop, nodes, &n, out_w, out_h, &ov);
    if (st) return st;
    if (!dst) return OR_OK;
    return or_pipeline_run(src, w, h, bands, fmt, nodes, n, ov, threads, dst, *out_w, *out_h);
}

int32_t or_resize_run(const void *src, uint32_t w, uint32_t h, uint32_t bands, int32_t fmt,
                      double hscale, double vscale, int32_t kernel, int32_t threads, void *dst,
                      uint32_t *out_w, uint32_t *out_h) {
    or_plan_node pn[16]; int32_t np;
    int32_t st = or_resize_plan(hscale, vscale, kernel, 2.0, w, h, pn, 16, &np, out_w, out_h);
    if (st) return st;
    if (!dst) return OR_OK;
    if (np == 0) {
        memcpy(dst, src, (size_t)w * h * bands * fmt_size(fmt));
        return OR_OK;
    }
    or_node nodes[16]; int32_t n;
    st = materialise(pn, np, 0, 0, nodes, &n);
    if (st) return st;
    return or_pipeline_run(src, w, h, bands, fmt, nodes, n, -1, threads, dst, *out_w, *out_h);
}

/* ------------------------------------------------------------------ */
/* mapim (mapim.rs), whole-image form                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    const void *src; uint32_t sw, sh, bands; int32_t fmt;
    const void *index; int32_t index_fmt; uint32_t iw, ih; int32_t kernel, extend_copy; double bg;
    int32_t premultiplied;
    void *dst; int64_t next_row; pthread_mutex_t mu;
} mapim_ctx;

/* Index sample i read as f64 whatever its format (mapim.rs:1135-1274 reads the
   index through ToF64 for every BandFormatId). */
static double mp_index(const mapim_ctx *c, size_t i) {
    switch (c->index_fmt) {
    case OR_U8: return (double)((const uint8_t *)c->index)[i];
    case OR_U16: return (double)((const uint16_t *)c->index)[i];
    default: return (double)((const float *)c->index)[i];
    }
}

static double mp_band(const mapim_ctx *c, const tile_t *s, int64_t ix, int64_t iy, int32_t band) {
    /* MapImOp::resolve_source_coord / sample_source_band (mapim.rs:306-384) */
    int64_t x, y;
    if (!c->extend_copy) {
        if (ix < 0 || ix >= (int64_t)c->sw || iy < 0 || iy >= (int64_t)c->sh) return c->bg;
        x = ix; y = iy;
    } else {
        int32_t lp, rp;
        kernel_padding(c->kernel, &lp, &rp);
        if (ix < -(int64_t)(lp + 1) || ix > (int64_t)c->sw + rp || iy < -(int64_t)(lp + 1) || iy > (int64_t)c->sh + rp)
            return c->bg;
        x = clampi(ix, 0, (int64_t)c->sw - 1); y = clampi(iy, 0, (int64_t)c->sh - 1);
    }
    return tget(s, ((size_t)y * c->sw + (size_t)x) * c->bands + (size_t)band);
}

/* sample_source_band_premultiplied (mapim.rs:616-636): colour bands scaled by
   the tap's alpha over alpha_max; out-of-range taps read the background for
   both the band and the alpha. */
static double mp_band_pm(const mapim_ctx *c, const tile_t *s, int64_t ix, int64_t iy, int32_t band,
                         int32_t ab, double amax) {
    double v = mp_band(c, s, ix, iy, band);
    if (band == ab) return v;
    return v * (mp_band(c, s, ix, iy, ab) / amax);
}

/* sample_at_premultiplied (mapim.rs:638-931) for the kernels this path
   carries: nearest and bilinear at floor(), the separable kernels over
   cx - (support - 1) .. cx + support with the weight-sum renormalisation
   (sample_at_premultiplied_separable, :935-991). */
static double mp_sample_pm(const mapim_ctx *c, const tile_t *s, double x, double y, int32_t band,
                           int32_t ab, double amax) {
    if (!isfinite(x) || !isfinite(y)) return c->bg;
    int32_t k = c->kernel;
    if (k == OR_K_NEAREST) return mp_band_pm(c, s, f2i(floor(x)), f2i(floor(y)), band, ab, amax);
    if (k == OR_K_BILINEAR) {
        int64_t x0 = f2i(floor(x)), y0 = f2i(floor(y));
        double fx = x - (double)x0, fy = y - (double)y0;
        return bilinear_mix(mp_band_pm(c, s, x0, y0, band, ab, amax), mp_band_pm(c, s, x0 + 1, y0, band, ab, amax),
                            mp_band_pm(c, s, x0, y0 + 1, band, ab, amax),
                            mp_band_pm(c, s, x0 + 1, y0 + 1, band, ab, amax), fx, fy);
    }
    int64_t support = k == OR_K_LANCZOS3 ? 3 : 2;
    int64_t cx = f2i(floor(x)), cy = f2i(floor(y));
    double acc = 0.0, wsum = 0.0;
    for (int64_t ky = -(support - 1); ky <= support; ky++) {
        int64_t iy = cy + ky;
        double wy = or_kernel_weight(k, fabs((double)iy - y));
        if (wy == 0.0) continue;
        for (int64_t kx = -(support - 1); kx <= support; kx++) {
            int64_t ix = cx + kx;
            double wx = or_kernel_weight(k, fabs((double)ix - x));
            if (wx != 0.0) {
                double w = wx * wy;
                wsum += w;
                acc = fma(mp_band_pm(c, s, ix, iy, band, ab, amax), w, acc);
            }
        }
    }
    return wsum > 0.0 ? acc / wsum : c->bg;
}

/* sample_source_with_premultiplied_alpha_into (mapim.rs:993-1040): the alpha
   band sampled from the premultiplied stencil and clamped to [0, alpha_max],
   each colour band sampled premultiplied and divided by the normalised alpha. */
static void mp_pixel_pm(const mapim_ctx *c, const tile_t *s, double x, double y, tile_t *o, size_t px) {
    const int32_t bands = (int32_t)c->bands, ab = bands - 1;
    if (!isfinite(x) || !isfinite(y)) {
        for (int32_t b = 0; b < bands; b++) tset_f64(o, px + (size_t)b, c->bg);
        return;
    }
    double amax = aff_alpha_max(c->fmt);
    double alpha = clampd(mp_sample_pm(c, s, x, y, ab, ab, amax), 0.0, amax);
    double na = alpha / amax;
    for (int32_t b = 0; b < ab; b++) {
        double p = mp_sample_pm(c, s, x, y, b, ab, amax);
        tset_f64(o, px + (size_t)b, na > 0.0 ? p / na : 0.0);
    }
    tset_f64(o, px + (size_t)ab, alpha);
}

static void *mapim_worker(void *arg) {
    mapim_ctx *c = (mapim_ctx *)arg;
    tile_t s; s.r.x = 0; s.r.y = 0; s.r.w = c->sw; s.r.h = c->sh; s.bands = (int32_t)c->bands; s.fmt = c->fmt; s.data = (void *)c->src;
    tile_t o; o.r.x = 0; o.r.y = 0; o.r.w = c->iw; o.r.h = c->ih; o.bands = (int32_t)c->bands; o.fmt = c->fmt; o.data = c->dst;
    /* the non-nearest/bilinear path samples through Affine::sample_at with Background(bg) and
       bounds = the source read region (mapim.rs:1178-1186, 1250-1271) */
    or_node an; memset(&an, 0, sizeof(an));
    an.kind = OR_OP_AFFINE; an.m[0] = 1.0; an.m[3] = 1.0; an.kernel = c->kernel;
    an.extend = OR_EXT_BACKGROUND; an.background = c->bg;
    node_rt nd; memset(&nd, 0, sizeof(nd)); nd.n = an; nd.in_w = c->sw; nd.in_h = c->sh;
    aff_ctx ac; ac.nd = &nd; ac.in = &s; ac.bands = (int32_t)c->bands;
    reg_t b = {0, 0, c->sw, c->sh}; ac.bounds = b;
    const size_t bands = c->bands;
    for (;;) {
        pthread_mutex_lock(&c->mu);
        int64_t row = c->next_row++;
        pthread_mutex_unlock(&c->mu);
        if (row >= (int64_t)c->ih) break;
        for (size_t col = 0; col < c->iw; col++) {
            size_t px = ((size_t)row * c->iw + col) * bands;
            size_t ix = ((size_t)row * c->iw + col) * 2;
            double rx = mp_index(c, ix), ry = mp_index(c, ix + 1);
            if (!c->premultiplied && (bands == 2 || bands == 4)) {
                mp_pixel_pm(c, &s, rx, ry, &o, px);
                continue;
            }
            if (!isfinite(rx) || !isfinite(ry)) {
                for (size_t b2 = 0; b2 < bands; b2++) tset_f64(&o, px + b2, c->bg);
                continue;
            }
            if (c->kernel == OR_K_NEAREST) {
                int64_t x0 = f2i(floor(rx)), y0 = f2i(floor(ry));
                for (size_t b2 = 0; b2 < bands; b2++) tset_f64(&o, px + b2, mp_band(c, &s, x0, y0, (int32_t)b2));
            } else if (c->kernel == OR_K_BILINEAR) {
                int64_t x0 = f2i(floor(rx)), y0 = f2i(floor(ry));
                double fx = rx - (double)x0, fy = ry - (double)y0;
                int interior = x0 >= 0 && x0 + 1 < (int64_t)c->sw && y0 >= 0 && y0 + 1 < (int64_t)c->sh;
                for (size_t b2 = 0; b2 < bands; b2++) {
                    double p00 = mp_band(c, &s, x0, y0, (int32_t)b2), p01 = mp_band(c, &s, x0 + 1, y0, (int32_t)b2);
                    double p10 = mp_band(c, &s, x0, y0 + 1, (int32_t)b2), p11 = mp_band(c, &s, x0 + 1, y0 + 1, (int32_t)b2);
                    double top, bottom;
                    if (interior) { top = fma(p01, fx, p00 * (1.0 - fx)); bottom = fma(p11, fx, p10 * (1.0 - fx)); }
                    else { top = fma(p00, 1.0 - fx, p01 * fx); bottom = p10 * (1.0 - fx) + p11 * fx; }
                    tset_f64(&o, px + b2, top * (1.0 - fy) + bottom * fy);
                }
            } else {
                for (size_t b2 = 0; b2 < bands; b2++)
                    tset_f64(&o, px + b2, aff_sample_at(&ac, rx, ry, (int32_t)b2, 0, 0, 1.0));
            }
        }
    }
    return NULL;
}

int32_t or_mapim_run(const void *src, uint32_t sw, uint32_t sh, uint32_t bands, int32_t fmt,
                     const void *index, int32_t index_fmt, uint32_t iw, uint32_t ih, int32_t kernel,
                     int32_t extend_copy, double background, int32_t premultiplied, int32_t threads,
                     void *dst) {
    if (!src || !index || !dst || bands == 0) return OR_EINVAL;
    if (index_fmt != OR_U8 && index_fmt != OR_U16 && index_fmt != OR_F32) return OR_EFORMAT;
    if (kernel == OR_K_NOHALO || kernel == OR_K_LBB || kernel == OR_K_VSQBS) return OR_EFORMAT;
    mapim_ctx c;
    memset(&c, 0, sizeof(c));
    c.src = src; c.sw = sw; c.sh = sh; c.bands = bands; c.fmt = fmt; c.index = index;
    c.index_fmt = index_fmt; c.iw = iw; c.ih = ih;
    c.kernel = kernel; c.extend_copy = extend_copy; c.bg = background; c.premultiplied = premultiplied; c.dst = dst;
    pthread_mutex_init(&c.mu, NULL);
    int32_t nt = threads > 0 ? threads : 1;
    if (nt > 256) nt = 256;
    pthread_t th[256];
    for (int32_t i = 1; i < nt; i++) pthread_create(&th[i], NULL, mapim_worker, &c);
    mapim_worker(&c);
    for (int32_t i = 1; i < nt; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&c.mu);
    return OR_OK;
}
