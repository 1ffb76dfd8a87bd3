// affine_dev.cuh -- device code of the affine and mapim interpolators (see
// affine.cu for the viprs files it follows).  Included by affine.cu and batch.cu.
#pragma once

#include "affine_launch.hpp"
#include "common.cuh"
#include "interp_weights.hpp"
#include "sin_rn.cuh"

namespace viprs {
namespace dev {

__device__ __forceinline__ int64_t trunc_i64(double v) {
    // Rust `as i64` for the finite, moderate values reaching here
    return (int64_t)v;
}

__device__ __forceinline__ int64_t tile_origin(int64_t v, int64_t off, int64_t t) {
    const int64_t d = v - off;
    if (d >= 0 && d <= 0x7fffffff && t <= 0x7fffffff)  // 32-bit division covers real images
        return off + (int64_t)((uint32_t)d / (uint32_t)t) * t;
    const int64_t q = d >= 0 ? d / t : -((-d + t - 1) / t);
    return off + q * t;
}

template <typename T>
struct AffineCtx {
    const AffineArgs& a;
    // the scheduler tile's input region (Affine::required_input_region clipped
    // to the source bounds): viprs samples outside it read the fill value
    int64_t rx0 = 0, rx1 = -1, ry0 = 0, ry1 = -1;
    __device__ AffineCtx(const AffineArgs& args) : a(args) {}

    __device__ void set_tile(int64_t X, int64_t Y) {
        rx0 = 0; rx1 = (int64_t)a.src_w - 1; ry0 = 0; ry1 = (int64_t)a.src_h - 1;
        if (X < a.tile_off_x || X >= a.tile_off_x + (int64_t)a.final_w || Y < a.tile_off_y ||
            Y >= a.tile_off_y + (int64_t)a.final_h)
            return;  // outside the tile grid (a downstream halo): image bounds only
        const int64_t X0 = tile_origin(X, a.tile_off_x, a.tile_w), Y0 = tile_origin(Y, a.tile_off_y, a.tile_h);
        const int64_t TW = min((int64_t)a.tile_w, a.tile_off_x + (int64_t)a.final_w - X0);
        const int64_t TH = min((int64_t)a.tile_h, a.tile_off_y + (int64_t)a.final_h - Y0);
        const double* m = a.m;
        const double xs[2] = {(double)X0, (double)X0 + (double)(TW - 1)};
        const double ys[2] = {(double)Y0, (double)Y0 + (double)(TH - 1)};
        double mnx = 0, mxx = 0, mny = 0, mxy = 0;
        for (int i = 0; i < 4; ++i) {
            const double x = xs[i & 1], y = ys[i >> 1];
            const double cx = fma(m[1], y, m[0] * x) + a.tx, cy = fma(m[3], y, m[2] * x) + a.ty;
            if (i == 0) { mnx = mxx = cx; mny = mxy = cy; }
            else { mnx = fmin(mnx, cx); mxx = fmax(mxx, cx); mny = fmin(mny, cy); mxy = fmax(mxy, cy); }
        }
        int lp = 1, rp = 2;
        if (a.kernel == 0) { lp = 0; rp = 0; }
        else if (a.kernel == 1) { lp = 0; rp = 1; }
        else if (a.kernel == 9 || a.kernel == 4) { lp = 2; rp = 3; }
        const int64_t x0 = trunc_i64(floor(mnx)) - lp, x1 = trunc_i64(floor(mxx)) + rp;
        const int64_t y0 = trunc_i64(floor(mny)) - lp, y1 = trunc_i64(floor(mxy)) + rp;
        rx0 = max(x0, (int64_t)0); rx1 = min(x1, (int64_t)a.src_w - 1);
        ry0 = max(y0, (int64_t)0); ry1 = min(y1, (int64_t)a.src_h - 1);
    }

    __device__ double fill() const {
        if (a.extend == 1) return sizeof(T) == 4 ? 1.0 : (sizeof(T) == 2 ? 65535.0 : 255.0);
        if (a.extend == 2) return a.background;
        return 0.0;
    }
    __device__ bool resolve(int64_t c, int64_t size, int64_t* r) const {
        if (size <= 0) return false;
        if (c >= 0 && c < size) { *r = c; return true; }
        switch (a.extend) {
        case 3: *r = c < 0 ? 0 : size - 1; return true;
        case 4: { int64_t m = c % size; if (m < 0) m += size; *r = m; return true; }
        case 5: {
            const int64_t p = size * 2;
            int64_t w = c % p;
            if (w < 0) w += p;
            *r = w < size ? w : p - 1 - w;
            return true;
        }
        default: return false;
        }
    }
    // Tap (ix, iy) resolved against the source bounds (extend) and the tile's
    // input region: its in-plane address (always readable) and whether it
    // reads the image (false: the fill value).
    __device__ __forceinline__ const T* tap(int64_t ix, int64_t iy, bool* ok) const {
        int64_t rx = 0, ry = 0;
        const bool okx = resolve(ix, a.src_w, &rx);
        const bool oky = resolve(iy, a.src_h, &ry);
        *ok = okx && oky && rx >= rx0 && rx <= rx1 && ry >= ry0 && ry <= ry1;
        return sample_ptr<T>(a.in, rx - a.in.x0, ry - a.in.y0, a.bands);
    }
    // Affine::sample_band: extend against the source bounds, read the plane
    __device__ double sb(int64_t ix, int64_t iy, int band) const {
        bool ok;
        const double v = (double)tap(ix, iy, &ok)[band];
        return ok ? v : fill();
    }
    __device__ double sbp(int64_t ix, int64_t iy, int band, int ab, double amax) const {
        const double v = sb(ix, iy, band);
        if (band == ab) return v;
        return v * (sb(ix, iy, ab) / amax);
    }
    __device__ double sample(double x, double y, int band, bool pm, int ab, double amax) const {
        if (!isfinite(x) || !isfinite(y)) return fill();
        const int k = a.kernel;
        if (k == 0) {
            const int64_t ix = trunc_i64(x), iy = trunc_i64(y);
            return pm ? sbp(ix, iy, band, ab, amax) : sb(ix, iy, band);
        }
        if (k == 1) {
            const int64_t x0 = trunc_i64(x), y0 = trunc_i64(y);
            const double fx = x - (double)x0, fy = y - (double)y0;
            double p00, p01, p10, p11;
            if (pm) {
                p00 = sbp(x0, y0, band, ab, amax); p01 = sbp(x0 + 1, y0, band, ab, amax);
                p10 = sbp(x0, y0 + 1, band, ab, amax); p11 = sbp(x0 + 1, y0 + 1, band, ab, amax);
            } else {
                p00 = sb(x0, y0, band); p01 = sb(x0 + 1, y0, band);
                p10 = sb(x0, y0 + 1, band); p11 = sb(x0 + 1, y0 + 1, band);
            }
            const double top = fma(p01, fx, p00 * (1.0 - fx));
            const double bottom = fma(p11, fx, p10 * (1.0 - fx));
            return top * (1.0 - fy) + bottom * fy;
        }
        // taps cx - (support - 1) .. cx + support per axis, each axis's
        // weights evaluated once, taps with a zero weight skipped
        const int support = k == 9 ? 3 : 2;
        const int nt = 2 * support;
        const int64_t cx = trunc_i64(floor(x)), cy = trunc_i64(floor(y));
        const int64_t tx0 = cx - (support - 1), ty0 = cy - (support - 1);
        double wxs[6], wys[6];
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            wxs[t] = t < nt ? kernel_w(k, fabs((double)(tx0 + t) - x)) : 0.0;
            wys[t] = t < nt ? kernel_w(k, fabs((double)(ty0 + t) - y)) : 0.0;
        }
        double acc = 0.0, wsum = 0.0;
        for (int j = 0; j < nt; ++j) {
            const double wy = wys[j];
            if (wy == 0.0) continue;
            const int64_t iy = ty0 + j;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                if (i >= nt) break;
                const double s = pm ? sbp(tx0 + i, iy, band, ab, amax) : sb(tx0 + i, iy, band);
                const double wx = wxs[i];
                if (wx != 0.0) {
                    const double w = wx * wy;
                    wsum += w;
                    acc = fma(s, w, acc);
                }
            }
        }
        return wsum > 0.0 ? acc / wsum : fill();
    }
    // Bilinear taps (x0 + dx, y0 + dy), dx, dy in {0, 1}, every band of a tap
    // read once: v[k][b] = sb(x0 + (k & 1), y0 + (k >> 1), b) for k = 0..3.
    template <int NB>
    __device__ void taps4(int64_t x0, int64_t y0, double (&v)[4][NB]) const {
        const double f = fill();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            bool ok;
            const T* px = tap(x0 + (k & 1), y0 + (k >> 1), &ok);
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const double s = (double)px[b];
                v[k][b] = ok ? s : f;
            }
        }
    }
    __device__ static double bil4(double p00, double p01, double p10, double p11, double fx, double fy) {
        const double top = fma(p01, fx, p00 * (1.0 - fx));
        const double bottom = fma(p11, fx, p10 * (1.0 - fx));
        return top * (1.0 - fy) + bottom * fy;
    }
    // pixel() for the bilinear kernel with NB == a.bands: the same arithmetic
    // per band as sample() / sbp(), with each tap read once.
    template <int NB>
    __device__ void pixel_bilinear(double x, double y, double* out) const {
        if (!isfinite(x) || !isfinite(y)) {
#pragma unroll
            for (int b = 0; b < NB; ++b) out[b] = fill();
            return;
        }
        const int64_t x0 = trunc_i64(x), y0 = trunc_i64(y);
        const double fx = x - (double)x0, fy = y - (double)y0;
        double v[4][NB];
        taps4<NB>(x0, y0, v);
        if (NB == 4 && !a.premultiplied) {
            constexpr int ab = NB - 1;
            const double amax = sizeof(T) == 4 ? 1.0 : (sizeof(T) == 2 ? 65535.0 : 255.0);
            double alpha = bil4(v[0][ab], v[1][ab], v[2][ab], v[3][ab], fx, fy);
            alpha = alpha < 0.0 ? 0.0 : (alpha > amax ? amax : alpha);
            const double na = alpha / amax;
            double s[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) s[k] = v[k][ab] / amax;
#pragma unroll
            for (int b = 0; b < ab; ++b) {
                const double p = bil4(v[0][b] * s[0], v[1][b] * s[1], v[2][b] * s[2], v[3][b] * s[3], fx, fy);
                out[b] = na > 0.0 ? p / na : 0.0;
            }
            out[ab] = alpha;
            return;
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) out[b] = bil4(v[0][b], v[1][b], v[2][b], v[3][b], fx, fy);
    }
    // Affine::sample_pixel_at into out[0..bands)
    // NB: compile-time band count (0: a.bands at run time) -- with it the
    // caller's per-band arrays stay in registers
    template <int NB = 0>
    __device__ void pixel(double x, double y, double* out) const {
        const int bands = NB > 0 ? NB : a.bands;
        if (NB > 0 && a.kernel == 1) {
            pixel_bilinear<(NB > 0 ? NB : 1)>(x, y, out);
            return;
        }
        if (a.kernel == 1) {
            switch (bands) {
            case 1: pixel_bilinear<1>(x, y, out); return;
            case 2: pixel_bilinear<2>(x, y, out); return;
            case 3: pixel_bilinear<3>(x, y, out); return;
            case 4: pixel_bilinear<4>(x, y, out); return;
            default: break;
            }
        }
        if (a.kernel >= 2) {
            // separable kernels: each axis's weights once for all bands (the
            // values sample() evaluates per band), then pixel_tab's taps
            if (!isfinite(x) || !isfinite(y)) {
                for (int b = 0; b < bands; ++b) out[b] = fill();
                return;
            }
            const int k = a.kernel, nt = separable_taps(k), support = nt / 2;
            const int64_t tx0 = trunc_i64(floor(x)) - (support - 1), ty0 = trunc_i64(floor(y)) - (support - 1);
            double wxs[kAxisTaps], wys[kAxisTaps];
#pragma unroll
            for (int t = 0; t < kAxisTaps; ++t) {
                wxs[t] = t < nt ? kernel_w(k, fabs((double)(tx0 + t) - x)) : 0.0;
                wys[t] = t < nt ? kernel_w(k, fabs((double)(ty0 + t) - y)) : 0.0;
            }
            pixel_tab<NB>(x, y, wxs, wys, out);
            return;
        }
        if (bands == 4 && !a.premultiplied) {
            if (!isfinite(x) || !isfinite(y)) {
                for (int b = 0; b < bands; ++b) out[b] = fill();
                return;
            }
            const int ab = bands - 1;
            const double amax = sizeof(T) == 4 ? 1.0 : (sizeof(T) == 2 ? 65535.0 : 255.0);
            double alpha = sample(x, y, ab, true, ab, amax);
            alpha = alpha < 0.0 ? 0.0 : (alpha > amax ? amax : alpha);
            const double na = alpha / amax;
            for (int b = 0; b < ab; ++b) {
                const double p = sample(x, y, b, true, ab, amax);
                out[b] = na > 0.0 ? p / na : 0.0;
            }
            out[ab] = alpha;
            return;
        }
        if (!isfinite(x) || !isfinite(y)) {
            for (int b = 0; b < bands; ++b) out[b] = fill();
            return;
        }
        if (a.kernel == 0) {
            const int64_t ix = trunc_i64(x), iy = trunc_i64(y);
            int64_t rx, ry;
            if (!resolve(ix, a.src_w, &rx) || !resolve(iy, a.src_h, &ry) || rx < rx0 || rx > rx1 || ry < ry0 ||
                ry > ry1) {
                for (int b = 0; b < bands; ++b) out[b] = fill();
                return;
            }
            for (int b = 0; b < bands; ++b) out[b] = (double)load_sample<T>(a.in, rx - a.in.x0, ry - a.in.y0, bands, b);
            return;
        }
        for (int b = 0; b < bands; ++b) out[b] = sample(x, y, b, false, 0, 1.0);
    }
    // pixel() for the separable kernels with the point-sampling weights of the
    // pixel's column and row given (kAxisTaps each): the taps, their order, the
    // weight sum and the fma accumulation of sample() / sbp(), every tap read
    // once for all bands.  x and y are finite (per-axis table positions).
    template <int NB = 0>
    __device__ void pixel_tab(double x, double y, const double* wxs, const double* wys, double* out) const {
        constexpr int MB = NB > 0 ? NB : 8;
        const int bands = NB > 0 ? NB : a.bands;
        const int nt = separable_taps(a.kernel), support = nt / 2;
        const int64_t tx0 = trunc_i64(floor(x)) - (support - 1), ty0 = trunc_i64(floor(y)) - (support - 1);
        const bool pm = bands == 4 && !a.premultiplied;
        const int ab = bands - 1;
        const double amax = sizeof(T) == 4 ? 1.0 : (sizeof(T) == 2 ? 65535.0 : 255.0);
        const double f = fill();
        if (!isfinite(x) || !isfinite(y)) {
            for (int b = 0; b < bands; ++b) out[b] = f;
            return;
        }
        double wx[kAxisTaps], acc[MB];
#pragma unroll
        for (int t = 0; t < kAxisTaps; ++t) wx[t] = wxs[t];
#pragma unroll
        for (int b = 0; b < MB; ++b) acc[b] = 0.0;
        double wsum = 0.0;
        // every tap inside the image, the tile's input region and the plane:
        // each reads the image at its own address (tap() would resolve to the
        // same), so the taps are loaded directly
        const int64_t px0 = tx0 - a.in.x0, py0 = ty0 - a.in.y0;
        const bool interior = tx0 >= rx0 && tx0 + nt - 1 <= rx1 && ty0 >= ry0 && ty0 + nt - 1 <= ry1 &&
                              px0 >= 0 && px0 + nt <= (int64_t)a.in.w && py0 >= 0 && py0 + nt <= (int64_t)a.in.h;
        if (interior && !pm) {
            const uint8_t* row = a.in.data + py0 * a.in.pitch;
            for (int j = 0; j < nt; ++j, row += a.in.pitch) {
                const double wy = wys[j];
                if (wy == 0.0) continue;
                const T* px = reinterpret_cast<const T*>(row) + px0 * bands;
#pragma unroll
                for (int i = 0; i < kAxisTaps; ++i) {
                    if (i >= nt) break;
                    if (wx[i] == 0.0) continue;
                    const double w = wx[i] * wy;
                    wsum += w;
#pragma unroll
                    for (int b = 0; b < MB; ++b) {
                        if (b >= bands) break;
                        acc[b] = fma((double)px[i * bands + b], w, acc[b]);
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < MB; ++b) {
                if (b >= bands) break;
                out[b] = wsum > 0.0 ? acc[b] / wsum : f;
            }
            return;
        }
        for (int j = 0; j < nt; ++j) {
            const double wy = wys[j];
            if (wy == 0.0) continue;
            const int64_t iy = ty0 + j;
#pragma unroll
            for (int i = 0; i < kAxisTaps; ++i) {
                if (i >= nt) break;
                if (wx[i] == 0.0) continue;
                const double w = wx[i] * wy;
                wsum += w;
                bool ok;
                const T* px = tap(tx0 + i, iy, &ok);
                if (pm) {
                    const double av = ok ? (double)px[ab] : f;
#pragma unroll
                    for (int b = 0; b < MB; ++b) {
                        if (b >= ab) break;
                        const double v = ok ? (double)px[b] : f;
                        acc[b] = fma(v * (av / amax), w, acc[b]);
                    }
                    acc[ab] = fma(av, w, acc[ab]);
                } else {
#pragma unroll
                    for (int b = 0; b < MB; ++b) {
                        if (b >= bands) break;
                        const double v = ok ? (double)px[b] : f;
                        acc[b] = fma(v, w, acc[b]);
                    }
                }
            }
        }
        if (pm) {
            double alpha = wsum > 0.0 ? acc[ab] / wsum : f;
            alpha = alpha < 0.0 ? 0.0 : (alpha > amax ? amax : alpha);
            const double na = alpha / amax;
#pragma unroll
            for (int b = 0; b < MB; ++b) {
                if (b >= ab) break;
                const double p = wsum > 0.0 ? acc[b] / wsum : f;
                out[b] = na > 0.0 ? p / na : 0.0;
            }
            out[ab] = alpha;
            return;
        }
#pragma unroll
        for (int b = 0; b < MB; ++b) {
            if (b >= bands) break;
            out[b] = wsum > 0.0 ? acc[b] / wsum : f;
        }
    }
};

template <typename T>
__device__ __forceinline__ T store_round(double v, bool u8_round_first) {
    if (sizeof(T) == 1 && u8_round_first) {
        double r = round(v);
        r = r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r);
        return (T)(uint32_t)r;
    }
    return from_f64<T>(v);
}

// Output pixel (lx, ly) from its sampled values: round, unpremultiply (u8), store.
template <typename T, int NB = 0>
__device__ __forceinline__ void affine_store(const AffineArgs& a, int64_t lx, int64_t ly, const double* v,
                                             bool u8_round_first) {
    const int bands = NB > 0 ? NB : a.bands;
    T* dst = reinterpret_cast<T*>(a.out.data + ly * a.out.pitch) + lx * bands;
    T o[NB > 0 ? NB : 8];
    for (int b = 0; b < bands; ++b) o[b] = store_round<T>(v[b], u8_round_first);
    if (sizeof(T) == 1 && a.unpremul_out && bands >= 2) {
        const uint32_t al = (uint32_t)o[bands - 1];
        for (int b = 0; b < bands - 1; ++b) o[b] = (T)unpremultiply_u8((uint32_t)o[b], al);
    }
    for (int b = 0; b < bands; ++b) dst[b] = o[b];
}

// State of one thread walking along an output row: the scheduler tile it is
// in (origin, and whether the pixel lies inside the tile grid -- together they
// decide the tile's input region, refreshed only when they change) and the
// incremental position walk.  viprs's position of pixel X of row Y is the
// tile row's start (the tile origin's position plus m1 / m3 added Y - Y0
// times) plus m0 / m2 added X - X0 times, so consecutive pixels of one tile
// add one step each and the walk restarts only where a tile begins.
struct AffineRow {
    int64_t tX0 = INT64_MIN;
    int grid = -1;
    int64_t wX = INT64_MIN, wX0 = INT64_MIN;  // last walked pixel and its tile
    double x = 0.0, y = 0.0;

    template <typename T>
    __device__ __forceinline__ void tile(const AffineArgs& a, AffineCtx<T>& c, int64_t X, int64_t Y) {
        const int64_t X0 = tile_origin(X, a.tile_off_x, a.tile_w);
        const int g = X >= a.tile_off_x && X < a.tile_off_x + (int64_t)a.final_w && Y >= a.tile_off_y &&
                      Y < a.tile_off_y + (int64_t)a.final_h;
        if (X0 != tX0 || g != grid) c.set_tile(X, Y);
        tX0 = X0;
        grid = g;
    }
    // position of (X, Y) by the walk; tile() has been called for X
    __device__ __forceinline__ void walk(const AffineArgs& a, int64_t X, int64_t Y) {
        const double* m = a.m;
        if (wX0 == tX0 && X == wX + 1) {
            x += m[0];
            y += m[2];
        } else {
            const int64_t Y0 = tile_origin(Y, a.tile_off_y, a.tile_h);
            double rx = fma(m[1], (double)Y0, m[0] * (double)tX0) + a.tx;
            double ry = fma(m[3], (double)Y0, m[2] * (double)tX0) + a.ty;
            for (int64_t r = Y0; r < Y; ++r) { rx += m[1]; ry += m[3]; }
            x = rx; y = ry;
            for (int64_t q = tX0; q < X; ++q) { x += m[0]; y += m[2]; }
        }
        wX = X;
        wX0 = tX0;
    }
};

// One output pixel (lx, ly) of the plane a.out; c and row carry the thread's
// state along the row (pixels of one thread advance left to right).
template <typename T, int NB = 0>
__device__ void affine_pixel(const AffineArgs& a, AffineCtx<T>& c, AffineRow& row, int64_t lx, int64_t ly) {
    const int64_t X = a.out.x0 + lx, Y = a.out.y0 + ly;
    const int bands = NB > 0 ? NB : a.bands;
    row.tile<T>(a, c, X, Y);
    double v[NB > 0 ? NB : 8];
    bool u8_round_first = false;
    const double* m = a.m;
    // fast paths and per-axis tables cover the affine's own output rectangle; a
    // region requested beyond it (a downstream op's halo) takes the general walk
    const bool inside = X >= 0 && X < (int64_t)a.total_w && Y >= 0 && Y < (int64_t)a.total_h;
    const int fast = inside ? a.fast : 0;
    if (fast == 1) {
        // process_region_nearest_fast (core.rs:1097-1143)
        const int64_t xc = trunc_i64(fma(m[0], (double)X, a.tx)), yc = trunc_i64(fma(m[3], (double)Y, a.ty));
        if (yc < 0 || yc >= (int64_t)a.src_h || xc < 0 || xc >= (int64_t)a.src_w) {
            for (int b = 0; b < bands; ++b) v[b] = c.fill();
        } else {
            for (int b = 0; b < bands; ++b) v[b] = (double)load_sample<T>(a.in, xc - a.in.x0, yc - a.in.y0, bands, b);
        }
    } else if (fast == 2) {
        // process_region_bilinear_fast (core.rs:1145-1219)
        const double cxr = fma(m[0], (double)X, a.tx), cyr = fma(m[3], (double)Y, a.ty);
        const int64_t xs = trunc_i64(cxr), ys = trunc_i64(cyr);
        const double wx1 = cxr - (double)xs, wx0 = 1.0 - wx1;
        const double wy1 = cyr - (double)ys, wy0 = 1.0 - wy1;
        if (ys < 0 || ys + 1 >= (int64_t)a.src_h || xs < 0 || xs + 1 >= (int64_t)a.src_w) {
            for (int b = 0; b < bands; ++b) v[b] = c.sample((double)xs + wx1, (double)ys + wy1, b, false, 0, 1.0);
        } else {
            for (int b = 0; b < bands; ++b) {
                const int64_t bx = xs - a.in.x0, by = ys - a.in.y0;
                const double p00 = (double)load_sample<T>(a.in, bx, by, bands, b);
                const double p01 = (double)load_sample<T>(a.in, bx + 1, by, bands, b);
                const double p10 = (double)load_sample<T>(a.in, bx, by + 1, bands, b);
                const double p11 = (double)load_sample<T>(a.in, bx + 1, by + 1, bands, b);
                const double top = fma(p01, wx1, p00 * wx0), bottom = fma(p11, wx1, p10 * wx0);
                v[b] = fma(bottom, wy1, top * wy0);
            }
        }
    } else if (fast == 3) {
        // process_region_bicubic_fast[_u8] (core.rs:1221-1513), build_cubic_axis (:163-189)
        const double cxr = fma(m[0], (double)X, a.tx), cyr = fma(m[3], (double)Y, a.ty);
        const int64_t xs = trunc_i64(floor(cxr)) - 1, ys = trunc_i64(floor(cyr)) - 1;
        u8_round_first = true;
        if (ys < 0 || ys + 3 >= (int64_t)a.src_h || xs < 0 || xs + 3 >= (int64_t)a.src_w) {
            if (sizeof(T) == 1) {
                for (int b = 0; b < bands; ++b) v[b] = c.sample(cxr, cyr, b, false, 0, 1.0);
            } else {
                c.template pixel<NB>(cxr, cyr, v);
                u8_round_first = false;
            }
        } else {
            double wx[4], wy[4], sx = 0.0, sy = 0.0;
            for (int t = 0; t < 4; ++t) {
                wx[t] = bicubic_w(fabs((double)(xs + t) - cxr));
                wy[t] = bicubic_w(fabs((double)(ys + t) - cyr));
            }
            for (int t = 0; t < 4; ++t) { sx += wx[t]; sy += wy[t]; }
            if (sx > 0.0) for (int t = 0; t < 4; ++t) wx[t] /= sx;
            if (sy > 0.0) for (int t = 0; t < 4; ++t) wy[t] /= sy;
            const int64_t bx = xs - a.in.x0, by = ys - a.in.y0;
            for (int b = 0; b < bands; ++b) {
                double acc = 0.0;
                for (int r = 0; r < 4; ++r) {
                    const double p0 = (double)load_sample<T>(a.in, bx, by + r, bands, b);
                    const double p1 = (double)load_sample<T>(a.in, bx + 1, by + r, bands, b);
                    const double p2 = (double)load_sample<T>(a.in, bx + 2, by + r, bands, b);
                    const double p3 = (double)load_sample<T>(a.in, bx + 3, by + r, bands, b);
                    const double ra = fma(p3, wx[3], fma(p2, wx[2], fma(p1, wx[1], p0 * wx[0])));
                    acc = fma(ra, wy[r], acc);
                }
                v[b] = acc;
            }
        }
    } else if (a.wx != nullptr && inside) {
        // separable walk, weights from the per-axis tables
        c.template pixel_tab<NB>(a.xs[X], a.ys[Y], a.wx + X * kAxisTaps, a.wy + Y * kAxisTaps, v);
    } else {
        double x_in, y_in;
        if (a.separable && a.xs != nullptr && inside) {
            x_in = a.xs[X];
            y_in = a.ys[Y];
        } else {
            row.walk(a, X, Y);
            x_in = row.x;
            y_in = row.y;
        }
        c.template pixel<NB>(x_in, y_in, v);
    }
    affine_store<T, NB>(a, lx, ly, v, u8_round_first);
}

// One output pixel with fresh per-thread state (threads striding over a row).
template <typename T>
__device__ void affine_pixel(const AffineArgs& a, int64_t lx, int64_t ly) {
    AffineCtx<T> c(a);
    AffineRow row;
    affine_pixel<T>(a, c, row, lx, ly);
}

// Threads over groups of a.group consecutive pixels of a row, block rows over
// the output rows (grid-stride): a thread's pixels share the tile region and
// the incremental walk.
template <typename T, int NB>
__global__ void __launch_bounds__(256, 2) affine_kernel(AffineArgs a) {
    const int G = a.group;
    const int64_t lx0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * G;
    if (lx0 >= a.out.w) return;
    const int64_t lx1 = min((int64_t)a.out.w, lx0 + G);
    for (int64_t ly = blockIdx.y; ly < a.out.h; ly += gridDim.y) {
        AffineCtx<T> c(a);
        AffineRow row;
        for (int64_t lx = lx0; lx < lx1; ++lx) affine_pixel<T, NB>(a, c, row, lx, ly);
    }
}


// ---------------------------------------------------------------- mapim
// Tap (ix, iy) of mapim's source read: its address (always readable) and
// whether it reads the image (false: the background).
template <typename T>
__device__ __forceinline__ const T* mp_tap(const MapimArgs& a, int64_t ix, int64_t iy, bool* ok) {
    if (!a.extend_copy) {
        *ok = !(ix < 0 || ix >= (int64_t)a.src_w || iy < 0 || iy >= (int64_t)a.src_h);
    } else {
        int lp = 1, rp = 2;
        if (a.kernel == 0) { lp = 0; rp = 0; }
        else if (a.kernel == 1) { lp = 0; rp = 1; }
        else if (a.kernel == 9 || a.kernel == 4) { lp = 2; rp = 3; }
        *ok = !(ix < -(int64_t)(lp + 1) || ix > (int64_t)a.src_w + rp || iy < -(int64_t)(lp + 1) ||
                iy > (int64_t)a.src_h + rp);
    }
    const int64_t x = clampi64(ix, 0, (int64_t)a.src_w - 1), y = clampi64(iy, 0, (int64_t)a.src_h - 1);
    return sample_ptr<T>(a.src, x, y, a.bands);
}

template <typename T>
__device__ __forceinline__ double mp_band(const MapimArgs& a, int64_t ix, int64_t iy, int band) {
    bool ok;
    const double v = (double)mp_tap<T>(a, ix, iy, &ok)[band];
    return ok ? v : a.background;
}

// Coordinates of output pixel (lx, ly) from the index image, read as f64
// whatever the index format (mapim.rs:1135-1274 reads them through ToF64).
__device__ __forceinline__ void mp_coords(const MapimArgs& a, int64_t lx, int64_t ly, double* rx, double* ry) {
    const uint8_t* row = a.index.data + ly * a.index.pitch;
    if (a.index_fmt == kF32) {
        const float2 v = *reinterpret_cast<const float2*>(row + lx * 8);
        *rx = (double)v.x; *ry = (double)v.y;
    } else if (a.index_fmt == kU16) {
        const ushort2 v = *reinterpret_cast<const ushort2*>(row + lx * 4);
        *rx = (double)v.x; *ry = (double)v.y;
    } else {
        *rx = (double)row[lx * 2]; *ry = (double)row[lx * 2 + 1];
    }
}

// NT: taps per axis of the separable samplers (4: support 2, 6: Lanczos3);
// 0 for the nearest / bilinear kernels.
template <typename T, int NT>
__device__ __forceinline__ void mapim_px(const MapimArgs& a, int64_t lx, int64_t ly) {
    double rx, ry;
    mp_coords(a, lx, ly, &rx, &ry);
    const int bands = a.bands;
    T* dst = reinterpret_cast<T*>(a.out.data + ly * a.out.pitch) + lx * bands;
    if (!isfinite(rx) || !isfinite(ry)) {
        for (int b = 0; b < bands; ++b) dst[b] = from_f64<T>(a.background);
        return;
    }
    if (NT == 0) {
        if (a.kernel == 0) {
            const int64_t x0 = trunc_i64(floor(rx)), y0 = trunc_i64(floor(ry));
            for (int b = 0; b < bands; ++b) dst[b] = from_f64<T>(mp_band<T>(a, x0, y0, b));
            return;
        }
        const int64_t x0 = trunc_i64(floor(rx)), y0 = trunc_i64(floor(ry));
        const double fx = rx - (double)x0, fy = ry - (double)y0;
        const bool interior = x0 >= 0 && x0 + 1 < (int64_t)a.src_w && y0 >= 0 && y0 + 1 < (int64_t)a.src_h;
        bool ok[4];
        const T* t[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) t[q] = mp_tap<T>(a, x0 + (q & 1), y0 + (q >> 1), &ok[q]);
        for (int b = 0; b < bands; ++b) {
            double v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double s = (double)t[q][b];
                v[q] = ok[q] ? s : a.background;
            }
            const double p00 = v[0], p01 = v[1], p10 = v[2], p11 = v[3];
            double top, bottom;
            if (interior) { top = fma(p01, fx, p00 * (1.0 - fx)); bottom = fma(p11, fx, p10 * (1.0 - fx)); }
            else { top = fma(p00, 1.0 - fx, p01 * fx); bottom = p10 * (1.0 - fx) + p11 * fx; }
            dst[b] = from_f64<T>(top * (1.0 - fy) + bottom * fy);
        }
        return;
    }
    // Affine sampler with Background(bg) over the source read region
    // (mapim.rs:1178-1186, 1250-1271): taps cx - (support - 1) .. cx + support
    // per axis, weights evaluated once per axis, the weight sum (the same for
    // every band) accumulated in the sampler's tap order.
    constexpr int nt = NT > 0 ? NT : 1;
    constexpr int support = nt / 2;
    const int k = a.kernel;
    const int64_t cx = trunc_i64(floor(rx)), cy = trunc_i64(floor(ry));
    const int64_t tx0 = cx - (support - 1), ty0 = cy - (support - 1);
    double wx[nt], wy[nt];
#pragma unroll
    for (int t = 0; t < nt; ++t) {
        wx[t] = kernel_w(k, fabs((double)(tx0 + t) - rx));
        wy[t] = kernel_w(k, fabs((double)(ty0 + t) - ry));
    }
    double wsum = 0.0;
#pragma unroll
    for (int j = 0; j < nt; ++j) {
        if (wy[j] == 0.0) continue;
#pragma unroll
        for (int i = 0; i < nt; ++i)
            if (wx[i] != 0.0) wsum += wx[i] * wy[j];
    }
    // per axis: in-bounds flags (background outside) and the clamped row
    // pointers / column offsets, so that every tap loads from a readable address
    bool okx[nt], oky[nt];
    int32_t col[nt];
    const T* rows[nt];
#pragma unroll
    for (int t = 0; t < nt; ++t) {
        const int64_t ix = tx0 + t, iy = ty0 + t;
        okx[t] = ix >= 0 && ix < (int64_t)a.src_w;
        oky[t] = iy >= 0 && iy < (int64_t)a.src_h;
        col[t] = (int32_t)clampi64(ix, 0, (int64_t)a.src_w - 1) * bands;
        rows[t] = reinterpret_cast<const T*>(a.src.data + clampi64(iy, 0, (int64_t)a.src_h - 1) * a.src.pitch);
    }
    for (int b = 0; b < bands; ++b) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < nt; ++j) {
            double sv[nt];
#pragma unroll
            for (int i = 0; i < nt; ++i) sv[i] = (double)rows[j][col[i] + b];
            if (wy[j] == 0.0) continue;
#pragma unroll
            for (int i = 0; i < nt; ++i) {
                if (wx[i] == 0.0) continue;
                const double s = okx[i] && oky[j] ? sv[i] : a.background;
                acc = fma(s, wx[i] * wy[j], acc);
            }
        }
        dst[b] = from_f64<T>(wsum > 0.0 ? acc / wsum : a.background);
    }
}

// Threads along an output row, block rows over the output rows (grid-stride).
template <typename T, int NT>
__global__ void __launch_bounds__(256, 4) mapim_kernel(MapimArgs a) {
    const int64_t lx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lx >= a.out.w) return;
    for (int64_t ly = blockIdx.y; ly < a.out.h; ly += gridDim.y) mapim_px<T, NT>(a, lx, ly);
}

// ---------------------------------------------------------------- mapim, alpha sampler
// 2/4-band sources that are not premultiplied (MapImOp's default): every tap
// is premultiplied by its own alpha / alpha_max before interpolation, the
// interpolated alpha is clamped to [0, alpha_max] and each colour band is
// divided by it (sample_source_with_premultiplied_alpha_into,
// mapim.rs:993-1040; taps through sample_source_band_premultiplied, :616-636,
// and mapim's own extend rules, :306-384).

template <typename T>
__device__ __forceinline__ double mp_band_pm(const MapimArgs& a, int64_t ix, int64_t iy, int band, int ab,
                                             double amax) {
    bool ok;
    const T* px = mp_tap<T>(a, ix, iy, &ok);
    const double v = ok ? (double)px[band] : a.background;
    if (band == ab) return v;
    const double al = ok ? (double)px[ab] : a.background;
    return v * (al / amax);
}

// sample_at_premultiplied (mapim.rs:638-931) for nearest, bilinear (both at
// floor()) and the separable kernels (sample_at_premultiplied_separable,
// :935-991: taps cx - (support - 1) .. cx + support, zero weights skipped,
// renormalised by the weight sum).
template <typename T>
__device__ double mp_sample_pm(const MapimArgs& a, double x, double y, int band, int ab, double amax) {
    const int k = a.kernel;
    const int64_t cx = trunc_i64(floor(x)), cy = trunc_i64(floor(y));
    if (k == 0) return mp_band_pm<T>(a, cx, cy, band, ab, amax);
    if (k == 1) {
        const double fx = x - (double)cx, fy = y - (double)cy;
        const double p00 = mp_band_pm<T>(a, cx, cy, band, ab, amax);
        const double p01 = mp_band_pm<T>(a, cx + 1, cy, band, ab, amax);
        const double p10 = mp_band_pm<T>(a, cx, cy + 1, band, ab, amax);
        const double p11 = mp_band_pm<T>(a, cx + 1, cy + 1, band, ab, amax);
        const double top = fma(p01, fx, p00 * (1.0 - fx));
        const double bottom = fma(p11, fx, p10 * (1.0 - fx));
        return top * (1.0 - fy) + bottom * fy;
    }
    const int support = k == 9 ? 3 : 2;
    double acc = 0.0, wsum = 0.0;
    for (int ky = -(support - 1); ky <= support; ++ky) {
        const int64_t iy = cy + ky;
        const double wy = kernel_w(k, fabs((double)iy - y));
        if (wy == 0.0) continue;
        for (int kx = -(support - 1); kx <= support; ++kx) {
            const int64_t ix = cx + kx;
            const double wx = kernel_w(k, fabs((double)ix - x));
            if (wx != 0.0) {
                const double w = wx * wy;
                wsum += w;
                acc = fma(mp_band_pm<T>(a, ix, iy, band, ab, amax), w, acc);
            }
        }
    }
    return wsum > 0.0 ? acc / wsum : a.background;
}

template <typename T>
__global__ void __launch_bounds__(256) mapim_alpha_kernel(MapimArgs a) {
    const int64_t lx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lx >= a.out.w) return;
    const int bands = a.bands, ab = bands - 1;
    const double amax = sizeof(T) == 4 ? 1.0 : (sizeof(T) == 2 ? 65535.0 : 255.0);
    for (int64_t ly = blockIdx.y; ly < a.out.h; ly += gridDim.y) {
        double rx, ry;
        mp_coords(a, lx, ly, &rx, &ry);
        T* dst = reinterpret_cast<T*>(a.out.data + ly * a.out.pitch) + lx * bands;
        if (!isfinite(rx) || !isfinite(ry)) {
            for (int b = 0; b < bands; ++b) dst[b] = from_f64<T>(a.background);
            continue;
        }
        double alpha = mp_sample_pm<T>(a, rx, ry, ab, ab, amax);
        alpha = alpha < 0.0 ? 0.0 : (alpha > amax ? amax : alpha);
        const double na = alpha / amax;
        for (int b = 0; b < ab; ++b) {
            const double p = mp_sample_pm<T>(a, rx, ry, b, ab, amax);
            dst[b] = from_f64<T>(na > 0.0 ? p / na : 0.0);
        }
        dst[ab] = from_f64<T>(alpha);
    }
}

}  // namespace dev
}  // namespace viprs
