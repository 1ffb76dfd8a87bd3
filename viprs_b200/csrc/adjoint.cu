// adjoint.cu -- backward (adjoint) kernels of the reduce, affine and mapim
// interpolators, f32 images, sm_100a.  No viprs counterpart: viprs's ops are
// forward only; each kernel is the exact transpose / derivative of the
// forward operator as this library evaluates it (forward: resample.cu,
// affine.cu, following resample/reduce*.rs, affine/core.rs, mapim.rs).
//
//   reduce_adjoint_kernel .. atomic-free gather over each input sample's
//                            contributing output span; the clamp-to-edge
//                            boundary folds edge taps onto the first / last
//                            sample, virtual rows fold onto the edge rows
//   affine_grad_kernel ..... d/d(image): scatter of the bilinear weights
//                            (f32 atomics, or a fixed-point accumulator whose
//                            integer adds make the result order-independent);
//                            d/d(matrix, translation): chain rule through the
//                            interpolator's derivative, per-block partial sums
//                            reduced in a fixed order
//   mapim_grad_kernel ...... d/d(image) scatter; d/d(coordinates) by the
//                            quotient rule over the renormalised separable
//                            weights (affine/core.rs:648-696)
#include <algorithm>

#include "adjoint_launch.hpp"
#include "affine_dev.cuh"

namespace viprs {
namespace dev {

// NB bands of one input pixel per thread (NB == 0: a.bands at run time),
// block rows over the input rows (grid-stride); 32-bit indexing (every plane
// holds fewer than 2^31 samples).  Each tap's weight is read once for the
// pixel's bands, 4-band pixels move as one 16-byte load.  f32 weights and
// accumulation, as a backward pass computes: a sample gathers at most a few
// dozen taps, so the rounding stays near f32 epsilon.
template <int NB>
__global__ void __launch_bounds__(256) reduce_adjoint_kernel(ReduceAdjArgs a) {
    constexpr int NBm = NB > 0 ? NB : 1;
    const int B = NB > 0 ? NB : a.bands;
    const int32_t ix = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (ix >= a.in_w) return;
    const int32_t gstride = a.out_w * B;  // g_out row length (samples)
    const int32_t rowlen = a.in_w * B;
    for (int32_t iy = (int32_t)blockIdx.y; iy < a.in_h; iy += (int32_t)gridDim.y) {
        const int32_t i = a.horizontal ? ix : iy;  // index along the folded axis
        // rows of g_out this input row gathers (H pass: one row, or the
        // virtual rows that the source read clamps onto an edge row)
        int32_t r0 = iy, r1 = iy;
        if (a.horizontal && a.fold_rows) {
            r0 = iy - a.mid_y0;
            r1 = r0;
            if (iy == 0) r0 = 0;
            if (iy == a.in_h - 1) r1 = a.out_h - 1;
            r0 = r0 < 0 ? 0 : r0;
            r1 = r1 >= a.out_h ? a.out_h - 1 : r1;
        }
        const int32_t olo = a.lo[i], n = a.hi[i] - olo + 1;
        const float* w = a.wt + (size_t)i * a.wstride;
        float* dst = a.g_in + (size_t)iy * rowlen + (size_t)ix * B;
        if constexpr (NB > 0) {
            float acc[NBm];
#pragma unroll
            for (int b = 0; b < NBm; ++b) acc[b] = 0.0f;
            // tap j of this pixel: g + j * step (H: the next output pixel of
            // the row; V: the next output row, same column)
            const size_t step = a.horizontal ? (size_t)NB : (size_t)gstride;
            for (int32_t r = (a.horizontal ? r0 : 0); r <= (a.horizontal ? r1 : 0); ++r) {
                const float* g = a.horizontal ? a.g_out + (size_t)r * gstride + (size_t)olo * NB
                                              : a.g_out + (size_t)olo * gstride + (size_t)ix * NB;
#pragma unroll 4
                for (int32_t j = 0; j < n; ++j) {
                    const float wj = w[j];
                    const float* q = g + (size_t)j * step;
                    if constexpr (NB == 4) {
                        const float4 v = *reinterpret_cast<const float4*>(q);
                        acc[0] = fmaf(v.x, wj, acc[0]);
                        acc[1] = fmaf(v.y, wj, acc[1]);
                        acc[2] = fmaf(v.z, wj, acc[2]);
                        acc[3] = fmaf(v.w, wj, acc[3]);
                    } else {
#pragma unroll
                        for (int b = 0; b < NBm; ++b) acc[b] = fmaf(q[b], wj, acc[b]);
                    }
                }
            }
            if constexpr (NB == 4) {
                *reinterpret_cast<float4*>(dst) = make_float4(acc[0], acc[1], acc[2], acc[3]);
            } else {
#pragma unroll
                for (int b = 0; b < NBm; ++b) dst[b] = acc[b];
            }
        } else {
            for (int b = 0; b < B; ++b) {
                float acc = 0.0f;
                if (a.horizontal) {
                    for (int32_t r = r0; r <= r1; ++r) {
                        const float* g = a.g_out + (size_t)r * gstride + (size_t)olo * B + b;
                        for (int32_t j = 0; j < n; ++j) acc = fmaf(g[j * B], w[j], acc);
                    }
                } else {
                    const float* g = a.g_out + (size_t)olo * gstride + (size_t)ix * B + b;
                    for (int32_t j = 0; j < n; ++j) acc = fmaf(g[(size_t)j * gstride], w[j], acc);
                }
                dst[b] = acc;
            }
        }
    }
}

// Image-gradient scatter; both targets null = the image gradient was not requested.
__device__ __forceinline__ void scatter(float* g, unsigned long long* fx, double scale, int64_t idx, double v) {
    if (fx) atomicAdd(fx + idx, (unsigned long long)(long long)llrint(v * scale));
    else if (g) atomicAdd(g + idx, (float)v);
}

// f32 contribution to the image gradient (fixed_scale is a power of two: the
// scaled value is exact).
__device__ __forceinline__ void scatter_f(float* g, unsigned long long* fx, double scale, int64_t idx, float v) {
    if (fx) atomicAdd(fx + idx, (unsigned long long)llrintf(v * (float)scale));
    else if (g) atomicAdd(g + idx, v);
}

// Bilinear forward of one band with derivative, from four samples.
template <typename R>
struct Bil {
    R out, dfx, dfy;
};
template <typename R>
__device__ __forceinline__ Bil<R> bil(R p00, R p01, R p10, R p11, R fx, R fy) {
    Bil<R> r;
    const R one = R(1);
    const R top = fma(p01, fx, p00 * (one - fx)), bottom = fma(p11, fx, p10 * (one - fx));
    r.out = top * (one - fy) + bottom * fy;
    r.dfx = (one - fy) * (p01 - p00) + fy * (p11 - p10);
    r.dfy = bottom - top;
    return r;
}

// Gradient contributions of one output pixel at position (x_in, y_in); NB
// bands (NB == 0: a.bands, up to 8, read at run time).  The position and the
// matrix-gradient sums are f64; the per-pixel interpolation derivative is
// f32 arithmetic (the samples and gradients are f32), as a backward pass
// computes.
template <int NB>
__device__ __forceinline__ void affine_grad_px(const AffineGradArgs& g, const AffineCtx<float>& c, double x_in,
                                               double y_in, int64_t X, int64_t Y, const float* gy, double* part) {
    const AffineArgs& a = g.fwd;
    constexpr int NBmax = NB > 0 ? NB : 8;
    const int bands = NB > 0 ? NB : a.bands;
    if (!isfinite(x_in) || !isfinite(y_in)) return;
    const int64_t x0 = trunc_i64(x_in), y0 = trunc_i64(y_in);
    const float fx = (float)(x_in - (double)x0), fy = (float)(y_in - (double)y0);
    const float w[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
    // element offset of each tap's first band in the input plane (-1: the
    // constant fill); every tap loads from a readable address
    const float* src = reinterpret_cast<const float*>(a.in.data);
    int64_t e[4];
    float sv[4][NBmax];
    const float fill = (float)c.fill();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        bool ok;
        const float* px = c.tap(x0 + (k & 1), y0 + (k >> 1), &ok);
        e[k] = ok ? (int64_t)(px - src) : -1;
#pragma unroll
        for (int b = 0; b < NBmax; ++b) {
            if (b >= bands) break;
            const float v = px[b];
            sv[k][b] = ok ? v : fill;
        }
    }
    float dx = 0.0f, dy = 0.0f;
    if (bands == 4 && !a.premultiplied) {
        // alpha-premultiplied sampler (affine/core.rs:988-1019), alpha_max = 1
        float al[4], pm[3][4];
#pragma unroll
        for (int k = 0; k < 4; ++k) al[k] = sv[k][3];
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int k = 0; k < 4; ++k) pm[b][k] = sv[k][b] * al[k];
        const Bil<float> A = bil<float>(al[0], al[1], al[2], al[3], fx, fy);
        Bil<float> P[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) P[b] = bil<float>(pm[b][0], pm[b][1], pm[b][2], pm[b][3], fx, fy);
        float dP[3] = {0, 0, 0}, dA = 0.0f;
        if (A.out > 0.0f && A.out < 1.0f) {
            const float inv = 1.0f / A.out;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                dP[b] = gy[b] * inv;
                dA -= gy[b] * P[b].out * inv * inv;
            }
            dA += gy[3];
        } else if (A.out >= 1.0f) {
#pragma unroll
            for (int b = 0; b < 3; ++b) dP[b] = gy[b];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (e[k] < 0) continue;
            float da = dA * w[k];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                scatter_f(g.g_in, g.g_fixed, g.fixed_scale, e[k] + b, dP[b] * w[k] * al[k]);
                da += dP[b] * w[k] * sv[k][b];
            }
            scatter_f(g.g_in, g.g_fixed, g.fixed_scale, e[k] + 3, da);
        }
#pragma unroll
        for (int b = 0; b < 3; ++b) { dx += dP[b] * P[b].dfx; dy += dP[b] * P[b].dfy; }
        dx += dA * A.dfx;
        dy += dA * A.dfy;
    } else {
#pragma unroll
        for (int b = 0; b < NBmax; ++b) {
            if (b >= bands) break;
            const float gb = gy[b];
            const Bil<float> v = bil<float>(sv[0][b], sv[1][b], sv[2][b], sv[3][b], fx, fy);
            dx += gb * v.dfx;
            dy += gb * v.dfy;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (e[k] >= 0) scatter_f(g.g_in, g.g_fixed, g.fixed_scale, e[k] + b, gb * w[k]);
        }
    }
    // x_in = m0 X + m1 Y + tx, y_in = m2 X + m3 Y + ty
    part[0] += (double)dx * (double)X; part[1] += (double)dx * (double)Y;
    part[2] += (double)dy * (double)X; part[3] += (double)dy * (double)Y;
    part[4] += (double)dx; part[5] += (double)dy;
}

// Threads over groups of a.group consecutive output pixels of a row, block
// rows over the output rows (grid-stride); positions as the forward kernel
// computes them (AffineRow's walk, the axis-aligned fast path or the per-axis
// tables).  Each thread sums its pixels' matrix-gradient terms in a fixed
// order, each block its threads' in a fixed tree.
template <int NB>
__global__ void __launch_bounds__(256, 2) affine_grad_kernel(AffineGradArgs g) {
    const AffineArgs& a = g.fwd;
    const int G = a.group;
    const int64_t lx0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * G;
    double part[6] = {0, 0, 0, 0, 0, 0};
    if (lx0 < a.out.w) {
        const int64_t lx1 = min((int64_t)a.out.w, lx0 + G);
        const double* m = a.m;
        for (int64_t ly = blockIdx.y; ly < a.out.h; ly += gridDim.y) {
            const int64_t Y = a.out.y0 + ly;
            AffineCtx<float> c(a);
            AffineRow row;
            for (int64_t lx = lx0; lx < lx1; ++lx) {
                const int64_t X = a.out.x0 + lx;
                row.tile<float>(a, c, X, Y);
                double x_in, y_in;
                if (a.fast == 2 && X >= 0 && X < (int64_t)a.total_w && Y >= 0 && Y < (int64_t)a.total_h) {
                    x_in = fma(m[0], (double)X, a.tx);
                    y_in = fma(m[3], (double)Y, a.ty);
                } else if (a.separable && a.xs != nullptr) {
                    x_in = a.xs[X];
                    y_in = a.ys[Y];
                } else {
                    row.walk(a, X, Y);
                    x_in = row.x;
                    y_in = row.y;
                }
                const float* gy = g.g_out + (ly * a.out.w + lx) * a.bands;
                affine_grad_px<NB>(g, c, x_in, y_in, X, Y, gy, part);
            }
        }
    }
    if (g.partial) {
        __shared__ double red[6][8];
        for (int q = 0; q < 6; ++q) {
            double v = part[q];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            double s = 0.0;
            for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) s += red[threadIdx.x][w8];
            g.partial[((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = s;
        }
    }
}

// d/dx of the kernel weight k(|i - x|) for the separable samplers.
__device__ __forceinline__ double kernel_dw(int k, double i_minus_x) {
    const double t = fabs(i_minus_x);
    const double s = i_minus_x > 0.0 ? -1.0 : (i_minus_x < 0.0 ? 1.0 : 0.0);  // d|i-x|/dx
    double dk = 0.0;
    if (k == 2 || k == 7) {
        if (t < 1.0) dk = 4.5 * t * t - 5.0 * t;
        else if (t < 2.0) dk = -1.5 * t * t + 5.0 * t - 4.0;
    } else if (k == 3) {
        if (t < 0.5) dk = -4.0 * t;
        else if (t < 1.5) dk = 2.0 * t - 2.5;
    } else if (k == 1) {
        if (t < 1.0) dk = -1.0;
    } else if (k == 8 || k == 9) {
        const double L = k == 9 ? 3.0 : 2.0;
        if (t > 0.0 && t < L) {
            const double pi = 3.141592653589793, p = pi * t;
            // d/dt [L sin(pi t) sin(pi t / L) / (pi t)^2]
            const double f = L * sin(p) * sin(p / L), df = L * pi * (cos(p) * sin(p / L) + sin(p) * cos(p / L) / L);
            dk = (df * p * p - f * 2.0 * pi * p) / (p * p * p * p);
        }
    }
    return dk * s;
}

// f32 forms of the separable kernels and their derivatives (the mapim
// gradient evaluates its weights in f32; sinpif / cospif give sin(pi t)).
__device__ __forceinline__ float kernel_wf(int k, float x) {
    x = fabsf(x);
    switch (k) {
    case 0: return x < 0.5f ? 1.0f : 0.0f;
    case 1: return x < 1.0f ? 1.0f - x : 0.0f;
    case 2: case 5: case 7:
        if (x < 1.0f) return fmaf(2.5f * x, -x, 1.5f * x * x * x) + 1.0f;
        if (x < 2.0f) return fmaf(4.0f, -x, fmaf(2.5f * x, x, -0.5f * x * x * x)) + 2.0f;
        return 0.0f;
    case 3:
        if (x < 0.5f) return fmaf(2.0f * x, -x, 1.0f);
        if (x < 1.5f) return fmaf(2.5f, -x, x * x) + 1.5f;
        return 0.0f;
    case 8: case 9: {
        const float L = k == 9 ? 3.0f : 2.0f;
        if (x < 1e-6f) return 1.0f;
        if (x < L) return L * sinpif(x) * sinpif(x / L) / (9.8696044f * x * x);
        return 0.0f;
    }
    default: return 0.0f;
    }
}

__device__ __forceinline__ float kernel_dwf(int k, float i_minus_x) {
    const float t = fabsf(i_minus_x);
    const float s = i_minus_x > 0.0f ? -1.0f : (i_minus_x < 0.0f ? 1.0f : 0.0f);  // d|i-x|/dx
    float dk = 0.0f;
    if (k == 2 || k == 5 || k == 7) {
        if (t < 1.0f) dk = 4.5f * t * t - 5.0f * t;
        else if (t < 2.0f) dk = -1.5f * t * t + 5.0f * t - 4.0f;
    } else if (k == 3) {
        if (t < 0.5f) dk = -4.0f * t;
        else if (t < 1.5f) dk = 2.0f * t - 2.5f;
    } else if (k == 1) {
        if (t < 1.0f) dk = -1.0f;
    } else if (k == 8 || k == 9) {
        const float L = k == 9 ? 3.0f : 2.0f;
        if (t > 0.0f && t < L) {
            const float pi = 3.14159265f, p = pi * t;
            const float sa = sinpif(t), sb = sinpif(t / L);
            const float f = L * sa * sb, df = L * pi * (cospif(t) * sb + sa * cospif(t / L) / L);
            dk = df / (p * p) - f * 2.0f * pi / (p * p * p);
        }
    }
    return dk * s;
}

// Image-gradient sink of one block of mapim_grad: while the block's scatter
// footprint (the bounding box of every tap it writes) fits in shared memory,
// contributions add there (shared atomics) and the block flushes the box to
// the global gradient once; otherwise they go to global atomics directly.
// Fixed-point sums stay integer all the way, so the deterministic mode keeps
// its order independence.
constexpr int kMapimTile = 16;           // 16 x 16 output pixels per block
constexpr int kMapimSmemElems = 4096;    // footprint capacity (elements x bands)

struct MapimSink {
    float* sf = nullptr;
    unsigned long long* su = nullptr;
    int32_t bx0 = 0, by0 = 0, bw = 0;
    bool local = false;
    const MapimGradArgs* g = nullptr;
    int64_t pitch_f = 0;
    int bands = 1;
    // element (rx, ry, b): local index li when the block accumulates
    // locally, global index gi otherwise
    __device__ __forceinline__ void add_at(int32_t li, int64_t gi, double v) const {
        if (local) {
            if (g->g_fixed) atomicAdd(su + li, (unsigned long long)(long long)llrint(v * g->fixed_scale));
            else atomicAdd(sf + li, (float)v);
        } else {
            scatter(g->g_src, g->g_fixed, g->fixed_scale, gi, v);
        }
    }
    // f32 contribution (fixed_scale is a power of two: the scaled value is exact)
    __device__ __forceinline__ void add_at(int32_t li, int64_t gi, float v) const {
        if (g->g_fixed) {
            const unsigned long long q = (unsigned long long)llrintf(v * (float)g->fixed_scale);
            if (local) atomicAdd(su + li, q);
            else atomicAdd(g->g_fixed + gi, q);
        } else {
            atomicAdd(local ? sf + li : g->g_src + gi, v);
        }
    }
    __device__ __forceinline__ void add(int64_t rx, int64_t ry, int b, double v) const {
        add_at(((int32_t)(ry - by0) * bw + (int32_t)(rx - bx0)) * bands + b, ry * pitch_f + rx * bands + b, v);
    }
};

// NT: taps per axis of the separable samplers (4: support 2, 6: Lanczos3);
// 0 for the nearest / bilinear kernels.
template <int NT>
__global__ void __launch_bounds__(256, 3) mapim_grad_kernel(MapimGradArgs g) {
    extern __shared__ __align__(16) unsigned char mg_smem[];
    __shared__ int32_t box[4];  // min x, max x, min y, max y of the block's taps
    const MapimArgs& a = g.fwd;
    const int64_t lx = (int64_t)blockIdx.x * kMapimTile + (threadIdx.x % kMapimTile);
    const int64_t ly = (int64_t)blockIdx.y * kMapimTile + (threadIdx.x / kMapimTile);
    const bool live = lx < a.out.w && ly < a.out.h;
    const int bands = a.bands;
    const int64_t p = ly * a.out.w + lx;
    double x = NAN, y = NAN;
    if (live) {
        const float2 idx = *reinterpret_cast<const float2*>(a.index.data + ly * a.index.pitch + lx * 8);
        x = (double)idx.x;
        y = (double)idx.y;
    }
    const bool valid = live && isfinite(x) && isfinite(y);
    const int k = a.kernel;
    const bool want_img = g.g_src != nullptr || g.g_fixed != nullptr;
    // tap bounding box of this pixel, clipped / clamped as the scatter resolves it
    int64_t tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
    const int64_t W = a.src_w, H = a.src_h;
    if (valid && want_img) {
        if (NT == 0) {
            const int64_t x0 = trunc_i64(floor(x)), y0 = trunc_i64(floor(y)), d = k;
            tx0 = x0; tx1 = x0 + d; ty0 = y0; ty1 = y0 + d;
            if (a.extend_copy) {
                tx0 = clampi64(tx0, 0, W - 1); tx1 = clampi64(tx1, 0, W - 1);
                ty0 = clampi64(ty0, 0, H - 1); ty1 = clampi64(ty1, 0, H - 1);
            } else {
                tx0 = max(tx0, (int64_t)0); tx1 = min(tx1, W - 1);
                ty0 = max(ty0, (int64_t)0); ty1 = min(ty1, H - 1);
            }
        } else {
            constexpr int64_t support = NT / 2;
            const int64_t cx = trunc_i64(floor(x)), cy = trunc_i64(floor(y));
            tx0 = max(cx - (support - 1), (int64_t)0); tx1 = min(cx + support, W - 1);
            ty0 = max(cy - (support - 1), (int64_t)0); ty1 = min(cy + support, H - 1);
        }
    }
    if (threadIdx.x == 0) { box[0] = INT32_MAX; box[1] = INT32_MIN; box[2] = INT32_MAX; box[3] = INT32_MIN; }
    __syncthreads();
    if (tx0 <= tx1 && ty0 <= ty1) {
        atomicMin(&box[0], (int32_t)tx0); atomicMax(&box[1], (int32_t)tx1);
        atomicMin(&box[2], (int32_t)ty0); atomicMax(&box[3], (int32_t)ty1);
    }
    __syncthreads();
    MapimSink sink;
    sink.g = &g;
    sink.bands = bands;
    sink.pitch_f = a.src.pitch / 4;
    const int64_t bw = (int64_t)box[1] - box[0] + 1, bh = (int64_t)box[3] - box[2] + 1;
    const int64_t n_local = (box[1] >= box[0] && box[3] >= box[2]) ? bw * bh * bands : 0;
    sink.local = n_local > 0 && n_local <= kMapimSmemElems;  // uniform across the block
    if (sink.local) {
        sink.bx0 = box[0]; sink.by0 = box[2]; sink.bw = (int32_t)bw;
        if (g.g_fixed) {
            sink.su = reinterpret_cast<unsigned long long*>(mg_smem);
            for (int i = threadIdx.x; i < (int)n_local; i += blockDim.x) sink.su[i] = 0ull;
        } else {
            sink.sf = reinterpret_cast<float*>(mg_smem);
            for (int i = threadIdx.x; i < (int)n_local; i += blockDim.x) sink.sf[i] = 0.0f;
        }
        __syncthreads();
    }
    const float* gy = g.g_out + p * bands;
    const float* src = reinterpret_cast<const float*>(a.src.data);
    const int64_t pitch_f = a.src.pitch / 4;
    double gx = 0.0, gyy = 0.0;
    if (valid) {
        auto inb = [&](int64_t ix, int64_t iy) { return ix >= 0 && ix < W && iy >= 0 && iy < H; };
        if (NT == 0 && k == 0) {
            const int64_t ix = trunc_i64(floor(x)), iy = trunc_i64(floor(y));
            int64_t rx = ix, ry = iy;
            bool ok = inb(ix, iy);
            if (!ok && a.extend_copy) {
                ok = !(ix < -1 || ix > W || iy < -1 || iy > H);
                rx = clampi64(ix, 0, W - 1);
                ry = clampi64(iy, 0, H - 1);
            }
            if (ok && want_img)
                for (int b = 0; b < bands; ++b) sink.add(rx, ry, b, gy[b]);
        } else if (NT == 0 && k == 1) {
            const int64_t x0 = trunc_i64(floor(x)), y0 = trunc_i64(floor(y));
            const double fx = x - (double)x0, fy = y - (double)y0;
            const double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
            int64_t rxq[4], ryq[4];
            bool okq[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                int64_t rx = x0 + (q & 1), ry = y0 + (q >> 1);
                bool ok = inb(rx, ry);
                if (!ok && a.extend_copy) {
                    ok = !(rx < -1 || rx > W + 1 || ry < -1 || ry > H + 1);
                    rx = clampi64(rx, 0, W - 1);
                    ry = clampi64(ry, 0, H - 1);
                }
                rxq[q] = rx; ryq[q] = ry; okq[q] = ok;
            }
            for (int b = 0; b < bands; ++b) {
                double sq[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    // every tap loads (a clamped, readable address); the background replaces it after
                    const double raw = (double)src[clampi64(ryq[q], 0, H - 1) * pitch_f + clampi64(rxq[q], 0, W - 1) * bands + b];
                    sq[q] = okq[q] ? raw : a.background;
                    if (okq[q] && want_img) sink.add(rxq[q], ryq[q], b, (double)gy[b] * w[q]);
                }
                const Bil<double> v = bil<double>(sq[0], sq[1], sq[2], sq[3], fx, fy);
                gx += (double)gy[b] * v.dfx;
                gyy += (double)gy[b] * v.dfy;
            }
        } else if (NT > 0) {
            // separable sampler y = N / W with N = sum_ij wx_i wy_j s_ij and
            // W = (sum_i wx_i)(sum_j wy_j), evaluated in f32; taps whose weight
            // and derivative are both zero are skipped, as the forward skips
            // zero weights
            constexpr int64_t support = NT / 2;
            constexpr int nt = NT > 0 ? NT : 1;
            const float xf = (float)x, yf = (float)y;  // the f32 coordinates themselves
            const int64_t cx = (int64_t)floorf(xf), cy = (int64_t)floorf(yf);
            const int64_t tx0 = cx - (support - 1), ty0 = cy - (support - 1);
            float wx[nt], dwx[nt], wy[nt], dwy[nt];
            bool okx[nt];
            int32_t col[nt], lcol[nt];
            float Sx = 0.0f, Sdx = 0.0f, Sy = 0.0f, Sdy = 0.0f;
#pragma unroll
            for (int t = 0; t < nt; ++t) {
                const int64_t ix = tx0 + t, iy = ty0 + t;
                const float ex = (float)ix - xf, ey = (float)iy - yf;
                wx[t] = kernel_wf(k, ex);
                dwx[t] = kernel_dwf(k, ex);
                wy[t] = kernel_wf(k, ey);
                dwy[t] = kernel_dwf(k, ey);
                Sx += wx[t]; Sdx += dwx[t]; Sy += wy[t]; Sdy += dwy[t];
                okx[t] = ix >= 0 && ix < W;
                col[t] = (int32_t)clampi64(ix, 0, W - 1) * bands;
                lcol[t] = (int32_t)(ix - sink.bx0) * bands;
            }
            const float Wt = Sx * Sy, Wx = Sdx * Sy, Wy = Sx * Sdy;
            if (Wt > 0.0f) {
                const float inv = 1.0f / Wt;
                const float bg = (float)a.background;
                for (int b = 0; b < bands; ++b) {
                    float Nv = 0.0f, Nx = 0.0f, Ny = 0.0f;
                    const float gb = gy[b];
#pragma unroll 1
                    for (int ty = 0; ty < nt; ++ty) {
                        if (wy[ty] == 0.0f && dwy[ty] == 0.0f) continue;
                        const int64_t iy = ty0 + ty;
                        const bool oky = iy >= 0 && iy < H;
                        const int64_t grow = clampi64(iy, 0, H - 1) * pitch_f + b;
                        // the row's taps load unconditionally (clamped addresses)
                        float sv[nt];
#pragma unroll
                        for (int tx = 0; tx < nt; ++tx) sv[tx] = src[grow + col[tx]];
                        float rv = 0.0f, rd = 0.0f;
#pragma unroll
                        for (int tx = 0; tx < nt; ++tx) {
                            if (wx[tx] == 0.0f && dwx[tx] == 0.0f) continue;
                            const float sval = okx[tx] && oky ? sv[tx] : bg;
                            rv = fmaf(wx[tx], sval, rv);
                            rd = fmaf(dwx[tx], sval, rd);
                        }
                        Nv = fmaf(wy[ty], rv, Nv);
                        Nx = fmaf(wy[ty], rd, Nx);
                        Ny = fmaf(dwy[ty], rv, Ny);
                        if (want_img && oky && wy[ty] != 0.0f) {
                            const float c = gb * inv * wy[ty];
                            const int32_t lrow = (int32_t)(iy - sink.by0) * sink.bw * bands + b;
#pragma unroll
                            for (int tx = 0; tx < nt; ++tx)
                                if (okx[tx] && wx[tx] != 0.0f) sink.add_at(lrow + lcol[tx], grow + col[tx], c * wx[tx]);
                        }
                    }
                    gx += (double)(gb * (Nx * Wt - Nv * Wx) * inv * inv);
                    gyy += (double)(gb * (Ny * Wt - Nv * Wy) * inv * inv);
                }
            }
        }
    }
    if (g.g_index && live) {
        g.g_index[p * 2] = (float)gx;
        g.g_index[p * 2 + 1] = (float)gyy;
    }
    if (sink.local) {
        __syncthreads();
        const int32_t rowe = sink.bw * bands;
        for (int i = threadIdx.x; i < (int)n_local; i += blockDim.x) {
            const int r = i / rowe, c = i - r * rowe;
            const int64_t gi = (int64_t)(sink.by0 + r) * pitch_f + (int64_t)sink.bx0 * bands + c;
            if (g.g_fixed) {
                const unsigned long long v = sink.su[i];
                if (v) atomicAdd(g.g_fixed + gi, v);
            } else {
                const float v = sink.sf[i];
                if (v != 0.0f) atomicAdd(g.g_src + gi, v);
            }
        }
    }
}

__global__ void fixed_to_f32_kernel(const unsigned long long* acc, float* out, int64_t n, double inv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)((double)(long long)acc[i] * inv);
}

__global__ void __launch_bounds__(192) sum_partials_kernel(const double* partial, int blocks, double* out) {
    // warp w sums component w: lane l takes blocks l, l + 32, ... and the lanes
    // combine in a fixed butterfly, so the result is the same on every run
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    double s = 0.0;
    for (int b = l; b < blocks; b += 32) s += partial[(int64_t)b * 6 + w];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (l == 0) out[w] = s;
}

}  // namespace dev

namespace launch {

cudaError_t reduce_adjoint(const ReduceAdjArgs& a, cudaStream_t s) {
    const int64_t rowlen = (int64_t)a.in_w * a.bands;
    if (rowlen <= 0 || a.in_h <= 0) return cudaSuccess;
    if (rowlen * a.in_h >= ((int64_t)1 << 31) || (int64_t)a.out_w * a.bands * a.out_h >= ((int64_t)1 << 31))
        return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((a.in_w + 255) / 256), (unsigned)std::min<int64_t>(a.in_h, 65535));
    // 16-byte loads of 4-band pixels need 16-byte aligned planes
    const bool al16 = (reinterpret_cast<uintptr_t>(a.g_out) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.g_in) & 15) == 0;
    switch (a.bands) {
    case 1: dev::reduce_adjoint_kernel<1><<<grid, 256, 0, s>>>(a); break;
    case 3: dev::reduce_adjoint_kernel<3><<<grid, 256, 0, s>>>(a); break;
    case 4:
        if (al16) dev::reduce_adjoint_kernel<4><<<grid, 256, 0, s>>>(a);
        else dev::reduce_adjoint_kernel<0><<<grid, 256, 0, s>>>(a);
        break;
    default: dev::reduce_adjoint_kernel<0><<<grid, 256, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

static dim3 affine_grad_grid(int32_t out_w, int32_t out_h, int group) {
    const int64_t gx = ((int64_t)out_w + group - 1) / group;
    return dim3((unsigned)((gx + 255) / 256), (unsigned)std::min<int32_t>(out_h, 65535));
}

int affine_grad_blocks(int32_t out_w, int32_t out_h) {
    const dim3 g = affine_grad_grid(out_w, out_h, affine_group((int64_t)out_w * out_h));
    return (int)(g.x * g.y);
}

cudaError_t affine_grad(const AffineGradArgs& a, int blocks, cudaStream_t s) {
    if (blocks <= 0) return cudaSuccess;
    if (a.fwd.bands > 8) return cudaErrorInvalidValue;
    AffineGradArgs k = a;
    k.fwd.group = affine_group((int64_t)a.fwd.out.w * a.fwd.out.h);
    const dim3 grid = affine_grad_grid(a.fwd.out.w, a.fwd.out.h, k.fwd.group);
    if ((int)(grid.x * grid.y) != blocks) return cudaErrorInvalidValue;
    switch (a.fwd.bands) {
    case 1: dev::affine_grad_kernel<1><<<grid, 256, 0, s>>>(k); break;
    case 3: dev::affine_grad_kernel<3><<<grid, 256, 0, s>>>(k); break;
    case 4: dev::affine_grad_kernel<4><<<grid, 256, 0, s>>>(k); break;
    default: dev::affine_grad_kernel<0><<<grid, 256, 0, s>>>(k); break;
    }
    return cudaGetLastError();
}

cudaError_t mapim_grad(const MapimGradArgs& a, cudaStream_t s) {
    const int64_t npx = (int64_t)a.fwd.out.w * a.fwd.out.h;
    if (npx <= 0) return cudaSuccess;
    const int64_t gx = ((int64_t)a.fwd.out.w + dev::kMapimTile - 1) / dev::kMapimTile;
    const int64_t gy = ((int64_t)a.fwd.out.h + dev::kMapimTile - 1) / dev::kMapimTile;
    if (gy > 65535 || (int64_t)a.fwd.src_w * a.fwd.bands >= ((int64_t)1 << 31) || a.fwd.src_h >= (1u << 31))
        return cudaErrorInvalidValue;
    const size_t smem = (size_t)dev::kMapimSmemElems * (a.g_fixed ? 8 : 4);
    const dim3 grid((unsigned)gx, (unsigned)gy);
    const int k = a.fwd.kernel;
    if (k == 0 || k == 1) dev::mapim_grad_kernel<0><<<grid, dev::kMapimTile * dev::kMapimTile, smem, s>>>(a);
    else if (k == 9) dev::mapim_grad_kernel<6><<<grid, dev::kMapimTile * dev::kMapimTile, smem, s>>>(a);
    else dev::mapim_grad_kernel<4><<<grid, dev::kMapimTile * dev::kMapimTile, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fixed_to_f32(const unsigned long long* acc, float* out, int64_t n, double inv_scale, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    dev::fixed_to_f32_kernel<<<grid, 256, 0, s>>>(acc, out, n, inv_scale);
    return cudaGetLastError();
}

cudaError_t sum_partials(const double* partial, int blocks, double* out, cudaStream_t s) {
    dev::sum_partials_kernel<<<1, 192, 0, s>>>(partial, blocks, out);
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
