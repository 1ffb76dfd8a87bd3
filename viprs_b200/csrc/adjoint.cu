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
#include "adjoint_launch.hpp"
#include "affine_dev.cuh"

namespace viprs {
namespace dev {

__global__ void __launch_bounds__(256) reduce_adjoint_kernel(ReduceAdjArgs a) {
    const int64_t n = (int64_t)a.in_w * a.in_h * a.bands;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int b = int(idx % a.bands);
    const int64_t px = idx / a.bands;
    const int32_t ix = int32_t(px % a.in_w), iy = int32_t(px / a.in_w);
    // the axis this pass folds, and the index along it
    const int32_t i = a.horizontal ? ix : iy;
    const int32_t n_axis = a.horizontal ? a.in_w : a.in_h;
    double acc = 0.0;
    // rows of g_out this input row gathers from (H pass: one row, or the
    // virtual rows that the source read clamps onto an edge row)
    int32_t r0 = iy, r1 = iy;
    if (a.horizontal && a.fold_rows) {
        const int32_t mrows = a.out_h;
        r0 = iy - a.mid_y0;
        r1 = r0;
        if (iy == 0) r0 = 0;
        if (iy == a.in_h - 1) r1 = mrows - 1;
        r0 = r0 < 0 ? 0 : r0;
        r1 = r1 >= mrows ? mrows - 1 : r1;
    }
    const int32_t olo = a.lo[i], ohi = a.hi[i];
    for (int32_t r = r0; r <= r1; ++r) {
        for (int32_t o = olo; o <= ohi; ++o) {
            double w;
            if (n_axis == 1) w = a.fold_lo[o] + 0.0;
            else if (i == 0) w = a.fold_lo[o];
            else if (i == n_axis - 1) w = a.fold_hi[o];
            else w = a.coeffs[a.phases[o] * a.taps + (i - a.starts[o])];
            const int64_t g = a.horizontal ? ((int64_t)r * a.out_w + o) * a.bands + b
                                           : ((int64_t)o * a.out_w + ix) * a.bands + b;
            acc = fma((double)a.g_out[g], w, acc);
        }
    }
    a.g_in[idx] = (float)acc;
}

// Image-gradient scatter; both targets null = the image gradient was not requested.
__device__ __forceinline__ void scatter(float* g, unsigned long long* fx, double scale, int64_t idx, double v) {
    if (fx) atomicAdd(fx + idx, (unsigned long long)(long long)llrint(v * scale));
    else if (g) atomicAdd(g + idx, (float)v);
}

// Bilinear forward of one band with derivative, from four samples.
struct Bil {
    double out, dfx, dfy;
};
__device__ __forceinline__ Bil bil(double p00, double p01, double p10, double p11, double fx, double fy) {
    Bil r;
    const double top = fma(p01, fx, p00 * (1.0 - fx)), bottom = fma(p11, fx, p10 * (1.0 - fx));
    r.out = top * (1.0 - fy) + bottom * fy;
    r.dfx = (1.0 - fy) * (p01 - p00) + fy * (p11 - p10);
    r.dfy = bottom - top;
    return r;
}

__global__ void __launch_bounds__(256) affine_grad_kernel(AffineGradArgs g) {
    const AffineArgs& a = g.fwd;
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double part[6] = {0, 0, 0, 0, 0, 0};
    if (p < npx) {
        const int64_t ly = p / a.out.w, lx = p - ly * a.out.w;
        const int64_t X = a.out.x0 + lx, Y = a.out.y0 + ly;
        AffineCtx<float> c(a);
        c.set_tile(X, Y);
        const double* m = a.m;
        double x_in, y_in;
        if (a.fast == 2 && X >= 0 && X < (int64_t)a.total_w && Y >= 0 && Y < (int64_t)a.total_h) {
            x_in = fma(m[0], (double)X, a.tx);
            y_in = fma(m[3], (double)Y, a.ty);
        } else if (a.separable && a.xs != nullptr) {
            x_in = a.xs[X];
            y_in = a.ys[Y];
        } else {
            const int64_t X0 = tile_origin(X, a.tile_off_x, a.tile_w), Y0 = tile_origin(Y, a.tile_off_y, a.tile_h);
            double rx = fma(m[1], (double)Y0, m[0] * (double)X0) + a.tx;
            double ry = fma(m[3], (double)Y0, m[2] * (double)X0) + a.ty;
            for (int64_t r = Y0; r < Y; ++r) { rx += m[1]; ry += m[3]; }
            x_in = rx; y_in = ry;
            for (int64_t q = X0; q < X; ++q) { x_in += m[0]; y_in += m[2]; }
        }
        const int bands = a.bands;
        const float* gy = g.g_out + p * bands;
        if (isfinite(x_in) && isfinite(y_in)) {
            const int64_t x0 = trunc_i64(x_in), y0 = trunc_i64(y_in);
            const double fx = x_in - (double)x0, fy = y_in - (double)y0;
            const double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
            const int64_t tx_[4] = {x0, x0 + 1, x0, x0 + 1}, ty_[4] = {y0, y0, y0 + 1, y0 + 1};
            // resolved in-plane sample index of each tap (-1: the constant fill)
            int64_t lin[4];
            for (int k = 0; k < 4; ++k) {
                int64_t rx, ry;
                const bool ok = c.resolve(tx_[k], a.src_w, &rx) && c.resolve(ty_[k], a.src_h, &ry) && rx >= c.rx0 &&
                                rx <= c.rx1 && ry >= c.ry0 && ry <= c.ry1;
                lin[k] = ok ? ((ry - a.in.y0) * (int64_t)a.in.w + (rx - a.in.x0)) : -1;
            }
            const float* src = reinterpret_cast<const float*>(a.in.data);
            const int64_t pitch_f = a.in.pitch / 4;
            auto sample = [&](int k, int band) -> double {
                if (lin[k] < 0) return c.fill();
                const int64_t ry = lin[k] / a.in.w, rx = lin[k] - ry * a.in.w;
                return (double)src[ry * pitch_f + rx * bands + band];
            };
            auto gidx = [&](int k, int band) -> int64_t {
                const int64_t ry = lin[k] / a.in.w, rx = lin[k] - ry * a.in.w;
                return ry * pitch_f + rx * bands + band;
            };
            double dx = 0.0, dy = 0.0;
            if (bands == 4 && !a.premultiplied) {
                // alpha-premultiplied sampler (affine/core.rs:988-1019), alpha_max = 1
                double al[4], pm[3][4];
                for (int k = 0; k < 4; ++k) al[k] = sample(k, 3);
                for (int b = 0; b < 3; ++b)
                    for (int k = 0; k < 4; ++k) pm[b][k] = sample(k, b) * al[k];
                const Bil A = bil(al[0], al[1], al[2], al[3], fx, fy);
                Bil P[3];
                for (int b = 0; b < 3; ++b) P[b] = bil(pm[b][0], pm[b][1], pm[b][2], pm[b][3], fx, fy);
                double dP[3] = {0, 0, 0}, dA = 0.0;
                if (A.out > 0.0 && A.out < 1.0) {
                    for (int b = 0; b < 3; ++b) {
                        dP[b] = (double)gy[b] / A.out;
                        dA -= (double)gy[b] * P[b].out / (A.out * A.out);
                    }
                    dA += (double)gy[3];
                } else if (A.out >= 1.0) {
                    for (int b = 0; b < 3; ++b) dP[b] = (double)gy[b];
                }
                for (int k = 0; k < 4; ++k) {
                    if (lin[k] < 0) continue;
                    double da = dA * w[k];
                    for (int b = 0; b < 3; ++b) {
                        scatter(g.g_in, g.g_fixed, g.fixed_scale, gidx(k, b), dP[b] * w[k] * al[k]);
                        da += dP[b] * w[k] * sample(k, b);
                    }
                    scatter(g.g_in, g.g_fixed, g.fixed_scale, gidx(k, 3), da);
                }
                for (int b = 0; b < 3; ++b) { dx += dP[b] * P[b].dfx; dy += dP[b] * P[b].dfy; }
                dx += dA * A.dfx;
                dy += dA * A.dfy;
            } else {
                for (int b = 0; b < bands; ++b) {
                    const double gb = (double)gy[b];
                    const Bil v = bil(sample(0, b), sample(1, b), sample(2, b), sample(3, b), fx, fy);
                    dx += gb * v.dfx;
                    dy += gb * v.dfy;
                    for (int k = 0; k < 4; ++k)
                        if (lin[k] >= 0) scatter(g.g_in, g.g_fixed, g.fixed_scale, gidx(k, b), gb * w[k]);
                }
            }
            // x_in = m0 X + m1 Y + tx, y_in = m2 X + m3 Y + ty
            part[0] = dx * (double)X; part[1] = dx * (double)Y;
            part[2] = dy * (double)X; part[3] = dy * (double)Y;
            part[4] = dx; part[5] = dy;
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
            g.partial[(int64_t)blockIdx.x * 6 + threadIdx.x] = s;
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

__global__ void __launch_bounds__(256) mapim_grad_kernel(MapimGradArgs g) {
    const MapimArgs& a = g.fwd;
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npx) return;
    const int64_t ly = p / a.out.w, lx = p - ly * a.out.w;
    const float2 idx = *reinterpret_cast<const float2*>(a.index.data + ly * a.index.pitch + lx * 8);
    const double x = (double)idx.x, y = (double)idx.y;
    const int bands = a.bands;
    const float* gy = g.g_out + p * bands;
    const float* src = reinterpret_cast<const float*>(a.src.data);
    const int64_t pitch_f = a.src.pitch / 4;
    double gx = 0.0, gyy = 0.0;
    if (isfinite(x) && isfinite(y)) {
        const int k = a.kernel;
        auto inb = [&](int64_t ix, int64_t iy) {
            return ix >= 0 && ix < (int64_t)a.src_w && iy >= 0 && iy < (int64_t)a.src_h;
        };
        if (k == 0) {
            const int64_t ix = trunc_i64(floor(x)), iy = trunc_i64(floor(y));
            int64_t rx = ix, ry = iy;
            bool ok = inb(ix, iy);
            if (!ok && a.extend_copy) {
                ok = !(ix < -1 || ix > (int64_t)a.src_w || iy < -1 || iy > (int64_t)a.src_h);
                rx = clampi64(ix, 0, (int64_t)a.src_w - 1);
                ry = clampi64(iy, 0, (int64_t)a.src_h - 1);
            }
            if (ok)
                for (int b = 0; b < bands; ++b) scatter(g.g_src, g.g_fixed, g.fixed_scale, ry * pitch_f + rx * bands + b, gy[b]);
        } else if (k == 1) {
            const int64_t x0 = trunc_i64(floor(x)), y0 = trunc_i64(floor(y));
            const double fx = x - (double)x0, fy = y - (double)y0;
            const double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
            const int64_t tx_[4] = {x0, x0 + 1, x0, x0 + 1}, ty_[4] = {y0, y0, y0 + 1, y0 + 1};
            for (int b = 0; b < bands; ++b) {
                double s[4];
                for (int q = 0; q < 4; ++q) {
                    int64_t rx = tx_[q], ry = ty_[q];
                    bool ok = inb(rx, ry);
                    if (!ok && a.extend_copy) {
                        ok = !(rx < -1 || rx > (int64_t)a.src_w + 1 || ry < -1 || ry > (int64_t)a.src_h + 1);
                        rx = clampi64(rx, 0, (int64_t)a.src_w - 1);
                        ry = clampi64(ry, 0, (int64_t)a.src_h - 1);
                    }
                    s[q] = ok ? (double)src[ry * pitch_f + rx * bands + b] : a.background;
                    if (ok) scatter(g.g_src, g.g_fixed, g.fixed_scale, ry * pitch_f + rx * bands + b, (double)gy[b] * w[q]);
                }
                const Bil v = bil(s[0], s[1], s[2], s[3], fx, fy);
                gx += (double)gy[b] * v.dfx;
                gyy += (double)gy[b] * v.dfy;
            }
        } else {
            const int64_t support = k == 9 ? 3 : 2;
            const int64_t cx = trunc_i64(floor(x)), cy = trunc_i64(floor(y));
            const int nt = int(2 * support);
            double wx[6], wy[6], dwx[6], dwy[6];
            for (int t = 0; t < nt; ++t) {
                const int64_t ix = cx - (support - 1) + t, iy = cy - (support - 1) + t;
                wx[t] = kernel_w(k, fabs((double)ix - x));
                wy[t] = kernel_w(k, fabs((double)iy - y));
                dwx[t] = kernel_dw(k, (double)ix - x);
                dwy[t] = kernel_dw(k, (double)iy - y);
            }
            double W = 0.0, Wx = 0.0, Wy = 0.0;
            for (int ty = 0; ty < nt; ++ty) {
                if (wy[ty] == 0.0) continue;
                for (int tx = 0; tx < nt; ++tx) {
                    if (wx[tx] == 0.0) continue;
                    W += wx[tx] * wy[ty];
                    Wx += dwx[tx] * wy[ty];
                    Wy += wx[tx] * dwy[ty];
                }
            }
            if (W > 0.0) {
                for (int b = 0; b < bands; ++b) {
                    double Nv = 0.0, Nx = 0.0, Ny = 0.0;
                    const double gb = (double)gy[b];
                    for (int ty = 0; ty < nt; ++ty) {
                        if (wy[ty] == 0.0) continue;
                        const int64_t iy = cy - (support - 1) + ty;
                        for (int tx = 0; tx < nt; ++tx) {
                            if (wx[tx] == 0.0) continue;
                            const int64_t ix = cx - (support - 1) + tx;
                            const bool ok = inb(ix, iy);
                            const double s = ok ? (double)src[iy * pitch_f + ix * bands + b] : a.background;
                            Nv += wx[tx] * wy[ty] * s;
                            Nx += dwx[tx] * wy[ty] * s;
                            Ny += wx[tx] * dwy[ty] * s;
                            if (ok) scatter(g.g_src, g.g_fixed, g.fixed_scale, iy * pitch_f + ix * bands + b, gb * wx[tx] * wy[ty] / W);
                        }
                    }
                    gx += gb * (Nx * W - Nv * Wx) / (W * W);
                    gyy += gb * (Ny * W - Nv * Wy) / (W * W);
                }
            }
        }
    }
    if (g.g_index) {
        g.g_index[p * 2] = (float)gx;
        g.g_index[p * 2 + 1] = (float)gyy;
    }
}

__global__ void fixed_to_f32_kernel(const unsigned long long* acc, float* out, int64_t n, double inv) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)((double)(long long)acc[i] * inv);
}

__global__ void sum_partials_kernel(const double* partial, int blocks, double* out) {
    // one thread per component, fixed order: deterministic
    if (threadIdx.x < 6) {
        double s = 0.0;
        for (int b = 0; b < blocks; ++b) s += partial[(int64_t)b * 6 + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

}  // namespace dev

namespace launch {

cudaError_t reduce_adjoint(const ReduceAdjArgs& a, cudaStream_t s) {
    const int64_t n = (int64_t)a.in_w * a.in_h * a.bands;
    if (n <= 0) return cudaSuccess;
    dev::reduce_adjoint_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t affine_grad(const AffineGradArgs& a, int blocks, cudaStream_t s) {
    if (blocks <= 0) return cudaSuccess;
    dev::affine_grad_kernel<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t mapim_grad(const MapimGradArgs& a, cudaStream_t s) {
    const int64_t npx = (int64_t)a.fwd.out.w * a.fwd.out.h;
    if (npx <= 0) return cudaSuccess;
    dev::mapim_grad_kernel<<<(unsigned)((npx + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fixed_to_f32(const unsigned long long* acc, float* out, int64_t n, double inv_scale, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    dev::fixed_to_f32_kernel<<<grid, 256, 0, s>>>(acc, out, n, inv_scale);
    return cudaGetLastError();
}

cudaError_t sum_partials(const double* partial, int blocks, double* out, cudaStream_t s) {
    dev::sum_partials_kernel<<<1, 32, 0, s>>>(partial, blocks, out);
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
