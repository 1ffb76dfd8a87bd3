// resample_dev.cuh -- device code of the box shrink and separable reduce ops
// (see resample.cu for the viprs files each routine follows).  Included by
// resample.cu (standalone kernels) and batch.cu (the persistent batch kernel).
#pragma once

#include <algorithm>

#include "common.cuh"
#include "tma.cuh"
#include "viprs_b200.h"

namespace viprs {
namespace dev {

constexpr int kShrinkThreads = 256;

// The routines below that a whole block runs together (the fused reduce
// tile, the reduce row chunks, the shrink edge items) use kCThreads threads
// (0..255) and barrier 1 for 256 threads: the standalone kernels launch
// exactly 256 threads, and the persistent batch kernel adds a producer warp
// (threads 256..287) that never joins barrier 1.
constexpr int kCThreads = 256;
__device__ __forceinline__ void csync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
constexpr int kShrinkMaxItems = 4;  // (column, band) outputs per thread
constexpr int kShrinkSegCap = 16384;  // target staging bytes per input row

// ---------------------------------------------------------------- shrink

// u8 rounding of ShrinkH (shrinkh.rs:323-397): factor 1 copies, 2 rounds up a
// half, 5 with 1/3/4 bands divides exactly, anything else uses libvips's
// multiplier (sum + f/2) * floor(2^32 / (256 f)) >> 24.
__device__ __forceinline__ uint32_t shrinkh_round_u8(uint32_t sum, uint32_t f, int bands) {
    if (f == 1) return sum;
    if (f == 2) return (sum + 1) >> 1;
    if (f == 5 && (bands == 1 || bands == 3 || bands == 4)) return (sum + 2) / 5;
    const unsigned long long mult = (1ull << 32) / (256ull * f);
    return static_cast<uint32_t>(((unsigned long long)(sum + f / 2) * mult) >> 24);
}
// u8 rounding of ShrinkV (shrinkv.rs:191-339): no factor-5 special case.
__device__ __forceinline__ uint32_t shrinkv_round_u8(uint32_t sum, uint32_t f) {
    if (f == 1) return sum;
    if (f == 2) return (sum + 1) >> 1;
    const unsigned long long mult = (uint32_t)((1ull << 32) / (256ull * f));
    return static_cast<uint32_t>(((unsigned long long)(sum + f / 2) * mult) >> 24);
}

// The same rounding with host-computed constants (mode 0 copy, 1 factor 2,
// 2 exact division by 5, 3 multiplier), avoiding 64-bit division on the device.
__device__ __forceinline__ uint32_t round_mode_u8(uint32_t sum, int mode, uint32_t f, uint64_t mult) {
    switch (mode) {
    case 0: return sum;
    case 1: return (sum + 1) >> 1;
    case 2: return (sum + 2) / 5;
    default: return (uint32_t)(((unsigned long long)(sum + f / 2) * mult) >> 24);
    }
}

template <typename T>
__device__ __forceinline__ double as_f64(T v) { return static_cast<double>(v); }

// Copy `nelem` samples of local row `ly`, starting at local column `c0`, into
// shared memory.  Interior segments use 16-byte loads of the aligned span
// that covers them; the returned pointer is the first sample.  Segments that
// leave the plane read per sample with clamped columns (edge replication).
template <typename T>
__device__ __forceinline__ const T* stage_row(const Plane& in, int64_t ly, int64_t c0, int nin, int bands,
                              uint8_t* raw) {
    ly = ly < 0 ? 0 : (ly >= in.h ? in.h - 1 : ly);
    const int nelem = nin * bands;
    const uint8_t* row = in.data + ly * in.pitch;
    if (c0 >= 0 && c0 + nin <= in.w) {
        const int64_t s = (row - in.data) + c0 * bands * (int64_t)sizeof(T);
        const int64_t e = s + (int64_t)nelem * sizeof(T);
        const int64_t as = s & ~int64_t(15);
        const int64_t ae = (e + 15) & ~int64_t(15);
        if (ae <= in.total_bytes && (reinterpret_cast<uintptr_t>(in.data) & 15) == 0) {
            const uint4* src = reinterpret_cast<const uint4*>(in.data + as);
            uint4* dst = reinterpret_cast<uint4*>(raw);
            const int nv = int((ae - as) >> 4);
            for (int i = threadIdx.x; i < nv; i += blockDim.x) dst[i] = __ldg(src + i);
            return reinterpret_cast<const T*>(raw + (s - as));
        }
        const T* srow = reinterpret_cast<const T*>(row) + c0 * bands;
        T* d = reinterpret_cast<T*>(raw);
        for (int i = threadIdx.x; i < nelem; i += blockDim.x) d[i] = srow[i];
        return d;
    }
    const T* srow = reinterpret_cast<const T*>(row);
    T* d = reinterpret_cast<T*>(raw);
    for (int i = threadIdx.x; i < nelem; i += blockDim.x) {
        int64_t col = c0 + i / bands;
        col = col < 0 ? 0 : (col >= in.w ? in.w - 1 : col);
        d[i] = srow[col * bands + (i % bands)];
    }
    return d;
}

// Premultiply the staged samples of a row in place (u8, alpha last).
__device__ __forceinline__ void premultiply_staged(uint8_t* seg, int nin, int bands) {
    const int ab = bands - 1;
    for (int p = threadIdx.x; p < nin; p += blockDim.x) {
        const uint32_t a = seg[p * bands + ab];
        for (int b = 0; b < ab; ++b) seg[p * bands + b] = (uint8_t)premultiply_u8(seg[p * bands + b], a);
    }
}

template <typename T>
__device__ __forceinline__ void store_sample(uint8_t* row, int64_t idx, T v) {
    reinterpret_cast<T*>(row)[idx] = v;
}

// One block: output row blockIdx.y, output columns [blockIdx.x*nx, +nx).
template <typename T, bool HV>
__global__ void __launch_bounds__(kShrinkThreads) shrink2d_kernel(ShrinkArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int bands = a.bands;
    const uint32_t fh = a.fh, fv = a.fv;
    const int nx = a.nx;
    const int64_t oy = blockIdx.y;
    const int64_t Y = a.out.y0 + oy;
    const int64_t xb = a.col_lo + (int64_t)blockIdx.x * nx;
    const int64_t rem = a.col_hi - xb;
    const int ncols = (int)(rem < nx ? rem : nx);
    if (ncols <= 0) return;
    const int64_t X0 = a.out.x0 + xb;
    const int64_t c0 = X0 * (int64_t)fh - a.in.x0;
    const int nin = ncols * (int)fh;
    const int nitems = ncols * bands;
    const int seg_bytes = ((nin * bands * (int)sizeof(T)) + 15) / 16 * 16 + 32;
    uint8_t* raw = smem;
    uint8_t* extra = smem + seg_bytes;  // VH accumulators / output staging
    const double inv_h = 1.0 / double(fh), inv_v = 1.0 / double(fv);

    if (HV) {
        uint32_t vacc_u[kShrinkMaxItems];
        double vacc_d[kShrinkMaxItems];
#pragma unroll
        for (int s = 0; s < kShrinkMaxItems; ++s) { vacc_u[s] = 0; vacc_d[s] = 0.0; }
        for (uint32_t k = 0; k < fv; ++k) {
            const int64_t ly = Y * (int64_t)fv + k - a.in.y0;
            const T* seg = stage_row<T>(a.in, ly, c0, nin, bands, raw);
            __syncthreads();
            if (sizeof(T) == 1 && a.premul_in) {
                premultiply_staged(reinterpret_cast<uint8_t*>(const_cast<T*>(seg)), nin, bands);
                __syncthreads();
            }
#pragma unroll
            for (int s = 0; s < kShrinkMaxItems; ++s) {
                const int item = threadIdx.x + s * kShrinkThreads;
                if (item < nitems) {
                    const int x = item / bands, b = item - (item / bands) * bands;
                    const T* p = seg + (int64_t)x * fh * bands + b;
                    if (sizeof(T) == 1) {
                        uint32_t sum = 0;
                        for (uint32_t j = 0; j < fh; ++j) sum += (uint32_t)p[j * bands];
                        vacc_u[s] += round_mode_u8(sum, a.hmode, fh, a.hmult);
                    } else {
                        double hv;
                        if (fh == 1) {
                            hv = as_f64(p[0]);
                        } else {
                            double sum = 0.0;
                            for (uint32_t j = 0; j < fh; ++j) sum += as_f64(p[j * bands]);
                            hv = as_f64(shrink_from_f64<T>(sum * inv_h));
                        }
                        vacc_d[s] += hv;
                    }
                }
            }
            __syncthreads();
        }
        T outv[kShrinkMaxItems];
#pragma unroll
        for (int s = 0; s < kShrinkMaxItems; ++s) {
            if (sizeof(T) == 1) outv[s] = (T)round_mode_u8(vacc_u[s], a.vmode, fv, a.vmult);
            else outv[s] = fv == 1 ? (T)vacc_d[s] : shrink_from_f64<T>(vacc_d[s] * inv_v);
        }
        uint8_t* orow = a.out.data + oy * a.out.pitch;
        if (sizeof(T) == 1 && a.unpremul_out) {
            uint8_t* ob = extra;
#pragma unroll
            for (int s = 0; s < kShrinkMaxItems; ++s) {
                const int item = threadIdx.x + s * kShrinkThreads;
                if (item < nitems) ob[item] = (uint8_t)outv[s];
            }
            __syncthreads();
            const int ab = bands - 1;
            for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
                const int x = item / bands, b = item - x * bands;
                uint32_t v = ob[item];
                if (b != ab) v = unpremultiply_u8(v, ob[x * bands + ab]);
                orow[xb * bands + item] = (uint8_t)v;
            }
        } else {
#pragma unroll
            for (int s = 0; s < kShrinkMaxItems; ++s) {
                const int item = threadIdx.x + s * kShrinkThreads;
                if (item < nitems) store_sample<T>(orow, xb * bands + item, outv[s]);
            }
        }
    } else {
        // ShrinkV first (per input sample), then ShrinkH (resize.rs:216-224 order).
        const int nelem = nin * bands;
        uint32_t* acc_u = reinterpret_cast<uint32_t*>(extra);
        double* acc_d = reinterpret_cast<double*>(extra);
        for (int i = threadIdx.x; i < nelem; i += blockDim.x) {
            if (sizeof(T) == 1) acc_u[i] = 0; else acc_d[i] = 0.0;
        }
        __syncthreads();
        for (uint32_t k = 0; k < fv; ++k) {
            const int64_t ly = Y * (int64_t)fv + k - a.in.y0;
            const T* seg = stage_row<T>(a.in, ly, c0, nin, bands, raw);
            __syncthreads();
            if (sizeof(T) == 1 && a.premul_in) {
                premultiply_staged(reinterpret_cast<uint8_t*>(const_cast<T*>(seg)), nin, bands);
                __syncthreads();
            }
            for (int i = threadIdx.x; i < nelem; i += blockDim.x) {
                if (sizeof(T) == 1) acc_u[i] += (uint32_t)seg[i]; else acc_d[i] += as_f64(seg[i]);
            }
            __syncthreads();
        }
        T* vvals = reinterpret_cast<T*>(raw);
        for (int i = threadIdx.x; i < nelem; i += blockDim.x) {
            if (sizeof(T) == 1) vvals[i] = (T)round_mode_u8(acc_u[i], a.vmode, fv, a.vmult);
            else vvals[i] = fv == 1 ? (T)acc_d[i] : shrink_from_f64<T>(acc_d[i] * inv_v);
        }
        __syncthreads();
        uint8_t* orow = a.out.data + oy * a.out.pitch;
        for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
            const int x = item / bands, b = item - x * bands;
            const T* p = vvals + (int64_t)x * fh * bands + b;
            T o;
            if (sizeof(T) == 1) {
                uint32_t sum = 0;
                for (uint32_t j = 0; j < fh; ++j) sum += (uint32_t)p[j * bands];
                o = (T)round_mode_u8(sum, a.hmode, fh, a.hmult);
            } else if (fh == 1) {
                o = p[0];
            } else {
                double sum = 0.0;
                for (uint32_t j = 0; j < fh; ++j) sum += as_f64(p[j * bands]);
                o = shrink_from_f64<T>(sum * inv_h);
            }
            store_sample<T>(orow, xb * bands + item, o);
        }
    }
}

// Premultiply<U8> in place over `npx` staged pixels of B bands (alpha last).
template <int B>
__device__ __forceinline__ void premultiply_pixels(uint8_t* seg, int npx) {
    for (int p = threadIdx.x; p < npx; p += kCThreads) {
        uint8_t* px = seg + p * B;
        const uint32_t a = px[B - 1];
#pragma unroll
        for (int b = 0; b < B - 1; ++b) px[b] = (uint8_t)premultiply_u8(px[b], a);
    }
}

// Output columns of the interior whose source boxes lie inside the plane are
// processed by the bulk-copy ring below; the few edge columns (the reduce
// halo beyond the image) by this routine: one (output row, column range)
// item, every source sample read with clamped coordinates.
template <int B>
__device__ void shrink_edge_item_u8(const ShrinkArgs& a, int32_t oy, int32_t c0, int32_t c1, uint8_t* buf) {
    const int32_t fh = int32_t(a.fh), fv = int32_t(a.fv);
    const int32_t ncols = c1 - c0;
    const int32_t per_row = ncols * fh * B;
    const int64_t Y = a.out.y0 + oy;
    for (int32_t i = threadIdx.x; i < fv * per_row; i += kCThreads) {
        const int32_t k = i / per_row, rem = i - k * per_row;
        const int32_t xb = rem / B, b = rem - xb * B;
        const int64_t sx = (a.out.x0 + c0) * (int64_t)fh + xb - a.in.x0;
        buf[i] = load_sample<uint8_t>(a.in, sx, Y * fv + k - a.in.y0, B, b);
    }
    csync();
    if (a.premul_in) {
        premultiply_pixels<B>(buf, fv * ncols * fh);
        csync();
    }
    uint8_t* ob = buf + fv * per_row;
    for (int32_t item = threadIdx.x; item < ncols * B; item += kCThreads) {
        const int32_t x = item / B, b = item - x * B;
        uint32_t vs = 0;
        for (int32_t k = 0; k < fv; ++k) {
            const uint8_t* p = buf + k * per_row + x * fh * B + b;
            uint32_t hs = 0;
            for (int32_t j = 0; j < fh; ++j) hs += p[j * B];
            vs += round_mode_u8(hs, a.hmode, uint32_t(fh), a.hmult);
        }
        ob[item] = (uint8_t)round_mode_u8(vs, a.vmode, uint32_t(fv), a.vmult);
    }
    csync();
    uint8_t* orow = a.out.data + (int64_t)oy * a.out.pitch + (int64_t)c0 * B;
    for (int32_t item = threadIdx.x; item < ncols * B; item += kCThreads) {
        const int32_t x = item / B, b = item - x * B;
        uint32_t v = ob[item];
        if (a.unpremul_out && b != B - 1) v = unpremultiply_u8(v, ob[x * B + B - 1]);
        orow[item] = (uint8_t)v;
    }
    csync();
}

// Column chunk `c` of a shrink item: output columns [lx0, lx0 + ncols) and the
// plane columns [s_lo, s_hi) its boxes read (clamped into the plane).
struct ShrinkChunk {
    int32_t lx0, ncols;
    int64_t s_lo, s_hi;
};

__device__ __forceinline__ ShrinkChunk shrink_chunk(const ShrinkArgs& a, int32_t c) {
    ShrinkChunk k;
    k.lx0 = c * a.nxf;
    k.ncols = min(a.nxf, a.out.w - k.lx0);
    const int64_t fh = a.fh;
    int64_t lo = (a.out.x0 + k.lx0) * fh - a.in.x0, hi = (a.out.x0 + k.lx0 + k.ncols) * fh - a.in.x0;
    lo = lo < 0 ? 0 : (lo >= a.in.w ? a.in.w - 1 : lo);
    hi = hi <= lo ? lo + 1 : (hi > a.in.w ? a.in.w : hi);
    k.s_lo = lo;
    k.s_hi = hi;
    return k;
}

// ---------------------------------------------------------------- u8 box sums
//
// Helpers of the u8 ShrinkH+ShrinkV kernels (shrink_warp.cuh): box sums of
// one output pixel from a staged source row segment, and the rounding.

// Threads of the blocks that run whole-block routines (reduce tiles and rows)
// plus the producer warp of the persistent batch kernel.
constexpr int kWsThreads = kCThreads + 32;

// 32-bit rounding of a box sum: (s * mul + add) >> 24 reproduces every u8
// rounding rule of ShrinkH / ShrinkV (shrinkh.rs:323-397, shrinkv.rs:191-339)
// with host-computed constants, and never overflows (s <= 255 f).
__device__ __forceinline__ uint32_t round_box(uint32_t s, uint32_t mul, uint32_t add) {
    return (s * mul + add) >> 24;
}

// Box sums of one output pixel's fh source pixels (B bands, u8) from shared
// memory at any byte alignment: words are realigned with a funnel shift and
// the bands are summed four bytes at a time with dp4a masks.  Words go in
// groups of G (3 for 3 bands: the band pattern repeats every 12 bytes, else
// 1); two accumulator sets halve the dp4a chains.  The last group is masked
// to the box and may read up to 16 bytes past it (stage buffers carry 32
// bytes of slack).
template <int B>
__device__ __forceinline__ void box_sums_u8(const uint8_t* p, int fh, uint32_t (&sums)[B]) {
    constexpr int G = B == 3 ? 3 : 1;
    const int o = int(reinterpret_cast<uintptr_t>(p) & 3);
    const uint32_t* wp = reinterpret_cast<const uint32_t*>(p - o);
    const int nbytes = fh * B;
    const int K = (nbytes + 3) >> 2;  // realigned words, the last one partial
    const int Kg = (K + G - 1) / G;   // groups, the last one masked
    const uint32_t sh = 8u * uint32_t(o);
    uint32_t sa[B], sb[B];
#pragma unroll
    for (int b = 0; b < B; ++b) { sa[b] = 0; sb[b] = 0; }
    // realigned word of phase `ph` within a group -> band sums
    auto acc = [&](uint32_t (&s)[B], uint32_t w, int ph) {
        if (B == 1) {
            s[0] = __dp4a(w, 0x01010101u, s[0]);
        } else if (B == 2) {
            s[0] = __dp4a(w, 0x00010001u, s[0]);
            s[1 % B] = __dp4a(w, 0x01000100u, s[1 % B]);
        } else if (B == 3) {
            const uint32_t m0 = ph == 0 ? 0x01000001u : (ph == 1 ? 0x00010000u : 0x00000100u);
            const uint32_t m1 = ph == 0 ? 0x00000100u : (ph == 1 ? 0x01000001u : 0x00010000u);
            const uint32_t m2 = ph == 0 ? 0x00010000u : (ph == 1 ? 0x00000100u : 0x01000001u);
            s[0] = __dp4a(w, m0, s[0]);
            s[1 % B] = __dp4a(w, m1, s[1 % B]);
            s[2 % B] = __dp4a(w, m2, s[2 % B]);
        } else {
#pragma unroll
            for (int b = 0; b < B; ++b) s[b] = __dp4a(w, 1u << (8 * b), s[b]);
        }
    };
    // unmasked groups [g0, g1): two accumulator sets halve the dp4a chains
    auto run = [&](int g0, int g1) {
        if (g0 >= g1) return;
        int k = g0 * G;
        uint32_t lo = wp[k];
        int g = g0;
        for (; g + 2 <= g1; g += 2, k += 2 * G) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const uint32_t hi = wp[k + j + 1];
                acc(sa, __funnelshift_r(lo, hi, sh), j);
                lo = hi;
            }
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const uint32_t hi = wp[k + G + j + 1];
                acc(sb, __funnelshift_r(lo, hi, sh), j);
                lo = hi;
            }
        }
        if (g < g1) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const uint32_t hi = wp[k + j + 1];
                acc(sa, __funnelshift_r(lo, hi, sh), j);
                lo = hi;
            }
        }
    };
    run(0, Kg - 1);
    {
        const int k = (Kg - 1) * G;
        uint32_t lo = wp[k];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const uint32_t hi = wp[k + j + 1];
            const int valid = nbytes - 4 * (k + j);
            const uint32_t m = valid >= 4 ? 0xFFFFFFFFu : (valid <= 0 ? 0u : ((1u << (8 * valid)) - 1u));
            acc(sb, __funnelshift_r(lo, hi, sh) & m, j);
            lo = hi;
        }
    }
#pragma unroll
    for (int b = 0; b < B; ++b) sums[b] = sa[b] + sb[b];
}

// Premultiplied box sums of fh 4-band pixels (Premultiply<U8> applied to each
// source pixel before the sum, as the separate Premultiply op would), from a
// 4-byte aligned box.  Every lane walks fh pixels starting at pixel q0 and
// wrapping around (the same trip count for every lane, so the warp does not
// diverge), which spreads the lanes' reads over the shared-memory banks when
// their boxes lie a multiple of 128 bytes apart.
// premultiply_u8(c, a) = (t + (t >> 8)) >> 8 with t = c a + 128 equals
// (c (257 a) + 32896) >> 16 for every c, a in 0..255 (t < 65536).
__device__ __forceinline__ void box_sums_premul4_rot(const uint8_t* p, int fh, int q0, uint32_t (&sums)[4]) {
    const uint32_t* wp = reinterpret_cast<const uint32_t*>(p);
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int j = q0;
    for (int t = 0; t < fh; ++t) {
        const uint32_t w = wp[j];
        j = j + 1 == fh ? 0 : j + 1;
        const uint32_t a = w >> 24;
        const uint32_t a257 = a * 257u;
        s0 += (__byte_perm(w, 0u, 0x4440) * a257 + 32896u) >> 16;
        s1 += (__byte_perm(w, 0u, 0x4441) * a257 + 32896u) >> 16;
        s2 += (__byte_perm(w, 0u, 0x4442) * a257 + 32896u) >> 16;
        s3 += a;
    }
    sums[0] = s0;
    sums[1] = s1;
    sums[2] = s2;
    sums[3] = s3;
}

// Box sums with columns clamped to the plane (boxes of the reduce halo), and
// for 2/4 bands optionally premultiplied.
template <int B>
__device__ __forceinline__ void box_sums_clamped_pm_u8(const uint8_t* span, int64_t first_col, int fh, int64_t c_lo,
                                                       int64_t w, bool premul, uint32_t (&sums)[B]) {
#pragma unroll
    for (int b = 0; b < B; ++b) sums[b] = 0;
    for (int j = 0; j < fh; ++j) {
        int64_t c = first_col + j;
        c = c < 0 ? 0 : (c >= w ? w - 1 : c);
        const uint8_t* px = span + (c - c_lo) * B;
        const uint32_t al = px[B - 1];
#pragma unroll
        for (int b = 0; b < B; ++b)
            sums[b] += (premul && b != B - 1) ? premultiply_u8(px[b], al) : (uint32_t)px[b];
    }
}

// Premultiplied box sums of fh pixels, 2 bands (grey, alpha).
__device__ __forceinline__ void box_sums_premul2_u8(const uint8_t* p, int fh, uint32_t (&sums)[2]) {
    uint32_t s0 = 0, s1 = 0;
    for (int j = 0; j < fh; ++j) {
        const uint32_t al = p[2 * j + 1];
        s0 += premultiply_u8(p[2 * j], al);
        s1 += al;
    }
    sums[0] = s0;
    sums[1] = s1;
}

// ---------------------------------------------------------------- reduce

template <typename T>
__device__ __forceinline__ uint32_t load_premul(const Plane& p, int64_t lx, int64_t ly, int bands, int b,
                                                bool premul) {
    uint32_t v = (uint32_t)load_sample<T>(p, lx, ly, bands, b);
    if (premul && b != bands - 1) v = premultiply_u8(v, (uint32_t)load_sample<T>(p, lx, ly, bands, bands - 1));
    return v;
}

// Store one output row chunk; unpremultiply (u8) needs the pixel's alpha, which
// another thread of the block computed: stage through shared memory.
template <typename T>
__device__ __forceinline__ void store_or_unpremul(uint8_t* orow, int64_t item, int nitems, T v, bool unpremul,
                                                  int bands, uint8_t* stage) {
    if (!unpremul) {
        if (item < nitems) reinterpret_cast<T*>(orow)[item] = v;
        return;
    }
    const int local = threadIdx.x;
    if (item < nitems) stage[local] = (uint8_t)v;
    csync();
    if (item < nitems) {
        const int b = int(item % bands);
        uint32_t o = stage[local];
        if (b != bands - 1) o = unpremultiply_u8(o, stage[local + (bands - 1 - b)]);
        orow[item] = (uint8_t)o;
    }
}

// One chunk of kCThreads output samples (`chunk`) of output row `oy`.
template <typename T, int MODE>
__device__ void reduce_h_chunk(const ReduceArgs& a, int64_t chunk, int64_t oy, uint8_t* smem) {
    const int taps = a.taps, bands = a.bands;
    const int coef_bytes = 65 * taps * (MODE == kReduceFixed ? 2 : 8);
    const bool coef_in_smem = coef_bytes <= 48 * 1024;
    const uint8_t* coef = reinterpret_cast<const uint8_t*>(a.coeffs);
    if (coef_in_smem) {
        for (int i = threadIdx.x * 4; i < coef_bytes; i += kCThreads * 4)
            *reinterpret_cast<uint32_t*>(smem + i) = *reinterpret_cast<const uint32_t*>(coef + i);
        csync();
        coef = smem;
    }
    uint8_t* stage = smem + ((coef_in_smem ? coef_bytes : 0) + 15) / 16 * 16;
    const int nitems = a.out.w * bands;
    const int64_t item = chunk * kCThreads + threadIdx.x;
    const int64_t ly = a.out.y0 + oy - a.in.y0;
    T outv = T(0);
    if (item < nitems) {
        const int x = int(item / bands), b = int(item - (item / bands) * bands);
        const int64_t base = (int64_t)a.starts[x] - a.in.x0;
        const int ph = a.phases[x];
        if (MODE == kReduceFixed) {
            const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
            int32_t acc = 0;
            for (int t = 0; t < taps; ++t)
                acc += (int32_t)c[t] * (int32_t)load_premul<T>(a.in, base + t, ly, bands, b, a.premul_in);
            outv = from_fixed<T>(acc);
        } else {
            const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
            double acc = 0.0;
            if (MODE == kReduceF32Simd) {
                // reduce_h_f32_avx2_pixel: 4-tap products summed in lane order, fma tail
                int t = 0;
                for (; t + 4 <= taps; t += 4) {
                    double lanes = as_f64(load_sample<T>(a.in, base + t, ly, bands, b)) * c[t];
                    lanes = lanes + as_f64(load_sample<T>(a.in, base + t + 1, ly, bands, b)) * c[t + 1];
                    lanes = lanes + as_f64(load_sample<T>(a.in, base + t + 2, ly, bands, b)) * c[t + 2];
                    lanes = lanes + as_f64(load_sample<T>(a.in, base + t + 3, ly, bands, b)) * c[t + 3];
                    acc = acc + lanes;
                }
                for (; t < taps; ++t) acc = fma(as_f64(load_sample<T>(a.in, base + t, ly, bands, b)), c[t], acc);
            } else {
                for (int t = 0; t < taps; ++t)
                    acc = fma(as_f64(load_sample<T>(a.in, base + t, ly, bands, b)), c[t], acc);
            }
            outv = from_f64<T>(acc);
        }
    }
    store_or_unpremul<T>(a.out.data + oy * a.out.pitch, item, nitems, outv, a.unpremul_out != 0, bands, stage);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) reduce_h_kernel(ReduceArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    reduce_h_chunk<T, MODE>(a, blockIdx.x, blockIdx.y, smem);
}

template <typename T, int MODE>
__device__ void reduce_v_chunk(const ReduceArgs& a, int64_t chunk, int64_t oy, uint8_t* smem) {
    const int taps = a.taps, bands = a.bands;
    const int coef_bytes = 65 * taps * (MODE == kReduceFixed ? 2 : 8);
    const bool coef_in_smem = coef_bytes <= 48 * 1024;
    const uint8_t* coef = reinterpret_cast<const uint8_t*>(a.coeffs);
    if (coef_in_smem) {
        for (int i = threadIdx.x * 4; i < coef_bytes; i += kCThreads * 4)
            *reinterpret_cast<uint32_t*>(smem + i) = *reinterpret_cast<const uint32_t*>(coef + i);
        csync();
        coef = smem;
    }
    uint8_t* stage = smem + ((coef_in_smem ? coef_bytes : 0) + 15) / 16 * 16;
    const int nitems = a.out.w * bands;
    const int64_t item = chunk * kCThreads + threadIdx.x;
    const int64_t base = (int64_t)a.starts[oy] - a.in.y0;
    const int ph = a.phases[oy];
    T outv = T(0);
    if (item < nitems) {
        const int x = int(item / bands), b = int(item - (item / bands) * bands);
        const int64_t lx = a.out.x0 + x - a.in.x0;
        if (MODE == kReduceFixed) {
            const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
            int32_t acc = 0;
            for (int t = 0; t < taps; ++t)
                acc += (int32_t)c[t] * (int32_t)load_premul<T>(a.in, lx, base + t, bands, b, a.premul_in);
            outv = from_fixed<T>(acc);
        } else {
            const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
            double acc = 0.0;
            if (MODE == kReduceF32Simd && item < a.vector_len) {
                for (int t = 0; t < taps; ++t) acc = acc + as_f64(load_sample<T>(a.in, lx, base + t, bands, b)) * c[t];
            } else {
                for (int t = 0; t < taps; ++t) acc = fma(as_f64(load_sample<T>(a.in, lx, base + t, bands, b)), c[t], acc);
            }
            outv = from_f64<T>(acc);
        }
    }
    store_or_unpremul<T>(a.out.data + oy * a.out.pitch, item, nitems, outv, a.unpremul_out != 0, bands, stage);
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) reduce_v_kernel(ReduceArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    reduce_v_chunk<T, MODE>(a, blockIdx.x, blockIdx.y, smem);
}

// ---------------------------------------------------------------- fused reduce
//
// ReduceH and ReduceV (either order) for one output tile, everything staged in
// shared memory: the tile's source rows are copied once with coalesced 16-byte
// loads, the first op's output (the mid tile, rounded to the sample type as
// viprs stores it) and the output tile never leave the SM.  Edge replication
// is a clamp of the tap index into the staged range: the staged range is the
// tile's tap span clamped to the source plane, so the clamp is the source
// read's clamp (and for the mid tile, clamp_axis of the second op).

// One sum of `taps` samples p[k * stride], k = clamp(s + t, 0, hi), with
// coefficient row c, in the accumulation order of `MODE`.
//   Fixed:      int32 sum of i16 x sample, (acc + 2048) >> 12 clamped
//   F32Simd, H: 4-lane partial sums of products, then sequential tail fmas
//               (reduce_h_f32 AVX2, reduce_simd.rs:2621-2694)
//   F32Simd, V: acc + v * w (mul then add) inside the vector body, fma in the
//               scalar tail (reduce_v_f32 AVX2, :2830-2888)
//   F64Fma:     sequential fma (scalar paths, ReduceOp)
template <typename T, int MODE, bool HORIZ>
__device__ __forceinline__ T fused_taps(const T* p, int s, int hi, int stride, int taps, const uint8_t* coef, int ph,
                                        bool simd_lane) {
    const bool inside = s >= 0 && s + taps - 1 <= hi;
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc = 0;
        if (inside) {
            const T* q = p + s * stride;
#pragma unroll 4
            for (int t = 0; t < taps; ++t) acc += (int32_t)c[t] * (int32_t)q[t * stride];
        } else {
            for (int t = 0; t < taps; ++t) {
                int k = s + t;
                k = k < 0 ? 0 : (k > hi ? hi : k);
                acc += (int32_t)c[t] * (int32_t)p[k * stride];
            }
        }
        return from_fixed<T>(acc);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        auto val = [&](int t) -> double {
            int k = s + t;
            if (!inside) k = k < 0 ? 0 : (k > hi ? hi : k);
            return as_f64(p[k * stride]);
        };
        double acc = 0.0;
        if (MODE == kReduceF32Simd && HORIZ) {
            int t = 0;
            for (; t + 4 <= taps; t += 4) {
                double lanes = val(t) * c[t];
                lanes = lanes + val(t + 1) * c[t + 1];
                lanes = lanes + val(t + 2) * c[t + 2];
                lanes = lanes + val(t + 3) * c[t + 3];
                acc = acc + lanes;
            }
            for (; t < taps; ++t) acc = fma(val(t), c[t], acc);
        } else if (MODE == kReduceF32Simd && simd_lane) {
            for (int t = 0; t < taps; ++t) acc = acc + val(t) * c[t];
        } else {
            for (int t = 0; t < taps; ++t) acc = fma(val(t), c[t], acc);
        }
        return from_f64<T>(acc);
    }
}

// The same vertical sum over staged source rows whose starts differ per row
// (`rowbase[k]` bytes from `base`).
template <typename T, int MODE>
__device__ __forceinline__ T fused_taps_rows(const uint8_t* base, const int32_t* rowbase, int col_bytes, int s, int hi,
                                             int taps, const uint8_t* coef, int ph, bool simd_lane) {
    auto at = [&](int t) -> T {
        int k = s + t;
        k = k < 0 ? 0 : (k > hi ? hi : k);
        return *reinterpret_cast<const T*>(base + rowbase[k] + col_bytes);
    };
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc = 0;
#pragma unroll 4
        for (int t = 0; t < taps; ++t) acc += (int32_t)c[t] * (int32_t)at(t);
        return from_fixed<T>(acc);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        double acc = 0.0;
        if (MODE == kReduceF32Simd && simd_lane) {
            for (int t = 0; t < taps; ++t) acc = acc + as_f64(at(t)) * c[t];
        } else {
            for (int t = 0; t < taps; ++t) acc = fma(as_f64(at(t)), c[t], acc);
        }
        return from_f64<T>(acc);
    }
}

// All NB bands of one output pixel at once: the coefficient of each tap is
// loaded once for the NB products.  p[k * stride + b] is band b of tap
// position k, k = clamp(s + t, 0, hi); each band keeps fused_taps' order.
// `lanes`: bit b set when band b lies in the V f32 vector body.
template <typename T, int MODE, bool HORIZ, int NB>
__device__ __forceinline__ void fused_taps_px(const T* p, int s, int hi, int stride, int taps, const uint8_t* coef,
                                              int ph, uint32_t lanes, T* out) {
    const bool inside = s >= 0 && s + taps - 1 <= hi;
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0;
        if (inside) {
            const T* q = p + s * stride;
#pragma unroll 4
            for (int t = 0; t < taps; ++t) {
                const int32_t ct = c[t];
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] += ct * (int32_t)q[t * stride + b];
            }
        } else {
            for (int t = 0; t < taps; ++t) {
                int k = s + t;
                k = k < 0 ? 0 : (k > hi ? hi : k);
                const int32_t ct = c[t];
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] += ct * (int32_t)p[k * stride + b];
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) out[b] = from_fixed<T>(acc[b]);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        auto pos = [&](int t) {
            int k = s + t;
            if (!inside) k = k < 0 ? 0 : (k > hi ? hi : k);
            return k * stride;
        };
        double acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0.0;
        if (MODE == kReduceF32Simd && HORIZ) {
            int t = 0;
            for (; t + 4 <= taps; t += 4) {
                const int k0 = pos(t), k1 = pos(t + 1), k2 = pos(t + 2), k3 = pos(t + 3);
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    double lanes4 = as_f64(p[k0 + b]) * c[t];
                    lanes4 = lanes4 + as_f64(p[k1 + b]) * c[t + 1];
                    lanes4 = lanes4 + as_f64(p[k2 + b]) * c[t + 2];
                    lanes4 = lanes4 + as_f64(p[k3 + b]) * c[t + 3];
                    acc[b] = acc[b] + lanes4;
                }
            }
            for (; t < taps; ++t) {
                const int k = pos(t);
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] = fma(as_f64(p[k + b]), c[t], acc[b]);
            }
        } else {
            for (int t = 0; t < taps; ++t) {
                const int k = pos(t);
                const double ct = c[t];
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    if (MODE == kReduceF32Simd && ((lanes >> b) & 1u)) acc[b] = acc[b] + as_f64(p[k + b]) * ct;
                    else acc[b] = fma(as_f64(p[k + b]), ct, acc[b]);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) out[b] = from_f64<T>(acc[b]);
    }
}

// The same vertical sum over staged source rows whose starts differ per row.
template <typename T, int MODE, int NB>
__device__ __forceinline__ void fused_taps_rows_px(const uint8_t* base, const int32_t* rowbase, int col_bytes, int s,
                                                   int hi, int taps, const uint8_t* coef, int ph, uint32_t lanes,
                                                   T* out) {
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0;
#pragma unroll 4
        for (int t = 0; t < taps; ++t) {
            int k = s + t;
            k = k < 0 ? 0 : (k > hi ? hi : k);
            const T* q = reinterpret_cast<const T*>(base + rowbase[k] + col_bytes);
            const int32_t ct = c[t];
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[b] += ct * (int32_t)q[b];
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) out[b] = from_fixed<T>(acc[b]);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        double acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0.0;
        for (int t = 0; t < taps; ++t) {
            int k = s + t;
            k = k < 0 ? 0 : (k > hi ? hi : k);
            const T* q = reinterpret_cast<const T*>(base + rowbase[k] + col_bytes);
            const double ct = c[t];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                if (MODE == kReduceF32Simd && ((lanes >> b) & 1u)) acc[b] = acc[b] + as_f64(q[b]) * ct;
                else acc[b] = fma(as_f64(q[b]), ct, acc[b]);
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) out[b] = from_f64<T>(acc[b]);
    }
}

// Walk the (row, column) pairs of a rows x cols grid, thread-strided.
template <typename F>
__device__ __forceinline__ void grid_walk(int rows, int cols, F&& f) {
    int r = threadIdx.x / cols, c = threadIdx.x - r * cols;
    const int dr = kCThreads / cols, dc = kCThreads - dr * cols;
    for (; r < rows;) {
        f(r, c);
        r += dr; c += dc;
        if (c >= cols) { c -= cols; ++r; }
    }
}

// Copy `bytes` (a multiple of 16, both pointers 16-byte aligned) global -> shared.
__device__ __forceinline__ void copy_table16(uint8_t* dst, const void* src, int bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (int i = threadIdx.x; i < bytes / 16; i += kCThreads) d[i] = s[i];
}

// Stage rows [0, nrows) of a source tile: row r is plane row row_of(r), columns
// [c0, c0 + ncols).  One warp per row: 16-byte loads for the aligned body, byte
// loads for the unaligned head and tail; the staged copy keeps the source's
// address modulo 16 so the vector stores stay aligned.
template <typename T, typename RowOf>
__device__ __forceinline__ void stage_tile_rows(const Plane& in, RowOf row_of, int nrows, int64_t c0, int ncols,
                                                int bands, uint8_t* dst_base, int pitch, int32_t* rowbase) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = kCThreads >> 5;
    const int nbytes = ncols * bands * int(sizeof(T));
    for (int r = warp; r < nrows; r += nw) {
        const uint8_t* src = in.data + row_of(r) * in.pitch + c0 * bands * int64_t(sizeof(T));
        const int off = int(reinterpret_cast<uintptr_t>(src) & 15);
        uint8_t* dst = dst_base + r * pitch + off;
        if (lane == 0) rowbase[r] = r * pitch + off;
        const int head = min((16 - off) & 15, nbytes);
        const int nvec = (nbytes - head) >> 4;
        const int tail0 = head + nvec * 16;
        if (lane < head) dst[lane] = __ldg(src + lane);
        if (lane < nbytes - tail0) dst[tail0 + lane] = __ldg(src + tail0 + lane);
        const uint4* vs = reinterpret_cast<const uint4*>(src + head);
        uint4* vd = reinterpret_cast<uint4*>(dst + head);
        for (int k = lane; k < nvec; k += 32) vd[k] = __ldg(vs + k);
    }
}

// NB: compile-time band count (0 = a.bands at run time), so that the
// per-sample index splits j -> (pixel, band) compile to multiply-shifts.
// Premultiply<U8> of the staged source tile (R rows of C pixels, alpha last).
__device__ __forceinline__ void premultiply_staged(uint8_t* ins, const int32_t* rowbase, int R, int C, int B) {
    int r = threadIdx.x / C, c = threadIdx.x - r * C;
    const int dr = kCThreads / C, dc = kCThreads - dr * C;
    for (; r < R;) {
        uint8_t* px = ins + rowbase[r] + c * B;
        const uint32_t al = px[B - 1];
        for (int b = 0; b < B - 1; ++b) px[b] = (uint8_t)premultiply_u8(px[b], al);
        r += dr; c += dc;
        if (c >= C) { c -= C; ++r; }
    }
}

template <typename T, int MH, int MV, int NB>
__device__ void reduce2d_tile(const Reduce2DArgs& a, int bx, int by, uint8_t* sm) {
    const Reduce2DLayout L = reduce2d_layout(a);
    const int B = NB > 0 ? NB : a.bands;
    const int tx0 = bx * a.tile_w, ty0 = by * a.tile_h;
    const int ncols = min(a.tile_w, a.out.w - tx0), nrows = min(a.tile_h, a.out.h - ty0);
    const uint8_t* ch = sm + L.coef_h;
    const uint8_t* cv = sm + L.coef_v;
    int32_t* sx = reinterpret_cast<int32_t*>(sm + L.tab);
    int32_t* sy = sx + a.tile_w;
    uint8_t* phx = reinterpret_cast<uint8_t*>(sy + a.tile_h);
    uint8_t* phy = phx + a.tile_w;
    int32_t* rowbase = reinterpret_cast<int32_t*>(sm + L.rowbase);
    uint8_t* ins = sm + L.in;
    T* mid = reinterpret_cast<T*>(sm + L.mid);
    T* ost = reinterpret_cast<T*>(sm + L.out);

    copy_table16(sm + L.coef_h, a.coeffs_h, r2_align16(L.coef_h_bytes));
    copy_table16(sm + L.coef_v, a.coeffs_v, r2_align16(L.coef_v_bytes));
    for (int i = threadIdx.x; i < ncols; i += kCThreads) { sx[i] = a.starts_h[tx0 + i]; phx[i] = a.phases_h[tx0 + i]; }
    for (int i = threadIdx.x; i < nrows; i += kCThreads) { sy[i] = a.starts_v[ty0 + i]; phy[i] = a.phases_v[ty0 + i]; }
    // tap spans of the tile (absolute coordinates of each op's input)
    const int64_t hs0 = a.starts_h[tx0], hs1 = (int64_t)a.starts_h[tx0 + ncols - 1] + a.taps_h - 1;
    const int64_t vs0 = a.starts_v[ty0], vs1 = (int64_t)a.starts_v[ty0 + nrows - 1] + a.taps_v - 1;
    const int64_t pw = a.in.w - 1, phh = a.in.h - 1;
    const bool premul = a.premul_in != 0;

    if (a.hfirst) {
        // mid rows [rlo, rhi]: the V taps clamped to the mid plane; each is the
        // H output of source row clamp(r - in.y0)
        const int64_t mlo = a.my0, mhi = a.my0 + a.mh - 1;
        const int64_t rlo = vs0 < mlo ? mlo : vs0, rhi = vs1 > mhi ? mhi : vs1;
        const int R = int(rhi - rlo + 1);
        const int64_t c0 = clampi64(hs0 - a.in.x0, 0, pw), c1 = clampi64(hs1 - a.in.x0, 0, pw);
        const int C = int(c1 - c0 + 1);
        stage_tile_rows<T>(a.in, [&](int r) { return clampi64(rlo + r - a.in.y0, 0, phh); }, R, c0, C, B, ins, L.pitch,
                           rowbase);
        csync();
        if (premul) {
            premultiply_staged(ins, rowbase, R, C, B);
            csync();
        }
        // H: mid[r][x*B + b]
        const int W1 = ncols * B;
        if constexpr (NB > 0) {
            // one thread per (mid row, pixel), all bands
            grid_walk(R, ncols, [&](int r, int x) {
                const T* row = reinterpret_cast<const T*>(ins + rowbase[r]);
                const int s = int(sx[x] - a.in.x0 - c0);
                fused_taps_px<T, MH, true, NB>(row, s, C - 1, NB, a.taps_h, ch, phx[x], 0u, mid + r * W1 + x * NB);
            });
        } else {
            int r = threadIdx.x / W1, j = threadIdx.x - r * W1;
            const int dr = kCThreads / W1, dj = kCThreads - dr * W1;
            for (; r < R;) {
                const int x = j / B, b = j - x * B;
                const T* row = reinterpret_cast<const T*>(ins + rowbase[r]) + b;
                const int s = int(sx[x] - a.in.x0 - c0);
                mid[r * W1 + j] = fused_taps<T, MH, true>(row, s, C - 1, B, a.taps_h, ch, phx[x], false);
                r += dr; j += dj;
                if (j >= W1) { j -= W1; ++r; }
            }
        }
        csync();
        // V: out[y][x*B + b]
        if constexpr (NB > 0) {
            grid_walk(nrows, ncols, [&](int y, int x) {
                const int s = int(sy[y] - rlo);
                uint32_t lanes = 0;
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    if ((int64_t)(tx0 + x) * NB + b < a.vector_len) lanes |= 1u << b;
                fused_taps_px<T, MV, false, NB>(mid + x * NB, s, R - 1, W1, a.taps_v, cv, phy[y], lanes,
                                                ost + y * W1 + x * NB);
            });
        } else {
            int y = threadIdx.x / W1, j = threadIdx.x - y * W1;
            const int dy = kCThreads / W1, dj = kCThreads - dy * W1;
            for (; y < nrows;) {
                const int s = int(sy[y] - rlo);
                const bool lane = (int64_t)tx0 * B + j < a.vector_len;
                ost[y * W1 + j] = fused_taps<T, MV, false>(mid + j, s, R - 1, W1, a.taps_v, cv, phy[y], lane);
                y += dy; j += dj;
                if (j >= W1) { j -= W1; ++y; }
            }
        }
    } else {
        // mid columns [clo, chi]: the H taps clamped to the mid plane; each is
        // the V output of source column clamp(c - in.x0)
        const int64_t mlo = a.mx0, mhi = a.mx0 + a.mw - 1;
        const int64_t clo = hs0 < mlo ? mlo : hs0, chi = hs1 > mhi ? mhi : hs1;
        const int Cm = int(chi - clo + 1);
        const int64_t c0 = clampi64(clo - a.in.x0, 0, pw), c1 = clampi64(chi - a.in.x0, 0, pw);
        const int C = int(c1 - c0 + 1);
        const int64_t r0 = clampi64(vs0 - a.in.y0, 0, phh), r1 = clampi64(vs1 - a.in.y0, 0, phh);
        const int R = int(r1 - r0 + 1);
        stage_tile_rows<T>(a.in, [&](int r) { return r0 + r; }, R, c0, C, B, ins, L.pitch, rowbase);
        csync();
        if (premul) {
            premultiply_staged(ins, rowbase, R, C, B);
            csync();
        }
        // V: mid[y][c*B + b]
        const int W1 = Cm * B;
        if constexpr (NB > 0) {
            grid_walk(nrows, Cm, [&](int y, int cc) {
                const int64_t mcol = clo + cc;
                const int col = int(clampi64(mcol - a.in.x0, 0, pw) - c0);
                const int s = int(sy[y] - a.in.y0 - r0);
                uint32_t lanes = 0;
#pragma unroll
                for (int b = 0; b < NB; ++b)
                    if ((mcol - a.mx0) * NB + b < a.vector_len) lanes |= 1u << b;
                fused_taps_rows_px<T, MV, NB>(ins, rowbase, col * NB * int(sizeof(T)), s, R - 1, a.taps_v, cv, phy[y],
                                              lanes, mid + y * W1 + cc * NB);
            });
        } else {
            int y = threadIdx.x / W1, j = threadIdx.x - y * W1;
            const int dy = kCThreads / W1, dj = kCThreads - dy * W1;
            for (; y < nrows;) {
                const int c = j / B, b = j - c * B;
                const int64_t mcol = clo + c;
                const int col = int(clampi64(mcol - a.in.x0, 0, pw) - c0);
                const int s = int(sy[y] - a.in.y0 - r0);
                const bool lane = (mcol - a.mx0) * B + b < a.vector_len;
                mid[y * W1 + j] = fused_taps_rows<T, MV>(ins, rowbase, (col * B + b) * int(sizeof(T)), s, R - 1,
                                                         a.taps_v, cv, phy[y], lane);
                y += dy; j += dj;
                if (j >= W1) { j -= W1; ++y; }
            }
        }
        csync();
        // H: out[y][x*B + b]
        const int W2 = ncols * B;
        if constexpr (NB > 0) {
            grid_walk(nrows, ncols, [&](int y, int x) {
                const int s = int(sx[x] - clo);
                fused_taps_px<T, MH, true, NB>(mid + y * W1, s, Cm - 1, NB, a.taps_h, ch, phx[x], 0u,
                                               ost + y * W2 + x * NB);
            });
        } else {
            int y = threadIdx.x / W2, j = threadIdx.x - y * W2;
            const int dy = kCThreads / W2, dj = kCThreads - dy * W2;
            for (; y < nrows;) {
                const int x = j / B, b = j - x * B;
                const int s = int(sx[x] - clo);
                ost[y * W2 + j] = fused_taps<T, MH, true>(mid + y * W1 + b, s, Cm - 1, B, a.taps_h, ch, phx[x], false);
                y += dy; j += dj;
                if (j >= W2) { j -= W2; ++y; }
            }
        }
    }
    csync();
    // store the output tile (unpremultiplied when the chain ends with it)
    const int Wo = ncols * B;
    const bool unpremul = a.unpremul_out != 0;
    int y = threadIdx.x / Wo, j = threadIdx.x - y * Wo;
    const int dy = kCThreads / Wo, dj = kCThreads - dy * Wo;
    for (; y < nrows;) {
        const int i = y * Wo + j;
        T v = ost[i];
        if (unpremul) {
            const int b = j % B;
            if (b != B - 1) v = (T)unpremultiply_u8((uint32_t)v, (uint32_t)ost[i + (B - 1 - b)]);
        }
        reinterpret_cast<T*>(a.out.data + (int64_t)(ty0 + y) * a.out.pitch)[(int64_t)tx0 * B + j] = v;
        y += dy; j += dj;
        if (j >= Wo) { j -= Wo; ++y; }
    }
}

template <typename T, int MH, int MV, int NB>
__global__ void __launch_bounds__(256) reduce2d_kernel(Reduce2DArgs a) {
    extern __shared__ __align__(16) uint8_t smem_r2[];
    reduce2d_tile<T, MH, MV, NB>(a, blockIdx.x, blockIdx.y, smem_r2);
}

// ---------------------------------------------------------------- pixel ops
template <typename T>
__global__ void pixel_kernel(PixelArgs a) {
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    const int bands = a.bands;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += (int64_t)gridDim.x * blockDim.x) {
        // the input plane of a pixel-local op or an ExtractArea starts at the
        // pixel that maps to the output's first pixel: local coordinates agree
        const int64_t y = p / a.out.w, x = p - y * a.out.w;
        const T* src = reinterpret_cast<const T*>(a.in.data + y * a.in.pitch) + x * bands;
        T* dst = reinterpret_cast<T*>(a.out.data + y * a.out.pitch) + x * bands;
        if (a.op == 0 || bands < 2) {
            for (int b = 0; b < bands; ++b) dst[b] = src[b];
        } else if (sizeof(T) == 1) {
            const uint32_t al = (uint32_t)src[bands - 1];
            for (int b = 0; b < bands - 1; ++b)
                dst[b] = (T)(a.op == 1 ? premultiply_u8((uint32_t)src[b], al) : unpremultiply_u8((uint32_t)src[b], al));
            dst[bands - 1] = src[bands - 1];
        } else if (sizeof(T) == 4 && a.op == 2) {
            // Unpremultiply<F32> (structural/unpremultiply.rs:137-170)
            const float al = (float)src[bands - 1];
            for (int b = 0; b < bands - 1; ++b) {
                float v = 0.0f;
                if (al > 0.0f) {
                    v = __fmul_rn((float)src[b], __frcp_rn(al));
                    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
                }
                dst[b] = (T)v;
            }
            dst[bands - 1] = src[bands - 1];
        } else {
            for (int b = 0; b < bands; ++b) dst[b] = src[b];
        }
    }
}

// Zoom: integer nearest-neighbour upscale (structural/zoom.rs:44-104): output
// (x, y) repeats source (x / zx, y / zy).  blockIdx.y walks output rows; each
// thread fills one 16-byte-aligned chunk of the row with a vector store,
// gathering its elements from the source row (L1-resident: a source row is
// read by zy output rows and each source pixel by zx output pixels) with the
// pixel and repeat counters stepped instead of divided.  The elements before
// the row's first 16-byte boundary and after its last are written singly.
template <typename T>
__global__ void __launch_bounds__(256) zoom_kernel(PixelArgs a) {
    constexpr int V = 16 / (int)sizeof(T);
    const int bands = a.bands;
    const int64_t n = (int64_t)a.out.w * bands;
    const int64_t zx = a.zx;
    for (int64_t y = blockIdx.y; y < a.out.h; y += gridDim.y) {
        const int64_t sy = (a.out.y0 + y) / a.zy - a.in.y0;
        const T* src = reinterpret_cast<const T*>(a.in.data + sy * a.in.pitch);
        T* dst = reinterpret_cast<T*>(a.out.data + y * a.out.pitch);
        const int64_t mis = (int64_t)(reinterpret_cast<uintptr_t>(dst) & 15);
        // a row not aligned to its element size never reaches a 16-byte
        // boundary at an element: all of it is written singly
        const int64_t head = mis % (int64_t)sizeof(T) ? n : (mis ? min(n, (16 - mis) / (int64_t)sizeof(T)) : 0);
        const int64_t chunks = (n - head) / V;
        const int64_t tail = head + chunks * V;
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < chunks; c += stride) {
            const int64_t e0 = head + c * V;
            const int64_t x = e0 / bands;
            int b = (int)(e0 - x * bands);
            const int64_t gx = a.out.x0 + x;
            int64_t q = gx / zx;
            int64_t r = gx - q * zx;
            union { T t[V]; uint4 u; } pk;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                pk.t[k] = src[(q - a.in.x0) * bands + b];
                if (++b == bands) {
                    b = 0;
                    if (++r == zx) { r = 0; ++q; }
                }
            }
            *reinterpret_cast<uint4*>(dst + e0) = pk.u;
        }
        const int64_t singles = head + (n - tail);
        for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < singles; t += stride) {
            const int64_t e = t < head ? t : tail + (t - head);
            const int64_t x = e / bands;
            const int b = (int)(e - x * bands);
            dst[e] = src[((a.out.x0 + x) / zx - a.in.x0) * bands + b];
        }
    }
}

// Zoom for destinations whose rows share their 16-byte phase (pitch a
// multiple of 16) and at most kZoomMaxBands bands.  blockIdx.y walks SOURCE
// rows: the zy output rows that repeat one source row are identical, so each
// 16-byte chunk is gathered once and stored to all of them.  A block takes
// kZoomChunks chunks of the row at a time (kZoomChunks / 256 per thread,
// strided so that a warp's stores are contiguous), stages the source span
// they read in shared memory with 4-byte loads (the span's first and last
// words may reach up to 3 bytes past it: a word never crosses a page), and
// gathers from there.
constexpr int kZoomMaxBands = 64;
constexpr int kZoomPerThread = 4;
constexpr int kZoomChunks = 256 * kZoomPerThread;
// span bytes: kZoomChunks 16-byte chunks read at most kZoomChunks * 16 - 1 + 3
// pixels' worth of sample bytes beyond them, plus 3 bytes of word alignment
constexpr int kZoomSpanWords = (kZoomChunks * 16 + 3 * kZoomMaxBands * 4 + 8) / 4;

template <typename T>
__global__ void __launch_bounds__(256) zoom_rows_kernel(PixelArgs a) {
    constexpr int V = 16 / (int)sizeof(T);
    __shared__ __align__(16) uint32_t span[kZoomSpanWords];
    const uint8_t* span_b = reinterpret_cast<const uint8_t*>(span);
    const int bands = a.bands;
    const int64_t n = (int64_t)a.out.w * bands;
    const int64_t zx = a.zx, zy = a.zy;
    const int64_t mis = (int64_t)(reinterpret_cast<uintptr_t>(a.out.data) & 15);
    const int64_t head = mis % (int64_t)sizeof(T) ? n : (mis ? min(n, (16 - mis) / (int64_t)sizeof(T)) : 0);
    const int64_t chunks = (n - head) / V;
    const int64_t tail = head + chunks * V;
    for (int64_t r = blockIdx.y; r < a.in.h; r += gridDim.y) {
        const int64_t gsy = a.in.y0 + r;
        const int64_t y_lo = max(gsy * zy - a.out.y0, (int64_t)0);
        const int64_t y_hi = min((gsy + 1) * zy - a.out.y0, (int64_t)a.out.h);
        if (y_lo >= y_hi) continue;  // the same for the whole block
        const T* src = reinterpret_cast<const T*>(a.in.data + r * a.in.pitch);
        for (int64_t c0 = (int64_t)blockIdx.x * kZoomChunks; c0 < chunks; c0 += (int64_t)gridDim.x * kZoomChunks) {
            const int64_t c1 = min(chunks, c0 + kZoomChunks);
            const int64_t e_first = head + c0 * V, e_last = head + c1 * V - 1;
            const int64_t p_first = (a.out.x0 + e_first / bands) / zx - a.in.x0;
            const int64_t p_last = (a.out.x0 + e_last / bands) / zx - a.in.x0;
            const uint8_t* sb = reinterpret_cast<const uint8_t*>(src + p_first * bands);
            const uint8_t* se = reinterpret_cast<const uint8_t*>(src + (p_last + 1) * bands);
            const uint32_t* w0 = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(sb) & ~(uintptr_t)3);
            const int delta = (int)(sb - reinterpret_cast<const uint8_t*>(w0));
            const int nw = (int)((se - reinterpret_cast<const uint8_t*>(w0) + 3) >> 2);
            __syncthreads();  // the previous span's readers are done
            for (int i = threadIdx.x; i < nw; i += blockDim.x) span[i] = __ldg(w0 + i);
            __syncthreads();
#pragma unroll
            for (int k = 0; k < kZoomPerThread; ++k) {
                const int64_t c = c0 + threadIdx.x + 256 * k;
                if (c >= c1) break;
                const int64_t e0 = head + c * V;
                const int64_t x = e0 / bands;
                int b = (int)(e0 - x * bands);
                const int64_t gx = a.out.x0 + x;
                const int64_t q = gx / zx;
                int64_t rem = gx - q * zx;
                int si = (int)((q - a.in.x0 - p_first) * bands) + b;
                union { T t[V]; uint4 u; } pk;
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    pk.t[j] = *reinterpret_cast<const T*>(span_b + delta + si * (int)sizeof(T));
                    ++si;
                    if (++b == bands) {
                        b = 0;
                        if (++rem == zx) rem = 0;  // next source pixel: si already points at it
                        else si -= bands;          // the same source pixel again
                    }
                }
                for (int64_t y = y_lo; y < y_hi; ++y)
                    *reinterpret_cast<uint4*>(reinterpret_cast<T*>(a.out.data + y * a.out.pitch) + e0) = pk.u;
            }
        }
        const int64_t singles = head + (n - tail);
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < singles; t += stride) {
            const int64_t e = t < head ? t : tail + (t - head);
            const int64_t x = e / bands;
            const int b = (int)(e - x * bands);
            const T v = src[((a.out.x0 + x) / zx - a.in.x0) * bands + b];
            for (int64_t y = y_lo; y < y_hi; ++y) reinterpret_cast<T*>(a.out.data + y * a.out.pitch)[e] = v;
        }
    }
}

}  // namespace dev
}  // namespace viprs
