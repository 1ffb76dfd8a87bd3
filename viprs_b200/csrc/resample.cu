// resample.cu -- sm_100a kernels for the box shrink and separable reduce ops
// of viprs's resample path, with their launch wrappers.
//
//   shrink2d_kernel ..... ShrinkH / ShrinkV / Shrink (resample/shrinkh.rs:255-874,
//                         shrinkv.rs:153-537, shrink.rs:179-293), premultiply fused
//                         into the source read, unpremultiply into the store
//   reduce_h_kernel ..... ReduceH (reduceh.rs:100-163; reduce_simd.rs:179-231,
//                         2421-2538 for u8, 2544-2615 u16, 2621-2694 f32) and the
//                         horizontal half of ReduceOp (reduce.rs:103-135)
//   reduce_v_kernel ..... ReduceV (reducev.rs:99-162; reduce_simd.rs:2700-2888) and
//                         the vertical half of ReduceOp (reduce.rs:137-170)
//   pixel_kernel ........ Premultiply / Unpremultiply / ExtractArea copies
//
// Memory traffic: the shrink reads every source sample exactly once with
// 16-byte loads into shared memory (coalesced across the block) and writes
// each output once; it is HBM-bound.  The reduce kernels gather taps from
// the (L2-resident) shrunk plane with coefficient tables in shared memory.
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "tma.cuh"
#include "viprs_b200.h"

namespace viprs {
namespace dev {

constexpr int kShrinkThreads = 256;
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
__device__ const T* stage_row(const Plane& in, int64_t ly, int64_t c0, int nin, int bands,
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
__device__ void premultiply_staged(uint8_t* seg, int nin, int bands) {
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

// Box sums of one output pixel's fh source pixels (B bands, u8) from shared
// memory at any byte alignment: words are realigned with a funnel shift and
// the bands are summed four bytes at a time with dp4a masks.  The word after
// the box is read (the stage buffers carry 32 bytes of slack) but masked out.
template <int B>
__device__ __forceinline__ void box_sums_u8(const uint8_t* p, int fh, uint32_t (&sums)[B]) {
    const int o = int(reinterpret_cast<uintptr_t>(p) & 3);
    const uint32_t* wp = reinterpret_cast<const uint32_t*>(p - o);
    const int nbytes = fh * B;
    const int K = (nbytes + 3) >> 2;
    const uint32_t sh = 8u * uint32_t(o);
    const uint32_t tail_mask = (nbytes & 3) ? ((1u << (8 * (nbytes & 3))) - 1u) : 0xFFFFFFFFu;
#pragma unroll
    for (int b = 0; b < B; ++b) sums[b] = 0;
    auto word = [&](int k) {
        uint32_t w = __funnelshift_r(wp[k], wp[k + 1], sh);
        return k == K - 1 ? (w & tail_mask) : w;
    };
    if (B == 1) {
        for (int k = 0; k < K; ++k) sums[0] = __dp4a(word(k), 0x01010101u, sums[0]);
    } else if (B == 2) {
        for (int k = 0; k < K; ++k) {
            const uint32_t w = word(k);
            sums[0] = __dp4a(w, 0x00010001u, sums[0]);
            sums[B > 1 ? 1 : 0] = __dp4a(w, 0x01000100u, sums[B > 1 ? 1 : 0]);
        }
    } else if (B == 3) {
        // byte j of the realigned stream is band j % 3: masks repeat every 3 words
        int k = 0;
        for (; k + 3 <= K; k += 3) {
            const uint32_t w0 = word(k), w1 = word(k + 1), w2 = word(k + 2);
            sums[0] = __dp4a(w0, 0x01000001u, sums[0]);
            sums[1 % B] = __dp4a(w0, 0x00000100u, sums[1 % B]);
            sums[2 % B] = __dp4a(w0, 0x00010000u, sums[2 % B]);
            sums[0] = __dp4a(w1, 0x00010000u, sums[0]);
            sums[1 % B] = __dp4a(w1, 0x01000001u, sums[1 % B]);
            sums[2 % B] = __dp4a(w1, 0x00000100u, sums[2 % B]);
            sums[0] = __dp4a(w2, 0x00000100u, sums[0]);
            sums[1 % B] = __dp4a(w2, 0x00010000u, sums[1 % B]);
            sums[2 % B] = __dp4a(w2, 0x01000001u, sums[2 % B]);
        }
        if (k < K) {
            const uint32_t w0 = word(k);
            sums[0] = __dp4a(w0, 0x01000001u, sums[0]);
            sums[1 % B] = __dp4a(w0, 0x00000100u, sums[1 % B]);
            sums[2 % B] = __dp4a(w0, 0x00010000u, sums[2 % B]);
        }
        if (k + 1 < K) {
            const uint32_t w1 = word(k + 1);
            sums[0] = __dp4a(w1, 0x00010000u, sums[0]);
            sums[1 % B] = __dp4a(w1, 0x01000001u, sums[1 % B]);
            sums[2 % B] = __dp4a(w1, 0x00000100u, sums[2 % B]);
        }
    } else {
        for (int k = 0; k < K; ++k) {
            const uint32_t w = word(k);
#pragma unroll
            for (int b = 0; b < B; ++b) sums[b] = __dp4a(w, 1u << (8 * b), sums[b]);
        }
    }
}

// Premultiply<U8> in place over `npx` staged pixels of B bands (alpha last).
template <int B>
__device__ __forceinline__ void premultiply_pixels(uint8_t* seg, int npx) {
    for (int p = threadIdx.x; p < npx; p += blockDim.x) {
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
    for (int32_t i = threadIdx.x; i < fv * per_row; i += blockDim.x) {
        const int32_t k = i / per_row, rem = i - k * per_row;
        const int32_t xb = rem / B, b = rem - xb * B;
        const int64_t sx = (a.out.x0 + c0) * (int64_t)fh + xb - a.in.x0;
        buf[i] = load_sample<uint8_t>(a.in, sx, Y * fv + k - a.in.y0, B, b);
    }
    __syncthreads();
    if (a.premul_in) {
        premultiply_pixels<B>(buf, fv * ncols * fh);
        __syncthreads();
    }
    uint8_t* ob = buf + fv * per_row;
    for (int32_t item = threadIdx.x; item < ncols * B; item += blockDim.x) {
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
    __syncthreads();
    uint8_t* orow = a.out.data + (int64_t)oy * a.out.pitch + (int64_t)c0 * B;
    for (int32_t item = threadIdx.x; item < ncols * B; item += blockDim.x) {
        const int32_t x = item / B, b = item - x * B;
        uint32_t v = ob[item];
        if (a.unpremul_out && b != B - 1) v = unpremultiply_u8(v, ob[x * B + B - 1]);
        orow[item] = (uint8_t)v;
    }
    __syncthreads();
}

// ShrinkH then ShrinkV over u8.  Items are (output row, column chunk) of the
// interior columns; a block owns every G-th item.  One thread per block fetches
// each source row segment of its items with a TMA bulk copy into a ring of S
// shared-memory buffers (the ring runs across item boundaries), so S rows are
// in flight while the block sums the current one; each thread owns one output
// pixel of the chunk and accumulates its B band sums over the fv rows.
// Every source byte is read from HBM once.  B is the band count (1..4).
template <int B>
__global__ void __launch_bounds__(kShrinkThreads) shrink_hv_u8_tma(ShrinkArgs a) {
    extern __shared__ __align__(128) uint8_t smem_tma[];
    uint8_t* smem = smem_tma;
    constexpr int S = 4;  // ring depth (power of two)
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    volatile int32_t* flag = reinterpret_cast<volatile int32_t*>(smem + 64);
    uint8_t* bufs = smem + 128;
    uint8_t* ostage = bufs + (size_t)S * a.stage_bytes;
    const int32_t fh = int32_t(a.fh), fv = int32_t(a.fv);
    const int32_t chunks = a.chunks;
    const int32_t G = gridDim.x;

    // edge columns first: small, clamped reads
    {
        const int32_t nl = a.col_lo > 0 ? a.out.h : 0, nr = a.col_hi < a.out.w ? a.out.h : 0;
        for (int32_t e = blockIdx.x; e < nl + nr; e += G) {
            if (e < nl) shrink_edge_item_u8<B>(a, e, 0, a.col_lo, bufs);
            else shrink_edge_item_u8<B>(a, e - nl, a.col_hi, a.out.w, bufs);
        }
    }

    const int32_t n_items = a.out.h * chunks;
    if ((int32_t)blockIdx.x >= n_items) return;
    const int32_t n_my = (n_items - 1 - (int32_t)blockIdx.x) / G + 1;
    const int64_t total = (int64_t)n_my * fv;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) mbar_init(&bars[i], 1);
        *flag = 0;
        mbar_fence_init();
    }
    __syncthreads();

    // per-item geometry: source byte offset of the chunk within a row and its length
    struct ItemGeom { int32_t oy, lx0, ncols; int64_t sbase, row0; int32_t nbytes; };
    auto item_geom = [&](int32_t item) {
        ItemGeom g;
        g.oy = item / chunks;
        const int32_t c = item - g.oy * chunks;
        g.lx0 = a.col_lo + c * a.nxf;
        g.ncols = min(a.nxf, a.col_hi - g.lx0);
        g.sbase = ((a.out.x0 + g.lx0) * (int64_t)fh - a.in.x0) * B;
        g.row0 = (a.out.y0 + g.oy) * (int64_t)fv - a.in.y0;
        g.nbytes = g.ncols * fh * B;
        return g;
    };
    auto row_span = [&](const ItemGeom& g, int32_t k, int64_t* as, uint32_t* bytes, int32_t* lead) {
        int64_t ly = g.row0 + k;
        ly = ly < 0 ? 0 : (ly >= a.in.h ? a.in.h - 1 : ly);
        const int64_t s0 = ly * a.in.pitch + g.sbase;
        *as = s0 & ~int64_t(15);
        *bytes = uint32_t(((s0 + g.nbytes + 15) & ~int64_t(15)) - *as);
        *lead = int32_t(s0 - *as);
    };

    // producer state (thread 0)
    int32_t p_item = blockIdx.x, p_k = 0;
    ItemGeom pg = item_geom(p_item);
    int64_t issued = 0;
    auto issue = [&]() {
        int64_t as; uint32_t bytes; int32_t lead;
        row_span(pg, p_k, &as, &bytes, &lead);
        const int st = int(issued & (S - 1));
        mbar_arrive_expect_tx(&bars[st], bytes);
        bulk_load(bufs + (size_t)st * a.stage_bytes, a.in.data + as, bytes, &bars[st]);
        ++issued;
        if (++p_k == fv) {
            p_k = 0;
            p_item += G;
            if (p_item < n_items) pg = item_geom(p_item);
        }
    };
    if (threadIdx.x == 0) {
        const int64_t first = total < S ? total : (int64_t)S;
        for (int64_t t = 0; t < first; ++t) issue();
    }

    int32_t c_item = blockIdx.x, c_k = 0;
    ItemGeom cg = item_geom(c_item);
    uint32_t vacc[B];
#pragma unroll
    for (int b = 0; b < B; ++b) vacc[b] = 0;
    int64_t t_fail = -1;
    const int32_t x = threadIdx.x;  // this thread's output pixel within the chunk (nxf <= blockDim)
    for (int64_t t = 0; t < total; ++t) {
        const int st = int(t & (S - 1));
        const uint32_t parity = uint32_t((t / S) & 1);
        if (threadIdx.x == 0 && !mbar_wait(&bars[st], parity)) *flag = 1;
        __syncthreads();
        if (*flag) { t_fail = t; break; }
        int64_t as; uint32_t bytes; int32_t lead;
        row_span(cg, c_k, &as, &bytes, &lead);
        uint8_t* row = bufs + (size_t)st * a.stage_bytes + lead;
        if (a.premul_in) {
            premultiply_pixels<B>(row, cg.ncols * fh);
            __syncthreads();
        }
        if (x < cg.ncols) {
            uint32_t sums[B];
            box_sums_u8<B>(row + x * fh * B, fh, sums);
#pragma unroll
            for (int b = 0; b < B; ++b) vacc[b] += round_mode_u8(sums[b], a.hmode, uint32_t(fh), a.hmult);
        }
        __syncthreads();  // all reads of this buffer are done
        if (threadIdx.x == 0 && issued < total) {
            fence_proxy_async_smem();
            issue();
        }
        if (++c_k == fv) {
            uint8_t o[B];
#pragma unroll
            for (int b = 0; b < B; ++b) o[b] = (uint8_t)round_mode_u8(vacc[b], a.vmode, uint32_t(fv), a.vmult);
            if (a.unpremul_out) {
#pragma unroll
                for (int b = 0; b < B - 1; ++b) o[b] = (uint8_t)unpremultiply_u8(o[b], o[B - 1]);
            }
            if (x < cg.ncols) {
                uint8_t* dst = a.out.data + (int64_t)cg.oy * a.out.pitch + (int64_t)(cg.lx0 + x) * B;
#pragma unroll
                for (int b = 0; b < B; ++b) dst[b] = o[b];
            }
#pragma unroll
            for (int b = 0; b < B; ++b) vacc[b] = 0;
            c_k = 0;
            c_item += G;
            if (c_item < n_items) cg = item_geom(c_item);
        }
    }
    (void)ostage;
    if (t_fail >= 0) {
        // a copy never completed: record it, then wait (bounded) for the copies
        // this block still has in flight before its shared memory goes away
        if (threadIdx.x == 0) {
            if (a.err) atomicExch(a.err, VIPRS_ERR_TIMEOUT);
            for (int64_t tt = t_fail + 1; tt < issued; ++tt) mbar_wait(&bars[tt & (S - 1)], uint32_t((tt / S) & 1));
        }
        __syncthreads();
    }
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
    __syncthreads();
    if (item < nitems) {
        const int b = int(item % bands);
        uint32_t o = stage[local];
        if (b != bands - 1) o = unpremultiply_u8(o, stage[local + (bands - 1 - b)]);
        orow[item] = (uint8_t)o;
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256) reduce_h_kernel(ReduceArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int taps = a.taps, bands = a.bands;
    const int coef_bytes = 65 * taps * (MODE == kReduceFixed ? 2 : 8);
    const bool coef_in_smem = coef_bytes <= 48 * 1024;
    const uint8_t* coef = reinterpret_cast<const uint8_t*>(a.coeffs);
    if (coef_in_smem) {
        for (int i = threadIdx.x * 4; i < coef_bytes; i += blockDim.x * 4)
            *reinterpret_cast<uint32_t*>(smem + i) = *reinterpret_cast<const uint32_t*>(coef + i);
        __syncthreads();
        coef = smem;
    }
    uint8_t* stage = smem + ((coef_in_smem ? coef_bytes : 0) + 15) / 16 * 16;
    const int nitems = a.out.w * bands;
    const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t oy = blockIdx.y;
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
__global__ void __launch_bounds__(256) reduce_v_kernel(ReduceArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int taps = a.taps, bands = a.bands;
    const int coef_bytes = 65 * taps * (MODE == kReduceFixed ? 2 : 8);
    const bool coef_in_smem = coef_bytes <= 48 * 1024;
    const uint8_t* coef = reinterpret_cast<const uint8_t*>(a.coeffs);
    if (coef_in_smem) {
        for (int i = threadIdx.x * 4; i < coef_bytes; i += blockDim.x * 4)
            *reinterpret_cast<uint32_t*>(smem + i) = *reinterpret_cast<const uint32_t*>(coef + i);
        __syncthreads();
        coef = smem;
    }
    uint8_t* stage = smem + ((coef_in_smem ? coef_bytes : 0) + 15) / 16 * 16;
    const int nitems = a.out.w * bands;
    const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t oy = blockIdx.y;
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

// ---------------------------------------------------------------- fused reduce

template <typename T, int MODE>
__device__ __forceinline__ T reduce_taps_global(const Plane& in, int64_t lx, int64_t ly, bool horizontal,
                                                int64_t start_local, int taps, int bands, int b,
                                                const uint8_t* coef, int ph, bool premul, bool simd_lane) {
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc = 0;
        for (int t = 0; t < taps; ++t) {
            const int64_t x = horizontal ? start_local + t : lx, y = horizontal ? ly : start_local + t;
            acc += (int32_t)c[t] * (int32_t)load_premul<T>(in, x, y, bands, b, premul);
        }
        return from_fixed<T>(acc);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        double acc = 0.0;
        if (MODE == kReduceF32Simd && horizontal) {
            int t = 0;
            for (; t + 4 <= taps; t += 4) {
                double lanes = as_f64(load_sample<T>(in, start_local + t, ly, bands, b)) * c[t];
                lanes = lanes + as_f64(load_sample<T>(in, start_local + t + 1, ly, bands, b)) * c[t + 1];
                lanes = lanes + as_f64(load_sample<T>(in, start_local + t + 2, ly, bands, b)) * c[t + 2];
                lanes = lanes + as_f64(load_sample<T>(in, start_local + t + 3, ly, bands, b)) * c[t + 3];
                acc = acc + lanes;
            }
            for (; t < taps; ++t) acc = fma(as_f64(load_sample<T>(in, start_local + t, ly, bands, b)), c[t], acc);
        } else if (MODE == kReduceF32Simd && simd_lane) {
            for (int t = 0; t < taps; ++t) acc = acc + as_f64(load_sample<T>(in, lx, start_local + t, bands, b)) * c[t];
        } else {
            for (int t = 0; t < taps; ++t) {
                const int64_t x = horizontal ? start_local + t : lx, y = horizontal ? ly : start_local + t;
                acc = fma(as_f64(load_sample<T>(in, x, y, bands, b)), c[t], acc);
            }
        }
        return from_f64<T>(acc);
    }
}

// Second pass over the shared-memory mid tile `m` (row stride `mstride` samples).
template <typename T, int MODE>
__device__ __forceinline__ T reduce_taps_smem(const T* m, int64_t first, int64_t lo, int64_t hi, int64_t origin,
                                              int64_t stride, int taps, const uint8_t* coef, int ph, bool horizontal,
                                              bool simd_lane) {
    // tap i reads mid index clamp(first + i, lo, hi) - origin along the pass axis
    if (MODE == kReduceFixed) {
        const int16_t* c = reinterpret_cast<const int16_t*>(coef) + ph * taps;
        int32_t acc = 0;
        for (int t = 0; t < taps; ++t) {
            int64_t q = first + t;
            q = q < lo ? lo : (q > hi ? hi : q);
            acc += (int32_t)c[t] * (int32_t)m[(q - origin) * stride];
        }
        return from_fixed<T>(acc);
    } else {
        const double* c = reinterpret_cast<const double*>(coef) + ph * taps;
        double acc = 0.0;
        auto val = [&](int t) {
            int64_t q = first + t;
            q = q < lo ? lo : (q > hi ? hi : q);
            return as_f64(m[(q - origin) * stride]);
        };
        if (MODE == kReduceF32Simd && horizontal) {
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

// One block: an output tile of tile_h rows x tile_w columns.
template <typename T, int MH, int MV>
__global__ void __launch_bounds__(256) reduce2d_kernel(Reduce2DArgs a) {
    extern __shared__ __align__(16) uint8_t smem_r2[];
    const int bands = a.bands;
    const int ch_bytes = 65 * a.taps_h * (MH == kReduceFixed ? 2 : 8);
    const int cv_bytes = 65 * a.taps_v * (MV == kReduceFixed ? 2 : 8);
    const int chp = (ch_bytes + 15) / 16 * 16, cvp = (cv_bytes + 15) / 16 * 16;
    uint8_t* ch = smem_r2;
    uint8_t* cv = smem_r2 + chp;
    for (int i = threadIdx.x * 4; i < ch_bytes; i += blockDim.x * 4)
        *reinterpret_cast<uint32_t*>(ch + i) = *reinterpret_cast<const uint32_t*>((const uint8_t*)a.coeffs_h + i);
    for (int i = threadIdx.x * 4; i < cv_bytes; i += blockDim.x * 4)
        *reinterpret_cast<uint32_t*>(cv + i) = *reinterpret_cast<const uint32_t*>((const uint8_t*)a.coeffs_v + i);
    T* mid = reinterpret_cast<T*>(smem_r2 + chp + cvp);
    const int tx0 = blockIdx.x * a.tile_w, ty0 = blockIdx.y * a.tile_h;
    const int ncols = min(a.tile_w, a.out.w - tx0), nrows = min(a.tile_h, a.out.h - ty0);
    uint8_t* stage = reinterpret_cast<uint8_t*>(mid) + (size_t)a.span_max * (a.hfirst ? ncols : nrows) * bands * sizeof(T);
    stage = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(stage) + 15) & ~uintptr_t(15));
    __syncthreads();
    const bool premul = a.premul_in != 0;
    if (a.hfirst) {
        // rows of the mid plane this tile's vertical taps read
        int64_t rlo = a.starts_v[ty0], rhi = (int64_t)a.starts_v[ty0 + nrows - 1] + a.taps_v - 1;
        const int64_t mlo = a.my0, mhi = a.my0 + a.mh - 1;
        rlo = rlo < mlo ? mlo : rlo;
        rhi = rhi > mhi ? mhi : rhi;
        const int R = int(rhi - rlo + 1);
        const int per_row = ncols * bands;
        for (int i = threadIdx.x; i < R * per_row; i += blockDim.x) {
            const int r = i / per_row, rem = i - r * per_row, x = rem / bands, b = rem - x * bands;
            const int64_t ly = rlo + r - a.in.y0;
            const int col = tx0 + x;
            mid[i] = reduce_taps_global<T, MH>(a.in, 0, ly, true, (int64_t)a.starts_h[col] - a.in.x0, a.taps_h, bands,
                                               b, ch, a.phases_h[col], premul, false);
        }
        __syncthreads();
        const int n_out = nrows * per_row;
        for (int base = 0; base < n_out; base += blockDim.x) {
            const int i = base + threadIdx.x;
            T v = T(0);
            if (i < n_out) {
                const int yy = i / per_row, rem = i - yy * per_row, x = rem / bands, b = rem - x * bands;
                const int y = ty0 + yy;
                const int64_t vidx = (int64_t)(tx0 + x) * bands + b;
                v = reduce_taps_smem<T, MV>(mid + x * bands + b, a.starts_v[y], mlo, mhi, rlo, per_row, a.taps_v, cv,
                                            a.phases_v[y], false, vidx < a.vector_len);
            }
            const int yy = i / per_row;
            uint8_t* orow = a.out.data + (int64_t)(ty0 + (i < n_out ? yy : 0)) * a.out.pitch;
            const int64_t col_item = (int64_t)tx0 * bands + (i - yy * per_row);
            if (a.unpremul_out) {
                stage[threadIdx.x] = (uint8_t)v;
                __syncthreads();
                if (i < n_out) {
                    const int b = int(col_item % bands);
                    uint32_t o = stage[threadIdx.x];
                    if (b != bands - 1) o = unpremultiply_u8(o, stage[threadIdx.x + (bands - 1 - b)]);
                    orow[col_item] = (uint8_t)o;
                }
                __syncthreads();
            } else if (i < n_out) {
                reinterpret_cast<T*>(orow)[col_item] = v;
            }
        }
    } else {
        // columns of the mid plane this tile's horizontal taps read
        int64_t clo = a.starts_h[tx0], chi = (int64_t)a.starts_h[tx0 + ncols - 1] + a.taps_h - 1;
        const int64_t mlo = a.mx0, mhi = a.mx0 + a.mw - 1;
        clo = clo < mlo ? mlo : clo;
        chi = chi > mhi ? mhi : chi;
        const int C = int(chi - clo + 1);
        const int per_row = C * bands;
        for (int i = threadIdx.x; i < nrows * per_row; i += blockDim.x) {
            const int yy = i / per_row, rem = i - yy * per_row, c = rem / bands, b = rem - c * bands;
            const int y = ty0 + yy;
            const int64_t mcol = clo + c;
            const int64_t vidx = (mcol - a.mx0) * bands + b;
            mid[i] = reduce_taps_global<T, MV>(a.in, mcol - a.in.x0, 0, false, (int64_t)a.starts_v[y] - a.in.y0, a.taps_v,
                                               bands, b, cv, a.phases_v[y], premul, vidx < a.vector_len);
        }
        __syncthreads();
        const int per_out = ncols * bands;
        const int n_out = nrows * per_out;
        for (int base = 0; base < n_out; base += blockDim.x) {
            const int i = base + threadIdx.x;
            T v = T(0);
            if (i < n_out) {
                const int yy = i / per_out, rem = i - yy * per_out, x = rem / bands, b = rem - x * bands;
                const int col = tx0 + x;
                v = reduce_taps_smem<T, MH>(mid + yy * per_row + b, a.starts_h[col], mlo, mhi, clo, bands, a.taps_h, ch,
                                            a.phases_h[col], true, false);
            }
            const int yy = i / per_out;
            uint8_t* orow = a.out.data + (int64_t)(ty0 + (i < n_out ? yy : 0)) * a.out.pitch;
            const int64_t col_item = (int64_t)tx0 * bands + (i - yy * per_out);
            if (a.unpremul_out) {
                stage[threadIdx.x] = (uint8_t)v;
                __syncthreads();
                if (i < n_out) {
                    const int b = int(col_item % bands);
                    uint32_t o = stage[threadIdx.x];
                    if (b != bands - 1) o = unpremultiply_u8(o, stage[threadIdx.x + (bands - 1 - b)]);
                    orow[col_item] = (uint8_t)o;
                }
                __syncthreads();
            } else if (i < n_out) {
                reinterpret_cast<T*>(orow)[col_item] = v;
            }
        }
    }
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

}  // namespace dev

namespace launch {

static int fmt_size(int32_t fmt) { return fmt == kU8 ? 1 : (fmt == kU16 ? 2 : 4); }

size_t shrink2d_smem_bytes(const ShrinkArgs& a, int32_t* nx_out) {
    const int es = fmt_size(a.fmt);
    const int64_t per_col = int64_t(a.fh) * a.bands * es;
    int64_t nx = std::max<int64_t>(1, dev::kShrinkSegCap / std::max<int64_t>(per_col, 1));
    nx = std::min<int64_t>(nx, (int64_t)dev::kShrinkMaxItems * dev::kShrinkThreads / a.bands);
    nx = std::max<int64_t>(1, std::min<int64_t>(nx, std::max(a.out.w, 1)));
    const int64_t nin = nx * a.fh;
    const int64_t seg = (nin * a.bands * es + 15) / 16 * 16 + 32;
    int64_t extra;
    if (a.hv_order) extra = a.unpremul_out ? (nx * a.bands + 15) / 16 * 16 : 0;
    else extra = nin * a.bands * (es == 1 ? 4 : 8);
    const int64_t total = seg + extra;
    *nx_out = int32_t(nx);
    if (total > 200 * 1024) return 0;
    return size_t(total);
}

template <typename T>
static cudaError_t shrink_typed(ShrinkArgs a, cudaStream_t s) {
    if (a.col_hi < 0) { a.col_lo = 0; a.col_hi = a.out.w; }
    if (a.col_hi <= a.col_lo) return cudaSuccess;
    int32_t nx;
    const size_t smem = shrink2d_smem_bytes(a, &nx);
    if (smem == 0) return cudaErrorInvalidValue;
    a.nx = nx;
    dim3 grid((unsigned)((a.col_hi - a.col_lo + nx - 1) / nx), (unsigned)a.out.h);
    if (a.hv_order) {
        auto k = dev::shrink2d_kernel<T, true>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, dev::kShrinkThreads, smem, s>>>(a);
    } else {
        auto k = dev::shrink2d_kernel<T, false>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, dev::kShrinkThreads, smem, s>>>(a);
    }
    return cudaGetLastError();
}

static int g_sm_count = 0;

static int sm_count() {
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

static void round_consts(uint32_t f, int bands, bool horizontal, int32_t* mode, uint64_t* mult) {
    *mult = (1ull << 32) / (256ull * f);
    if (f == 1) *mode = 0;
    else if (f == 2) *mode = 1;
    else if (horizontal && f == 5 && (bands == 1 || bands == 3 || bands == 4)) *mode = 2;
    else *mode = 3;
    if (!horizontal) *mult = (uint32_t)*mult;
}

// Interior output columns [lo, hi): their source span lies inside the plane
// and its 16-byte aligned cover lies inside the buffer for every row.
static void interior_columns(const ShrinkArgs& a, int32_t* lo, int32_t* hi) {
    const int64_t fh = a.fh;
    int64_t xlo = (a.in.x0 + fh - 1) / fh;  // ceil for non-negative x0
    if (a.in.x0 < 0) xlo = -((-a.in.x0) / fh);
    int64_t xhi = (a.in.x0 + a.in.w) >= 0 ? (a.in.x0 + a.in.w) / fh : -1;
    int64_t l = std::max<int64_t>(xlo - a.out.x0, 0), h = std::min<int64_t>(xhi - a.out.x0, a.out.w);
    // the last source row's aligned span must stay inside the buffer
    while (h > l) {
        const int64_t ly = a.in.h - 1;
        const int64_t e = ly * a.in.pitch + ((a.out.x0 + h) * fh - a.in.x0) * a.bands;
        if (((e + 15) & ~int64_t(15)) <= a.in.total_bytes) break;
        --h;
    }
    *lo = int32_t(l);
    *hi = int32_t(std::max(l, h));
}

cudaError_t shrink2d(ShrinkArgs a, cudaStream_t s) {
    if (a.out.w <= 0 || a.out.h <= 0) return cudaSuccess;
    round_consts(a.fh, a.bands, true, &a.hmode, &a.hmult);
    round_consts(a.fv, a.bands, false, &a.vmode, &a.vmult);
    if (a.fmt == kU8 && a.hv_order && (reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0 && a.bands <= 4) {
        int32_t lo, hi;
        interior_columns(a, &lo, &hi);
        const int64_t iw = hi - lo;
        const int64_t per_col = int64_t(a.fh) * a.bands;
        // one output pixel per thread: chunks of at most 256 columns, about 16 KB per row
        int64_t nxf = std::min<int64_t>(dev::kShrinkThreads, std::max<int64_t>(1, 16384 / std::max<int64_t>(per_col, 1)));
        const int64_t chunks = iw > 0 ? (iw + nxf - 1) / nxf : 0;
        if (chunks > 0) nxf = (iw + chunks - 1) / chunks;
        const int64_t edge_cols = std::max<int64_t>(lo, a.out.w - hi);
        const int64_t edge_bytes = int64_t(a.fv) * edge_cols * per_col + edge_cols * a.bands + 64;
        const uint32_t stage_bytes = uint32_t((std::max<int64_t>(nxf * per_col, 1) + 32 + 127) / 128 * 128);
        const size_t smem = 128 + std::max<size_t>(size_t(4) * stage_bytes, size_t(edge_bytes)) + 16;
        if (iw > 0 && per_col <= 16384 && smem <= 200 * 1024 && int64_t(a.out.h) * chunks < (int64_t(1) << 30)) {
            ShrinkArgs f = a;
            f.col_lo = lo; f.col_hi = hi; f.nxf = int32_t(nxf); f.chunks = int32_t(chunks);
            f.stages = 4; f.stage_bytes = stage_bytes;
            void (*k)(ShrinkArgs) = a.bands == 1 ? dev::shrink_hv_u8_tma<1>
                                   : a.bands == 2 ? dev::shrink_hv_u8_tma<2>
                                   : a.bands == 3 ? dev::shrink_hv_u8_tma<3> : dev::shrink_hv_u8_tma<4>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, dev::kShrinkThreads, smem);
            const int64_t items = std::max<int64_t>(int64_t(a.out.h) * chunks, 2 * int64_t(a.out.h));
            const int64_t grid = std::min<int64_t>(items, int64_t(std::max(per_sm, 1)) * sm_count());
            k<<<(unsigned)grid, dev::kShrinkThreads, smem, s>>>(f);
            return cudaGetLastError();
        }
    }
    switch (a.fmt) {
    case kU8: return shrink_typed<uint8_t>(a, s);
    case kU16: return shrink_typed<uint16_t>(a, s);
    default: return shrink_typed<float>(a, s);
    }
}

template <typename T, int MODE, bool H>
static cudaError_t reduce_typed(const ReduceArgs& a, cudaStream_t s) {
    const int coef_bytes = 65 * a.taps * (MODE == kReduceFixed ? 2 : 8);
    size_t smem = (coef_bytes <= 48 * 1024 ? (coef_bytes + 15) / 16 * 16 : 0) + 256;
    const int64_t nitems = (int64_t)a.out.w * a.bands;
    dim3 grid((unsigned)((nitems + 255) / 256), (unsigned)a.out.h);
    if (H) {
        auto k = dev::reduce_h_kernel<T, MODE>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, 256, smem, s>>>(a);
    } else {
        auto k = dev::reduce_v_kernel<T, MODE>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, 256, smem, s>>>(a);
    }
    return cudaGetLastError();
}

template <bool H>
static cudaError_t reduce_any(const ReduceArgs& a, cudaStream_t s) {
    if (a.out.w <= 0 || a.out.h <= 0) return cudaSuccess;
    if (a.unpremul_out && (256 % a.bands) != 0) return cudaErrorInvalidValue;
    switch (a.fmt) {
    case kU8:
        if (a.mode == kReduceFixed) return reduce_typed<uint8_t, kReduceFixed, H>(a, s);
        return reduce_typed<uint8_t, kReduceF64Fma, H>(a, s);
    case kU16:
        if (a.mode == kReduceFixed) return reduce_typed<uint16_t, kReduceFixed, H>(a, s);
        return reduce_typed<uint16_t, kReduceF64Fma, H>(a, s);
    default:
        if (a.mode == kReduceF32Simd) return reduce_typed<float, kReduceF32Simd, H>(a, s);
        return reduce_typed<float, kReduceF64Fma, H>(a, s);
    }
}

cudaError_t reduce_h(const ReduceArgs& a, cudaStream_t s) { return reduce_any<true>(a, s); }
cudaError_t reduce_v(const ReduceArgs& a, cudaStream_t s) { return reduce_any<false>(a, s); }

size_t reduce2d_smem_bytes(const Reduce2DArgs& a) {
    const int es = fmt_size(a.fmt);
    const int mh_b = a.mode_h == kReduceFixed ? 2 : 8, mv_b = a.mode_v == kReduceFixed ? 2 : 8;
    const size_t ch = (65 * a.taps_h * mh_b + 15) / 16 * 16, cv = (65 * a.taps_v * mv_b + 15) / 16 * 16;
    const size_t mid = size_t(a.span_max) * (a.hfirst ? a.tile_w : a.tile_h) * a.bands * es;
    const size_t total = ch + cv + (mid + 15) / 16 * 16 + 256 + 16;
    return total <= 200 * 1024 ? total : 0;
}

template <typename T, int MH, int MV>
static cudaError_t r2d(const Reduce2DArgs& a, size_t smem, cudaStream_t s) {
    auto k = dev::reduce2d_kernel<T, MH, MV>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((a.out.w + a.tile_w - 1) / a.tile_w), (unsigned)((a.out.h + a.tile_h - 1) / a.tile_h));
    k<<<grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t reduce2d(const Reduce2DArgs& a, cudaStream_t s) {
    if (a.out.w <= 0 || a.out.h <= 0) return cudaSuccess;
    if (a.unpremul_out && (256 % a.bands) != 0) return cudaErrorInvalidValue;
    const size_t smem = reduce2d_smem_bytes(a);
    if (smem == 0) return cudaErrorInvalidValue;
    switch (a.fmt) {
    case kU8:
        if (a.mode_h == kReduceFixed) return r2d<uint8_t, kReduceFixed, kReduceFixed>(a, smem, s);
        return r2d<uint8_t, kReduceF64Fma, kReduceF64Fma>(a, smem, s);
    case kU16:
        if (a.mode_h == kReduceFixed) return r2d<uint16_t, kReduceFixed, kReduceFixed>(a, smem, s);
        return r2d<uint16_t, kReduceF64Fma, kReduceF64Fma>(a, smem, s);
    default:
        if (a.mode_h == kReduceF64Fma && a.mode_v == kReduceF64Fma) return r2d<float, kReduceF64Fma, kReduceF64Fma>(a, smem, s);
        if (a.mode_h == kReduceF64Fma) return r2d<float, kReduceF64Fma, kReduceF32Simd>(a, smem, s);
        return r2d<float, kReduceF32Simd, kReduceF32Simd>(a, smem, s);
    }
}

cudaError_t pixel(const PixelArgs& a, cudaStream_t s) {
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    if (npx <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<int64_t>((npx + 255) / 256, 148 * 16);
    switch (a.fmt) {
    case kU8: dev::pixel_kernel<uint8_t><<<grid, 256, 0, s>>>(a); break;
    case kU16: dev::pixel_kernel<uint16_t><<<grid, 256, 0, s>>>(a); break;
    default: dev::pixel_kernel<float><<<grid, 256, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
