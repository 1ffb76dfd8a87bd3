// reduce_strip.cuh -- f32 ReduceH + ReduceV (either order) as a streaming
// row-strip kernel.
//
// A block owns a strip of `tw` output columns and a band of output rows.  It
// streams the f32 source row segments the strip needs, top to bottom, into a
// ring of shared-memory slots by TMA bulk copies (`cp.async.bulk`, no
// multicast), eight rows per mbarrier, issued by one lane of each of the
// block's eight warps; rows further ahead are pulled into L2 by bulk
// prefetches.  The staged f32 rows are read in place (each tap converts its
// sample to f64), so a row costs one copy and one wait per eight rows.
//   V first (resize: ReduceV then ReduceH): per group of output rows the V
//     pass reads the staged source rows and makes the group's mid rows of the
//     strip (rounded to f32 as viprs stores them), the H pass the output rows;
//   H first (reduce_h then reduce_v): the H pass turns each staged source row
//     into a mid row (rounded to f32) kept in a ring of f64 rows; per group of
//     output rows the V pass reads that ring.
// Every source and mid sample is computed once per strip (no halo
// recomputation between row tiles), and the arithmetic is the fused reduce's:
// f64 products and sums in viprs's order (the AVX2 lane order of
// reduce_simd.rs:2621-2694 / 2830-2888, or sequential fma for ReduceOp), the
// same clamps of tap rows and columns to the source plane and the mid plane.
#pragma once

#include "resample_dev.cuh"

namespace viprs {
namespace dev {

constexpr int kStripThreads = 256;
constexpr int kStripWarps = kStripThreads / 32;
constexpr int kStripBatch = kStripWarps;  // staged rows per mbarrier (one copy per warp)
constexpr int kStripMaxSlots = 64;        // staged rows per block, at most (a power of two >= kStripBatch)
constexpr int kStripMaxBars = kStripMaxSlots / kStripBatch;
constexpr int kStripPrefetch = 48;        // rows ahead of the copies pulled into L2
constexpr int kStripGroup = 8;            // output rows per pass of the block
constexpr int kStripUnit = 128;           // V-first V-pass values per warp unit (4 per lane)
static_assert(kStripThreads == kCThreads, "grid_walk strides by kCThreads");

// Taps of one output value in the order of MODE (fused_taps_px): `v(t)` reads
// tap t's sample as f64, `c` the phase's coefficient row.  Used where taps
// clamp to a plane edge.
template <int MODE, bool HORIZ, typename V>
__device__ __forceinline__ double strip_taps(V v, const double* c, int taps, bool simd_lane) {
    double acc = 0.0;
    if (MODE == kReduceF32Simd && HORIZ) {
        int t = 0;
        for (; t + 4 <= taps; t += 4) {
            double lanes4 = v(t) * c[t];
            lanes4 = lanes4 + v(t + 1) * c[t + 1];
            lanes4 = lanes4 + v(t + 2) * c[t + 2];
            lanes4 = lanes4 + v(t + 3) * c[t + 3];
            acc = acc + lanes4;
        }
        for (; t < taps; ++t) acc = fma(v(t), c[t], acc);
    } else if (MODE == kReduceF32Simd && simd_lane) {
        for (int t = 0; t < taps; ++t) acc = acc + v(t) * c[t];
    } else {
        for (int t = 0; t < taps; ++t) acc = fma(v(t), c[t], acc);
    }
    return acc;
}

// V taps p[0], p[stride], ... p[(n - 1) * stride] against c[0 .. n) in the
// order of MODE (a sequential sum: the fma chain of ReduceOp, or the f32 SIMD
// V lanes' product then add), continuing `acc`.  A ring read that wraps is two
// calls.
template <int MODE>
__device__ __forceinline__ double strip_seq(const double* p, int stride, const double* c, int n, bool simd_lane,
                                            double acc) {
    if (MODE == kReduceF32Simd && simd_lane) {
#pragma unroll 4
        for (int t = 0; t < n; ++t) acc = acc + p[t * stride] * c[t];
    } else {
#pragma unroll 4
        for (int t = 0; t < n; ++t) acc = fma(p[t * stride], c[t], acc);
    }
    return acc;
}

// H taps of one output value from consecutive pixels (p[t * NB], f64 or f32
// samples) in the order of MODE: the f32 SIMD H lanes add four products before
// adding them to the sum, the tail and ReduceOp use fma.
template <int MODE, int NB, typename S>
__device__ __forceinline__ double strip_h(const S* p, const double* c, int taps) {
    double acc = 0.0;
    int t = 0;
    if (MODE == kReduceF32Simd) {
        for (; t + 4 <= taps; t += 4) {
            double lanes4 = double(p[t * NB]) * c[t];
            lanes4 = lanes4 + double(p[(t + 1) * NB]) * c[t + 1];
            lanes4 = lanes4 + double(p[(t + 2) * NB]) * c[t + 2];
            lanes4 = lanes4 + double(p[(t + 3) * NB]) * c[t + 3];
            acc = acc + lanes4;
        }
    }
#pragma unroll 4
    for (; t < taps; ++t) acc = fma(double(p[t * NB]), c[t], acc);
    return acc;
}

// V-first V pass of one warp unit: four values per lane (staged-row float
// offsets o[0..3]) of one mid row, taps rows of the ring from `row` (bytes,
// `n1` rows before the ring wraps to `wrap`), `sb` bytes between rows.
// SIMD: 0 = every value in the f32 SIMD body (product then add), 1 = none
// (fma), 2 = mixed (bit j of `lanes` set for SIMD values).
template <int SIMD>
__device__ __forceinline__ void strip_v4(const uint8_t* row, const uint8_t* wrap, int n1, int taps, int sb,
                                         const int32_t* o, const double* c, uint32_t lanes, double* acc) {
    for (int t = 0; t < taps; ++t) {
        if (t == n1) row = wrap;
        const float* r = reinterpret_cast<const float*>(row);
        const double ct = c[t];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double v = double(r[o[j]]);
            if (SIMD == 0) acc[j] = acc[j] + v * ct;
            else if (SIMD == 1) acc[j] = fma(v, ct, acc[j]);
            else acc[j] = ((lanes >> j) & 1u) ? acc[j] + v * ct : fma(v, ct, acc[j]);
        }
        row += sb;
    }
}

// The same for a unit whose four values per lane sit at p[0], p[32], p[64],
// p[96] of every staged row (no column clamp): `p` points into the first tap's
// row, `pw` into the row the ring wraps to after `n1` taps, `sbf` floats
// between rows.
template <int SIMD>
__device__ __forceinline__ void strip_v4_lin(const float* p, const float* pw, int n1, int taps, int sbf,
                                             const double* c, uint32_t lanes, double* acc) {
    auto step = [&](const float* r, double ct) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double v = double(r[32 * j]);
            if (SIMD == 0) acc[j] = acc[j] + v * ct;
            else if (SIMD == 1) acc[j] = fma(v, ct, acc[j]);
            else acc[j] = ((lanes >> j) & 1u) ? acc[j] + v * ct : fma(v, ct, acc[j]);
        }
    };
    int t = 0;
#pragma unroll 2
    for (; t < n1; ++t, p += sbf) step(p, c[t]);
#pragma unroll 2
    for (; t < taps; ++t, pw += sbf) step(pw, c[t]);
}

// Launch parameters of the strip kernel beside the fused-reduce arguments.
struct StripArgs {
    Reduce2DArgs r;
    int32_t tw = 16;          // output columns per strip
    int32_t seg = 64;         // output rows per block
    int32_t cs_max = 0;       // most source columns one strip stages
    int32_t ring = 32;        // H first: rows of the f64 mid ring (a power of two)
    int32_t slots = 32;       // staged rows (a power of two, kStripBatch .. kStripMaxSlots)
    int32_t stage_bytes = 0;  // bytes of one staged row (16-byte lead + row rounded up to kStripUnit + slack)
    int64_t z_in = 0, z_out = 0;  // bytes between consecutive images (gridDim.z images)
    int32_t* err = nullptr;       // device error word (timeout), may be null
};

// Shared-memory layout of one strip block (byte offsets, 16-aligned).
struct StripLayout {
    int32_t bars, stop, coef_h, coef_v, tab, stage, ring, scratch, total;
};

__host__ __device__ inline int32_t strip_align16(int64_t v) { return int32_t((v + 15) / 16 * 16); }

// stage: `slots` staged f32 rows; ring (H first): `ring` rows of tw x bands
// f64 mid values; scratch (V first): kStripGroup mid rows of cs_max x bands
// f64 values.
__host__ __device__ inline StripLayout strip_layout(const StripArgs& a) {
    const Reduce2DArgs& r = a.r;
    StripLayout L;
    L.bars = 0;
    L.stop = kStripMaxBars * 8;
    L.coef_h = L.stop + 16;
    L.coef_v = L.coef_h + strip_align16(int64_t(65) * r.taps_h * 8);
    L.tab = L.coef_v + strip_align16(int64_t(65) * r.taps_v * 8);
    L.stage = L.tab + strip_align16(int64_t(a.tw) * 5 + int64_t(a.seg) * 5 + 16);
    L.ring = L.stage + strip_align16(int64_t(a.slots) * a.stage_bytes);
    const int64_t ring_bytes = r.hfirst ? int64_t(a.ring) * a.tw * r.bands * 8 : 0;
    L.scratch = L.ring + strip_align16(ring_bytes);
    const int64_t scratch_bytes = r.hfirst ? 0 : int64_t(kStripGroup) * a.cs_max * r.bands * 8;
    L.total = L.scratch + strip_align16(scratch_bytes);
    return L;
}

// The block's source-row stream: row q of the sequence is a plane row
// (clamped to the plane), staged in slot q % slots by one bulk copy of the 16-byte aligned
// cover of columns [c0, c0 + ncols) (bytes whose cover would pass the end of
// the buffer by plain loads).  Rows come in batches of kStripBatch sharing one
// mbarrier; lane 0 of warp w issues row w of a batch and pulls row
// q + kStripPrefetch into L2.  The plane pitch is a multiple of 16 bytes, so
// every staged row starts at the same offset (`lead`) in its slot.
struct StripStream {
    const PlaneArg* in;
    uint64_t* bars;
    uint8_t* stage;
    int32_t stage_bytes;
    int64_t c0;
    int32_t ncols, bands, nrows;  // nrows: length of the sequence
    int32_t slots;
};

// Row batch*kStripBatch + w, whose segment starts at byte s0 of the plane
// (its plane row clamped to the plane); the prefetch goes kStripPrefetch rows
// further down (not clamped: a hint, kept inside the buffer).
__device__ __forceinline__ void strip_issue_row(const StripStream& s, int64_t s0, int32_t batch, int w) {
    uint64_t* bar = &s.bars[batch & (s.slots / kStripBatch - 1)];
    const int32_t q = batch * kStripBatch + w;
    if (q >= s.nrows) {
        mbar_arrive(bar);  // past the end of the sequence: an arrival without bytes
        return;
    }
    uint8_t* dst = s.stage + size_t(q & (s.slots - 1)) * s.stage_bytes;
    const int64_t n = int64_t(s.ncols) * s.bands * 4;
    const int64_t e0 = s0 + n;
    const int64_t base = int64_t(reinterpret_cast<uintptr_t>(s.in->data) & 15);  // planes are 4-byte aligned
    const int64_t as = ((base + s0) & ~int64_t(15)) - base;
    const int64_t ae = ((base + e0 + 15) & ~int64_t(15)) - base;
    const int64_t total = s.in->total_bytes;
    if (ae > total || as < 0) {
        // the cover leaves the buffer: plain loads for the bytes outside the copy
        const int64_t cs = as < 0 ? as + 16 : as;
        const int64_t ce = ae > total ? ae - 16 : ae;
        for (int64_t b = s0; b < e0; ++b)
            if (b < cs || b >= ce) dst[b - as] = s.in->data[b];
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, uint32_t(ce > cs ? ce - cs : 0));
        if (ce > cs) bulk_load(dst + (cs - as), s.in->data + cs, uint32_t(ce - cs), bar);
    } else {
        mbar_arrive_expect_tx(bar, uint32_t(ae - as));
        bulk_load(dst, s.in->data + as, uint32_t(ae - as), bar);
    }
    if (q + kStripPrefetch < s.nrows) {
        const int64_t f0 = s0 + int64_t(kStripPrefetch) * s.in->pitch;
        const int64_t fa = ((base + f0) & ~int64_t(15)) - base;
        int64_t fe = ((base + f0 + n + 15) & ~int64_t(15)) - base;
        const int64_t lim = ((base + total) & ~int64_t(15)) - base;
        fe = fe > lim ? lim : fe;
        if (fa >= 0 && fe > fa) bulk_prefetch_l2(s.in->data + fa, uint32_t(fe - fa));
    }
}

// Block (strip blockIdx.x, row band blockIdx.y, image blockIdx.z); HF: H first.
template <int NB, int MH, int MV, bool HF>
__global__ void __launch_bounds__(kStripThreads, 2) reduce_strip_kernel(StripArgs sa) {
    extern __shared__ __align__(128) uint8_t smem_st[];
    const StripLayout L = strip_layout(sa);
    Reduce2DArgs a = sa.r;
    a.in.data += int64_t(blockIdx.z) * sa.z_in;
    a.out.data += int64_t(blockIdx.z) * sa.z_out;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int32_t x0 = int32_t(blockIdx.x) * sa.tw, x1 = min(x0 + sa.tw, a.out.w);
    const int32_t y0 = int32_t(blockIdx.y) * sa.seg, y1 = min(y0 + sa.seg, a.out.h);
    if (x0 >= x1 || y0 >= y1) return;
    const int32_t ncx = x1 - x0, W2 = ncx * NB;
    const int32_t P = sa.slots, NBAR = P / kStripBatch, SB = sa.stage_bytes, R = sa.ring;
    const int32_t Pm = P - 1, Rm = R - 1, NBm = NBAR - 1, NBs = __ffs(NBAR) - 1;  // all powers of two
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_st + L.bars);
    volatile int32_t* stop = reinterpret_cast<volatile int32_t*>(smem_st + L.stop);
    double* ch = reinterpret_cast<double*>(smem_st + L.coef_h);
    double* cv = reinterpret_cast<double*>(smem_st + L.coef_v);
    int32_t* sx = reinterpret_cast<int32_t*>(smem_st + L.tab);
    int32_t* sy = sx + sa.tw;
    uint8_t* phx = reinterpret_cast<uint8_t*>(sy + sa.seg);
    uint8_t* phy = phx + sa.tw;
    uint8_t* stage = smem_st + L.stage;
    double* ring = reinterpret_cast<double*>(smem_st + L.ring);
    double* scratch = reinterpret_cast<double*>(smem_st + L.scratch);
    const int64_t pw = a.in.w - 1, phh = a.in.h - 1;
    const int taps_h = a.taps_h, taps_v = a.taps_v;

    for (int i = tid; i < 65 * taps_h; i += kStripThreads) ch[i] = reinterpret_cast<const double*>(a.coeffs_h)[i];
    for (int i = tid; i < 65 * taps_v; i += kStripThreads) cv[i] = reinterpret_cast<const double*>(a.coeffs_v)[i];
    for (int i = tid; i < ncx; i += kStripThreads) { sx[i] = a.starts_h[x0 + i]; phx[i] = a.phases_h[x0 + i]; }
    for (int i = tid; i < y1 - y0; i += kStripThreads) { sy[i] = a.starts_v[y0 + i]; phy[i] = a.phases_v[y0 + i]; }

    // source columns staged per row and the row sequence
    const int64_t hs0 = a.starts_h[x0], hs1 = int64_t(a.starts_h[x1 - 1]) + taps_h - 1;
    const int64_t vs0 = a.starts_v[y0], vs1 = int64_t(a.starts_v[y1 - 1]) + taps_v - 1;
    int64_t clo = 0, chi = 0, c0, q0;
    int32_t C, nrows;
    if (HF) {
        c0 = clampi64(hs0 - a.in.x0, 0, pw);
        C = int32_t(clampi64(hs1 - a.in.x0, 0, pw) - c0 + 1);
        // mid rows [q0, q0 + nrows): the V taps clamped to the mid plane
        q0 = vs0 < a.my0 ? a.my0 : vs0;
        const int64_t m1 = vs1 > a.my0 + a.mh - 1 ? a.my0 + a.mh - 1 : vs1;
        nrows = int32_t(m1 - q0 + 1);
    } else {
        // mid columns [clo, chi]: the H taps clamped to the mid plane
        clo = hs0 < a.mx0 ? a.mx0 : hs0;
        chi = hs1 > a.mx0 + a.mw - 1 ? a.mx0 + a.mw - 1 : hs1;
        c0 = clampi64(clo - a.in.x0, 0, pw);
        C = int32_t(clampi64(chi - a.in.x0, 0, pw) - c0 + 1);
        q0 = vs0 - a.in.y0;  // unclamped local source rows
        nrows = int32_t(vs1 - vs0 + 1);
    }
    // float offset of a staged row's first value in its slot
    const int32_t lead4 = int32_t(((reinterpret_cast<uintptr_t>(a.in.data) + uint64_t(c0) * NB * 4) & 15) >> 2);
    const int64_t iny0 = a.in.y0;
    const StripStream st{&a.in, bars, stage, SB, c0, C, NB, nrows, P};
    if (tid == 0) {
        for (int i = 0; i < NBAR; ++i) mbar_init(&bars[i], kStripBatch);
        *stop = 0;
        mbar_fence_init();
    }
    __syncthreads();

    int32_t issued = 0, waited = 0;  // batches issued / waited for (the same in every thread)
    // issue every batch whose slots hold only rows below `free_below`
    // lane 0 of each warp keeps the plane row (unclamped) and segment offset
    // of its next row, warp + kStripBatch * issued, stepping kStripBatch rows
    // at a time (a multiply only where the clamp to the plane bites)
    const int64_t seg0 = c0 * NB * 4, pitch = a.in.pitch;
    int64_t my_raw = (HF ? q0 - iny0 : q0) + warp;
    auto seg_of = [&](int64_t raw) { return (raw < 0 ? 0 : (raw > phh ? phh : raw)) * pitch + seg0; };
    int64_t my_off = seg_of(my_raw);
    auto issue_until = [&](int32_t free_below) {
        while (issued * kStripBatch < nrows && (issued + 1) * kStripBatch - P <= free_below) {
            if (lane == 0) {
                strip_issue_row(st, my_off, issued, warp);
                my_raw += kStripBatch;
                if (my_raw - kStripBatch >= 0 && my_raw <= phh) my_off += kStripBatch * pitch;
                else my_off = seg_of(my_raw);
            }
            ++issued;
        }
    };
    // wait until sequence rows [.., hi] are staged; false (in every thread)
    // when a wait gave up
    auto wait_rows = [&](int32_t hi) -> bool {
        bool ok = true;
        while (ok && waited * kStripBatch <= hi) {
            ok = waited < issued && mbar_wait(&bars[waited & NBm], uint32_t((waited >> NBs) & 1));
            if (ok) ++waited;
        }
        return __syncthreads_or(!ok) == 0;
    };
    issue_until(0);

    if (HF) {
        int32_t done = 0;  // mid rows made by the H pass (sequence rows taken from the stream)
        const int64_t mlo = a.my0, mhi = a.my0 + a.mh - 1;
        for (int32_t ya = y0; ya < y1; ya += kStripGroup) {
            const int32_t yb = min(ya + kStripGroup, y1), ng = yb - ya;
            const int64_t last = int64_t(sy[yb - 1 - y0]) + taps_v - 1;
            const int32_t need = int32_t((last > mhi ? mhi : last) - q0 + 1);
            if (need > done) {
                issue_until(done);
                if (!wait_rows(need - 1)) { if (tid == 0) *stop = 1; break; }
                // H pass of sequence rows [done, need): mid values of the strip, rounded to f32
                grid_walk(need - done, W2, [&](int j, int col) {
                    const int32_t q = done + j;
                    const int x = col / NB, b = col - (col / NB) * NB;
                    const int s = int(sx[x] - a.in.x0 - c0);
                    const float* row =
                        reinterpret_cast<const float*>(stage + size_t(q & Pm) * SB) + lead4 + b;
                    const double* cp = ch + phx[x] * taps_h;
                    double acc;
                    if (s >= 0 && s + taps_h <= C) {
                        acc = strip_h<MH, NB>(row + s * NB, cp, taps_h);
                    } else {
                        auto v = [&](int t) -> double {
                            int k = s + t;
                            k = k < 0 ? 0 : (k > C - 1 ? C - 1 : k);
                            return double(row[k * NB]);
                        };
                        acc = strip_taps<MH, true>(v, cp, taps_h, false);
                    }
                    ring[size_t(q & Rm) * W2 + col] = double(__double2float_rn(acc));
                });
                __syncthreads();
                done = need;
            }
            // V pass from the ring of mid rows -> output rows
            grid_walk(ng, W2, [&](int yy, int col) {
                const int y = ya + yy - y0;
                const int x = col / NB, b = col - (col / NB) * NB;
                const int64_t sv = sy[y];
                const double* cp = cv + phy[y] * taps_v;
                const bool lane_simd = int64_t(x0 + x) * NB + b < a.vector_len;
                double acc;
                if (sv >= mlo && sv + taps_v - 1 <= mhi) {
                    const int slot = int(sv - q0) & Rm;
                    const int n1 = min(taps_v, R - slot);
                    acc = strip_seq<MV>(ring + size_t(slot) * W2 + col, W2, cp, n1, lane_simd, 0.0);
                    if (n1 < taps_v) acc = strip_seq<MV>(ring + col, W2, cp + n1, taps_v - n1, lane_simd, acc);
                } else {
                    auto v = [&](int t) -> double {
                        int64_t m = sv + t;
                        m = m < mlo ? mlo : (m > mhi ? mhi : m);
                        return ring[size_t(int32_t(m - q0) & Rm) * W2 + col];
                    };
                    acc = strip_taps<MV, false>(v, cp, taps_v, lane_simd);
                }
                reinterpret_cast<float*>(a.out.data + int64_t(ya + yy) * a.out.pitch)[int64_t(x0) * NB + col] =
                    __double2float_rn(acc);
            });
            __syncthreads();
        }
    } else {
        const int32_t Cm = int32_t(chi - clo + 1), Wm = Cm * NB;  // mid values per scratch row
        const int32_t units_row = (Wm + kStripUnit - 1) / kStripUnit;
        // no mid column clamps into the source plane: staged value c is mid value c
        const bool vlin = clo - a.in.x0 >= 0 && chi - a.in.x0 <= pw;
        for (int32_t ya = y0; ya < y1; ya += kStripGroup) {
            const int32_t yb = min(ya + kStripGroup, y1), ng = yb - ya;
            // sequence rows [lo, hi] the group's V taps reach
            const int32_t lo = int32_t(sy[ya - y0] - vs0);
            const int32_t hi = int32_t(int64_t(sy[yb - 1 - y0]) + taps_v - 1 - vs0);
            issue_until(lo);
            if (!wait_rows(hi)) { if (tid == 0) *stop = 1; break; }
            // V pass: warp units of (mid row, kStripUnit values), four values per lane
            for (int32_t u = warp; u < ng * units_row; u += kStripWarps) {
                const int yy = u / units_row, cu = u - yy * units_row;
                const int y = ya + yy - y0;
                const int cb = cu * kStripUnit + lane;  // value of j = 0
                uint32_t simd = 0;
                if (MV == kReduceF32Simd) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int c = min(cb + 32 * j, Wm - 1);
                        const int mc = c / NB;
                        if ((clo + mc - a.mx0) * NB + (c - mc * NB) < a.vector_len) simd |= 1u << j;
                    }
                }
                const int32_t k0 = int32_t(sy[y] - vs0);
                const int slot0 = k0 & Pm;
                const int n1 = min(taps_v, P - slot0);
                const double* cp = cv + phy[y] * taps_v;
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                const int mode = MV != kReduceF32Simd ? 1
                               : __all_sync(0xffffffffu, simd == 0xFu) ? 0
                               : __all_sync(0xffffffffu, simd == 0u) ? 1 : 2;
                if (vlin) {
                    // staged value c of a row is float lead4 + c of its slot (no column clamp)
                    const float* p = reinterpret_cast<const float*>(stage + size_t(slot0) * SB) + lead4 + cb;
                    const float* pw = reinterpret_cast<const float*>(stage) + lead4 + cb;
                    if (mode == 0) strip_v4_lin<0>(p, pw, n1, taps_v, SB / 4, cp, simd, acc);
                    else if (mode == 1) strip_v4_lin<1>(p, pw, n1, taps_v, SB / 4, cp, simd, acc);
                    else strip_v4_lin<2>(p, pw, n1, taps_v, SB / 4, cp, simd, acc);
                } else {
                    int32_t o[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int c = min(cb + 32 * j, Wm - 1);
                        const int mc = c / NB, b = c - mc * NB;
                        o[j] = lead4 + int32_t(clampi64(clo + mc - a.in.x0, 0, pw) - c0) * NB + b;
                    }
                    const uint8_t* row = stage + size_t(slot0) * SB;
                    if (mode == 0) strip_v4<0>(row, stage, n1, taps_v, SB, o, cp, simd, acc);
                    else if (mode == 1) strip_v4<1>(row, stage, n1, taps_v, SB, o, cp, simd, acc);
                    else strip_v4<2>(row, stage, n1, taps_v, SB, o, cp, simd, acc);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = cb + 32 * j;
                    if (c < Wm) scratch[size_t(yy) * Wm + c] = double(__double2float_rn(acc[j]));
                }
            }
            __syncthreads();
            // H pass from the mid rows -> output rows
            grid_walk(ng, W2, [&](int yy, int col) {
                const int x = col / NB, b = col - (col / NB) * NB;
                const int s = int(sx[x] - clo);
                const double* row = scratch + size_t(yy) * Wm + b;
                const double* cp = ch + phx[x] * taps_h;
                double acc;
                if (s >= 0 && s + taps_h <= Cm) {
                    acc = strip_h<MH, NB>(row + s * NB, cp, taps_h);
                } else {
                    auto v = [&](int t) -> double {
                        int k = s + t;
                        k = k < 0 ? 0 : (k > Cm - 1 ? Cm - 1 : k);
                        return row[k * NB];
                    };
                    acc = strip_taps<MH, true>(v, cp, taps_h, false);
                }
                reinterpret_cast<float*>(a.out.data + int64_t(ya + yy) * a.out.pitch)[int64_t(x0) * NB + col] =
                    __double2float_rn(acc);
            });
            __syncthreads();
        }
    }
    if (tid == 0) {
        // copies still in flight (a wait that gave up) land before the block exits (bounded)
        for (int32_t b = waited; b < issued; ++b) mbar_wait(&bars[b & NBm], uint32_t((b >> NBs) & 1));
        if (*stop && sa.err) atomicExch(sa.err, VIPRS_ERR_TIMEOUT);
    }
}

}  // namespace dev
}  // namespace viprs
