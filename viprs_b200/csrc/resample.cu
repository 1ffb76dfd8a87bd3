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
//   zoom_kernel ......... Zoom (structural/zoom.rs:44-149), 16-byte stores
//
// Memory traffic: the shrink reads every source sample exactly once with
// 16-byte loads into shared memory (coalesced across the block) and writes
// each output once; it is HBM-bound.  The reduce kernels gather taps from
// the (L2-resident) shrunk plane with coefficient tables in shared memory.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <type_traits>
#include <vector>

#include "reduce_strip.cuh"
#include "shrink_warp.cuh"
#include "shrink_warp.hpp"

namespace viprs {
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

// The same rounding as (s * mul + add) >> 24 in 32 bits, exact for every box
// sum s <= 255 f: factor 1 copies (mul 2^24), 2 rounds up a half (2^23, 2^23),
// the ShrinkH factor-5 division is (s + 2) * ceil(2^24 / 5) >> 24, and the
// multiplier rule ((s + f/2) * m) >> 24 distributes (its product stays below
// 2^32 because m = floor(2^32 / (256 f))).
static void round_consts32(uint32_t f, int32_t mode, uint32_t* mul, uint32_t* add) {
    switch (mode) {
    case 0: *mul = 1u << 24; *add = 0; break;
    case 1: *mul = 1u << 23; *add = 1u << 23; break;
    case 2: *mul = 3355444u; *add = 2u * 3355444u; break;
    default: {
        const uint32_t m = uint32_t((1ull << 32) / (256ull * f));
        *mul = m;
        *add = (f / 2) * m;
    }
    }
}

static void shrink_round_all(ShrinkArgs* a) {
    round_consts(a->fh, a->bands, true, &a->hmode, &a->hmult);
    round_consts(a->fv, a->bands, false, &a->vmode, &a->vmult);
    round_consts32(a->fh, a->hmode, &a->hmul, &a->hadd);
    round_consts32(a->fv, a->vmode, &a->vmul, &a->vadd);
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

// Bank-conflict cost of a warp's box walk in shared memory for lane rotation
// `shift`: lanes read word base + ((q0 + t) % Kg) * G + j at step t, with
// q0 = (lane >> shift) % Kg; the cost is the sum over steps of the most
// distinct words any bank serves (the wavefronts of that load).
static int64_t walk_cost(int B, int fh, int pw, bool premul4, int shift) {
    const int lp = 32 / pw;
    const int G = (B == 3 && !premul4) ? 3 : 1;
    int64_t cost = 0;
    const int leads = premul4 ? 1 : 4;
    for (int o = 0; o < leads; ++o) {
        int base[32], kg[32], q0[32], steps = 0;
        for (int l = 0; l < 32; ++l) {
            const int pix = l % pw, part = l / pw;
            const int j0 = part * fh / lp, j1 = (part + 1) * fh / lp, npix = j1 - j0;
            const int start = o + (pix * fh + j0) * B;
            base[l] = start / 4;
            if (premul4) kg[l] = std::max(npix, 1);
            else kg[l] = std::max(1, (((npix * B + 3) >> 2) + G - 1) / G);
            q0[l] = (l >> shift) % kg[l];
            steps = std::max(steps, kg[l]);
        }
        for (int t = 0; t < steps; ++t)
            for (int j = 0; j < G; ++j) {
                int64_t words[32];
                int n = 0;
                for (int l = 0; l < 32; ++l) {
                    if (t >= kg[l]) continue;
                    words[n++] = base[l] + int64_t((q0[l] + t) % kg[l]) * G + j;
                }
                int worst = 0;
                for (int b = 0; b < 32; ++b) {
                    int distinct = 0;
                    for (int i = 0; i < n; ++i) {
                        if (((words[i] % 32) + 32) % 32 != b) continue;
                        bool seen = false;
                        for (int q = 0; q < i; ++q) seen |= words[q] == words[i];
                        distinct += seen ? 0 : 1;
                    }
                    worst = std::max(worst, distinct);
                }
                cost += worst;
            }
    }
    return cost;
}

// Resident blocks per SM of a warp-shrink kernel with `smem` bytes of shared
// memory; the kernel's shared-memory limit is raised once per (bands, size)
// and the answer cached, so that launches make no driver queries.
static int warp_blocks_per_sm(void (*kern)(ShrinkArgs), int bands, size_t smem) {
    struct Entry { int bands; size_t smem; int bps; };
    static std::vector<Entry> cache;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    bool raised = false;
    for (const Entry& e : cache) {
        if (e.bands == bands && e.smem == smem) return e.bps;
        raised |= e.bands == bands;
    }
    // one limit for every size this kernel is launched with (a lower limit
    // set later would refuse the larger launches)
    if (!raised) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    int bps = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kWarpBlockThreads, smem);
    bps = std::max(1, bps);
    cache.push_back(Entry{bands, smem, bps});
    return bps;
}

static uint32_t warp_stage_bytes(int64_t seg_bytes) { return uint32_t((15 + seg_bytes + 32 + 15) / 16 * 16); }

bool shrink_warp_setup(ShrinkArgs* a, uint32_t stage_budget, int64_t item_bytes, int64_t min_items) {
    const int64_t s = int64_t(a->fh) * a->bands;
    int pw = 32;
    const int64_t w = std::max<int64_t>(a->out.w, 1);
    while (pw > 8 && pw / 2 >= w) pw /= 2;  // narrow outputs: spare lanes split the boxes
    while (pw > 8 && warp_stage_bytes(pw * s) > stage_budget) pw /= 2;
    if (warp_stage_bytes(pw * s) > stage_budget) return false;
    a->nxf = pw;
    a->row_cap = warp_stage_bytes(pw * s);
    const int64_t per_row = std::max<int64_t>(1, pw * s * int64_t(a->fv));
    int64_t rows = std::max<int64_t>(1, std::min<int64_t>(a->out.h, item_bytes / per_row));
    const int64_t groups = (a->out.w + pw - 1) / pw;
    if (min_items > 0) rows = std::max<int64_t>(1, std::min<int64_t>(rows, groups * a->out.h / min_items));
    a->rows_per_item = int32_t(rows);
    // only the premultiplied 4-band walk is rotated (uniform trip counts);
    // its best rotation per (fh, pw) is cached
    a->rot_shift = 5;
    if (a->premul_in && a->bands == 4) {
        struct Entry { uint32_t fh; int pw; int shift; };
        static std::vector<Entry> cache;
        static std::mutex mu;
        std::lock_guard<std::mutex> lock(mu);
        for (const Entry& e : cache)
            if (e.fh == a->fh && e.pw == pw) { a->rot_shift = e.shift; return true; }
        int best = 5;
        int64_t best_cost = walk_cost(4, int(a->fh), pw, true, 5);
        for (int sh = 0; sh < 5; ++sh) {
            const int64_t c = walk_cost(4, int(a->fh), pw, true, sh);
            if (c < best_cost) { best_cost = c; best = sh; }
        }
        cache.push_back(Entry{a->fh, pw, best});
        a->rot_shift = best;
    }
    return true;
}

int64_t shrink_warp_items(const ShrinkArgs& a) {
    const int64_t groups = (a.out.w + a.nxf - 1) / a.nxf;
    return ((a.out.h + a.rows_per_item - 1) / a.rows_per_item) * groups;
}

void shrink_prepare(ShrinkArgs* a, int32_t* lo, int32_t* hi) {
    shrink_round_all(a);
    interior_columns(*a, lo, hi);
}

cudaError_t shrink2d(ShrinkArgs a, cudaStream_t s) {
    if (a.out.w <= 0 || a.out.h <= 0) return cudaSuccess;
    shrink_round_all(&a);
    if (a.fmt == kU8 && a.hv_order && (reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0 && a.bands <= 4) {
        // independent warps, each streaming its own source rows (shrink_warp.cuh)
        ShrinkArgs f = a;
        // items small enough that every resident warp gets several
        if (shrink_warp_setup(&f, 2048, 48 * 1024, int64_t(sm_count()) * 24 * 4)) {
            const size_t smem = size_t(kWarpBlockThreads / 32) * (dev::kWarpBars + kWarpStagesHost * size_t(f.row_cap));
            void (*kern)(ShrinkArgs) = a.bands == 1 ? dev::shrink_warp_kernel<1>
                                      : a.bands == 2 ? dev::shrink_warp_kernel<2>
                                      : a.bands == 3 ? dev::shrink_warp_kernel<3> : dev::shrink_warp_kernel<4>;
            const int bps = warp_blocks_per_sm(kern, a.bands, smem);
            // one warp per item up to the resident grid; warps then stride over the items
            const int64_t items = shrink_warp_items(f);
            const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((items + 7) / 8, int64_t(bps) * sm_count()));
            kern<<<(unsigned)grid, kWarpBlockThreads, smem, s>>>(f);
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

// Strip-kernel launch parameters of a configured f32 stage (strip_configure
// stores the staged-row slots in in_rows_max).
static dev::StripArgs strip_args(const Reduce2DArgs& a) {
    dev::StripArgs sa;
    sa.r = a;
    sa.tw = a.tile_w;
    sa.seg = a.tile_h;
    sa.cs_max = a.in_cols_max;
    sa.ring = a.span_max;
    sa.slots = a.in_rows_max;
    sa.err = a.err;
    // V first reads whole kStripUnit values per warp unit from a staged row
    const int64_t vals = int64_t(a.in_cols_max) * a.bands;
    const int64_t units = (vals + dev::kStripUnit - 1) / dev::kStripUnit * dev::kStripUnit;
    sa.stage_bytes = a.hfirst ? dev::strip_align16(vals * 4 + 32) : dev::strip_align16((units + 4) * 4);
    return sa;
}

size_t reduce2d_smem_bytes(const Reduce2DArgs& a) {
    if (a.strip) {
        const dev::StripLayout L = dev::strip_layout(strip_args(a));
        return L.total <= 200 * 1024 ? size_t(L.total) : 0;
    }
    if (a.tile_w <= 0 || a.tile_h <= 0 || a.span_max <= 0 || a.in_rows_max <= 0 || a.in_cols_max <= 0) return 0;
    const Reduce2DLayout L = reduce2d_layout(a);
    return L.total <= 200 * 1024 ? size_t(L.total) : 0;
}

// f32 stages with 1, 3 or 4 bands and a source pitch that is a multiple of 16
// bytes run as row strips (reduce_strip.cuh): the widest strip whose block
// fits 110 KB of shared memory (two blocks per SM) with staged rows (a power of
// two) for twice the span of one group of output rows, else for that span plus
// one batch, and rows per block for about four waves of blocks.
static bool strip_configure(Reduce2DArgs* a, const int32_t* sh, const int32_t* sv, int64_t in_x0, int64_t in_w) {
    if (a->fmt != kF32 || a->premul_in || a->unpremul_out) return false;
    if (a->bands != 1 && a->bands != 3 && a->bands != 4) return false;
    if (a->mode_h == kReduceFixed || a->mode_v == kReduceFixed) return false;
    if (a->in.pitch <= 0 || a->in.pitch % 16 != 0) return false;
    const int64_t ow = a->out.w, oh = a->out.h;
    if (ow <= 0 || oh <= 0) return false;
    // every block's taps must reach the mid plane (the kernel's row and column
    // sequences are its intersection with the mid plane)
    if (a->hfirst && (sv[oh - 1] > a->my0 + a->mh - 1 || int64_t(sv[0]) + a->taps_v - 1 < a->my0)) return false;
    if (!a->hfirst && (sh[ow - 1] > a->mx0 + a->mw - 1 || int64_t(sh[0]) + a->taps_h - 1 < a->mx0)) return false;
    const int G = dev::kStripGroup, B = dev::kStripBatch;
    // span: the most rows one group of output rows reaches (groups start at
    // multiples of G: blocks cover multiples of G rows)
    int64_t span = 1;
    for (int64_t y = 0; y < oh; y += G) {
        const int64_t yb = std::min(oh, y + G) - 1;
        int64_t v0 = sv[y], v1 = int64_t(sv[yb]) + a->taps_v - 1;
        if (a->hfirst) {
            v0 = std::max<int64_t>(v0, a->my0);
            v1 = std::min<int64_t>(v1, int64_t(a->my0) + a->mh - 1);
        }
        span = std::max(span, v1 - v0 + 1);
    }
    // staged rows: a power of two, the group's span plus at least one batch in flight
    int64_t min_slots = B;
    while (min_slots < span + B) min_slots *= 2;
    if (min_slots > dev::kStripMaxSlots) return false;
    int64_t ring = 1;  // H first: mid ring rows, a power of two
    while (ring < span) ring *= 2;
    const int tws[3] = {a->bands == 1 ? 128 : 32, a->bands == 1 ? 64 : 16, a->bands == 1 ? 32 : 8};
    const int64_t budget = 110 * 1024;
    for (int pass = 0; pass < 2; ++pass) {
        // first the most slots (a batch or more beyond one group), then the fewest
        const int64_t want = pass == 0 ? std::min<int64_t>(dev::kStripMaxSlots, 2 * min_slots) : min_slots;
        for (int tw : tws) {
            int64_t cs = 1;
            for (int64_t x = 0; x < ow; x += tw) {
                const int64_t xb = std::min(ow, x + tw) - 1;
                const int64_t h0 = sh[x], h1 = int64_t(sh[xb]) + a->taps_h - 1;
                if (a->hfirst) {
                    const int64_t c0 = std::min(std::max(h0 - in_x0, int64_t(0)), in_w - 1);
                    const int64_t c1 = std::min(std::max(h1 - in_x0, int64_t(0)), in_w - 1);
                    cs = std::max(cs, c1 - c0 + 1);
                } else {
                    const int64_t lo = std::max<int64_t>(h0, a->mx0);
                    const int64_t hi = std::min<int64_t>(h1, int64_t(a->mx0) + a->mw - 1);
                    cs = std::max(cs, hi - lo + 1);
                }
            }
            Reduce2DArgs c = *a;
            c.strip = 1;
            c.tile_w = tw;
            c.tile_h = 1024;  // the table size of the largest band: fixed below
            c.in_cols_max = int32_t(cs);
            c.span_max = int32_t(ring);
            int64_t slots = 0;
            for (int64_t p = dev::kStripMaxSlots; p >= want; p /= 2) {
                c.in_rows_max = int32_t(p);
                if (dev::strip_layout(strip_args(c)).total <= budget) { slots = p; break; }
            }
            if (slots == 0) continue;
            c.in_rows_max = int32_t(slots);
            const int64_t total = dev::strip_layout(strip_args(c)).total;
            const int64_t per_sm = std::max<int64_t>(1, std::min<int64_t>(8, (228 * 1024) / (total + 1024)));
            const int64_t strips = (ow + tw - 1) / tw;
            const int64_t min_blocks = 4 * per_sm * 148;
            const int64_t bands_rows = std::max<int64_t>(1, (min_blocks + strips - 1) / strips);
            int64_t seg = (oh + bands_rows - 1) / bands_rows;
            seg = std::max<int64_t>(G, (seg + G - 1) / G * G);
            c.tile_h = int32_t(std::min<int64_t>(seg, 1024));
            *a = c;
            return true;
        }
    }
    return false;
}

bool reduce2d_configure(Reduce2DArgs* a, const int32_t* sh, const int32_t* sv, int64_t in_x0, int64_t in_y0,
                        int64_t in_w, int64_t in_h, int64_t min_tiles, size_t smem_budget) {
    a->strip = 0;
    if (strip_configure(a, sh, sv, in_x0, in_w)) return true;
    static const int32_t kShapes[][2] = {{128, 32}, {64, 64}, {64, 32}, {32, 64}, {32, 32}, {64, 16}, {32, 16},
                                         {16, 32}, {16, 16}, {32, 8}, {16, 8}, {8, 8}, {8, 4}, {4, 4},
                                         {4, 2}, {2, 2}, {2, 1}, {1, 1}};
    const int64_t ow = a->out.w, oh = a->out.h;
    // per-axis extents of every tile of a given size: (first, last) tap of the tile
    auto axis = [&](const int32_t* st, int64_t n, int tile, int taps, auto&& fn) {
        for (int64_t t0 = 0; t0 < n; t0 += tile) {
            const int64_t t1 = std::min(n, t0 + tile) - 1;
            fn(int64_t(st[t0]), int64_t(st[t1]) + taps - 1);
        }
    };
    Reduce2DArgs best = *a;
    bool found = false;
    int64_t best_tiles = 0;
    for (const auto& sz : kShapes) {
        Reduce2DArgs c = *a;
        c.tile_w = sz[0];
        c.tile_h = sz[1];
        int64_t span = 1, rows = 1, cols = 1;
        if (c.hfirst) {
            const int64_t mlo = c.my0, mhi = c.my0 + c.mh - 1;
            axis(sv, oh, c.tile_h, c.taps_v, [&](int64_t v0, int64_t v1) {
                span = std::max(span, std::min(v1, mhi) - std::max(v0, mlo) + 1);
            });
            rows = span;
            axis(sh, ow, c.tile_w, c.taps_h, [&](int64_t h0, int64_t h1) {
                const int64_t c0 = std::min(std::max(h0 - in_x0, int64_t(0)), in_w - 1);
                const int64_t c1 = std::min(std::max(h1 - in_x0, int64_t(0)), in_w - 1);
                cols = std::max(cols, c1 - c0 + 1);
            });
        } else {
            const int64_t mlo = c.mx0, mhi = c.mx0 + c.mw - 1;
            axis(sh, ow, c.tile_w, c.taps_h, [&](int64_t h0, int64_t h1) {
                const int64_t lo = std::max(h0, mlo), hi = std::min(h1, mhi);
                span = std::max(span, hi - lo + 1);
                const int64_t c0 = std::min(std::max(lo - in_x0, int64_t(0)), in_w - 1);
                const int64_t c1 = std::min(std::max(hi - in_x0, int64_t(0)), in_w - 1);
                cols = std::max(cols, c1 - c0 + 1);
            });
            axis(sv, oh, c.tile_h, c.taps_v, [&](int64_t v0, int64_t v1) {
                const int64_t r0 = std::min(std::max(v0 - in_y0, int64_t(0)), in_h - 1);
                const int64_t r1 = std::min(std::max(v1 - in_y0, int64_t(0)), in_h - 1);
                rows = std::max(rows, r1 - r0 + 1);
            });
        }
        c.span_max = int32_t(span);
        c.in_rows_max = int32_t(rows);
        c.in_cols_max = int32_t(cols);
        const size_t need = reduce2d_smem_bytes(c);
        if (need == 0 || need > smem_budget) continue;
        const int64_t tiles = ((ow + c.tile_w - 1) / c.tile_w) * ((oh + c.tile_h - 1) / c.tile_h);
        if (!found || (best_tiles < min_tiles && tiles > best_tiles)) {
            best = c;
            best_tiles = tiles;
            found = true;
        }
        if (tiles >= min_tiles) break;
    }
    if (!found) return false;
    *a = best;
    return true;
}

template <typename T, int MH, int MV>
static cudaError_t r2d(const Reduce2DArgs& a, size_t smem, cudaStream_t s) {
    auto k = a.bands == 1 ? dev::reduce2d_kernel<T, MH, MV, 1>
           : a.bands == 2 ? dev::reduce2d_kernel<T, MH, MV, 2>
           : a.bands == 3 ? dev::reduce2d_kernel<T, MH, MV, 3>
           : a.bands == 4 ? dev::reduce2d_kernel<T, MH, MV, 4>
                          : dev::reduce2d_kernel<T, MH, MV, 0>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((a.out.w + a.tile_w - 1) / a.tile_w), (unsigned)((a.out.h + a.tile_h - 1) / a.tile_h));
    k<<<grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

template <int MH, int MV>
static cudaError_t strip_launch(const Reduce2DArgs& a, size_t smem, cudaStream_t s) {
    const dev::StripArgs sa = strip_args(a);
    auto pick = [&](auto hf) {
        constexpr bool HF = decltype(hf)::value;
        return a.bands == 1 ? dev::reduce_strip_kernel<1, MH, MV, HF>
             : a.bands == 3 ? dev::reduce_strip_kernel<3, MH, MV, HF> : dev::reduce_strip_kernel<4, MH, MV, HF>;
    };
    auto k = a.hfirst ? pick(std::true_type{}) : pick(std::false_type{});
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((a.out.w + a.tile_w - 1) / a.tile_w), (unsigned)((a.out.h + a.tile_h - 1) / a.tile_h));
    k<<<grid, dev::kStripThreads, smem, s>>>(sa);
    return cudaGetLastError();
}

cudaError_t reduce2d(const Reduce2DArgs& a, cudaStream_t s) {
    if (a.out.w <= 0 || a.out.h <= 0) return cudaSuccess;
    if (a.unpremul_out && (256 % a.bands) != 0) return cudaErrorInvalidValue;
    const size_t smem = reduce2d_smem_bytes(a);
    if (smem == 0) return cudaErrorInvalidValue;
    if (a.strip) {
        if (a.mode_h == kReduceF64Fma && a.mode_v == kReduceF64Fma) return strip_launch<kReduceF64Fma, kReduceF64Fma>(a, smem, s);
        if (a.mode_h == kReduceF64Fma) return strip_launch<kReduceF64Fma, kReduceF32Simd>(a, smem, s);
        if (a.mode_v == kReduceF64Fma) return strip_launch<kReduceF32Simd, kReduceF64Fma>(a, smem, s);
        return strip_launch<kReduceF32Simd, kReduceF32Simd>(a, smem, s);
    }
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
    if (a.op == 3) {
        // one block row per output row (grid-strided past 65535), enough
        // blocks along x for one 16-byte chunk per thread
        const int64_t row_bytes = (int64_t)a.out.w * a.bands * fmt_size(a.fmt);
        const int64_t chunks = row_bytes / 16 + 1;
        const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((chunks + 255) / 256, 64));
        if (a.out.pitch % 16 == 0 && a.bands <= dev::kZoomMaxBands && a.in.h > 0) {
            // output rows of one source row together (see zoom_rows_kernel)
            const unsigned gxr = (unsigned)std::max<int64_t>(
                1, std::min<int64_t>((chunks + dev::kZoomChunks - 1) / dev::kZoomChunks, 64));
            const dim3 grid(gxr, (unsigned)std::min<int64_t>(a.in.h, 65535));
            switch (a.fmt) {
            case kU8: dev::zoom_rows_kernel<uint8_t><<<grid, 256, 0, s>>>(a); break;
            case kU16: dev::zoom_rows_kernel<uint16_t><<<grid, 256, 0, s>>>(a); break;
            default: dev::zoom_rows_kernel<float><<<grid, 256, 0, s>>>(a); break;
            }
            return cudaGetLastError();
        }
        const dim3 grid(gx, (unsigned)std::min<int64_t>(a.out.h, 65535));
        switch (a.fmt) {
        case kU8: dev::zoom_kernel<uint8_t><<<grid, 256, 0, s>>>(a); break;
        case kU16: dev::zoom_kernel<uint16_t><<<grid, 256, 0, s>>>(a); break;
        default: dev::zoom_kernel<float><<<grid, 256, 0, s>>>(a); break;
        }
        return cudaGetLastError();
    }
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
