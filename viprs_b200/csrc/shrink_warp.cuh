// shrink_warp.cuh -- u8 ShrinkH then ShrinkV (shrinkh.rs:323-397,
// shrinkv.rs:191-339) by independent warps.
//
// A warp owns `pw` consecutive output pixels (32, 16 or 8: 32 / pw lanes
// share one pixel's box) of a band of output rows.  It streams the source row
// segment its boxes cover through a private kWarpStages-deep buffer in shared
// memory: lane 0 issues one TMA bulk copy (`cp.async.bulk`, no multicast) per
// source row, completing on the stage's mbarrier in the warp's own shared
// memory, so that the next rows are in flight while the warp sums the current
// one; rows further ahead are pulled into L2 by bulk prefetches, so that the
// stage copies wait for L2 rather than DRAM.  Nothing is shared with other warps -- no producer warp, no block
// barrier -- and warps pick their work independently.  Per source row each
// lane sums its part of its pixel's box (dp4a over realigned words, or
// premultiplied 4-band pixels), the parts are combined with shuffles and
// rounded as ShrinkH rounds; per output row the rounded sums are rounded as
// ShrinkV rounds, unpremultiplied when the chain ends there, and stored.
// Boxes that leave the plane (the reduce halo beyond the image) read clamped
// columns from the staged segment.
//
// ShrinkArgs fields used here: nxf = pw, rows_per_item = output rows per
// work item, row_cap = bytes of one stage buffer (source segment + 16-byte
// alignment + 32 bytes of over-read slack), rot_shift = lane rotation of the
// premultiplied 4-band walk (chosen on the host to spread shared-memory
// banks).  Every wait on
// a stage is bounded: a wait that gives up records VIPRS_ERR_TIMEOUT in
// a.err, waits (bounded) for the warp's copies still in flight and makes the
// warp stop.
#pragma once

#include "resample_dev.cuh"

namespace viprs {
namespace dev {

constexpr int kWarpStages = 4;    // source rows in flight to shared memory per warp
constexpr int kWarpPrefetch = 8;   // rows ahead of the consumed one pulled into L2
// Shared memory ahead of a warp's stage buffers: its kWarpStages mbarriers.
constexpr uint32_t kWarpBars = 128;

// A warp's copy pipeline: the stage mbarriers and the number of rows issued
// and consumed so far (row n uses stage n % kWarpStages, phase parity
// (n / kWarpStages) & 1), kept across the warp's work items.
struct WarpPipe {
    uint64_t* bars;
    uint32_t issued = 0, consumed = 0;
    bool ok = true;
};

// Lane 0: initialise the pipe's barriers (one arrival each: lane 0's
// arrive.expect_tx).
__device__ __forceinline__ void warp_pipe_init(WarpPipe& p, uint8_t* warp_smem) {
    p.bars = reinterpret_cast<uint64_t*>(warp_smem);
    if ((threadIdx.x & 31) == 0) {
        for (int s = 0; s < kWarpStages; ++s) mbar_init(&p.bars[s], 1);
        mbar_fence_init();
    }
    __syncwarp();
}

// Box sums of a pixel whose box leaves the plane (the reduce halo): the
// columns beyond the plane read its edge columns, so the sum is the box over
// the part inside the plane plus each edge pixel times the columns clamped
// onto it (premultiplied when `premul`).  `row` holds plane columns from c_lo.
template <int B>
__device__ __forceinline__ void box_sums_edge(const uint8_t* row, int64_t fcol, int32_t fh, int64_t c_lo, int64_t w,
                                              bool premul, uint32_t (&sums)[B]) {
    const int64_t ca = fcol < 0 ? 0 : (fcol > w ? w : fcol);
    const int64_t cb = fcol + fh > w ? w : (fcol + fh < 0 ? 0 : fcol + fh);
    const int32_t n_in = cb > ca ? int32_t(cb - ca) : 0;
    const int32_t left = int32_t((fcol < 0 ? (fcol + fh < 0 ? fh : -fcol) : 0));
    const int32_t right = fh - n_in - left;
#pragma unroll
    for (int b = 0; b < B; ++b) sums[b] = 0;
    if (n_in > 0) {
        const uint8_t* p = row + (ca - c_lo) * B;
        if (premul && B == 4) box_sums_premul4_rot(p, n_in, 0, *reinterpret_cast<uint32_t(*)[4]>(sums));
        else if (premul && B == 2) box_sums_premul2_u8(p, n_in, *reinterpret_cast<uint32_t(*)[2]>(sums));
        else box_sums_u8<B>(p, n_in, sums);
    }
    auto add_px = [&](int64_t c, int32_t times) {
        if (times <= 0) return;
        const uint8_t* px = row + (c - c_lo) * B;
        const uint32_t al = px[B - 1];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const uint32_t v = (premul && b != B - 1 && B >= 2) ? premultiply_u8(px[b], al) : uint32_t(px[b]);
            sums[b] += v * uint32_t(times);
        }
    };
    add_px(0, left);
    add_px(w - 1, right);
}

// One work item: output columns [x0, x0 + pw) (local to a.out) of output rows
// [oy0, oy1).  `wbuf`: this warp's kWarpStages * a.row_cap bytes of shared
// memory (16-byte aligned).  Every lane of the warp calls it; on a timeout it
// clears p.ok.
template <int B, bool PAIR>
__device__ void shrink_warp_item(const ShrinkArgs& a, int32_t x0, int32_t oy0, int32_t oy1, uint8_t* wbuf,
                                 WarpPipe& p) {
    constexpr int D = kWarpStages;
    const int lane = threadIdx.x & 31;
    const int pw = a.nxf, lp = 32 / pw;
    const int pix = lane & (pw - 1), part = lane / pw;
    const int32_t fh = int32_t(a.fh), fv = int32_t(a.fv);
    const int32_t x = x0 + pix;
    const bool mine = x < a.out.w;
    const int64_t fcol = (a.out.x0 + x) * (int64_t)fh - a.in.x0;
    const bool inside = fcol >= 0 && fcol + fh <= a.in.w;
    // source columns [c_lo, c_hi) of the warp's boxes, clamped into the plane
    const int32_t xe = min(x0 + pw, a.out.w);
    int64_t c_lo = (a.out.x0 + x0) * (int64_t)fh - a.in.x0, c_hi = (a.out.x0 + xe) * (int64_t)fh - a.in.x0;
    c_lo = c_lo < 0 ? 0 : (c_lo >= a.in.w ? a.in.w - 1 : c_lo);
    c_hi = c_hi <= c_lo ? c_lo + 1 : (c_hi > a.in.w ? a.in.w : c_hi);
    const int64_t seg_bytes = (c_hi - c_lo) * B;
    const uint32_t rb = a.row_cap;
    // this lane's part of its pixel's box: pixels [j0, j1)
    const int32_t j0 = part * fh / lp, j1 = (part + 1) * fh / lp;
    const int32_t npix = j1 - j0;
    const int32_t off = inside ? int32_t(fcol + j0 - c_lo) * B : 0;
    const bool premul = a.premul_in != 0;
    const bool premul4 = premul && B == 4;
    // lane rotation of the premultiplied walk (the dp4a walk is not rotated:
    // its split loops would diverge)
    const int q0 = premul4 ? (lane >> a.rot_shift) % (npix > 0 ? npix : 1) : 0;
    const int32_t T = (oy1 - oy0) * fv;
    const int64_t total = a.in.total_bytes;
    // flattened row i of the item is plane row ly0 + i (clamped to the plane)
    const int64_t ly0 = (a.out.y0 + oy0) * (int64_t)fv - a.in.y0;
    const int64_t hmax = a.in.h - 1;
    // byte offset of flattened row i's segment, and the same advanced one row
    // at a time (the rows of an item are consecutive, clamped at the plane's
    // edges: the offset moves by a pitch only while the clamped row moves)
    struct Cursor {
        int64_t raw, off;
    };
    auto cursor_at = [&](int32_t i) -> Cursor {
        const int64_t ly = ly0 + i;
        const int64_t c = ly < 0 ? 0 : (ly > hmax ? hmax : ly);
        return Cursor{ly, c * a.in.pitch + c_lo * B};
    };
    auto step = [&](Cursor& c) {
        ++c.raw;
        if (uint64_t(c.raw - 1) < uint64_t(hmax)) c.off += a.in.pitch;
    };
    Cursor cur_issue = cursor_at(0);
    // staged-row leads (segment offset mod 16), one byte per stage
    uint32_t leads = 0;
    // the row kWarpPrefetch below the one being issued is pulled into L2 (its
    // offset is not clamped at the plane's edges: the prefetch is only a hint,
    // kept inside the buffer below)
    const int64_t pref_ahead = int64_t(kWarpPrefetch) * a.in.pitch;
    // A 16-byte aligned plane streams each row segment's aligned cover by one
    // bulk copy; bytes whose cover would pass the end of the buffer go by
    // plain loads first.  Any other plane is copied byte by byte by the whole
    // warp (the stage's barrier then completes with no transaction bytes).
    const bool al16 = (reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0;
    // copy rows [first, first + n) of the item (n <= 2) into their
    // stages: lanes 0 .. n-1 issue one bulk copy each, in parallel, and pull
    // the row kWarpPrefetch below theirs into L2, so that its copy finds its
    // bytes there
    auto issue2 = [&](int32_t first, int n) {
        const int64_t o0 = cur_issue.off;
        step(cur_issue);
        const int64_t o1 = cur_issue.off;
        if (n > 1) step(cur_issue);
        // stages follow the warp's running count of issued rows (items chain
        // on one pipe), exactly as the consumer's count of consumed rows does
        const int st0 = int(p.issued % kWarpStages), st1 = int((p.issued + 1) % kWarpStages);
        leads = (leads & ~(0xFFu << (8 * st0))) | (uint32_t(o0 & 15) << (8 * st0));
        if (n > 1) leads = (leads & ~(0xFFu << (8 * st1))) | (uint32_t(o1 & 15) << (8 * st1));
        if (!al16) {
            for (int k = 0; k < n; ++k) {
                uint8_t* dst = wbuf + uint32_t(k == 0 ? st0 : st1) * rb;
                const int64_t s0 = k == 0 ? o0 : o1;
                for (int32_t v = lane; v < int32_t(seg_bytes); v += 32) dst[v] = a.in.data[s0 + v];
                __syncwarp();
                if (lane == 0) mbar_arrive_expect_tx(&p.bars[k == 0 ? st0 : st1], 0);
            }
        } else if (lane < n) {
            const int stage = lane == 0 ? st0 : st1;
            const int64_t s0 = lane == 0 ? o0 : o1;
            const int32_t i = first + lane;
            uint8_t* dst = wbuf + uint32_t(stage) * rb;
            const int64_t e0 = s0 + seg_bytes;
            const int64_t as = s0 & ~int64_t(15);
            int64_t ae = (e0 + 15) & ~int64_t(15);
            if (ae > total) {
                const int64_t ab = e0 & ~int64_t(15);
                for (int64_t q = ab > as ? ab : as; q < e0; ++q) dst[q - as] = a.in.data[q];
                ae = ab > as ? ab : as;
            }
            if (ae != ((e0 + 15) & ~int64_t(15))) fence_proxy_async_smem();  // plain stores above
            mbar_arrive_expect_tx(&p.bars[stage], uint32_t(ae - as));
            if (ae > as) bulk_load(dst, a.in.data + as, uint32_t(ae - as), &p.bars[stage]);
            if (i + kWarpPrefetch < T) {
                const int64_t f0 = (s0 + pref_ahead) & ~int64_t(15);
                int64_t fe = (f0 + seg_bytes + 31) & ~int64_t(15);
                fe = fe > (total & ~int64_t(15)) ? (total & ~int64_t(15)) : fe;
                if (fe > f0) bulk_prefetch_l2(a.in.data + f0, uint32_t(fe - f0));
            }
        }
        p.issued += uint32_t(n);
    };
    // wait (bounded) for the oldest issued row; false on a timeout
    auto arrive = [&]() -> bool {
        const int stage = int(p.consumed % kWarpStages);
        const bool got = mbar_wait(&p.bars[stage], (p.consumed / kWarpStages) & 1u);
        return __all_sync(0xffffffffu, got);
    };

    // PAIR: rows are issued two at a time, when a pair of stages has been
    // consumed (half the issue instructions per row, more registers); else one
    // at a time, D - 1 rows ahead of the one being consumed.
    // prologue: the rows up to kWarpPrefetch - 1 that no issue prefetches go
    // to L2, then the first rows (D of them in pairs, D - 1 singly) in flight
    static_assert(kWarpStages == 4, "rows are issued in pairs into two of four stages");
    constexpr int kFirst = PAIR ? D : D - 1;
    if (al16 && lane == 0) {
        Cursor c = cursor_at(kFirst);
        for (int32_t i = kFirst; i < kWarpPrefetch && i < T; ++i, step(c)) {
            const int64_t f0 = c.off & ~int64_t(15);
            int64_t fe = (f0 + seg_bytes + 31) & ~int64_t(15);
            fe = fe > (total & ~int64_t(15)) ? (total & ~int64_t(15)) : fe;
            if (fe > f0) bulk_prefetch_l2(a.in.data + f0, uint32_t(fe - f0));
        }
    }
    if (PAIR) {
        issue2(0, min(T, 2));
        if (T > 2) issue2(2, min(T - 2, 2));
    } else {
        for (int32_t i = 0; i < D - 1 && i < T; ++i) issue2(i, 1);
    }
    uint32_t vacc[B];
#pragma unroll
    for (int b = 0; b < B; ++b) vacc[b] = 0;
    int32_t coy = oy0, ck = 0;  // output row and source row within it being consumed
    for (int32_t i = 0; i < T; ++i) {
        if (!PAIR && i + D - 1 < T) issue2(i + D - 1, 1);
        if (!arrive()) {
            p.ok = false;
            break;
        }
        const uint32_t cst = p.consumed % kWarpStages;
        const uint8_t* row = wbuf + cst * rb + (al16 ? (leads >> (8 * cst)) & 0xFFu : 0u);
        uint32_t sums[B];
#pragma unroll
        for (int b = 0; b < B; ++b) sums[b] = 0;
        if (mine) {
            if (!inside) {
                if (part == 0) box_sums_edge<B>(row, fcol, fh, c_lo, a.in.w, premul, sums);
            } else if (premul4) {
                box_sums_premul4_rot(row + off, npix, q0, *reinterpret_cast<uint32_t(*)[4]>(sums));
            } else if (premul && B == 2) {
                box_sums_premul2_u8(row + off, npix, *reinterpret_cast<uint32_t(*)[2]>(sums));
            } else if (npix > 0) {
                box_sums_u8<B>(row + off, npix, sums);
            }
        }
        // the parts of a pixel's box sit pw lanes apart
        for (int m = 16; m >= pw; m >>= 1) {
#pragma unroll
            for (int b = 0; b < B; ++b) sums[b] += __shfl_xor_sync(0xffffffffu, sums[b], m);
        }
#pragma unroll
        for (int b = 0; b < B; ++b) vacc[b] += round_box(sums[b], a.hmul, a.hadd);
        if (++ck == fv) {
            if (mine && part == 0) {
                uint32_t o[B];
#pragma unroll
                for (int b = 0; b < B; ++b) o[b] = round_box(vacc[b], a.vmul, a.vadd);
                if (a.unpremul_out) {
#pragma unroll
                    for (int b = 0; b < B - 1; ++b) o[b] = unpremultiply_u8(o[b], o[B - 1]);
                }
                uint8_t* dst = a.out.data + (int64_t)coy * a.out.pitch + (int64_t)x * B;
                if (B == 4 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
                    *reinterpret_cast<uint32_t*>(dst) = o[0] | (o[1 % B] << 8) | (o[2 % B] << 16) | (o[3 % B] << 24);
                } else {
#pragma unroll
                    for (int b = 0; b < B; ++b) dst[b] = uint8_t(o[b]);
                }
            }
#pragma unroll
            for (int b = 0; b < B; ++b) vacc[b] = 0;
            ck = 0;
            ++coy;
        }
        ++p.consumed;
        __syncwarp();  // every lane is done with the stage before it is refilled
        // a pair of rows consumed: their two stages take rows i + 3 and i + 4
        if (PAIR && (i & 1) && i + 3 < T) issue2(i + 3, min(T - (i + 3), 2));
    }
    if (!p.ok) {
        // record the timeout, then let the copies still in flight land (bounded)
        if (lane == 0 && a.err) atomicExch(a.err, VIPRS_ERR_TIMEOUT);
        while (p.consumed < p.issued) {
            mbar_wait(&p.bars[p.consumed % kWarpStages], (p.consumed / kWarpStages) & 1u);
            ++p.consumed;
        }
        __syncwarp();
    }
}

// Work items of one shrink stage: bands of a.rows_per_item output rows x
// groups of pw output columns.
__device__ __forceinline__ int32_t warp_items(const ShrinkArgs& a) {
    const int32_t groups = (a.out.w + a.nxf - 1) / a.nxf;
    return ((a.out.h + a.rows_per_item - 1) / a.rows_per_item) * groups;
}

template <int B, bool PAIR>
__device__ __forceinline__ void shrink_warp_index(const ShrinkArgs& a, int32_t item, uint8_t* wbuf, WarpPipe& p) {
    const int32_t groups = (a.out.w + a.nxf - 1) / a.nxf;
    const int32_t band = item / groups, g = item - band * groups;
    const int32_t oy0 = band * a.rows_per_item, oy1 = min(a.out.h, oy0 + a.rows_per_item);
    shrink_warp_item<B, PAIR>(a, g * a.nxf, oy0, oy1, wbuf, p);
}

// Standalone ShrinkH+ShrinkV (u8, B <= 4 bands): warp w of the grid takes
// items w, w + (warps in the grid), ...  Each warp's shared memory: its
// barriers (kWarpBars bytes), then kWarpStages buffers of a.row_cap bytes.
template <int B>
__global__ void __launch_bounds__(256) shrink_warp_kernel(ShrinkArgs a) {
    extern __shared__ __align__(128) uint8_t smem_sw[];
    const int warp = threadIdx.x >> 5;
    uint8_t* mine = smem_sw + size_t(warp) * (kWarpBars + size_t(kWarpStages) * a.row_cap);
    WarpPipe p;
    warp_pipe_init(p, mine);
    uint8_t* wbuf = mine + kWarpBars;
    const int32_t n = warp_items(a);
    const int32_t stride = int32_t(gridDim.x) * (blockDim.x >> 5);
    for (int32_t item = int32_t(blockIdx.x) * (blockDim.x >> 5) + warp; item < n && p.ok; item += stride)
        shrink_warp_index<B, true>(a, item, wbuf, p);
}

}  // namespace dev
}  // namespace viprs
