// shrink_warp.cuh -- u8 ShrinkH then ShrinkV (shrinkh.rs:323-397,
// shrinkv.rs:191-339) by independent warps.
//
// A warp owns `pw` consecutive output pixels (32, 16 or 8: 32 / pw lanes
// share one pixel's box) of a band of output rows.  It streams the source row
// segment its boxes cover through a private kWarpStages-deep buffer in shared
// memory with cp.async (16-byte copies, L1 bypassed), so that the next rows
// are in flight while it sums the current one; nothing is shared with other
// warps -- no producer warp, no block barrier, no mbarrier -- and warps pick
// their work independently.  Per source row each lane sums its part of its
// pixel's box (dp4a over realigned words, or premultiplied 4-band pixels),
// the parts are combined with shuffles and rounded as ShrinkH rounds; per
// output row the rounded sums are rounded as ShrinkV rounds, unpremultiplied
// when the chain ends there, and stored.  Boxes that leave the plane (the
// reduce halo beyond the image) read clamped columns from the staged segment.
//
// ShrinkArgs fields used here: nxf = pw, rows_per_item = output rows per
// work item, row_cap = bytes of one stage buffer (source segment + 16-byte
// alignment + 32 bytes of over-read slack), rot_shift = lane rotation of the
// box walk (chosen on the host to spread shared-memory banks).  cp.async
// completes by itself (no flag to spin on), so the warp never waits on
// another warp or thread.
#pragma once

#include "resample_dev.cuh"

namespace viprs {
namespace dev {

constexpr int kWarpStages = 4;  // source rows in flight per warp

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Groups of the dp4a box walk for `npix` pixels of B bands (G words per
// group: 3 for 3 bands, else 1), or pixels for the premultiplied 4-band walk.
__device__ __forceinline__ int warp_walk_groups(int npix, int B, bool premul4) {
    if (premul4) return npix > 0 ? npix : 1;
    const int G = B == 3 ? 3 : 1;
    const int K = (npix * B + 3) >> 2;
    const int Kg = (K + G - 1) / G;
    return Kg > 0 ? Kg : 1;
}

// One work item: output columns [x0, x0 + pw) (local to a.out) of output rows
// [oy0, oy1).  `wbuf`: this warp's kWarpStages * a.row_cap bytes of shared
// memory (16-byte aligned).  Every lane of the warp calls it.
template <int B>
__device__ void shrink_warp_item(const ShrinkArgs& a, int32_t x0, int32_t oy0, int32_t oy1, uint8_t* wbuf) {
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
    const uint32_t sbase = smem_u32(wbuf);
    // this lane's part of its pixel's box: pixels [j0, j1)
    const int32_t j0 = part * fh / lp, j1 = (part + 1) * fh / lp;
    const int32_t npix = j1 - j0;
    const int32_t off = inside ? int32_t(fcol + j0 - c_lo) * B : 0;
    const bool premul = a.premul_in != 0;
    const bool premul4 = premul && B == 4;
    const int q0 = (lane >> a.rot_shift) % warp_walk_groups(npix, B, premul4);
    const int32_t T = (oy1 - oy0) * fv;
    const int64_t total = a.in.total_bytes;

    // source row of flattened row index (oy, k) and its first byte
    auto row_start = [&](int32_t oy, int32_t k) -> int64_t {
        int64_t ly = (a.out.y0 + oy) * (int64_t)fv + k - a.in.y0;
        ly = ly < 0 ? 0 : (ly >= a.in.h ? a.in.h - 1 : ly);
        return ly * a.in.pitch + c_lo * B;
    };
    // A 16-byte aligned plane streams each row segment's aligned cover with
    // cp.async (a copy passing the end of the buffer takes only the bytes
    // inside it); any other plane copies the segment byte by byte.
    const bool al16 = (reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0;
    auto lead_of = [&](int64_t s0) -> uint32_t { return al16 ? uint32_t(s0 & 15) : 0u; };
    // copy row (oy, k) into stage buffer `stage`
    auto issue = [&](int32_t oy, int32_t k, int stage) {
        const int64_t s0 = row_start(oy, k);
        if (!al16) {
            uint8_t* d = wbuf + uint32_t(stage) * rb;
            for (int32_t v = lane; v < int32_t(seg_bytes); v += 32) d[v] = a.in.data[s0 + v];
            return;
        }
        const int64_t as = s0 & ~int64_t(15);
        const int32_t nv = int32_t((((s0 + seg_bytes + 15) & ~int64_t(15)) - as) >> 4);
        const uint32_t dst = sbase + uint32_t(stage) * rb;
        for (int32_t v = lane; v < nv; v += 32) {
            const int64_t g = as + 16 * int64_t(v);
            const int64_t left = total - g;
            if (left > 0) cp_async16(dst + 16u * uint32_t(v), a.in.data + g, left >= 16 ? 16u : uint32_t(left));
        }
    };

    // prologue: rows 0 .. D-2 in flight
    int32_t ioy = oy0, ik = 0;  // next row to issue
    for (int s = 0; s < D - 1; ++s) {
        if (s < T) {
            issue(ioy, ik, s);
            if (++ik == fv) { ik = 0; ++ioy; }
        }
        cp_async_commit();
    }
    uint32_t vacc[B];
#pragma unroll
    for (int b = 0; b < B; ++b) vacc[b] = 0;
    int32_t coy = oy0, ck = 0;  // row being consumed
    for (int32_t i = 0; i < T; ++i) {
        if (i + D - 1 < T) {
            issue(ioy, ik, (i + D - 1) % D);
            if (++ik == fv) { ik = 0; ++ioy; }
        }
        cp_async_commit();
        cp_async_wait<D - 1>();
        __syncwarp();
        const uint8_t* row = wbuf + uint32_t(i % D) * rb + lead_of(row_start(coy, ck));
        uint32_t sums[B];
#pragma unroll
        for (int b = 0; b < B; ++b) sums[b] = 0;
        if (mine) {
            if (!inside) {
                if (part == 0) box_sums_clamped_pm_u8<B>(row, fcol, fh, c_lo, a.in.w, premul, sums);
            } else if (premul4) {
                box_sums_premul4_rot(row + off, npix, q0, *reinterpret_cast<uint32_t(*)[4]>(sums));
            } else if (premul && B == 2) {
                box_sums_premul2_u8(row + off, npix, *reinterpret_cast<uint32_t(*)[2]>(sums));
            } else if (npix > 0) {
                box_sums_rot_u8<B>(row + off, npix, q0, sums);
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
        __syncwarp();
    }
    cp_async_wait<0>();
    __syncwarp();
}

// Work items of one shrink stage: bands of a.rows_per_item output rows x
// groups of pw output columns.
__device__ __forceinline__ int32_t warp_items(const ShrinkArgs& a) {
    const int32_t groups = (a.out.w + a.nxf - 1) / a.nxf;
    return ((a.out.h + a.rows_per_item - 1) / a.rows_per_item) * groups;
}

template <int B>
__device__ __forceinline__ void shrink_warp_index(const ShrinkArgs& a, int32_t item, uint8_t* wbuf) {
    const int32_t groups = (a.out.w + a.nxf - 1) / a.nxf;
    const int32_t band = item / groups, g = item - band * groups;
    const int32_t oy0 = band * a.rows_per_item, oy1 = min(a.out.h, oy0 + a.rows_per_item);
    shrink_warp_item<B>(a, g * a.nxf, oy0, oy1, wbuf);
}

// Standalone ShrinkH+ShrinkV (u8, B <= 4 bands): warp w of the grid takes
// items w, w + (warps in the grid), ...
template <int B>
__global__ void __launch_bounds__(256) shrink_warp_kernel(ShrinkArgs a) {
    extern __shared__ __align__(128) uint8_t smem_sw[];
    const int warp = threadIdx.x >> 5;
    uint8_t* wbuf = smem_sw + size_t(warp) * kWarpStages * a.row_cap;
    const int32_t n = warp_items(a);
    const int32_t stride = int32_t(gridDim.x) * (blockDim.x >> 5);
    for (int32_t item = int32_t(blockIdx.x) * (blockDim.x >> 5) + warp; item < n; item += stride)
        shrink_warp_index<B>(a, item, wbuf);
}

}  // namespace dev
}  // namespace viprs
