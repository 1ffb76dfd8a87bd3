// batch.cu -- the persistent batched-thumbnail kernel (sm_100a).
//
// One launch processes the thumbnails of many images of uneven size.  Blocks
// (a few per SM, all resident) claim work items from a device list with an
// atomic cursor; an item is one piece of one stage of one image's plan:
//   shrink   (output row, column chunk)  ShrinkH+ShrinkV, TMA ring as in resample.cu
//   reduce2d (output tile)               fused ReduceH+ReduceV
//   affine   (output row)                the bicubic correction (rare)
//   pixel    (output row)                copy / premultiply / unpremultiply
// A stage waits for the stage it reads: thread 0 polls the producer stage's
// completion counter with an acquire load, bounded by kMaxPolls; on timeout
// the block records VIPRS_ERR_TIMEOUT and stops claiming work.  Producers
// publish with __threadfence() + atomicAdd after the block's stores.
#include "affine_dev.cuh"
#include "batch_launch.hpp"
#include "resample_dev.cuh"

namespace viprs {
namespace dev {

__device__ __forceinline__ int32_t ld_acquire_i32(const int32_t* p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr int kRing = 4;

// One interior shrink item -- output rows [oy0, oy1) of a column chunk --
// through the TMA ring.  The item's source rows are consecutive plane rows
// (oy0 * fv + k), so the ring streams them without a break at output-row
// boundaries.  `pos` counts ring loads issued so far by this block (identical
// in every thread).  Returns false on a timed-out copy.
template <int B>
__device__ bool batch_shrink_interior(const ShrinkArgs& a, int32_t oy0, int32_t oy1, int32_t c0, int32_t ncols,
                                      uint64_t* bars, uint8_t* bufs, uint32_t stage_bytes, int64_t& pos,
                                      volatile int32_t* flag) {
    const int32_t fh = int32_t(a.fh), fv = int32_t(a.fv);
    const int64_t sbase = ((a.out.x0 + c0) * (int64_t)fh - a.in.x0) * B;
    const int64_t row0 = (a.out.y0 + oy0) * (int64_t)fv - a.in.y0;
    const int32_t nbytes = ncols * fh * B;
    const int32_t total = (oy1 - oy0) * fv;
    auto span = [&](int32_t k, int64_t* as, uint32_t* bytes, int32_t* lead) {
        int64_t ly = row0 + k;
        ly = ly < 0 ? 0 : (ly >= a.in.h ? a.in.h - 1 : ly);
        const int64_t s0 = ly * a.in.pitch + sbase;
        *as = s0 & ~int64_t(15);
        *bytes = uint32_t(((s0 + nbytes + 15) & ~int64_t(15)) - *as);
        *lead = int32_t(s0 - *as);
    };
    auto issue = [&](int32_t k) {
        int64_t as; uint32_t bytes; int32_t lead;
        span(k, &as, &bytes, &lead);
        const int st = int((pos + k) & (kRing - 1));
        mbar_arrive_expect_tx(&bars[st], bytes);
        bulk_load(bufs + (size_t)st * stage_bytes, a.in.data + as, bytes, &bars[st]);
    };
    const int32_t first = total < kRing ? total : kRing;
    if (threadIdx.x == 0)
        for (int32_t k = 0; k < first; ++k) issue(k);
    uint32_t vacc[B];
#pragma unroll
    for (int b = 0; b < B; ++b) vacc[b] = 0;
    const int32_t x = threadIdx.x;
    const uint32_t hhalf = uint32_t(fh) / 2;
    const bool hmult = a.hmode == 3;
    bool ok = true;
    int32_t k = 0, kv = 0, oy = oy0;
    for (; k < total; ++k) {
        const int st = int((pos + k) & (kRing - 1));
        const uint32_t parity = uint32_t(((pos + k) / kRing) & 1);
        if (threadIdx.x == 0 && !mbar_wait(&bars[st], parity)) *flag = 1;
        __syncthreads();
        if (*flag) { ok = false; break; }
        int64_t as; uint32_t bytes; int32_t lead;
        span(k, &as, &bytes, &lead);
        uint8_t* row = bufs + (size_t)st * stage_bytes + lead;
        if (a.premul_in) {
            premultiply_pixels<B>(row, ncols * fh);
            __syncthreads();
        }
        if (x < ncols) {
            uint32_t sums[B];
            box_sums_u8<B>(row + x * fh * B, fh, sums);
            if (hmult) {
#pragma unroll
                for (int b = 0; b < B; ++b) vacc[b] += round_mult_u8(sums[b], hhalf, a.hmult);
            } else {
#pragma unroll
                for (int b = 0; b < B; ++b) vacc[b] += round_mode_u8(sums[b], a.hmode, uint32_t(fh), a.hmult);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && k + kRing < total) {
            fence_proxy_async_smem();
            issue(k + kRing);
        }
        if (++kv == fv) {
            if (x < ncols) {
                uint8_t o[B];
#pragma unroll
                for (int b = 0; b < B; ++b) o[b] = (uint8_t)round_mode_u8(vacc[b], a.vmode, uint32_t(fv), a.vmult);
                if (a.unpremul_out) {
#pragma unroll
                    for (int b = 0; b < B - 1; ++b) o[b] = (uint8_t)unpremultiply_u8(o[b], o[B - 1]);
                }
                uint8_t* dst = a.out.data + (int64_t)oy * a.out.pitch + (int64_t)(c0 + x) * B;
#pragma unroll
                for (int b = 0; b < B; ++b) dst[b] = o[b];
            }
#pragma unroll
            for (int b = 0; b < B; ++b) vacc[b] = 0;
            kv = 0;
            ++oy;
        }
    }
    if (!ok) {
        // wait (bounded) for the copies of this item still in flight
        if (threadIdx.x == 0) {
            const int32_t last = (k + kRing < total) ? k + kRing : total;
            for (int32_t kk = k + 1; kk < last; ++kk)
                mbar_wait(&bars[(pos + kk) & (kRing - 1)], uint32_t(((pos + kk) / kRing) & 1));
        }
        __syncthreads();
        return false;
    }
    pos += total;
    return true;
}

template <int B>
__device__ bool batch_shrink_item(const BatchStage& st, const ShrinkArgs& a, int32_t index, uint64_t* bars,
                                  uint8_t* work, uint32_t stage_bytes, int64_t& pos, volatile int32_t* flag) {
    const int32_t band = index / st.n_chunks;
    int32_t c = index - band * st.n_chunks;
    const int32_t oy0 = band * st.rows_per_item, oy1 = min(a.out.h, oy0 + st.rows_per_item);
    const int32_t left = st.lo > 0 ? 1 : 0;
    const int32_t n_int = st.hi > st.lo ? (st.hi - st.lo + st.chunk_cols - 1) / st.chunk_cols : 0;
    int32_t c0, c1;
    bool interior = false;
    if (c < left) { c0 = 0; c1 = st.lo; }
    else if (c - left < n_int) {
        c0 = st.lo + (c - left) * st.chunk_cols;
        c1 = min(st.hi, c0 + st.chunk_cols);
        interior = true;
    } else { c0 = st.hi; c1 = a.out.w; }
    if (c1 <= c0 || oy1 <= oy0) return true;
    // the bulk copy needs a 16-byte aligned source buffer
    if (interior && (reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0)
        return batch_shrink_interior<B>(a, oy0, oy1, c0, c1 - c0, bars, work, stage_bytes, pos, flag);
    // edge (or unaligned) columns: clamped loads, a few columns at a time
    const int32_t per_col = int32_t(a.fv) * int32_t(a.fh) * B;
    const int32_t step = max(1, int32_t((kRing * stage_bytes - 64) / (per_col + B)));
    for (int32_t oy = oy0; oy < oy1; ++oy)
        for (int32_t x0 = c0; x0 < c1; x0 += step) shrink_edge_item_u8<B>(a, oy, x0, min(c1, x0 + step), work);
    return true;
}

__device__ void batch_pixel_row(const PixelArgs& a, int32_t ly) {
    const int bands = a.bands;
    const uint8_t* src = a.in.data + (int64_t)ly * a.in.pitch;
    uint8_t* dst = a.out.data + (int64_t)ly * a.out.pitch;
    for (int32_t x = threadIdx.x; x < a.out.w; x += blockDim.x) {
        const uint8_t* s = src + (int64_t)x * bands;
        uint8_t* d = dst + (int64_t)x * bands;
        if (a.op == 0 || bands < 2) {
            for (int b = 0; b < bands; ++b) d[b] = s[b];
        } else {
            const uint32_t al = s[bands - 1];
            for (int b = 0; b < bands - 1; ++b)
                d[b] = (uint8_t)(a.op == 1 ? premultiply_u8(s[b], al) : unpremultiply_u8(s[b], al));
            d[bands - 1] = s[bands - 1];
        }
    }
}

__global__ void __launch_bounds__(256) batch_kernel(BatchArgs g) {
    extern __shared__ __align__(128) uint8_t smem_b[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_b);
    volatile int32_t* flag = reinterpret_cast<volatile int32_t*>(smem_b + 64);
    volatile int32_t* sidx = reinterpret_cast<volatile int32_t*>(smem_b + 72);
    BatchStage* sst = reinterpret_cast<BatchStage*>(smem_b + 128);
    uint8_t* work = smem_b + 128 + ((sizeof(BatchStage) + 127) / 128) * 128;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) mbar_init(&bars[i], 1);
        *flag = 0;
        mbar_fence_init();
    }
    __syncthreads();
    int64_t pos = 0;
    for (;;) {
        if (threadIdx.x == 0) *sidx = atomicAdd(g.cursor, 1);
        __syncthreads();
        const int32_t idx = *sidx;
        if (idx >= g.n_items) break;
        const WorkItem it = g.items[idx];
        // stage descriptor into shared memory, plane pointers resolved for this launch
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(g.stages + it.stage);
            uint32_t* dst = reinterpret_cast<uint32_t*>(sst);
            for (int i = threadIdx.x; i < int(sizeof(BatchStage) / 4); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            BatchStage& s = *sst;
            const uint8_t* in = reinterpret_cast<const uint8_t*>(g.srcs[s.image]);
            uint8_t* out = reinterpret_cast<uint8_t*>(g.dsts[s.image]);
            if (s.in_src) { s.sh.in.data = in; s.r2.in.data = in; s.px.in.data = in; s.af.in.data = in; s.rd.in.data = in; }
            if (s.out_dst) {
                s.sh.out.data = out; s.r2.out.data = out; s.px.out.data = out; s.af.out.data = out; s.rd.out.data = out;
            }
            if (s.dep >= 0) {
                bool done = ld_acquire_i32(g.counters + s.dep) >= s.dep_items;
                const uint64_t t0 = global_ns();
                for (uint32_t i = 0; !done && i < kMaxPolls; ++i) {
                    __nanosleep(64);
                    if (ld_acquire_i32(g.counters + s.dep) >= s.dep_items) done = true;
                    else if ((i & 63) == 63 && global_ns() - t0 > kWaitLimitNs) break;
                }
                if (!done) {
                    *flag = 1;
                    atomicExch(g.err, VIPRS_ERR_TIMEOUT);
                }
            }
        }
        __syncthreads();
        if (*flag) break;
        const BatchStage& s = *sst;
        bool ok = true;
        switch (s.type) {
        case kBatchShrink:
            switch (s.sh.bands) {
            case 1: ok = batch_shrink_item<1>(s, s.sh, it.index, bars, work, g.ring_stage_bytes, pos, flag); break;
            case 2: ok = batch_shrink_item<2>(s, s.sh, it.index, bars, work, g.ring_stage_bytes, pos, flag); break;
            case 3: ok = batch_shrink_item<3>(s, s.sh, it.index, bars, work, g.ring_stage_bytes, pos, flag); break;
            default: ok = batch_shrink_item<4>(s, s.sh, it.index, bars, work, g.ring_stage_bytes, pos, flag); break;
            }
            break;
        case kBatchReduce2D: {
            const int nbx = (s.r2.out.w + s.r2.tile_w - 1) / s.r2.tile_w;
            const int tbx = it.index % nbx, tby = it.index / nbx;
            if (s.r2.bands == 3) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 3>(s.r2, tbx, tby, work);
            else if (s.r2.bands == 4) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 4>(s.r2, tbx, tby, work);
            else reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 0>(s.r2, tbx, tby, work);
            break;
        }
        case kBatchAffine:
            for (int32_t x = threadIdx.x; x < s.af.out.w; x += blockDim.x) affine_pixel<uint8_t>(s.af, x, it.index);
            break;
        case kBatchReduceH:
        case kBatchReduceV: {
            const int32_t chunks = (s.rd.out.w * s.rd.bands + 255) / 256;
            const int32_t oy = it.index / chunks, ch = it.index - oy * chunks;
            if (s.type == kBatchReduceH) reduce_h_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            else reduce_v_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            break;
        }
        default:
            batch_pixel_row(s.px, it.index);
            break;
        }
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(g.err, VIPRS_ERR_TIMEOUT);
            break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(g.counters + it.stage, 1);
        }
    }
}

}  // namespace dev

namespace launch {

int batch_blocks_per_sm(size_t smem) {
    cudaFuncSetAttribute(dev::batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::batch_kernel, 256, smem);
    return per_sm;
}

cudaError_t batch(const BatchArgs& a, int grid, cudaStream_t s) {
    if (a.n_items <= 0) return cudaSuccess;
    cudaFuncSetAttribute(dev::batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem_bytes);
    dev::batch_kernel<<<grid, 256, a.smem_bytes, s>>>(a);
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
