// batch.cu -- the persistent batched-thumbnail kernels (sm_100a).
//
// A few launches process the thumbnails of many images of uneven size.  Each
// launch walks a device work list with an atomic cursor; an item is one
// piece of one stage of one image's plan:
//   shrink   (band of output rows, group of pw output columns)  ShrinkH+ShrinkV
//   reduce2d (output tile)                                      fused ReduceH+ReduceV
//   reduce h/v (output row chunk)                               one reduce pass
//   affine   (output row)                                       the bicubic correction (rare)
//   pixel    (output row)                                       copy / premultiply / unpremultiply
//
// Shrink items run in batch_warp_kernel: every warp claims items on its own
// and streams its source rows through its own stage buffers by TMA bulk
// copies (shrink_warp.cuh), so warps never wait for each other.  The other item kinds run in
// batch_kernel: a producer warp (threads kCThreads..) claims items one ahead
// and copies each item's stage descriptor into a queue slot in shared memory
// (pointers resolved for this launch); the eight consumer warps run the items
// in queue order, using barrier 1 (256 threads), which the producer never
// joins.
//
// The batch runs as one launch per stage level and kind (batch_plan.cpp), so
// an item's input is complete when its launch starts.  Every wait of the
// queue is bounded; a timeout is recorded as VIPRS_ERR_TIMEOUT.
#include "affine_dev.cuh"
#include "batch_launch.hpp"
#include "shrink_warp.cuh"

namespace viprs {
namespace dev {

constexpr int kQueue = 3;  // items the producer may prepare ahead of the consumers

// Control block at the start of the dynamic shared memory.
struct BatchCtl {
    uint64_t qfull[kQueue];   // producer prepared the entry (1 arrival)
    uint64_t qempty[kQueue];  // consumers finished the entry's item (1 arrival)
    int32_t qidx[kQueue];     // work item index within the stage, or -1: no more work
    int32_t cur;              // consumers: the queue entry's item index, or -1
    int32_t cstop;            // consumers: a bounded wait gave up
};

// Producer warp: copy stage `stage` into queue slot `dst` (the whole warp) and
// resolve its source / destination pointers for this launch (lane 0).
__device__ __forceinline__ void prepare_stage(const BatchArgs& g, int32_t stage, BatchStage* dst, int lane) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(g.stages + stage);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int i = lane; i < int(sizeof(BatchStage) / 4); i += 32) d[i] = src[i];
    __syncwarp();
    if (lane == 0) {
        BatchStage& s = *dst;
        const uint8_t* in = reinterpret_cast<const uint8_t*>(g.srcs[s.image]);
        uint8_t* out = reinterpret_cast<uint8_t*>(g.dsts[s.image]);
        if (s.in_src) { s.sh.in.data = in; s.r2.in.data = in; s.px.in.data = in; s.af.in.data = in; s.rd.in.data = in; }
        if (s.out_dst) {
            s.sh.out.data = out; s.r2.out.data = out; s.px.out.data = out; s.af.out.data = out; s.rd.out.data = out;
        }
    }
    __syncwarp();
}

// Producer warp: claim items (one ahead, so the atomic's latency overlaps the
// current item), prepare each in a queue slot and publish it.
__device__ void batch_producer(const BatchArgs& g, BatchCtl* ctl, BatchStage* qstage) {
    const int lane = threadIdx.x & 31;
    int q = 0;
    uint32_t qph = 0;
    bool fail = false;
    int32_t idx = 0;
    if (lane == 0) idx = atomicAdd(g.cursor, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    for (;;) {
        int ok = 1;
        if (lane == 0) ok = mbar_wait(&ctl->qempty[q], qph ^ 1u) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) { fail = true; break; }
        const bool more = idx < g.n_items;
        int32_t next = g.n_items;
        WorkItem it = {0, 0};
        if (more) {
            if (lane == 0) next = atomicAdd(g.cursor, 1);  // used one iteration later
            it = g.items[idx];
            prepare_stage(g, it.stage, &qstage[q], lane);
        }
        if (lane == 0) {
            ctl->qidx[q] = more ? it.index : -1;
            mbar_arrive(&ctl->qfull[q]);  // releases the slot's stage and index
        }
        if (++q == kQueue) { q = 0; qph ^= 1u; }
        if (!more) break;
        idx = __shfl_sync(0xffffffffu, next, 0);
    }
    if (lane == 0 && fail) {
        atomicExch(g.err, VIPRS_ERR_TIMEOUT);
        // publish an end marker if a queue slot frees, so consumers stop promptly
        if (mbar_wait(&ctl->qempty[q], qph ^ 1u)) {
            ctl->qidx[q] = -1;
            mbar_arrive(&ctl->qfull[q]);
        }
    }
}

__device__ void batch_pixel_row(const PixelArgs& a, int32_t ly) {
    const int bands = a.bands;
    const uint8_t* src = a.in.data + (int64_t)ly * a.in.pitch;
    uint8_t* dst = a.out.data + (int64_t)ly * a.out.pitch;
    if (a.op == 3) {
        // Zoom: the source row and pixel of each output pixel (zoom.rs:44-104)
        src = a.in.data + ((a.out.y0 + ly) / a.zy - a.in.y0) * a.in.pitch;
        for (int32_t x = threadIdx.x; x < a.out.w; x += kCThreads) {
            const uint8_t* s = src + ((a.out.x0 + x) / a.zx - a.in.x0) * bands;
            uint8_t* d = dst + (int64_t)x * bands;
            for (int b = 0; b < bands; ++b) d[b] = s[b];
        }
        return;
    }
    for (int32_t x = threadIdx.x; x < a.out.w; x += kCThreads) {
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

// R2B 3 or 4: a launch of fused-reduce tiles of R2B-band images only (the
// code of the other item kinds is left out); 0: every item kind.
template <int R2B>
__device__ void batch_consumers(const BatchArgs& g, BatchCtl* ctl, const BatchStage* qstage, uint8_t* work) {
    int q = 0;
    uint32_t qph = 0;
    for (;;) {
        // next queue entry: one thread waits; `cur` is written only by thread 0
        // before the barrier and rewritten only after the next barrier
        if (threadIdx.x == 0) {
            int32_t index = -1;
            if (!ctl->cstop) {
                if (mbar_wait(&ctl->qfull[q], qph)) index = ctl->qidx[q];
                else ctl->cstop = 1;
            }
            ctl->cur = index;
        }
        csync();
        const int32_t index = ctl->cur;
        if (index < 0) break;
        const BatchStage& s = qstage[q];
        if (R2B != 0) {
            const int nbx = (s.r2.out.w + s.r2.tile_w - 1) / s.r2.tile_w;
            reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, R2B>(s.r2, index % nbx, index / nbx, work);
        } else switch (s.type) {
        case kBatchReduce2D: {
            const int nbx = (s.r2.out.w + s.r2.tile_w - 1) / s.r2.tile_w;
            const int tbx = index % nbx, tby = index / nbx;
            if (s.r2.bands == 3) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 3>(s.r2, tbx, tby, work);
            else if (s.r2.bands == 4) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 4>(s.r2, tbx, tby, work);
            else reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 0>(s.r2, tbx, tby, work);
            break;
        }
        case kBatchAffine:
            for (int32_t x = threadIdx.x; x < s.af.out.w; x += kCThreads) affine_pixel<uint8_t>(s.af, x, index);
            break;
        case kBatchReduceH:
        case kBatchReduceV: {
            const int32_t chunks = (s.rd.out.w * s.rd.bands + kCThreads - 1) / kCThreads;
            const int32_t oy = index / chunks, ch = index - oy * chunks;
            if (s.type == kBatchReduceH) reduce_h_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            else reduce_v_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            break;
        }
        default:
            batch_pixel_row(s.px, index);
            break;
        }
        csync();  // every consumer is done with the entry
        if (threadIdx.x == 0) mbar_arrive(&ctl->qempty[q]);
        if (++q == kQueue) { q = 0; qph ^= 1u; }
    }
}

// The other item kinds (fused reduce tiles, reduce rows, affine and pixel
// rows), with the work region in shared memory.
template <int R2B>
__global__ void __launch_bounds__(kWsThreads, 3) batch_kernel(BatchArgs g) {
    extern __shared__ __align__(128) uint8_t smem_b[];
    BatchCtl* ctl = reinterpret_cast<BatchCtl*>(smem_b);
    const size_t ctl_bytes = (sizeof(BatchCtl) + 127) / 128 * 128;
    BatchStage* qstage = reinterpret_cast<BatchStage*>(smem_b + ctl_bytes);
    uint8_t* work = smem_b + ctl_bytes + kQueue * ((sizeof(BatchStage) + 127) / 128 * 128);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kQueue; ++i) {
            mbar_init(&ctl->qfull[i], 1);
            mbar_init(&ctl->qempty[i], 1);
        }
        ctl->cstop = 0;
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x >= kCThreads) {
        batch_producer(g, ctl, qstage);
        return;
    }
    batch_consumers<R2B>(g, ctl, qstage, work);
}

constexpr uint32_t kWarpDesc = (sizeof(ShrinkArgs) + 127) / 128 * 128;

// Shrink items by independent warps: each warp claims items (atomic cursor),
// copies the item's stage descriptor into its own shared memory, resolves the
// image pointers for this launch and runs the item with its own stage
// buffers.  A warp's shared memory: barriers, descriptor, stage buffers.
template <int B>
__global__ void __launch_bounds__(256, 3) batch_warp_kernel(BatchArgs g) {
    extern __shared__ __align__(128) uint8_t smem_w[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t* mine = smem_w + size_t(warp) * (kWarpBars + kWarpDesc + size_t(kWarpStages) * g.ring_stage_bytes);
    WarpPipe p;
    warp_pipe_init(p, mine);
    ShrinkArgs* d = reinterpret_cast<ShrinkArgs*>(mine + kWarpBars);
    uint8_t* wbuf = mine + kWarpBars + kWarpDesc;
    while (p.ok) {
        int32_t idx = 0;
        if (lane == 0) idx = atomicAdd(g.cursor, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= g.n_items) break;
        const WorkItem it = g.items[idx];
        const BatchStage* st = g.stages + it.stage;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&st->sh);
        uint32_t* dst = reinterpret_cast<uint32_t*>(d);
        for (int i = lane; i < int(sizeof(ShrinkArgs) / 4); i += 32) dst[i] = src[i];
        __syncwarp();
        if (lane == 0) {
            if (st->in_src) d->in.data = reinterpret_cast<const uint8_t*>(g.srcs[st->image]);
            if (st->out_dst) d->out.data = reinterpret_cast<uint8_t*>(g.dsts[st->image]);
            d->err = g.err;
        }
        __syncwarp();
        shrink_warp_index<B, true>(*d, it.index, wbuf, p);
        __syncwarp();
    }
}

}  // namespace dev

namespace launch {

size_t batch_ctl_bytes() {
    return (sizeof(dev::BatchCtl) + 127) / 128 * 128 + dev::kQueue * ((sizeof(BatchStage) + 127) / 128 * 128);
}

size_t batch_warp_smem_bytes(uint32_t stage_bytes) {
    return size_t(8) * (dev::kWarpBars + dev::kWarpDesc + size_t(dev::kWarpStages) * stage_bytes);
}

// The persistent kernel of a launch: the tile variant (ring_bands 0) or the
// warp shrink of images with ring_bands bands.
static void (*batch_kernel_of(int ring_bands))(BatchArgs) {
    switch (ring_bands) {
    case 0: return dev::batch_kernel<0>;
    case kBatchTile3: return dev::batch_kernel<3>;
    case kBatchTile4: return dev::batch_kernel<4>;
    case 1: return dev::batch_warp_kernel<1>;
    case 2: return dev::batch_warp_kernel<2>;
    case 3: return dev::batch_warp_kernel<3>;
    default: return dev::batch_warp_kernel<4>;
    }
}

int batch_blocks_per_sm(size_t smem, int ring_bands) {
    void (*k)(BatchArgs) = batch_kernel_of(ring_bands);
    const int threads = ring_bands >= 1 && ring_bands <= 4 ? 256 : dev::kWsThreads;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
    return per_sm;
}

cudaError_t batch(const BatchArgs& a, int grid, int ring_bands, cudaStream_t s) {
    if (a.n_items <= 0) return cudaSuccess;
    void (*k)(BatchArgs) = batch_kernel_of(ring_bands);
    const int threads = ring_bands >= 1 && ring_bands <= 4 ? 256 : dev::kWsThreads;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem_bytes);
    k<<<grid, threads, a.smem_bytes, s>>>(a);
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
