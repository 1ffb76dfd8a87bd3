// batch.cu -- the persistent batched-thumbnail kernel (sm_100a).
//
// A few launches process the thumbnails of many images of uneven size.  Blocks
// (resident on every SM) claim work items from a device list with an atomic
// cursor; an item is one piece of one stage of one image's plan:
//   shrink   (band of output rows, column chunk)  ShrinkH+ShrinkV
//   reduce2d (output tile)                        fused ReduceH+ReduceV
//   reduce h/v (output row chunk)                 one reduce pass
//   affine   (output row)                         the bicubic correction (rare)
//   pixel    (output row)                         copy / premultiply / unpremultiply
//
// Each block is warp-specialised.  The producer warp (threads kCThreads..)
// claims items one ahead of its queue, copies each item's stage descriptor
// into a queue slot in shared memory (pointers resolved for this launch) and,
// for shrink items, issues the source row segments as TMA bulk copies into the
// block's ring (the warp-specialised ring of resample_dev.cuh), so the next
// items are ready while the consumers finish the current one.  The eight
// consumer warps run the items in queue order; block-wide steps among them use
// barrier 1 (256 threads), which the producer never joins.
//
// The batch runs as one launch per stage level and kind (batch_plan.cpp), so
// an item's input is complete when its launch starts.  Every wait is bounded;
// a timeout is recorded as VIPRS_ERR_TIMEOUT and the producer drains its
// in-flight copies before the block exits.
#include "affine_dev.cuh"
#include "batch_launch.hpp"
#include "resample_dev.cuh"

namespace viprs {
namespace dev {

constexpr int kQueue = 3;  // items the producer may prepare ahead of the consumers

// Control block at the start of the dynamic shared memory.
struct BatchCtl {
    WsRing ring;
    uint64_t qfull[kQueue];   // producer prepared the entry (1 arrival)
    uint64_t qempty[kQueue];  // consumers finished the entry's item (1 arrival)
    int32_t qidx[kQueue];     // work item index within the stage, or -1: no more work
    int32_t cur;              // consumers: the queue entry's item index, or -1
    int32_t cstop;            // consumers: a bounded wait gave up
};

// Band of output rows and column chunk of shrink item `index`.
__device__ __forceinline__ void shrink_item_geom(const BatchStage& st, const ShrinkArgs& a, int32_t index,
                                                 int32_t* oy0, int32_t* oy1, ShrinkChunk* c) {
    const int32_t band = index / st.n_chunks;
    *oy0 = band * st.rows_per_item;
    *oy1 = min(a.out.h, *oy0 + st.rows_per_item);
    *c = shrink_chunk(a, index - band * st.n_chunks);
}

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
// current item), prepare each in a queue slot, publish it, and for shrink
// items stream the source rows into the ring (lane 0).
template <bool RING>
__device__ void batch_producer(const BatchArgs& g, BatchCtl* ctl, BatchStage* qstage, uint8_t* bufs) {
    const int lane = threadIdx.x & 31;
    int q = 0;
    uint32_t qph = 0;
    int slot = 0;
    uint32_t ph = 0;
    int64_t issued = 0;
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
        const int pq = q;
        if (++q == kQueue) { q = 0; qph ^= 1u; }
        if (!more) break;
        if constexpr (RING) {
            if (lane == 0) {
                const BatchStage& st = qstage[pq];
                const ShrinkArgs& a = st.sh;
                if ((reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0) {
                    int32_t oy0, oy1;
                    ShrinkChunk c;
                    shrink_item_geom(st, a, it.index, &oy0, &oy1, &c);
                    bool r;
                    switch (a.bands) {
                    case 1: r = ws_produce<1>(a, a.in.data, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph, issued); break;
                    case 2: r = ws_produce<2>(a, a.in.data, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph, issued); break;
                    case 3: r = ws_produce<3>(a, a.in.data, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph, issued); break;
                    default: r = ws_produce<4>(a, a.in.data, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph, issued); break;
                    }
                    ok = r ? 1 : 0;
                }
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) { fail = true; break; }
        }
        idx = __shfl_sync(0xffffffffu, next, 0);
    }
    if (lane == 0) {
        if (fail) {
            atomicExch(g.err, VIPRS_ERR_TIMEOUT);
            // publish an end marker if a queue slot frees, so consumers stop promptly
            if (mbar_wait(&ctl->qempty[q], qph ^ 1u)) {
                ctl->qidx[q] = -1;
                mbar_arrive(&ctl->qfull[q]);
            }
        }
        if (RING) ws_drain(&ctl->ring, g.ring_slots, issued);
    }
}

// Consumers: one shrink item.
template <int B>
__device__ bool consume_shrink(const BatchArgs& g, const BatchStage& st, int32_t index, BatchCtl* ctl,
                               const uint8_t* bufs, uint8_t* work, int& slot, uint32_t& ph) {
    const ShrinkArgs& a = st.sh;
    int32_t oy0, oy1;
    ShrinkChunk c;
    shrink_item_geom(st, a, index, &oy0, &oy1, &c);
    if ((reinterpret_cast<uintptr_t>(a.in.data) & 15) == 0)
        return ws_consume<B>(a, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph,
                             reinterpret_cast<volatile int32_t*>(&ctl->cstop));
    // unaligned source: clamped plain loads, a few columns at a time
    const int32_t per_col = int32_t(a.fv) * int32_t(a.fh) * B;
    const int32_t step = max(1, int32_t((g.work_bytes - 64) / (per_col + B)));
    for (int32_t oy = oy0; oy < oy1; ++oy)
        for (int32_t x0 = c.lx0; x0 < c.lx0 + c.ncols; x0 += step)
            shrink_edge_item_u8<B>(a, oy, x0, min(c.lx0 + c.ncols, x0 + step), work);
    return true;
}

__device__ void batch_pixel_row(const PixelArgs& a, int32_t ly) {
    const int bands = a.bands;
    const uint8_t* src = a.in.data + (int64_t)ly * a.in.pitch;
    uint8_t* dst = a.out.data + (int64_t)ly * a.out.pitch;
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

template <bool RING>
__device__ void batch_consumers(const BatchArgs& g, BatchCtl* ctl, const BatchStage* qstage, const uint8_t* bufs,
                                uint8_t* work) {
    int q = 0;
    uint32_t qph = 0;
    int slot = 0;
    uint32_t ph = 0;
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
        bool ok = true;
        if constexpr (RING) {
            // a ring launch runs shrink items only
            switch (s.sh.bands) {
            case 1: ok = consume_shrink<1>(g, s, index, ctl, bufs, work, slot, ph); break;
            case 2: ok = consume_shrink<2>(g, s, index, ctl, bufs, work, slot, ph); break;
            case 3: ok = consume_shrink<3>(g, s, index, ctl, bufs, work, slot, ph); break;
            default: ok = consume_shrink<4>(g, s, index, ctl, bufs, work, slot, ph); break;
            }
        } else {
            switch (s.type) {
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
        }
        if (!ok && threadIdx.x == 0) atomicExch(g.err, VIPRS_ERR_TIMEOUT);
        csync();  // every consumer is done with the entry
        if (threadIdx.x == 0) mbar_arrive(&ctl->qempty[q]);
        if (++q == kQueue) { q = 0; qph ^= 1u; }
    }
}

// RING: a launch of shrink items (the ring in shared memory); otherwise a
// launch of the other item kinds (the work region in shared memory).
template <bool RING>
__global__ void __launch_bounds__(kWsThreads, RING ? 4 : 3) batch_kernel(BatchArgs g) {
    extern __shared__ __align__(128) uint8_t smem_b[];
    BatchCtl* ctl = reinterpret_cast<BatchCtl*>(smem_b);
    const size_t ctl_bytes = (sizeof(BatchCtl) + 127) / 128 * 128;
    BatchStage* qstage = reinterpret_cast<BatchStage*>(smem_b + ctl_bytes);
    uint8_t* bufs = smem_b + ctl_bytes + kQueue * ((sizeof(BatchStage) + 127) / 128 * 128);
    uint8_t* work = bufs + (size_t)g.ring_slots * g.ring_stage_bytes;
    if (threadIdx.x == 0) {
        if (RING) ws_ring_init(&ctl->ring, g.ring_slots);
        for (int i = 0; i < kQueue; ++i) {
            mbar_init(&ctl->qfull[i], 1);
            mbar_init(&ctl->qempty[i], 1);
        }
        ctl->cstop = 0;
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x >= kCThreads) {
        batch_producer<RING>(g, ctl, qstage, bufs);
        return;
    }
    batch_consumers<RING>(g, ctl, qstage, bufs, work);
}

}  // namespace dev

namespace launch {

size_t batch_ctl_bytes() {
    return (sizeof(dev::BatchCtl) + 127) / 128 * 128 + dev::kQueue * ((sizeof(BatchStage) + 127) / 128 * 128);
}

int batch_blocks_per_sm(size_t smem, bool ring) {
    void (*k)(BatchArgs) = ring ? dev::batch_kernel<true> : dev::batch_kernel<false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, dev::kWsThreads, smem);
    return per_sm;
}

cudaError_t batch(const BatchArgs& a, int grid, bool ring, cudaStream_t s) {
    if (a.n_items <= 0) return cudaSuccess;
    void (*k)(BatchArgs) = ring ? dev::batch_kernel<true> : dev::batch_kernel<false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.smem_bytes);
    k<<<grid, dev::kWsThreads, a.smem_bytes, s>>>(a);
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
