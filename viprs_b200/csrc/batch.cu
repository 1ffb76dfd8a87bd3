// batch.cu -- the persistent batched-thumbnail kernel (sm_100a).
//
// One launch processes the thumbnails of many images of uneven size.  Blocks
// (resident on every SM) claim work items from a device list with an atomic
// cursor; an item is one piece of one stage of one image's plan:
//   shrink   (band of output rows, column chunk)  ShrinkH+ShrinkV
//   reduce2d (output tile)                        fused ReduceH+ReduceV
//   reduce h/v (output row chunk)                 one reduce pass
//   affine   (output row)                         the bicubic correction (rare)
//   pixel    (output row)                         copy / premultiply / unpremultiply
//
// Each block is warp-specialised.  The producer warp (thread kCThreads) claims
// items ahead of the consumers into a small queue and, for shrink items, issues
// the source row segments as TMA bulk copies into the block's ring (the
// warp-specialised ring of resample_dev.cuh), so the copies of the next items
// are in flight while the consumers finish the current one.  The eight
// consumer warps process the items in queue order; block-wide steps among them
// use barrier 1 (256 threads), which the producer never joins.
//
// A stage waits for the stage it reads: one consumer thread polls the producer
// stage's completion counter with an acquire load, bounded by kMaxPolls and
// 2 s; producers publish with __threadfence() + atomicAdd after the item's
// stores.  Items are claimed in list order and each block runs its claimed
// items in that order, so the earliest unfinished item never waits on a later
// one.  Every wait is bounded; a timeout is recorded as VIPRS_ERR_TIMEOUT and
// the block drains its in-flight copies before it exits.
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

constexpr int kQueue = 3;  // items the producer may hold ahead of the consumers

// Control block at the start of the dynamic shared memory.
struct BatchCtl {
    WsRing ring;
    uint64_t qfull[kQueue];   // producer published the entry (1 arrival)
    uint64_t qempty[kQueue];  // consumers read the entry (1 arrival)
    int32_t qidx[kQueue];     // work-list index, or >= n_items: no more work
    int32_t cur;              // consumers: the item being processed
    int32_t go;               // consumers: the item's dependency is satisfied
    int32_t cstop;            // consumers: a bounded wait gave up
    int32_t pstop;            // producer: a bounded wait gave up
};

// Band of output rows and column chunk of shrink item `index`.
__device__ __forceinline__ void shrink_item_geom(const BatchStage& st, const ShrinkArgs& a, int32_t index,
                                                 int32_t* oy0, int32_t* oy1, ShrinkChunk* c) {
    const int32_t band = index / st.n_chunks;
    *oy0 = band * st.rows_per_item;
    *oy1 = min(a.out.h, *oy0 + st.rows_per_item);
    *c = shrink_chunk(a, index - band * st.n_chunks);
}

__device__ __forceinline__ const uint8_t* shrink_source(const BatchArgs& g, const BatchStage& st) {
    return st.in_src ? reinterpret_cast<const uint8_t*>(g.srcs[st.image]) : st.sh.in.data;
}

// Producer (one thread): claim items, publish them, stream shrink rows.
template <int B>
__device__ bool produce_shrink(const BatchArgs& g, const BatchStage& st, int32_t index, BatchCtl* ctl, uint8_t* bufs,
                               int& slot, uint32_t& ph, int64_t& issued) {
    const uint8_t* in = shrink_source(g, st);
    if ((reinterpret_cast<uintptr_t>(in) & 15) != 0) return true;  // consumers take the plain-load path
    int32_t oy0, oy1;
    ShrinkChunk c;
    shrink_item_geom(st, st.sh, index, &oy0, &oy1, &c);
    return ws_produce<B>(st.sh, in, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph,
                         issued);
}

template <bool RING>
__device__ void batch_producer(const BatchArgs& g, BatchCtl* ctl, uint8_t* bufs) {
    int q = 0;
    uint32_t qph = 0;
    int slot = 0;
    uint32_t ph = 0;
    int64_t issued = 0;
    for (;;) {
        if (!mbar_wait(&ctl->qempty[q], qph ^ 1u)) {
            ctl->pstop = 1;
            break;
        }
        const int32_t idx = ctl->pstop ? g.n_items : atomicAdd(g.cursor, 1);
        ctl->qidx[q] = idx;
        mbar_arrive(&ctl->qfull[q]);  // releases the qidx store
        if (++q == kQueue) { q = 0; qph ^= 1u; }
        if (idx >= g.n_items) break;
        if constexpr (!RING) continue;
        const WorkItem it = g.items[idx];
        const BatchStage& st = g.stages[it.stage];
        if (st.type != kBatchShrink) continue;
        bool ok;
        switch (st.sh.bands) {
        case 1: ok = produce_shrink<1>(g, st, it.index, ctl, bufs, slot, ph, issued); break;
        case 2: ok = produce_shrink<2>(g, st, it.index, ctl, bufs, slot, ph, issued); break;
        case 3: ok = produce_shrink<3>(g, st, it.index, ctl, bufs, slot, ph, issued); break;
        default: ok = produce_shrink<4>(g, st, it.index, ctl, bufs, slot, ph, issued); break;
        }
        if (!ok) {
            ctl->pstop = 1;
            atomicExch(g.err, VIPRS_ERR_TIMEOUT);
            // publish an end marker if a queue slot frees, so consumers stop promptly
            if (mbar_wait(&ctl->qempty[q], qph ^ 1u)) {
                ctl->qidx[q] = g.n_items;
                mbar_arrive(&ctl->qfull[q]);
            }
            break;
        }
    }
    ws_drain(&ctl->ring, g.ring_slots, issued);
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
        return ws_consume<B, 2>(a, oy0, oy1, c, &ctl->ring, bufs, g.ring_stage_bytes, g.ring_slots, slot, ph,
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
__device__ void batch_consumers(const BatchArgs& g, BatchCtl* ctl, BatchStage* sst, const uint8_t* bufs,
                                uint8_t* work) {
    int q = 0;
    uint32_t qph = 0;
    int slot = 0;
    uint32_t ph = 0;
    for (;;) {
        // next queue entry: one thread waits, everyone reads the same answer
        // (decisions that every consumer takes are read from fields that only
        // thread 0 writes before the barrier and nobody rewrites until all
        // consumers have passed the next barrier: `cur` and `go`)
        if (threadIdx.x == 0) {
            int32_t idx = g.n_items;
            if (!ctl->cstop) {
                if (mbar_wait(&ctl->qfull[q], qph)) idx = ctl->qidx[q];
                else ctl->cstop = 1;
            }
            ctl->cur = idx;
        }
        csync();
        const int32_t idx = ctl->cur;
        if (idx >= g.n_items) break;
        const WorkItem it = g.items[idx];
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(g.stages + it.stage);
            uint32_t* dst = reinterpret_cast<uint32_t*>(sst);
            for (int i = threadIdx.x; i < int(sizeof(BatchStage) / 4); i += kCThreads) dst[i] = src[i];
        }
        csync();
        if (threadIdx.x == 0) {
            mbar_arrive(&ctl->qempty[q]);
            BatchStage& s = *sst;
            const uint8_t* in = reinterpret_cast<const uint8_t*>(g.srcs[s.image]);
            uint8_t* out = reinterpret_cast<uint8_t*>(g.dsts[s.image]);
            if (s.in_src) { s.sh.in.data = in; s.r2.in.data = in; s.px.in.data = in; s.af.in.data = in; s.rd.in.data = in; }
            if (s.out_dst) {
                s.sh.out.data = out; s.r2.out.data = out; s.px.out.data = out; s.af.out.data = out; s.rd.out.data = out;
            }
            ctl->go = 1;
            if (s.dep >= 0) {
                bool done = ld_acquire_i32(g.counters + s.dep) >= s.dep_items;
                const uint64_t t0 = global_ns();
                for (uint32_t i = 0; !done && i < kMaxPolls; ++i) {
                    __nanosleep(64);
                    if (ld_acquire_i32(g.counters + s.dep) >= s.dep_items) done = true;
                    else if ((i & 63) == 63 && global_ns() - t0 > kWaitLimitNs) break;
                }
                if (!done) {
                    ctl->cstop = 1;
                    ctl->go = 0;
                    atomicExch(g.err, VIPRS_ERR_TIMEOUT);
                }
            }
        }
        if (++q == kQueue) { q = 0; qph ^= 1u; }
        csync();
        if (!ctl->go) break;
        const BatchStage& s = *sst;
        bool ok = true;
        if constexpr (RING) {
            // a ring launch runs shrink items only
            switch (s.sh.bands) {
            case 1: ok = consume_shrink<1>(g, s, it.index, ctl, bufs, work, slot, ph); break;
            case 2: ok = consume_shrink<2>(g, s, it.index, ctl, bufs, work, slot, ph); break;
            case 3: ok = consume_shrink<3>(g, s, it.index, ctl, bufs, work, slot, ph); break;
            default: ok = consume_shrink<4>(g, s, it.index, ctl, bufs, work, slot, ph); break;
            }
        } else {
        switch (s.type) {
        case kBatchReduce2D: {
            const int nbx = (s.r2.out.w + s.r2.tile_w - 1) / s.r2.tile_w;
            const int tbx = it.index % nbx, tby = it.index / nbx;
            if (s.r2.bands == 3) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 3>(s.r2, tbx, tby, work);
            else if (s.r2.bands == 4) reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 4>(s.r2, tbx, tby, work);
            else reduce2d_tile<uint8_t, kReduceFixed, kReduceFixed, 0>(s.r2, tbx, tby, work);
            break;
        }
        case kBatchAffine:
            for (int32_t x = threadIdx.x; x < s.af.out.w; x += kCThreads) affine_pixel<uint8_t>(s.af, x, it.index);
            break;
        case kBatchReduceH:
        case kBatchReduceV: {
            const int32_t chunks = (s.rd.out.w * s.rd.bands + kCThreads - 1) / kCThreads;
            const int32_t oy = it.index / chunks, ch = it.index - oy * chunks;
            if (s.type == kBatchReduceH) reduce_h_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            else reduce_v_chunk<uint8_t, kReduceFixed>(s.rd, ch, oy, work);
            break;
        }
        default:
            batch_pixel_row(s.px, it.index);
            break;
        }
        }
        if (!ok && threadIdx.x == 0) atomicExch(g.err, VIPRS_ERR_TIMEOUT);
        csync();  // the item's stores are done in every consumer
        // a timed-out item is not published; the loop top then stops this block
        if (threadIdx.x == 0 && !ctl->cstop) {
            __threadfence();
            atomicAdd(g.counters + it.stage, 1);
        }
    }
}

// RING: a launch of shrink items (the ring in shared memory); otherwise a
// launch of the other item kinds (the work region in shared memory).
template <bool RING>
__global__ void __launch_bounds__(kWsThreads, 3) batch_kernel(BatchArgs g) {
    extern __shared__ __align__(128) uint8_t smem_b[];
    BatchCtl* ctl = reinterpret_cast<BatchCtl*>(smem_b);
    const size_t ctl_bytes = (sizeof(BatchCtl) + 127) / 128 * 128;
    BatchStage* sst = reinterpret_cast<BatchStage*>(smem_b + ctl_bytes);
    uint8_t* bufs = smem_b + ctl_bytes + (sizeof(BatchStage) + 127) / 128 * 128;
    uint8_t* work = bufs + (size_t)g.ring_slots * g.ring_stage_bytes;
    if (threadIdx.x == 0) {
        if (RING) ws_ring_init(&ctl->ring, g.ring_slots);
        for (int i = 0; i < kQueue; ++i) {
            mbar_init(&ctl->qfull[i], 1);
            mbar_init(&ctl->qempty[i], 1);
        }
        ctl->cstop = 0;
        ctl->pstop = 0;
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x >= kCThreads) {
        if (threadIdx.x == kCThreads) batch_producer<RING>(g, ctl, bufs);
        return;
    }
    batch_consumers<RING>(g, ctl, sst, bufs, work);
}

}  // namespace dev

namespace launch {

size_t batch_ctl_bytes() {
    return (sizeof(dev::BatchCtl) + 127) / 128 * 128 + (sizeof(BatchStage) + 127) / 128 * 128;
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
