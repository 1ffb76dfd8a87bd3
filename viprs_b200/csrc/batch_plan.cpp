// batch_plan.cpp -- batched thumbnails: one plan per image, executed either
// as ONE persistent launch over a device work list (optionally captured in a
// CUDA graph) or image by image (the plain per-image GPU path).
//
// Each image's plan is PipelineBuilder::thumbnail over an in-memory source
// (builder/resample.rs:871-979); the persistent kernel runs exactly the same
// stages with the same tables, so both paths give identical bytes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <memory>
#include <new>
#include <numeric>
#include <vector>

#include "batch_launch.hpp"
#include "chain.hpp"
#include "shrink_warp.hpp"
#include "viprs_b200.h"

using namespace viprs;

// One launch of the persistent kernel: a contiguous range of the work list.
struct BatchLaunch {
    int32_t level = 0;        // stage level: launches of one level are independent
    bool ring = false;        // shrink items (the warp shrink variant)
    int32_t bands = 0;        // kernel variant: the band count of a shrink launch, else 0 or kBatchTile3/4
    int64_t offset = 0, count = 0;
    int32_t ring_slots = 0;
    uint32_t work_bytes = 0;
    size_t smem = 0;
    int grid = 0;
};

struct viprs_batch {
    int n = 0;
    std::vector<uint32_t> w, h, bands;
    std::vector<viprs_plan*> plans;
    // knobs (autotuned)
    uint32_t ring_target = 2048;  // bytes of one shrink warp's stage buffer (source row segment)
    int32_t ring_slots_knob = 0;  // kept for the configuration API; the warp shrink ignores it
    int32_t blocks_per_sm = 0;    // cap of the shrink launches (0 = occupancy maximum)
    uint32_t reduce_smem_budget = 64 * 1024;  // shared memory of one fused-reduce tile
    int64_t item_bytes = 32 * 1024;           // source bytes per shrink work item
    // device work list
    std::vector<BatchStage> stages;
    std::vector<WorkItem> items;
    std::vector<BatchLaunch> launches;
    BatchStage* d_stages = nullptr;
    WorkItem* d_items = nullptr;
    int32_t* d_counters = nullptr;
    int32_t* d_ctrl = nullptr;  // [0] error, [1 + k] cursor of launch k
    size_t counters_cap = 0, stages_cap = 0, items_cap = 0;
    uint32_t ring_stage_bytes = 0;
    // the 4-band images' launches run on a second stream beside the others
    // (each stream's order carries its images' dependencies), joined around
    // the launches that hold items of every band count
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_main = nullptr, ev_aux = nullptr;
    // captured graph
    cudaGraphExec_t graph = nullptr;
    const uint64_t* graph_srcs = nullptr;
    const uint64_t* graph_dsts = nullptr;
};

constexpr int kMaxLaunches = 64;

namespace {

int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

void free_list(viprs_batch* b) {
    if (b->d_stages) cudaFree(b->d_stages);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counters) cudaFree(b->d_counters);
    b->d_stages = nullptr; b->d_items = nullptr; b->d_counters = nullptr;
    b->stages_cap = b->items_cap = b->counters_cap = 0;
}

void drop_graph(viprs_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_srcs = b->graph_dsts = nullptr;
}

// Convert one image's plan into batch stages; returns status.
int plan_stages(viprs_batch* b, int image, std::vector<std::vector<BatchStage>>* per_image) {
    viprs_plan* p = b->plans[size_t(image)];
    std::vector<BatchStage> out;
    const int last_plane = int(p->planes.size()) - 1;
    for (size_t si = 0; si < p->stages.size(); ++si) {
        const Stage& st = p->stages[si];
        BatchStage bs;
        bs.image = image;
        bs.in_src = st.in_plane == 0 ? 1 : 0;
        bs.out_dst = st.out_plane == last_plane ? 1 : 0;
        const PlaneArg in = plane_in_arg(p, st.in_plane, nullptr);
        const OutPlaneArg outp = plane_out_arg(p, st.out_plane, nullptr);
        switch (st.type) {
        case StageType::Shrink: {
            if (p->fmt != kU8 || !st.sh.hv_order || p->bands > 4) return VIPRS_ERR_UNSUPPORTED_FORMAT;
            bs.type = kBatchShrink;
            bs.sh = st.sh;
            bs.sh.in = in;
            bs.sh.out = outp;
            int32_t lo, hi;
            launch::shrink_prepare(&bs.sh, &lo, &hi);
            bs.lo = lo; bs.hi = hi;
            // independent warps: pixels per warp, stage buffers of at most
            // `ring_target` bytes, about `item_bytes` of source per item
            if (!launch::shrink_warp_setup(&bs.sh, b->ring_target, b->item_bytes, 0)) return VIPRS_ERR_INVALID_ARGUMENT;
            bs.n_items = int32_t(launch::shrink_warp_items(bs.sh));
            b->ring_stage_bytes = std::max(b->ring_stage_bytes, bs.sh.row_cap);
            break;
        }
        case StageType::Reduce2D: {
            if (p->fmt != kU8 || st.r2.mode_h != kReduceFixed || st.r2.mode_v != kReduceFixed)
                return VIPRS_ERR_UNSUPPORTED_FORMAT;
            bs.type = kBatchReduce2D;
            bs.r2 = st.r2;
            bs.r2.in = in;
            bs.r2.out = outp;
            bs.r2.starts_h = reinterpret_cast<const int32_t*>(p->d_tables + st.starts_off);
            bs.r2.phases_h = p->d_tables + st.phases_off;
            bs.r2.starts_v = reinterpret_cast<const int32_t*>(p->d_tables + st.starts2_off);
            bs.r2.phases_v = p->d_tables + st.phases2_off;
            bs.r2.coeffs_h = p->d_tables + st.coeffs_off;
            bs.r2.coeffs_v = p->d_tables + st.coeffs2_off;
            // many images keep every SM busy: take the largest tile (least halo
            // work) within the batch's shared-memory budget
            if (!launch::reduce2d_configure(&bs.r2, reinterpret_cast<const int32_t*>(p->host_tables.data() + st.starts_off),
                                            reinterpret_cast<const int32_t*>(p->host_tables.data() + st.starts2_off),
                                            in.x0, in.y0, in.w, in.h, 0, b->reduce_smem_budget))
                return VIPRS_ERR_UNSUPPORTED_FORMAT;
            const int nbx = (outp.w + bs.r2.tile_w - 1) / bs.r2.tile_w;
            const int nby = (outp.h + bs.r2.tile_h - 1) / bs.r2.tile_h;
            bs.n_items = nbx * nby;
            break;
        }
        case StageType::Affine: {
            bs.type = kBatchAffine;
            bs.af = st.af;
            bs.af.in = in;
            bs.af.out = outp;
            if (bs.af.separable && !bs.af.fast) {
                bs.af.xs = reinterpret_cast<const double*>(p->d_tables + st.starts_off);
                bs.af.ys = reinterpret_cast<const double*>(p->d_tables + st.phases_off);
            }
            if (st.axis_weights) {
                bs.af.wx = reinterpret_cast<const double*>(p->d_tables + st.coeffs_off);
                bs.af.wy = reinterpret_cast<const double*>(p->d_tables + st.coeffs2_off);
            }
            bs.n_items = outp.h;
            break;
        }
        case StageType::ReduceH:
        case StageType::ReduceV: {
            if (p->fmt != kU8 || st.rd.mode != kReduceFixed) return VIPRS_ERR_UNSUPPORTED_FORMAT;
            bs.type = st.type == StageType::ReduceH ? kBatchReduceH : kBatchReduceV;
            bs.rd = st.rd;
            bs.rd.in = in;
            bs.rd.out = outp;
            bs.rd.starts = reinterpret_cast<const int32_t*>(p->d_tables + st.starts_off);
            bs.rd.phases = p->d_tables + st.phases_off;
            bs.rd.coeffs = p->d_tables + st.coeffs_off;
            bs.n_items = outp.h * ((outp.w * int32_t(p->bands) + 255) / 256);
            break;
        }
        case StageType::Pixel: {
            bs.type = kBatchPixel;
            bs.px = st.px;
            bs.px.in = in;
            bs.px.out = outp;
            bs.n_items = outp.h;
            break;
        }
        default:
            return VIPRS_ERR_UNSUPPORTED_FORMAT;
        }
        out.push_back(bs);
    }
    (*per_image)[size_t(image)] = std::move(out);
    return VIPRS_OK;
}

size_t reduce2d_need(const Reduce2DArgs& a) { return launch::reduce2d_smem_bytes(a); }

// Build the device work list for the current knobs.
//
// Stages are grouped into levels: a shrink runs at level 0, the stage after it
// at level 1, and so on; a chain that does not start with a shrink starts at
// level 1, so that each level holds one kind of work.  Each level becomes one
// launch of its shrink items (the ring variant) and one of its other items
// (the tile variant).  A stage reads only stages of lower levels, so launch
// order in the stream is the whole dependency structure: no item waits.
int build_list(viprs_batch* b) {
    b->ring_stage_bytes = 0;
    std::vector<std::vector<BatchStage>> per(size_t(b->n));
    for (int i = 0; i < b->n; ++i) {
        const int st = plan_stages(b, i, &per);
        if (st) return st;
    }
    b->ring_stage_bytes = std::max<uint32_t>(b->ring_stage_bytes, 256);

    // flatten the stages; levels
    b->stages.clear();
    std::vector<std::vector<int>> gidx(size_t(b->n)), level(size_t(b->n));
    int max_level = 0;
    for (int i = 0; i < b->n; ++i) {
        const int shift = (!per[size_t(i)].empty() && per[size_t(i)][0].type != kBatchShrink) ? 1 : 0;
        for (size_t j = 0; j < per[size_t(i)].size(); ++j) {
            BatchStage s = per[size_t(i)][j];
            s.dep = -1;  // ordered by the launches
            gidx[size_t(i)].push_back(int(b->stages.size()));
            level[size_t(i)].push_back(int(j) + shift);
            max_level = std::max(max_level, int(j) + shift);
            b->stages.push_back(s);
        }
    }
    // images large first inside every launch (the long items start early)
    std::vector<int> order(size_t(b->n));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return uint64_t(b->w[size_t(x)]) * b->h[size_t(x)] * b->bands[size_t(x)] >
               uint64_t(b->w[size_t(y)]) * b->h[size_t(y)] * b->bands[size_t(y)];
    });
    b->items.clear();
    b->launches.clear();
    const size_t ctl = launch::batch_ctl_bytes();
    for (int L = 0; L <= max_level; ++L) {
        // shrink items of 1, 2, 3 and 4-band images (one launch each, a
        // kernel specialised to the band count), the fused-reduce tiles of 3-
        // and 4-band images (one launch each), then every other item
        for (int kind = 1; kind <= 7; ++kind) {
            const bool ring = kind <= 4;
            BatchLaunch l;
            l.level = L;
            l.ring = ring;
            l.bands = ring ? kind : (kind == 5 ? launch::kBatchTile3 : kind == 6 ? launch::kBatchTile4 : 0);
            l.offset = int64_t(b->items.size());
            size_t work = 0;
            for (int image : order) {
                for (size_t j = 0; j < gidx[size_t(image)].size(); ++j) {
                    if (level[size_t(image)][j] != L) continue;
                    const int g = gidx[size_t(image)][j];
                    const BatchStage& s = b->stages[size_t(g)];
                    if ((s.type == kBatchShrink) != ring) continue;
                    if (ring && s.sh.bands != l.bands) continue;
                    if (!ring) {
                        const int tb = s.type == kBatchReduce2D && s.r2.bands == 3   ? launch::kBatchTile3
                                       : s.type == kBatchReduce2D && s.r2.bands == 4 ? launch::kBatchTile4
                                                                                      : 0;
                        if (tb != l.bands) continue;
                    }
                    for (int32_t k = 0; k < s.n_items; ++k) b->items.push_back(WorkItem{g, k});
                    if (s.type == kBatchShrink) continue;
                    if (s.type == kBatchReduce2D) work = std::max(work, reduce2d_need(s.r2));
                    else if (s.type == kBatchReduceH || s.type == kBatchReduceV)
                        work = std::max(work, size_t(65 * s.rd.taps * 2 + 15) / 16 * 16 + 256);
                    else work = std::max<size_t>(work, 1024);
                }
            }
            l.count = int64_t(b->items.size()) - l.offset;
            if (l.count == 0) continue;
            if (int(b->launches.size()) >= kMaxLaunches) return VIPRS_ERR_UNSUPPORTED_FORMAT;
            l.work_bytes = uint32_t((std::max<size_t>(work, 256) + 127) / 128 * 128);
            l.ring_slots = 0;
            l.smem = ring ? launch::batch_warp_smem_bytes(b->ring_stage_bytes) : ctl + l.work_bytes;
            if (l.smem > 220 * 1024) return VIPRS_ERR_INVALID_ARGUMENT;
            int per_sm = launch::batch_blocks_per_sm(l.smem, l.bands);
            if (per_sm <= 0) return VIPRS_ERR_INVALID_ARGUMENT;
            if (ring && b->blocks_per_sm > 0) per_sm = std::min(per_sm, b->blocks_per_sm);
            l.grid = int(std::min<int64_t>(int64_t(per_sm) * sm_count(), l.count));
            b->launches.push_back(l);
        }
    }

    // upload
    if (b->stages.size() > b->stages_cap || b->items.size() > b->items_cap || b->stages.size() > b->counters_cap) {
        free_list(b);
        b->stages_cap = std::max<size_t>(b->stages.size(), 1);
        b->items_cap = std::max<size_t>(b->items.size(), 1);
        b->counters_cap = b->stages_cap;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_stages), b->stages_cap * sizeof(BatchStage));
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_items), b->items_cap * sizeof(WorkItem));
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&b->d_counters), b->counters_cap * sizeof(int32_t));
        if (e != cudaSuccess) return cuda_status(e);
    }
    cudaError_t e = cudaMemcpy(b->d_stages, b->stages.data(), b->stages.size() * sizeof(BatchStage), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, b->items.data(), b->items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice);
    return cuda_status(e);
}

int launch_batch(viprs_batch* b, const uint64_t* d_srcs, const uint64_t* d_dsts, cudaStream_t s) {
    if (!b->aux) return VIPRS_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaMemsetAsync(b->d_ctrl, 0, (1 + b->launches.size()) * sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_status(e);
    // join the two streams: `to` waits for everything enqueued on `from`
    auto join = [&](cudaStream_t from, cudaEvent_t ev, cudaStream_t to) {
        cudaError_t r = cudaEventRecord(ev, from);
        return r == cudaSuccess ? cudaStreamWaitEvent(to, ev, 0) : r;
    };
    e = join(s, b->ev_main, b->aux);
    if (e != cudaSuccess) return cuda_status(e);
    // A stage reads only its own image's earlier stages, so each stream's own
    // order carries the dependencies of its images (4-band on aux, the rest on
    // s).  A generic launch (items of any band count) waits for aux first, and
    // aux waits for it before its next launch.
    bool aux_behind = false;
    for (size_t k = 0; k < b->launches.size(); ++k) {
        const BatchLaunch& l = b->launches[k];
        const bool on_aux = l.bands == 4 || l.bands == launch::kBatchTile4;
        if (on_aux && aux_behind) {
            e = join(s, b->ev_main, b->aux);
            if (e != cudaSuccess) return cuda_status(e);
            aux_behind = false;
        }
        if (!l.ring && l.bands == 0) {
            e = join(b->aux, b->ev_aux, s);
            if (e != cudaSuccess) return cuda_status(e);
            aux_behind = true;
        }
        const cudaStream_t ls = on_aux ? b->aux : s;
        BatchArgs a;
        a.stages = b->d_stages;
        a.items = b->d_items + l.offset;
        a.n_items = int32_t(l.count);
        a.counters = b->d_counters;
        a.cursor = b->d_ctrl + 1 + k;
        a.err = b->d_ctrl;
        a.srcs = d_srcs;
        a.dsts = d_dsts;
        a.ring_stage_bytes = b->ring_stage_bytes;
        a.ring_slots = l.ring_slots;
        a.work_bytes = l.work_bytes;
        a.smem_bytes = uint32_t(l.smem);
        e = launch::batch(a, l.grid, l.bands, ls);
        if (e != cudaSuccess) return cuda_status(e);
    }
    e = join(b->aux, b->ev_aux, s);  // the caller's stream ends after both
    return cuda_status(e);
}

// A batch of one u8 chain plan per image (`chain_of(i, &chain)` builds image
// i's chain), its control words and work list.
template <typename ChainOf>
int32_t batch_create(int32_t n, const uint32_t* widths, const uint32_t* heights, const uint32_t* bands,
                     viprs_batch** out, ChainOf chain_of) {
    std::unique_ptr<viprs_batch> b(new (std::nothrow) viprs_batch());
    if (!b) return VIPRS_ERR_OUT_OF_MEMORY;
    b->n = n;
    b->w.assign(widths, widths + n);
    b->h.assign(heights, heights + n);
    b->bands.assign(bands, bands + n);
    b->plans.assign(size_t(n), nullptr);
    int st = VIPRS_OK;
    for (int i = 0; i < n && st == VIPRS_OK; ++i) {
        Chain c;
        st = chain_of(i, &c);
        if (st == VIPRS_OK) st = create_chain_plan(widths[i], heights[i], bands[i], VIPRS_U8, c, &b->plans[size_t(i)]);
    }
    if (st == VIPRS_OK) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_ctrl), (1 + kMaxLaunches) * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_main, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_aux, cudaEventDisableTiming);
        st = cuda_status(e);
    }
    if (st == VIPRS_OK) st = build_list(b.get());
    if (st != VIPRS_OK) {
        viprs_batch_destroy(b.release());
        return st;
    }
    *out = b.release();
    return VIPRS_OK;
}

}  // namespace

extern "C" {

int32_t viprs_thumbnail_batch_create(int32_t n, const uint32_t* widths, const uint32_t* heights,
                                     const uint32_t* bands, int32_t target, uint32_t tw, uint32_t th,
                                     int32_t kernel, int32_t crop, viprs_batch** out) {
    if (!out || !widths || !heights || !bands) return VIPRS_ERR_NULL_POINTER;
    *out = nullptr;
    if (n <= 0 || target < 0 || target > 3) return VIPRS_ERR_INVALID_ARGUMENT;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    return batch_create(n, widths, heights, bands, out, [&](int i, Chain* c) {
        return builder_thumbnail_chain(widths[i], heights[i], bands[i], ThumbTarget(target), tw, th, Kernel(kernel),
                                       crop != 0, c);
    });
}

int32_t viprs_chain_batch_create(int32_t n, const uint32_t* widths, const uint32_t* heights, const uint32_t* bands,
                                 const viprs_node* nodes, int32_t n_nodes, int32_t demand_override,
                                 viprs_batch** out) {
    if (!out || !widths || !heights || !bands) return VIPRS_ERR_NULL_POINTER;
    *out = nullptr;
    if (n <= 0) return VIPRS_ERR_INVALID_ARGUMENT;
    Chain chain;
    const int32_t st = nodes_to_chain(nodes, n_nodes, demand_override, &chain);
    if (st) return st;
    return batch_create(n, widths, heights, bands, out, [&](int, Chain* c) {
        *c = chain;
        return int(VIPRS_OK);
    });
}

int32_t viprs_batch_output_size(const viprs_batch* b, int32_t i, uint32_t* w, uint32_t* h) {
    if (!b || !w || !h) return VIPRS_ERR_NULL_POINTER;
    if (i < 0 || i >= b->n) return VIPRS_ERR_INVALID_ARGUMENT;
    *w = b->plans[size_t(i)]->out_w;
    *h = b->plans[size_t(i)]->out_h;
    return VIPRS_OK;
}

int32_t viprs_batch_work_items(const viprs_batch* b, int32_t* items, int32_t* stages, int32_t* grid) {
    if (!b) return VIPRS_ERR_NULL_POINTER;
    if (items) *items = int32_t(b->items.size());
    if (stages) *stages = int32_t(b->stages.size());
    if (grid) {
        int g = 0;
        for (const auto& l : b->launches) g = std::max(g, l.grid);
        *grid = g;
    }
    return VIPRS_OK;
}

int32_t viprs_batch_execute(viprs_batch* b, const uint64_t* d_srcs, const uint64_t* d_dsts, void* stream) {
    if (!b || !d_srcs || !d_dsts) return VIPRS_ERR_NULL_POINTER;
    return launch_batch(b, d_srcs, d_dsts, static_cast<cudaStream_t>(stream));
}

int32_t viprs_batch_execute_graph(viprs_batch* b, const uint64_t* d_srcs, const uint64_t* d_dsts, void* stream) {
    if (!b || !d_srcs || !d_dsts) return VIPRS_ERR_NULL_POINTER;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!b->graph || b->graph_srcs != d_srcs || b->graph_dsts != d_dsts) {
        drop_graph(b);
        cudaStream_t cs;
        cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e);
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        int st = VIPRS_OK;
        if (e == cudaSuccess) st = launch_batch(b, d_srcs, d_dsts, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && st == VIPRS_OK) e = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (st != VIPRS_OK) return st;
        if (e != cudaSuccess) { b->graph = nullptr; return cuda_status(e); }
        b->graph_srcs = d_srcs;
        b->graph_dsts = d_dsts;
    }
    return cuda_status(cudaGraphLaunch(b->graph, s));
}

int32_t viprs_batch_execute_per_image(viprs_batch* b, const uint64_t* h_srcs, const uint64_t* h_dsts, void* stream) {
    if (!b || !h_srcs || !h_dsts) return VIPRS_ERR_NULL_POINTER;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int i = 0; i < b->n; ++i) {
        const int st = execute_plan(b->plans[size_t(i)], reinterpret_cast<const void*>(h_srcs[i]),
                                    reinterpret_cast<void*>(h_dsts[i]), s);
        if (st) return st;
    }
    return VIPRS_OK;
}

int32_t viprs_batch_launch_count(const viprs_batch* b, int32_t* batched, int32_t* per_image) {
    if (!b) return VIPRS_ERR_NULL_POINTER;
    if (batched) *batched = int32_t(b->launches.size());
    if (per_image) {
        int32_t n = 0;
        for (auto* p : b->plans) n += int32_t(p->stages.size());
        *per_image = n;
    }
    return VIPRS_OK;
}

int32_t viprs_batch_set_config(viprs_batch* b, uint32_t ring_bytes, int32_t ring_slots, int32_t blocks_per_sm) {
    if (!b) return VIPRS_ERR_NULL_POINTER;
    if (ring_bytes < 1024 || ring_bytes > 32768 || ring_slots < 0 || ring_slots > 16 || blocks_per_sm < 0)
        return VIPRS_ERR_INVALID_ARGUMENT;
    b->ring_target = ring_bytes;
    b->ring_slots_knob = ring_slots;
    b->blocks_per_sm = blocks_per_sm;
    drop_graph(b);
    return build_list(b);
}

int32_t viprs_batch_get_config(const viprs_batch* b, uint32_t* ring_bytes, int32_t* ring_slots, int32_t* blocks_per_sm) {
    if (!b) return VIPRS_ERR_NULL_POINTER;
    if (ring_bytes) *ring_bytes = b->ring_target;
    if (ring_slots) *ring_slots = b->ring_slots_knob;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    return VIPRS_OK;
}

int32_t viprs_batch_autotune(viprs_batch* b, const uint64_t* d_srcs, const uint64_t* d_dsts, void* stream,
                             int32_t repeats, float* best_ms) {
    if (!b || !d_srcs || !d_dsts) return VIPRS_ERR_NULL_POINTER;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t rings[] = {1536, 2048, 3072, 4096};  // warp stage buffer bytes
    const int32_t lags[] = {0};
    const int32_t caps[] = {0, 2, 3};
    float best = 1e30f;
    uint32_t br = b->ring_target;
    int32_t bl = b->ring_slots_knob, bc = b->blocks_per_sm;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    repeats = std::max(repeats, 1);
    for (uint32_t r : rings)
        for (int32_t l : lags)
            for (int32_t c : caps) {
                if (viprs_batch_set_config(b, r, l, c) != VIPRS_OK) continue;
                if (launch_batch(b, d_srcs, d_dsts, s) != VIPRS_OK) continue;  // warm
                cudaEventRecord(e0, s);
                for (int k = 0; k < repeats; ++k) launch_batch(b, d_srcs, d_dsts, s);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= float(repeats);
                if (ms < best) { best = ms; br = r; bl = l; bc = c; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_ms) *best_ms = best;
    return viprs_batch_set_config(b, br, bl, bc);
}

int32_t viprs_batch_status(viprs_batch* b, void* stream) {
    if (!b) return VIPRS_ERR_NULL_POINTER;
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e);
    int32_t h = 0;
    e = cudaMemcpy(&h, b->d_ctrl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    return h;
}

void viprs_batch_destroy(viprs_batch* b) {
    if (!b) return;
    drop_graph(b);
    free_list(b);
    if (b->d_ctrl) cudaFree(b->d_ctrl);
    if (b->ev_main) cudaEventDestroy(b->ev_main);
    if (b->ev_aux) cudaEventDestroy(b->ev_aux);
    if (b->aux) cudaStreamDestroy(b->aux);
    for (auto* p : b->plans) free_plan(p);
    delete b;
}

}  // extern "C"
