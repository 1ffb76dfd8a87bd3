// adjoint_plan.cpp -- host side of the adjoint (backward) entry points.
//
// The forward operators are the library's own (f32): ReduceH / ReduceV and
// their chain (resample/reduceh.rs, reducev.rs with bound input lengths), the
// Affine of PipelineBuilder::affine semantics with a backward matrix
// (affine/core.rs) and MapImOp (mapim.rs).  Tables and positions are built
// exactly as for the forward pass, so each kernel computes the exact
// transpose / derivative of what the forward kernels compute.  Scratch
// (the transposed mid plane, position tables, fixed-point accumulators,
// per-block partial sums) is allocated stream-ordered on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "adjoint_launch.hpp"
#include "chain.hpp"
#include "viprs_b200.h"

using namespace viprs;

namespace {

// The library's own stream-ordered memory pool on the current device.  Its
// release threshold is unbounded, so memory freed at the end of one backward
// call stays mapped for the next (a deterministic mapim gradient of a 4096^2
// image needs a 512 MB accumulator every call; mapping it afresh each time
// would cost more than the kernels).  nullptr: fall back to the device's
// default pool.
cudaMemPool_t scratch_pool() {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        pool = nullptr;
    } else {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pools.emplace(dev, pool);
    return pool;
}

// Stream-ordered scratch from scratch_pool(): freed on the stream when the
// guard goes away.
struct Scratch {
    cudaStream_t s;
    cudaMemPool_t pool;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t st) : s(st), pool(scratch_pool()) {}
    ~Scratch() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
    template <typename T>
    T* alloc(size_t n, cudaError_t* e) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(n * sizeof(T), 16);
        *e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, s) : cudaMallocAsync(&p, bytes, s);
        if (*e == cudaSuccess) ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    template <typename T>
    T* upload(const std::vector<T>& v, cudaError_t* e) {
        T* d = alloc<T>(v.size(), e);
        if (*e == cudaSuccess && !v.empty()) *e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
        return d;
    }
};

int check_f32(const viprs_image* im) {
    if (!im || !im->data) return VIPRS_ERR_NULL_POINTER;
    if (im->format != VIPRS_F32) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    if (im->bands == 0 || im->width == 0 || im->height == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    const uint64_t packed = uint64_t(im->width) * im->bands * 4;
    if (im->row_stride && im->row_stride != packed) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    return VIPRS_OK;
}

// Tables of one transposed reduce pass.  `out_origin`/`out_len`: the pass's
// output positions; the pass input has `in_len` samples starting at `in_origin`
// (clamp folding at both ends when `fold`).  Input index i gathers outputs
// [lo[i], hi[i]] with weights wt[i * wstride + (o - lo[i])].
struct PassTables {
    std::vector<int32_t> lo, hi;
    std::vector<double> wt;
    int32_t wstride = 1;
};

PassTables pass_tables(const ReduceKernel& rk, int64_t out_origin, int64_t out_len, int64_t in_origin,
                       int64_t in_len, bool fold) {
    std::vector<int64_t> starts(size_t(out_len), 0);
    std::vector<int32_t> phases(size_t(out_len), 0);
    std::vector<double> fold_lo(size_t(out_len), 0.0), fold_hi(size_t(out_len), 0.0);
    for (int64_t o = 0; o < out_len; ++o) {
        int64_t s; int32_t ph;
        rk.plan(rk.source_position(double(out_origin + o)), &s, &ph);
        starts[size_t(o)] = s - in_origin;
        phases[size_t(o)] = ph;
        const double* c = &rk.coeffs_f64[size_t(ph) * rk.taps];
        const int64_t rel = s - in_origin;
        if (fold) {
            for (int32_t k = 0; k < rk.taps; ++k) {
                // a one-sample axis: every tap clamps onto it
                if (rel + k <= 0 || in_len == 1) fold_lo[size_t(o)] += c[k];
                else if (rel + k >= in_len - 1) fold_hi[size_t(o)] += c[k];
            }
        }
    }
    PassTables t;
    t.lo.assign(size_t(in_len), 0);
    t.hi.assign(size_t(in_len), -1);
    // outputs whose taps reach input index i (after the clamp when folding)
    for (int64_t o = 0; o < out_len; ++o) {
        int64_t a = starts[size_t(o)], b = a + rk.taps - 1;
        if (fold) { a = std::max<int64_t>(a, 0); b = std::min<int64_t>(b, in_len - 1); a = std::min(a, in_len - 1); b = std::max<int64_t>(b, 0); }
        else { a = std::max<int64_t>(a, 0); b = std::min<int64_t>(b, in_len - 1); }
        for (int64_t i = a; i <= b; ++i) {
            if (t.hi[size_t(i)] < t.lo[size_t(i)]) { t.lo[size_t(i)] = int32_t(o); t.hi[size_t(i)] = int32_t(o); }
            else { t.lo[size_t(i)] = std::min(t.lo[size_t(i)], int32_t(o)); t.hi[size_t(i)] = std::max(t.hi[size_t(i)], int32_t(o)); }
        }
    }
    int32_t ws = 1;
    for (int64_t i = 0; i < in_len; ++i) ws = std::max(ws, t.hi[size_t(i)] - t.lo[size_t(i)] + 1);
    t.wstride = ws;
    t.wt.assign(size_t(in_len) * size_t(ws), 0.0);
    for (int64_t i = 0; i < in_len; ++i) {
        for (int32_t o = t.lo[size_t(i)]; o <= t.hi[size_t(i)]; ++o) {
            double w;
            const int64_t k = i - starts[size_t(o)];
            if (fold && (in_len == 1 || i == 0)) w = fold_lo[size_t(o)];
            else if (fold && i == in_len - 1) w = fold_hi[size_t(o)];
            else w = (k >= 0 && k < rk.taps) ? rk.coeffs_f64[size_t(phases[size_t(o)]) * rk.taps + size_t(k)] : 0.0;
            t.wt[size_t(i) * size_t(ws) + size_t(o - t.lo[size_t(i)])] = w;
        }
    }
    return t;
}

// The tables of a pass packed in one buffer: lo, hi (int32, in_len each), then
// the weights rounded to f32 (16-byte aligned).
std::vector<uint8_t> pack_tables(const PassTables& t, size_t* wt_off) {
    const size_t n = t.lo.size();
    *wt_off = (n * 8 + 15) / 16 * 16;
    std::vector<uint8_t> buf(*wt_off + t.wt.size() * 4);
    std::memcpy(buf.data(), t.lo.data(), n * 4);
    std::memcpy(buf.data() + n * 4, t.hi.data(), n * 4);
    for (size_t k = 0; k < t.wt.size(); ++k) {
        const float w = float(t.wt[k]);
        std::memcpy(buf.data() + *wt_off + k * 4, &w, 4);
    }
    return buf;
}

// Device copies of pass tables, kept per device and geometry: a backward pass
// over the same shapes (every training step) reuses them instead of uploading
// again.  Entries are immutable and live until the process exits; past
// kMaxCached entries a pass uploads its tables stream-ordered per call.
struct TableKey {
    int device;
    int32_t kernel, fold;
    uint64_t factor_bits;
    int64_t bound, out_origin, out_len, in_origin, in_len;
    bool operator<(const TableKey& o) const {
        return std::tie(device, kernel, fold, factor_bits, bound, out_origin, out_len, in_origin, in_len) <
               std::tie(o.device, o.kernel, o.fold, o.factor_bits, o.bound, o.out_origin, o.out_len, o.in_origin,
                        o.in_len);
    }
};
struct DevTables {
    const uint8_t* data = nullptr;
    size_t wt_off = 0;
    int32_t wstride = 1;
};
constexpr size_t kMaxCached = 256;
std::mutex g_table_mu;
std::map<TableKey, DevTables> g_tables;

int launch_pass(Scratch& sc, const ReduceKernel& rk, int32_t kernel, double factor, int64_t bound,
                int64_t out_origin, int64_t out_len, int64_t in_origin, int64_t in_len, bool fold, ReduceAdjArgs a,
                cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    uint64_t fb;
    std::memcpy(&fb, &factor, 8);
    const TableKey key{dev, kernel, fold ? 1 : 0, fb, bound, out_origin, out_len, in_origin, in_len};
    DevTables d;
    {
        std::lock_guard<std::mutex> lk(g_table_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) d = it->second;
    }
    if (!d.data) {
        const PassTables t = pass_tables(rk, out_origin, out_len, in_origin, in_len, fold);
        const std::vector<uint8_t> buf = pack_tables(t, &d.wt_off);
        d.wstride = t.wstride;
        std::lock_guard<std::mutex> lk(g_table_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) {
            d = it->second;
        } else if (g_tables.size() < kMaxCached) {
            void* p = nullptr;
            e = cudaMalloc(&p, buf.size());
            if (e == cudaSuccess) e = cudaMemcpy(p, buf.data(), buf.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                if (p) cudaFree(p);
                return cuda_status(e);
            }
            d.data = static_cast<const uint8_t*>(p);
            g_tables.emplace(key, d);
        } else {
            d.data = sc.upload(buf, &e);
            if (e != cudaSuccess) return cuda_status(e);
        }
    }
    a.lo = reinterpret_cast<const int32_t*>(d.data);
    a.hi = reinterpret_cast<const int32_t*>(d.data + size_t(in_len) * 4);
    a.wt = reinterpret_cast<const float*>(d.data + d.wt_off);
    a.wstride = d.wstride;
    return cuda_status(launch::reduce_adjoint(a, s));
}

}  // namespace

extern "C" {

int32_t viprs_reduce_adjoint(const viprs_image* grad_out, const viprs_image* grad_in, double factor,
                             int32_t kernel, int32_t horizontal, void* stream) {
    int st = check_f32(grad_out);
    if (st) return st;
    st = check_f32(grad_in);
    if (st) return st;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    if (grad_out->bands != grad_in->bands) return VIPRS_ERR_SIZE_MISMATCH;
    ReduceKernel rk;
    st = rk.init(factor, Kernel(kernel));
    if (st) return st;
    const uint32_t n_in = horizontal ? grad_in->width : grad_in->height;
    rk.bind_input_len(n_in);
    const uint32_t n_out = reduce_output_len(factor, n_in);
    if ((horizontal ? grad_out->width : grad_out->height) != n_out) return VIPRS_ERR_SIZE_MISMATCH;
    if ((horizontal ? grad_out->height : grad_out->width) != (horizontal ? grad_in->height : grad_in->width))
        return VIPRS_ERR_SIZE_MISMATCH;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc(s);
    ReduceAdjArgs a;
    a.g_out = static_cast<const float*>(grad_out->data);
    a.g_in = static_cast<float*>(grad_in->data);
    a.horizontal = horizontal ? 1 : 0;
    a.out_w = int32_t(grad_out->width); a.out_h = int32_t(grad_out->height);
    a.in_w = int32_t(grad_in->width); a.in_h = int32_t(grad_in->height);
    a.bands = int32_t(grad_in->bands);
    return launch_pass(sc, rk, kernel, factor, n_in, 0, n_out, 0, n_in, true, a, s);
}

int32_t viprs_reduce_hv_adjoint(const viprs_image* grad_out, const viprs_image* grad_in, double hfactor,
                                double vfactor, int32_t kernel, void* stream) {
    int st = check_f32(grad_out);
    if (st) return st;
    st = check_f32(grad_in);
    if (st) return st;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    if (grad_out->bands != grad_in->bands) return VIPRS_ERR_SIZE_MISMATCH;
    const uint32_t W = grad_in->width, H = grad_in->height, B = grad_in->bands;
    ReduceKernel rh, rv;
    st = rh.init(hfactor, Kernel(kernel));
    if (st) return st;
    st = rv.init(vfactor, Kernel(kernel));
    if (st) return st;
    rh.bind_input_len(W);
    const uint32_t OW = reduce_output_len(hfactor, W);
    rv.bind_input_len(H);
    const uint32_t OH = reduce_output_len(vfactor, H);
    if (grad_out->width != OW || grad_out->height != OH) return VIPRS_ERR_SIZE_MISMATCH;
    // mid plane: the ReduceH output rows the ReduceV taps read (virtual rows
    // beyond the image are ReduceH of clamped source rows)
    int64_t my0, mh;
    rv.required_axis(0, OH, &my0, &mh);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc(s);
    cudaError_t e = cudaSuccess;
    float* g_mid = sc.alloc<float>(size_t(mh) * OW * B, &e);
    if (e != cudaSuccess) return cuda_status(e);
    // V^T: no clamp inside the mid plane (it covers every tap)
    ReduceAdjArgs av;
    av.g_out = static_cast<const float*>(grad_out->data);
    av.g_in = g_mid;
    av.horizontal = 0;
    av.out_w = int32_t(OW); av.out_h = int32_t(OH);
    av.in_w = int32_t(OW); av.in_h = int32_t(mh);
    av.bands = int32_t(B);
    st = launch_pass(sc, rv, kernel, vfactor, H, 0, OH, my0, mh, false, av, s);
    if (st) return st;
    // H^T with the source clamp: edge columns fold, virtual mid rows fold onto edge rows
    ReduceAdjArgs ah;
    ah.g_out = g_mid;
    ah.g_in = static_cast<float*>(grad_in->data);
    ah.horizontal = 1;
    ah.out_w = int32_t(OW); ah.out_h = int32_t(mh);
    ah.in_w = int32_t(W); ah.in_h = int32_t(H);
    ah.bands = int32_t(B);
    ah.fold_rows = 1;
    ah.mid_y0 = int32_t(my0);
    return launch_pass(sc, rh, kernel, hfactor, W, 0, OW, 0, W, true, ah, s);
}

int32_t viprs_affine_grad(const viprs_image* in, const viprs_image* grad_out, const viprs_image* grad_in,
                          const double backward[4], double tx, double ty, int32_t kernel, int32_t extend,
                          double background, int32_t premultiplied, uint32_t tile_w, uint32_t tile_h,
                          int32_t deterministic, double* grad_matrix, void* stream) {
    int st = check_f32(in);
    if (st) return st;
    st = check_f32(grad_out);
    if (st) return st;
    if (grad_in) {
        st = check_f32(grad_in);
        if (st) return st;
        if (grad_in->width != in->width || grad_in->height != in->height || grad_in->bands != in->bands)
            return VIPRS_ERR_SIZE_MISMATCH;
    }
    if (!backward) return VIPRS_ERR_NULL_POINTER;
    if (kernel != VIPRS_KERNEL_BILINEAR) return VIPRS_ERR_INVALID_KERNEL;
    if (extend < 0 || extend > 5) return VIPRS_ERR_INVALID_ARGUMENT;
    if (grad_out->bands != in->bands || in->bands > 8) return VIPRS_ERR_SIZE_MISMATCH;
    PlanNode n;
    n.kind = NodeKind::Affine;
    std::memcpy(n.m, backward, sizeof(n.m));
    n.tx = tx; n.ty = ty; n.kernel = Kernel(kernel);
    n.out_w = grad_out->width; n.out_h = grad_out->height;
    n.extend = Extend(extend); n.background = background; n.premultiplied = premultiplied != 0;
    n.ew = tile_w; n.eh = tile_h;
    AffineGradArgs g;
    st = affine_stage_setup(n, in->width, in->height, in->bands, VIPRS_F32, -1, Demand::SmallTile, n.out_w, n.out_h,
                            0, 0, &g.fwd);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc(s);
    cudaError_t e = cudaSuccess;
    if (g.fwd.separable && !g.fwd.fast) {
        std::vector<double> xs(n.out_w), ys(n.out_h);
        affine_axis_tables(g.fwd, xs.data(), ys.data());
        g.fwd.xs = sc.upload(xs, &e);
        if (e == cudaSuccess) g.fwd.ys = sc.upload(ys, &e);
    }
    g.fwd.in.data = static_cast<const uint8_t*>(in->data);
    g.fwd.in.w = int32_t(in->width); g.fwd.in.h = int32_t(in->height);
    g.fwd.in.pitch = int64_t(in->width) * in->bands * 4;
    g.fwd.in.total_bytes = g.fwd.in.pitch * in->height;
    g.fwd.out.w = int32_t(grad_out->width); g.fwd.out.h = int32_t(grad_out->height);
    g.fwd.out.pitch = int64_t(grad_out->width) * grad_out->bands * 4;
    g.g_out = static_cast<const float*>(grad_out->data);
    const int blocks = launch::affine_grad_blocks(int32_t(grad_out->width), int32_t(grad_out->height));
    const int64_t n_in = int64_t(in->width) * in->height * in->bands;
    if (grad_in) {
        if (deterministic) {
            g.g_fixed = sc.alloc<unsigned long long>(size_t(n_in), &e);
            if (e == cudaSuccess) e = cudaMemsetAsync(g.g_fixed, 0, size_t(n_in) * 8, s);
            g.fixed_scale = 4294967296.0;  // 2^32: exact, order-independent integer sums
        } else {
            g.g_in = static_cast<float*>(grad_in->data);
            if (e == cudaSuccess) e = cudaMemsetAsync(g.g_in, 0, size_t(n_in) * 4, s);
        }
    }
    if (grad_matrix && e == cudaSuccess) g.partial = sc.alloc<double>(size_t(blocks) * 6, &e);
    if (e != cudaSuccess) return cuda_status(e);
    e = launch::affine_grad(g, blocks, s);
    if (e == cudaSuccess && grad_in && deterministic)
        e = launch::fixed_to_f32(g.g_fixed, static_cast<float*>(grad_in->data), n_in, 1.0 / g.fixed_scale, s);
    if (e == cudaSuccess && grad_matrix) e = launch::sum_partials(g.partial, blocks, grad_matrix, s);
    return cuda_status(e);
}

int32_t viprs_mapim_grad(const viprs_image* src, const viprs_image* index, const viprs_image* grad_out,
                         const viprs_image* grad_src, const viprs_image* grad_index, int32_t kernel,
                         int32_t extend_copy, double background, int32_t premultiplied, int32_t deterministic,
                         void* stream) {
    int st = check_f32(src);
    if (st) return st;
    st = check_f32(index);
    if (st) return st;
    st = check_f32(grad_out);
    if (st) return st;
    if (index->bands != 2) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    if (grad_out->width != index->width || grad_out->height != index->height || grad_out->bands != src->bands)
        return VIPRS_ERR_SIZE_MISMATCH;
    // the alpha-premultiplying sampler of 2/4-band images is forward only
    if ((src->bands == 2 || src->bands == 4) && !premultiplied) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    if (src->bands > 8) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    if (kernel < 0 || kernel > 9 || !affine_kernel_supported(Kernel(kernel))) return VIPRS_ERR_INVALID_KERNEL;
    if (grad_src) {
        st = check_f32(grad_src);
        if (st) return st;
        if (grad_src->width != src->width || grad_src->height != src->height || grad_src->bands != src->bands)
            return VIPRS_ERR_SIZE_MISMATCH;
    }
    if (grad_index) {
        st = check_f32(grad_index);
        if (st) return st;
        if (grad_index->width != index->width || grad_index->height != index->height || grad_index->bands != 2)
            return VIPRS_ERR_SIZE_MISMATCH;
    }
    MapimGradArgs g;
    MapimArgs& a = g.fwd;
    a.src.data = static_cast<const uint8_t*>(src->data);
    a.src.w = int32_t(src->width); a.src.h = int32_t(src->height); a.src.pitch = int64_t(src->width) * src->bands * 4;
    a.index.data = static_cast<const uint8_t*>(index->data);
    a.index.w = int32_t(index->width); a.index.h = int32_t(index->height); a.index.pitch = int64_t(index->width) * 8;
    a.out.w = int32_t(grad_out->width); a.out.h = int32_t(grad_out->height);
    a.bands = int32_t(src->bands); a.fmt = VIPRS_F32; a.kernel = kernel; a.extend_copy = extend_copy != 0;
    a.background = background; a.src_w = src->width; a.src_h = src->height;
    g.g_out = static_cast<const float*>(grad_out->data);
    g.g_index = grad_index ? static_cast<float*>(grad_index->data) : nullptr;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc(s);
    cudaError_t e = cudaSuccess;
    const int64_t n_src = int64_t(src->width) * src->height * src->bands;
    if (grad_src) {
        if (deterministic) {
            g.g_fixed = sc.alloc<unsigned long long>(size_t(n_src), &e);
            if (e == cudaSuccess) e = cudaMemsetAsync(g.g_fixed, 0, size_t(n_src) * 8, s);
            g.fixed_scale = 4294967296.0;
        } else {
            g.g_src = static_cast<float*>(grad_src->data);
            e = cudaMemsetAsync(g.g_src, 0, size_t(n_src) * 4, s);
        }
    }
    if (e != cudaSuccess) return cuda_status(e);
    e = launch::mapim_grad(g, s);
    if (e == cudaSuccess && grad_src && deterministic)
        e = launch::fixed_to_f32(g.g_fixed, static_cast<float*>(grad_src->data), n_src, 1.0 / g.fixed_scale, s);
    return cuda_status(e);
}

}  // extern "C"
