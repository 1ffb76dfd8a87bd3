// capi.cpp -- the extern "C" boundary and the chain executor.
//
// A chain is what PipelineBuilder materialises (builder/resample.rs): a list
// of nodes applied to a MemorySource.  viprs runs it tile by tile
// (rayon_scheduler/execute.rs:174-480): each node's required input region is
// propagated upstream unclipped and only the source read edge-replicates.
// Here the whole output is one region: regions are propagated once on the
// host, every intermediate is a device-resident plane covering exactly the
// region its consumer requested, and each fused stage is one kernel launch.
// Every pixel of viprs's virtual intermediate planes is independent of the
// tile that computes it, so the results match viprs's tiled run (the u8
// ReduceH position walk starts at the region origin, which is x = 0 for the
// full-width strips that ThinStrip tiling uses).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "chain.hpp"
#include "sin_rn.cuh"
#include "viprs_b200.h"

using namespace viprs;

namespace {
thread_local int32_t g_last_cuda_error = 0;
}  // namespace

int32_t viprs::cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return VIPRS_OK;
    g_last_cuda_error = int32_t(e);
    if (e == cudaErrorMemoryAllocation) return VIPRS_ERR_OUT_OF_MEMORY;
    return VIPRS_ERR_CUDA;
}

namespace {

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

size_t push_table(std::vector<uint8_t>& t, const void* data, size_t bytes) {
    const size_t off = align_up(t.size(), 16);
    t.resize(off + align_up(bytes, 16), 0);  // padded: kernels copy tables in 4-byte words
    if (bytes) std::memcpy(t.data() + off, data, bytes);
    return off;
}

// Region a node needs from its input to produce `out` (the required_input_region
// of each op; see plan.hpp for the files).
int required_region(const PlanNode& n, const ReduceKernel* rk, const ReduceKernel* rk2, uint32_t in_w,
                    uint32_t in_h, const Region& out, Region* in) {
    *in = out;
    switch (n.kind) {
    case NodeKind::ShrinkH: in->x = out.x * n.ufactor; in->w = out.w * n.ufactor; break;
    case NodeKind::ShrinkV: in->y = out.y * n.ufactor; in->h = out.h * n.ufactor; break;
    case NodeKind::Shrink:
        in->x = out.x * n.ufactor; in->w = out.w * n.ufactor;
        in->y = out.y * n.vufactor; in->h = out.h * n.vufactor;
        break;
    case NodeKind::ReduceH: rk->required_axis(out.x, out.w, &in->x, &in->w); break;
    case NodeKind::ReduceV: rk->required_axis(out.y, out.h, &in->y, &in->h); break;
    case NodeKind::Reduce: {
        Region mid = out;
        rk2->config_required_axis(out.y, out.h, &mid.y, &mid.h);
        *in = mid;
        rk->config_required_axis(mid.x, mid.w, &in->x, &in->w);
        break;
    }
    case NodeKind::Affine: *in = affine_required_region(n, in_w, in_h, out); break;
    case NodeKind::ExtractArea: in->x = out.x + n.ex; in->y = out.y + n.ey; break;
    case NodeKind::Zoom:
        // Zoom::required_input_region (structural/zoom.rs:343-349)
        if (out.w > 0) { in->x = out.x / n.zx; in->w = (out.x + out.w - 1) / n.zx - in->x + 1; }
        if (out.h > 0) { in->y = out.y / n.zy; in->h = (out.y + out.h - 1) / n.zy - in->y + 1; }
        break;
    default: break;
    }
    return VIPRS_OK;
}

struct NodeRt {
    PlanNode n;
    uint32_t in_w = 0, in_h = 0, out_w = 0, out_h = 0;
    ReduceKernel rk, rk2;
};

int add_plane(viprs_plan* p, const Region& r, size_t es, size_t* ws) {
    PlaneInfo pi;
    pi.r = r;
    pi.pitch = int64_t(std::max<int64_t>(r.w, 0)) * p->bands * es;
    pi.offset = align_up(*ws, 256);
    *ws = pi.offset + size_t(pi.pitch) * size_t(std::max<int64_t>(r.h, 0)) + 16;
    p->planes.push_back(pi);
    return int(p->planes.size()) - 1;
}

// Position tables of a reduce stage over `out_len` outputs starting at `origin`.
void reduce_tables(const ReduceKernel& rk, int64_t origin, int64_t len, bool incremental,
                   std::vector<int32_t>* starts, std::vector<uint8_t>* phases) {
    starts->resize(size_t(std::max<int64_t>(len, 1)));
    phases->resize(size_t(std::max<int64_t>(len, 1)));
    if (incremental) {
        // ReduceH<U8>::process_region (reduceh.rs:111-118): += factor from the region origin
        double sx = rk.source_position(double(origin));
        for (int64_t i = 0; i < len; ++i) {
            int64_t s; int32_t ph;
            rk.plan(sx, &s, &ph);
            (*starts)[i] = int32_t(s); (*phases)[i] = uint8_t(ph);
            sx += rk.factor;
        }
    } else {
        for (int64_t i = 0; i < len; ++i) {
            int64_t s; int32_t ph;
            rk.plan(rk.source_position(double(origin) + double(i)), &s, &ph);
            (*starts)[i] = int32_t(s); (*phases)[i] = uint8_t(ph);
        }
    }
}

int add_reduce_stage(viprs_plan* p, const ReduceKernel& rk, bool horizontal, int mode, int in_plane,
                     int out_plane, bool incremental) {
    Stage st;
    st.type = horizontal ? StageType::ReduceH : StageType::ReduceV;
    st.in_plane = in_plane;
    st.out_plane = out_plane;
    const Region& o = p->planes[out_plane].r;
    std::vector<int32_t> starts;
    std::vector<uint8_t> phases;
    reduce_tables(rk, horizontal ? o.x : o.y, horizontal ? o.w : o.h, incremental, &starts, &phases);
    st.starts_off = push_table(p->host_tables, starts.data(), starts.size() * 4);
    st.phases_off = push_table(p->host_tables, phases.data(), phases.size());
    if (mode == kReduceFixed) {
        // int32 accumulation must hold sum |c| * max sample exactly
        const double maxv = p->fmt == kU8 ? 255.0 : 65535.0;
        if (double(rk.max_abs_i16_sum()) * maxv >= 2147483647.0) return VIPRS_ERR_TOO_MANY_TAPS;
        st.coeffs_off = push_table(p->host_tables, rk.coeffs_i16.data(), rk.coeffs_i16.size() * 2);
    } else {
        st.coeffs_off = push_table(p->host_tables, rk.coeffs_f64.data(), rk.coeffs_f64.size() * 8);
    }
    st.rd.bands = int32_t(p->bands);
    st.rd.fmt = p->fmt;
    st.rd.mode = mode;
    st.rd.taps = rk.taps;
    st.rd.vector_len = int32_t(o.w * p->bands / 4 * 4);
    p->stages.push_back(st);
    return VIPRS_OK;
}

int mode_for(int32_t fmt, bool horizontal, uint32_t bands);

// ReduceH and ReduceV fused into one launch (either order).  `first` produces
// the mid region `mid`; `second` produces `outr`.  Returns false (and adds
// nothing) when the tile does not fit in shared memory.
bool add_reduce2d_stage(viprs_plan* p, const ReduceKernel& first, const ReduceKernel& second, bool hfirst,
                        int mode_first, int mode_second, const Region& mid, const Region& outr, int in_plane,
                        int out_plane, bool incremental_h) {
    Stage st;
    st.type = StageType::Reduce2D;
    st.in_plane = in_plane;
    st.out_plane = out_plane;
    const ReduceKernel& rh = hfirst ? first : second;
    const ReduceKernel& rv = hfirst ? second : first;
    // H tables run over the columns of the H op's output, V tables over the rows of the V op's output
    const Region& hreg = hfirst ? mid : outr;
    const Region& vreg = hfirst ? outr : mid;
    std::vector<int32_t> sh, sv;
    std::vector<uint8_t> ph, pv;
    reduce_tables(rh, hreg.x, hreg.w, incremental_h, &sh, &ph);
    reduce_tables(rv, vreg.y, vreg.h, false, &sv, &pv);
    Reduce2DArgs& a = st.r2;
    a.bands = int32_t(p->bands);
    a.fmt = p->fmt;
    a.hfirst = hfirst ? 1 : 0;
    a.mx0 = mid.x; a.my0 = mid.y; a.mw = int32_t(mid.w); a.mh = int32_t(mid.h);
    a.taps_h = rh.taps; a.taps_v = rv.taps;
    a.mode_h = hfirst ? mode_first : mode_second;
    a.mode_v = hfirst ? mode_second : mode_first;
    a.vector_len = int32_t((hfirst ? outr.w : mid.w) * p->bands / 4 * 4);
    const double maxv = p->fmt == kU8 ? 255.0 : 65535.0;
    if (a.mode_h == kReduceFixed && double(rh.max_abs_i16_sum()) * maxv >= 2147483647.0) return false;
    if (a.mode_v == kReduceFixed && double(rv.max_abs_i16_sum()) * maxv >= 2147483647.0) return false;
    // tile shape: the largest whose staged rows, mid tile and output tile fit
    // 64 KB of shared memory while the launch still has two tiles per SM
    a.out.w = int32_t(outr.w);
    a.out.h = int32_t(outr.h);
    const Region& ir = p->planes[size_t(in_plane)].r;
    a.in.pitch = p->planes[size_t(in_plane)].pitch;
    if (!launch::reduce2d_configure(&a, sh.data(), sv.data(), ir.x, ir.y, ir.w, ir.h, 2 * 148, 64 * 1024))
        return false;
    if (launch::reduce2d_smem_bytes(a) == 0) return false;
    st.starts_off = push_table(p->host_tables, sh.data(), sh.size() * 4);
    st.phases_off = push_table(p->host_tables, ph.data(), ph.size());
    st.starts2_off = push_table(p->host_tables, sv.data(), sv.size() * 4);
    st.phases2_off = push_table(p->host_tables, pv.data(), pv.size());
    if (a.mode_h == kReduceFixed) st.coeffs_off = push_table(p->host_tables, rh.coeffs_i16.data(), rh.coeffs_i16.size() * 2);
    else st.coeffs_off = push_table(p->host_tables, rh.coeffs_f64.data(), rh.coeffs_f64.size() * 8);
    if (a.mode_v == kReduceFixed) st.coeffs2_off = push_table(p->host_tables, rv.coeffs_i16.data(), rv.coeffs_i16.size() * 2);
    else st.coeffs2_off = push_table(p->host_tables, rv.coeffs_f64.data(), rv.coeffs_f64.size() * 8);
    p->stages.push_back(st);
    return true;
}

int mode_for(int32_t fmt, bool horizontal, uint32_t bands) {
    if (fmt == kU8 || fmt == kU16) return kReduceFixed;
    // f32: x86 AVX2 order for 1-band H and for V; scalar fma for multi-band H
    if (horizontal && bands != 1) return kReduceF64Fma;
    return kReduceF32Simd;
}

int build_chain(viprs_plan* p, const Chain& chain) {
    const size_t es = format_size(Format(p->fmt));
    const int n = int(chain.nodes.size());
    std::vector<NodeRt> rt(size_t(std::max(n, 1)));
    uint32_t cw = p->in_w, ch = p->in_h;
    for (int i = 0; i < n; ++i) {
        NodeRt& r = rt[i];
        r.n = chain.nodes[i];
        r.in_w = cw; r.in_h = ch;
        int st = node_output_dims(r.n, cw, ch, &r.out_w, &r.out_h);
        if (st) return st;
        if (r.n.kind == NodeKind::ReduceH || r.n.kind == NodeKind::ReduceV || r.n.kind == NodeKind::Reduce) {
            st = r.rk.init(r.n.factor, r.n.kernel);
            if (st) return st;
            if (r.n.kind == NodeKind::ReduceH) r.rk.bind_input_len(cw);
            if (r.n.kind == NodeKind::ReduceV) r.rk.bind_input_len(ch);
            if (r.n.kind == NodeKind::Reduce) {
                st = r.rk2.init(r.n.vfactor, r.n.kernel);
                if (st) return st;
            }
        }
        if ((r.n.kind == NodeKind::Premultiply || r.n.kind == NodeKind::Unpremultiply) && p->bands < 2)
            return VIPRS_ERR_INVALID_ARGUMENT;
        if (r.n.kind == NodeKind::Premultiply && p->fmt != kU8) return VIPRS_ERR_UNSUPPORTED_FORMAT;
        if (r.n.kind == NodeKind::Unpremultiply && p->fmt == kU16) return VIPRS_ERR_UNSUPPORTED_FORMAT;
        if (r.n.kind == NodeKind::Affine) {
            if (!affine_kernel_supported(r.n.kernel)) return VIPRS_ERR_INVALID_KERNEL;
        }
        cw = r.out_w; ch = r.out_h;
    }
    p->out_w = cw; p->out_h = ch;
    if (chain.out_w != 0 && (chain.out_w != cw || chain.out_h != ch)) return VIPRS_ERR_SIZE_MISMATCH;

    // regions: out[i] = output region of node i
    std::vector<Region> out(size_t(std::max(n, 1)));
    if (n > 0) {
        out[n - 1] = Region{0, 0, int64_t(cw), int64_t(ch)};
        for (int i = n - 1; i > 0; --i) {
            int st = required_region(rt[i].n, &rt[i].rk, &rt[i].rk2, rt[i].in_w, rt[i].in_h, out[i], &out[i - 1]);
            if (st) return st;
        }
    }

    size_t ws = 0;
    p->planes.clear();
    PlaneInfo src;
    src.r = Region{0, 0, int64_t(p->in_w), int64_t(p->in_h)};
    src.pitch = p->in_pitch;
    p->planes.push_back(src);
    // plane index holding each node's output
    std::vector<int> node_plane(size_t(std::max(n, 1)), 0);
    auto plane_for = [&](int i) -> int {
        if (i == n - 1) return -1;  // destination, appended at the end
        return add_plane(p, out[i], es, &ws);
    };

    int cur = 0;  // plane holding the current value
    bool pending_premul = false;
    int i = 0;
    while (i < n) {
        const PlanNode& nd = rt[i].n;
        if (nd.kind == NodeKind::Premultiply) {
            const bool fusable = i + 1 < n && p->fmt == kU8 &&
                                 (rt[i + 1].n.kind == NodeKind::ShrinkH || rt[i + 1].n.kind == NodeKind::ShrinkV ||
                                  rt[i + 1].n.kind == NodeKind::ReduceH || rt[i + 1].n.kind == NodeKind::ReduceV);
            if (fusable) { pending_premul = true; ++i; continue; }
            Stage st; st.type = StageType::Pixel; st.in_plane = cur; st.out_plane = plane_for(i);
            st.px.bands = int32_t(p->bands); st.px.fmt = p->fmt; st.px.op = 1;
            p->stages.push_back(st);
            cur = st.out_plane; ++i;
            continue;
        }
        if (nd.kind == NodeKind::Unpremultiply) {
            if (!p->stages.empty() && p->fmt == kU8 && i == n - 1 && cur != 0) {
                Stage& last = p->stages.back();
                const bool ok = (last.type == StageType::Shrink && last.sh.hv_order) ||
                                ((last.type == StageType::ReduceH || last.type == StageType::ReduceV ||
                                  last.type == StageType::Reduce2D) &&
                                 (256 % p->bands) == 0) ||
                                last.type == StageType::Affine;
                if (ok && last.out_plane == cur) {
                    // retarget the previous stage's output to this node's output and
                    // unpremultiply in its store
                    last.sh.unpremul_out = 1; last.rd.unpremul_out = 1; last.af.unpremul_out = 1;
                    last.r2.unpremul_out = 1;
                    last.out_plane = -1;
                    // the intermediate plane that stage wrote is no longer needed
                    cur = -1; ++i;
                    continue;
                }
            }
            Stage st; st.type = StageType::Pixel; st.in_plane = cur; st.out_plane = plane_for(i);
            st.px.bands = int32_t(p->bands); st.px.fmt = p->fmt; st.px.op = 2;
            p->stages.push_back(st);
            cur = st.out_plane; ++i;
            continue;
        }
        if (nd.kind == NodeKind::ShrinkH || nd.kind == NodeKind::ShrinkV || nd.kind == NodeKind::Shrink) {
            Stage st; st.type = StageType::Shrink; st.in_plane = cur;
            st.sh.bands = int32_t(p->bands); st.sh.fmt = p->fmt;
            st.sh.premul_in = pending_premul ? 1 : 0;
            pending_premul = false;
            int last = i;
            if (nd.kind == NodeKind::Shrink) {
                st.sh.fh = nd.ufactor; st.sh.fv = nd.vufactor; st.sh.hv_order = 1;
            } else if (nd.kind == NodeKind::ShrinkH) {
                st.sh.fh = nd.ufactor; st.sh.hv_order = 1;
                if (i + 1 < n && rt[i + 1].n.kind == NodeKind::ShrinkV && !rt[i + 1].n.ceil && !nd.ceil) {
                    st.sh.fv = rt[i + 1].n.ufactor; last = i + 1;
                }
            } else {
                st.sh.fv = nd.ufactor; st.sh.hv_order = 0;
                if (i + 1 < n && rt[i + 1].n.kind == NodeKind::ShrinkH && !rt[i + 1].n.ceil && !nd.ceil) {
                    st.sh.fh = rt[i + 1].n.ufactor; last = i + 1;
                }
                if (st.sh.fh == 1) st.sh.hv_order = 1;  // a lone ShrinkV is the same either way
            }
            st.out_plane = plane_for(last);
            p->stages.push_back(st);
            cur = st.out_plane; i = last + 1;
            continue;
        }
        if ((nd.kind == NodeKind::ReduceH || nd.kind == NodeKind::ReduceV) && i + 1 < n &&
            ((nd.kind == NodeKind::ReduceH && rt[i + 1].n.kind == NodeKind::ReduceV) ||
             (nd.kind == NodeKind::ReduceV && rt[i + 1].n.kind == NodeKind::ReduceH))) {
            const bool hfirst = nd.kind == NodeKind::ReduceH;
            const int op = plane_for(i + 1);
            if (op < 0) { PlaneInfo dst; dst.r = out[i + 1]; p->planes.push_back(dst); }
            const int oplane = op < 0 ? int(p->planes.size()) - 1 : op;
            const bool ok = add_reduce2d_stage(p, rt[i].rk, rt[i + 1].rk, hfirst, mode_for(p->fmt, hfirst, p->bands),
                                               mode_for(p->fmt, !hfirst, p->bands), out[i], out[i + 1], cur, oplane,
                                               p->fmt == kU8);
            if (op < 0) p->planes.pop_back();
            if (ok) {
                if (op < 0) p->stages.back().out_plane = -1;
                if (pending_premul) { p->stages.back().r2.premul_in = 1; pending_premul = false; }
                cur = op; i += 2;
                continue;
            }
            if (op >= 0) p->planes.pop_back();  // not fusable: fall through to two launches
        }
        if (nd.kind == NodeKind::ReduceH || nd.kind == NodeKind::ReduceV) {
            const bool h = nd.kind == NodeKind::ReduceH;
            const int op = plane_for(i);
            const int mode = mode_for(p->fmt, h, p->bands);
            const bool incremental = h && p->fmt == kU8;
            // the destination plane is appended after the loop; use a placeholder region
            if (op < 0) {
                PlaneInfo dst; dst.r = out[i]; p->planes.push_back(dst);
            }
            const int oplane = op < 0 ? int(p->planes.size()) - 1 : op;
            int st = add_reduce_stage(p, rt[i].rk, h, mode, cur, oplane, incremental);
            if (st) return st;
            if (op < 0) { p->planes.pop_back(); p->stages.back().out_plane = -1; }
            if (pending_premul) { p->stages.back().rd.premul_in = 1; pending_premul = false; }
            cur = op; ++i;
            continue;
        }
        if (nd.kind == NodeKind::Reduce) {
            // ReduceOp: H into the intermediate ReduceConfig region, then V (reduce.rs:103-251)
            Region mid = out[i];
            rt[i].rk2.config_required_axis(out[i].y, out[i].h, &mid.y, &mid.h);
            {
                const int op = plane_for(i);
                if (op < 0) { PlaneInfo dst; dst.r = out[i]; p->planes.push_back(dst); }
                const int oplane = op < 0 ? int(p->planes.size()) - 1 : op;
                const bool ok = add_reduce2d_stage(p, rt[i].rk, rt[i].rk2, true, kReduceF64Fma, kReduceF64Fma, mid,
                                                   out[i], cur, oplane, false);
                if (op < 0) p->planes.pop_back();
                if (ok) {
                    if (op < 0) p->stages.back().out_plane = -1;
                    cur = op; ++i;
                    continue;
                }
                if (op >= 0) p->planes.pop_back();
            }
            const int midp = add_plane(p, mid, es, &ws);
            int st = add_reduce_stage(p, rt[i].rk, true, kReduceF64Fma, cur, midp, false);
            if (st) return st;
            const int op = plane_for(i);
            if (op < 0) { PlaneInfo dst; dst.r = out[i]; p->planes.push_back(dst); }
            const int oplane = op < 0 ? int(p->planes.size()) - 1 : op;
            st = add_reduce_stage(p, rt[i].rk2, false, kReduceF64Fma, midp, oplane, false);
            if (st) return st;
            if (op < 0) { p->planes.pop_back(); p->stages.back().out_plane = -1; }
            cur = op; ++i;
            continue;
        }
        if (nd.kind == NodeKind::Affine) {
            Stage st; st.type = StageType::Affine; st.in_plane = cur; st.out_plane = plane_for(i);
            // tiles cover the final output; an ExtractArea after the affine shifts them
            int64_t offx = 0, offy = 0;
            if (i + 1 < n && rt[i + 1].n.kind == NodeKind::ExtractArea) { offx = rt[i + 1].n.ex; offy = rt[i + 1].n.ey; }
            int s2 = affine_stage_setup(nd, rt[i].in_w, rt[i].in_h, p->bands, p->fmt, chain.demand_override,
                                        default_demand(chain), cw, ch, offx, offy, &st.af);
            if (s2) return s2;
            if (st.af.separable && !st.af.fast) {
                std::vector<double> xs(std::max<uint32_t>(st.af.total_w, 1)), ys(std::max<uint32_t>(st.af.total_h, 1));
                affine_axis_tables(st.af, xs.data(), ys.data());
                st.starts_off = push_table(p->host_tables, xs.data(), xs.size() * 8);
                st.phases_off = push_table(p->host_tables, ys.data(), ys.size() * 8);
                if (affine_weight_tables_apply(st.af)) {
                    std::vector<double> wx(xs.size() * kAxisTaps), wy(ys.size() * kAxisTaps);
                    affine_weight_tables(st.af, xs.data(), ys.data(), wx.data(), wy.data());
                    st.coeffs_off = push_table(p->host_tables, wx.data(), wx.size() * 8);
                    st.coeffs2_off = push_table(p->host_tables, wy.data(), wy.size() * 8);
                    st.axis_weights = true;
                }
            }
            p->stages.push_back(st);
            cur = st.out_plane; ++i;
            continue;
        }
        if (nd.kind == NodeKind::Zoom) {
            Stage st; st.type = StageType::Pixel; st.in_plane = cur; st.out_plane = plane_for(i);
            st.px.bands = int32_t(p->bands); st.px.fmt = p->fmt; st.px.op = 3;
            st.px.zx = int32_t(nd.zx); st.px.zy = int32_t(nd.zy);
            p->stages.push_back(st);
            cur = st.out_plane; ++i;
            continue;
        }
        if (nd.kind == NodeKind::ExtractArea) {
            Stage st; st.type = StageType::Pixel; st.in_plane = cur; st.out_plane = plane_for(i);
            st.px.bands = int32_t(p->bands); st.px.fmt = p->fmt; st.px.op = 0;
            p->stages.push_back(st);
            cur = st.out_plane; ++i;
            continue;
        }
        return VIPRS_ERR_UNSUPPORTED_FORMAT;
    }
    if (n == 0 || p->stages.empty()) {
        // identity: a copy
        Stage st; st.type = StageType::Pixel; st.in_plane = 0; st.out_plane = -1;
        st.px.bands = int32_t(p->bands); st.px.fmt = p->fmt; st.px.op = 0;
        p->stages.push_back(st);
    }
    // destination plane
    PlaneInfo dst;
    dst.r = Region{0, 0, int64_t(p->out_w), int64_t(p->out_h)};
    dst.pitch = p->out_pitch;
    p->planes.push_back(dst);
    const int dst_idx = int(p->planes.size()) - 1;
    for (auto& s : p->stages)
        if (s.out_plane < 0) s.out_plane = dst_idx;
    p->work_bytes = ws;
    return VIPRS_OK;
}

int alloc_plan(viprs_plan* p, cudaStream_t stream, bool stream_ordered) {
    cudaGetDevice(&p->device);
    p->stream_ordered_alloc = stream_ordered;
    p->alloc_stream = stream;
    static const int32_t zero[4] = {0, 0, 0, 0};
    p->err_off = push_table(p->host_tables, zero, sizeof(zero));
    const size_t tb = std::max<size_t>(p->host_tables.size(), 16);
    cudaError_t e;
    if (stream_ordered) {
        e = cudaMallocAsync(reinterpret_cast<void**>(&p->d_tables), tb, stream);
        if (e == cudaSuccess && p->work_bytes) e = cudaMallocAsync(reinterpret_cast<void**>(&p->d_work), p->work_bytes, stream);
        if (e == cudaSuccess && !p->host_tables.empty())
            e = cudaMemcpyAsync(p->d_tables, p->host_tables.data(), p->host_tables.size(), cudaMemcpyHostToDevice, stream);
    } else {
        e = cudaMalloc(reinterpret_cast<void**>(&p->d_tables), tb);
        if (e == cudaSuccess && p->work_bytes) e = cudaMalloc(reinterpret_cast<void**>(&p->d_work), p->work_bytes);
        if (e == cudaSuccess && !p->host_tables.empty())
            e = cudaMemcpy(p->d_tables, p->host_tables.data(), p->host_tables.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) p->d_err = reinterpret_cast<int32_t*>(p->d_tables + p->err_off);
    return cuda_status(e);
}

void free_plan_a(viprs_plan* p) {
    if (!p) return;
    if (p->stream_ordered_alloc) {
        if (p->d_tables) cudaFreeAsync(p->d_tables, p->alloc_stream);
        if (p->d_work) cudaFreeAsync(p->d_work, p->alloc_stream);
    } else {
        if (p->d_tables) cudaFree(p->d_tables);
        if (p->d_work) cudaFree(p->d_work);
    }
    if (p->d_in) cudaFree(p->d_in);
    if (p->d_out) cudaFree(p->d_out);
    delete p;
}

PlaneArg in_arg_a(const viprs_plan* p, int idx, const uint8_t* src) {
    const PlaneInfo& pi = p->planes[idx];
    PlaneArg a;
    a.x0 = pi.r.x; a.y0 = pi.r.y; a.w = int32_t(pi.r.w); a.h = int32_t(pi.r.h);
    a.pitch = pi.pitch;
    if (idx == 0) a.data = src;
    else a.data = p->d_work + pi.offset;
    const int64_t row_bytes = std::max<int64_t>(pi.r.w, 0) * p->bands * int64_t(format_size(Format(p->fmt)));
    a.total_bytes = pi.r.h > 0 ? pi.pitch * (pi.r.h - 1) + row_bytes : 0;
    return a;
}

OutPlaneArg out_arg_a(const viprs_plan* p, int idx, uint8_t* dst) {
    const PlaneInfo& pi = p->planes[idx];
    OutPlaneArg a;
    a.x0 = pi.r.x; a.y0 = pi.r.y; a.w = int32_t(pi.r.w); a.h = int32_t(pi.r.h);
    a.pitch = pi.pitch;
    a.data = idx == int(p->planes.size()) - 1 ? dst : p->d_work + pi.offset;
    return a;
}

int execute_a(viprs_plan* p, const void* src, void* dst, cudaStream_t s, int first = 0, int count = -1) {
    const uint8_t* in = static_cast<const uint8_t*>(src);
    uint8_t* out = static_cast<uint8_t*>(dst);
    const int nst = int(p->stages.size());
    const int last = count < 0 ? nst : std::min(nst, first + count);
    for (int si = std::max(first, 0); si < last; ++si) {
        Stage& st = p->stages[size_t(si)];
        const PlaneArg ia = in_arg_a(p, st.in_plane, in);
        const OutPlaneArg oa = out_arg_a(p, st.out_plane, out);
        cudaError_t e = cudaSuccess;
        switch (st.type) {
        case StageType::Shrink: {
            ShrinkArgs a = st.sh; a.in = ia; a.out = oa; a.err = p->d_err;
            e = launch::shrink2d(a, s);
            break;
        }
        case StageType::ReduceH:
        case StageType::ReduceV: {
            ReduceArgs a = st.rd; a.in = ia; a.out = oa;
            a.starts = reinterpret_cast<const int32_t*>(p->d_tables + st.starts_off);
            a.phases = p->d_tables + st.phases_off;
            a.coeffs = p->d_tables + st.coeffs_off;
            e = st.type == StageType::ReduceH ? launch::reduce_h(a, s) : launch::reduce_v(a, s);
            break;
        }
        case StageType::Reduce2D: {
            Reduce2DArgs a = st.r2; a.in = ia; a.out = oa;
            a.starts_h = reinterpret_cast<const int32_t*>(p->d_tables + st.starts_off);
            a.phases_h = p->d_tables + st.phases_off;
            a.starts_v = reinterpret_cast<const int32_t*>(p->d_tables + st.starts2_off);
            a.phases_v = p->d_tables + st.phases2_off;
            a.coeffs_h = p->d_tables + st.coeffs_off;
            a.coeffs_v = p->d_tables + st.coeffs2_off;
            a.err = p->d_err;
            e = launch::reduce2d(a, s);
            break;
        }
        case StageType::Pixel: {
            PixelArgs a = st.px; a.in = ia; a.out = oa;
            e = launch::pixel(a, s);
            break;
        }
        case StageType::Affine: {
            AffineArgs a = st.af; a.in = ia; a.out = oa;
            if (a.separable && !a.fast) {
                a.xs = reinterpret_cast<const double*>(p->d_tables + st.starts_off);
                a.ys = reinterpret_cast<const double*>(p->d_tables + st.phases_off);
            }
            if (st.axis_weights) {
                a.wx = reinterpret_cast<const double*>(p->d_tables + st.coeffs_off);
                a.wy = reinterpret_cast<const double*>(p->d_tables + st.coeffs2_off);
            }
            e = launch::affine(a, s);
            break;
        }
        }
        if (e != cudaSuccess) return cuda_status(e);
    }
    return VIPRS_OK;
}

int check_image(const viprs_image* im) {
    if (!im || !im->data) return VIPRS_ERR_NULL_POINTER;
    if (im->bands == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    if (im->format < 0 || im->format > 2) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    // a row must start on a sample and hold a whole row of pixels
    const uint64_t es = format_size(Format(im->format));
    if (reinterpret_cast<uintptr_t>(im->data) % es) return VIPRS_ERR_INVALID_ARGUMENT;
    if (im->row_stride && (im->row_stride % es || im->row_stride < uint64_t(im->width) * im->bands * es))
        return VIPRS_ERR_INVALID_ARGUMENT;
    return VIPRS_OK;
}

int64_t pitch_of(const viprs_image* im) {
    const int64_t packed = int64_t(im->width) * im->bands * format_size(Format(im->format));
    return im->row_stride ? int64_t(im->row_stride) : packed;
}

// One-shot execution of a single-node chain with stream-ordered allocations.
int run_single(const viprs_image* in, const viprs_image* out, const PlanNode& node, void* stream) {
    int st = check_image(in);
    if (st) return st;
    if (in->width == 0 || in->height == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    {
        // parameter errors first (BuildError happens before any pixel is touched)
        uint32_t ow, oh;
        st = node_output_dims(node, in->width, in->height, &ow, &oh);
        if (st) return st;
        if (node.kind == NodeKind::ReduceH || node.kind == NodeKind::ReduceV || node.kind == NodeKind::Reduce) {
            ReduceKernel rk;
            st = rk.init(node.factor, node.kernel);
            if (st == VIPRS_OK && node.kind == NodeKind::Reduce) st = rk.init(node.vfactor, node.kernel);
            if (st) return st;
        }
    }
    if (!out) return VIPRS_ERR_NULL_POINTER;
    if (out->width == 0 || out->height == 0) return VIPRS_ERR_SIZE_MISMATCH;
    st = check_image(out);
    if (st) return st;
    if (in->format != out->format || in->bands != out->bands) return VIPRS_ERR_SIZE_MISMATCH;
    std::unique_ptr<viprs_plan> p(new (std::nothrow) viprs_plan());
    if (!p) return VIPRS_ERR_OUT_OF_MEMORY;
    p->in_w = in->width; p->in_h = in->height; p->bands = in->bands; p->fmt = in->format;
    p->in_pitch = pitch_of(in);
    p->out_pitch = pitch_of(out);
    Chain c;
    c.nodes.push_back(node);
    st = build_chain(p.get(), c);
    if (st) return st;
    if (p->out_w != out->width || p->out_h != out->height) return VIPRS_ERR_SIZE_MISMATCH;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    st = alloc_plan(p.get(), s, true);
    if (st == VIPRS_OK) st = execute_a(p.get(), in->data, out->data, s);
    free_plan_a(p.release());
    return st;
}

int create_chain_plan_a(uint32_t w, uint32_t h, uint32_t bands, int32_t format, const Chain& chain,
                      viprs_plan** out) {
    if (!out) return VIPRS_ERR_NULL_POINTER;
    *out = nullptr;
    if (bands == 0 || w == 0 || h == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    if (format < 0 || format > 2) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    std::unique_ptr<viprs_plan> p(new (std::nothrow) viprs_plan());
    if (!p) return VIPRS_ERR_OUT_OF_MEMORY;
    p->in_w = w; p->in_h = h; p->bands = bands; p->fmt = format;
    p->in_pitch = int64_t(w) * bands * format_size(Format(format));
    int st = build_chain(p.get(), chain);
    if (st) return st;
    p->out_pitch = int64_t(p->out_w) * bands * format_size(Format(format));
    p->planes.back().pitch = p->out_pitch;
    st = alloc_plan(p.get(), nullptr, false);
    if (st) { free_plan_a(p.release()); return st; }
    *out = p.release();
    return VIPRS_OK;
}

}  // namespace

namespace viprs {
int32_t nodes_to_chain(const viprs_node* nodes, int32_t n_nodes, int32_t demand_override, Chain* out) {
    if (n_nodes < 0 || (n_nodes > 0 && !nodes) || !out) return VIPRS_ERR_NULL_POINTER;
    Chain c;
    c.demand_override = demand_override < 0 ? -1 : demand_override;
    if (demand_override > 5) return VIPRS_ERR_INVALID_ARGUMENT;
    for (int32_t i = 0; i < n_nodes; ++i) {
        const viprs_node& v = nodes[i];
        PlanNode n;
        switch (v.kind) {
        case VIPRS_NODE_PREMULTIPLY: n.kind = NodeKind::Premultiply; break;
        case VIPRS_NODE_UNPREMULTIPLY: n.kind = NodeKind::Unpremultiply; break;
        case VIPRS_NODE_SHRINKH: n.kind = NodeKind::ShrinkH; break;
        case VIPRS_NODE_SHRINKV: n.kind = NodeKind::ShrinkV; break;
        case VIPRS_NODE_SHRINK: n.kind = NodeKind::Shrink; break;
        case VIPRS_NODE_REDUCEH: n.kind = NodeKind::ReduceH; break;
        case VIPRS_NODE_REDUCEV: n.kind = NodeKind::ReduceV; break;
        case VIPRS_NODE_REDUCE: n.kind = NodeKind::Reduce; break;
        case VIPRS_NODE_AFFINE: n.kind = NodeKind::Affine; break;
        case VIPRS_NODE_EXTRACT_AREA: n.kind = NodeKind::ExtractArea; break;
        case VIPRS_NODE_ZOOM: n.kind = NodeKind::Zoom; break;
        default: return VIPRS_ERR_INVALID_ARGUMENT;
        }
        if (v.kernel < 0 || v.kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
        if (v.extend < 0 || v.extend > 5) return VIPRS_ERR_INVALID_ARGUMENT;
        if (v.demand_hint < 0 || v.demand_hint > 5) return VIPRS_ERR_INVALID_ARGUMENT;
        n.ufactor = v.factor_u; n.vufactor = v.vfactor_u; n.ceil = v.ceil_mode != 0;
        n.factor = v.factor; n.vfactor = v.vfactor; n.kernel = Kernel(v.kernel);
        std::memcpy(n.m, v.matrix, sizeof(n.m));
        n.tx = v.tx; n.ty = v.ty; n.out_w = v.out_width; n.out_h = v.out_height;
        n.extend = Extend(v.extend); n.background = v.background; n.premultiplied = v.premultiplied != 0;
        n.ex = v.area_x; n.ey = v.area_y;
        if (n.kind == NodeKind::ExtractArea) { n.ew = v.area_width; n.eh = v.area_height; }
        if (n.kind == NodeKind::Zoom) { n.zx = v.factor_u; n.zy = v.vfactor_u; }
        n.demand = Demand(v.demand_hint);
        c.nodes.push_back(n);
    }
    *out = c;
    return VIPRS_OK;
}

int create_chain_plan(uint32_t w, uint32_t h, uint32_t bands, int32_t format, const Chain& chain, viprs_plan** out) {
    return create_chain_plan_a(w, h, bands, format, chain, out);
}
int execute_plan(viprs_plan* p, const void* src, void* dst, cudaStream_t s, int first, int count) {
    return execute_a(p, src, dst, s, first, count);
}
void free_plan(viprs_plan* p) { free_plan_a(p); }
PlaneArg plane_in_arg(const viprs_plan* p, int idx, const uint8_t* src) { return in_arg_a(p, idx, src); }
OutPlaneArg plane_out_arg(const viprs_plan* p, int idx, uint8_t* dst) { return out_arg_a(p, idx, dst); }

// Host-side planning of a one-node chain for `in` -> `out`, with the same
// checks, in the same order, as the allocating single-op entry points; the
// plan's device pointers are left null for the caller to point at memory it
// already has.
int plan_single_node(const viprs_image* in, const viprs_image* out, const PlanNode& node, viprs_plan* p) {
    int st = check_image(in);
    if (st) return st;
    if (in->width == 0 || in->height == 0) return VIPRS_ERR_INVALID_ARGUMENT;
    uint32_t ow, oh;
    st = node_output_dims(node, in->width, in->height, &ow, &oh);
    if (st) return st;
    if (node.kind == NodeKind::ReduceH || node.kind == NodeKind::ReduceV || node.kind == NodeKind::Reduce) {
        ReduceKernel rk;
        st = rk.init(node.factor, node.kernel);
        if (st == VIPRS_OK && node.kind == NodeKind::Reduce) st = rk.init(node.vfactor, node.kernel);
        if (st) return st;
    }
    if (!out) return VIPRS_ERR_NULL_POINTER;
    if (out->width == 0 || out->height == 0) return VIPRS_ERR_SIZE_MISMATCH;
    st = check_image(out);
    if (st) return st;
    if (in->format != out->format || in->bands != out->bands) return VIPRS_ERR_SIZE_MISMATCH;
    p->in_w = in->width; p->in_h = in->height; p->bands = in->bands; p->fmt = in->format;
    p->in_pitch = pitch_of(in);
    p->out_pitch = pitch_of(out);
    Chain c;
    c.nodes.push_back(node);
    st = build_chain(p, c);
    if (st) return st;
    if (p->out_w != out->width || p->out_h != out->height) return VIPRS_ERR_SIZE_MISMATCH;
    return VIPRS_OK;
}
}  // namespace viprs

extern "C" {

const char* viprs_status_string(int32_t status) {
    switch (status) {
    case VIPRS_OK: return "ok";
    case VIPRS_ERR_INVALID_ARGUMENT: return "invalid argument";
    case VIPRS_ERR_UNSUPPORTED_FORMAT: return "unsupported format or node";
    case VIPRS_ERR_TOO_MANY_TAPS: return "factor produces too many filter taps";
    case VIPRS_ERR_OUT_OF_MEMORY: return "out of device memory";
    case VIPRS_ERR_CUDA: return "CUDA error";
    case VIPRS_ERR_TIMEOUT: return "device wait timed out";
    case VIPRS_ERR_INVALID_KERNEL: return "interpolation kernel not valid for this op";
    case VIPRS_ERR_DEGENERATE_AFFINE: return "affine matrix determinant is singular";
    case VIPRS_ERR_NULL_POINTER: return "null pointer";
    case VIPRS_ERR_SIZE_MISMATCH: return "image size, bands or format mismatch";
    case VIPRS_ERR_SCRATCH_LIMIT: return "work exceeds the static scratch of the no-alloc entry point";
    default: return "unknown status";
    }
}

int32_t viprs_last_cuda_error(void) { return g_last_cuda_error; }

int32_t viprs_sin_rn(const double* x, double* out, int64_t n) {
    if (n > 0 && (!x || !out)) return VIPRS_ERR_INVALID_ARGUMENT;
    for (int64_t i = 0; i < n; ++i) out[i] = sinrn::sin_rn(x[i]);
    return VIPRS_OK;
}

uint32_t viprs_reduce_output_len(double factor, uint32_t input_len) {
    return reduce_output_len(factor, input_len);
}

int32_t viprs_reduce_kernel_table(double factor, int32_t kernel, int32_t* taps, int16_t* coeffs) {
    ReduceKernel rk;
    const int st = rk.init(factor, Kernel(kernel));
    if (st) return st;
    if (taps) *taps = rk.taps;
    if (coeffs) std::memcpy(coeffs, rk.coeffs_i16.data(), rk.coeffs_i16.size() * 2);
    return VIPRS_OK;
}

int32_t viprs_reduceh(const viprs_image* in, const viprs_image* out, double factor, int32_t kernel, void* stream) {
    PlanNode n; n.kind = NodeKind::ReduceH; n.factor = factor; n.kernel = Kernel(kernel);
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    return run_single(in, out, n, stream);
}

int32_t viprs_reducev(const viprs_image* in, const viprs_image* out, double factor, int32_t kernel, void* stream) {
    PlanNode n; n.kind = NodeKind::ReduceV; n.factor = factor; n.kernel = Kernel(kernel);
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    return run_single(in, out, n, stream);
}

int32_t viprs_reduce(const viprs_image* in, const viprs_image* out, double hfactor, double vfactor, int32_t kernel,
                     void* stream) {
    PlanNode n; n.kind = NodeKind::Reduce; n.factor = hfactor; n.vfactor = vfactor; n.kernel = Kernel(kernel);
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    return run_single(in, out, n, stream);
}

int32_t viprs_shrinkh(const viprs_image* in, const viprs_image* out, uint32_t factor, int32_t ceil_mode, void* stream) {
    PlanNode n; n.kind = NodeKind::ShrinkH; n.ufactor = factor; n.ceil = ceil_mode != 0;
    return run_single(in, out, n, stream);
}

int32_t viprs_shrinkv(const viprs_image* in, const viprs_image* out, uint32_t factor, int32_t ceil_mode, void* stream) {
    PlanNode n; n.kind = NodeKind::ShrinkV; n.ufactor = factor; n.ceil = ceil_mode != 0;
    return run_single(in, out, n, stream);
}

int32_t viprs_shrink(const viprs_image* in, const viprs_image* out, uint32_t hf, uint32_t vf, void* stream) {
    PlanNode n; n.kind = NodeKind::Shrink; n.ufactor = hf; n.vufactor = vf;
    return run_single(in, out, n, stream);
}

int32_t viprs_similarity(const viprs_image* in, const viprs_image* out, double scale, double angle, int32_t kernel,
                         void* stream) {
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    if (!std::isfinite(angle)) return VIPRS_ERR_INVALID_ARGUMENT;
    if (!in) return VIPRS_ERR_NULL_POINTER;
    const PlanNode n = similarity_node(scale, angle, Kernel(kernel), in->width, in->height);
    return run_single(in, out, n, stream);
}

int32_t viprs_zoom(const viprs_image* in, const viprs_image* out, uint32_t xfac, uint32_t yfac, void* stream) {
    PlanNode n; n.kind = NodeKind::Zoom; n.zx = xfac; n.zy = yfac;
    return run_single(in, out, n, stream);
}

int32_t viprs_premultiply(const viprs_image* in, const viprs_image* out, void* stream) {
    PlanNode n; n.kind = NodeKind::Premultiply;
    return run_single(in, out, n, stream);
}

int32_t viprs_unpremultiply(const viprs_image* in, const viprs_image* out, void* stream) {
    PlanNode n; n.kind = NodeKind::Unpremultiply;
    return run_single(in, out, n, stream);
}

int32_t viprs_affine(const viprs_image* in, const viprs_image* out, const double matrix[4], double tx, double ty,
                     int32_t kernel, void* stream) {
    if (!matrix) return VIPRS_ERR_NULL_POINTER;
    PlanNode n; n.kind = NodeKind::Affine;
    double b[4], btx, bty;
    const int st = forward_affine_to_backward(matrix, tx, ty, b, &btx, &bty);
    if (st) return st;
    std::memcpy(n.m, b, sizeof(b));
    n.tx = btx; n.ty = bty;
    n.kernel = Kernel(kernel);
    n.out_w = out ? out->width : 0; n.out_h = out ? out->height : 0;
    n.extend = Extend::Background; n.background = 0.0;
    n.demand = Demand::SmallTile;
    return run_single(in, out, n, stream);
}

int32_t viprs_affine_backward_matrix(const viprs_image* in, const viprs_image* out, const double m[4], double tx,
                                     double ty, int32_t kernel, int32_t extend, double background,
                                     int32_t premultiplied, uint32_t tile_w, uint32_t tile_h, void* stream) {
    if (!m) return VIPRS_ERR_NULL_POINTER;
    if (extend < 0 || extend > 5) return VIPRS_ERR_INVALID_ARGUMENT;
    PlanNode n; n.kind = NodeKind::Affine;
    std::memcpy(n.m, m, sizeof(n.m));
    n.tx = tx; n.ty = ty;
    n.kernel = Kernel(kernel);
    n.out_w = out ? out->width : 0; n.out_h = out ? out->height : 0;
    n.extend = Extend(extend); n.background = background; n.premultiplied = premultiplied != 0;
    n.demand = Demand::SmallTile;
    n.ew = tile_w; n.eh = tile_h;  // explicit tile grid (0 = from the demand hint)
    return run_single(in, out, n, stream);
}

int32_t viprs_mapim(const viprs_image* src, const viprs_image* index, const viprs_image* out, int32_t kernel,
                    int32_t extend_copy, double background, int32_t premultiplied, void* stream) {
    int st = check_image(src);
    if (st) return st;
    st = check_image(index);
    if (st) return st;
    st = check_image(out);
    if (st) return st;
    // any index format is read as f64 (mapim.rs:1135-1274)
    if (index->bands != 2) return VIPRS_ERR_UNSUPPORTED_FORMAT;
    if (out->format != src->format || out->bands != src->bands) return VIPRS_ERR_SIZE_MISMATCH;
    if (index->width != out->width || index->height != out->height) return VIPRS_ERR_SIZE_MISMATCH;
    if (kernel < 0 || kernel > 9 || !affine_kernel_supported(Kernel(kernel))) return VIPRS_ERR_INVALID_KERNEL;
    if (src->bands > 8) return VIPRS_ERR_INVALID_ARGUMENT;
    MapimArgs a;
    a.src.data = static_cast<const uint8_t*>(src->data);
    a.src.w = int32_t(src->width); a.src.h = int32_t(src->height); a.src.pitch = pitch_of(src);
    a.src.total_bytes = a.src.pitch * src->height;
    a.index.data = static_cast<const uint8_t*>(index->data);
    a.index.w = int32_t(index->width); a.index.h = int32_t(index->height); a.index.pitch = pitch_of(index);
    a.out.data = static_cast<uint8_t*>(out->data);
    a.out.w = int32_t(out->width); a.out.h = int32_t(out->height); a.out.pitch = pitch_of(out);
    a.bands = int32_t(src->bands); a.fmt = src->format; a.kernel = kernel; a.extend_copy = extend_copy != 0;
    a.index_fmt = index->format;
    // 2/4-band sources are alpha-premultiplied inside the sampler unless the
    // caller says they already are (MapImOp::has_alpha, mapim.rs:157-159)
    a.alpha = !premultiplied && (src->bands == 2 || src->bands == 4);
    a.background = background; a.src_w = src->width; a.src_h = src->height;
    return cuda_status(launch::mapim(a, static_cast<cudaStream_t>(stream)));
}

int32_t viprs_forward_affine_to_backward(const double f[4], double tx, double ty, double b[4], double* btx,
                                         double* bty) {
    if (!f || !b || !btx || !bty) return VIPRS_ERR_NULL_POINTER;
    return forward_affine_to_backward(f, tx, ty, b, btx, bty);
}

int32_t viprs_chain_plan_create(uint32_t w, uint32_t h, uint32_t bands, int32_t format, const viprs_node* nodes,
                                int32_t n_nodes, int32_t demand_override, viprs_plan** out) {
    Chain c;
    const int32_t st = nodes_to_chain(nodes, n_nodes, demand_override, &c);
    if (st) return st;
    return create_chain_plan_a(w, h, bands, format, c, out);
}

// The C-ABI form of planned nodes (kind 9 = the Zoom upscale); SIZE_MISMATCH
// when `capacity` nodes do not suffice.
static int32_t export_nodes(const std::vector<PlanNode>& planned, viprs_node* nodes, int32_t capacity) {
    if (int64_t(planned.size()) > capacity) return VIPRS_ERR_SIZE_MISMATCH;
    for (size_t i = 0; i < planned.size(); ++i) {
        const PlanNode& n = planned[i];
        viprs_node v;
        std::memset(&v, 0, sizeof(v));
        v.kind = int32_t(n.kind);
        v.factor_u = n.kind == NodeKind::Zoom ? n.zx : n.ufactor;
        v.vfactor_u = n.kind == NodeKind::Zoom ? n.zy : n.vufactor;
        v.ceil_mode = n.ceil ? 1 : 0;
        v.factor = n.factor; v.vfactor = n.vfactor; v.kernel = int32_t(n.kernel);
        std::memcpy(v.matrix, n.m, sizeof(v.matrix));
        v.tx = n.tx; v.ty = n.ty; v.out_width = n.out_w; v.out_height = n.out_h;
        v.extend = int32_t(n.extend); v.background = n.background; v.premultiplied = n.premultiplied ? 1 : 0;
        v.area_x = n.ex; v.area_y = n.ey; v.area_width = n.ew; v.area_height = n.eh;
        v.demand_hint = int32_t(n.demand);
        nodes[i] = v;
    }
    return VIPRS_OK;
}

int32_t viprs_thumbnail_plan_nodes(int32_t target, uint32_t tw, uint32_t th, int32_t kernel, int32_t crop,
                                   uint32_t w, uint32_t h, uint32_t bands, int32_t allow_shrink_hint,
                                   viprs_node* nodes, int32_t capacity, int32_t* n_nodes, uint32_t* out_w,
                                   uint32_t* out_h, uint32_t* shrink_factor) {
    if (!n_nodes || !out_w || !out_h || !shrink_factor || (capacity > 0 && !nodes)) return VIPRS_ERR_NULL_POINTER;
    if (target < 0 || target > 3 || capacity < 0) return VIPRS_ERR_INVALID_ARGUMENT;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    const ThumbnailPlan plan =
        thumbnail_plan(ThumbTarget(target), tw, th, Kernel(kernel), crop != 0, w, h, bands, allow_shrink_hint != 0);
    *n_nodes = int32_t(plan.nodes.size());
    *out_w = plan.output_width;
    *out_h = plan.output_height;
    *shrink_factor = plan.shrink_factor;
    return export_nodes(plan.nodes, nodes, capacity);
}

int32_t viprs_resize_plan_nodes(double hscale, double vscale, int32_t kernel, double gap, uint32_t w, uint32_t h,
                                viprs_node* nodes, int32_t capacity, int32_t* n_nodes, uint32_t* out_w,
                                uint32_t* out_h) {
    if (!n_nodes || !out_w || !out_h || (capacity > 0 && !nodes)) return VIPRS_ERR_NULL_POINTER;
    if (capacity < 0 || !(hscale > 0.0) || !(vscale > 0.0) || !std::isfinite(hscale) || !std::isfinite(vscale))
        return VIPRS_ERR_INVALID_ARGUMENT;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    const ResizePlan plan = resize_plan(hscale, vscale, Kernel(kernel), gap, w, h);
    *n_nodes = int32_t(plan.nodes.size());
    *out_w = plan.output_width;
    *out_h = plan.output_height;
    return export_nodes(plan.nodes, nodes, capacity);
}

int32_t viprs_chain_output_size(uint32_t w, uint32_t h, const viprs_node* nodes, int32_t n_nodes, uint32_t* out_w,
                                uint32_t* out_h) {
    if (!out_w || !out_h) return VIPRS_ERR_NULL_POINTER;
    Chain c;
    int32_t st = nodes_to_chain(nodes, n_nodes, -1, &c);
    if (st) return st;
    for (const PlanNode& n : c.nodes) {
        st = node_output_dims(n, w, h, &w, &h);
        if (st) return st;
    }
    *out_w = w;
    *out_h = h;
    return VIPRS_OK;
}

int32_t viprs_similarity_node(double scale, double angle, int32_t kernel, uint32_t w, uint32_t h, viprs_node* node) {
    if (!node) return VIPRS_ERR_NULL_POINTER;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    if (!std::isfinite(angle)) return VIPRS_ERR_INVALID_ARGUMENT;
    return export_nodes({similarity_node(scale, angle, Kernel(kernel), w, h)}, node, 1);
}

int32_t viprs_thumbnail_plan_create(uint32_t w, uint32_t h, uint32_t bands, int32_t format, int32_t target,
                                    uint32_t tw, uint32_t th, int32_t kernel, int32_t crop, viprs_plan** out) {
    if (target < 0 || target > 3) return VIPRS_ERR_INVALID_ARGUMENT;
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    Chain c;
    int st = builder_thumbnail_chain(w, h, bands, ThumbTarget(target), tw, th, Kernel(kernel), crop != 0, &c);
    if (st) return st;
    return create_chain_plan_a(w, h, bands, format, c, out);
}

int32_t viprs_resize_plan_create(uint32_t w, uint32_t h, uint32_t bands, int32_t format, double hscale,
                                 double vscale, int32_t kernel, viprs_plan** out) {
    if (kernel < 0 || kernel > 9) return VIPRS_ERR_INVALID_KERNEL;
    Chain c;
    int st = builder_resize_chain(w, h, bands, hscale, vscale, Kernel(kernel), &c);
    if (st) return st;
    return create_chain_plan_a(w, h, bands, format, c, out);
}

int32_t viprs_plan_status(viprs_plan* p, void* stream) {
    if (!p) return VIPRS_ERR_NULL_POINTER;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    int32_t h = 0;
    if (p->d_err) {
        e = cudaMemcpy(&h, p->d_err, sizeof(h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && h != 0) e = cudaMemset(p->d_err, 0, sizeof(h));
        if (e != cudaSuccess) return cuda_status(e);
    }
    return h;
}

int32_t viprs_plan_output_size(const viprs_plan* p, uint32_t* w, uint32_t* h) {
    if (!p || !w || !h) return VIPRS_ERR_NULL_POINTER;
    *w = p->out_w; *h = p->out_h;
    return VIPRS_OK;
}

int32_t viprs_plan_workspace_bytes(const viprs_plan* p, uint64_t* bytes) {
    if (!p || !bytes) return VIPRS_ERR_NULL_POINTER;
    *bytes = p->work_bytes + p->host_tables.size();
    return VIPRS_OK;
}

int32_t viprs_plan_launch_count(const viprs_plan* p, int32_t* launches) {
    if (!p || !launches) return VIPRS_ERR_NULL_POINTER;
    *launches = int32_t(p->stages.size());
    return VIPRS_OK;
}

int32_t viprs_plan_execute(viprs_plan* p, const void* src, void* dst, void* stream) {
    if (!p || !src || !dst) return VIPRS_ERR_NULL_POINTER;
    return execute_a(p, src, dst, static_cast<cudaStream_t>(stream));
}

int32_t viprs_plan_execute_stages(viprs_plan* p, int32_t first, int32_t count, const void* src, void* dst,
                                  void* stream) {
    if (!p || !src || !dst) return VIPRS_ERR_NULL_POINTER;
    if (first < 0 || count < 0) return VIPRS_ERR_INVALID_ARGUMENT;
    return execute_a(p, src, dst, static_cast<cudaStream_t>(stream), first, count);
}

int32_t viprs_plan_execute_host(viprs_plan* p, const void* hsrc, void* hdst, void* stream) {
    if (!p || !hsrc || !hdst) return VIPRS_ERR_NULL_POINTER;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = format_size(Format(p->fmt));
    const size_t in_bytes = size_t(p->in_w) * p->in_h * p->bands * es;
    const size_t out_bytes = size_t(p->out_w) * p->out_h * p->bands * es;
    cudaError_t e = cudaSuccess;
    if (!p->d_in) e = cudaMalloc(reinterpret_cast<void**>(&p->d_in), std::max<size_t>(in_bytes, 16));
    if (e == cudaSuccess && !p->d_out) e = cudaMalloc(reinterpret_cast<void**>(&p->d_out), std::max<size_t>(out_bytes, 16));
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaMemcpyAsync(p->d_in, hsrc, in_bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e);
    int st = execute_a(p, p->d_in, p->d_out, s);
    if (st) return st;
    e = cudaMemcpyAsync(hdst, p->d_out, out_bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e);
}

void viprs_plan_destroy(viprs_plan* p) { free_plan_a(p); }

}  // extern "C"
