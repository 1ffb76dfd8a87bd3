// launch.hpp -- host-visible argument blocks and launch wrappers of the
// resample kernels.  Plain structs only, so that host C++ (capi.cpp) and
// device code (resample.cu, affine.cu, batch.cu) share one definition.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace viprs {

struct PlaneArg {
    const uint8_t* data = nullptr;
    int64_t x0 = 0, y0 = 0;
    int32_t w = 0, h = 0;
    int64_t pitch = 0;
    int64_t total_bytes = 0;
};

struct OutPlaneArg {
    uint8_t* data = nullptr;
    int64_t x0 = 0, y0 = 0;
    int32_t w = 0, h = 0;
    int64_t pitch = 0;
};

// Sample formats (values of viprs_format).
enum : int32_t { kU8 = 0, kU16 = 1, kF32 = 2 };

// Box shrink of one or two axes (ShrinkH then ShrinkV when hv_order, ShrinkV
// then ShrinkH otherwise); factor 1 on an axis means that op is absent.
struct ShrinkArgs {
    PlaneArg in;
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kU8;
    uint32_t fh = 1, fv = 1;
    int32_t hv_order = 1;
    int32_t premul_in = 0;     // apply Premultiply<U8> to every source sample read
    int32_t unpremul_out = 0;  // apply Unpremultiply<U8> to every stored pixel
    int32_t nx = 0;            // output columns per block (set by the launcher)
    int32_t col_lo = 0;        // local output columns [col_lo, col_hi) handled
    int32_t col_hi = -1;       //   (-1: all)
    // rounding constants of ShrinkH / ShrinkV for u8 (host-computed)
    int32_t hmode = 0, vmode = 0;       // 0 copy, 1 factor 2, 2 exact /5, 3 multiplier
    uint64_t hmult = 0, vmult = 0;
    // the same roundings as one 32-bit multiply-add: round(s) = (s * mul + add) >> 24
    uint32_t hmul = 0, hadd = 0, vmul = 0, vadd = 0;
    // warp shrink (u8, ShrinkH then ShrinkV; shrink_warp.cuh): nxf output
    // pixels per warp, rows_per_item output rows per work item, stage buffers
    // of row_cap bytes, box walks rotated by (lane >> rot_shift) groups
    int32_t nxf = 0, rows_per_item = 1;
    uint32_t row_cap = 0;
    int32_t rot_shift = 5;
    int32_t* err = nullptr;    // device error word (timeout), may be null
};

// Reduce accumulation modes.
enum : int32_t {
    kReduceFixed = 0,    // u8/u16: i16 x sample, int32 accumulator, (acc+2048)>>12
    kReduceF32Simd = 1,  // f32: x86 AVX2 order of viprs (f64 products, lane sums)
    kReduceF64Fma = 2    // sequential f64 fma, FromF64 rounding (ReduceOp, scalar paths)
};

struct ReduceArgs {
    PlaneArg in;
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kU8;
    int32_t mode = kReduceFixed;
    int32_t taps = 1;
    const int32_t* starts = nullptr;  // absolute first tap per output column (H) or row (V)
    const uint8_t* phases = nullptr;  // phase row (0..64) per output column / row
    const void* coeffs = nullptr;     // 65 x taps, int16 (fixed) or double (float modes)
    int32_t vector_len = 0;           // V f32: samples below this index use mul+add
    int32_t premul_in = 0;
    int32_t unpremul_out = 0;
};

// ReduceH and ReduceV fused (either order): the first op's output tile stays
// in shared memory.  Tables follow ReduceArgs; the mid plane is the first op's
// output region.
struct Reduce2DArgs {
    PlaneArg in;
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kU8;
    int32_t hfirst = 1;
    int64_t mx0 = 0, my0 = 0;
    int32_t mw = 0, mh = 0;
    int32_t taps_h = 1, taps_v = 1;
    int32_t mode_h = kReduceFixed, mode_v = kReduceFixed;
    const int32_t* starts_h = nullptr;
    const uint8_t* phases_h = nullptr;
    const int32_t* starts_v = nullptr;
    const uint8_t* phases_v = nullptr;
    const void* coeffs_h = nullptr;
    const void* coeffs_v = nullptr;
    int32_t vector_len = 0;   // V f32 split, index within a V output row
    int32_t premul_in = 0;
    int32_t unpremul_out = 0;
    int32_t tile_w = 64, tile_h = 16;
    int32_t span_max = 0;     // largest mid rows (hfirst) or columns (vfirst) one tile reads
    int32_t in_rows_max = 0;  // largest source rows one tile stages in shared memory
    int32_t in_cols_max = 0;  // largest source columns one tile stages
    // f32: the row-strip kernel (reduce_strip.cuh) instead of tiles: tile_w
    // output columns per strip, tile_h output rows per block, in_cols_max the
    // widest source / mid column span of a strip, span_max the rows of its
    // ring, in_rows_max the source rows in flight per block
    int32_t strip = 0;
    int32_t* err = nullptr;   // device error word (a bounded wait that gave up), may be null
};

#if defined(__CUDACC__)
#define VIPRS_HD __host__ __device__
#else
#define VIPRS_HD
#endif

// Shrink ring slot (u8 box shrink) for a source row segment of n bytes: the
// segment sits at its plane offset mod 16 within the slot (the 16-byte aligned
// cover is copied), with 32 bytes of slack after it for the box sums'
// over-read.


// Shared-memory layout of one fused-reduce tile (byte offsets, 16-aligned):
// both coefficient tables, the tile's start/phase tables, one offset per
// staged source row, the staged source rows, the mid tile and the output tile.
struct Reduce2DLayout {
    int32_t coef_h = 0, coef_v = 0, tab = 0, rowbase = 0, in = 0, mid = 0, out = 0, total = 0;
    int32_t coef_h_bytes = 0, coef_v_bytes = 0;
    int32_t pitch = 0;  // bytes per staged source row
};

VIPRS_HD inline int32_t r2_align16(int64_t v) { return int32_t((v + 15) / 16 * 16); }

VIPRS_HD inline Reduce2DLayout reduce2d_layout(const Reduce2DArgs& a) {
    Reduce2DLayout L;
    const int es = a.fmt == kU8 ? 1 : (a.fmt == kU16 ? 2 : 4);
    L.coef_h_bytes = 65 * a.taps_h * (a.mode_h == kReduceFixed ? 2 : 8);
    L.coef_v_bytes = 65 * a.taps_v * (a.mode_v == kReduceFixed ? 2 : 8);
    L.coef_h = 0;
    L.coef_v = r2_align16(L.coef_h_bytes);
    L.tab = L.coef_v + r2_align16(L.coef_v_bytes);
    const int64_t tab_bytes = int64_t(a.tile_w + a.tile_h) * 4 + a.tile_w + a.tile_h;
    L.rowbase = L.tab + r2_align16(tab_bytes);
    L.in = L.rowbase + r2_align16(int64_t(a.in_rows_max) * 4);
    L.pitch = r2_align16(int64_t(a.in_cols_max) * a.bands * es + 16);
    L.mid = L.in + r2_align16(int64_t(a.in_rows_max) * L.pitch);
    const int64_t mid_bytes = int64_t(a.span_max) * (a.hfirst ? a.tile_w : a.tile_h) * a.bands * es;
    L.out = L.mid + r2_align16(mid_bytes);
    L.total = L.out + r2_align16(int64_t(a.tile_w) * a.tile_h * a.bands * es);
    return L;
}

struct PixelArgs {
    PlaneArg in;
    OutPlaneArg out;
    int32_t bands = 1;
    int32_t fmt = kU8;
    int32_t op = 0;  // 0 copy, 1 premultiply, 2 unpremultiply, 3 zoom
    // zoom: output (x, y) takes source (x / zx, y / zy), both in image
    // coordinates (the planes' origins x0 / y0 map them to local ones)
    int32_t zx = 1, zy = 1;
};

namespace launch {
cudaError_t shrink2d(ShrinkArgs a, cudaStream_t s);
cudaError_t reduce_h(const ReduceArgs& a, cudaStream_t s);
cudaError_t reduce_v(const ReduceArgs& a, cudaStream_t s);
cudaError_t reduce2d(const Reduce2DArgs& a, cudaStream_t s);
// Shared memory a reduce2d launch needs for its tile shape; 0 if too large.
size_t reduce2d_smem_bytes(const Reduce2DArgs& a);
// Choose the tile shape of a fused reduce and fill span_max / in_rows_max /
// in_cols_max.  `sh`/`sv`: host copies of the H and V start tables (absolute
// first tap per output column / row); `in_*`: the source plane's rectangle.
// Picks the largest tile that fits `smem_budget` bytes and still gives at
// least `min_tiles` tiles (when any shape does).  False if nothing fits.
bool reduce2d_configure(Reduce2DArgs* a, const int32_t* sh, const int32_t* sv, int64_t in_x0, int64_t in_y0,
                        int64_t in_w, int64_t in_h, int64_t min_tiles, size_t smem_budget);
cudaError_t pixel(const PixelArgs& a, cudaStream_t s);
// Dynamic shared memory a shrink2d launch needs; 0 if the factor is too large.
size_t shrink2d_smem_bytes(const ShrinkArgs& a, int32_t* nx);
// Set the u8 rounding constants of `a` and return its interior output columns
// [lo, hi) (source boxes inside the plane, aligned spans inside the buffer).
void shrink_prepare(ShrinkArgs* a, int32_t* lo, int32_t* hi);
}  // namespace launch

}  // namespace viprs
