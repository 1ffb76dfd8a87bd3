// affine.cu -- sm_100a kernels for viprs's affine and mapim interpolators.
//
// One thread per output pixel (all bands); the kernels of each sample format
// are instantiated in affine_u8.cu, affine_u16.cu and affine_f32.cu.  All
// coordinate and weight arithmetic is f64 in viprs's operation order (these
// TUs are compiled with --fmad=false; fma() appears exactly where viprs calls
// mul_add), so u8 and
// f32 outputs reproduce viprs bit for bit.  The Lanczos2/3 weights take their
// sines from sin_rn.cuh (rounded to nearest); glibc's sin, which viprs calls,
// differs from it by one ulp on about 0.13% of the arguments (glibc's own
// rounding error, up to about 0.51 ulp), which moves a weight by one ulp and
// an u8 output only when its weighted sum lies within about 1e-16 of a
// rounding boundary.
//
//   Affine::process_region ........ affine/core.rs:1593-1632 (incremental walk
//                                   from each scheduler tile's origin)
//   fast paths .................... affine/core.rs:1057-1513
//   sample_pixel_at / _with_alpha . affine/core.rs:1001-1054, 988-1019
//   sample_at / separable ......... affine/core.rs:640-760
//   extend modes .................. affine/interpolation.rs:43-137
//   MapImOp::process_typed ........ mapim.rs:1135-1274 (bilinear 1043-1096,
//                                   nearest 1099-1132, extend 306-384,
//                                   alpha sampler 616-1040)
#include <algorithm>

#include "affine_fmt.hpp"

namespace viprs {
namespace launch {

int affine_group(int64_t npx) {
    // enough threads for a few waves of 2048 per SM on 148 SMs, then up to
    // 8 pixels per thread (the walk and the tile region are shared along them)
    const int64_t per = npx / (148ll * 2048 * 2);
    return (int)std::max<int64_t>(1, std::min<int64_t>(8, per));
}

cudaError_t affine(const AffineArgs& a, cudaStream_t s) {
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    if (npx <= 0) return cudaSuccess;
    if (a.bands > 8) return cudaErrorInvalidValue;
    AffineArgs k = a;
    k.group = affine_group(npx);
    const int64_t gx = ((int64_t)a.out.w + k.group - 1) / k.group;
    const dim3 grid((unsigned)((gx + 255) / 256), (unsigned)std::min<int64_t>(a.out.h, 65535));
    switch (a.fmt) {
    case kU8: affine_u8(k, grid, s); break;
    case kU16: affine_u16(k, grid, s); break;
    default: affine_f32(k, grid, s); break;
    }
    return cudaGetLastError();
}

cudaError_t mapim(const MapimArgs& a, cudaStream_t s) {
    const int64_t npx = (int64_t)a.out.w * a.out.h;
    if (npx <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((a.out.w + 255) / 256), (unsigned)std::min<int64_t>(a.out.h, 65535));
    // the kernels index a source row with 32-bit element offsets
    if ((int64_t)a.src_w * a.bands >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
    const int nt = (a.kernel == 0 || a.kernel == 1) ? 0 : (a.kernel == 9 ? 6 : 4);
    switch (a.fmt) {
    case kU8: return mapim_u8(a, grid, nt, s);
    case kU16: return mapim_u16(a, grid, nt, s);
    case kF32: return mapim_f32(a, grid, nt, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace launch
}  // namespace viprs
