// common.cuh -- device-side helpers shared by the resample kernels.
//
// Every device translation unit of this library is compiled with
// --fmad=false: a product and a sum are fused only where fma() is written,
// which is where viprs calls `mul_add`.  Together with the host tables of
// plan.cpp this reproduces viprs's f64 arithmetic bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "launch.hpp"

namespace viprs {
namespace dev {

// A plane (PlaneArg): a rectangle (x0, y0, w, h) of the virtual image plane
// of one pipeline stage, stored row-major with `pitch` bytes per row.  Reads
// are clamped to the rectangle.  For the source image this is viprs's
// MemorySource edge replication (sources/memory.rs:186-215); for an
// intermediate it is the reduce ops' clamp_axis (reduce_common.rs:318-322),
// whose rectangle is exactly the region the downstream op requested.
using Plane = PlaneArg;

template <typename T>
__device__ __forceinline__ T load_sample(const Plane& p, int64_t lx, int64_t ly, int bands, int b) {
    lx = lx < 0 ? 0 : (lx >= p.w ? p.w - 1 : lx);
    ly = ly < 0 ? 0 : (ly >= p.h ? p.h - 1 : ly);
    const T* row = reinterpret_cast<const T*>(p.data + ly * p.pitch);
    return row[lx * bands + b];
}

// Zeroed stand-in address for a tap of an empty plane.  The interpolators
// load every tap of a pixel unconditionally, so that all of its loads are in
// flight together, and select the fill value for taps outside the image
// afterwards; a tap therefore always needs a readable address.
__device__ __align__(16) static const unsigned char kNoSample[64] = {0};

// Address of sample (lx, ly), band 0, of plane p with load_sample's clamp to
// the plane; kNoSample for an empty plane.
template <typename T>
__device__ __forceinline__ const T* sample_ptr(const Plane& p, int64_t lx, int64_t ly, int bands) {
    if (p.w <= 0 || p.h <= 0) return reinterpret_cast<const T*>(kNoSample);
    lx = lx < 0 ? 0 : (lx >= p.w ? p.w - 1 : lx);
    ly = ly < 0 ? 0 : (ly >= p.h ? p.h - 1 : ly);
    return reinterpret_cast<const T*>(p.data + ly * p.pitch) + lx * bands;
}

__device__ __forceinline__ int64_t clampi64(int64_t v, int64_t lo, int64_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// FromF64 (viprs-core/src/shared_ops/sample_conv.rs): clamp, then round half
// away from zero; f32 is a plain round-to-nearest cast.
template <typename T> __device__ __forceinline__ T from_f64(double v);
template <> __device__ __forceinline__ uint8_t from_f64<uint8_t>(double v) {
    v = v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v);
    return static_cast<uint8_t>(static_cast<uint32_t>(round(v)));
}
template <> __device__ __forceinline__ uint16_t from_f64<uint16_t>(double v) {
    v = v < 0.0 ? 0.0 : (v > 65535.0 ? 65535.0 : v);
    return static_cast<uint16_t>(static_cast<uint32_t>(round(v)));
}
template <> __device__ __forceinline__ float from_f64<float>(double v) { return __double2float_rn(v); }

// ShrinkSample::from_f64_clamped (resample/shrinkh.rs:44-128): round, then clamp.
template <typename T> __device__ __forceinline__ T shrink_from_f64(double v);
template <> __device__ __forceinline__ uint8_t shrink_from_f64<uint8_t>(double v) {
    double r = round(v);
    r = r < 0.0 ? 0.0 : (r > 255.0 ? 255.0 : r);
    return static_cast<uint8_t>(static_cast<uint32_t>(r));
}
template <> __device__ __forceinline__ uint16_t shrink_from_f64<uint16_t>(double v) {
    double r = round(v);
    r = r < 0.0 ? 0.0 : (r > 65535.0 ? 65535.0 : r);
    return static_cast<uint16_t>(static_cast<uint32_t>(r));
}
template <> __device__ __forceinline__ float shrink_from_f64<float>(double v) { return __double2float_rn(v); }

// Fixed-point reduce output (resample/sample_conv.rs:24-33): (acc + 2048) >> 12, clamped.
template <typename T> __device__ __forceinline__ T from_fixed(int32_t acc);
template <> __device__ __forceinline__ uint8_t from_fixed<uint8_t>(int32_t acc) {
    int32_t v = (acc + 2048) >> 12;
    return static_cast<uint8_t>(v < 0 ? 0 : (v > 255 ? 255 : v));
}
template <> __device__ __forceinline__ uint16_t from_fixed<uint16_t>(int32_t acc) {
    int32_t v = (acc + 2048) >> 12;
    return static_cast<uint16_t>(v < 0 ? 0 : (v > 65535 ? 65535 : v));
}
// f32 never takes the fixed-point path; defined so that dead template branches compile.
template <> __device__ __forceinline__ float from_fixed<float>(int32_t acc) { return float(acc); }

// Premultiply<U8> (structural/premultiply.rs:84-121) computes
// round(c * fl(a / 255)) in f64.  c*a/255 is never within 1/510 of a
// half-integer (2ca is even, 255(2k+1) is odd) while the f64 error is below
// 1e-13, so the result equals the exact rational rounding below.
__device__ __forceinline__ uint32_t premultiply_u8(uint32_t c, uint32_t a) {
    // == (2ca + 255) / 510 for all c, a in 0..255 (checked exhaustively in the tests)
    const uint32_t t = c * a + 128u;
    return (t + (t >> 8)) >> 8;
}
// Unpremultiply<U8> (structural/unpremultiply.rs:76-113): round(c*255 / a),
// clamped; a == 0 gives 0.  255c/a is either an exact half-integer (kept
// exactly by f64, rounded up) or at least 1/(2a) away from one, far beyond
// the f64 error, so integer rounding reproduces it.
__device__ __forceinline__ uint32_t unpremultiply_u8(uint32_t c, uint32_t a) {
    if (a == 0) return 0;
    uint32_t v = (510u * c + a) / (2u * a);
    return v > 255u ? 255u : v;
}

}  // namespace dev
}  // namespace viprs
