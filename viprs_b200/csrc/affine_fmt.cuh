// affine_fmt.cuh -- the launch templates the per-format translation units
// instantiate (see affine_fmt.hpp).
#pragma once

#include "affine_dev.cuh"
#include "affine_fmt.hpp"

namespace viprs {
namespace launch {

template <typename T>
inline void affine_bands(const AffineArgs& k, dim3 grid, cudaStream_t s) {
    switch (k.bands) {
    case 1: dev::affine_kernel<T, 1><<<grid, 256, 0, s>>>(k); break;
    case 3: dev::affine_kernel<T, 3><<<grid, 256, 0, s>>>(k); break;
    case 4: dev::affine_kernel<T, 4><<<grid, 256, 0, s>>>(k); break;
    default: dev::affine_kernel<T, 0><<<grid, 256, 0, s>>>(k); break;
    }
}

template <typename T>
inline cudaError_t mapim_taps(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s) {
    if (a.alpha) {
        dev::mapim_alpha_kernel<T><<<grid, 256, 0, s>>>(a);
        return cudaGetLastError();
    }
    switch (nt) {
    case 0: dev::mapim_kernel<T, 0><<<grid, 256, 0, s>>>(a); break;
    case 4: dev::mapim_kernel<T, 4><<<grid, 256, 0, s>>>(a); break;
    case 6: dev::mapim_kernel<T, 6><<<grid, 256, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace launch
}  // namespace viprs
