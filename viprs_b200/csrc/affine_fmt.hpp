// affine_fmt.hpp -- per-sample-format launchers of the affine and mapim
// kernels.  Each format's kernels live in their own translation unit
// (affine_u8.cu, affine_u16.cu, affine_f32.cu) so that they compile in
// parallel; affine.cu dispatches to them.
#pragma once

#include <cuda_runtime.h>

#include "affine_launch.hpp"

namespace viprs {
namespace launch {

// affine_kernel<T, NB> with the band count as a template parameter for 1, 3
// and 4 bands (0: run-time band count).
void affine_u8(const AffineArgs& k, dim3 grid, cudaStream_t s);
void affine_u16(const AffineArgs& k, dim3 grid, cudaStream_t s);
void affine_f32(const AffineArgs& k, dim3 grid, cudaStream_t s);
// mapim_kernel<T, nt> (nt taps per axis: 0 nearest/bilinear, 4, 6), or the
// alpha-premultiplying sampler when a.alpha.
cudaError_t mapim_u8(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s);
cudaError_t mapim_u16(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s);
cudaError_t mapim_f32(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s);

}  // namespace launch
}  // namespace viprs
