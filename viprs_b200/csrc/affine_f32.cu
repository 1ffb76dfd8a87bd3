// affine_f32.cu -- the affine and mapim kernels for float samples (see affine.cu
// for the viprs files they follow).
#include "affine_fmt.cuh"

namespace viprs {
namespace launch {

void affine_f32(const AffineArgs& k, dim3 grid, cudaStream_t s) { affine_bands<float>(k, grid, s); }

cudaError_t mapim_f32(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s) { return mapim_taps<float>(a, grid, nt, s); }

}  // namespace launch
}  // namespace viprs
