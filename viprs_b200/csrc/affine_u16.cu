// affine_u16.cu -- the affine and mapim kernels for uint16_t samples (see affine.cu
// for the viprs files they follow).
#include "affine_fmt.cuh"

namespace viprs {
namespace launch {

void affine_u16(const AffineArgs& k, dim3 grid, cudaStream_t s) { affine_bands<uint16_t>(k, grid, s); }

cudaError_t mapim_u16(const MapimArgs& a, dim3 grid, int nt, cudaStream_t s) { return mapim_taps<uint16_t>(a, grid, nt, s); }

}  // namespace launch
}  // namespace viprs
