// sphb_pass_cubic2d.cu -- the density and force passes with the cubic spline
// kernel in 2D.

#include "sphb_density_pass.cuh"
#include "sphb_force_pass.cuh"
#include "sphb_tiled.cuh"

namespace sphb {

template void launch_density_kt<SPHB_KERNEL_CUBIC, 2>(const sphb_engine &, int, uint32_t, int,
                                           cudaStream_t);
template void launch_force_kt<SPHB_KERNEL_CUBIC, 2>(const sphb_engine &, int, uint32_t, int, int,
                                         cudaStream_t);

}  // namespace sphb
