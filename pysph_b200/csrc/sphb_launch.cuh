// sphb_launch.cuh -- the pair-pass launchers, one instantiation per
// (smoothing kernel, dimension) in the sphb_pass_*.cu translation units, so
// the kernel variants compile in parallel.

#pragma once

#include "sphb_common.cuh"

namespace sphb {

// SPHRho (+ Tait epilogue, list recording): flags as sphb_density
template <int KT, int DIM>
void launch_density_kt(const sphb_engine &e, int cur, uint32_t dm, int flags, cudaStream_t st);

// MomentumEquation / SPHPressureGradient (+ gravity, continuity terms)
template <int KT, int DIM>
void launch_force_kt(const sphb_engine &e, int cur, uint32_t dm, int grav, int mode,
                     cudaStream_t st);

// the same passes with shared-memory staging (pair_mode SPHB_PAIRS_TILED,
// 2D FP32C; sphb_tiled.cuh)
template <int KT>
void launch_density_tiled(const sphb_engine &e, int cur, uint32_t dm, int flags, cudaStream_t st);
template <int KT>
void launch_force_tiled(const sphb_engine &e, int cur, uint32_t dm, int grav, int mode,
                        cudaStream_t st);

// kernel * 10 + dim of the built pair passes (the cubic in 2D and 3D, the
// quintic and Wendland kernels in 2D, as the reference has them); 0 if the
// configuration has no pass
inline int pass_variant(const sphb_config &c)
{
    const int v = (c.kernel == 0 ? (int)SPHB_KERNEL_CUBIC : c.kernel) * 10 + c.dim;
    return (v == 12 || v == 13 || v == 32 || v == 42) ? v : 0;
}

}  // namespace sphb
