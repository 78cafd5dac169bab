// sphb_force.cu -- the force entry point: MomentumEquation /
// SPHPressureGradient + GravityForce, with the continuity scheme's
// SPHDensityRate and XSPHCorrection terms (the pass is in
// sphb_force_pass.cuh).

#include "sphb_launch.cuh"

namespace sphb {

int check_engine_public(const sphb_engine *e, int cur);
int check_pair_cfg(const sphb_engine *e);

}  // namespace sphb

using namespace sphb;

extern "C" int sphb_momentum(const sphb_engine *e, int cur, uint32_t dest_mask,
                             int with_gravity, int mode, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if ((rc = check_pair_cfg(e))) return rc;
    if ((mode & ~SPHB_FORCE_USE_LIST) != 0 && (mode & ~SPHB_FORCE_USE_LIST) != 1)
        return SPHB_ERR_ARG;
    if (!e->f.au || !e->f.av || (e->cfg.dim == 3 && !e->f.aw)) return SPHB_ERR_ARG;
    if ((mode & 15) == 0 && !e->f.dt_fac) return SPHB_ERR_ARG;
    for (int a = 0; a < SPHB_MAX_ARRAYS; ++a) {
        if (e->cfg.rate_src[a] && !e->f.drho) return SPHB_ERR_ARG;
        if (e->cfg.xsph_src[a] && (!e->f.xu || !e->f.xv || (e->cfg.dim == 3 && !e->f.xw)))
            return SPHB_ERR_ARG;
    }
    if (e->num_pair_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const sphb_config &c = e->cfg;
    if (c.precision == SPHB_FP32C) {
        if (!e->f.geo || !e->f.thermo || !e->f.vel || (c.dim == 3 && !e->f.mass))
            return SPHB_ERR_ARG;
    } else {
        if (!e->f.rho || !e->f.p || !e->f.cs) return SPHB_ERR_ARG;
    }
    const int g = with_gravity;
    switch (pass_variant(c)) {
    case 12: launch_force_kt<SPHB_KERNEL_CUBIC, 2>(*e, cur, dest_mask, g, mode, st); break;
    case 13: launch_force_kt<SPHB_KERNEL_CUBIC, 3>(*e, cur, dest_mask, g, mode, st); break;
    case 32: launch_force_kt<SPHB_KERNEL_QUINTIC, 2>(*e, cur, dest_mask, g, mode, st); break;
    case 42: launch_force_kt<SPHB_KERNEL_WENDLAND, 2>(*e, cur, dest_mask, g, mode, st); break;
    default: return SPHB_ERR_UNSUPPORTED;
    }
    return launch_status("sphb_momentum");
}
