// sphb_force.cu -- the force entry point: MomentumEquation /
// SPHPressureGradient + GravityForce, with the continuity scheme's
// SPHDensityRate and XSPHCorrection terms (the pass is in
// sphb_force_pass.cuh).

#include "sphb_launch.cuh"

namespace sphb {

int check_engine_public(const sphb_engine *e, int cur);
int check_pair_cfg(const sphb_engine *e);
int check_stage_sums(const sphb_engine *e, int cur, int kind);

}  // namespace sphb

using namespace sphb;

extern "C" int sphb_momentum(const sphb_engine *e, int cur, uint32_t dest_mask,
                             int with_gravity, int mode, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if ((rc = check_pair_cfg(e))) return rc;
    const int fmode = mode & ~(SPHB_FORCE_USE_LIST | SPHB_FORCE_NO_MAXIMA | SPHB_FORCE_STAGE_MASK);
    if (fmode != 0 && fmode != 1 && fmode != 2) return SPHB_ERR_ARG;
    const int kind = ((mode & SPHB_FORCE_STAGE_MASK) >> 8) - 1;
    if (kind > 7) return SPHB_ERR_ARG;
    if ((rc = check_stage_sums(e, cur, kind))) return rc;
    if (kind >= 0) {
        // the fused stage: FP32C, both record copies, the stage buffers,
        // and every stepped / density-rate array a dest of this pass
        const sphb_config &c = e->cfg;
        if (c.precision != SPHB_FP32C || !e->f.geo_next || !e->f.vel_next) return SPHB_ERR_ARG;
        const sphb_buffers &B = e->buf[cur];
        if (!B.x0 || !B.y0 || !B.u0 || !B.v0 || (c.dim == 3 && (!B.z0 || !B.w0)))
            return SPHB_ERR_ARG;
        for (int a = 0; a < c.num_arrays; ++a) {
            const bool pair_dest = ((dest_mask >> a) & 1u) &&
                                   (c.mom_src[a] | c.rate_src[a] | c.xsph_src[a]) != 0u;
            if ((((c.step_on >> a) & 1u) || c.rate_src[a]) && !pair_dest) return SPHB_ERR_ARG;
            if (c.rate_src[a] && (!B.rho || !B.rho0)) return SPHB_ERR_ARG;
        }
    }
    if (!e->f.au || !e->f.av || (e->cfg.dim == 3 && !e->f.aw)) return SPHB_ERR_ARG;
    if ((fmode == 0 || fmode == 2) && !e->f.dt_fac) return SPHB_ERR_ARG;
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
