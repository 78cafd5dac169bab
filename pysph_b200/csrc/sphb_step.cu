// sphb_step.cu -- predictor-corrector stages, the per-step prologue (count,
// CFL time step), user <-> engine order exchange, and the host helpers of
// the C ABI (sm_100a).
//
// PredictorCorrectorIntegrator (S/solver/integrator.py:614-683):
//   predict   X0 = X;  X = X0 + dt/2 F(X)                      (step, :340-367)
//   correct   X = X0 + dt/2 F(X_half);  final  X = 2 X - X0    (:632-644)
// F is the acceleration for u, v, w and, through PositionStepping
// (S/sph/funcs/position_funcs.pyx:10-56), the velocity for x, y, z.  The
// state stays FP64; products and sums round separately (numpy's
// `initial + step * dt`, no FMA), so FP64 runs track the reference closely.

#include <stdio.h>
#include <string.h>

#include "sphb_common.cuh"

namespace sphb {

int check_engine_public(const sphb_engine *e, int cur);

static thread_local char g_last_error[256] = "";

void record_cuda_error(const char *what, cudaError_t err)
{
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(err));
}

int launch_status(const char *what)
{
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what,
                 cudaGetErrorString(err));
        return SPHB_ERR_CUDA;
    }
    return SPHB_OK;
}

__device__ __forceinline__ double axpy_rn(double x0, double a, double dt)
{
    return __dadd_rn(x0, __dmul_rn(a, dt));
}

template <int DIM, bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_pc_stage(const __grid_constant__ sphb_engine e, int cur, int stage)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the particles move: the lists are not known to be complete until
        // the next rebin decision, and the positions leave the anchors
        e.work.meta[2] = 0;
        e.work.meta[3] = 0;
    }
    if (stage == 0 && blockIdx.x == 0) {
        // the CFL rule reads the maxima of the corrector's force pass only
        // (dt_fac is reset per calc, S/sph/sph_calc.pyx:324): clear what the
        // predictor's pass accumulated
        for (int q = threadIdx.x; q < e.cfg.num_scenes; q += blockDim.x) {
            e.sstate[q].max_dtfac = 0ull;
            e.sstate[q].max_acc2 = 0ull;
        }
    }
    const int k = t.begin + threadIdx.x;
    const bool active = k < t.end;
    const sphb_buffers &B = e.buf[cur];
    const sphb_scene_state &st = e.sstate[s];
    const double dt2 = st.dt / 2;
    // the stage: 0 save X0, X = X0 + dt/2 F; 1 X = 2 (X0 + dt/2 F) - X0;
    // 2 save X0, X = X0 + dt F; 3 X = X0 + dt F
    const bool save = stage == 0 || stage == 2;
    const double hstep = stage == 0 ? dt2 : st.dt;
    auto advance = [&](double cur0, double init, double rate) {
        if (stage == 1) return __dadd_rn(2 * axpy_rn(init, rate, dt2), -init);
        return axpy_rn(save ? cur0 : init, rate, hstep);
    };
    // continuity scheme: the density of every SPHDensityRate dest is
    // integrated like the other stepped properties
    if (active && B.rho && B.rho0 && e.f.drho && e.cfg.rate_src[a]) {
        const double dr = F32 ? (double)((const float *)e.f.drho)[k] : ((const double *)e.f.drho)[k];
        const double r = B.rho[k];
        const double r0 = save ? r : B.rho0[k];
        if (save) B.rho0[k] = r;
        B.rho[k] = advance(r, r0, dr);
    }
    if (!((e.cfg.step_on >> a) & 1u)) return;  // block-uniform
    // XSPHCorrection adds to PositionStepping's rate
    const bool xsph = e.cfg.xsph_src[a] && e.f.xu && e.f.xv && (DIM == 2 || e.f.xw);
    const bool rec = F32 && e.f.geo && e.f.vel;   // FP32 pair records
    const bool disp = e.f.anchor != nullptr;      // displacement check
    float d2 = 0.f;
    if (active) {
        // every load first, so a thread's loads are in flight together
        double *X[3] = {B.x, B.y, B.z};
        double *V[3] = {B.u, B.v, B.w};
        double *X0[3] = {B.x0, B.y0, B.z0};
        double *V0[3] = {B.u0, B.v0, B.w0};
        const bool real = B.tag[k] == 0;
        double f[3] = {0.0, 0.0, 0.0}, x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0};
        double x0[3] = {0.0, 0.0, 0.0}, v0[3] = {0.0, 0.0, 0.0}, xv[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const void *fa = d == 0 ? e.f.au : (d == 1 ? e.f.av : e.f.aw);
            f[d] = F32 ? (double)((const float *)fa)[k] : ((const double *)fa)[k];
            if (xsph) {
                const void *xa = d == 0 ? e.f.xu : (d == 1 ? e.f.xv : e.f.xw);
                xv[d] = F32 ? (double)((const float *)xa)[k] : ((const double *)xa)[k];
            }
            x[d] = X[d][k];
            v[d] = V[d][k];
            if (!save) {
                x0[d] = X0[d][k];
                v0[d] = V0[d][k];
            }
        }
        int local = (rec || disp) ? e.f.cell[k] : 0;
        float an[3] = {0.f, 0.f, 0.f};
        if (disp) {
            if (DIM == 2) {
                const float2 q = ((const float2 *)e.f.anchor)[k];
                an[0] = q.x;
                an[1] = q.y;
            } else {
                const float4 q = ((const float4 *)e.f.anchor)[k];
                an[0] = q.x;
                an[1] = q.y;
                an[2] = q.z;
            }
        }
        const float hk = (rec && DIM == 3) ? (float)B.h[k] : 0.f;
        // the stage
        double p[3] = {0.0, 0.0, 0.0}, vn[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double fd = real ? f[d] : 0.0;
            // PositionStepping: F_x = u (+ the XSPH velocity)
            const double fx = real ? (xsph ? __dadd_rn(v[d], xv[d]) : v[d]) : 0.0;
            if (save) {
                X0[d][k] = x[d];
                V0[d][k] = v[d];
            }
            p[d] = advance(x[d], x0[d], fx);
            vn[d] = advance(v[d], v0[d], fd);
            X[d][k] = p[d];
            V[d][k] = vn[d];
        }
        // FP32 pair records of the new state, relative to the particle's
        // cell of the last bin, and how far it has moved from where that bin
        // put it
        if (rec || disp) {
            if (local < 0 || local >= st.ncells) {
                flag(e, SPHB_ST_BAD_INDEX);
                local = 0;
            }
            const double cs = e.scene[s].cell_size;
            int c[3];
            cell_coords(local, st.n, c[0], c[1], c[2]);
            float xr[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int d = 0; d < DIM; ++d) xr[d] = (float)(p[d] - (double)(st.lo[d] + c[d]) * cs);
            if (rec) {
                if (DIM == 2) {
                    ((float2 *)e.f.geo)[2 * k] = make_float2(xr[0], xr[1]);
                    ((float2 *)e.f.vel)[k] = make_float2((float)vn[0], (float)vn[1]);
                } else {
                    ((float4 *)e.f.geo)[k] = make_float4(xr[0], xr[1], xr[2], hk);
                    ((float4 *)e.f.vel)[k] =
                        make_float4((float)vn[0], (float)vn[1], (float)vn[2], 0.f);
                }
            }
            if (disp) {
                const float q0 = xr[0] - an[0], q1 = xr[1] - an[1], q2 = xr[2] - an[2];
                d2 = q0 * q0 + q1 * q1 + q2 * q2;
                // a non-finite position can never be within the skin
                if (!(d2 <= 3.0e38f)) d2 = 3.0e38f;
            }
        }
    }
    if (disp) {
        // non-negative floats order like their bits: one warp reduction
        const float wd = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(d2)));
        if ((threadIdx.x & 31) == 0 && wd > 0.f)
            atomic_max_nonneg(&e.sstate[s].max_disp2, (double)wd);
    }
}

// Solver.solve per-step prologue for every scene.
__global__ void k_step_begin(const __grid_constant__ sphb_engine e)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.cfg.num_scenes) return;
    const sphb_scene &sc = e.scene[s];
    sphb_scene_state &st = e.sstate[s];
    st.count += 1;
    if (sc.use_cfl) {
        const double dtfac = __longlong_as_double((long long)st.max_dtfac);
        const double acc2 = __longlong_as_double((long long)st.max_acc2);
        double dt = 1.0;
        // ViscousTimeStep: min(cfl * h / (co + max dt_fac))
        const double dv = __ddiv_rn(__dmul_rn(sc.cfl, sc.h_min), __dadd_rn(sc.c0, dtfac));
        dt = dv < dt ? dv : dt;
        // force criterion (use_cfl == 1): cfl * min(sqrt(h / fmax)), with
        // fmax = solver.dt at count 1; use_cfl == 2 is ViscousTimeStep alone
        if (sc.use_cfl == 1) {
            const double fmax = st.count == 1 ? sc.dt_initial : sqrt(acc2);
            const double df = __dmul_rn(sc.cfl, sqrt(__ddiv_rn(sc.h_min, fmax)));
            dt = dt < df ? dt : df;
        }
        st.dt = dt;
    }
    st.t += st.dt;
    // the maxima served this step's rule: the step's own force passes
    // accumulate them afresh (a single-stage integrator has no stage that
    // clears them)
    st.max_dtfac = 0ull;
    st.max_acc2 = 0ull;
}

__global__ void k_set_dt(const __grid_constant__ sphb_engine e, double dt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.cfg.num_scenes || e.scene[s].use_cfl) return;
    e.sstate[s].dt = dt;
}

__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_init_index(const __grid_constant__ sphb_engine e, int cur)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    e.buf[cur].idx[k] = k - e.seg_offset[t.seg];
}

template <bool F32>
__device__ __forceinline__ double *field_ptr(const sphb_engine &e, int cur, int field)
{
    const sphb_buffers &B = e.buf[cur];
    switch (field) {
    case 0: return B.x;
    case 1: return B.y;
    case 2: return B.z;
    case 3: return B.u;
    case 4: return B.v;
    case 5: return B.w;
    case 6: return B.x0;
    case 7: return B.y0;
    case 8: return B.z0;
    case 9: return B.u0;
    case 10: return B.v0;
    case 11: return B.w0;
    case 12: return B.m;
    case 13: return B.h;
    case 21: return B.rho;
    case 22: return B.rho0;
    }
    return nullptr;
}

template <bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_exchange(const __grid_constant__ sphb_engine e, int cur, int array, int field,
           int dir, double *user, const int *user_offset)
{
    // new positions, velocities, masses or smoothing lengths: the lists and
    // the FP32 records must be rebuilt before they are reused
    if (dir == 0 && (field <= 5 || field == 12 || field == 13) && blockIdx.x == 0 &&
        threadIdx.x == 0) {
        e.work.meta[2] = 0;
        e.work.meta[3] = 0;
        e.work.meta[4] = 0;
    }
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (a != array) return;
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const int n_seg = e.seg_offset[t.seg + 1] - e.seg_offset[t.seg];
    const int li = e.buf[cur].idx[k];
    if (li < 0 || li >= n_seg) {
        flag(e, SPHB_ST_BAD_INDEX);
        return;
    }
    const long long ui = (long long)user_offset[s] + li;
    if (field <= 13 || field == 21 || field == 22) {
        double *f = field_ptr<F32>(e, cur, field);
        if (dir == 0) f[k] = user[ui];
        else user[ui] = f[k];
        return;
    }
    if (field >= 23) {   // _a_rho_1, XSPH velocity: scatter only
        const void *src = field == 23 ? e.f.drho : field == 24 ? e.f.xu
                        : field == 25 ? e.f.xv : e.f.xw;
        user[ui] = F32 ? (double)((const float *)src)[k] : ((const double *)src)[k];
        return;
    }
    if (F32) {
        if (field <= 16) {
            float4 *th = (float4 *)e.f.thermo;
            float4 v = th[k];
            if (dir == 0) {
                const float x = (float)user[ui];
                if (field == 14) v.x = x;
                else if (field == 15) v.y = x;
                else v.z = x;
                v.w = v.x != 0.f ? v.y / (v.x * v.x) : 0.f;
                th[k] = v;
            } else {
                user[ui] = field == 14 ? v.x : (field == 15 ? v.y : v.z);
            }
            return;
        }
        float *f = (float *)(field == 17 ? e.f.au : field == 18 ? e.f.av
                             : field == 19 ? e.f.aw : e.f.dt_fac);
        if (dir == 0) f[k] = (float)user[ui];
        else user[ui] = f[k];
    } else {
        double *f = (double *)(field == 14 ? e.f.rho : field == 15 ? e.f.p
                              : field == 16 ? e.f.cs : field == 17 ? e.f.au
                              : field == 18 ? e.f.av : field == 19 ? e.f.aw
                              : e.f.dt_fac);
        if (dir == 0) f[k] = user[ui];
        else user[ui] = f[k];
    }
}

__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_exchange_tag(const __grid_constant__ sphb_engine e, int cur, int array, int dir,
               int *user, const int *user_offset)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (a != array) return;
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const int n_seg = e.seg_offset[t.seg + 1] - e.seg_offset[t.seg];
    const int li = e.buf[cur].idx[k];
    if (li < 0 || li >= n_seg) {
        flag(e, SPHB_ST_BAD_INDEX);
        return;
    }
    const long long ui = (long long)user_offset[s] + li;
    if (dir == 0) e.buf[cur].tag[k] = user[ui];
    else user[ui] = e.buf[cur].tag[k];
}

}  // namespace sphb

using namespace sphb;

extern "C" int sphb_abi_version(void) { return SPHB_ABI_VERSION; }

extern "C" const char *sphb_last_cuda_error(void) { return g_last_error; }

extern "C" int sphb_make_tiles(const int32_t *seg_offset_host, int32_t nseg,
                               int32_t tile_size, sphb_tile *tiles,
                               int32_t *num_tiles)
{
    if (!seg_offset_host || nseg < 0 || tile_size < 1 || !num_tiles) return SPHB_ERR_ARG;
    int32_t cnt = 0;
    for (int32_t g = 0; g < nseg; ++g) {
        const int32_t b = seg_offset_host[g], en = seg_offset_host[g + 1];
        if (en < b) return SPHB_ERR_ARG;
        for (int32_t i = b; i < en; i += tile_size) {
            if (tiles) {
                tiles[cnt].seg = g;
                tiles[cnt].begin = i;
                tiles[cnt].end = (en - i > tile_size) ? i + tile_size : en;
                tiles[cnt].pad0 = 0;
            }
            ++cnt;
        }
    }
    *num_tiles = cnt;
    return SPHB_OK;
}

extern "C" int sphb_workspace_layout(const sphb_config *cfg, size_t offsets[9],
                                     size_t *total_bytes)
{
    if (!cfg || !offsets || !total_bytes) return SPHB_ERR_ARG;
    if (cfg->num_particles < 0 || cfg->cell_capacity < 1) return SPHB_ERR_ARG;
    const size_t N = (size_t)cfg->num_particles, C = (size_t)cfg->cell_capacity;
    const size_t nb = (C + SPHB_SCAN_CHUNK - 1) / SPHB_SCAN_CHUNK;
    const size_t sizes[9] = {C * 4, (C + 1) * 4, N * 4, N * 4, N * 4,
                             (nb + 1) * 4, 8 * 4, 4, 4 * 8};
    size_t off = 0;
    for (int i = 0; i < 9; ++i) {
        offsets[i] = off;
        off += (sizes[i] + 255) & ~(size_t)255;
    }
    *total_bytes = off;
    return SPHB_OK;
}

extern "C" int sphb_pc_stage(const sphb_engine *e, int cur, int stage, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (stage < 0 || stage > 3) return SPHB_ERR_ARG;
    if (!e->f.au || !e->f.av) return SPHB_ERR_ARG;
    const sphb_buffers &B = e->buf[cur];
    if (!B.x0 || !B.y0 || !B.u0 || !B.v0) return SPHB_ERR_ARG;
    if (e->cfg.dim == 3 && (!B.z0 || !B.w0 || !e->f.aw)) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int nt = e->num_tiles;
    const bool f32 = e->cfg.precision == SPHB_FP32C;
    if (e->cfg.dim == 2) {
        if (f32) k_pc_stage<2, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, stage);
        else k_pc_stage<2, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, stage);
    } else {
        if (f32) k_pc_stage<3, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, stage);
        else k_pc_stage<3, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, stage);
    }
    return launch_status("sphb_pc_stage");
}

extern "C" int sphb_step_begin(const sphb_engine *e, void *stream)
{
    int rc = check_engine_public(e, 0);
    if (rc) return rc;
    k_step_begin<<<(e->cfg.num_scenes + 127) / 128, 128, 0, (cudaStream_t)stream>>>(*e);
    return launch_status("sphb_step_begin");
}

extern "C" int sphb_set_dt(const sphb_engine *e, double dt, void *stream)
{
    int rc = check_engine_public(e, 0);
    if (rc) return rc;
    if (!(dt > 0.0) || !isfinite(dt)) return SPHB_ERR_ARG;
    k_set_dt<<<(e->cfg.num_scenes + 127) / 128, 128, 0, (cudaStream_t)stream>>>(*e, dt);
    return launch_status("sphb_set_dt");
}

extern "C" int sphb_init_index(const sphb_engine *e, int cur, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!e->buf[cur].idx) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    k_init_index<<<e->num_tiles, SPHB_ELEM_TILE, 0, (cudaStream_t)stream>>>(*e, cur);
    return launch_status("sphb_init_index");
}

extern "C" int sphb_exchange(const sphb_engine *e, int cur, int array, int field,
                             int dir, double *user, const int32_t *user_offset,
                             void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!user || !user_offset || array < 0 || array >= e->cfg.num_arrays) return SPHB_ERR_ARG;
    if (field < 0 || field > 26 || (dir != 0 && dir != 1)) return SPHB_ERR_ARG;
    if (dir == 0 && ((field >= 17 && field <= 20) || field >= 23)) return SPHB_ERR_ARG;
    const bool f32 = e->cfg.precision == SPHB_FP32C;
    const sphb_buffers &B = e->buf[cur];
    const void *ptrs[27] = {B.x, B.y, B.z, B.u, B.v, B.w, B.x0, B.y0, B.z0, B.u0,
                            B.v0, B.w0, B.m, B.h,
                            f32 ? e->f.thermo : e->f.rho, f32 ? e->f.thermo : e->f.p,
                            f32 ? e->f.thermo : e->f.cs, e->f.au, e->f.av, e->f.aw,
                            e->f.dt_fac, B.rho, B.rho0, e->f.drho,
                            e->f.xu, e->f.xv, e->f.xw};
    if (!ptrs[field] || !B.idx) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (f32)
        k_exchange<true><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, field, dir, user, user_offset);
    else
        k_exchange<false><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, field, dir, user, user_offset);
    return launch_status("sphb_exchange");
}

extern "C" int sphb_exchange_tag(const sphb_engine *e, int cur, int array, int dir,
                                 int32_t *user, const int32_t *user_offset,
                                 void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!user || !user_offset || array < 0 || array >= e->cfg.num_arrays) return SPHB_ERR_ARG;
    if ((dir != 0 && dir != 1) || !e->buf[cur].tag || !e->buf[cur].idx) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    k_exchange_tag<<<e->num_tiles, SPHB_ELEM_TILE, 0, (cudaStream_t)stream>>>(*e, cur, array, dir, user, user_offset);
    return launch_status("sphb_exchange_tag");
}
