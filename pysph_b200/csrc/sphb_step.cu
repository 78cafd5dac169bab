// sphb_step.cu -- integrator stages (the per-particle stage itself is in
// sphb_stage.cuh), the per-step prologue (count, CFL time step), user <->
// engine order exchange, and the host helpers of the C ABI (sm_100a).

#include <stdio.h>
#include <string.h>

#include "sphb_common.cuh"
#include "sphb_stage.cuh"

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
    if ((stage == 0 || (stage >= 4 && stage <= 6)) && blockIdx.x == 0) {
        // the CFL rule reads the maxima of the step's last force pass only
        // (dt_fac is reset per calc, S/sph/sph_calc.pyx:324): clear what the
        // earlier stages' passes accumulated
        for (int q = threadIdx.x; q < e.cfg.num_scenes; q += blockDim.x) {
            e.sstate[q].max_dtfac = 0ull;
            e.sstate[q].max_acc2 = 0ull;
        }
    }
    const int k = t.begin + threadIdx.x;
    const bool rate = e.buf[cur].rho && e.f.drho && e.cfg.rate_src[a];
    const bool stepped = (e.cfg.step_on >> a) & 1u;
    if (!rate && !stepped) return;   // block-uniform
    float d2 = 0.f;
    if (k < t.end) {
        // the rates the force pass left: accelerations, XSPH velocity,
        // density rate
        auto ld = [&](const void *q) {
            return F32 ? (double)((const float *)q)[k] : ((const double *)q)[k];
        };
        const bool xsph = e.cfg.xsph_src[a] && e.f.xu && e.f.xv && (DIM == 2 || e.f.xw);
        double f[3] = {0.0, 0.0, 0.0}, xv[3] = {0.0, 0.0, 0.0};
        if (stepped) {
            const void *fa[3] = {e.f.au, e.f.av, e.f.aw};
            const void *xa[3] = {e.f.xu, e.f.xv, e.f.xw};
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                f[d] = ld(fa[d]);
                if (xsph) xv[d] = ld(xa[d]);
            }
        }
        const double dr = rate ? ld(e.f.drho) : 0.0;
        // FP32 pair records rewritten in place
        const bool rec = F32 && e.f.geo && e.f.vel && stepped;
        float4 *geo = rec ? (float4 *)e.f.geo : nullptr;
        const float4 g_old = rec ? geo[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        d2 = stage_particle<DIM, F32>(e, cur, k, s, a, stage, f, xsph, xv, dr, geo,
                                      rec ? e.f.vel : nullptr, g_old);
    }
    if (stepped && e.f.anchor) warp_max_disp(e, s, d2);
}

// Solver.solve per-step prologue for every scene.
__global__ void k_step_begin(const __grid_constant__ sphb_engine e)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.cfg.num_scenes) return;
    step_begin_scene(e, s);
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

// Import marks of a gather (dir 0): new masses or smoothing lengths mean
// the lists must be recorded again; new positions or velocities mean the
// records are stale and the particles may have left their anchors, so the
// next decision rebins unless sphb_refresh measures them first (meta[5]).
__device__ __forceinline__ void exchange_marks(const sphb_engine &e, int field, int dir)
{
    if (dir == 0 && (field <= 5 || field == 12 || field == 13)) {
        e.work.meta[2] = 0;
        e.work.meta[3] = 0;
        if (field <= 5) e.work.meta[5] = 1;
        else e.work.meta[4] = 0;
    }
}

// Engine position k <-> user position ui of one field.
template <bool F32>
__device__ __forceinline__ void exchange_field(const sphb_engine &e, int cur, int field, int dir,
                                               double *user, long long ui, int k)
{
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

// Engine position of this thread, and its user position in the array
// `array` (false when the thread has no particle of that array).
__device__ __forceinline__ bool exchange_slot(const sphb_engine &e, int cur, int array,
                                              const int *user_offset, int &k, long long &ui)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (a != array) return false;
    k = t.begin + threadIdx.x;
    if (k >= t.end) return false;
    const int n_seg = e.seg_offset[t.seg + 1] - e.seg_offset[t.seg];
    const int li = e.buf[cur].idx[k];
    if (li < 0 || li >= n_seg) {
        flag(e, SPHB_ST_BAD_INDEX);
        return false;
    }
    ui = (long long)user_offset[s] + li;
    return true;
}

template <bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_exchange(const __grid_constant__ sphb_engine e, int cur, int array, int field,
           int dir, double *user, const int *user_offset)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) exchange_marks(e, field, dir);
    int k;
    long long ui;
    if (exchange_slot(e, cur, array, user_offset, k, ui))
        exchange_field<F32>(e, cur, field, dir, user, ui, k);
}

// Several fields of one array: the tile, index and offset loads once.
struct ExchangeList {
    int count;
    int field[SPHB_EXCHANGE_MAX];
    double *user[SPHB_EXCHANGE_MAX];
};

template <bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_exchange_many(const __grid_constant__ sphb_engine e, int cur, int array, int dir,
                const __grid_constant__ ExchangeList l, const int *user_offset)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int i = 0; i < l.count; ++i) exchange_marks(e, l.field[i], dir);
    int k;
    long long ui;
    if (!exchange_slot(e, cur, array, user_offset, k, ui)) return;
    for (int i = 0; i < l.count; ++i) exchange_field<F32>(e, cur, l.field[i], dir, l.user[i], ui, k);
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
    // bsum: the scan's chunk totals, then the rebin barrier's counters
    const size_t sizes[9] = {C * 4, (C + 1) * 4, N * 4, N * 4, N * 4,
                             (nb + 1 + 64) * 4, 8 * 4, 4, 4 * 8};
    size_t off = 0;
    for (int i = 0; i < 9; ++i) {
        offsets[i] = off;
        off += (sizes[i] + 255) & ~(size_t)255;
    }
    *total_bytes = off;
    return SPHB_OK;
}

// RK4's stages (kinds 4-7) need the running sums of every integrated
// property: x, y(, z), u, v(, w) of the stepped arrays, rho of the density
// rate dests.
namespace sphb {
int check_stage_sums(const sphb_engine *e, int cur, int kind)
{
    if (kind < 4) return SPHB_OK;
    const sphb_config &c = e->cfg;
    const sphb_buffers &B = e->buf[cur];
    if (c.step_on && (!B.kx || !B.ky || !B.ku || !B.kv || (c.dim == 3 && (!B.kz || !B.kw))))
        return SPHB_ERR_ARG;
    for (int a = 0; a < c.num_arrays; ++a)
        if (c.rate_src[a] && B.rho && !B.krho) return SPHB_ERR_ARG;
    return SPHB_OK;
}
}  // namespace sphb

extern "C" int sphb_pc_stage(const sphb_engine *e, int cur, int stage, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (stage < 0 || stage > 7) return SPHB_ERR_ARG;
    if ((rc = check_stage_sums(e, cur, stage))) return rc;
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

// SPHB_OK when `field` can be exchanged in direction `dir` on this engine.
static int exchange_field_ok(const sphb_engine *e, int cur, int field, int dir)
{
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
    return SPHB_OK;
}

extern "C" int sphb_exchange(const sphb_engine *e, int cur, int array, int field,
                             int dir, double *user, const int32_t *user_offset,
                             void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!user || !user_offset || array < 0 || array >= e->cfg.num_arrays) return SPHB_ERR_ARG;
    rc = exchange_field_ok(e, cur, field, dir);
    if (rc) return rc;
    const bool f32 = e->cfg.precision == SPHB_FP32C;
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (f32)
        k_exchange<true><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, field, dir, user, user_offset);
    else
        k_exchange<false><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, field, dir, user, user_offset);
    return launch_status("sphb_exchange");
}

extern "C" int sphb_exchange_many(const sphb_engine *e, int cur, int array, int dir,
                                  int32_t count, const int32_t *fields, double *const *users,
                                  const int32_t *user_offset, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!fields || !users || !user_offset || array < 0 || array >= e->cfg.num_arrays ||
        count < 1 || count > SPHB_EXCHANGE_MAX)
        return SPHB_ERR_ARG;
    ExchangeList l;
    l.count = count;
    for (int i = 0; i < count; ++i) {
        rc = exchange_field_ok(e, cur, fields[i], dir);
        if (rc) return rc;
        if (!users[i]) return SPHB_ERR_ARG;
        l.field[i] = fields[i];
        l.user[i] = users[i];
    }
    for (int i = count; i < SPHB_EXCHANGE_MAX; ++i) {
        l.field[i] = 0;
        l.user[i] = nullptr;
    }
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (e->cfg.precision == SPHB_FP32C)
        k_exchange_many<true><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, dir, l, user_offset);
    else
        k_exchange_many<false><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, array, dir, l, user_offset);
    return launch_status("sphb_exchange_many");
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
