// sphb_density.cu -- the density entry point (the pass itself is in
// sphb_density_pass.cuh), the stand-alone Tait kernel, neighbour-list
// emission and cell coordinates (sm_100a).
//
// TaitEquation (S/sph/funcs/eos_funcs.pyx:88-129): p = B((rho/rho0)^gamma-1),
// cs = c0 (rho/rho0)^((gamma-1)/2).  Non-LocalReal dests get 0
// (S/sph/sph_func.pyx:220-227).

#include "sphb_launch.cuh"
#include "sphb_pairs.cuh"

namespace sphb {

int check_engine_public(const sphb_engine *e, int cur);


// Tait alone (rho given).
template <bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_tait(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask)
{
    // the force pass that follows may launch once every block has started
    pdl_trigger();
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (!((dest_mask >> a) & 1u)) return;
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const sphb_scene &sc = e.scene[s];
    const sphb_buffers &B = e.buf[cur];
    const bool real = B.tag[k] == 0;
    // continuity scheme: the density is the integrated state, which the
    // pair passes then read from the same place as a summed one
    const bool state = B.rho != nullptr && e.cfg.rate_src[a] != 0u;
    double rho;
    if (state) rho = B.rho[k];
    else if constexpr (F32) rho = ((const float4 *)e.f.thermo)[k].x;
    else rho = ((const double *)e.f.rho)[k];
    double p = 0.0, c = 0.0;
    if (real) {
        const double ratio = rho / sc.rho0;
        p = (eos_pow<F32>(ratio, sc.gamma) - 1.0) * sc.B;
        c = eos_pow<F32>(ratio, 0.5 * (sc.gamma - 1.0)) * sc.c0;
    }
    if constexpr (F32) {
        float4 *th = (float4 *)e.f.thermo;
        float4 v = th[k];
        if (state) v.x = (float)rho;
        v.y = (float)p;
        v.z = (float)c;
        v.w = v.x != 0.f ? v.y / (v.x * v.x) : 0.f;
        th[k] = v;
        if (state && !(isfinite(v.x) && isfinite(v.y))) flag(e, SPHB_ST_NONFINITE_RHO);
    } else {
        if (state) ((double *)e.f.rho)[k] = rho;
        ((double *)e.f.p)[k] = p;
        ((double *)e.f.cs)[k] = c;
        if (state && !(isfinite(rho) && isfinite(p))) flag(e, SPHB_ST_NONFINITE_RHO);
    }
}

// Neighbour lists with the reference's exact FP64 predicate (the symmetric
// one with variable h).
template <int DIM, int R>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_neighbors(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask, uint32_t src_mask,
            int *counts, const long long *offs, int *out, long long cap)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    if (!((dest_mask >> a) & 1u)) return;
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const sphb_scene_state &st = e.sstate[s];
    const int n[3] = {st.n[0], st.n[1], st.n[2]};
    const sphb_buffers &B = e.buf[cur];
    const double xk = B.x[k], yk = B.y[k], zk = DIM == 3 ? B.z[k] : 0.0;
    const double rad = B.h[k] * e.scene[s].radius_scale;
    const double rad2 = __dmul_rn(rad, rad);
    const bool vh = e.scene[s].variable_h != 0;
    int cx, cy, cz;
    cell_coords(e.f.cell[k], n, cx, cy, cz);
    int cnt = 0;
    const long long base = offs ? offs[k] : 0;
    for_each_candidate<DIM, R, 1>(
        e.work.start, A, src_mask, st.cell_base, st.ncells, n, cx, cy, cz, 0,
        e.cfg.num_particles, e.work.status, CellTrim{},
        [&](int j, int, int, int) {
            const double dx = B.x[j] - xk;
            const double dy = B.y[j] - yk;
            const double dz = DIM == 3 ? B.z[j] - zk : 0.0;
            const double d2 = dist2_ref<DIM>(dx, dy, dz);
            bool in = d2 < rad2;
            if (vh && !in) {
                // variable h: also the particles whose own support holds k
                const double rj = B.h[j] * e.scene[s].radius_scale;
                in = d2 < __dmul_rn(rj, rj);
            }
            if (in) {
                if (offs) {
                    const long long pos = base + cnt;
                    if (pos < cap) out[pos] = j;
                    else flag(e, SPHB_ST_NBR_CAPACITY);
                }
                ++cnt;
            }
        });
    counts[k] = cnt;
}

__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_cell_coords(const __grid_constant__ sphb_engine e, int *out)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const int s = t.seg / e.cfg.num_arrays;
    const sphb_scene_state &st = e.sstate[s];
    int cx, cy, cz;
    cell_coords(e.f.cell[k], st.n, cx, cy, cz);
    out[3 * k + 0] = st.lo[0] + cx;
    out[3 * k + 1] = st.lo[1] + cy;
    out[3 * k + 2] = e.cfg.dim == 3 ? st.lo[2] + cz : 0;
}


int check_pair_cfg(const sphb_engine *e)
{
    const sphb_config &c = e->cfg;
    if (c.lanes != 1 && c.lanes != 2 && c.lanes != 4 && c.lanes != 8) return SPHB_ERR_UNSUPPORTED;
    if (c.pair_block < 32 || c.pair_block > 256 || (c.pair_block & 31)) return SPHB_ERR_ARG;
    if (c.list_batch != 0 && c.list_batch != 2 && c.list_batch != 4) return SPHB_ERR_ARG;
    if (!e->pair_tiles || e->num_pair_tiles < 0) return SPHB_ERR_ARG;
    if (!e->work.start || !e->f.cell) return SPHB_ERR_ARG;
    if (!pass_variant(c)) return SPHB_ERR_UNSUPPORTED;   // kernel type / dimension
    if (c.pair_mode != SPHB_PAIRS_LISTS && c.pair_mode != SPHB_PAIRS_TILED) return SPHB_ERR_ARG;
    if (c.pair_mode == SPHB_PAIRS_TILED) {
        // 2D FP32C, one thread per dest, the summation-density scheme
        if (c.dim != 2 || c.precision != SPHB_FP32C || c.lanes != 1) return SPHB_ERR_UNSUPPORTED;
        for (int a = 0; a < SPHB_MAX_ARRAYS; ++a)
            if (c.rate_src[a] || c.xsph_src[a]) return SPHB_ERR_UNSUPPORTED;
        if (c.num_particles >= (1 << SPHB_NBR_IDX_BITS_2D)) return SPHB_ERR_UNSUPPORTED;
    }
    return SPHB_OK;
}

}  // namespace sphb

using namespace sphb;

extern "C" int sphb_density(const sphb_engine *e, int cur, uint32_t dest_mask,
                            int with_eos, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if ((rc = check_pair_cfg(e))) return rc;
    if (with_eos & ~(SPHB_DENSITY_EOS | SPHB_DENSITY_USE_LIST | SPHB_DENSITY_LIST_IF_VALID |
                     SPHB_DENSITY_LISTS_ONLY))
        return SPHB_ERR_ARG;
    if (e->cfg.pair_mode == SPHB_PAIRS_TILED && (with_eos & SPHB_DENSITY_LISTS_ONLY))
        return SPHB_ERR_UNSUPPORTED;
    if (e->num_pair_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const sphb_config &c = e->cfg;
    if (c.precision == SPHB_FP32C) {
        if (!e->f.geo || !e->f.thermo || (c.dim == 3 && !e->f.mass)) return SPHB_ERR_ARG;
    } else {
        if (!e->f.rho || !e->f.p || !e->f.cs) return SPHB_ERR_ARG;
    }
    switch (pass_variant(c)) {
    case 12: launch_density_kt<SPHB_KERNEL_CUBIC, 2>(*e, cur, dest_mask, with_eos, st); break;
    case 13: launch_density_kt<SPHB_KERNEL_CUBIC, 3>(*e, cur, dest_mask, with_eos, st); break;
    case 32: launch_density_kt<SPHB_KERNEL_QUINTIC, 2>(*e, cur, dest_mask, with_eos, st); break;
    case 42: launch_density_kt<SPHB_KERNEL_WENDLAND, 2>(*e, cur, dest_mask, with_eos, st); break;
    default: return SPHB_ERR_UNSUPPORTED;
    }
    return launch_status("sphb_density");
}

extern "C" int sphb_tait(const sphb_engine *e, int cur, uint32_t dest_mask, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (e->cfg.precision == SPHB_FP32C)
        k_tait<true><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask);
    else
        k_tait<false><<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask);
    return launch_status("sphb_tait");
}

extern "C" int sphb_neighbors(const sphb_engine *e, int cur, uint32_t dest_mask,
                              uint32_t src_mask, int32_t *counts,
                              const int64_t *nbr_offsets, int32_t *nbr_index,
                              int64_t nbr_capacity, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!counts || (nbr_offsets && !nbr_index) || !e->work.start || !e->f.cell)
        return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const long long *offs = (const long long *)nbr_offsets;
    const int nt = e->num_tiles;
    const int key = e->cfg.dim * 10 + e->cfg.stencil;
    switch (key) {
    case 21: k_neighbors<2, 1><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask, src_mask, counts, offs, nbr_index, nbr_capacity); break;
    case 22: k_neighbors<2, 2><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask, src_mask, counts, offs, nbr_index, nbr_capacity); break;
    case 31: k_neighbors<3, 1><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask, src_mask, counts, offs, nbr_index, nbr_capacity); break;
    case 32: k_neighbors<3, 2><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, dest_mask, src_mask, counts, offs, nbr_index, nbr_capacity); break;
    default: return SPHB_ERR_UNSUPPORTED;
    }
    return launch_status("sphb_neighbors");
}

extern "C" int sphb_cell_coords(const sphb_engine *e, int cur, int32_t *out, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!out || !e->f.cell) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    k_cell_coords<<<e->num_tiles, SPHB_ELEM_TILE, 0, (cudaStream_t)stream>>>(*e, out);
    return launch_status("sphb_cell_coords");
}
