// sphb_bin.cu -- cell binning for the particle engine (sm_100a).
//
// One rebin = scene boxes -> per-scene grids -> cell key per particle ->
// counting sort (histogram, two-level scan, scatter) -> gather of the
// particle state into the other buffer in cell order, ranking the members of
// each cell by particle index so the order is canonical, plus the FP32 pair
// records and the anchors (binned positions).  With SPHB_BIN_IF_NEEDED a
// one-block kernel first decides on the device whether the lists still
// cover every pair (no particle has moved skin/2 from its anchor); when they
// do, every later kernel of the rebin returns at once, and when they do not,
// the gathered state is copied back so it stays in buf[cur].
//
// The reference bins with a Python dict of cells keyed by floor(x / cs)
// (CellManager._insert_particles, S/base/cell.pyx:1229-1300); its OpenCL
// manager hashes to a flattened cell id and radix-sorts the keys
// (RadixSortManager._cl_update, S/base/domain_manager.py:901-972;
// bin / compute_cell_counts, S/base/radix_sort.cl:31-108).  Here the keys are
// bounded by the grid, so a counting sort replaces the radix sort and the
// state itself is permuted so every later kernel reads it coalesced.

#include <mutex>

#include "sphb_common.cuh"
#include "sphb_stage.cuh"

namespace sphb {

// ---------------------------------------------------------------- boxes --
// work.meta[1] == 0 after a decision to keep the lists: the rebin is off
__device__ __forceinline__ bool skip_rebin(const sphb_engine &e, int gated)
{
    return gated && *(volatile int *)&e.work.meta[1] == 0;
}

// One block.  No rebin while the particles sit where the last rebin put
// them (work.meta[3] == 2); otherwise rebin unless the lists were recorded
// with the skin at those positions (work.meta[4]) and no particle of any
// scene has moved skin_max / 2 (less a relative 1e-4 for the FP32 rounding
// of the displacement) from its anchor.  max_disp2 restarts either way.
__global__ void k_bin_decide(const __grid_constant__ sphb_engine e,
                             cudaGraphConditionalHandle cond, int set_cond, int step_begin)
{
    // launched as a programmatic dependent of the stage before: its
    // displacements and meta must be complete
    pdl_wait();
    __shared__ int s_far;
    if (threadIdx.x == 0) s_far = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < e.cfg.num_scenes; s += blockDim.x) {
        if (step_begin) step_begin_scene(e, s);
        sphb_scene_state &st = e.sstate[s];
        const double d2 = __longlong_as_double((long long)st.max_disp2);
        const double lim = 0.5 * e.scene[s].skin_max * (1.0 - 1e-4);
        if (!(d2 < lim * lim)) s_far = 1;
        st.max_disp2 = 0ull;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool at_anchor = e.work.meta[3] == 2;
        // host-written state nobody has measured: no trusting the lists
        const bool lists = e.work.meta[4] == 1 && e.work.meta[5] == 0;
        const bool keep = at_anchor || (lists && !s_far);
        e.work.meta[1] = keep ? 0 : 1;
        e.work.meta[2] = (keep && lists) ? 1 : 0;
        if (!keep) e.work.pairs[3] += 1ull;   // rebins decided on the device
        // inside a captured graph: run the rebin's conditional body or not
        if (set_cond) cudaGraphSetConditional(cond, keep ? 0u : 1u);
    }
}

__global__ void k_box_reset(const __grid_constant__ sphb_engine e, int gated)
{
    if (skip_rebin(e, gated)) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= e.cfg.num_scenes) return;
    for (int d = 0; d < 3; ++d) {
        e.sstate[s].box[d] = enc_double(INFINITY);
        e.sstate[s].box[3 + d] = enc_double(-INFINITY);
    }
}

__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_box_accum(const __grid_constant__ sphb_engine e, int cur, int gated)
{
    if (skip_rebin(e, gated)) return;
    const sphb_tile t = e.tiles[blockIdx.x];
    const int s = t.seg / e.cfg.num_arrays;
    const int k = t.begin + threadIdx.x;
    const sphb_buffers &B = e.buf[cur];
    const int dim = e.cfg.dim;
    double p[3] = {0.0, 0.0, 0.0};
    bool ok = false;
    if (k < t.end) {
        p[0] = B.x[k];
        p[1] = B.y[k];
        if (dim == 3) p[2] = B.z[k];
        ok = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
    }
    for (int d = 0; d < dim; ++d) {
        double lo = block_reduce(ok ? p[d] : INFINITY, OpMin(), (double)INFINITY);
        if (threadIdx.x == 0 && lo < INFINITY)
            atomic_min_enc(&e.sstate[s].box[d], enc_double(lo));
        double hi = block_reduce(ok ? p[d] : -INFINITY, OpMax(), (double)-INFINITY);
        if (threadIdx.x == 0 && hi > -INFINITY)
            atomic_max_enc(&e.sstate[s].box[3 + d], enc_double(hi));
    }
}

// FP32 pair records from the FP64 state without reordering (FP32C):
// positions relative to the origin of each particle's cell of the last bin,
// velocities, into both record copies.  With anchors, every particle's
// displacement from its anchor goes into its scene's max_disp2, and the
// host-written state counts as measured (meta[5]).
template <int DIM, bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_refresh(const __grid_constant__ sphb_engine e, int cur)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A;
    if (blockIdx.x == 0 && threadIdx.x == 0) e.work.meta[5] = 0;
    float d2 = 0.f;
    if (k < t.end) {
        const sphb_scene_state &st = e.sstate[s];
        const double cs = e.scene[s].cell_size;
        const sphb_buffers &B = e.buf[cur];
        int local = e.f.cell[k];
        if (local < 0 || local >= st.ncells) {
            flag(e, SPHB_ST_BAD_INDEX);
            local = 0;
        }
        int cx, cy, cz;
        cell_coords(local, st.n, cx, cy, cz);
        const float xr = (float)(B.x[k] - (double)(st.lo[0] + cx) * cs);
        const float yr = (float)(B.y[k] - (double)(st.lo[1] + cy) * cs);
        const float zr = DIM == 3 ? (float)(B.z[k] - (double)(st.lo[2] + cz) * cs) : 0.f;
        if (F32) {
            float4 *geo = (float4 *)e.f.geo;
            const float4 g = geo[k];
            // both copies of the records when the force pass steps the state
            const float4 gn = DIM == 2 ? make_float4(xr, yr, g.z, g.w)
                                       : make_float4(xr, yr, zr, g.w);
            geo[k] = gn;
            if (e.f.geo_next) ((float4 *)e.f.geo_next)[k] = gn;
            if (DIM == 2) {
                const float2 vv = make_float2((float)B.u[k], (float)B.v[k]);
                ((float2 *)e.f.vel)[k] = vv;
                if (e.f.vel_next) ((float2 *)e.f.vel_next)[k] = vv;
            } else {
                const float4 vv = make_float4((float)B.u[k], (float)B.v[k], (float)B.w[k], 0.f);
                ((float4 *)e.f.vel)[k] = vv;
                if (e.f.vel_next) ((float4 *)e.f.vel_next)[k] = vv;
            }
        }
        if (e.f.anchor) {
            float q0, q1, q2 = 0.f;
            if (DIM == 2) {
                const float2 an = ((const float2 *)e.f.anchor)[k];
                q0 = xr - an.x;
                q1 = yr - an.y;
            } else {
                const float4 an = ((const float4 *)e.f.anchor)[k];
                q0 = xr - an.x;
                q1 = yr - an.y;
                q2 = zr - an.z;
            }
            d2 = q0 * q0 + q1 * q1 + q2 * q2;
            // a non-finite position can never be within the skin
            if (!(d2 <= 3.0e38f)) d2 = 3.0e38f;
        }
    }
    // a block never spans two scenes
    if (e.f.anchor) warp_max_disp(e, s, d2);
}

// ----------------------------------------------------------- grid setup --
// One block.  Grid of scene s: cells floor(lo/cs)-R .. floor(hi/cs)+R per
// axis (R padding cells, so every stencil row of every particle exists);
// exclusive prefix of A*ncells over scenes gives the scene key bases.
__global__ void __launch_bounds__(1024) k_grid_setup(const __grid_constant__ sphb_engine e, int gated)
{
    if (skip_rebin(e, gated)) return;
    __shared__ long long sh[1024];
    __shared__ long long s_carry;
    const int S = e.cfg.num_scenes, A = e.cfg.num_arrays, R = e.cfg.stencil;
    const int dim = e.cfg.dim;
    const long long cap = e.cfg.cell_capacity;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < S; base += blockDim.x) {
        const int s = base + threadIdx.x;
        long long need = 0;
        int lo[3] = {0, 0, 0}, n[3] = {1, 1, 1};
        bool bad = false;
        if (s < S) {
            const sphb_scene &sc = e.scene[s];
            sphb_scene_state &st = e.sstate[s];
            const double cs = sc.cell_size;
            for (int d = 0; d < dim; ++d) {
                double blo = dec_double(st.box[d]);
                double bhi = dec_double(st.box[3 + d]);
                if (!(blo <= bhi)) { blo = 0.0; bhi = 0.0; }
                const double flo = floor(blo / cs), fhi = floor(bhi / cs);
                if (!(fabs(flo) < 1.0e9) || !(fabs(fhi) < 1.0e9) ||
                    !(fhi - flo < 1.0e8)) {
                    bad = true;
                    lo[d] = 0;
                    n[d] = 1;
                } else {
                    lo[d] = (int)flo - R;
                    n[d] = (int)(fhi - flo) + 1 + 2 * R;
                }
            }
            need = (long long)A * n[0] * n[1] * n[2];
            if (bad || need > cap) { bad = true; need = 0; }
        }
        sh[threadIdx.x] = need;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            long long v = (int)threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += v;
            __syncthreads();
        }
        const long long incl = sh[threadIdx.x];
        const long long total = sh[blockDim.x - 1];
        if (s < S) {
            sphb_scene_state &st = e.sstate[s];
            const long long cb = s_carry + incl - need;
            if (bad || cb + need > cap) {
                flag(e, SPHB_ST_GRID_OVERFLOW);
                for (int d = 0; d < 3; ++d) { st.lo[d] = 0; st.n[d] = 1; }
                st.cell_base = 0;
                st.ncells = 0;
            } else {
                for (int d = 0; d < 3; ++d) { st.lo[d] = lo[d]; st.n[d] = n[d]; }
                st.cell_base = (int)cb;
                st.ncells = n[0] * n[1] * n[2];
            }
            st.max_disp2 = 0ull;   // the anchors are the new positions
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        long long used = s_carry;
        if (used > cap) {
            flag(e, SPHB_ST_GRID_OVERFLOW);
            used = 0;
        }
        e.work.meta[0] = (int)used;
        // new order: the lists must be recorded again before they are
        // reused; the positions are the anchors
        e.work.meta[1] = 1;
        e.work.meta[2] = 0;
        e.work.meta[3] = 2;
        // tiled pair passes search the cells, which stay complete while no
        // particle has moved half the skin from where this rebin put it
        e.work.meta[4] = e.cfg.pair_mode == SPHB_PAIRS_TILED ? 1 : 0;
        e.work.meta[5] = 0;
    }
}

// ----------------------------------------------------------------- hash --
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_hash(const __grid_constant__ sphb_engine e, int cur, int gated)
{
    if (skip_rebin(e, gated)) return;
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    const sphb_scene_state &st = e.sstate[s];
    const double cs = e.scene[s].cell_size;
    const sphb_buffers &B = e.buf[cur];
    const int dim = e.cfg.dim;
    double p[3] = {B.x[k], B.y[k], dim == 3 ? B.z[k] : 0.0};
    int c[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) {
        if (!isfinite(p[d])) {
            flag(e, SPHB_ST_NONFINITE_POS);
            e.work.key[k] = -1;
            return;
        }
        // floor(x / cs) exactly as find_cell_id (S/base/cell.pyx:44-84)
        const double f = floor(p[d] / cs) - (double)st.lo[d];
        if (!(f >= 0.0) || !(f < (double)st.n[d])) {
            flag(e, SPHB_ST_OUT_OF_GRID);
            e.work.key[k] = -1;
            return;
        }
        c[d] = (int)f;
    }
    const int local = (c[2] * st.n[1] + c[1]) * st.n[0] + c[0];
    const long long key = (long long)st.cell_base + (long long)a * st.ncells + local;
    if (local >= st.ncells || key >= (long long)e.work.meta[0]) {
        flag(e, SPHB_ST_OUT_OF_GRID);
        e.work.key[k] = -1;
        return;
    }
    e.work.slot[k] = atomicAdd(&e.work.count[key], 1);
    e.work.key[k] = (int)key;
}

// ----------------------------------------------------------------- scan --
__device__ __forceinline__ int block_excl_scan_int(int v, int &total)
{
    __shared__ int wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        int w = lane < nw ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    total = wsum[(blockDim.x >> 5) - 1];
    const int before = warp > 0 ? wsum[warp - 1] : 0;
    return before + x - v;
}

__global__ void __launch_bounds__(SPHB_SCAN_THREADS)
k_scan_reduce(const __grid_constant__ sphb_engine e, int gated)
{
    if (skip_rebin(e, gated)) return;
    const int T = e.work.meta[0];
    const long long base = (long long)blockIdx.x * SPHB_SCAN_CHUNK;
    int sum = 0;
    if (base < T) {
#pragma unroll
        for (int i = 0; i < SPHB_SCAN_ITEMS; ++i) {
            const long long c = base + (long long)i * SPHB_SCAN_THREADS + threadIdx.x;
            if (c < T) sum += e.work.count[c];
        }
    }
    int total;
    block_excl_scan_int(sum, total);
    if (threadIdx.x == 0) e.work.bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SPHB_SCAN_THREADS)
k_scan_top(const __grid_constant__ sphb_engine e, int nb, int gated)
{
    if (skip_rebin(e, gated)) return;
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? e.work.bsum[i] : 0;
        int total;
        const int ex = block_excl_scan_int(v, total);
        const int carry = s_carry;
        if (i < nb) e.work.bsum[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) e.work.bsum[nb] = s_carry;
}

__global__ void __launch_bounds__(SPHB_SCAN_THREADS)
k_scan_apply(const __grid_constant__ sphb_engine e, int gated)
{
    if (skip_rebin(e, gated)) return;
    const int T = e.work.meta[0];
    const long long base = (long long)blockIdx.x * SPHB_SCAN_CHUNK;
    if (T == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) e.work.start[0] = 0;
        return;
    }
    if (base >= T) return;
    const long long c0 = base + (long long)threadIdx.x * SPHB_SCAN_ITEMS;
    int v[SPHB_SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SPHB_SCAN_ITEMS; ++i) {
        v[i] = (c0 + i < T) ? e.work.count[c0 + i] : 0;
        sum += v[i];
    }
    int total;
    int run = block_excl_scan_int(sum, total) + e.work.bsum[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SPHB_SCAN_ITEMS; ++i) {
        const long long c = c0 + i;
        if (c < T) {
            e.work.start[c] = run;
            e.work.count[c] = 0;  // ready for the next bin
            run += v[i];
            if (c == T - 1) e.work.start[T] = run;
        }
    }
}

// -------------------------------------------------------------- scatter --
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_scatter(const __grid_constant__ sphb_engine e, int gated)
{
    if (skip_rebin(e, gated)) return;
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const int key = e.work.key[k];
    if (key < 0) return;
    const int pos = e.work.start[key] + e.work.slot[k];
    if (pos < 0 || pos >= e.cfg.num_particles) {
        flag(e, SPHB_ST_BAD_INDEX);
        return;
    }
    e.work.perm[pos] = k;
}

// -------------------------------------------------------------- reorder --
// Thread k takes particle p = perm[k] (the scatter put it somewhere inside
// its cell's range [b, e)), ranks it among the cell's members by their index
// in the particle array, and writes it to b + rank: the order inside a cell
// is canonical whatever order the atomics handed out the slots, and it does
// not depend on the order the particles had before.
template <int DIM, bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_reorder(const __grid_constant__ sphb_engine e, int cur, int move_initial, int gated)
{
    if (skip_rebin(e, gated)) return;
    const sphb_tile t = e.tiles[blockIdx.x];
    const int kk = t.begin + threadIdx.x;
    if (kk >= t.end) return;
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    const int seg_lo = e.seg_offset[t.seg], seg_hi = e.seg_offset[t.seg + 1];
    const int p = e.work.perm[kk];
    if (p < seg_lo || p >= seg_hi) {
        flag(e, SPHB_ST_BAD_INDEX);
        return;
    }
    int k = kk;
    {
        const int key = e.work.key[p];
        const int b = key >= 0 ? e.work.start[key] : -1;
        const int en = key >= 0 ? e.work.start[key + 1] : -1;
        if (b < seg_lo || en > seg_hi || kk < b || kk >= en) {
            flag(e, SPHB_ST_BAD_INDEX);
            return;
        }
        // canonical order inside a cell: by the particle's index in its
        // array, so the order depends on the positions alone
        const int *__restrict__ sidx = e.buf[cur].idx;
        const int me = sidx[p];
        int rank = 0;
        for (int i = b; i < en; ++i) rank += (sidx[e.work.perm[i]] < me) ? 1 : 0;
        k = b + rank;
    }
    const sphb_buffers &S = e.buf[cur];
    const sphb_buffers &D = e.buf[cur ^ 1];
    const double x = S.x[p], y = S.y[p];
    const double u = S.u[p], v = S.v[p];
    const double m = S.m[p], h = S.h[p];
    D.x[k] = x;
    D.y[k] = y;
    D.u[k] = u;
    D.v[k] = v;
    D.m[k] = m;
    D.h[k] = h;
    D.idx[k] = S.idx[p];
    D.tag[k] = S.tag[p];
    if (S.rho && D.rho) D.rho[k] = S.rho[p];   // integrated density (continuity)
    if (move_initial && S.rho0 && D.rho0) D.rho0[k] = S.rho0[p];
    double z = 0.0, w = 0.0;
    if (DIM == 3) {
        z = S.z[p];
        w = S.w[p];
        D.z[k] = z;
        D.w[k] = w;
    }
    if (move_initial) {
        D.x0[k] = S.x0[p];
        D.y0[k] = S.y0[p];
        D.u0[k] = S.u0[p];
        D.v0[k] = S.v0[p];
        if (DIM == 3) {
            D.z0[k] = S.z0[p];
            D.w0[k] = S.w0[p];
        }
    }
    const sphb_scene_state &st = e.sstate[s];
    const int key = e.work.key[p];
    int local = key - st.cell_base - a * st.ncells;
    if (key < 0 || local < 0 || local >= st.ncells) {
        flag(e, SPHB_ST_BAD_INDEX);
        local = 0;
    }
    e.f.cell[k] = local;
    if (!F32 && !e.f.anchor) return;
    const double cs = e.scene[s].cell_size;
    int cx, cy, cz;
    cell_coords(local, st.n, cx, cy, cz);
    // position relative to the origin of the particle's own cell
    const float xr = (float)(x - (double)(st.lo[0] + cx) * cs);
    const float yr = (float)(y - (double)(st.lo[1] + cy) * cs);
    const float zr = DIM == 3 ? (float)(z - (double)(st.lo[2] + cz) * cs) : 0.f;
    if (F32) {
        // both copies of the records when the force pass steps the state
        const float4 g = DIM == 2 ? make_float4(xr, yr, (float)h, (float)m)
                                  : make_float4(xr, yr, zr, (float)h);
        ((float4 *)e.f.geo)[k] = g;
        if (e.f.geo_next) ((float4 *)e.f.geo_next)[k] = g;
        if (DIM == 2) {
            const float2 vv = make_float2((float)u, (float)v);
            ((float2 *)e.f.vel)[k] = vv;
            if (e.f.vel_next) ((float2 *)e.f.vel_next)[k] = vv;
        } else {
            ((float *)e.f.mass)[k] = (float)m;
            const float4 vv = make_float4((float)u, (float)v, (float)w, 0.f);
            ((float4 *)e.f.vel)[k] = vv;
            if (e.f.vel_next) ((float4 *)e.f.vel_next)[k] = vv;
        }
    }
    if (e.f.anchor) {
        if (DIM == 2) ((float2 *)e.f.anchor)[k] = make_float2(xr, yr);
        else ((float4 *)e.f.anchor)[k] = make_float4(xr, yr, zr, 0.f);
    }
}

// After a rebin decided on the device: the gathered state back into
// buf[cur], same order (the records, anchors and cells already follow it).
template <int DIM>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_copy_back(const __grid_constant__ sphb_engine e, int cur, int move_initial, int gated)
{
    if (skip_rebin(e, gated)) return;
    const sphb_tile t = e.tiles[blockIdx.x];
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    const sphb_buffers &S = e.buf[cur ^ 1];
    const sphb_buffers &D = e.buf[cur];
    D.x[k] = S.x[k];
    D.y[k] = S.y[k];
    D.u[k] = S.u[k];
    D.v[k] = S.v[k];
    D.m[k] = S.m[k];
    D.h[k] = S.h[k];
    D.idx[k] = S.idx[k];
    D.tag[k] = S.tag[k];
    if (S.rho && D.rho) D.rho[k] = S.rho[k];
    if (move_initial && S.rho0 && D.rho0) D.rho0[k] = S.rho0[k];
    if (DIM == 3) {
        D.z[k] = S.z[k];
        D.w[k] = S.w[k];
    }
    if (move_initial) {
        D.x0[k] = S.x0[k];
        D.y0[k] = S.y0[k];
        D.u0[k] = S.u0[k];
        D.v0[k] = S.v0[k];
        if (DIM == 3) {
            D.z0[k] = S.z0[k];
            D.w0[k] = S.w0[k];
        }
    }
}

// --------------------------------------------------------- entry points --
static int check_engine(const sphb_engine *e, int cur)
{
    if (!e || (cur != 0 && cur != 1)) return SPHB_ERR_ARG;
    const sphb_config &c = e->cfg;
    if (c.dim != 2 && c.dim != 3) return SPHB_ERR_UNSUPPORTED;
    if (c.precision != SPHB_FP64 && c.precision != SPHB_FP32C) return SPHB_ERR_UNSUPPORTED;
    if (c.stencil < 1 || c.stencil > SPHB_MAX_STENCIL) return SPHB_ERR_UNSUPPORTED;
    if (c.num_scenes < 1 || c.num_arrays < 1 || c.num_arrays > SPHB_MAX_ARRAYS)
        return SPHB_ERR_ARG;
    if (c.num_particles < 0 || c.cell_capacity < 1) return SPHB_ERR_ARG;
    if (!e->tiles || e->num_tiles < 0 || !e->seg_offset || !e->scene || !e->sstate)
        return SPHB_ERR_ARG;
    return SPHB_OK;
}

int check_engine_public(const sphb_engine *e, int cur) { return check_engine(e, cur); }

int bin_scan_blocks(const sphb_config &c)
{
    return (int)((c.cell_capacity + SPHB_SCAN_CHUNK - 1) / SPHB_SCAN_CHUNK);
}

}  // namespace sphb

using namespace sphb;

extern "C" int sphb_box_init(const sphb_engine *e, int cur, void *stream)
{
    int rc = check_engine(e, cur);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    k_box_reset<<<(e->cfg.num_scenes + 127) / 128, 128, 0, st>>>(*e, 0);
    if (e->num_tiles > 0)
        k_box_accum<<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, 0);
    return launch_status("sphb_box_init");
}

extern "C" int sphb_refresh(const sphb_engine *e, int cur, void *stream)
{
    int rc = check_engine(e, cur);
    if (rc) return rc;
    if (e->num_tiles == 0) return SPHB_OK;
    const bool f32 = e->cfg.precision == SPHB_FP32C;
    if (!e->f.cell || (f32 && (!e->f.geo || !e->f.vel))) return SPHB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int nt = e->num_tiles;
    if (e->cfg.dim == 2) {
        if (f32) k_refresh<2, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur);
        else k_refresh<2, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur);
    } else {
        if (f32) k_refresh<3, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur);
        else k_refresh<3, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur);
    }
    return launch_status("sphb_refresh");
}

// The kernels of one rebin, gated on work.meta[1] when gated.
static void launch_rebin(const sphb_engine *e, int cur, int flags, int gated, cudaStream_t st)
{
    const sphb_config &c = e->cfg;
    // every rebin measures the scene boxes afresh (only a rebin needs them)
    k_box_reset<<<(c.num_scenes + 127) / 128, 128, 0, st>>>(*e, gated);
    if (e->num_tiles > 0) k_box_accum<<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur, gated);
    k_grid_setup<<<1, 1024, 0, st>>>(*e, gated);
    const int nt = e->num_tiles;
    if (nt > 0) k_hash<<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, gated);
    const int nb = bin_scan_blocks(c);
    k_scan_reduce<<<nb, SPHB_SCAN_THREADS, 0, st>>>(*e, gated);
    k_scan_top<<<1, SPHB_SCAN_THREADS, 0, st>>>(*e, nb, gated);
    k_scan_apply<<<nb, SPHB_SCAN_THREADS, 0, st>>>(*e, gated);
    if (nt > 0) {
        k_scatter<<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, gated);
        const int mi = (flags & SPHB_BIN_MOVE_INITIAL) ? 1 : 0;
        if (c.dim == 2 && c.precision == SPHB_FP32C)
            k_reorder<2, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
        else if (c.dim == 2)
            k_reorder<2, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
        else if (c.precision == SPHB_FP32C)
            k_reorder<3, true><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
        else
            k_reorder<3, false><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
        if (gated) {
            if (c.dim == 2) k_copy_back<2><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
            else k_copy_back<3><<<nt, SPHB_ELEM_TILE, 0, st>>>(*e, cur, mi, gated);
        }
    }
}

// A stream of the library's own per device, to capture the body of the
// conditional rebin node into (cudaStreamBeginCaptureToGraph needs a stream
// that is not capturing already); one capture at a time.
static std::mutex g_body_mu;
static cudaStream_t g_body_stream[128];

static int body_stream(cudaStream_t *out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return SPHB_ERR_CUDA;
    if (!g_body_stream[dev] &&
        cudaStreamCreateWithFlags(&g_body_stream[dev], cudaStreamNonBlocking) != cudaSuccess)
        return SPHB_ERR_CUDA;
    *out = g_body_stream[dev];
    return SPHB_OK;
}

static int cuda_fail(const char *what, cudaError_t err)
{
    record_cuda_error(what, err);
    return SPHB_ERR_CUDA;
}

// Captured form of a device-decided rebin: the decision kernel sets a graph
// conditional handle, and the rebin kernels form the body of an IF node, so
// a replay that keeps the lists launches none of them.
static int bin_conditional(const sphb_engine *e, int cur, int flags, cudaStream_t st,
                           cudaGraph_t graph)
{
    cudaError_t err;
    cudaGraphConditionalHandle cond;
    if ((err = cudaGraphConditionalHandleCreate(&cond, graph, 0, cudaGraphCondAssignDefault)))
        return cuda_fail("sphb_bin: conditional handle", err);
    if ((err = launch_pdl(k_bin_decide, dim3(1), dim3(256), st, *e, cond, 1,
                          (flags & SPHB_BIN_STEP_BEGIN) ? 1 : 0)))
        return cuda_fail("sphb_bin: decision", err);
    cudaStreamCaptureStatus cs;
    unsigned long long id;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    if ((err = cudaStreamGetCaptureInfo(st, &cs, &id, &graph, &deps, &ndeps)))
        return cuda_fail("sphb_bin: capture info", err);
    // (the union inside has no default constructor: zeroed storage)
    alignas(cudaGraphNodeParams) unsigned char pbuf[sizeof(cudaGraphNodeParams)];
    memset(pbuf, 0, sizeof(pbuf));
    cudaGraphNodeParams &p = *reinterpret_cast<cudaGraphNodeParams *>(pbuf);
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if ((err = cudaGraphAddNode(&node, graph, deps, ndeps, &p)))
        return cuda_fail("sphb_bin: conditional node", err);
    cudaGraph_t body = p.conditional.phGraph_out[0];
    {
        std::lock_guard<std::mutex> lock(g_body_mu);
        cudaStream_t bs;
        if (body_stream(&bs)) return cuda_fail("sphb_bin: body stream", cudaGetLastError());
        if ((err = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeRelaxed)))
            return cuda_fail("sphb_bin: body capture", err);
        launch_rebin(e, cur, flags, 1, bs);
        const cudaError_t lerr = cudaGetLastError();
        cudaGraph_t done;
        err = cudaStreamEndCapture(bs, &done);
        if (lerr) return cuda_fail("sphb_bin: body launch", lerr);
        if (err) return cuda_fail("sphb_bin: body capture end", err);
    }
    if ((err = cudaStreamUpdateCaptureDependencies(st, &node, 1,
                                                   cudaStreamSetCaptureDependencies)))
        return cuda_fail("sphb_bin: capture dependencies", err);
    return SPHB_OK;
}

extern "C" int sphb_bin(const sphb_engine *e, int cur, int flags, void *stream)
{
    int rc = check_engine(e, cur);
    if (rc) return rc;
    if (flags & ~(SPHB_BIN_MOVE_INITIAL | SPHB_BIN_BOX | SPHB_BIN_IF_NEEDED |
                  SPHB_BIN_STEP_BEGIN))
        return SPHB_ERR_ARG;
    if ((flags & SPHB_BIN_STEP_BEGIN) && !(flags & SPHB_BIN_IF_NEEDED)) return SPHB_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int gated = (flags & SPHB_BIN_IF_NEEDED) ? 1 : 0;
    if (!gated) {
        launch_rebin(e, cur, flags, 0, st);
        return launch_status("sphb_bin");
    }
    // the decision needs the displacements sphb_pc_stage measures from the
    // anchors
    if (!e->f.anchor || !e->f.cell) return SPHB_ERR_ARG;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(st, &cs);
    if (err) return cuda_fail("sphb_bin: capture status", err);
    if (cs == cudaStreamCaptureStatusActive) {
        cudaGraph_t graph;
        unsigned long long id;
        if ((err = cudaStreamGetCaptureInfo(st, &cs, &id, &graph, nullptr, nullptr)))
            return cuda_fail("sphb_bin: capture info", err);
        return bin_conditional(e, cur, flags, st, graph);
    }
    launch_pdl(k_bin_decide, dim3(1), dim3(256), st, *e, cudaGraphConditionalHandle(), 0,
               (flags & SPHB_BIN_STEP_BEGIN) ? 1 : 0);
    launch_rebin(e, cur, flags, 1, st);
    return launch_status("sphb_bin");
}
