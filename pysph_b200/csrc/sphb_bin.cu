// sphb_bin.cu -- cell binning for the particle engine (sm_100a).
//
// One rebin = scene boxes -> per-scene grids -> cell key per particle ->
// counting sort (histogram, two-level scan, scatter) -> gather of the
// particle state into the other buffer in cell order, ranking the members of
// each cell by particle index so the order is canonical, plus the FP32 pair
// records and the anchors (binned positions).  With SPHB_BIN_IF_NEEDED the
// device first decides whether the lists (or, for tiled pair passes, the
// cells) still cover every pair (no particle has moved skin/2 from its
// anchor); when they do, the rebin ends there, and when they do not, the
// gathered state is copied back so it stays in buf[cur].
//
// The whole rebin is one cooperative launch (every block resident, so a
// grid-wide barrier between phases cannot deadlock): decision, boxes, grids,
// hash, scan, scatter, gather, copy back, each a grid-stride loop over tiles
// or scan chunks, separated by a bounded barrier.  A step that keeps its
// cells costs one short launch, and a CUDA graph needs no conditional node.
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

// ------------------------------------------------------- grid barrier --
// polls of the barrier's generation word before giving up (each poll sleeps
// ~100 ns; every block of a cooperative launch is resident, so the barrier
// completes in microseconds)
constexpr long BARRIER_POLLS = 1L << 24;

// Grid-wide barrier of a cooperative launch, two-level so that no counter
// takes more than a few dozen same-address atomics: block b arrives on
// counter b % BARRIER_GROUPS (in the words after the scan's chunk totals,
// bsum[nb + 1 ..]), the last of each group on the top counter, and the last
// of those advances the generation work.meta[7] that every block polls.
// Each counter is reset by its last arriver before the release.  The wait
// is bounded: on the limit it sets SPHB_ST_STAGE_TIMEOUT and goes on.
constexpr int BARRIER_GROUPS = 32;

__device__ __forceinline__ void grid_barrier(const sphb_engine &e, int *cnt)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int *gen = (volatile int *)&e.work.meta[7];
        const int g = *gen;
        const int nb = (int)gridDim.x;
        const int grp = (int)blockIdx.x % BARRIER_GROUPS;
        const int ngrp = nb < BARRIER_GROUPS ? nb : BARRIER_GROUPS;
        const int members = nb / BARRIER_GROUPS + (grp < nb % BARRIER_GROUPS ? 1 : 0);
        __threadfence();
        bool release = false;
        if (atomicAdd(&cnt[grp], 1) == members - 1) {
            cnt[grp] = 0;
            __threadfence();
            if (atomicAdd(&cnt[BARRIER_GROUPS], 1) == ngrp - 1) {
                cnt[BARRIER_GROUPS] = 0;
                release = true;
            }
        }
        if (release) {
            __threadfence();
            atomicAdd(&e.work.meta[7], 1);
        } else {
            long it = 0;
            while (*gen == g) {
                if (++it > BARRIER_POLLS) {
                    flag(e, SPHB_ST_STAGE_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// ---------------------------------------------------------------- boxes --
// Block 0.  No rebin while the particles sit where the last rebin put
// them (work.meta[3] == 2); otherwise rebin unless the lists were recorded
// with the skin at those positions (work.meta[4]) and no particle of any
// scene has moved skin_max / 2 (less a relative 1e-4 for the FP32 rounding
// of the displacement) from its anchor.  max_disp2 restarts either way.
__device__ void decide_block(const sphb_engine &e, int step_begin)
{
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
    }
}

__device__ __forceinline__ void box_reset_scene(const sphb_engine &e, int s)
{
    for (int d = 0; d < 3; ++d) {
        e.sstate[s].box[d] = enc_double(INFINITY);
        e.sstate[s].box[3 + d] = enc_double(-INFINITY);
    }
}

__global__ void k_box_reset(const __grid_constant__ sphb_engine e)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < e.cfg.num_scenes) box_reset_scene(e, s);
}

// The bounding box of a tile's particles into its scene's box (every thread
// of the block calls it).
__device__ __forceinline__ void box_accum_tile(const sphb_engine &e, int cur, const sphb_tile &t)
{
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

__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_box_accum(const __grid_constant__ sphb_engine e, int cur)
{
    box_accum_tile(e, cur, e.tiles[blockIdx.x]);
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
// Block 0 (<= 1024 threads).  Grid of scene s: cells floor(lo/cs)-R .. floor(hi/cs)+R per
// axis (R padding cells, so every stencil row of every particle exists);
// exclusive prefix of A*ncells over scenes gives the scene key bases.
__device__ void grid_setup_block(const sphb_engine &e)
{
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
__device__ __forceinline__ void hash_tile(const sphb_engine &e, int cur, const sphb_tile &t)
{
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

// Chunk b of SPHB_SCAN_CHUNK cells: its count total into bsum[b].
__device__ __forceinline__ void scan_reduce_chunk(const sphb_engine &e, int b)
{
    const int T = e.work.meta[0];
    const long long base = (long long)b * SPHB_SCAN_CHUNK;
    int sum = 0;
    for (long long c = base + threadIdx.x; c < base + SPHB_SCAN_CHUNK && c < T; c += blockDim.x)
        sum += e.work.count[c];
    int total;
    block_excl_scan_int(sum, total);
    if (threadIdx.x == 0) e.work.bsum[b] = total;
}

// One block: the exclusive scan of the nb chunk totals (bsum[nb] = all).
__device__ void scan_top_block(const sphb_engine &e, int nb)
{
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

// Chunk b: start[c] for its cells (ITEMS consecutive cells per thread,
// ITEMS x blockDim.x = SPHB_SCAN_CHUNK), and the counts cleared for the
// next bin.
template <int ITEMS>
__device__ __forceinline__ void scan_apply_chunk(const sphb_engine &e, int b)
{
    const int T = e.work.meta[0];
    const long long base = (long long)b * SPHB_SCAN_CHUNK;
    if (T == 0) {
        if (b == 0 && threadIdx.x == 0) e.work.start[0] = 0;
        return;
    }
    if (base >= T) return;   // block-uniform
    const long long c0 = base + (long long)threadIdx.x * ITEMS;
    int v[ITEMS];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        v[i] = (c0 + i < T) ? e.work.count[c0 + i] : 0;
        sum += v[i];
    }
    int total;
    int run = block_excl_scan_int(sum, total) + e.work.bsum[b];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
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
__device__ __forceinline__ void scatter_tile(const sphb_engine &e, const sphb_tile &t)
{
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
__device__ __forceinline__ void reorder_tile(const sphb_engine &e, int cur, int move_initial,
                                             const sphb_tile &t)
{
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
__device__ __forceinline__ void copy_back_tile(const sphb_engine &e, int cur, int move_initial,
                                               const sphb_tile &t)
{
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


// ---------------------------------------------------------- the rebin --
// One cooperative launch: [decision] -> boxes -> grids -> hash -> scan ->
// scatter -> gather [-> copy back], the phases separated by grid_barrier.
// With SPHB_BIN_IF_NEEDED block 0 decides first and every block returns
// when the cells are kept; the gathered state then goes back to buf[cur].
template <int DIM, bool F32>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_rebin(const __grid_constant__ sphb_engine e, int cur, int flags)
{
    const bool if_needed = (flags & SPHB_BIN_IF_NEEDED) != 0;
    const int mi = (flags & SPHB_BIN_MOVE_INITIAL) ? 1 : 0;
    const int nt = e.num_tiles;
    const int nb = (int)((e.cfg.cell_capacity + SPHB_SCAN_CHUNK - 1) / SPHB_SCAN_CHUNK);
    int *const bar = e.work.bsum + nb + 1;   // the barrier's counters
    if (blockIdx.x == 0) {
        if (if_needed) decide_block(e, (flags & SPHB_BIN_STEP_BEGIN) ? 1 : 0);
        // every rebin measures the scene boxes afresh (only a rebin reads them)
        for (int s = threadIdx.x; s < e.cfg.num_scenes; s += blockDim.x) box_reset_scene(e, s);
    }
    grid_barrier(e, bar);
    if (if_needed && *(volatile int *)&e.work.meta[1] == 0) {   // kept (grid-uniform)
        pdl_trigger();   // the density pass may launch
        return;
    }
    for (int t = blockIdx.x; t < nt; t += gridDim.x) box_accum_tile(e, cur, e.tiles[t]);
    grid_barrier(e, bar);
    if (blockIdx.x == 0) grid_setup_block(e);
    grid_barrier(e, bar);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) hash_tile(e, cur, e.tiles[t]);
    grid_barrier(e, bar);
    for (int b = blockIdx.x; b < nb; b += gridDim.x) scan_reduce_chunk(e, b);
    grid_barrier(e, bar);
    if (blockIdx.x == 0) scan_top_block(e, nb);
    grid_barrier(e, bar);
    for (int b = blockIdx.x; b < nb; b += gridDim.x)
        scan_apply_chunk<SPHB_SCAN_CHUNK / SPHB_ELEM_TILE>(e, b);
    grid_barrier(e, bar);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) scatter_tile(e, e.tiles[t]);
    grid_barrier(e, bar);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) reorder_tile<DIM, F32>(e, cur, mi, e.tiles[t]);
    if (!if_needed) return;
    grid_barrier(e, bar);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) copy_back_tile<DIM>(e, cur, mi, e.tiles[t]);
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
    k_box_reset<<<(e->cfg.num_scenes + 127) / 128, 128, 0, st>>>(*e);
    if (e->num_tiles > 0)
        k_box_accum<<<e->num_tiles, SPHB_ELEM_TILE, 0, st>>>(*e, cur);
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

static int cuda_fail(const char *what, cudaError_t err)
{
    record_cuda_error(what, err);
    return SPHB_ERR_CUDA;
}

// Blocks of one cooperative rebin launch: every block resident at once
// (occupancy x SMs), looked up once per device and instantiation.
template <int DIM, bool F32>
static int rebin_grid(int *out)
{
    static std::mutex mu;
    static int cache[128];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err || dev < 0 || dev >= 128) return cuda_fail("sphb_bin: device", err);
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        int per_sm = 0, sms = 0;
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rebin<DIM, F32>,
                                                                 SPHB_ELEM_TILE, 0)))
            return cuda_fail("sphb_bin: occupancy", err);
        if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)))
            return cuda_fail("sphb_bin: SM count", err);
        if (per_sm < 1 || sms < 1) return cuda_fail("sphb_bin: occupancy", cudaErrorInvalidValue);
        cache[dev] = per_sm * sms;
    }
    *out = cache[dev];
    return SPHB_OK;
}

// Blocks of a launch: about 4 tiles each, between 2 per SM (a kept-cells
// launch costs little more than one small kernel) and every resident block
// (measured on B200 with the 332k-particle dam break: 2 per SM keep the
// cells in 2 us over a plain launch against 4 us at 3 per SM, while a full
// rebin takes 88 us at 3 per SM and 94 us at 2)
template <int DIM, bool F32>
static int launch_rebin_t(const sphb_engine *e, int cur, int flags, cudaStream_t st)
{
    int resident = 0, sms = 0, dev = 0;
    int rc = rebin_grid<DIM, F32>(&resident);
    if (rc) return rc;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        sms = 1;
    int blocks = (e->num_tiles + 3) / 4;
    if (blocks < 2 * sms) blocks = 2 * sms;
    if (blocks > resident) blocks = resident;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(SPHB_ELEM_TILE);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t err = cudaLaunchKernelEx(&cfg, k_rebin<DIM, F32>, *e, cur, flags);
    if (err) return cuda_fail("sphb_bin: cooperative launch", err);
    return SPHB_OK;
}

static int launch_rebin(const sphb_engine *e, int cur, int flags, cudaStream_t st)
{
    const sphb_config &c = e->cfg;
    if (c.dim == 2 && c.precision == SPHB_FP32C) return launch_rebin_t<2, true>(e, cur, flags, st);
    if (c.dim == 2) return launch_rebin_t<2, false>(e, cur, flags, st);
    if (c.precision == SPHB_FP32C) return launch_rebin_t<3, true>(e, cur, flags, st);
    return launch_rebin_t<3, false>(e, cur, flags, st);
}

extern "C" int sphb_bin(const sphb_engine *e, int cur, int flags, void *stream)
{
    int rc = check_engine(e, cur);
    if (rc) return rc;
    if (flags & ~(SPHB_BIN_MOVE_INITIAL | SPHB_BIN_BOX | SPHB_BIN_IF_NEEDED |
                  SPHB_BIN_STEP_BEGIN))
        return SPHB_ERR_ARG;
    if ((flags & SPHB_BIN_STEP_BEGIN) && !(flags & SPHB_BIN_IF_NEEDED)) return SPHB_ERR_ARG;
    // the decision needs the displacements the stages measure from the
    // anchors
    if ((flags & SPHB_BIN_IF_NEEDED) && (!e->f.anchor || !e->f.cell)) return SPHB_ERR_ARG;
    if ((rc = launch_rebin(e, cur, flags, (cudaStream_t)stream))) return rc;
    return launch_status("sphb_bin");
}
