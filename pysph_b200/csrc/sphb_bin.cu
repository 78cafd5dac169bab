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
// polls of the barrier word before giving up (every block of a cooperative
// launch is resident, so the barrier completes in microseconds)
constexpr long BARRIER_POLLS = 1L << 22;

// Grid-wide barrier of a cooperative launch on one word (the first word
// after the scan's chunk totals, bsum[nb + 1]).  Each block adds 1 to it,
// except block 0, which adds 2^31 - (blocks - 1): the word's top bit flips
// exactly when the last block has arrived, and its low bits are back where
// they were, so the word needs no reset between barriers or launches.  The
// wait is bounded: on the limit it sets SPHB_ST_STAGE_TIMEOUT and goes on.
__device__ __forceinline__ void grid_barrier(const sphb_engine &e, int *word_)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned *word = (unsigned *)word_;
        const unsigned nb = gridDim.x;
        const unsigned add = blockIdx.x == 0 ? 0x80000000u - (nb - 1u) : 1u;
        __threadfence();
        const unsigned old = atomicAdd(word, add);
        long it = 0;
        while (((old ^ *(volatile unsigned *)word) & 0x80000000u) == 0u) {
            if (++it > BARRIER_POLLS) {
                flag(e, SPHB_ST_STAGE_TIMEOUT);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
}

// ------------------------------------------------------------ decision --
// No rebin while the particles sit where the last rebin put them
// (work.meta[3] == 2); otherwise rebin unless the lists were recorded with
// the skin at those positions (work.meta[4]) and no particle of any scene
// has moved skin_max / 2 (less a relative 1e-4 for the FP32 rounding of the
// displacement) from its anchor.  Every block reads the same words, written
// by earlier launches, and reaches the same decision (block-uniform), so a
// launch that keeps the cells needs no grid barrier; *lists tells whether
// the kept lists hold every pair.
__device__ bool decide_keep(const sphb_engine &e, bool *lists)
{
    __shared__ int s_far;
    if (threadIdx.x == 0) s_far = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < e.cfg.num_scenes; s += blockDim.x) {
        const double d2 = __longlong_as_double((long long)e.sstate[s].max_disp2);
        const double lim = 0.5 * e.scene[s].skin_max * (1.0 - 1e-4);
        if (!(d2 < lim * lim)) s_far = 1;
    }
    __syncthreads();
    const bool at_anchor = e.work.meta[3] == 2;
    // host-written state nobody has measured: no trusting the lists
    *lists = e.work.meta[4] == 1 && e.work.meta[5] == 0;
    return at_anchor || (*lists && !s_far);
}

// One block, once every block has read the decision's inputs: the step
// prologue when asked, max_disp2 restarting, and the decision published
// (meta[1] = 1 when it rebins, meta[2] = 1 when it kept the lists).
__device__ void decide_commit(const sphb_engine &e, int step_begin, bool keep, bool lists)
{
    for (int s = threadIdx.x; s < e.cfg.num_scenes; s += blockDim.x) {
        if (step_begin) step_begin_scene(e, s);
        e.sstate[s].max_disp2 = 0ull;
    }
    if (threadIdx.x == 0) {
        e.work.meta[1] = keep ? 0 : 1;
        e.work.meta[2] = (keep && lists) ? 1 : 0;
        if (!keep) e.work.pairs[3] += 1ull;   // rebins decided on the device
    }
}

// ---------------------------------------------------------------- boxes --
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

// ------------------------------------------------------- block work runs --
// The rebin's per-particle phases give each block a contiguous run of tiles
// and walk it RU tiles at a time, issuing every load of the RU particles a
// thread owns before any of them is used.  The launch keeps only 2-3 blocks
// per SM (a kept-cells launch must stay cheap), so with one particle per
// thread in flight the phases waited one memory latency per tile; this way
// they wait one per RU tiles.
constexpr int RU = 4;
// tiles at a time of the phases that carry little per particle (boxes,
// keys, scatter)
constexpr int RU8 = 8;

__device__ __forceinline__ void block_tile_run(int nt, int &t0, int &t1)
{
    const long long G = gridDim.x, b = blockIdx.x;
    t0 = (int)(b * nt / G);
    t1 = (int)((b + 1) * nt / G);
}

// The particles of tiles [t, t + U) this thread owns (-1: none) and their
// segments.
template <int U>
__device__ __forceinline__ void run_particles(const sphb_engine &e, int t, int t1, int *kk,
                                              int *seg)
{
#pragma unroll
    for (int u = 0; u < U; ++u) {
        kk[u] = -1;
        seg[u] = -1;
        if (t + u < t1) {
            const sphb_tile tl = e.tiles[t + u];
            seg[u] = tl.seg;
            const int k = tl.begin + (int)threadIdx.x;
            if (k < tl.end) kk[u] = k;
        }
    }
}

// ---------------------------------------------------------------- boxes --
// This block's minima / maxima into scene s's box (a block-uniform call),
// then the partials restart.
__device__ __forceinline__ void box_flush(const sphb_engine &e, int s, int dim, double *lo,
                                          double *hi)
{
    __shared__ double sh[SPHB_ELEM_TILE / 32][6];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = warp_reduce(lo[d], OpMin());
        hi[d] = warp_reduce(hi[d], OpMax());
    }
    if (lane == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sh[w][d] = lo[d];
            sh[w][3 + d] = hi[d];
        }
    }
    __syncthreads();
    // one thread per bound: its value over the warps, then one fire-and-
    // forget atomic (the encoded doubles order like the doubles)
    const int t = threadIdx.x;
    if (t < 2 * dim) {
        const bool is_lo = t < dim;
        const int c = is_lo ? t : 3 + (t - dim);
        double v = sh[0][c];
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i)
            v = is_lo ? fmin(v, sh[i][c]) : fmax(v, sh[i][c]);
        if (is_lo && v < INFINITY) atomicMin(&e.sstate[s].box[c], enc_double(v));
        if (!is_lo && v > -INFINITY) atomicMax(&e.sstate[s].box[c], enc_double(v));
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = INFINITY;
        hi[d] = -INFINITY;
    }
}

// The scene boxes from the block's run of tiles: partials in registers,
// published whenever the run passes into another scene and at its end.
template <int DIM>
__device__ void box_accum_run(const sphb_engine &e, int cur, int t0, int t1)
{
    if (t0 >= t1) return;   // block-uniform
    const int A = e.cfg.num_arrays;
    const sphb_buffers &B = e.buf[cur];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int s_cur = e.tiles[t0].seg / A;
    for (int t = t0; t < t1; t += RU8) {
        int kk[RU8], seg[RU8];
        run_particles<RU8>(e, t, t1, kk, seg);
        double px[RU8], py[RU8], pz[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            px[u] = py[u] = pz[u] = 0.0;
            if (kk[u] >= 0) {
                px[u] = B.x[kk[u]];
                py[u] = B.y[kk[u]];
                if (DIM == 3) pz[u] = B.z[kk[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            if (seg[u] < 0) break;   // block-uniform
            const int su = seg[u] / A;
            if (su != s_cur) {
                box_flush(e, s_cur, DIM, lo, hi);
                s_cur = su;
            }
            if (kk[u] >= 0 && isfinite(px[u]) && isfinite(py[u]) && isfinite(pz[u])) {
                lo[0] = fmin(lo[0], px[u]);
                hi[0] = fmax(hi[0], px[u]);
                lo[1] = fmin(lo[1], py[u]);
                hi[1] = fmax(hi[1], py[u]);
                if (DIM == 3) {
                    lo[2] = fmin(lo[2], pz[u]);
                    hi[2] = fmax(hi[2], pz[u]);
                }
            }
        }
    }
    box_flush(e, s_cur, DIM, lo, hi);
}

// ----------------------------------------------------------------- hash --
// Global cell key of a particle of segment seg at (x, y, z), or -1 (status
// flagged) for a non-finite position or one outside its scene's grid.
template <int DIM>
__device__ __forceinline__ long long cell_key(const sphb_engine &e, int seg, double x, double y,
                                              double z)
{
    const int A = e.cfg.num_arrays;
    const int s = seg / A, a = seg - s * A;
    const sphb_scene_state &st = e.sstate[s];
    const double cs = e.scene[s].cell_size;
    const double p[3] = {x, y, z};
    int c[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        if (!isfinite(p[d])) {
            flag(e, SPHB_ST_NONFINITE_POS);
            return -1;
        }
        // floor(x / cs) exactly as find_cell_id (S/base/cell.pyx:44-84)
        const double f = floor(p[d] / cs) - (double)st.lo[d];
        if (!(f >= 0.0) || !(f < (double)st.n[d])) {
            flag(e, SPHB_ST_OUT_OF_GRID);
            return -1;
        }
        c[d] = (int)f;
    }
    const int local = (c[2] * st.n[1] + c[1]) * st.n[0] + c[0];
    const long long key = (long long)st.cell_base + (long long)a * st.ncells + local;
    if (local >= st.ncells || key >= (long long)e.work.meta[0]) {
        flag(e, SPHB_ST_OUT_OF_GRID);
        return -1;
    }
    return key;
}

// Keys and the cell histogram: RU positions loaded, RU keys, RU atomics in
// flight, then the stores.
template <int DIM>
__device__ void hash_run(const sphb_engine &e, int cur, int t0, int t1)
{
    const sphb_buffers &B = e.buf[cur];
    for (int t = t0; t < t1; t += RU8) {
        int kk[RU8], seg[RU8];
        run_particles<RU8>(e, t, t1, kk, seg);
        double px[RU8], py[RU8], pz[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            px[u] = py[u] = pz[u] = 0.0;
            if (kk[u] >= 0) {
                px[u] = B.x[kk[u]];
                py[u] = B.y[kk[u]];
                if (DIM == 3) pz[u] = B.z[kk[u]];
            }
        }
        long long key[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u)
            key[u] = kk[u] >= 0 ? cell_key<DIM>(e, seg[u], px[u], py[u], pz[u]) : -1;
        int slot[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u) slot[u] = key[u] >= 0 ? atomicAdd(&e.work.count[key[u]], 1) : 0;
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            if (kk[u] < 0) continue;
            if (key[u] >= 0) e.work.slot[kk[u]] = slot[u];
            e.work.key[kk[u]] = (int)key[u];
        }
    }
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

// Cells per thread in a scan chunk (256 threads x 16 = SPHB_SCAN_CHUNK).
constexpr int SCAN_ITEMS = SPHB_SCAN_CHUNK / SPHB_ELEM_TILE;
static_assert(SCAN_ITEMS % 4 == 0, "scan items come in int4 groups");

// The counts of the thread's SCAN_ITEMS consecutive cells from c0 (zero past
// T): int4 loads when the table is 16-byte aligned, all issued before use.
__device__ __forceinline__ void scan_load(const int *count, long long c0, long long T, bool vec,
                                          int *v)
{
    if (vec && c0 + SCAN_ITEMS <= T) {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS / 4; ++i) {
            const int4 q = ((const int4 *)(count + c0))[i];
            v[4 * i] = q.x;
            v[4 * i + 1] = q.y;
            v[4 * i + 2] = q.z;
            v[4 * i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i) v[i] = (c0 + i < T) ? count[c0 + i] : 0;
    }
}

// Chunk b of the T used cells: its count total into bsum[b].
__device__ __forceinline__ void scan_reduce_chunk(const sphb_engine &e, int b, long long T,
                                                  bool vec)
{
    const long long c0 = (long long)b * SPHB_SCAN_CHUNK + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    scan_load(e.work.count, c0, T, vec, v);
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) sum += v[i];
    const int total = block_reduce(sum, OpSumInt(), 0);
    if (threadIdx.x == 0) e.work.bsum[b] = total;
}

// Chunk b: start[c] for its cells, start[T] after the last, and the counts
// cleared for the next bin.  The chunk's offset is the sum of the totals
// of the chunks before it, which every block adds up itself (a few
// thousand L2-resident words at most), so no phase scans the totals.
__device__ __forceinline__ void scan_apply_chunk(const sphb_engine &e, int b, long long T,
                                                 bool vec)
{
    int pre = 0;
    for (int i = threadIdx.x; i < b; i += blockDim.x) pre += e.work.bsum[i];
    __shared__ int s_pre;
    pre = block_reduce(pre, OpSumInt(), 0);
    if (threadIdx.x == 0) s_pre = pre;
    const long long c0 = (long long)b * SPHB_SCAN_CHUNK + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    scan_load(e.work.count, c0, T, vec, v);
    int sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) sum += v[i];
    int total;
    int run = block_excl_scan_int(sum, total);   // (its barriers publish s_pre)
    run += s_pre;
    int st[SCAN_ITEMS];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        st[i] = run;
        run += v[i];
    }
    if (vec && c0 + SCAN_ITEMS <= T) {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS / 4; ++i) {
            ((int4 *)(e.work.start + c0))[i] =
                make_int4(st[4 * i], st[4 * i + 1], st[4 * i + 2], st[4 * i + 3]);
            ((int4 *)(e.work.count + c0))[i] = make_int4(0, 0, 0, 0);
        }
    } else {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i) {
            if (c0 + i < T) {
                e.work.start[c0 + i] = st[i];
                e.work.count[c0 + i] = 0;
            }
        }
    }
    if (c0 <= T - 1 && T - 1 < c0 + SCAN_ITEMS) e.work.start[T] = run;
}

// -------------------------------------------------------------- scatter --
__device__ void scatter_run(const sphb_engine &e, int t0, int t1)
{
    const int N = e.cfg.num_particles;
    for (int t = t0; t < t1; t += RU8) {
        int kk[RU8], seg[RU8];
        run_particles<RU8>(e, t, t1, kk, seg);
        int key[RU8], sl[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            key[u] = -1;
            sl[u] = 0;
            if (kk[u] >= 0) {
                key[u] = e.work.key[kk[u]];
                sl[u] = e.work.slot[kk[u]];
            }
        }
        int pos[RU8];
#pragma unroll
        for (int u = 0; u < RU8; ++u) pos[u] = key[u] >= 0 ? e.work.start[key[u]] + sl[u] : -1;
#pragma unroll
        for (int u = 0; u < RU8; ++u) {
            if (kk[u] < 0 || key[u] < 0) continue;
            if (pos[u] < 0 || pos[u] >= N) flag(e, SPHB_ST_BAD_INDEX);
            else e.work.perm[pos[u]] = kk[u];
        }
    }
}

// -------------------------------------------------------------- reorder --
// The state one particle carries through a rebin.
template <int DIM>
struct Carried {
    double x, y, z, u, v, w, m, h, rho, rho0;
    double x0, y0, z0, u0, v0, w0;
    int idx, tag;
};

// Every load of particle p's state, issued together.
template <int DIM>
__device__ __forceinline__ Carried<DIM> carried_load(const sphb_buffers &S, int p, int mi)
{
    Carried<DIM> c;
    c.x = S.x[p];
    c.y = S.y[p];
    c.u = S.u[p];
    c.v = S.v[p];
    c.m = S.m[p];
    c.h = S.h[p];
    c.idx = S.idx[p];
    c.tag = S.tag[p];
    c.z = c.w = c.rho = c.rho0 = c.z0 = c.w0 = 0.0;
    c.x0 = c.y0 = c.u0 = c.v0 = 0.0;
    if (S.rho) c.rho = S.rho[p];
    if (mi && S.rho0) c.rho0 = S.rho0[p];
    if (DIM == 3) {
        c.z = S.z[p];
        c.w = S.w[p];
    }
    if (mi) {
        c.x0 = S.x0[p];
        c.y0 = S.y0[p];
        c.u0 = S.u0[p];
        c.v0 = S.v0[p];
        if (DIM == 3) {
            c.z0 = S.z0[p];
            c.w0 = S.w0[p];
        }
    }
    return c;
}

template <int DIM>
__device__ __forceinline__ void carried_store(const sphb_buffers &S, const sphb_buffers &D, int k,
                                              int mi, const Carried<DIM> &c)
{
    D.x[k] = c.x;
    D.y[k] = c.y;
    D.u[k] = c.u;
    D.v[k] = c.v;
    D.m[k] = c.m;
    D.h[k] = c.h;
    D.idx[k] = c.idx;
    D.tag[k] = c.tag;
    if (S.rho && D.rho) D.rho[k] = c.rho;   // integrated density (continuity)
    if (mi && S.rho0 && D.rho0) D.rho0[k] = c.rho0;
    if (DIM == 3) {
        D.z[k] = c.z;
        D.w[k] = c.w;
    }
    if (mi) {
        D.x0[k] = c.x0;
        D.y0[k] = c.y0;
        D.u0[k] = c.u0;
        D.v0[k] = c.v0;
        if (DIM == 3) {
            D.z0[k] = c.z0;
            D.w0[k] = c.w0;
        }
    }
}

// RK4's running sums of particle p to position k (engines that step RK4
// have them; the pointers decide, uniformly over the launch).
template <int DIM>
__device__ __forceinline__ void carry_sums(const sphb_buffers &S, const sphb_buffers &D, int p,
                                           int k)
{
    if (S.kx && D.kx) {
        double q[6];
        q[0] = S.kx[p];
        q[1] = S.ky[p];
        q[2] = S.ku[p];
        q[3] = S.kv[p];
        if (DIM == 3) {
            q[4] = S.kz[p];
            q[5] = S.kw[p];
        }
        D.kx[k] = q[0];
        D.ky[k] = q[1];
        D.ku[k] = q[2];
        D.kv[k] = q[3];
        if (DIM == 3) {
            D.kz[k] = q[4];
            D.kw[k] = q[5];
        }
    }
    if (S.krho && D.krho) D.krho[k] = S.krho[p];
}

// Engine position kk takes particle p = perm[kk] (the scatter put it
// somewhere inside its cell's range [b, e)), ranked among the cell's
// members by their index in the particle array and written to b + rank: the
// order inside a cell is canonical whatever order the atomics handed out the
// slots, and it does not depend on the order the particles had before.  The
// lookups run RU particles abreast (perm, then key and index, then the
// cell's range, then the ranks), the state moves two particles at a time,
// each with all its loads ahead of its stores.
template <int DIM, bool F32>
__device__ void reorder_run(const sphb_engine &e, int cur, int mi, int t0, int t1)
{
    const int A = e.cfg.num_arrays;
    const sphb_buffers &S = e.buf[cur];
    const sphb_buffers &D = e.buf[cur ^ 1];
    const int *__restrict__ sidx = S.idx;
    const int *__restrict__ perm = e.work.perm;
    for (int t = t0; t < t1; t += RU) {
        int kk[RU], seg[RU];
        run_particles<RU>(e, t, t1, kk, seg);
        int p[RU], key[RU], me[RU], cb[RU], ce[RU], k[RU];
#pragma unroll
        for (int u = 0; u < RU; ++u) p[u] = kk[u] >= 0 ? perm[kk[u]] : -1;
#pragma unroll
        for (int u = 0; u < RU; ++u) {
            key[u] = -1;
            me[u] = 0;
            if (kk[u] < 0) continue;
            const int lo = e.seg_offset[seg[u]], hi = e.seg_offset[seg[u] + 1];
            if (p[u] < lo || p[u] >= hi) {
                flag(e, SPHB_ST_BAD_INDEX);
                kk[u] = -1;
                continue;
            }
            key[u] = e.work.key[p[u]];
            me[u] = sidx[p[u]];
        }
#pragma unroll
        for (int u = 0; u < RU; ++u) {
            cb[u] = ce[u] = -1;
            if (kk[u] >= 0 && key[u] >= 0) {
                cb[u] = e.work.start[key[u]];
                ce[u] = e.work.start[key[u] + 1];
            }
        }
#pragma unroll
        for (int u = 0; u < RU; ++u) {
            k[u] = -1;
            if (kk[u] < 0) continue;
            const int lo = e.seg_offset[seg[u]], hi = e.seg_offset[seg[u] + 1];
            if (key[u] < 0 || cb[u] < lo || ce[u] > hi || kk[u] < cb[u] || kk[u] >= ce[u]) {
                flag(e, SPHB_ST_BAD_INDEX);
                continue;
            }
            // canonical order inside a cell: by the particle's index in its
            // array, so the order depends on the positions alone
            int rank = 0;
            for (int i = cb[u]; i < ce[u]; ++i) rank += (sidx[perm[i]] < me[u]) ? 1 : 0;
            k[u] = cb[u] + rank;
        }
#pragma unroll
        for (int u0 = 0; u0 < RU; u0 += 2) {
            Carried<DIM> c[2];
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (k[u0 + j] >= 0) c[j] = carried_load<DIM>(S, p[u0 + j], mi);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int u = u0 + j;
                if (k[u] < 0) continue;
                carried_store<DIM>(S, D, k[u], mi, c[j]);
                if (mi) carry_sums<DIM>(S, D, p[u], k[u]);
                const int s = seg[u] / A, a = seg[u] - s * A;
                const sphb_scene_state &st = e.sstate[s];
                int local = key[u] - st.cell_base - a * st.ncells;
                if (local < 0 || local >= st.ncells) {
                    flag(e, SPHB_ST_BAD_INDEX);
                    local = 0;
                }
                e.f.cell[k[u]] = local;
                if (!F32 && !e.f.anchor) continue;
                const double cs = e.scene[s].cell_size;
                int cx, cy, cz;
                cell_coords(local, st.n, cx, cy, cz);
                // position relative to the origin of the particle's own cell
                const float xr = (float)(c[j].x - (double)(st.lo[0] + cx) * cs);
                const float yr = (float)(c[j].y - (double)(st.lo[1] + cy) * cs);
                const float zr = DIM == 3 ? (float)(c[j].z - (double)(st.lo[2] + cz) * cs) : 0.f;
                if (F32) {
                    // both copies of the records when the force pass steps the state
                    const float4 g = DIM == 2 ? make_float4(xr, yr, (float)c[j].h, (float)c[j].m)
                                              : make_float4(xr, yr, zr, (float)c[j].h);
                    ((float4 *)e.f.geo)[k[u]] = g;
                    if (e.f.geo_next) ((float4 *)e.f.geo_next)[k[u]] = g;
                    if (DIM == 2) {
                        const float2 vv = make_float2((float)c[j].u, (float)c[j].v);
                        ((float2 *)e.f.vel)[k[u]] = vv;
                        if (e.f.vel_next) ((float2 *)e.f.vel_next)[k[u]] = vv;
                    } else {
                        ((float *)e.f.mass)[k[u]] = (float)c[j].m;
                        const float4 vv =
                            make_float4((float)c[j].u, (float)c[j].v, (float)c[j].w, 0.f);
                        ((float4 *)e.f.vel)[k[u]] = vv;
                        if (e.f.vel_next) ((float4 *)e.f.vel_next)[k[u]] = vv;
                    }
                }
                if (e.f.anchor) {
                    if (DIM == 2) ((float2 *)e.f.anchor)[k[u]] = make_float2(xr, yr);
                    else ((float4 *)e.f.anchor)[k[u]] = make_float4(xr, yr, zr, 0.f);
                }
            }
        }
    }
}

// After a rebin decided on the device: the gathered state back into
// buf[cur], same order (the records, anchors and cells already follow it),
// two particles' loads ahead of their stores.
template <int DIM>
__device__ void copy_back_run(const sphb_engine &e, int cur, int mi, int t0, int t1)
{
    const sphb_buffers &S = e.buf[cur ^ 1];
    const sphb_buffers &D = e.buf[cur];
    for (int t = t0; t < t1; t += RU) {
        int kk[RU], seg[RU];
        run_particles<RU>(e, t, t1, kk, seg);
#pragma unroll
        for (int u0 = 0; u0 < RU; u0 += 2) {
            Carried<DIM> c[2];
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (kk[u0 + j] >= 0) c[j] = carried_load<DIM>(S, kk[u0 + j], mi);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (kk[u0 + j] < 0) continue;
                carried_store<DIM>(S, D, kk[u0 + j], mi, c[j]);
                if (mi) carry_sums<DIM>(S, D, kk[u0 + j], kk[u0 + j]);
            }
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
    int *const bar = e.work.bsum + nb + 1;   // the barrier's word
    const int step_begin = (flags & SPHB_BIN_STEP_BEGIN) ? 1 : 0;
    if (if_needed) {
        bool lists;
        if (decide_keep(e, &lists)) {   // block-uniform, the same in every block
            // kept: the last block to arrive (every block has read the
            // inputs by then) commits; nobody waits
            __shared__ int s_last;
            if (threadIdx.x == 0) {
                __threadfence();
                int *arrive = bar + 1;
                s_last = atomicAdd(arrive, 1) == (int)gridDim.x - 1;
                if (s_last) *arrive = 0;
            }
            __syncthreads();
            if (s_last) decide_commit(e, step_begin, true, lists);
            pdl_trigger();   // the density pass may launch
            return;
        }
        grid_barrier(e, bar);   // every block has read the inputs
        if (blockIdx.x == 0) decide_commit(e, step_begin, false, lists);
    }
    // every rebin measures the scene boxes afresh (only a rebin reads them)
    if (blockIdx.x == 0)
        for (int s = threadIdx.x; s < e.cfg.num_scenes; s += blockDim.x) box_reset_scene(e, s);
    grid_barrier(e, bar);
    int t0, t1;
    block_tile_run(nt, t0, t1);
    box_accum_run<DIM>(e, cur, t0, t1);
    grid_barrier(e, bar);
    if (blockIdx.x == 0) grid_setup_block(e);
    grid_barrier(e, bar);
    hash_run<DIM>(e, cur, t0, t1);
    grid_barrier(e, bar);
    // the scan covers the cells the grids use, not the whole capacity
    const long long T = *(volatile int *)&e.work.meta[0];
    const int nbu = (int)((T + SPHB_SCAN_CHUNK - 1) / SPHB_SCAN_CHUNK);
    const bool vec = ((reinterpret_cast<uintptr_t>(e.work.count) |
                       reinterpret_cast<uintptr_t>(e.work.start)) & 15) == 0;
    for (int b = blockIdx.x; b < nbu; b += gridDim.x) scan_reduce_chunk(e, b, T, vec);
    grid_barrier(e, bar);
    if (T == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) e.work.start[0] = 0;
    }
    for (int b = blockIdx.x; b < nbu; b += gridDim.x) scan_apply_chunk(e, b, T, vec);
    grid_barrier(e, bar);
    scatter_run(e, t0, t1);
    grid_barrier(e, bar);
    reorder_run<DIM, F32>(e, cur, mi, t0, t1);
    if (!if_needed) return;
    grid_barrier(e, bar);
    copy_back_run<DIM>(e, cur, mi, t0, t1);
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
// (2 per SM at the rebin's 128 registers).  Measured on B200 with the
// 332k-particle dam break: a kept-cells launch 4.6 us in a graph (a
// one-block kernel 3.1 us), a full rebin 86-92 us; 256 drops (2.9M
// particles) 375 us, of which the gather and the copy back, near the HBM
// rate, are 260 us.
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
