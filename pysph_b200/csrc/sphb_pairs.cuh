// sphb_pairs.cuh -- neighbour traversal for the pair kernels.
//
// Cells are keyed row-major with x fastest, so the 2R+1 cells of one stencil
// row (cx-R .. cx+R at fixed y, z) hold one contiguous particle range
// [start[row-R], start[row+R+1]).  A dest particle visits (2R+1)^(DIM-1) such
// ranges instead of (2R+1)^DIM cells; the 2R inner boundaries tell which
// cell (x offset o) a candidate sits in, which the FP32 path needs because
// its positions are stored relative to their own cell origin.

#pragma once

#include "sphb_common.cuh"

namespace sphb {

// A dest cell must lie at least R cells inside its grid (the grid is padded
// by R cells), so every stencil row exists.  Anything else means the binning
// state is corrupt (the status word says why); the particle is skipped.
template <int DIM, int R>
__device__ __forceinline__ bool dest_cell_ok(int cx, int cy, int cz, const int *n)
{
    bool ok = cx >= R && cx < n[0] - R && cy >= R && cy < n[1] - R;
    if (DIM == 3) ok = ok && cz >= R && cz < n[2] - R;
    return ok;
}

// Which stencil cells a dest particle can reach.  Right after a bin every
// particle lies inside its own cell, and nothing a pass accepts (list
// radius with the skin, larger h of a variable-h pair) lies beyond R cell
// widths: the cell size is radius_scale max h (1 + skin margin) / R.  A
// cell whose box is R cell widths or more from the dest's position then
// holds no candidate that can pass the predicate, so it is not visited.
// The test is in cell units with a 1e-3 margin (the dest's offset inside its
// cell is rounded to float).  `on` is false whenever the particles may have
// moved since the bin; every cell of the stencil is visited then.  3D only
// (measured on B200: the density pass of a 128^3 lattice searching cells
// 2.34 -> 2.25 ms; in 2D, with one cell of reach, it trims little and the
// 332k-particle dam break's recording pass went 83 -> 86 us).
struct CellTrim {
    bool on = false;
    float f[3] = {0.f, 0.f, 0.f};   // dest position in its cell, in cell widths
};

// distance (cell widths) from offset f to the cells [d, d + 1) of a row
__device__ __forceinline__ float row_gap(float f, int d)
{
    return fmaxf(0.f, fmaxf((float)d - f, f - (float)(d + 1)));
}

// The trim of a dest whose FP32 record holds its offset from its cell origin.
__device__ __forceinline__ CellTrim cell_trim_rel(const sphb_engine &e, float xr, float yr,
                                                  float zr, float cs)
{
    CellTrim t;
    t.on = e.work.meta[3] == 2;
    const float ic = 1.0f / cs;
    t.f[0] = xr * ic;
    t.f[1] = yr * ic;
    t.f[2] = zr * ic;
    return t;
}

// The trim of a dest at FP64 position (x, y, z) in local cell (cx, cy, cz).
template <int DIM>
__device__ __forceinline__ CellTrim cell_trim_abs(const sphb_engine &e,
                                                  const sphb_scene_state &st, double cs,
                                                  double x, double y, double z, int cx, int cy,
                                                  int cz)
{
    CellTrim t;
    t.on = e.work.meta[3] == 2;
    t.f[0] = (float)((x - (double)(st.lo[0] + cx) * cs) / cs);
    t.f[1] = (float)((y - (double)(st.lo[1] + cy) * cs) / cs);
    t.f[2] = DIM == 3 ? (float)((z - (double)(st.lo[2] + cz) * cs) / cs) : 0.f;
    return t;
}

// Visits every candidate j of the stencil rows (or of the cells `trim`
// keeps), in the order of the full stencil; returns false (visiting nothing
// more) if a row range falls outside [0, num_particles).
template <int DIM, int R, int LANES, typename F>
__device__ __forceinline__ bool for_each_candidate(
    const int *__restrict__ start, int num_arrays, uint32_t src_mask,
    int cell_base, int ncells, const int *n, int cx, int cy, int cz, int lane,
    int num_particles, unsigned *status, const CellTrim &trim, F &&f)
{
    // one loop over the whole row range in 3D (cells of ~2.6 particles: the
    // per-cell loops of a warp diverge) and with cells of half the reach
    // (R = 2, ~2.3 particles a cell in 2D), one per cell in 2D with cells of
    // the whole reach (measured: 3D density search 2.53 -> 2.33 ms; the
    // dam break's recording pass 86.4 -> 83.1 us at R = 2, 83 -> 88 us the
    // other way at R = 1)
    constexpr bool SPAN = LANES > 1 || DIM == 3 || R == 2;
    constexpr float RC2 = (R + 1e-3f) * (R + 1e-3f);
    if (!dest_cell_ok<DIM, R>(cx, cy, cz, n)) {
        atomicOr(status, (unsigned)SPHB_ST_BAD_INDEX);
        return false;
    }
    for (int b = 0; b < num_arrays; ++b) {
        if (!((src_mask >> b) & 1u)) continue;
        const int base = cell_base + b * ncells;
#pragma unroll 1
        for (int dz = (DIM == 3 ? -R : 0); dz <= (DIM == 3 ? R : 0); ++dz) {
#pragma unroll 1
            for (int dy = -R; dy <= R; ++dy) {
                int clo = -R, chi = R;   // x offsets of the cells to visit
                if (DIM == 3 && trim.on) {
                    const float ey = row_gap(trim.f[1], dy);
                    const float ez = DIM == 3 ? row_gap(trim.f[2], dz) : 0.f;
                    const float rem = RC2 - ey * ey - ez * ez;
                    if (rem < 0.f) continue;
                    const float ex = sqrtf(rem);
                    clo = max(-R, (int)floorf(trim.f[0] - ex));
                    chi = min(R, (int)floorf(trim.f[0] + ex));
                    if (clo > chi) continue;
                }
                const int row = base + ((cz + dz) * n[1] + (cy + dy)) * n[0] + cx;
                int bd[2 * R + 2];
#pragma unroll
                for (int i = 0; i < 2 * R + 2; ++i) bd[i] = __ldg(start + row - R + i);
                if (bd[0] < 0 || bd[2 * R + 1] > num_particles || bd[0] > bd[2 * R + 1]) {
                    atomicOr(status, (unsigned)SPHB_ST_BAD_INDEX);
                    return false;
                }
                if (!SPAN) {
                    // one loop per cell: the x offset is loop-invariant
#pragma unroll
                    for (int c = 0; c <= 2 * R; ++c)
                        if (c - R >= clo && c - R <= chi)
                            for (int j = bd[c]; j < bd[c + 1]; ++j) f(j, c - R, dy, dz);
                } else {
                    int js = bd[0], je = bd[2 * R + 1];
#pragma unroll
                    for (int i = 0; i <= 2 * R + 1; ++i) {
                        if (i == clo + R) js = bd[i];
                        if (i == chi + R + 1) je = bd[i];
                    }
                    for (int j = js + lane; j < je; j += LANES) {
                        int o = -R;
#pragma unroll
                        for (int i = 1; i <= 2 * R; ++i) o += (j >= bd[i]) ? 1 : 0;
                        f(j, o, dy, dz);
                    }
                }
            }
        }
    }
    return true;
}

// Neighbour-list entries: index plus the candidate's cell offsets.
template <int DIM>
__device__ __forceinline__ uint32_t nbr_pack(int j, int o, int dy, int dz)
{
    constexpr int B = DIM == 2 ? SPHB_NBR_IDX_BITS_2D : SPHB_NBR_IDX_BITS_3D;
    uint32_t v = (uint32_t)j | ((uint32_t)(o + 2) << B) | ((uint32_t)(dy + 2) << (B + 3));
    if constexpr (DIM == 3) v |= (uint32_t)(dz + 2) << (B + 6);
    return v;
}

// Each lane's list is padded with nbr_pad entries to a multiple of
// SPHB_LIST_PAD slots, so the FP32 list loops load whole batches without a
// per-entry bound.  A pad entry is the dest itself five cells away along x
// (offset field 7): its squared distance exceeds every support radius
// (cells are at least half the largest reach wide), so every pass rejects
// it with the ordinary neighbour test.
constexpr int SPHB_LIST_PAD = 4;

template <int DIM>
__device__ __forceinline__ uint32_t nbr_pad(int k)
{
    constexpr int B = DIM == 2 ? SPHB_NBR_IDX_BITS_2D : SPHB_NBR_IDX_BITS_3D;
    return (uint32_t)k | (7u << B);
}

template <int DIM>
__device__ __forceinline__ void nbr_unpack(uint32_t v, int &j, int &o, int &dy, int &dz)
{
    constexpr int B = DIM == 2 ? SPHB_NBR_IDX_BITS_2D : SPHB_NBR_IDX_BITS_3D;
    j = (int)(v & ((1u << B) - 1u));
    o = (int)((v >> B) & 7u) - 2;
    dy = (int)((v >> (B + 3)) & 7u) - 2;
    dz = DIM == 3 ? (int)((v >> (B + 6)) & 7u) - 2 : 0;
}

// Sources a dest array's neighbour lists are recorded over: every source
// of every pair function on it (SPHRho, MomentumEquation, SPHDensityRate,
// XSPHCorrection), so one list serves all of them.
__device__ __forceinline__ uint32_t list_sources(const sphb_config &c, int a)
{
    return c.rho_src[a] | c.mom_src[a] | c.rate_src[a] | c.xsph_src[a];
}

// Array index of engine position j inside scene s (segments of a scene are
// consecutive: seg_offset[s*A + b] is where array b starts).
struct SegBounds {
    int b1, b2, b3;   // starts of arrays 1, 2, 3 (INT_MAX when absent)
    __device__ __forceinline__ SegBounds(const sphb_engine &e, int s)
    {
        const int A = e.cfg.num_arrays;
        const int *so = e.seg_offset + s * A;
        b1 = A > 1 ? so[1] : 0x7fffffff;
        b2 = A > 2 ? so[2] : 0x7fffffff;
        b3 = A > 3 ? so[3] : 0x7fffffff;
    }
    __device__ __forceinline__ int array_of(int j) const
    {
        return (j >= b1) + (j >= b2) + (j >= b3);
    }
};

// A list entry unpacked, with the cell offsets as floats.  The 3-bit fields
// become floats through the exponent of 2^23 (exact, no conversion
// instruction): float(0x4B000000 | b) = 2^23 + b.
struct EntryF {
    int j;
    float o, dy, dz;
};

template <int DIM>
__device__ __forceinline__ EntryF entry_unpack_f(uint32_t v)
{
    constexpr int B = DIM == 2 ? SPHB_NBR_IDX_BITS_2D : SPHB_NBR_IDX_BITS_3D;
    constexpr float BIAS = 8388608.0f + 2.0f;
    EntryF r;
    r.j = (int)(v & ((1u << B) - 1u));
    r.o = __int_as_float(0x4B000000 | (int)((v >> B) & 7u)) - BIAS;
    r.dy = __int_as_float(0x4B000000 | (int)((v >> (B + 3)) & 7u)) - BIAS;
    r.dz = DIM == 3 ? __int_as_float(0x4B000000 | (int)((v >> (B + 6)) & 7u)) - BIAS : 0.f;
    return r;
}

// Entries of dest k this lane owns (-1 when some lane's list overflowed),
// or -1 when the lists are not to be used.
template <int LANES>
__device__ __forceinline__ int list_count(const sphb_engine &e, bool use_list, int k, int lane)
{
    if (!use_list) return -1;
    const int N = e.cfg.num_particles;
    int mine = 0;
    bool ok = true;
#pragma unroll
    for (int l = 0; l < LANES; ++l) {
        const int c = __ldg(e.f.nbr_cnt + (size_t)l * N + k);
        ok = ok && c >= 0;
        if (l == lane) mine = c;
    }
    return ok ? mine : -1;
}

// use(load(entry)) over the cnt list entries of (k, lane), in batches of
// U: a batch's U neighbour records are loaded before any is used, and the
// next batch's list entries are fetched before this batch's records, so a
// thread keeps U record gathers and U list loads in flight instead of one
// dependent chain.  The last batch reads the list's pad entries (U divides
// SPHB_LIST_PAD), which the neighbour test rejects.
template <int DIM, int LANES, int U, typename Load, typename Use>
__device__ __forceinline__ void list_loop(const sphb_engine &e, int k, int lane, int cnt,
                                          Load &&load, Use &&use)
{
    static_assert(SPHB_LIST_PAD % U == 0, "batches must end inside the padding");
    const int N = e.cfg.num_particles;
    const uint32_t *__restrict__ p = e.f.nbr + (size_t)lane * N + k;
    const size_t stride = (size_t)LANES * N;
    const int nb = (cnt + U - 1) / U;
    auto fetch = [&](int b, uint32_t *v) {
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = __ldg(p + (size_t)(b * U + u) * stride);
    };
    uint32_t v[U];
    if (nb > 0) fetch(0, v);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        uint32_t w[U];
        if (b + 1 < nb) fetch(b + 1, w);
        decltype(load(EntryF{})) r[U];
#pragma unroll
        for (int u = 0; u < U; ++u) r[u] = load(entry_unpack_f<DIM>(v[u]));
#pragma unroll
        for (int u = 0; u < U; ++u) use(r[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = w[u];
    }
}

// The pairs of dest k: its list from the last density pass when use_list
// and every lane's list is complete, else the cell search.
template <int DIM, int R, int LANES, typename F>
__device__ __forceinline__ void traverse(const sphb_engine &e, bool use_list, int k, int lane,
                                         const int *__restrict__ start, int num_arrays,
                                         uint32_t src_mask, int cell_base, int ncells,
                                         const int *n, int cx, int cy, int cz,
                                         const CellTrim &trim, F &&f)
{
    const int N = e.cfg.num_particles;
    if (use_list) {
        bool ok = true;
        int mine = 0;
#pragma unroll
        for (int l = 0; l < LANES; ++l) {
            const int c = __ldg(e.f.nbr_cnt + (size_t)l * N + k);
            ok = ok && c >= 0;
            if (l == lane) mine = c;
        }
        if (ok) {
            const uint32_t *__restrict__ nbr = e.f.nbr;
            for (int c = 0; c < mine; ++c) {
                int j, o, dy, dz;
                nbr_unpack<DIM>(__ldg(nbr + (size_t)(lane + LANES * c) * N + k), j, o, dy, dz);
                if (j < N) f(j, o, dy, dz);
                else atomicOr(e.work.status, (unsigned)SPHB_ST_BAD_INDEX);
            }
            return;
        }
    }
    for_each_candidate<DIM, R, LANES>(start, num_arrays, src_mask, cell_base, ncells, n, cx, cy,
                                      cz, lane, N, e.work.status, trim, f);
}

// Squared distance with the reference's rounding (no FMA contraction):
// cPoint_distance2 (S/base/point.pxd:35-37).
template <int DIM>
__device__ __forceinline__ double dist2_ref(double dx, double dy, double dz)
{
    double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    if (DIM == 3) d2 = __dadd_rn(d2, __dmul_rn(dz, dz));
    return d2;
}

}  // namespace sphb
