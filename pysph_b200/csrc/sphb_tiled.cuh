// sphb_tiled.cuh -- the pair passes of pair_mode SPHB_PAIRS_TILED (2D
// FP32C): SPHRho + Tait, and MomentumEquation / SPHPressureGradient +
// gravity with the integrator stage in the epilogue, with every neighbour
// record read from shared memory.
//
// Staging.  A block owns the dests [k0, k1) of one pair tile, sorted by
// cell, so their cells run from c_first to c_last in key order (row-major,
// x fastest).  For a source array b and a stencil row offset dy, every
// candidate of every dest lies in the cells c + dy nx + (-R .. R) of its own
// cell c, all inside the key range [c_first + dy nx - R, c_last + dy nx + R]:
// one contiguous particle range [start[..], start[..]) of the sorted order.
// One thread copies each of these (2R+1) x (source arrays) ranges into
// shared memory with 1D bulk copies (cp.async.bulk, completion on an
// mbarrier; this GPU's memory only), while every thread loads its own
// dest.  A block whose ranges do not fit its shared memory (a tile spanning
// many short rows, e.g. a side wall) reads the same records from global
// memory instead, through the same code.
//
// Per dest, two phases over its (2R+1)^2 stencil cells per source array:
//   filter  every candidate's squared distance from shared memory with the
//           cell offset applied to the dest (one subtraction per axis),
//           accepted into a per-thread list in shared memory when within
//           the support radius (1 + 1e-5)^2;
//   math    the accepted entries, each re-tested with the exact predicate
//           and arithmetic of the list passes (r_ab^2 < (radius_scale h_a)^2
//           on ((x_a - x_b) - o cs, (y_a - y_b) - dy cs)), then SPHRho or
//           the momentum terms.
// The filter's cheap test only pre-selects; the exact test decides, so the
// pairs and their order (stencil rows, then cells, then ascending index)
// are those of the list passes.  Separating the two keeps the expensive
// pair arithmetic off the ~75% of candidates that fail the test (in one
// loop, a warp would run it whenever any lane accepts).  The list holds
// TILE_LCAP entries per thread; a dest with more runs the math on each full
// list and continues.
//
// Formulas, sources and outputs are those of k_density and k_force (the
// reference citations are there): SPHRho (S/sph/funcs/density_funcs.pyx:
// 37-73), TaitEquation (S/sph/funcs/eos_funcs.pyx:88-129),
// MomentumEquation / SPHPressureGradient (S/sph/funcs/pressure_funcs.pyx:
// 19-391), GravityForce (S/sph/funcs/external_force.pyx:13-62); the
// neighbour predicate of FixedDestNbrParticleLocator (S/base/nnps.pyx:
// 271-356); the cell-range walk of the reference's GPU locator
// (RadixSortNeighborLocator, S/base/locator.py:515-553).

#pragma once

#include "sphb_density_pass.cuh"
#include "sphb_force_pass.cuh"

namespace sphb {

constexpr int TILE_LCAP = 32;   // accepted entries a thread holds at once
constexpr int TILE_MAX_RANGES = SPHB_MAX_ARRAYS * (2 * SPHB_MAX_STENCIL + 1);
// polls of a bulk-copy completion before the block gives up (each poll
// suspends for a hardware-chosen time; a copy of ~50 KB completes in
// microseconds)
constexpr long TILE_WAIT_POLLS = 1L << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    // make the initialised barrier visible to the bulk-copy (async) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// global -> shared 1D bulk copy completing on bar; bytes a multiple of 16,
// both addresses 16-byte aligned (no multicast)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of bar: false when it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t parity)
{
    for (long i = 0; i < TILE_WAIT_POLLS; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// The staged ranges of one block, in static shared memory.  Range r =
// b (2R+1) + dy + R holds the particles [gstart, gend) at shared slots
// sbase + (j - gstart).
struct TileRanges {
    int gstart[TILE_MAX_RANGES];
    int gend[TILE_MAX_RANGES];
    int sbase[TILE_MAX_RANGES];
    int fallback;   // 1: read the records from global memory
    int bad;        // 1: the block's cell / start data failed a bounds check
};

// Warp 0: plan and issue the staging of the block's dests [k0, k1) of scene
// s over the source arrays of src.  Lane r computes range r's particle
// bounds; every lane then places the ranges in order (a slot's parity
// equals its particle's and one spare slot surrounds each range, so that
// 8-byte records copy as whole 16-byte units); when they fit cap slots,
// lane 0 arms the barrier with the byte count and each lane issues its own
// range's bulk copies of the float4 array g4 (and, when non-null, of the
// float4 array t4 and the float2 array v2).  A float2 element that would
// widen a copy past the array's end is copied by its lane.
template <int R>
__device__ __forceinline__ void tile_plan_stage(const sphb_engine &e, TileRanges &tr, int s,
                                                int k0, int k1, uint32_t src, int cap,
                                                const float4 *g4, float4 *sg4, const float4 *t4,
                                                float4 *st4, const float2 *v2, float2 *sv2,
                                                unsigned long long *bar)
{
    constexpr int NR = 2 * R + 1;
    const int lane = threadIdx.x & 31;
    const sphb_scene_state &st = e.sstate[s];
    const int A = e.cfg.num_arrays;
    const int N = e.cfg.num_particles;
    const int nx = st.n[0], ncells = st.ncells;
    const bool tile_ok = k0 >= 0 && k1 > k0 && k1 <= N;
    const int c_first = tile_ok ? e.f.cell[k0] : 0, c_last = tile_ok ? e.f.cell[k1 - 1] : -1;
    int g0 = 0, g1 = 0;
    bool bad = !tile_ok;
    const int b = lane / NR, dy = lane - b * NR - R;
    if (lane < A * NR && ((src >> b) & 1u) && tile_ok) {
        const long long lo = (long long)c_first + (long long)dy * nx - R;
        const long long hi = (long long)c_last + (long long)dy * nx + R + 1;
        if (c_first < 0 || c_last < c_first || lo < 0 || hi > ncells) {
            bad = true;
        } else {
            const int base = st.cell_base + b * ncells;
            g0 = e.work.start[base + (int)lo];
            g1 = e.work.start[base + (int)hi];
            if (g0 < 0 || g1 < g0 || g1 > N) {
                bad = true;
                g0 = g1 = 0;
            }
        }
    }
    bad = __any_sync(0xffffffffu, bad);
    // place the ranges in order (every lane walks all of them)
    int cursor = 0, my_sb = 1;
    for (int r = 0; r < A * NR; ++r) {
        const int rg0 = __shfl_sync(0xffffffffu, g0, r);
        const int n = __shfl_sync(0xffffffffu, g1 - g0, r);
        int sb = cursor + 1;
        if ((sb & 1) != (rg0 & 1)) ++sb;
        if (lane == r) my_sb = sb;
        if (n > 0) cursor = sb + n + 1;
    }
    const bool fb = bad || cursor > cap;
    if (lane < TILE_MAX_RANGES) {
        tr.gstart[lane] = g0;
        tr.gend[lane] = g1;
        tr.sbase[lane] = my_sb;
    }
    if (lane == 0) {
        tr.fallback = fb ? 1 : 0;
        tr.bad = bad ? 1 : 0;
        mbar_init(bar, 1);
    }
    if (fb) return;
    // bytes of this lane's copies
    const int n = g1 - g0;
    int a0 = 0, a1 = 0;
    uint32_t bytes = 0;
    if (n > 0) {
        bytes = 16u * n * (t4 ? 2u : 1u);
        if (v2) {
            a0 = g0 & ~1;
            a1 = (g1 + 1) & ~1;
            if (a1 > N) a1 -= 2;   // N odd: the last element goes by hand
            if (a1 > a0) bytes += 8u * (a1 - a0);
        }
    }
    uint32_t total = bytes;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) mbar_arrive_expect_tx(bar, total);
    __syncwarp();
    if (n > 0) {
        bulk_g2s(sg4 + my_sb, g4 + g0, 16u * n, bar);
        if (t4) bulk_g2s(st4 + my_sb, t4 + g0, 16u * n, bar);
        if (v2) {
            if (((g1 + 1) & ~1) > N) sv2[my_sb + (N - 1 - g0)] = v2[N - 1];
            if (a1 > a0) bulk_g2s(sv2 + my_sb - (g0 - a0), v2 + a0, 8u * (a1 - a0), bar);
        }
    }
}

// The stencil cells of a dest in cell (cx, cy) of source array b, row dy:
// the particle bounds bd[0 .. 2R+1] of its 2R+1 cells; false (visit
// nothing) when they leave the staged range r.
template <int R>
__device__ __forceinline__ bool tile_row(const sphb_engine &e, const TileRanges &tr, int r,
                                         int base, int nx, int cx, int cy, int dy, int *bd)
{
    const int row = base + (cy + dy) * nx + cx;
#pragma unroll
    for (int i = 0; i < 2 * R + 2; ++i) bd[i] = __ldg(e.work.start + row - R + i);
    return bd[0] >= tr.gstart[r] && bd[2 * R + 1] <= tr.gend[r] && bd[0] <= bd[2 * R + 1];
}

// One dest's candidate search.  SH: the records come from shared memory
// (slot = j - gstart + sbase per range), else from global memory.  rec(i)
// gives the geo record of slot / index i; every candidate within the
// pre-selection radius goes into this thread's list (column `list`,
// stride blockDim.x) as index | cell offsets, and flush(cnt) consumes the
// list whenever the next cell could overflow it, and at the end.  The loop
// body has no branch: the entry is stored unconditionally and the count
// advances only when accepted.
template <int R, bool SH, typename Rec, typename Flush>
__device__ __forceinline__ void tile_search(const sphb_engine &e, const TileRanges &tr,
                                            uint32_t src, int A, int s, int cx, int cy, float xk,
                                            float yk, float csf, float pre2, uint32_t *list,
                                            Rec &&rec, Flush &&flush)
{
    const sphb_scene_state &st = e.sstate[s];
    const int nx = st.n[0], ncells = st.ncells;
    const int T = blockDim.x;
    int cnt = 0;
    for (int b = 0; b < A; ++b) {
        if (!((src >> b) & 1u)) continue;
        const int base = st.cell_base + b * ncells;
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy) {
            const int r = b * (2 * R + 1) + dy + R;
            int bd[2 * R + 2];
            if (!tile_row<R>(e, tr, r, base, nx, cx, cy, dy, bd)) {
                atomicOr(e.work.status, (unsigned)SPHB_ST_BAD_INDEX);
                continue;
            }
            const int off = SH ? tr.sbase[r] - tr.gstart[r] : 0;
            const float yo = yk - (float)dy * csf;
#pragma unroll
            for (int c = 0; c <= 2 * R; ++c) {
                const int o = c - R;
                const float xo = xk - (float)o * csf;
                const uint32_t tag = ((uint32_t)(o + 2) << SPHB_NBR_IDX_BITS_2D) |
                                     ((uint32_t)(dy + 2) << (SPHB_NBR_IDX_BITS_2D + 3));
                const int hi = bd[c + 1] + off;
                for (int j = bd[c] + off; j < hi;) {
                    if (cnt > 0 && cnt + (hi - j) > TILE_LCAP) {
                        flush(cnt);
                        cnt = 0;
                    }
                    const int jl = min(hi, j + (TILE_LCAP - cnt));
#pragma unroll 4
                    for (; j < jl; ++j) {
                        const float4 g = rec(j);
                        const float ddx = xo - g.x, ddy = yo - g.y;
                        list[cnt * T] = (uint32_t)j | tag;
                        cnt += (ddx * ddx + ddy * ddy < pre2) ? 1 : 0;
                    }
                }
            }
        }
    }
    if (cnt > 0) flush(cnt);
}

// SPHRho + Tait (2D FP32C, tiled).  Dynamic shared memory: cap float4
// records, then TILE_LCAP x blockDim.x list entries.  With e.f.nbr the
// accepted entries of every dest also go to the per-stage lists
// nbr[slot][N] (count in nbr_cnt[k], -1 when more than list_cap), which the
// force pass of the same stage reads instead of searching again.
template <int KT, int R>
__global__ void __launch_bounds__(256, 4)
k_density_tiled(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask, int flags,
                int cap)
{
    // a programmatic dependent of the rebin before it (see k_density)
    pdl_wait();
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileRanges tr;
    __shared__ unsigned long long bar;
    float4 *s_geo = (float4 *)smem;
    uint32_t *s_list = (uint32_t *)(s_geo + cap);
    const sphb_tile tl = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = tl.seg / A, a = tl.seg - s * A;
    const uint32_t src = e.cfg.rho_src[a];
    if (!((dest_mask >> a) & 1u) || src == 0u) return;   // block-uniform
    const int N = e.cfg.num_particles;
    const float4 *__restrict__ geo = (const float4 *)e.f.geo;
    if (threadIdx.x < 32)
        tile_plan_stage<R>(e, tr, s, tl.begin, tl.end, src, cap, geo, s_geo, nullptr, nullptr,
                           nullptr, nullptr, &bar);
    __syncthreads();
    const int k = tl.begin + (int)threadIdx.x;
    bool active = k < tl.end;
    const sphb_scene &sc = e.scene[s];
    const sphb_scene_state &st = e.sstate[s];
    unsigned int np = 0;
    Kahan acc;
    float4 gk = make_float4(0.f, 0.f, 0.f, 0.f);
    int ck = 0;
    if (active) {
        gk = geo[k];
        ck = e.f.cell[k];
    }
    if (tr.bad && threadIdx.x == 0) flag(e, SPHB_ST_BAD_INDEX);
    if (!tr.fallback && !mbar_wait_bounded(&bar, 0)) {
        flag(e, SPHB_ST_STAGE_TIMEOUT);
        mbar_wait_bounded(&bar, 0);   // the copies in flight, once more
        active = false;
    }
    if (sc.variable_h || sc.hks) {   // not a tiled configuration
        if (threadIdx.x == 0) flag(e, SPHB_ST_BAD_INDEX);
        active = false;
    }
    uint32_t *__restrict__ gl = e.f.list_cap > 0 ? e.f.nbr : nullptr;
    int exported = 0;
    if (active) {
        int cx, cy, cz;
        cell_coords(ck, st.n, cx, cy, cz);
        if (!dest_cell_ok<2, R>(cx, cy, 0, st.n)) {
            flag(e, SPHB_ST_BAD_INDEX);
            exported = -1;
        } else {
            const float csf = (float)sc.cell_size;
            const float xk = gk.x, yk = gk.y, hk = gk.z;
            const float rad = hk * (float)sc.radius_scale;
            const float rad2 = rad * rad;
            const float pre2 = rad2 * (1.0f + 1e-5f);
            const float kf = (float)Kern<KT>::template norm<2>();
            const float ihk = __fdividef(1.0f, hk);
            const float fack = kf * ihk * ihk;
            const bool uh = sc.uniform_h != 0;
            const int T = blockDim.x;
            const int lcap = e.f.list_cap;
            uint32_t *list = s_list + threadIdx.x;
            auto body = [&](auto shared) {
                constexpr bool SH = decltype(shared)::value;
                auto rec = [&](int i) { return SH ? s_geo[i] : __ldg(geo + i); };
                auto math = [&](uint32_t v) {
                    const EntryF en = entry_unpack_f<2>(v);
                    const float4 g = rec(en.j);
                    const float dx = (xk - g.x) - en.o * csf;
                    const float ddy = (yk - g.y) - en.dy * csf;
                    const float r2 = dx * dx + ddy * ddy;
                    if (!(r2 < rad2)) return;
                    const float ir = rsqrtf(fmaxf(r2, 1e-30f));   // q = 0 at r = 0
                    float w;
                    if (uh) {
                        w = Kern<KT>::w_bf(r2 * ir * ihk, fack);
                    } else {
                        // W(r, h_ab), h_ab = (h_a + h_b) / 2
                        const float hs = 0.5f * (hk + g.z);
                        const float ih = __fdividef(1.0f, hs);
                        w = Kern<KT>::w_bf(r2 * ir * ih, kf * ih * ih);
                    }
                    acc.add(g.w * w);
                    ++np;
                };
                auto flush = [&](int cnt) {
#pragma unroll 1
                    for (int i = 0; i < cnt; ++i) {
                        const uint32_t v = list[i * T];
                        math(v);
                        if (gl && exported + i < lcap) gl[(size_t)(exported + i) * N + k] = v;
                    }
                    exported += cnt;
                };
                tile_search<R, SH>(e, tr, src, A, s, cx, cy, xk, yk, csf, pre2, list, rec,
                                   flush);
            };
            if (tr.fallback) body(std::false_type{});
            else body(std::true_type{});
        }
    } else {
        exported = -1;
    }
    if (gl && k < tl.end) e.f.nbr_cnt[k] = (exported >= 0 && exported <= e.f.list_cap) ? exported : -1;
    if (tr.fallback && threadIdx.x == 0) atomicAdd(&e.work.pairs[2], 1ull);
    density_finish<true>(e, cur, k, s, a, active, 0, acc.value(), flags & SPHB_DENSITY_EOS, np);
}

// MomentumEquation (mode 0) / SPHPressureGradient (mode 1) / the split
// MonaghanArtificialViscosity (mode 2) + gravity, with
// the stage in the epilogue (2D FP32C, tiled).  Dynamic shared memory: cap
// float4 geo and thermo records, cap float2 velocities, then TILE_LCAP x
// blockDim.x list entries.  With SPHB_FORCE_USE_LIST and the density pass of
// this stage run over the same sources, each dest reads its accepted
// entries from that pass's per-stage list; otherwise (or when its list
// overflowed) it searches its cells.
template <int KT, int R>
__global__ void __launch_bounds__(256, 3)
k_force_tiled(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask,
              int with_gravity, int mode, int cap)
{
    // a programmatic dependent of the density pass: the records it wrote
    // are read (by the bulk copies too) only after this
    pdl_wait();
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileRanges tr;
    __shared__ unsigned long long bar;
    float4 *s_geo = (float4 *)smem;
    float4 *s_th = s_geo + cap;
    float2 *s_vel = (float2 *)(s_th + cap);
    uint32_t *s_list = (uint32_t *)(s_vel + cap);
    const sphb_tile tl = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = tl.seg / A, a = tl.seg - s * A;
    const uint32_t mm = e.cfg.mom_src[a];
    if (!((dest_mask >> a) & 1u) || mm == 0u) return;   // block-uniform
    const int N = e.cfg.num_particles;
    const float4 *__restrict__ geo = (const float4 *)e.f.geo;
    const float4 *__restrict__ th = (const float4 *)e.f.thermo;
    const float2 *__restrict__ vel = (const float2 *)e.f.vel;
    if (threadIdx.x < 32)
        tile_plan_stage<R>(e, tr, s, tl.begin, tl.end, mm, cap, geo, s_geo, th, s_th, vel,
                           s_vel, &bar);
    __syncthreads();
    const int k = tl.begin + (int)threadIdx.x;
    bool active = k < tl.end;
    const sphb_scene &sc = e.scene[s];
    const sphb_scene_state &st = e.sstate[s];
    const bool visc = (mode & 15) == 0;
    const bool avisc = (mode & 15) == 2;   // split-form viscosity alone
    // the density pass's per-stage lists hold this array's SPHRho sources
    const bool use_list = (mode & SPHB_FORCE_USE_LIST) && e.f.list_cap > 0 && e.f.nbr &&
                          e.f.nbr_cnt && e.cfg.rho_src[a] == mm;
    unsigned int np = 0;
    Kahan ax, ay;
    float dtmax = 0.f;
    float4 gk = make_float4(0.f, 0.f, 0.f, 0.f), tk = gk;
    float2 vk = make_float2(0.f, 0.f);
    int ck = 0, lc = -1;
    if (active) {
        gk = geo[k];
        tk = th[k];
        vk = vel[k];
        ck = e.f.cell[k];
        if (use_list) lc = e.f.nbr_cnt[k];
    }
    if (tr.bad && threadIdx.x == 0) flag(e, SPHB_ST_BAD_INDEX);
    if (!tr.fallback && !mbar_wait_bounded(&bar, 0)) {
        flag(e, SPHB_ST_STAGE_TIMEOUT);
        mbar_wait_bounded(&bar, 0);
        active = false;
    }
    if (sc.variable_h || sc.hks) {
        if (threadIdx.x == 0) flag(e, SPHB_ST_BAD_INDEX);
        active = false;
    }
    if (active) {
        int cx, cy, cz;
        cell_coords(ck, st.n, cx, cy, cz);
        if (!dest_cell_ok<2, R>(cx, cy, 0, st.n)) {
            flag(e, SPHB_ST_BAD_INDEX);
        } else {
            const float csf = (float)sc.cell_size;
            const float xk = gk.x, yk = gk.y, hk = gk.z;
            const float uk = vk.x, vvk = vk.y;
            const float rad = hk * (float)sc.radius_scale;
            const float rad2 = rad * rad;
            const float pre2 = rad2 * (1.0f + 1e-5f);
            const float alpha = (float)sc.alpha, beta = (float)sc.beta;
            const float eta2 = (float)(sc.eta * sc.eta);
            const float kf = (float)Kern<KT>::template norm<2>();
            const float ihk = __fdividef(1.0f, hk);
            const float fihk = kf * ihk * ihk * ihk;   // fac / h of the dest
            const float eh2k = eta2 * hk * hk;
            const bool uh = sc.uniform_h != 0;
            const int T = blockDim.x;
            uint32_t *list = s_list + threadIdx.x;
            auto body = [&](auto shared) {
                constexpr bool SH = decltype(shared)::value;
                auto rec = [&](int i) { return SH ? s_geo[i] : __ldg(geo + i); };
                auto math = [&](uint32_t v) {
                    const EntryF en = entry_unpack_f<2>(v);
                    const float4 g = rec(en.j);
                    const float rx = (xk - g.x) - en.o * csf;
                    const float ry = (yk - g.y) - en.dy * csf;
                    const float r2 = rx * rx + ry * ry;
                    if (!(r2 < rad2)) return;
                    const float4 t = SH ? s_th[en.j] : __ldg(th + en.j);
                    float hab = hk, eh2 = eh2k, gw;
                    const float ir = rsqrtf(fmaxf(r2, 1e-30f));
                    if (uh) {
                        gw = Kern<KT>::gw_bf(r2 * ir * ihk, ir, ihk, fihk);
                    } else {
                        hab = 0.5f * (hk + g.z);
                        eh2 = eta2 * hab * hab;
                        const float ih = __fdividef(1.0f, hab);
                        gw = Kern<KT>::gw_bf(r2 * ir * ih, ir, ih, kf * ih * ih * ih);
                    }
                    ++np;
                    // P_a/rho_a^2 + P_b/rho_b^2 (none in the split viscosity)
                    float tmp = avisc ? 0.f : tk.w + t.w;
                    if (visc || avisc) {
                        const float2 vb = SH ? s_vel[en.j] : __ldg(vel + en.j);
                        const float vx = uk - vb.x, vy = vvk - vb.y;
                        const float dot = vx * rx + vy * ry;
                        const float mu = __fdividef(hab * dot, r2 + eh2);
                        dtmax = fmaxf(dtmax, fabsf(avisc ? __fdividef(hab * dot,
                                                                       r2 + 0.01f * hab * hab)
                                                         : mu));
                        // Pi_ab = (-alpha c_ab mu + beta mu^2) / rho_ab when mu < 0
                        const float mn = fminf(mu, 0.f);
                        const float cab = 0.5f * (tk.z + t.z);
                        const float rhoab = 0.5f * (tk.x + t.x);
                        tmp += __fdividef(-alpha * cab * mn + beta * mn * mn, rhoab);
                    }
                    const float f = -g.w * tmp * gw;
                    ax.add(f * rx);
                    ay.add(f * ry);
                };
                if (lc >= 0) {
                    // the density pass's accepted entries, 4 loads ahead
                    const uint32_t *__restrict__ p = e.f.nbr + k;
                    uint32_t v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) v[u] = u < lc ? __ldg(p + (size_t)u * N) : 0u;
#pragma unroll 1
                    for (int i = 0; i < lc; i += 4) {
                        uint32_t w[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            w[u] = i + 4 + u < lc ? __ldg(p + (size_t)(i + 4 + u) * N) : 0u;
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (i + u < lc) math(v[u]);
#pragma unroll
                        for (int u = 0; u < 4; ++u) v[u] = w[u];
                    }
                    return;
                }
                auto flush = [&](int cnt) {
#pragma unroll 1
                    for (int i = 0; i < cnt; ++i) math(list[i * T]);
                };
                tile_search<R, SH>(e, tr, mm, A, s, cx, cy, xk, yk, csf, pre2, list, rec,
                                   flush);
            };
            if (tr.fallback) body(std::false_type{});
            else body(std::true_type{});
        }
    }
    if (tr.fallback && threadIdx.x == 0) atomicAdd(&e.work.pairs[2], 1ull);
    double acc[3] = {ax.value(), ay.value(), 0.0};
    const double xs[3] = {0.0, 0.0, 0.0};
    force_finish<2, true, false>(e, cur, k, s, a, active, 0, acc, (double)dtmax, 0.0, xs,
                                 visc || avisc, mm, 0u, 0u, with_gravity, mode, np);
}

// Shared-memory slots of a tiled block: the (2R+1) rows of T dests plus
// their halos, with spare slots between ranges.  Blocks whose ranges
// exceed it read from global memory (counted in work.pairs[2]).
inline int tile_cap(int T, int R)
{
    return ((2 * R + 1) * (T + 64) + 32 + 1) & ~1;
}

inline size_t tile_smem_density(int T, int cap)
{
    return (size_t)cap * 16 + (size_t)TILE_LCAP * T * 4;
}

inline size_t tile_smem_force(int T, int cap)
{
    return (size_t)cap * 40 + (size_t)TILE_LCAP * T * 4;
}

template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int KT>
void launch_density_tiled(const sphb_engine &e, int cur, uint32_t dm, int flags, cudaStream_t st)
{
    const int T = e.cfg.pair_block;
    const int R = e.cfg.stencil;
    const int cap = tile_cap(T, R);
    const size_t sm = tile_smem_density(T, cap);
    const dim3 g(e.num_pair_tiles), b(T);
    auto go = [&](auto kern) {
        if (allow_smem(kern, sm) != cudaSuccess) return;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = b;
        cfg.dynamicSmemBytes = sm;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, e, cur, dm, flags, cap);
    };
    if (R == 1) go(k_density_tiled<KT, 1>);
    else go(k_density_tiled<KT, 2>);
}

template <int KT>
void launch_force_tiled(const sphb_engine &e, int cur, uint32_t dm, int grav, int mode,
                        cudaStream_t st)
{
    const int T = e.cfg.pair_block;
    const int R = e.cfg.stencil;
    const int cap = tile_cap(T, R);
    const size_t sm = tile_smem_force(T, cap);
    const dim3 g(e.num_pair_tiles), b(T);
    auto go = [&](auto kern) {
        if (allow_smem(kern, sm) != cudaSuccess) return;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = b;
        cfg.dynamicSmemBytes = sm;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, kern, e, cur, dm, grav, mode, cap);
    };
    if (R == 1) go(k_force_tiled<KT, 1>);
    else go(k_force_tiled<KT, 2>);
}

}  // namespace sphb
