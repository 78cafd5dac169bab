// sphb_density_pass.cuh -- the summation-density pass (SPHRho + Tait
// epilogue, neighbour-list recording), templated on the smoothing kernel.
// Included by one translation unit per kernel type (sphb_pass_*.cu), which
// instantiates launch_density_kt for its kernel and dimensions.
//
// SPHRho (S/sph/funcs/density_funcs.pyx:37-73; OpenCL S/sph/funcs/
// density_funcs.clt:3-53): rho_a = sum_b m_b W(r_ab, (h_a + h_b)/2) over the
// neighbours r_ab^2 < (radius_scale h_a)^2 of every source array, self
// included.  TaitEquation (S/sph/funcs/eos_funcs.pyx:88-129): p =
// B((rho/rho0)^gamma-1), cs = c0 (rho/rho0)^((gamma-1)/2), fused as the
// epilogue.  Non-LocalReal dests get 0 (S/sph/sph_func.pyx:220-227).
//
// FP32C: pair geometry in FP32 from cell-relative positions, the sum in FP32
// with Kahan compensation, the EOS in FP64.  FP64: the reference's
// arithmetic, with its exact neighbour predicate.
//
// Variable smoothing length (scene.variable_h): the neighbours are the
// symmetric set of VarHNbrParticleLocator (S/base/nnps.pyx:691-786),
// r^2 < (radius_scale h_a)^2 or r^2 < (radius_scale h_b)^2.  With scene.hks
// the pair's W is the mean of W(r, h_a) and W(r, h_b) (density_funcs.pyx:
// 56-63) instead of W(r, (h_a + h_b) / 2).

#pragma once

#include <type_traits>

#include "sphb_kernels.cuh"
#include "sphb_launch.cuh"
#include "sphb_pairs.cuh"

namespace sphb {

// The outputs of dest k after its density sum: rho (0 for non-LocalReal
// dests), the Tait EOS when asked and the array is a Tait dest, the FP32C
// record {rho, p, cs, p / rho^2}, and the pair count.  Every thread of the
// block calls it; rho is valid in lane 0 of each dest.
template <bool F32>
__device__ __forceinline__ void density_finish(const sphb_engine &e, int cur, int k, int s, int a,
                                               bool active, int lane, double rho, int with_eos,
                                               unsigned int np)
{
    const sphb_scene &sc = e.scene[s];
    if (active && lane == 0) {
        const bool real = e.buf[cur].tag[k] == 0;
        if (!real) rho = 0.0;
        const bool eos = with_eos && ((e.cfg.tait_on >> a) & 1u);
        double p = 0.0, c = 0.0;
        if (eos && real) {
            const double ratio = rho / sc.rho0;
            p = (eos_pow<F32>(ratio, sc.gamma) - 1.0) * sc.B;
            c = eos_pow<F32>(ratio, 0.5 * (sc.gamma - 1.0)) * sc.c0;
        }
        if constexpr (F32) {
            float4 *th = (float4 *)e.f.thermo;
            float4 t = th[k];
            t.x = (float)rho;
            if (eos) {
                t.y = (float)p;
                t.z = (float)c;
            }
            t.w = t.x != 0.f ? t.y / (t.x * t.x) : 0.f;
            th[k] = t;
            if (!isfinite(t.x) || !isfinite(t.y)) flag(e, SPHB_ST_NONFINITE_RHO);
        } else {
            ((double *)e.f.rho)[k] = rho;
            if (eos) {
                ((double *)e.f.p)[k] = p;
                ((double *)e.f.cs)[k] = c;
            }
            if (!isfinite(rho) || !isfinite(p)) flag(e, SPHB_ST_NONFINITE_RHO);
        }
    }
    block_add_u64(&e.work.pairs[0], np);
}

// The 2D FP32C variants are held to 48 registers, five 256-thread blocks per
// SM (62 registers and four blocks otherwise): 2-12% shorter passes on the
// dam break, the list-recording pass gaining most.  The 3D FP32C variants are
// held to four blocks (64 registers) and the FP64 ones to three (80; they
// would take 86 and fit two).
template <int KT, int DIM, bool F32, int LANES, int R>
__global__ void __launch_bounds__(256, F32 ? (DIM == 2 ? 5 : 4) : 3)
k_density(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask, int flags)
{
    // launched as a programmatic dependent of the rebin before it: the cells,
    // records and lists are read only after this; the force pass that
    // follows may launch once every block has started
    pdl_wait();
    pdl_trigger();
    const int with_eos = flags & SPHB_DENSITY_EOS;
    // list reuse: read the lists when the last rebin decision kept them
    // (work.meta[2]); otherwise record them, with the skin
    const bool reuse = (flags & SPHB_DENSITY_LIST_IF_VALID) && e.f.list_cap > 0;
    const bool from_list = e.f.list_cap > 0 && ((flags & SPHB_DENSITY_USE_LIST) ||
                                                (reuse && e.work.meta[2] == 1));
    // lists only (continuity scheme): record the lists after a rebin, no
    // density; with the lists kept there is nothing to do
    const bool lists_only = (flags & SPHB_DENSITY_LISTS_ONLY) != 0;
    const sphb_tile tl = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = tl.seg / A, a = tl.seg - s * A;
    const uint32_t rsrc = e.cfg.rho_src[a];           // SPHRho sources
    const uint32_t lsrc = list_sources(e.cfg, a);     // sources the lists hold
    if (!((dest_mask >> a) & 1u) || (lists_only ? lsrc : rsrc) == 0u) return;  // block-uniform
    if (lists_only && (from_list || e.f.list_cap == 0)) return;
    // recording, or reading the lists: every list source; a cell search
    // without recording: the SPHRho sources alone
    const bool records = e.f.list_cap > 0 && !from_list;
    const uint32_t src = (records || from_list) ? lsrc : rsrc;
    // neighbours outside the SPHRho sources are skipped by the sum
    const bool filt = src != rsrc;
    const SegBounds seg(e, s);
    const int lane = threadIdx.x & (LANES - 1);
    const int k = tl.begin + (int)(threadIdx.x / LANES);
    const bool active = k < tl.end;
    const sphb_scene_state &st = e.sstate[s];
    const int n[3] = {st.n[0], st.n[1], st.n[2]};
    const int cell_base = st.cell_base, ncells = st.ncells;
    const sphb_scene &sc = e.scene[s];
    const int *__restrict__ start = e.work.start;
    unsigned int np = 0;   // pairs of this thread
    double rho = 0.0;
    // neighbour list of this lane: slots lane, lane + LANES, ... of k,
    // recorded (unless this pass reads them) with the skin when they are
    // meant for reuse
    const int N = e.cfg.num_particles;
    uint32_t *__restrict__ nbr = (e.f.list_cap > 0 && !from_list) ? e.f.nbr : nullptr;
    // a lane's slots, whole pads of SPHB_LIST_PAD
    const int cap_lane = (e.f.list_cap / LANES) & ~(SPHB_LIST_PAD - 1);
    const double skin = (nbr && reuse) ? sc.skin_max : 0.0;
    if (nbr && blockIdx.x == 0 && threadIdx.x == 0) {
        // reusable only when recorded with the skin at the anchors (the
        // positions of the last rebin, work.meta[3] == 2); no pass of this
        // kernel reads meta[4], and a plain record also withdraws meta[2]
        e.work.meta[4] = (reuse && e.work.meta[3] == 2) ? 1 : 0;
        if (!reuse) e.work.meta[2] = 0;
    }
    int cnt = 0;
    auto record = [&](int j, int o, int dy, int dz) {
        if (nbr) {
            if (cnt < cap_lane)
                nbr[(size_t)(lane + LANES * cnt) * N + k] = nbr_pack<DIM>(j, o, dy, dz);
            ++cnt;
        }
    };

    if constexpr (F32) {
        Kahan acc;
        if (active) {
            const float4 *__restrict__ geo = (const float4 *)e.f.geo;
            const float *__restrict__ mass = (const float *)e.f.mass;
            const float4 gk = geo[k];
            const float csf = (float)sc.cell_size;
            const float xk = gk.x, yk = gk.y, zk = DIM == 3 ? gk.z : 0.f;
            const float hk = DIM == 3 ? gk.w : gk.z;
            const float rad = hk * (float)sc.radius_scale;
            const float rad2 = rad * rad;
            const float radl = (float)((hk * sc.radius_scale + skin) * (1.0 + 1e-5));
            const float radl2 = nbr ? radl * radl : rad2;
            const float kf = (float)Kern<KT>::template norm<DIM>();
            const float ihk = __fdividef(1.0f, hk);
            const float fack = DIM == 2 ? kf * ihk * ihk : kf * ihk * ihk * ihk;
            // variable h: symmetric lists and, with hks, W averaged over h_a, h_b
            const bool vh = sc.variable_h != 0, hks = sc.hks != 0;
            const float rsf = (float)sc.radius_scale;
            const float skinf = (float)skin;
            struct Rec {
                float4 g;
                float m, o, dy, dz;
                bool ok;
            };
            auto load = [&](const EntryF &en) {
                Rec r;
                // list entries index the set (pads the dest itself); the
                // clamp only keeps a damaged list inside the arrays
                const int j = min(en.j, N - 1);
                r.ok = !filt || ((rsrc >> seg.array_of(j)) & 1u);
                r.g = __ldg(geo + j);
                r.m = DIM == 3 ? __ldg(mass + j) : r.g.w;
                r.o = en.o;
                r.dy = en.dy;
                r.dz = en.dz;
                return r;
            };
            auto dist2 = [&](const Rec &r) {
                const float dx = (xk - r.g.x) - r.o * csf;
                const float ddy = (yk - r.g.y) - r.dy * csf;
                float r2 = dx * dx + ddy * ddy;
                if (DIM == 3) {
                    const float ddz = (zk - r.g.z) - r.dz * csf;
                    r2 += ddz * ddz;
                }
                return r2;
            };
            // uniform h (every particle of the scene): h_ab = h_a, and the
            // kernel's 1/h and normalisation are the dest's
            auto pass = [&](auto uniform) {
                constexpr bool UH = decltype(uniform)::value;
                auto use = [&](const Rec &r, float r2) {
                    if (lists_only || !r.ok) return;
                    const float hj = DIM == 3 ? r.g.w : r.g.z;
                    if (UH || !vh) {
                        if (!(r2 < rad2)) return;
                    } else {
                        const float rj = hj * rsf;   // r < radius_scale max(h_a, h_b)
                        if (!(r2 < rad2 || r2 < rj * rj)) return;
                    }
                    const float ir = rsqrtf(fmaxf(r2, 1e-30f));   // q = 0 at r = 0
                    float w;
                    if (UH) {
                        w = Kern<KT>::w_bf(r2 * ir * ihk, fack);
                    } else {
                        // W(r, h_ab), or with hks (W(r, h_a) + W(r, h_b)) / 2; one
                        // kernel evaluation in a loop keeps the register count
                        const float rr = r2 * ir;
                        float hs = hks ? hk : 0.5f * (hk + hj);
                        w = 0.f;
#pragma unroll 1
                        for (int t = 0;; ++t) {
                            const float ih = __fdividef(1.0f, hs);
                            const float fac = DIM == 2 ? kf * ih * ih : kf * ih * ih * ih;
                            w += Kern<KT>::w_bf(rr * ih, fac);
                            if (!hks || t == 1) break;
                            hs = hj;
                        }
                        if (hks) w *= 0.5f;
                    }
                    acc.add(r.m * w);
                    ++np;
                };
                // the common case (one h, every source summed, densities
                // wanted) with the tests that cannot fail there out of the
                // loops: the same arithmetic as load() and use()
                const bool plain = UH && !filt && !lists_only;
                auto load_all = [&](const EntryF &en) {
                    Rec r;
                    const int j = min(en.j, N - 1);
                    r.ok = true;
                    r.g = __ldg(geo + j);
                    r.m = DIM == 3 ? __ldg(mass + j) : r.g.w;
                    r.o = en.o;
                    r.dy = en.dy;
                    r.dz = en.dz;
                    return r;
                };
                auto sum_plain = [&](const Rec &r, float r2) {
                    if (r2 < rad2) {
                        const float ir = rsqrtf(fmaxf(r2, 1e-30f));   // q = 0 at r = 0
                        acc.add(r.m * Kern<KT>::w_bf(r2 * ir * ihk, fack));
                        ++np;
                    }
                };
                const int lc = list_count<LANES>(e, from_list, k, lane);
                if (lc >= 0) {
                    if (plain) {
                        list_loop<DIM, LANES, 4>(e, k, lane, lc, load_all,
                                                 [&](const Rec &r) { sum_plain(r, dist2(r)); });
                        return;
                    }
                    list_loop<DIM, LANES, 4>(e, k, lane, lc, load,
                                             [&](const Rec &r) { use(r, dist2(r)); });
                    return;
                }
                int cx, cy, cz;
                cell_coords(e.f.cell[k], n, cx, cy, cz);
                if (plain && nbr) {
                    // the recording pass of the common case
                    for_each_candidate<DIM, R, LANES>(
                        start, A, src, cell_base, ncells, n, cx, cy, cz, lane, N, e.work.status,
                        cell_trim_rel(e, xk, yk, zk, csf), [&](int j, int o, int dy, int dz) {
                            const Rec r = load_all(EntryF{j, (float)o, (float)dy, (float)dz});
                            const float r2 = dist2(r);
                            if (r2 < radl2) {
                                if (cnt < cap_lane)
                                    nbr[(size_t)(lane + LANES * cnt) * N + k] =
                                        nbr_pack<DIM>(j, o, dy, dz);
                                ++cnt;
                            }
                            sum_plain(r, r2);
                        });
                    return;
                }
                for_each_candidate<DIM, R, LANES>(
                    start, A, src, cell_base, ncells, n, cx, cy, cz, lane, N, e.work.status,
                    cell_trim_rel(e, xk, yk, zk, csf), [&](int j, int o, int dy, int dz) {
                        const Rec r = load(EntryF{j, (float)o, (float)dy, (float)dz});
                        const float r2 = dist2(r);
                        bool rec = r2 < radl2;
                        if (!UH && vh && nbr && !rec) {
                            // the larger of the two supports, with the skin
                            const float hj = DIM == 3 ? r.g.w : r.g.z;
                            const float rl = (hj * rsf + skinf) * (1.0f + 1e-5f);
                            rec = hj > hk && r2 < rl * rl;
                        }
                        if (rec) record(j, o, dy, dz);
                        use(r, r2);
                    });
            };
            if (sc.uniform_h) pass(std::true_type{});
            else pass(std::false_type{});
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            const float os = __shfl_xor_sync(0xffffffffu, acc.sum, o);
            const float oc = __shfl_xor_sync(0xffffffffu, acc.c, o);
            acc.merge(os, oc);
        }
        rho = acc.value();
    } else {
        double sum = 0.0;
        if (active) {
            const sphb_buffers &B = e.buf[cur];
            const double xk = B.x[k], yk = B.y[k], zk = DIM == 3 ? B.z[k] : 0.0;
            const double hk = B.h[k];
            const double rad = hk * sc.radius_scale;
            const double rad2 = __dmul_rn(rad, rad);
            const double radl = (rad + skin) * (1.0 + 1e-5);
            const double radl2 = nbr ? radl * radl : rad2;
            // with one h in the scene the symmetric set and the averaged
            // kernel are the plain ones
            const bool uh = sc.uniform_h != 0;
            const bool vh = !uh && sc.variable_h != 0, hks = !uh && sc.hks != 0;
            int cx, cy, cz;
            cell_coords(e.f.cell[k], n, cx, cy, cz);
            traverse<DIM, R, LANES>(
                e, from_list, k, lane, start, A, src, cell_base, ncells, n, cx, cy, cz,
                cell_trim_abs<DIM>(e, st, sc.cell_size, xk, yk, zk, cx, cy, cz),
                [&](int j, int o, int oy, int oz) {
                    const double dx = xk - __ldg(B.x + j);
                    const double dy = yk - __ldg(B.y + j);
                    const double dz = DIM == 3 ? zk - __ldg(B.z + j) : 0.0;
                    const double d2 = dist2_ref<DIM>(dx, dy, dz);
                    double hb = 0.0, radj2 = rad2, radlj2 = radl2;
                    if (vh) {
                        // symmetric: r^2 < (radius_scale h_a)^2 or (radius_scale h_b)^2
                        hb = __ldg(B.h + j);
                        const double rj = hb * sc.radius_scale;
                        radj2 = fmax(rad2, __dmul_rn(rj, rj));
                        const double rl = (fmax(rad, rj) + skin) * (1.0 + 1e-5);
                        radlj2 = nbr ? rl * rl : radj2;
                    }
                    if (d2 < radlj2) {
                        record(j, o, oy, oz);
                        const bool sums =
                            !lists_only && (!filt || ((rsrc >> seg.array_of(j)) & 1u));
                        if (sums && d2 < radj2) {
                            if (!vh) hb = uh ? hk : __ldg(B.h + j);
                            double w;
                            if (hks)
                                w = 0.5 * (Kern<KT>::template w_d<DIM>(sqrt(d2), hk) + Kern<KT>::template w_d<DIM>(sqrt(d2), hb));
                            else
                                w = Kern<KT>::template w_d<DIM>(sqrt(d2), 0.5 * (hk + hb));
                            sum += w * __ldg(B.m + j);
                            ++np;
                        }
                    }
                });
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        rho = sum;
    }

    if (active && nbr) {
        const int c_ok = cnt <= cap_lane ? cnt : -1;
        if (c_ok >= 0) {
            const int c_end = (c_ok + SPHB_LIST_PAD - 1) & ~(SPHB_LIST_PAD - 1);
            for (int c = c_ok; c < c_end; ++c)
                nbr[(size_t)(lane + LANES * c) * N + k] = nbr_pad<DIM>(k);
        }
        e.f.nbr_cnt[(size_t)lane * N + k] = c_ok;
    }
    density_finish<F32>(e, cur, k, s, a, active && !lists_only, lane, rho, with_eos, np);
}

template <int KT, int DIM, bool F32>
static void launch_density_p(const sphb_engine &e, int cur, uint32_t dm, int eos,
                             cudaStream_t st)
{
    const dim3 g(e.num_pair_tiles), b(e.cfg.pair_block);
#define SPHB_L(LV, RV) launch_pdl(k_density<KT, DIM, F32, LV, RV>, g, b, st, e, cur, dm, eos)
    switch (e.cfg.lanes * 10 + e.cfg.stencil) {
    case 11: SPHB_L(1, 1); break;
    case 12: SPHB_L(1, 2); break;
    case 21: SPHB_L(2, 1); break;
    case 22: SPHB_L(2, 2); break;
    case 41: SPHB_L(4, 1); break;
    case 42: SPHB_L(4, 2); break;
    case 81: SPHB_L(8, 1); break;
    case 82: SPHB_L(8, 2); break;
    }
#undef SPHB_L
}

template <int KT, int DIM>
void launch_density_kt(const sphb_engine &e, int cur, uint32_t dm, int flags, cudaStream_t st)
{
    if constexpr (DIM == 2) {
        if (e.cfg.pair_mode == SPHB_PAIRS_TILED) {
            launch_density_tiled<KT>(e, cur, dm, flags, st);
            return;
        }
    }
    if (e.cfg.precision == SPHB_FP32C) launch_density_p<KT, DIM, true>(e, cur, dm, flags, st);
    else launch_density_p<KT, DIM, false>(e, cur, dm, flags, st);
}

}  // namespace sphb
