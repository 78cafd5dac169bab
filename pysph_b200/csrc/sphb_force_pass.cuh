// sphb_force_pass.cuh -- the force pass, templated on the smoothing kernel.
// Included by one translation unit per kernel type (sphb_pass_*.cu), which
// instantiates launch_force_kt for its kernel and dimensions.
//
// MomentumEquation.eval_nbr (S/sph/funcs/pressure_funcs.pyx:246-391; OpenCL
// pressure_funcs.clt:69-157), per neighbour b of dest a:
//   dot = v_ab . r_ab,  dt_fac_a = max |h_ab dot / (r_ab^2 + eta^2 h_ab^2)|
//   tmp = P_a/rho_a^2 + P_b/rho_b^2 (+ Pi_ab when dot < 0,
//         Pi_ab = (-alpha c_ab mu + beta mu^2) / rho_ab, mu = h_ab dot /
//         (r_ab^2 + eta^2 h_ab^2))
//   a_a += -m_b tmp grad W(r_ab, h_ab)
// SPHPressureGradient (:62-161) is the same without Pi and dt_fac.
// GravityForce (S/sph/funcs/external_force.pyx:13-62) adds g afterwards.
// Per scene the kernel also keeps max dt_fac and max |a|^2 for the CFL rule.
// Variable h (scene.variable_h): the symmetric neighbour set r < radius_scale
// max(h_a, h_b); with scene.hks every pair function's W and grad W are the
// means of their values at h_a and h_b (pressure_funcs.pyx:141-149,
// 371-381), the viscosity and dt_fac keep h_ab.

#pragma once

#include <type_traits>

#include "sphb_kernels.cuh"
#include "sphb_launch.cuh"
#include "sphb_pairs.cuh"
#include "sphb_stage.cuh"

namespace sphb {

// Everything after the pair sums of dest k: its outputs (non-LocalReal
// dests get 0), gravity, dt_fac, the per-scene CFL maxima, the integrator
// stage fused into the epilogue (FP32C) and the pair count.  Every thread
// of the block calls it (block reductions inside); acc, dtf, drho and xs
// are valid in lane 0 of each dest; visc: the pass has a viscous term
// and writes dt_fac.
template <int DIM, bool F32, bool CONT>
__device__ __forceinline__ void force_finish(const sphb_engine &e, int cur, int k, int s, int a,
                                             bool active, int lane, double *acc, double dtf,
                                             double drho, const double *xs, bool visc,
                                             uint32_t mm, uint32_t rm, uint32_t xm,
                                             int with_gravity, int mode, unsigned int np)
{
    const sphb_scene &sc = e.scene[s];
    double a2 = 0.0, dtf_out = 0.0;
    if (CONT && active && lane == 0) {
        // non-LocalReal dests get 0 (S/sph/sph_func.pyx:220-227)
        const bool real = e.buf[cur].tag[k] == 0;
        if (rm) {
            const double v = real ? drho : 0.0;
            if (F32) ((float *)e.f.drho)[k] = (float)v;
            else ((double *)e.f.drho)[k] = v;
            if (!isfinite(v)) flag(e, SPHB_ST_NONFINITE_RHO);
        }
        if (xm) {
            void *xo[3] = {e.f.xu, e.f.xv, e.f.xw};
            for (int d = 0; d < DIM; ++d) {
                const double v = real ? xs[d] : 0.0;
                if (F32) ((float *)xo[d])[k] = (float)v;
                else ((double *)xo[d])[k] = v;
            }
        }
    }
    if (active && lane == 0 && mm) {
        const bool real = e.buf[cur].tag[k] == 0;
        if (real) {
            if (with_gravity) {
                acc[0] += sc.g[0];
                acc[1] += sc.g[1];
                if (DIM == 3) acc[2] += sc.g[2];
            }
            dtf_out = visc ? dtf : 0.0;
        } else {
            acc[0] = acc[1] = acc[2] = 0.0;
        }
        if (F32) {
            const float fx = (float)acc[0], fy = (float)acc[1], fz = (float)acc[2];
            ((float *)e.f.au)[k] = fx;
            ((float *)e.f.av)[k] = fy;
            if (DIM == 3) ((float *)e.f.aw)[k] = fz;
            if (visc) ((float *)e.f.dt_fac)[k] = (float)dtf_out;
            a2 = (double)fx * fx + (double)fy * fy + (double)fz * fz;
        } else {
            ((double *)e.f.au)[k] = acc[0];
            ((double *)e.f.av)[k] = acc[1];
            if (DIM == 3) ((double *)e.f.aw)[k] = acc[2];
            if (visc) ((double *)e.f.dt_fac)[k] = dtf_out;
            a2 = acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2];
        }
        if (!isfinite(a2)) flag(e, SPHB_ST_NONFINITE_ACC);
    }
    if (!(mode & SPHB_FORCE_NO_MAXIMA)) {
        // one atomic per block and quantity (a block never spans two scenes)
        const double bdt = block_reduce(dtf_out, OpMax(), 0.0);
        const double ba2 = block_reduce(isfinite(a2) ? a2 : 0.0, OpMax(), 0.0);
        if (threadIdx.x == 0) {
            sphb_scene_state &sw = e.sstate[s];
            atomic_max_nonneg(&sw.max_dtfac, bdt);
            atomic_max_nonneg(&sw.max_acc2, ba2);
        }
    }
    if constexpr (F32) {
        // the integrator stage fused into the epilogue (FP32C): the rates
        // as stored above, the new records into the second copy
        const int kind = ((mode & SPHB_FORCE_STAGE_MASK) >> 8) - 1;
        if (kind >= 0) {
            const bool stepped = (e.cfg.step_on >> a) & 1u;
            float d2 = 0.f;
            if (active && lane == 0 && (stepped || rm)) {
                const bool real = e.buf[cur].tag[k] == 0;
                double f[3], xv[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    f[d] = (double)(float)acc[d];
                    xv[d] = (double)(float)(real ? xs[d] : 0.0);
                }
                const double dr = (double)(float)(real ? drho : 0.0);
                const float4 g_old = ((const float4 *)e.f.geo)[k];
                d2 = stage_particle<DIM, true>(e, cur, k, s, a, kind, f, xm != 0u, xv, dr,
                                               (float4 *)e.f.geo_next, e.f.vel_next, g_old);
            }
            if (stepped && e.f.anchor) warp_max_disp(e, s, d2);
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                // the particles move: the lists are not known to be complete
                // until the next rebin decision, and they leave the anchors
                e.work.meta[2] = 0;
                e.work.meta[3] = 0;
            }
        }
    }
    block_add_u64(&e.work.pairs[1], np);
}

// CONT: the continuity scheme's pair terms too -- SPHDensityRate
// (density_funcs.pyx:119-156) and XSPHCorrection (xsph_funcs.pyx:40-86),
// each over its own sources, in the same traversal as the momentum.
// The 2D FP32C momentum-only variants are held to 80 registers (three
// 256-thread blocks per SM) with list batches of 4, and to 64 (four blocks)
// with batches of 2, which then need no spills: on the dam break the
// latter's pass is 3% shorter (51.6 against 53.4 us), while batches of 4
// at 64 registers spill 256 B and take 67.5 us.  Left alone, the fused
// stage in the epilogue would take them to 96 (two blocks).  Every other
// variant is held to 128 (two blocks): the FP64 continuity pass would
// otherwise take 132 and fit one block per SM.
template <int KT, int DIM, bool F32, int LANES, int R, int U, bool CONT>
__global__ void __launch_bounds__(256, (F32 && !CONT && DIM == 2) ? (U == 2 ? 4 : 3) : 2)
k_force(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask,
        int with_gravity, int mode)
{
    // launched as a programmatic dependent of the density pass: everything
    // below reads what that pass wrote; the next rebin decision may launch
    // once every block of this pass has started
    pdl_wait();
    pdl_trigger();
    const sphb_tile tl = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = tl.seg / A, a = tl.seg - s * A;
    const uint32_t mm = e.cfg.mom_src[a];
    const uint32_t rm = CONT ? e.cfg.rate_src[a] : 0u;
    const uint32_t xm = CONT ? e.cfg.xsph_src[a] : 0u;
    if (!((dest_mask >> a) & 1u) || (mm | rm | xm) == 0u) return;  // block-uniform
    // sources visited: those the lists hold (every pair function's); each
    // term keeps to its own sources when they differ
    const uint32_t src = CONT ? list_sources(e.cfg, a) : mm;
    const bool filt = CONT && ((mm && mm != src) || (rm && rm != src) || (xm && xm != src));
    const SegBounds seg(e, s);
    const int lane = threadIdx.x & (LANES - 1);
    const int k = tl.begin + (int)(threadIdx.x / LANES);
    const bool active = k < tl.end;
    const sphb_scene_state &st = e.sstate[s];
    const int n[3] = {st.n[0], st.n[1], st.n[2]};
    const int cell_base = st.cell_base, ncells = st.ncells;
    const sphb_scene &sc = e.scene[s];
    const int *__restrict__ start = e.work.start;
    const bool visc = (mode & 15) == 0;
    // split-form MonaghanArtificialViscosity alone (no pressure terms)
    const bool avisc = (mode & 15) == 2;
    // reuse the density pass's lists (recorded over list_sources); without
    // the per-source filter they must hold the momentum sources exactly
    const bool use_list = (mode & SPHB_FORCE_USE_LIST) && e.f.list_cap > 0 && e.f.nbr &&
                          e.f.nbr_cnt && (CONT || list_sources(e.cfg, a) == mm);
    unsigned int np = 0;   // pairs of this thread
    double acc[3] = {0.0, 0.0, 0.0};
    double dtf = 0.0;
    double drho = 0.0, xs[3] = {0.0, 0.0, 0.0};   // continuity scheme sums

    if constexpr (F32) {
        Kahan ax, ay, az;
        Kahan kr, kxx, kxy, kxz;   // density rate, XSPH velocity (CONT)
        float dtmax = 0.f;
        if (active) {
            const int N = e.cfg.num_particles;
            const float4 *__restrict__ geo = (const float4 *)e.f.geo;
            const float *__restrict__ mass = (const float *)e.f.mass;
            const float4 *__restrict__ th = (const float4 *)e.f.thermo;
            const float csf = (float)sc.cell_size;
            const float4 gk = geo[k];
            const float4 tk = th[k];
            float uk, vk, wk = 0.f;
            if (DIM == 2) {
                const float2 vv = ((const float2 *)e.f.vel)[k];
                uk = vv.x;
                vk = vv.y;
            } else {
                const float4 vv = ((const float4 *)e.f.vel)[k];
                uk = vv.x;
                vk = vv.y;
                wk = vv.z;
            }
            const float xk = gk.x, yk = gk.y, zk = DIM == 3 ? gk.z : 0.f;
            const float hk = DIM == 3 ? gk.w : gk.z;
            const float rad = hk * (float)sc.radius_scale;
            const float rad2 = rad * rad;
            const float alpha = (float)sc.alpha, beta = (float)sc.beta;
            const float eta2 = (float)(sc.eta * sc.eta);
            const float kf = (float)Kern<KT>::template norm<DIM>();
            const float ihk = __fdividef(1.0f, hk);
            // fac / h of the dest: 2D kf/h^3, 3D kf/h^4
            const float fihk = DIM == 2 ? kf * ihk * ihk * ihk : kf * ihk * ihk * ihk * ihk;
            const float eh2k = eta2 * hk * hk;
            // variable h: symmetric lists and, with hks, W and grad W
            // averaged over h_a and h_b (the AV and the CFL keep h_ab)
            const bool vh = sc.variable_h != 0, hks = sc.hks != 0;
            const float rsf = (float)sc.radius_scale;
            struct Rec {
                float4 g, t;
                float vx, vy, vz, m, o, dy, dz;
                uint32_t bit;   // the source's array as a mask bit (CONT)
                bool ok;
            };
            auto load = [&](const EntryF &en) {
                Rec r;
                // list entries index the set (pads the dest itself); the
                // clamp only keeps a damaged list inside the arrays
                const int j = min(en.j, N - 1);
                r.ok = true;
                r.bit = filt ? 1u << seg.array_of(j) : ~0u;
                r.g = __ldg(geo + j);
                r.t = __ldg(th + j);
                r.m = DIM == 3 ? __ldg(mass + j) : r.g.w;
                if (visc || avisc || CONT) {
                    if (DIM == 2) {
                        const float2 vv = __ldg((const float2 *)e.f.vel + j);
                        r.vx = vv.x;
                        r.vy = vv.y;
                        r.vz = 0.f;
                    } else {
                        const float4 vv = __ldg((const float4 *)e.f.vel + j);
                        r.vx = vv.x;
                        r.vy = vv.y;
                        r.vz = vv.z;
                    }
                } else {
                    r.vx = r.vy = r.vz = 0.f;
                }
                r.o = en.o;
                r.dy = en.dy;
                r.dz = en.dz;
                return r;
            };
            auto pass = [&](auto uniform) {
                constexpr bool UH = decltype(uniform)::value;
                // the pair body; with the force mode known at compile time
                // (KM = 0 MomentumEquation, 1 SPHPressureGradient, 2 the
                // split viscosity; -1 read at run time) the list loop
                // carries no test of it
                auto make_use = [&](auto known) {
                    constexpr int KM = decltype(known)::value;
                    const bool visc_k = KM < 0 ? visc : KM == 0;
                    const bool avisc_k = KM < 0 ? avisc : KM == 2;
                    return [&, visc_k, avisc_k](const Rec &r) {
                        const float rx = (xk - r.g.x) - r.o * csf;
                        const float ry = (yk - r.g.y) - r.dy * csf;
                        float rz = 0.f;
                        float r2 = rx * rx + ry * ry;
                        if (DIM == 3) {
                            rz = (zk - r.g.z) - r.dz * csf;
                            r2 += rz * rz;
                        }
                        if (!r.ok) return;
                        const float hj = DIM == 3 ? r.g.w : r.g.z;
                        if (UH || !vh) {
                            if (!(r2 < rad2)) return;
                        } else {
                            const float rj = hj * rsf;   // r < radius_scale max(h_a, h_b)
                            if (!(r2 < rad2 || r2 < rj * rj)) return;
                        }
                        ++np;
                        const bool mom_on = !CONT || (mm & r.bit);
                        const bool rate_on = CONT && (rm & r.bit);
                        const bool xs_on = CONT && (xm & r.bit);
                        float hab = hk, eh2 = eh2k;
                        if (!UH) {
                            hab = 0.5f * (hk + hj);
                            eh2 = eta2 * hab * hab;
                        }
                        // P_a/rho_a^2 + P_b/rho_b^2 (none in the split viscosity)
                        float tmp = avisc_k ? 0.f : tk.w + r.t.w;
                        const float vx = uk - r.vx, vy = vk - r.vy, vz = wk - r.vz;
                        float dot = vx * rx + vy * ry;
                        if (DIM == 3) dot += vz * rz;
                        // r = 0 (self) gives q = 0 and a finite gradient times r_ab = 0
                        const float ir = rsqrtf(fmaxf(r2, 1e-30f));
                        // grad W / r (and W for XSPH) at h_ab, or with hks the means
                        // of the values at h_a and h_b: one evaluation in a loop
                        // keeps the register count of the uniform-h path
                        float gw, w = 0.f;
                        if (UH) {
                            const float q = r2 * ir * ihk;
                            gw = Kern<KT>::gw_bf(q, ir, ihk, fihk);
                            if (CONT && xs_on) w = Kern<KT>::w_bf(q, fihk * hk);
                        } else {
                            const float rr = r2 * ir;
                            float hs = hks ? hk : hab;
                            gw = 0.f;
    #pragma unroll 1
                            for (int t = 0;; ++t) {
                                const float ih = __fdividef(1.0f, hs);
                                const float fih = DIM == 2 ? kf * ih * ih * ih : kf * ih * ih * ih * ih;
                                const float q = rr * ih;
                                gw += Kern<KT>::gw_bf(q, ir, ih, fih);
                                if (CONT && xs_on) w += Kern<KT>::w_bf(q, fih * hs);
                                if (!hks || t == 1) break;
                                hs = hj;
                            }
                            if (hks) {
                                gw *= 0.5f;
                                w *= 0.5f;
                            }
                        }
                        if (CONT) {
                            // drho_a += m_b (v_a - v_b) . grad_a W
                            if (rate_on) kr.add(r.m * (dot * gw));
                            // XSPH: eps m_b W_ab (v_b - v_a) / rho_ab (eps at the end)
                            if (xs_on) {
                                const float temp = __fdividef(r.m * w, 0.5f * (tk.x + r.t.x));
                                kxx.add(-temp * vx);
                                kxy.add(-temp * vy);
                                if (DIM == 3) kxz.add(-temp * vz);
                            }
                            if (!mom_on) return;
                        }
                        if (visc_k || avisc_k) {
                            const float mu = __fdividef(hab * dot, r2 + eh2);
                            // the split viscosity's dt_fac has 0.01 h_ab^2 written in
                            // (viscosity_funcs.pyx:103) whatever its eta
                            dtmax = fmaxf(dtmax, fabsf(avisc_k ? __fdividef(hab * dot,
                                                                           r2 + 0.01f * hab * hab)
                                                             : mu));
                            // Monaghan Pi_ab = (-alpha c_ab mu + beta mu^2) / rho_ab
                            // when v_ab . r_ab < 0, i.e. mu < 0; else 0: min(mu, 0)
                            const float mn = fminf(mu, 0.f);
                            const float cab = 0.5f * (tk.z + r.t.z);
                            const float rhoab = 0.5f * (tk.x + r.t.x);
                            tmp += __fdividef(-alpha * cab * mn + beta * mn * mn, rhoab);
                        }
                        const float f = -r.m * tmp * gw;
                        ax.add(f * rx);
                        ay.add(f * ry);
                        if (DIM == 3) az.add(f * rz);
                    };
                };
                const int lc = list_count<LANES>(e, use_list, k, lane);
                if (lc >= 0) {
                    switch (mode & 15) {   // block-uniform
                    case 0:
                        list_loop<DIM, LANES, U>(e, k, lane, lc, load,
                                                 make_use(std::integral_constant<int, 0>{}));
                        break;
                    case 1:
                        list_loop<DIM, LANES, U>(e, k, lane, lc, load,
                                                 make_use(std::integral_constant<int, 1>{}));
                        break;
                    default:
                        list_loop<DIM, LANES, U>(e, k, lane, lc, load,
                                                 make_use(std::integral_constant<int, 2>{}));
                        break;
                    }
                    return;
                }
                auto use = make_use(std::integral_constant<int, -1>{});
                int cx, cy, cz;
                cell_coords(e.f.cell[k], n, cx, cy, cz);
                for_each_candidate<DIM, R, LANES>(
                    start, A, src, cell_base, ncells, n, cx, cy, cz, lane, N, e.work.status,
                    cell_trim_rel(e, xk, yk, zk, csf), [&](int j, int o, int dy, int dz) {
                        use(load(EntryF{j, (float)o, (float)dy, (float)dz}));
                    });
            };
            if (sc.uniform_h) pass(std::true_type{});
            else pass(std::false_type{});
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            ax.merge(__shfl_xor_sync(0xffffffffu, ax.sum, o), __shfl_xor_sync(0xffffffffu, ax.c, o));
            ay.merge(__shfl_xor_sync(0xffffffffu, ay.sum, o), __shfl_xor_sync(0xffffffffu, ay.c, o));
            if (DIM == 3)
                az.merge(__shfl_xor_sync(0xffffffffu, az.sum, o), __shfl_xor_sync(0xffffffffu, az.c, o));
            dtmax = fmaxf(dtmax, __shfl_xor_sync(0xffffffffu, dtmax, o));
        }
        acc[0] = ax.value();
        acc[1] = ay.value();
        acc[2] = az.value();
        dtf = dtmax;
        if (CONT) {
#pragma unroll
            for (int o = LANES / 2; o > 0; o >>= 1) {
                kr.merge(__shfl_xor_sync(0xffffffffu, kr.sum, o), __shfl_xor_sync(0xffffffffu, kr.c, o));
                kxx.merge(__shfl_xor_sync(0xffffffffu, kxx.sum, o), __shfl_xor_sync(0xffffffffu, kxx.c, o));
                kxy.merge(__shfl_xor_sync(0xffffffffu, kxy.sum, o), __shfl_xor_sync(0xffffffffu, kxy.c, o));
                if (DIM == 3)
                    kxz.merge(__shfl_xor_sync(0xffffffffu, kxz.sum, o),
                              __shfl_xor_sync(0xffffffffu, kxz.c, o));
            }
            drho = kr.value();
            xs[0] = kxx.value() * sc.xsph_eps;
            xs[1] = kxy.value() * sc.xsph_eps;
            xs[2] = kxz.value() * sc.xsph_eps;
        }
    } else {
        if (active) {
            const sphb_buffers &B = e.buf[cur];
            const double *__restrict__ rho = (const double *)e.f.rho;
            const double *__restrict__ pr = (const double *)e.f.p;
            const double *__restrict__ csnd = (const double *)e.f.cs;
            const double xk = B.x[k], yk = B.y[k], zk = DIM == 3 ? B.z[k] : 0.0;
            const double uk = B.u[k], vk = B.v[k], wk = DIM == 3 ? B.w[k] : 0.0;
            const double hk = B.h[k];
            const double rhoa = rho[k], Pa = pr[k], ca = csnd[k];
            const double rhoa2 = 1.0 / (rhoa * rhoa);
            const double rad = hk * sc.radius_scale;
            const double rad2 = __dmul_rn(rad, rad);
            const double alpha = sc.alpha, beta = sc.beta, eta = sc.eta;
            // with one h in the scene the symmetric set and the averaged
            // kernels are the plain ones
            const bool uh = sc.uniform_h != 0;
            const bool vh = !uh && sc.variable_h != 0, hks = !uh && sc.hks != 0;
            int cx, cy, cz;
            cell_coords(e.f.cell[k], n, cx, cy, cz);
            traverse<DIM, R, LANES>(
                e, use_list, k, lane, start, A, src, cell_base, ncells, n, cx, cy, cz,
                cell_trim_abs<DIM>(e, st, sc.cell_size, xk, yk, zk, cx, cy, cz),
                [&](int j, int, int, int) {
                    const double rx = xk - __ldg(B.x + j);
                    const double ry = yk - __ldg(B.y + j);
                    const double rz = DIM == 3 ? zk - __ldg(B.z + j) : 0.0;
                    const double rab2 = dist2_ref<DIM>(rx, ry, rz);
                    double hb = 0.0, radj2 = rad2;
                    if (vh) {
                        // symmetric: r^2 < (radius_scale h_a)^2 or (radius_scale h_b)^2
                        hb = __ldg(B.h + j);
                        const double rj = hb * sc.radius_scale;
                        radj2 = fmax(rad2, __dmul_rn(rj, rj));
                    }
                    if (!(rab2 < radj2)) return;
                    if (!vh) hb = uh ? hk : __ldg(B.h + j);
                    ++np;
                    const uint32_t bit = filt ? 1u << seg.array_of(j) : ~0u;
                    const double hab = 0.5 * (hk + hb);
                    const double rhob = __ldg(rho + j), Pb = __ldg(pr + j);
                    const double mb = __ldg(B.m + j);
                    // grad_a W: at h_ab, or with hks the mean of the gradients
                    // at h_a and h_b (pressure_funcs.pyx:371-381)
                    double gx, gy, gz = 0.0;
                    if (hks) {
                        const double ga = Kern<KT>::template gw_d<DIM>(sqrt(rab2), hk);
                        const double gb = Kern<KT>::template gw_d<DIM>(sqrt(rab2), hb);
                        gx = (rx * ga + rx * gb) * 0.5;
                        gy = (ry * ga + ry * gb) * 0.5;
                        if (DIM == 3) gz = (rz * ga + rz * gb) * 0.5;
                    } else {
                        const double g = Kern<KT>::template gw_d<DIM>(sqrt(rab2), hab);
                        gx = rx * g;
                        gy = ry * g;
                        if (DIM == 3) gz = rz * g;
                    }
                    if (CONT) {
                        const double vbx = __ldg(B.u + j), vby = __ldg(B.v + j);
                        const double vbz = DIM == 3 ? __ldg(B.w + j) : 0.0;
                        if (rm & bit) {
                            // SPHDensityRate: ((v_a - v_b) . grad_a W) m_b
                            double d = (uk - vbx) * gx + (vk - vby) * gy;
                            if (DIM == 3) d += (wk - vbz) * gz;
                            drho += d * mb;
                        }
                        if (xm & bit) {
                            // XSPHCorrection: m_b W_ab / rho_ab (v_b - v_a) eps
                            const double w =
                                hks ? 0.5 * (Kern<KT>::template w_d<DIM>(sqrt(rab2), hk) +
                                             Kern<KT>::template w_d<DIM>(sqrt(rab2), hb))
                                    : Kern<KT>::template w_d<DIM>(sqrt(rab2), hab);
                            const double temp = mb * w / (0.5 * (rhob + rhoa));
                            xs[0] += temp * (vbx - uk) * sc.xsph_eps;
                            xs[1] += temp * (vby - vk) * sc.xsph_eps;
                            if (DIM == 3) xs[2] += temp * (vbz - wk) * sc.xsph_eps;
                        }
                        if (!(mm & bit)) return;
                    }
                    // P_a/rho_a^2 + P_b/rho_b^2; the split viscosity has none
                    // (tmp = piab; tmp *= -mb, viscosity_funcs.pyx:125-126)
                    double tmp = avisc ? 0.0 : Pa * rhoa2 + Pb * (1.0 / (rhob * rhob));
                    if (visc || avisc) {
                        const double vx = uk - __ldg(B.u + j);
                        const double vy = vk - __ldg(B.v + j);
                        const double vz = DIM == 3 ? wk - __ldg(B.w + j) : 0.0;
                        double dot = vx * rx + vy * ry;
                        if (DIM == 3) dot += vz * rz;
                        const double den = rab2 + eta * eta * hab * hab;
                        dtf = fmax(dtf, fabs(hab * dot /
                                             (avisc ? rab2 + 0.01 * hab * hab : den)));
                        if (dot < 0) {
                            const double cab = 0.5 * (ca + __ldg(csnd + j));
                            const double rhoab = 0.5 * (rhoa + rhob);
                            double mu = hab * dot;
                            mu /= den;
                            double piab = -alpha * cab * mu + beta * mu * mu;
                            piab /= rhoab;
                            tmp += piab;
                        }
                    }
                    tmp *= -mb;
                    acc[0] += tmp * gx;
                    acc[1] += tmp * gy;
                    if (DIM == 3) acc[2] += tmp * gz;
                });
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o);
            acc[1] += __shfl_xor_sync(0xffffffffu, acc[1], o);
            if (DIM == 3) acc[2] += __shfl_xor_sync(0xffffffffu, acc[2], o);
            dtf = fmax(dtf, __shfl_xor_sync(0xffffffffu, dtf, o));
            if (CONT) {
                drho += __shfl_xor_sync(0xffffffffu, drho, o);
                for (int d = 0; d < DIM; ++d) xs[d] += __shfl_xor_sync(0xffffffffu, xs[d], o);
            }
        }
    }

    force_finish<DIM, F32, CONT>(e, cur, k, s, a, active, lane, acc, dtf, drho, xs,
                                 visc || avisc, mm, rm, xm, with_gravity, mode, np);
}

template <int KT, int DIM, bool F32, int LV, int RV>
static void launch_force_lr(const sphb_engine &e, int cur, uint32_t dm, int grav, int mode,
                            bool cont, cudaStream_t st)
{
    const dim3 g(e.num_pair_tiles), b(e.cfg.pair_block);
    if (cont) {
        launch_pdl(k_force<KT, DIM, F32, LV, RV, 4, true>, g, b, st, e, cur, dm, grav, mode);
        return;
    }
    // the load-ahead depth only shapes the FP32C list loop of the cubic (the
    // other kernels and FP64 load 4 ahead)
    if constexpr (F32 && KT == SPHB_KERNEL_CUBIC) {
        if (e.cfg.list_batch == 2) {
            launch_pdl(k_force<KT, DIM, F32, LV, RV, 2, false>, g, b, st, e, cur, dm, grav,
                       mode);
            return;
        }
    }
    launch_pdl(k_force<KT, DIM, F32, LV, RV, 4, false>, g, b, st, e, cur, dm, grav, mode);
}

template <int KT, int DIM, bool F32>
static void launch_force_p(const sphb_engine &e, int cur, uint32_t dm, int grav,
                           int mode, cudaStream_t st)
{
    bool cont = false;
    for (int a = 0; a < SPHB_MAX_ARRAYS; ++a) cont = cont || e.cfg.rate_src[a] || e.cfg.xsph_src[a];
#define SPHB_L(LV, RV) launch_force_lr<KT, DIM, F32, LV, RV>(e, cur, dm, grav, mode, cont, st)
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
void launch_force_kt(const sphb_engine &e, int cur, uint32_t dm, int grav, int mode,
                     cudaStream_t st)
{
    if constexpr (DIM == 2) {
        if (e.cfg.pair_mode == SPHB_PAIRS_TILED) {
            launch_force_tiled<KT>(e, cur, dm, grav, mode, st);
            return;
        }
    }
    if (e.cfg.precision == SPHB_FP32C) launch_force_p<KT, DIM, true>(e, cur, dm, grav, mode, st);
    else launch_force_p<KT, DIM, false>(e, cur, dm, grav, mode, st);
}

}  // namespace sphb
