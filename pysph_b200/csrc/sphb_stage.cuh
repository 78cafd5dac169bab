// sphb_stage.cuh -- one particle's integrator stage, shared by sphb_pc_stage
// and the stage fused into the force pass's epilogue.
//
// PredictorCorrectorIntegrator (S/solver/integrator.py:614-683):
//   predict   X0 = X;  X = X0 + dt/2 F(X)                      (step, :340-367)
//   correct   X = X0 + dt/2 F(X_half);  final  X = 2 X - X0    (:632-644)
// EulerIntegrator (:420-447): X0 = X; X = X0 + dt F.  RK2Integrator
// (:452-499): the predictor, then X = X0 + dt F(X_half).
// F is the acceleration for u, v, w and, through PositionStepping
// (S/sph/funcs/position_funcs.pyx:10-56), the velocity (+ the XSPH
// correction) for x, y, z; with the continuity equation also the density
// rate for rho.  The state stays FP64; products and sums round separately
// (numpy's `initial + step * dt`, no FMA), so FP64 runs track the reference
// closely.

#pragma once

#include "sphb_common.cuh"

namespace sphb {

__device__ __forceinline__ double axpy_rn(double x0, double a, double dt)
{
    return __dadd_rn(x0, __dmul_rn(a, dt));
}

// Stage kind `stage` (0 predict / RK2 first, 1 correct + final, 2 Euler,
// 3 RK2 second, 4-7 the four RK4 stages) of particle k of array a in scene
// s, from its rates: f the
// acceleration, xv the XSPH velocity (when xsph), dr the density rate (used
// for density-rate dests).  Non-LocalReal particles get zero rates.  With
// geo_out / vel_out (FP32C) the particle's new pair records are written
// there: g_old is its current geo record (the h, m it keeps).  Returns the
// squared FP32 distance from its anchor (0 without anchors or when the
// array is not stepped).
template <int DIM, bool F32>
__device__ __forceinline__ float stage_particle(const sphb_engine &e, int cur, int k, int s,
                                                int a, int stage, const double *f, bool xsph,
                                                const double *xv, double dr, float4 *geo_out,
                                                void *vel_out, float4 g_old)
{
    const sphb_buffers &B = e.buf[cur];
    const sphb_scene_state &st = e.sstate[s];
    const double dt2 = st.dt / 2;
    // the stage: 0 save X0, X = X0 + dt/2 F; 1 X = 2 (X0 + dt/2 F) - X0;
    // 2 save X0, X = X0 + dt F; 3 X = X0 + dt F.  RK4Integrator
    // (S/solver/integrator.py:504-609), S the running sum in buf.k*: 4 save
    // X0, S = F, X = X0 + dt/2 F; 5 S = S + 2 F, X = X0 + dt/2 F; 6 S = S +
    // 2 F, X = X0 + dt F; 7 X = X0 + (1/6 dt) (S + F), numpy's order of
    // final_step's X0 + fac dt (K1 + 2 K2 + 2 K3 + K4)
    const bool save = stage == 0 || stage == 2 || stage == 4;
    const double hstep = (stage == 0 || stage == 4 || stage == 5) ? dt2 : st.dt;
    auto advance = [&](double cur0, double init, double rate, double *ks) {
        switch (stage) {
        case 1: return __dadd_rn(2 * axpy_rn(init, rate, dt2), -init);
        case 4: ks[k] = rate; break;
        case 5:
        case 6: ks[k] = __dadd_rn(ks[k], 2 * rate); break;
        case 7: return __dadd_rn(init, __dmul_rn(__dmul_rn(1.0 / 6.0, st.dt),
                                                 __dadd_rn(ks[k], rate)));
        default: break;
        }
        return axpy_rn(save ? cur0 : init, rate, hstep);
    };
    // continuity scheme: the density of every SPHDensityRate dest is
    // integrated like the other stepped properties
    if (B.rho && B.rho0 && e.cfg.rate_src[a]) {
        const double r = B.rho[k];
        const double r0 = save ? r : B.rho0[k];
        if (save) B.rho0[k] = r;
        B.rho[k] = advance(r, r0, dr, B.krho);
    }
    if (!((e.cfg.step_on >> a) & 1u)) return 0.f;
    const bool disp = e.f.anchor != nullptr;   // displacement check
    double *X[3] = {B.x, B.y, B.z};
    double *V[3] = {B.u, B.v, B.w};
    double *X0[3] = {B.x0, B.y0, B.z0};
    double *V0[3] = {B.u0, B.v0, B.w0};
    double *KX[3] = {B.kx, B.ky, B.kz};
    double *KV[3] = {B.ku, B.kv, B.kw};
    const bool real = B.tag[k] == 0;
    // every load first, so a thread's loads are in flight together
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0};
    double x0[3] = {0.0, 0.0, 0.0}, v0[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        x[d] = X[d][k];
        v[d] = V[d][k];
        if (!save) {
            x0[d] = X0[d][k];
            v0[d] = V0[d][k];
        }
    }
    int local = (geo_out || disp) ? e.f.cell[k] : 0;
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
        p[d] = advance(x[d], x0[d], fx, KX[d]);
        vn[d] = advance(v[d], v0[d], fd, KV[d]);
        X[d][k] = p[d];
        V[d][k] = vn[d];
    }
    float d2 = 0.f;
    // FP32 pair records of the new state, relative to the particle's cell of
    // the last bin, and how far it has moved from where that bin put it
    if (geo_out || disp) {
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
        if (geo_out) {
            if (DIM == 2) {
                geo_out[k] = make_float4(xr[0], xr[1], g_old.z, g_old.w);
                ((float2 *)vel_out)[k] = make_float2((float)vn[0], (float)vn[1]);
            } else {
                geo_out[k] = make_float4(xr[0], xr[1], xr[2], g_old.w);
                ((float4 *)vel_out)[k] = make_float4((float)vn[0], (float)vn[1], (float)vn[2], 0.f);
            }
        }
        if (disp) {
            const float q0 = xr[0] - an[0], q1 = xr[1] - an[1], q2 = xr[2] - an[2];
            d2 = q0 * q0 + q1 * q1 + q2 * q2;
            // a non-finite position can never be within the skin
            if (!(d2 <= 3.0e38f)) d2 = 3.0e38f;
        }
    }
    return d2;
}

// The largest d2 of the warp into the scene's max_disp2 (non-negative floats
// order like their bits); every lane of the warp calls it.
__device__ __forceinline__ void warp_max_disp(const sphb_engine &e, int s, float d2)
{
    const float wd = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(d2)));
    if ((threadIdx.x & 31) == 0 && wd > 0.f) atomic_max_nonneg(&e.sstate[s].max_disp2, (double)wd);
}

// The Solver's per-step prologue for scene s (S/solver/solver.py:546-566):
// count += 1; with use_cfl, dt from ViscousAndForceBasedTimeStep
// (S/solver/time_step_functions.py:8-57) over the maxima of the last force
// passes; t += dt; the maxima restart.  Run by k_step_begin, or by the rebin
// decision of a step's first bin (SPHB_BIN_STEP_BEGIN).
__device__ __forceinline__ void step_begin_scene(const sphb_engine &e, int s)
{
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

}  // namespace sphb
