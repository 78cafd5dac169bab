// sphb_adjoint.cu -- hand-written reverse-mode (vector-Jacobian) kernels of
// the particle update: MomentumEquation (pressure gradient + Monaghan
// artificial viscosity), the Tait EOS and summation density (sm_100a).
//
// Forward, per dest a and neighbour b (r = x_a - x_b, h = (h_a + h_b)/2):
//   rho_a = sum_b m_b W(r)                          (SPHRho)
//   p_a = B((rho_a/rho0)^g - 1), c_a = c0 (rho_a/rho0)^((g-1)/2)   (Tait)
//   T_ab = -m_b (A_ab + Pi_ab) G(r),  A_ab = p_a/rho_a^2 + p_b/rho_b^2,
//   G(r) = r g(|r|) = grad W,  Pi_ab = (-alpha cbar mu + beta mu^2)/rhobar
//   when v_ab . r < 0, mu = h v_ab.r / (r.r + eta^2 h^2)  (MomentumEquation)
//   a_a = sum_b T_ab
// Given lam_a (the adjoint of a_a) the kernels accumulate the adjoints of x,
// v, rho, p, c in gather form: each particle k visits its neighbours j once
// and adds both its dest-role terms (pair (k, j), weighted by lam_k) and
// its source-role terms (pair (j, k), weighted by lam_j), so no atomics are
// needed and the result is deterministic.  Role predicates follow the
// forward neighbour search: pair (a, b) exists when |r|^2 < (2 h_a)^2.
// All adjoint arithmetic and sums are FP64.

#include "sphb_pairs.cuh"

namespace sphb {

int check_engine_public(const sphb_engine *e, int cur);

template <int DIM>
struct V3 {
    double c[3];
};

// g(s) with grad W = r g and dg/ds (the cubic spline of
// CubicSplineKernel.gradient, S/base/kernels.pyx:380-417, and its
// derivative).  Returns g, writes dg/ds / s into dgs (for r (x) r terms).
// Two reciprocals (1/h, 1/s) replace the divisions of the textbook form.
template <int DIM>
__device__ __forceinline__ double kernel_g(double s, double h, double &dgs)
{
    const double ih = 1.0 / h;
    const double q = s * ih;
    const double fac = (DIM == 2 ? ih * ih : ih * ih * ih) * kfac_unit<DIM>();
    double g = 0.0;
    dgs = 0.0;
    if (q > 2.0) {
    } else if (q >= 1.0) {
        const double is = 1.0 / s;
        // g = -0.75 (2 - q)^2 / (h s) fac
        const double t = 2.0 - q;
        g = -0.75 * t * t * ih * is * fac;
        // dg/ds = fac (1.5 t / (h^2 s) + 0.75 t^2 / (h s^2))
        const double dg = fac * ih * is * (1.5 * t * ih + 0.75 * t * t * is);
        dgs = dg * is;
    } else if (q > 1e-14) {
        g = 3.0 * (0.75 * q - 1.0) * ih * ih * fac;
        dgs = fac * 2.25 * ih * ih * ih / s;
    }
    return g;
}

struct AdjPtrs {
    const double *lam_a;   // [DIM][N] adjoint of the acceleration (SoA)
    double *lam_x;         // [DIM][N] accumulated (+=)
    double *lam_v;         // [DIM][N] accumulated (+=)
    double *lam_rho;       // [N] written (=)
    double *lam_p;         // [N] written (=)
    double *lam_c;         // [N] written (=)
};

// The sum of v over the LANES lanes of a particle (every lane of the warp
// calls it); valid in every lane.
template <int LANES>
__device__ __forceinline__ double lane_sum(double v)
{
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Force VJP.  Inputs: positions, velocities, h, m (buf[cur]) and rho, p, cs
// (FP64 fields) of the current stage, cell tables of the current bin.  One
// pair tile per block, LANES threads per particle (the engine's pair-pass
// shape): each lane takes its share of the neighbours and the lanes' sums
// meet with shuffles.
template <int DIM, int R, int LANES>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_force_vjp(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask, AdjPtrs P)
{
    const sphb_tile t = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    const int lane = threadIdx.x & (LANES - 1);
    const int k_raw = t.begin + (int)(threadIdx.x / LANES);
    const bool active = k_raw < t.end;
    const int k = active ? k_raw : t.begin;   // inactive lanes read a valid particle
    const int N = e.cfg.num_particles;
    const sphb_buffers &B = e.buf[cur];
    const sphb_scene &sc = e.scene[s];
    const sphb_scene_state &st = e.sstate[s];
    const int n[3] = {st.n[0], st.n[1], st.n[2]};
    const double *rho = (const double *)e.f.rho;
    const double *pr = (const double *)e.f.p;
    const double *cs = (const double *)e.f.cs;
    const double alpha = sc.alpha, beta = sc.beta, eta2 = sc.eta * sc.eta;
    const double rs = sc.radius_scale;

    double xk[3] = {B.x[k], B.y[k], DIM == 3 ? B.z[k] : 0.0};
    double vk[3] = {B.u[k], B.v[k], DIM == 3 ? B.w[k] : 0.0};
    const double hk = B.h[k], mk = B.m[k];
    const double rhok = rho[k], pk = pr[k], ck = cs[k];
    const double irhok = 1.0 / rhok;
    const bool k_dest = ((dest_mask >> a) & 1u) && B.tag[k] == 0;
    double lk[3] = {0, 0, 0};
    for (int d = 0; d < DIM; ++d) lk[d] = k_dest ? P.lam_a[(size_t)d * N + k] : 0.0;
    const double radk2 = (hk * rs) * (hk * rs);

    double gx[3] = {0, 0, 0}, gv[3] = {0, 0, 0};
    double grho = 0.0, gp = 0.0, gc = 0.0;
    int cx, cy, cz;
    cell_coords(e.f.cell[k], n, cx, cy, cz);
    // every array holds candidates of both roles; mom_src of the dest's
    // array decides the dest-role sources, mom_src of the neighbour's array
    // the source role
    const uint32_t all = (1u << A) - 1u;
    // the lists of the density pass (recorded one lane per particle) hold
    // every pair of both roles when h is uniform (the predicate is then
    // symmetric)
    const bool use_list = sc.uniform_h && e.cfg.rho_src[a] != 0u && e.cfg.lanes == LANES &&
                          e.f.list_cap > 0 && e.f.nbr && e.f.nbr_cnt;
    if (active) traverse<DIM, R, LANES>(
        e, use_list, k, lane, e.work.start, A, all, st.cell_base, st.ncells, n, cx, cy, cz,
        CellTrim{}, [&](int j, int, int, int) {
            if (j == k) return;
            double r[3] = {xk[0] - B.x[j], xk[1] - B.y[j], DIM == 3 ? xk[2] - B.z[j] : 0.0};
            const double r2 = dist2_ref<DIM>(r[0], r[1], r[2]);
            const double hj = B.h[j];
            const double radj2 = (hj * rs) * (hj * rs);
            const bool role1 = k_dest && r2 < radk2;
            // j as a dest: its array must take k's array as a MomentumEquation source
            int arr_j = 0;
            for (int q = 1; q < A; ++q)
                if (j >= e.seg_offset[s * A + q]) arr_j = q;
            const bool j_dest = ((dest_mask >> arr_j) & 1u) &&
                                ((e.cfg.mom_src[arr_j] >> a) & 1u) && B.tag[j] == 0;
            const bool role2 = j_dest && r2 < radj2;
            const bool r1 = role1 && ((e.cfg.mom_src[a] >> arr_j) & 1u);
            if (!r1 && !role2) return;
            const double sdist = sqrt(r2);
            const double h = 0.5 * (hk + hj);
            double dgs;
            const double g = kernel_g<DIM>(sdist, h, dgs);
            const double G[3] = {r[0] * g, r[1] * g, r[2] * g};
            const double vj[3] = {B.u[j], B.v[j], DIM == 3 ? B.w[j] : 0.0};
            const double rhoj = rho[j], pj = pr[j], cj = cs[j], mj = B.m[j];
            const double v[3] = {vk[0] - vj[0], vk[1] - vj[1], vk[2] - vj[2]};
            const double dot = v[0] * r[0] + v[1] * r[1] + v[2] * r[2];
            // reciprocals once per pair instead of a division per term
            const double iden = 1.0 / (r2 + eta2 * h * h);
            const double mu = h * dot * iden;
            const double rhobar = 0.5 * (rhok + rhoj), cbar = 0.5 * (ck + cj);
            const double irb = 1.0 / rhobar;
            const double irhoj = 1.0 / rhoj;
            double Pi = 0.0, dPi_dmu = 0.0;
            if (dot < 0.0) {
                Pi = (-alpha * cbar * mu + beta * mu * mu) * irb;
                dPi_dmu = (-alpha * cbar + 2.0 * beta * mu) * irb;
            }
            // dmu/dr = h (v / den - 2 dot r / den^2); dmu/dv_a = h r / den
            double dmu_dr[3], dmu_dv[3];
            for (int d = 0; d < 3; ++d) {
                dmu_dr[d] = h * iden * (v[d] - 2.0 * dot * r[d] * iden);
                dmu_dv[d] = h * r[d] * iden;
            }
            // 1 / rho of each particle of the pair
            const double irho_k = irhok;
            // The pair term T = -m_b (A + Pi) G(r) is symmetric in which
            // particle is "a"; both roles use r = x_a - x_b.
            auto accumulate = [&](const double *lam, double mb, double irho_a, double p_a,
                                  double irho_b, double p_b, double sign_r, bool k_is_a) {
                // r_role = sign_r * r (role 2 has a = j, so r_role = -r)
                double rr[3] = {sign_r * r[0], sign_r * r[1], sign_r * r[2]};
                double GG[3] = {sign_r * G[0], sign_r * G[1], sign_r * G[2]};
                const double lg = lam[0] * GG[0] + lam[1] * GG[1] + lam[2] * GG[2];
                const double lr = lam[0] * rr[0] + lam[1] * rr[1] + lam[2] * rr[2];
                const double pa_r2 = p_a * irho_a * irho_a, pb_r2 = p_b * irho_b * irho_b;
                const double AP = (pa_r2 + pb_r2) + Pi;
                // lam^T dT/dr_role = -m_b [ (A+Pi)(g lam + (lam.r) dgs r) + (lam.G) dPi/dr ]
                double dT_dr[3];
                for (int d = 0; d < 3; ++d) {
                    const double dpi_dr = dPi_dmu * sign_r * dmu_dr[d];
                    dT_dr[d] = -mb * (AP * (g * lam[d] + lr * dgs * rr[d]) + lg * dpi_dr);
                }
                // dPi/dv_a = dPi_dmu * h r_role / den = dPi_dmu * sign_r * dmu_dv
                double dT_dva[3];
                for (int d = 0; d < 3; ++d)
                    dT_dva[d] = -mb * lg * dPi_dmu * sign_r * dmu_dv[d];
                const double dT_drho_a = -mb * lg * (-2.0 * pa_r2 * irho_a - 0.5 * Pi * irb);
                const double dT_drho_b = -mb * lg * (-2.0 * pb_r2 * irho_b - 0.5 * Pi * irb);
                const double dT_dp_a = -mb * lg * irho_a * irho_a;
                const double dT_dp_b = -mb * lg * irho_b * irho_b;
                const double dT_dc = (dot < 0.0) ? -mb * lg * (-alpha * mu * 0.5 * irb) : 0.0;
                if (k_is_a) {
                    for (int d = 0; d < DIM; ++d) {
                        gx[d] += dT_dr[d];    // dr/dx_a = +I
                        gv[d] += dT_dva[d];   // dv/dv_a = +I
                    }
                    grho += dT_drho_a;
                    gp += dT_dp_a;
                    gc += dT_dc;
                } else {
                    for (int d = 0; d < DIM; ++d) {
                        gx[d] -= dT_dr[d];    // dr/dx_b = -I
                        gv[d] -= dT_dva[d];
                    }
                    grho += dT_drho_b;
                    gp += dT_dp_b;
                    gc += dT_dc;
                }
            };
            if (r1) accumulate(lk, mj, irho_k, pk, irhoj, pj, 1.0, true);
            if (role2) {
                double lj[3] = {0, 0, 0};
                for (int d = 0; d < DIM; ++d) lj[d] = P.lam_a[(size_t)d * N + j];
                accumulate(lj, mk, irhoj, pj, irho_k, pk, -1.0, false);
            }
        });
    for (int d = 0; d < DIM; ++d) {
        gx[d] = lane_sum<LANES>(gx[d]);
        gv[d] = lane_sum<LANES>(gv[d]);
    }
    grho = lane_sum<LANES>(grho);
    gp = lane_sum<LANES>(gp);
    gc = lane_sum<LANES>(gc);
    if (!active || lane != 0) return;
    for (int d = 0; d < DIM; ++d) {
        P.lam_x[(size_t)d * N + k] += gx[d];
        P.lam_v[(size_t)d * N + k] += gv[d];
    }
    P.lam_rho[k] = grho;
    P.lam_p[k] = gp;
    P.lam_c[k] = gc;
}

// lam_rho_total = lam_rho + lam_p dP/drho + lam_c dC/drho (Tait), in place
// on lam_rho, for the Tait dests; others keep lam_rho.
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_eos_vjp(const __grid_constant__ sphb_engine e, int cur, double *lam_rho,
          const double *lam_p, const double *lam_c)
{
    const sphb_tile t = e.tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    const int k = t.begin + threadIdx.x;
    if (k >= t.end) return;
    if (!((e.cfg.tait_on >> a) & 1u) || e.buf[cur].tag[k] != 0) return;
    const sphb_scene &sc = e.scene[s];
    const double rho = ((const double *)e.f.rho)[k];
    const double ratio = rho / sc.rho0;
    const double dP = sc.B * sc.gamma * pow(ratio, sc.gamma - 1.0) / sc.rho0;
    const double dC = sc.c0 * 0.5 * (sc.gamma - 1.0) * pow(ratio, 0.5 * (sc.gamma - 3.0)) / sc.rho0;
    lam_rho[k] += lam_p[k] * dP + lam_c[k] * dC;
}

// Density VJP: lam_x_k += sum_j (lam_rho_k m_j [k dest] + lam_rho_j m_k
// [j dest]) G(x_k - x_j).  The force VJP's launch shape.
template <int DIM, int R, int LANES>
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_density_vjp(const __grid_constant__ sphb_engine e, int cur, uint32_t dest_mask,
              const double *lam_rho, double *lam_x)
{
    const sphb_tile t = e.pair_tiles[blockIdx.x];
    const int A = e.cfg.num_arrays;
    const int s = t.seg / A, a = t.seg - s * A;
    const int lane = threadIdx.x & (LANES - 1);
    const int k_raw = t.begin + (int)(threadIdx.x / LANES);
    const bool active = k_raw < t.end;
    const int k = active ? k_raw : t.begin;   // inactive lanes read a valid particle
    const int N = e.cfg.num_particles;
    const sphb_buffers &B = e.buf[cur];
    const sphb_scene &sc = e.scene[s];
    const sphb_scene_state &st = e.sstate[s];
    const int n[3] = {st.n[0], st.n[1], st.n[2]};
    const double rs = sc.radius_scale;
    const double xk[3] = {B.x[k], B.y[k], DIM == 3 ? B.z[k] : 0.0};
    const double hk = B.h[k], mk = B.m[k];
    const bool k_dest = ((dest_mask >> a) & 1u) && B.tag[k] == 0;
    const double lk = k_dest ? lam_rho[k] : 0.0;
    const double radk2 = (hk * rs) * (hk * rs);
    double gx[3] = {0, 0, 0};
    int cx, cy, cz;
    cell_coords(e.f.cell[k], n, cx, cy, cz);
    const uint32_t all = (1u << A) - 1u;
    // the lists of the density pass (recorded one lane per particle) hold
    // every pair of both roles when h is uniform (the predicate is then
    // symmetric)
    const bool use_list = sc.uniform_h && e.cfg.rho_src[a] != 0u && e.cfg.lanes == LANES &&
                          e.f.list_cap > 0 && e.f.nbr && e.f.nbr_cnt;
    if (active) traverse<DIM, R, LANES>(
        e, use_list, k, lane, e.work.start, A, all, st.cell_base, st.ncells, n, cx, cy, cz,
        CellTrim{}, [&](int j, int, int, int) {
            if (j == k) return;
            const double r[3] = {xk[0] - B.x[j], xk[1] - B.y[j], DIM == 3 ? xk[2] - B.z[j] : 0.0};
            const double r2 = dist2_ref<DIM>(r[0], r[1], r[2]);
            const double hj = B.h[j];
            int arr_j = 0;
            for (int q = 1; q < A; ++q)
                if (j >= e.seg_offset[s * A + q]) arr_j = q;
            const bool r1 = k_dest && r2 < radk2 && ((e.cfg.rho_src[a] >> arr_j) & 1u);
            const bool r2ok = ((dest_mask >> arr_j) & 1u) && B.tag[j] == 0 &&
                              r2 < (hj * rs) * (hj * rs) && ((e.cfg.rho_src[arr_j] >> a) & 1u);
            if (!r1 && !r2ok) return;
            double w = 0.0;
            if (r1) w += lk * B.m[j];
            if (r2ok) w += lam_rho[j] * mk;
            double dgs;
            const double g = kernel_g<DIM>(sqrt(r2), 0.5 * (hk + hj), dgs);
            for (int d = 0; d < DIM; ++d) gx[d] += w * g * r[d];
        });
    for (int d = 0; d < DIM; ++d) gx[d] = lane_sum<LANES>(gx[d]);
    if (!active || lane != 0) return;
    for (int d = 0; d < DIM; ++d) lam_x[(size_t)d * N + k] += gx[d];
}

// Generic permutation between the caller's order and the engine's.
__global__ void __launch_bounds__(SPHB_ELEM_TILE)
k_permute(const __grid_constant__ sphb_engine e, int cur, int array, int dir,
          double *user, double *eng, const int *user_offset)
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
    if (dir == 0) eng[k] = user[ui];
    else user[ui] = eng[k];
}

}  // namespace sphb

using namespace sphb;

// The pair kernels' launch shape: pair tiles of pair_block / lanes
// particles, lanes a power of two up to 8, blocks of at most 256 threads.
static int adj_shape(const sphb_engine *e)
{
    const sphb_config &c = e->cfg;
    if (c.lanes != 1 && c.lanes != 2 && c.lanes != 4 && c.lanes != 8) return SPHB_ERR_ARG;
    if (c.pair_block < 32 || c.pair_block > SPHB_ELEM_TILE || (c.pair_block & 31))
        return SPHB_ERR_ARG;
    if (e->num_pair_tiles < 0 || (e->num_pair_tiles > 0 && !e->pair_tiles)) return SPHB_ERR_ARG;
    return SPHB_OK;
}

static int adj_check(const sphb_engine *e, int cur)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (e->cfg.precision != SPHB_FP64) return SPHB_ERR_UNSUPPORTED;
    if (!e->f.rho || !e->f.p || !e->f.cs || !e->f.cell || !e->work.start) return SPHB_ERR_ARG;
    return SPHB_OK;
}

extern "C" int sphb_force_vjp(const sphb_engine *e, int cur, uint32_t dest_mask,
                              const double *lam_a, double *lam_x, double *lam_v,
                              double *lam_rho, double *lam_p, double *lam_c, void *stream)
{
    int rc = adj_check(e, cur);
    if (rc) return rc;
    if (!lam_a || !lam_x || !lam_v || !lam_rho || !lam_p || !lam_c) return SPHB_ERR_ARG;
    if ((rc = adj_shape(e))) return rc;
    if (e->num_pair_tiles == 0) return SPHB_OK;
    AdjPtrs P{lam_a, lam_x, lam_v, lam_rho, lam_p, lam_c};
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 g(e->num_pair_tiles), b(e->cfg.pair_block);
    switch (e->cfg.dim * 100 + e->cfg.stencil * 10 + e->cfg.lanes) {
#define SPHB_FV(D, RR, L)                                                         \
    case D * 100 + RR * 10 + L:                                                  \
        k_force_vjp<D, RR, L><<<g, b, 0, st>>>(*e, cur, dest_mask, P);           \
        break;
    SPHB_FV(2, 1, 1) SPHB_FV(2, 1, 2) SPHB_FV(2, 1, 4) SPHB_FV(2, 1, 8)
    SPHB_FV(2, 2, 1) SPHB_FV(2, 2, 2) SPHB_FV(2, 2, 4) SPHB_FV(2, 2, 8)
    SPHB_FV(3, 1, 1) SPHB_FV(3, 1, 2) SPHB_FV(3, 1, 4) SPHB_FV(3, 1, 8)
    SPHB_FV(3, 2, 1) SPHB_FV(3, 2, 2) SPHB_FV(3, 2, 4) SPHB_FV(3, 2, 8)
#undef SPHB_FV
    default: return SPHB_ERR_UNSUPPORTED;
    }
    return launch_status("sphb_force_vjp");
}

extern "C" int sphb_eos_vjp(const sphb_engine *e, int cur, double *lam_rho,
                            const double *lam_p, const double *lam_c, void *stream)
{
    int rc = adj_check(e, cur);
    if (rc) return rc;
    if (!lam_rho || !lam_p || !lam_c) return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    k_eos_vjp<<<e->num_tiles, SPHB_ELEM_TILE, 0, (cudaStream_t)stream>>>(*e, cur, lam_rho, lam_p, lam_c);
    return launch_status("sphb_eos_vjp");
}

extern "C" int sphb_density_vjp(const sphb_engine *e, int cur, uint32_t dest_mask,
                                const double *lam_rho, double *lam_x, void *stream)
{
    int rc = adj_check(e, cur);
    if (rc) return rc;
    if (!lam_rho || !lam_x) return SPHB_ERR_ARG;
    if ((rc = adj_shape(e))) return rc;
    if (e->num_pair_tiles == 0) return SPHB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 g(e->num_pair_tiles), b(e->cfg.pair_block);
    switch (e->cfg.dim * 100 + e->cfg.stencil * 10 + e->cfg.lanes) {
#define SPHB_DV(D, RR, L)                                                                 \
    case D * 100 + RR * 10 + L:                                                          \
        k_density_vjp<D, RR, L><<<g, b, 0, st>>>(*e, cur, dest_mask, lam_rho, lam_x);    \
        break;
    SPHB_DV(2, 1, 1) SPHB_DV(2, 1, 2) SPHB_DV(2, 1, 4) SPHB_DV(2, 1, 8)
    SPHB_DV(2, 2, 1) SPHB_DV(2, 2, 2) SPHB_DV(2, 2, 4) SPHB_DV(2, 2, 8)
    SPHB_DV(3, 1, 1) SPHB_DV(3, 1, 2) SPHB_DV(3, 1, 4) SPHB_DV(3, 1, 8)
    SPHB_DV(3, 2, 1) SPHB_DV(3, 2, 2) SPHB_DV(3, 2, 4) SPHB_DV(3, 2, 8)
#undef SPHB_DV
    default: return SPHB_ERR_UNSUPPORTED;
    }
    return launch_status("sphb_density_vjp");
}

extern "C" int sphb_permute(const sphb_engine *e, int cur, int array, int dir, double *user,
                            double *engine_buf, const int32_t *user_offset, void *stream)
{
    int rc = check_engine_public(e, cur);
    if (rc) return rc;
    if (!user || !engine_buf || !user_offset || array < 0 || array >= e->cfg.num_arrays ||
        (dir != 0 && dir != 1) || !e->buf[cur].idx)
        return SPHB_ERR_ARG;
    if (e->num_tiles == 0) return SPHB_OK;
    k_permute<<<e->num_tiles, SPHB_ELEM_TILE, 0, (cudaStream_t)stream>>>(*e, cur, array, dir, user,
                                                                         engine_buf, user_offset);
    return launch_status("sphb_permute");
}
