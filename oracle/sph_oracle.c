/*
 * sph_oracle.c -- CPU restatement of PySPH's FP64 particle-update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * pysph_b200/csrc and the timed CPU baseline of bench.py.  Nothing in the
 * product imports, links or calls it.
 *
 * Each routine restates the reference algorithm it cites (paths relative to
 * the reference project, S/ = source/pysph/), including the operand order of
 * every floating-point expression and the order in which neighbours are
 * visited, so that its FP64 results reproduce the reference's own Cython
 * results bit for bit (pinned by tests/golden fixtures made by the reference
 * itself).  Build with -ffp-contract=off: the reference is compiled for
 * x86-64 without FMA contraction.
 *
 *   cubic spline W, grad W ........ S/base/kernels.pyx:349-454 (h_dim :59-66)
 *   quintic spline, Wendland ....... S/base/kernels.pyx:461-640 (2D only, as
 *                                    there; their quirks kept, see below)
 *   cell id = floor(x / cs) ........ S/base/cell.pyx:44-84
 *   cell size = scale * max h ...... S/base/cell.pyx:911-941
 *   stencil order (x, y, z) ........ S/base/cell.pyx:95-118, :996-1032
 *   neighbour predicate, self last . S/base/nnps.pyx:271-356, :525-621
 *   variable h (symmetric lists) ... S/base/nnps.pyx:691-786
 *   hks (kernel averaged over h_a, h_b) the `if self.hks` branches of each
 *                                    function
 *   SPHRho ......................... S/sph/funcs/density_funcs.pyx:37-73,
 *                                    S/sph/sph_func.pyx:513-531
 *   SPHDensityRate ................. S/sph/funcs/density_funcs.pyx:88-161
 *   XSPHCorrection ................. S/sph/funcs/xsph_funcs.pyx:9-90,
 *                                    S/sph/sph_func.pyx:500-531 (CSPH eval)
 *   TaitEquation ................... S/sph/funcs/eos_funcs.pyx:88-129
 *   MomentumEquation ............... S/sph/funcs/pressure_funcs.pyx:246-391
 *   SPHPressureGradient ............ S/sph/funcs/pressure_funcs.pyx:62-161
 *   MonaghanArtificialViscosity .... S/sph/funcs/viscosity_funcs.pyx:19-157
 *                                    (the split form; its quirks kept)
 *   GravityForce, PositionStepping . S/sph/funcs/external_force.pyx:13-62,
 *                                    S/sph/funcs/position_funcs.pyx:10-56
 *   SPHFunction.eval (+= / tag) .... S/sph/sph_func.pyx:208-227
 *   SPHCalc.sph resets ............. S/sph/sph_calc.pyx:307-331, :431-440
 *   PredictorCorrector ............. S/solver/integrator.py:262-367, :614-683
 *   Euler, RK2, RK4 ................ S/solver/integrator.py:420-609
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_ARRAYS 4
#define ORC_PI 3.141592653589793

typedef struct {
    int64_t n;
    double *x, *y, *z, *u, *v, *w, *m, *h, *rho, *p, *cs;
    double *au, *av, *aw;      /* _a_u_1, _a_v_1, _a_w_1 */
    double *ax, *ay, *az;      /* _a_x_1, _a_y_1, _a_z_1 (PositionStepping) */
    double *dt_fac;
    double *x0, *y0, *z0, *u0, *v0, *w0;
    double *arho;              /* _a_rho_1 (SPHDensityRate) */
    double *rho0;              /* _rho0 */
    int64_t *tag;              /* 0 == LocalReal */
} orc_array;

typedef struct {
    int32_t dim;
    int32_t narrays;
    double radius_scale;       /* kernel support in units of h: 2 */
    double cell_scale;         /* cell size = cell_scale * max h: 2 */
    uint32_t rho_src[ORC_MAX_ARRAYS];  /* SPHRho sources per dest (bitmask) */
    uint32_t tait_on;                  /* TaitEquation dests (bitmask) */
    uint32_t mom_src[ORC_MAX_ARRAYS];  /* MomentumEquation sources per dest */
    uint32_t step_on;                  /* arrays stepped by the integrator */
    double c0, rho0, gamma_eos;
    double alpha, beta, gamma_av, eta;
    double gx, gy, gz;
    int32_t nthreads;
    int32_t pad_;
    orc_array a[ORC_MAX_ARRAYS];
    int64_t pairs;             /* pair interactions evaluated by orc_eval */
    uint32_t rate_src[ORC_MAX_ARRAYS]; /* SPHDensityRate sources per dest */
    uint32_t xsph_src[ORC_MAX_ARRAYS]; /* XSPHCorrection sources per dest */
    double xsph_eps;
    int32_t variable_h;        /* VarHNbrParticleLocator lists */
    int32_t hks;               /* kernels averaged over h_a and h_b */
    int32_t kernel;            /* get_type(): 1 cubic, 3 quintic, 4 Wendland */
    int32_t pad2_;
    /* split momentum: SPHPressureGradient then MonaghanArtificialViscosity
     * (S/sph/funcs/viscosity_funcs.pyx:19-157) on the mom_src pairs, with
     * the viscosity's own eta (av_eta; the reference never sets it: 0),
     * instead of MomentumEquation */
    int32_t split_av;
    int32_t pad3_;
    double av_eta;
} orc_system;

typedef struct {
    double cell_size;
    int32_t g0[3];
    int32_t gn[3];
    int64_t ncells;
    int64_t *cstart[ORC_MAX_ARRAYS];   /* ncells + 1 */
    int32_t *cidx[ORC_MAX_ARRAYS];     /* particle indices sorted by cell */
    int64_t *off[ORC_MAX_ARRAYS][ORC_MAX_ARRAYS];
    int32_t *idx[ORC_MAX_ARRAYS][ORC_MAX_ARRAYS];
    int64_t nn[ORC_MAX_ARRAYS];        /* dest sizes the lists were built for */
} orc_nnps;

/* ------------------------------------------------------------------ */
/* cubic spline (S/base/kernels.pyx:349-454)                          */
/* ------------------------------------------------------------------ */
static double kfac_unit(int dim)
{
    /* _fac(1.0), S/base/kernels.pyx:441-447 */
    double h = 1.0;
    if (dim == 1) return (2. / 3.) / h;
    if (dim == 2) return 10 / (7 * ORC_PI) / (h * h);
    return 1. / ORC_PI / (h * h * h);
}

static double h_dim(double h, int dim)
{
    if (dim == 1) return 1 / h;
    if (dim == 2) return 1 / (h * h);
    return 1 / (h * h * h);
}

/* CubicSplineKernel.function(pa, pb, h) */
static double cs_function(double pax, double pay, double paz,
                          double pbx, double pby, double pbz,
                          double h, int dim, double kfac)
{
    double rab = sqrt((pax - pbx) * (pax - pbx) + (pay - pby) * (pay - pby) +
                      (paz - pbz) * (paz - pbz));
    double q = rab / h;
    double val;
    double fac = h_dim(h, dim) * kfac;
    if (q > 2.0)
        val = 0.0;
    else if (q > 1.0)
        val = 0.25 * (2 - q) * (2 - q) * (2 - q);
    else
        val = 1 - 1.5 * (q * q) * (1 - 0.5 * q);
    return val * fac;
}

/* CubicSplineKernel.gradient(pa, pb, h) */
static void cs_gradient(double pax, double pay, double paz,
                        double pbx, double pby, double pbz,
                        double h, int dim, double kfac, double *g)
{
    double rab = sqrt((pax - pbx) * (pax - pbx) + (pay - pby) * (pay - pby) +
                      (paz - pbz) * (paz - pbz));
    double q = rab / h;
    double val = 0.0;
    double fac = h_dim(h, dim) * kfac;
    double rx = pax - pbx, ry = pay - pby, rz = paz - pbz;
    if (q > 2.0) {
    } else if (q >= 1.0) {
        val = -0.75 * (2 - q) * (2 - q) / (h * rab);
    } else if (q > 1e-14) {
        val = 3.0 * (0.75 * q - 1) / (h * h);
    }
    g[0] = rx * (val * fac);
    g[1] = ry * (val * fac);
    g[2] = rz * (val * fac);
}

/* QuinticSplineKernel (S/base/kernels.pyx:461-560), 2D: fac = _fac(1) =
 * 7 / (478 pi), support 3h.  As in the reference, W adds (1 - q)^5 with
 * weight 1 (not 15), and the gradient carries +5 (3-q)^4 - 30 (2-q)^4 +
 * 75 (1-q)^4, the opposite sign of dW/dq. */
static double qs_fac(void)
{
    double h = 1.0;
    return 7. / (478 * ORC_PI * h * h);
}

static double qs_function(double pax, double pay, double paz,
                          double pbx, double pby, double pbz,
                          double h, int dim, double kfac)
{
    double fac = kfac * h_dim(h, dim);
    double rab = sqrt((pax - pbx) * (pax - pbx) + (pay - pby) * (pay - pby) +
                      (paz - pbz) * (paz - pbz));
    double q = rab / h;
    double val;
    double tmp1 = (3 - q), tmp2 = (2 - q), tmp3 = (1 - q);
    if (q > 3.0) {
        val = 0.0;
    } else {
        tmp1 *= (tmp1 * tmp1 * tmp1 * tmp1);
        if (q > 2.0) {
            val = tmp1;
        } else {
            tmp2 *= (tmp2 * tmp2 * tmp2 * tmp2);
            val = tmp1 - 6 * tmp2;
            if (!(q > 1.0)) {
                tmp3 *= (tmp3 * tmp3 * tmp3 * tmp3);
                val += tmp3;
            }
        }
    }
    return val * fac;
}

static void qs_gradient(double pax, double pay, double paz,
                        double pbx, double pby, double pbz,
                        double h, int dim, double kfac, double *g)
{
    double fac = kfac * h_dim(h, dim);
    double rx = pax - pbx, ry = pay - pby, rz = paz - pbz;
    double rab = sqrt(rx * rx + ry * ry + rz * rz);
    double q = rab / h;
    double val;
    double tmp1 = (3 - q), tmp2 = (2 - q), tmp3 = (1 - q);
    if (rab < 1e-16) {
        val = 0.0;
    } else {
        fac *= 1. / (h * rab);
        if (q > 3.0) {
            val = 0.0;
        } else {
            tmp1 *= (tmp1 * tmp1 * tmp1);
            if (q > 2.0) {
                val = 5 * tmp1;
            } else {
                tmp2 *= (tmp2 * tmp2 * tmp2);
                val = 5 * tmp1 - 30 * tmp2;
                if (!(q > 1.0)) {
                    tmp3 *= (tmp3 * tmp3 * tmp3);
                    val += 75 * tmp3;
                }
            }
        }
    }
    g[0] = rx * (val * fac);
    g[1] = ry * (val * fac);
    g[2] = rz * (val * fac);
}

/* WendlandQuinticSplineKernel (S/base/kernels.pyx:562-640), 2D: support 2h;
 * _fac(h) is written (7./4*PI*h*h), so fac = _fac(1) = 7 pi / 4 as there. */
static double wq_fac(void)
{
    double h = 1.0;
    return (7. / 4 * ORC_PI * h * h);
}

static double wq_function(double pax, double pay, double paz,
                          double pbx, double pby, double pbz,
                          double h, int dim, double kfac)
{
    double fac = kfac * h_dim(h, dim);
    double rab = sqrt((pax - pbx) * (pax - pbx) + (pay - pby) * (pay - pby) +
                      (paz - pbz) * (paz - pbz));
    double q = rab / h;
    double val;
    double tmp = (1 - 0.5 * q);
    if (q > 2.0) {
        val = 0.0;
    } else {
        tmp *= (tmp * tmp * tmp);
        tmp *= (2 * q + 1);
        val = tmp;
    }
    return val * fac;
}

static void wq_gradient(double pax, double pay, double paz,
                        double pbx, double pby, double pbz,
                        double h, int dim, double kfac, double *g)
{
    double fac = kfac * h_dim(h, dim);
    double rx = pax - pbx, ry = pay - pby, rz = paz - pbz;
    double rab = sqrt(rx * rx + ry * ry + rz * rz);
    double q = rab / h;
    double val;
    double tmp = (1 - 0.5 * q);
    if (rab < 1e-16) {
        val = 0.0;
    } else {
        fac *= 1. / (h * rab);
        if (q > 2.0) {
            val = 0;
        } else {
            tmp *= (tmp * tmp);
            val = tmp * -5 * q;
        }
    }
    g[0] = rx * (val * fac);
    g[1] = ry * (val * fac);
    g[2] = rz * (val * fac);
}

/* the kernel's fac = _fac(1.0) and its function / gradient */
static double kern_fac(const orc_system *s, int dim)
{
    if (s->kernel == 3) return qs_fac();
    if (s->kernel == 4) return wq_fac();
    return kfac_unit(dim);
}

static double kern_function(int kernel, double pax, double pay, double paz,
                            double pbx, double pby, double pbz, double h, int dim,
                            double kfac)
{
    if (kernel == 3) return qs_function(pax, pay, paz, pbx, pby, pbz, h, dim, kfac);
    if (kernel == 4) return wq_function(pax, pay, paz, pbx, pby, pbz, h, dim, kfac);
    return cs_function(pax, pay, paz, pbx, pby, pbz, h, dim, kfac);
}

static void kern_gradient(int kernel, double pax, double pay, double paz,
                          double pbx, double pby, double pbz, double h, int dim,
                          double kfac, double *g)
{
    if (kernel == 3) qs_gradient(pax, pay, paz, pbx, pby, pbz, h, dim, kfac, g);
    else if (kernel == 4) wq_gradient(pax, pay, paz, pbx, pby, pbz, h, dim, kfac, g);
    else cs_gradient(pax, pay, paz, pbx, pby, pbz, h, dim, kfac, g);
}

/* W and grad W of a pair as the functions evaluate them: at h_ab =
 * (h_a + h_b) / 2, or with hks the average of the values at h_a and h_b
 * (e.g. S/sph/funcs/density_funcs.pyx:56-63, pressure_funcs.pyx:371-381). */
static double pair_w(const orc_system *s, const orc_array *D, int64_t i,
                     const orc_array *S, int64_t j, double hab, int dim, double kfac)
{
    const int k = s->kernel;
    if (s->hks) {
        double wa = kern_function(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j],
                                  D->h[i], dim, kfac);
        double wb = kern_function(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j],
                                  S->h[j], dim, kfac);
        return 0.5 * (wa + wb);
    }
    return kern_function(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j], hab, dim,
                         kfac);
}

static void pair_grad(const orc_system *s, const orc_array *D, int64_t i,
                      const orc_array *S, int64_t j, double hab, int dim, double kfac,
                      double *g)
{
    const int k = s->kernel;
    if (s->hks) {
        double ga[3], gb[3];
        kern_gradient(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j], D->h[i], dim,
                      kfac, ga);
        kern_gradient(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j], S->h[j], dim,
                      kfac, gb);
        for (int d = 0; d < 3; ++d) g[d] = (ga[d] + gb[d]) * 0.5;
        return;
    }
    kern_gradient(k, D->x[i], D->y[i], D->z[i], S->x[j], S->y[j], S->z[j], hab, dim, kfac, g);
}

double orc_kernel_w(double dx, double dy, double dz, double h, int dim)
{
    return cs_function(dx, dy, dz, 0.0, 0.0, 0.0, h, dim, kfac_unit(dim));
}

void orc_kernel_grad(double dx, double dy, double dz, double h, int dim,
                     double *g)
{
    cs_gradient(dx, dy, dz, 0.0, 0.0, 0.0, h, dim, kfac_unit(dim), g);
}

/* W and grad W of kernel type `kernel` (get_type ids) at (dx, dy, dz) */
double orc_kernel_w2(int kernel, double dx, double dy, double dz, double h, int dim)
{
    orc_system s;
    s.kernel = kernel;
    return kern_function(kernel, dx, dy, dz, 0.0, 0.0, 0.0, h, dim, kern_fac(&s, dim));
}

void orc_kernel_grad2(int kernel, double dx, double dy, double dz, double h, int dim,
                      double *g)
{
    orc_system s;
    s.kernel = kernel;
    kern_gradient(kernel, dx, dy, dz, 0.0, 0.0, 0.0, h, dim, kern_fac(&s, dim), g);
}

/* ------------------------------------------------------------------ */
/* binning (S/base/cell.pyx:44-84, :911-941, :1229-1300)              */
/* ------------------------------------------------------------------ */
static inline int real_to_int(double real_val, double step)
{
    return (int)floor(real_val / step);
}

void orc_cell_ids(int64_t n, const double *x, const double *y,
                  const double *z, double cell_size, int32_t *out)
{
    for (int64_t i = 0; i < n; ++i) {
        out[3 * i + 0] = real_to_int(x[i], cell_size);
        out[3 * i + 1] = real_to_int(y[i], cell_size);
        out[3 * i + 2] = real_to_int(z[i], cell_size);
    }
}

orc_nnps *orc_nnps_new(void)
{
    return (orc_nnps *)calloc(1, sizeof(orc_nnps));
}

static void nnps_clear(orc_nnps *c)
{
    for (int a = 0; a < ORC_MAX_ARRAYS; ++a) {
        free(c->cstart[a]);
        free(c->cidx[a]);
        c->cstart[a] = NULL;
        c->cidx[a] = NULL;
        for (int b = 0; b < ORC_MAX_ARRAYS; ++b) {
            free(c->off[a][b]);
            free(c->idx[a][b]);
            c->off[a][b] = NULL;
            c->idx[a][b] = NULL;
        }
    }
}

void orc_nnps_free(orc_nnps *c)
{
    if (!c) return;
    nnps_clear(c);
    free(c);
}

double orc_cell_size(const orc_nnps *c) { return c->cell_size; }

void orc_grid(const orc_nnps *c, int32_t *g0, int32_t *gn)
{
    for (int d = 0; d < 3; ++d) {
        g0[d] = c->g0[d];
        gn[d] = c->gn[d];
    }
}

/* CellManager.compute_cell_size: cell_size = radius_scale * max_h over all
 * binned arrays; 0 -> 1 (S/base/cell.pyx:911-941). */
static double compute_cell_size(const orc_system *s)
{
    double max_h = -INFINITY;
    int any = 0;
    for (int a = 0; a < s->narrays; ++a)
        for (int64_t i = 0; i < s->a[a].n; ++i) {
            if (!any || s->a[a].h[i] > max_h) max_h = s->a[a].h[i];
            any = 1;
        }
    if (!any) max_h = 0.0;
    double cs = s->cell_scale * max_h;
    if (cs == 0.0) cs = 1.0;
    return cs;
}

static int bin_all(const orc_system *s, orc_nnps *c)
{
    double cs = c->cell_size;
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX};
    int32_t hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    int any = 0;
    for (int a = 0; a < s->narrays; ++a) {
        const orc_array *A = &s->a[a];
        for (int64_t i = 0; i < A->n; ++i) {
            int32_t id[3] = {real_to_int(A->x[i], cs), real_to_int(A->y[i], cs),
                             real_to_int(A->z[i], cs)};
            for (int d = 0; d < 3; ++d) {
                if (id[d] < lo[d]) lo[d] = id[d];
                if (id[d] > hi[d]) hi[d] = id[d];
            }
            any = 1;
        }
    }
    if (!any) {
        for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = 0; }
    }
    int64_t ncells = 1;
    for (int d = 0; d < 3; ++d) {
        c->g0[d] = lo[d];
        c->gn[d] = hi[d] - lo[d] + 1;
        ncells *= c->gn[d];
    }
    if (ncells > ((int64_t)1 << 28)) return -2;
    c->ncells = ncells;
    for (int a = 0; a < s->narrays; ++a) {
        const orc_array *A = &s->a[a];
        int64_t *start = (int64_t *)calloc((size_t)ncells + 1, sizeof(int64_t));
        int32_t *idx = (int32_t *)malloc(sizeof(int32_t) * (size_t)(A->n > 0 ? A->n : 1));
        int64_t *key = (int64_t *)malloc(sizeof(int64_t) * (size_t)(A->n > 0 ? A->n : 1));
        if (!start || !idx || !key) { free(start); free(idx); free(key); return -3; }
        for (int64_t i = 0; i < A->n; ++i) {
            int64_t ix = real_to_int(A->x[i], cs) - lo[0];
            int64_t iy = real_to_int(A->y[i], cs) - lo[1];
            int64_t iz = real_to_int(A->z[i], cs) - lo[2];
            key[i] = (ix * c->gn[1] + iy) * c->gn[2] + iz;
            start[key[i] + 1]++;
        }
        for (int64_t k = 0; k < ncells; ++k) start[k + 1] += start[k];
        int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncells);
        if (!cur) { free(start); free(idx); free(key); return -3; }
        memcpy(cur, start, sizeof(int64_t) * (size_t)ncells);
        /* ascending particle index inside each cell, as _insert_particles
         * appends indices in order (S/base/cell.pyx:1272-1291) */
        for (int64_t i = 0; i < A->n; ++i) idx[cur[key[i]]++] = (int32_t)i;
        free(cur);
        free(key);
        c->cstart[a] = start;
        c->cidx[a] = idx;
    }
    return 0;
}

/* One dest particle's neighbours in source array `sa`, in the reference
 * order: stencil cells x-major, then y, then z (construct_immediate_neighbor_
 * list), ascending index inside a cell, strict d2 < (scale*h)^2, then self
 * swapped to the last slot when source is dest (S/base/nnps.pyx:612-619).
 * Returns the count; writes up to `cap` indices when out != NULL. */
static int64_t query(const orc_system *s, const orc_nnps *c, int da, int sa,
                     int64_t i, int32_t *out, int swap_self)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    double cs = c->cell_size;
    double px = D->x[i], py = D->y[i], pz = D->z[i];
    double radius = D->h[i] * s->radius_scale;
    double radius2 = radius * radius;
    int dist = (int)ceil(radius / cs);
    int32_t cx = real_to_int(px, cs), cy = real_to_int(py, cs),
            cz = real_to_int(pz, cs);
    int64_t cnt = 0;
    for (int di = -dist; di <= dist; ++di) {
        int64_t ix = (int64_t)cx + di - c->g0[0];
        if (ix < 0 || ix >= c->gn[0]) continue;
        for (int dj = -dist; dj <= dist; ++dj) {
            int64_t iy = (int64_t)cy + dj - c->g0[1];
            if (iy < 0 || iy >= c->gn[1]) continue;
            for (int dk = -dist; dk <= dist; ++dk) {
                int64_t iz = (int64_t)cz + dk - c->g0[2];
                if (iz < 0 || iz >= c->gn[2]) continue;
                int64_t key = (ix * c->gn[1] + iy) * c->gn[2] + iz;
                for (int64_t k = c->cstart[sa][key]; k < c->cstart[sa][key + 1]; ++k) {
                    int32_t j = c->cidx[sa][k];
                    double sx = S->x[j], sy = S->y[j], sz = S->z[j];
                    double d2 = (sx - px) * (sx - px) + (sy - py) * (sy - py) +
                                (sz - pz) * (sz - pz);
                    if (d2 < radius2) {
                        if (out) out[cnt] = j;
                        cnt++;
                    }
                }
            }
        }
    }
    if (out && da == sa && swap_self) {
        for (int64_t j = 0; j < cnt - 1; ++j) {
            if (out[j] == (int32_t)i) {
                out[j] = out[cnt - 1];
                out[cnt - 1] = (int32_t)i;
                break;
            }
        }
    }
    return cnt;
}

/* VarHNbrParticleLocator._update_cache (S/base/nnps.pyx:748-784): dest i's
 * own query (radius from h_i, no self swap), then every source j, in index
 * order, whose reversed query (radius from h_j, self swapped last) holds i
 * and that is not yet in i's list. */
static int build_lists_varh(const orc_system *s, orc_nnps *c, int da, int sa)
{
    int64_t nd = s->a[da].n, ns = s->a[sa].n;
    int64_t *cnt = (int64_t *)calloc((size_t)nd, sizeof(int64_t));
    int64_t *capa = (int64_t *)calloc((size_t)nd, sizeof(int64_t));
    int32_t **lst = (int32_t **)calloc((size_t)nd, sizeof(int32_t *));
    if (!cnt || !capa || !lst) return -3;
    for (int64_t i = 0; i < nd; ++i) {
        int64_t m = query(s, c, da, sa, i, NULL, 0);
        capa[i] = m + 8;
        lst[i] = (int32_t *)malloc(sizeof(int32_t) * (size_t)capa[i]);
        if (!lst[i]) return -3;
        cnt[i] = query(s, c, da, sa, i, lst[i], 0);
    }
    int32_t *rev = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nd + 1));
    if (!rev) return -3;
    int64_t nsr = 0;   /* the reversed locator covers the real particles */
    for (int64_t j = 0; j < ns; ++j) nsr += s->a[sa].tag[j] == 0;
    for (int64_t j = 0; j < nsr; ++j) {
        int64_t m = query(s, c, sa, da, j, NULL, 1);
        int32_t *rv = m > nd ? (int32_t *)malloc(sizeof(int32_t) * (size_t)m) : rev;
        query(s, c, sa, da, j, rv, 1);
        for (int64_t q = 0; q < m; ++q) {
            int32_t k = rv[q];
            int found = 0;
            for (int64_t t = 0; t < cnt[k]; ++t)
                if (lst[k][t] == (int32_t)j) { found = 1; break; }
            if (found) continue;
            if (cnt[k] == capa[k]) {
                capa[k] *= 2;
                lst[k] = (int32_t *)realloc(lst[k], sizeof(int32_t) * (size_t)capa[k]);
                if (!lst[k]) return -3;
            }
            lst[k][cnt[k]++] = (int32_t)j;
        }
        if (rv != rev) free(rv);
    }
    free(rev);
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nd + 1));
    if (!off) return -3;
    off[0] = 0;
    for (int64_t i = 0; i < nd; ++i) off[i + 1] = off[i] + cnt[i];
    int32_t *idx = (int32_t *)malloc(sizeof(int32_t) * (size_t)(off[nd] > 0 ? off[nd] : 1));
    if (!idx) return -3;
    for (int64_t i = 0; i < nd; ++i) {
        memcpy(idx + off[i], lst[i], sizeof(int32_t) * (size_t)cnt[i]);
        free(lst[i]);
    }
    free(lst);
    free(cnt);
    free(capa);
    c->off[da][sa] = off;
    c->idx[da][sa] = idx;
    c->nn[da] = nd;
    return 0;
}

static int build_lists(const orc_system *s, orc_nnps *c, int da, int sa)
{
    if (s->variable_h) return build_lists_varh(s, c, da, sa);
    int64_t n = s->a[da].n;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    if (!off) return -3;
    off[0] = 0;
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < n; ++i) off[i + 1] = query(s, c, da, sa, i, NULL, 1);
    for (int64_t i = 0; i < n; ++i) off[i + 1] += off[i];
    int32_t *idx = (int32_t *)malloc(sizeof(int32_t) * (size_t)(off[n] > 0 ? off[n] : 1));
    if (!idx) { free(off); return -3; }
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < n; ++i) query(s, c, da, sa, i, idx + off[i], 1);
    c->off[da][sa] = off;
    c->idx[da][sa] = idx;
    c->nn[da] = n;
    return 0;
}

static void set_threads(const orc_system *s)
{
#ifdef _OPENMP
    if (s->nthreads > 0) omp_set_num_threads(s->nthreads);
#else
    (void)s;
#endif
}

/* Particles.update(): recompute the cell size, rebin every array and rebuild
 * the cached neighbour lists of every (dest, source) pair in pair_mask
 * (bit dest*4 + source). */
int orc_update(const orc_system *s, orc_nnps *c, uint32_t pair_mask)
{
    set_threads(s);
    nnps_clear(c);
    c->cell_size = compute_cell_size(s);
    int rc = bin_all(s, c);
    if (rc) return rc;
    for (int da = 0; da < s->narrays; ++da)
        for (int sa = 0; sa < s->narrays; ++sa)
            if (pair_mask & (1u << (da * 4 + sa))) {
                rc = build_lists(s, c, da, sa);
                if (rc) return rc;
            }
    return 0;
}

int64_t orc_nbr_total(const orc_nnps *c, int da, int sa)
{
    if (!c->off[da][sa]) return -1;
    return c->off[da][sa][c->nn[da]];
}

int orc_nbr_copy(const orc_nnps *c, int da, int sa, int64_t *off, int32_t *idx)
{
    if (!c->off[da][sa]) return -1;
    int64_t n = c->nn[da];
    memcpy(off, c->off[da][sa], sizeof(int64_t) * (size_t)(n + 1));
    memcpy(idx, c->idx[da][sa], sizeof(int32_t) * (size_t)c->off[da][sa][n]);
    return 0;
}

static int cmp_i32(const void *a, const void *b)
{
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* The lists of orc_nbr_copy with each dest's list sorted ascending: the
 * canonical form neighbour sets are compared in (a comparison aid, not a
 * reference routine). */
int orc_nbr_copy_sorted(const orc_nnps *c, int da, int sa, int64_t *off, int32_t *idx,
                        int nthreads)
{
    if (orc_nbr_copy(c, da, sa, off, idx)) return -1;
    const int64_t n = c->nn[da];
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i)
        qsort(idx + off[i], (size_t)(off[i + 1] - off[i]), sizeof(int32_t), cmp_i32);
    return 0;
}

/* ------------------------------------------------------------------ */
/* SPH functions, function-level semantics of SPHFunction.eval:        */
/* out[i] += result for LocalReal dests, out[i] = 0 otherwise.          */
/* ------------------------------------------------------------------ */
int orc_sph_rho(const orc_system *s, const orc_nnps *c, int da, int sa,
                double *out1)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = 0; continue; }
        double nr = 0.0;
        double ha = D->h[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double hb = S->h[j];
            double hab = 0.5 * (ha + hb);
            double w = pair_w(s, D, i, S, j, hab, dim, kfac);
            nr += w * S->m[j];
        }
        out1[i] += nr;
    }
    return 0;
}

int orc_tait(const orc_system *s, int da, double co, double ro, double gamma,
             double *out1, double *out2)
{
    const orc_array *D = &s->a[da];
    double B = co * co * ro / gamma;
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = 0; out2[i] = 0; continue; }
        double rhoa = D->rho[i];
        double ratio = rhoa / ro;
        double gamma2 = 0.5 * (gamma - 1.0);
        double tmp = pow(ratio, gamma);
        out1[i] += (tmp - 1.0) * B;
        out2[i] += pow(ratio, gamma2) * co;
    }
    return 0;
}

int orc_momentum(const orc_system *s, const orc_nnps *c, int da, int sa,
                 double alpha, double beta, double eta, double *out1,
                 double *out2, double *out3, double *dt_fac)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = out2[i] = out3[i] = 0; continue; }
        double nr0 = 0.0, nr1 = 0.0, nr2 = 0.0;
        double ha = D->h[i];
        double ca = D->cs[i];
        double Pa = D->p[i];
        double rhoa = D->rho[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double hb = S->h[j];
            double hab = 0.5 * (ha + hb);
            double cb = S->cs[j];
            double rx = D->x[i] - S->x[j];
            double ry = D->y[i] - S->y[j];
            double rz = D->z[i] - S->z[j];
            double vx = D->u[i] - S->u[j];
            double vy = D->v[i] - S->v[j];
            double vz = D->w[i] - S->w[j];
            double dot = vx * rx + vy * ry + vz * rz;
            double rab2 = rx * rx + ry * ry + rz * rz;
            double dtf = fabs(hab * dot / (rab2 + eta * eta * hab * hab));
            dt_fac[i] = dt_fac[i] > dtf ? dt_fac[i] : dtf;
            double Pb = S->p[j];
            double rhob = S->rho[j];
            double mb = S->m[j];
            double rhoa2 = 1.0 / (rhoa * rhoa);
            double rhob2 = 1.0 / (rhob * rhob);
            double tmp = Pa * rhoa2 + Pb * rhob2;
            double piab = 0;
            if (dot < 0) {
                double cab = 0.5 * (ca + cb);
                double rhoab = 0.5 * (rhoa + rhob);
                double mu = hab * dot;
                mu /= (rab2 + eta * eta * hab * hab);
                piab = -alpha * cab * mu + beta * mu * mu;
                piab /= rhoab;
            }
            tmp += piab;
            tmp *= -mb;
            double g[3];
            pair_grad(s, D, i, S, j, hab, dim, kfac, g);
            nr0 += tmp * g[0];
            nr1 += tmp * g[1];
            nr2 += tmp * g[2];
        }
        out1[i] += nr0;
        out2[i] += nr1;
        out3[i] += nr2;
    }
    return 0;
}

/* MonaghanArtificialViscosity.eval_nbr (S/sph/funcs/viscosity_funcs.pyx:
 * 75-157), the split form of the momentum equation's viscous term: per
 * neighbour, dt_fac = max |h_ab dot / (r_ab^2 + 0.01 h_ab^2)| (the 0.01 is
 * written into the reference, :103) and, when dot < 0, a += -m_b Pi_ab
 * grad W(h_ab) with mu = h_ab dot / (r_ab^2 + eta^2 h_ab^2), where eta is
 * the function's attribute, which its constructor never sets (:30-45), so
 * 0 unless the caller assigns it. */
int orc_monaghan_av(const orc_system *s, const orc_nnps *c, int da, int sa,
                    double alpha, double beta, double eta, double *out1,
                    double *out2, double *out3, double *dt_fac)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = out2[i] = out3[i] = 0; continue; }
        double nr0 = 0.0, nr1 = 0.0, nr2 = 0.0;
        double ha = D->h[i];
        double ca = D->cs[i];
        double rhoa = D->rho[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double hb = S->h[j];
            double hab = 0.5 * (ha + hb);
            double cb = S->cs[j];
            double rx = D->x[i] - S->x[j];
            double ry = D->y[i] - S->y[j];
            double rz = D->z[i] - S->z[j];
            double vx = D->u[i] - S->u[j];
            double vy = D->v[i] - S->v[j];
            double vz = D->w[i] - S->w[j];
            double dot = vx * rx + vy * ry + vz * rz;
            double rab2 = rx * rx + ry * ry + rz * rz;
            double dtf = fabs(hab * dot / (rab2 + 0.01 * hab * hab));
            dt_fac[i] = dt_fac[i] < dtf ? dtf : dt_fac[i];
            double rhob = S->rho[j];
            double mb = S->m[j];
            double piab = 0;
            if (dot < 0) {
                double cab = 0.5 * (ca + cb);
                double rhoab = 0.5 * (rhoa + rhob);
                double mu = hab * dot;
                mu /= (rab2 + eta * eta * hab * hab);
                piab = -alpha * cab * mu + beta * mu * mu;
                piab /= rhoab;
            }
            double tmp = piab;
            tmp *= -mb;
            double g[3];
            pair_grad(s, D, i, S, j, hab, dim, kfac, g);
            nr0 += tmp * g[0];
            nr1 += tmp * g[1];
            nr2 += tmp * g[2];
        }
        out1[i] += nr0;
        out2[i] += nr1;
        out3[i] += nr2;
    }
    return 0;
}

int orc_pgrad(const orc_system *s, const orc_nnps *c, int da, int sa,
              double *out1, double *out2, double *out3)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = out2[i] = out3[i] = 0; continue; }
        double nr0 = 0.0, nr1 = 0.0, nr2 = 0.0;
        double ha = D->h[i];
        double pa = D->p[i];
        double rhoa = D->rho[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double mb = S->m[j];
            double rhob = S->rho[j];
            double pb = S->p[j];
            double hb = S->h[j];
            double h = 0.5 * (ha + hb);
            double rhoa2 = 1.0 / (rhoa * rhoa);
            double rhob2 = 1.0 / (rhob * rhob);
            double temp = -mb * (pa * rhoa2 + pb * rhob2);
            double artificial_stress = 0.0;
            temp = temp + artificial_stress;
            double g[3];
            pair_grad(s, D, i, S, j, h, dim, kfac, g);
            nr0 += temp * g[0];
            nr1 += temp * g[1];
            nr2 += temp * g[2];
        }
        out1[i] += nr0;
        out2[i] += nr1;
        out3[i] += nr2;
    }
    return 0;
}

/* SPHDensityRate.eval_nbr (S/sph/funcs/density_funcs.pyx:119-156), hks
 * off: drho_a += ((v_a - v_b) . grad_a W(r_ab, h_ab)) m_b. */
int orc_density_rate(const orc_system *s, const orc_nnps *c, int da, int sa,
                     double *out1)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = 0; continue; }
        double nr = 0.0;
        double ha = D->h[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double hb = S->h[j];
            double hab = 0.5 * (ha + hb);
            double vx = D->u[i] - S->u[j];
            double vy = D->v[i] - S->v[j];
            double vz = D->w[i] - S->w[j];
            double g[3];
            pair_grad(s, D, i, S, j, hab, dim, kfac, g);
            double dot = vx * g[0] + vy * g[1] + vz * g[2];
            nr += dot * S->m[j];
        }
        out1[i] += nr;
    }
    return 0;
}

/* XSPHCorrection.eval_nbr_csph (S/sph/funcs/xsph_funcs.pyx:40-86), hks and
 * kernel correction off, so the CSPH denominator stays 0 and is not applied
 * (S/sph/sph_func.pyx:513-531): x_a' += eps m_b W_ab (v_b - v_a) / rho_ab,
 * rho_ab = (rho_b + rho_a) / 2. */
int orc_xsph(const orc_system *s, const orc_nnps *c, int da, int sa, double eps,
             double *out1, double *out2, double *out3)
{
    const orc_array *D = &s->a[da];
    const orc_array *S = &s->a[sa];
    const int64_t *off = c->off[da][sa];
    const int32_t *idx = c->idx[da][sa];
    if (!off) return -1;
    int dim = s->dim;
    double kfac = kern_fac(s, dim);
    set_threads(s);
#pragma omp parallel for schedule(dynamic, 512)
    for (int64_t i = 0; i < D->n; ++i) {
        if (D->tag[i] != 0) { out1[i] = out2[i] = out3[i] = 0; continue; }
        double nr0 = 0.0, nr1 = 0.0, nr2 = 0.0;
        double ha = D->h[i];
        for (int64_t k = off[i]; k < off[i + 1]; ++k) {
            int32_t j = idx[k];
            double hb = S->h[j];
            double hab = 0.5 * (ha + hb);
            double rhoab = 0.5 * (S->rho[j] + D->rho[i]);
            double vbx = S->u[j] - D->u[i];
            double vby = S->v[j] - D->v[i];
            double vbz = S->w[j] - D->w[i];
            double mb = S->m[j];
            double w = pair_w(s, D, i, S, j, hab, dim, kfac);
            double temp = mb * w / rhoab;
            nr0 += temp * vbx * eps;
            nr1 += temp * vby * eps;
            nr2 += temp * vbz * eps;
        }
        out1[i] += nr0;
        out2[i] += nr1;
        out3[i] += nr2;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* the pinned scheme: SPHRho -> Tait -> MomentumEquation -> Gravity ->  */
/* PositionStepping, evaluated as Integrator.eval does                  */
/* ------------------------------------------------------------------ */
static uint32_t pair_mask_of(const orc_system *s)
{
    uint32_t mask = 0;
    for (int d = 0; d < s->narrays; ++d)
        for (int a = 0; a < s->narrays; ++a)
            if ((s->rho_src[d] | s->mom_src[d] | s->rate_src[d] | s->xsph_src[d]) &
                (1u << a))
                mask |= 1u << (d * 4 + a);
    return mask;
}

uint32_t orc_scheme_pairs(const orc_system *s) { return pair_mask_of(s); }

int orc_eval(orc_system *s, const orc_nnps *c)
{
    int rc;
    /* SPHRho: non-integrating calc resets rho, _tmpy, _tmpz then adds each
     * source in array order */
    for (int d = 0; d < s->narrays; ++d) {
        if (!s->rho_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) D->rho[i] = 0.0;
        for (int a = 0; a < s->narrays; ++a)
            if (s->rho_src[d] & (1u << a)) {
                rc = orc_sph_rho(s, c, d, a, D->rho);
                if (rc) return rc;
                s->pairs += c->off[d][a][D->n];
            }
    }
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->tait_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) { D->p[i] = 0.0; D->cs[i] = 0.0; }
        orc_tait(s, d, s->c0, s->rho0, s->gamma_eos, D->p, D->cs);
    }
    /* SPHDensityRate (the continuity scheme): integrating, adds into
     * _a_rho_1 source by source */
    for (int d = 0; d < s->narrays; ++d) {
        if (!s->rate_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int a = 0; a < s->narrays; ++a)
            if (s->rate_src[d] & (1u << a)) {
                rc = orc_density_rate(s, c, d, a, D->arho);
                if (rc) return rc;
                s->pairs += c->off[d][a][D->n];
            }
    }
    /* the split form: SPHPressureGradient's calc, then
     * MonaghanArtificialViscosity's (its to_reset clears dt_fac), each
     * adding into the accelerations source by source */
    if (s->split_av) {
        for (int d = 0; d < s->narrays; ++d) {
            if (!s->mom_src[d]) continue;
            const orc_array *D = &s->a[d];
            for (int a = 0; a < s->narrays; ++a)
                if (s->mom_src[d] & (1u << a)) {
                    rc = orc_pgrad(s, c, d, a, D->au, D->av, D->aw);
                    if (rc) return rc;
                    s->pairs += c->off[d][a][D->n];
                }
        }
        for (int d = 0; d < s->narrays; ++d) {
            if (!s->mom_src[d]) continue;
            const orc_array *D = &s->a[d];
            for (int64_t i = 0; i < D->n; ++i) D->dt_fac[i] = 0.0;
            for (int a = 0; a < s->narrays; ++a)
                if (s->mom_src[d] & (1u << a)) {
                    rc = orc_monaghan_av(s, c, d, a, s->alpha, s->beta, s->av_eta, D->au,
                                         D->av, D->aw, D->dt_fac);
                    if (rc) return rc;
                    s->pairs += c->off[d][a][D->n];
                }
        }
    }
    /* accelerations were reset by reset_accelerations; dt_fac by to_reset */
    for (int d = 0; d < s->narrays && !s->split_av; ++d) {
        if (!s->mom_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) D->dt_fac[i] = 0.0;
        for (int a = 0; a < s->narrays; ++a)
            if (s->mom_src[d] & (1u << a)) {
                rc = orc_momentum(s, c, d, a, s->alpha, s->beta, s->eta, D->au,
                                  D->av, D->aw, D->dt_fac);
                if (rc) return rc;
                s->pairs += c->off[d][a][D->n];
            }
    }
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->step_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) {
            if (D->tag[i] != 0) {
                D->au[i] = D->av[i] = D->aw[i] = 0;
                D->ax[i] = D->ay[i] = D->az[i] = 0;
                continue;
            }
            D->au[i] += s->gx;
            D->av[i] += s->gy;
            D->aw[i] += s->gz;
            D->ax[i] = D->u[i];
            D->ay[i] = D->v[i];
            D->az[i] = D->w[i];
        }
    }
    /* XSPHCorrection: integrating, updates x, y (z) after PositionStepping */
    for (int d = 0; d < s->narrays; ++d) {
        if (!s->xsph_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int a = 0; a < s->narrays; ++a)
            if (s->xsph_src[d] & (1u << a)) {
                rc = orc_xsph(s, c, d, a, s->xsph_eps, D->ax, D->ay, D->az);
                if (rc) return rc;
                s->pairs += c->off[d][a][D->n];
            }
    }
    return 0;
}

static void reset_acc(const orc_system *s)
{
    for (int d = 0; d < s->narrays; ++d) {
        if (s->rate_src[d]) {
            const orc_array *D = &s->a[d];
            for (int64_t i = 0; i < D->n; ++i) D->arho[i] = 0.0;
        }
    }
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->step_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) {
            D->au[i] = D->av[i] = D->aw[i] = 0.0;
            D->ax[i] = D->ay[i] = D->az[i] = 0.0;
        }
    }
}

/* Integrator.step: prop = initial + step_arr * dt (numpy, no FMA) */
static void half_step(const orc_system *s, double dt)
{
    for (int d = 0; d < s->narrays; ++d) {
        if (!s->rate_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) {
            double t = D->arho[i] * dt;
            D->rho[i] = D->rho0[i] + t;
        }
    }
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->step_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) {
            double t;
            t = D->ax[i] * dt; D->x[i] = D->x0[i] + t;
            t = D->ay[i] * dt; D->y[i] = D->y0[i] + t;
            t = D->au[i] * dt; D->u[i] = D->u0[i] + t;
            t = D->av[i] * dt; D->v[i] = D->v0[i] + t;
            if (s->dim == 3) {
                t = D->az[i] * dt; D->z[i] = D->z0[i] + t;
                t = D->aw[i] * dt; D->w[i] = D->w0[i] + t;
            }
        }
    }
}

/* One PredictorCorrectorIntegrator.integrate(dt) preceded by the
 * particles.update() of Solver.solve (S/solver/solver.py:546-566). */
int orc_pc_step(orc_system *s, orc_nnps *c, double dt)
{
    uint32_t pm = pair_mask_of(s);
    int rc = orc_update(s, c, pm);
    if (rc) return rc;
    for (int d = 0; d < s->narrays; ++d)
        if (s->rate_src[d])
            memcpy(s->a[d].rho0, s->a[d].rho, sizeof(double) * (size_t)s->a[d].n);
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->step_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        memcpy(D->x0, D->x, sizeof(double) * (size_t)D->n);
        memcpy(D->y0, D->y, sizeof(double) * (size_t)D->n);
        memcpy(D->u0, D->u, sizeof(double) * (size_t)D->n);
        memcpy(D->v0, D->v, sizeof(double) * (size_t)D->n);
        if (s->dim == 3) {
            memcpy(D->z0, D->z, sizeof(double) * (size_t)D->n);
            memcpy(D->w0, D->w, sizeof(double) * (size_t)D->n);
        }
    }
    double half = dt / 2;
    reset_acc(s);
    rc = orc_eval(s, c);
    if (rc) return rc;
    half_step(s, half);
    rc = orc_update(s, c, pm);
    if (rc) return rc;
    reset_acc(s);
    rc = orc_eval(s, c);
    if (rc) return rc;
    half_step(s, half);
    for (int d = 0; d < s->narrays; ++d) {
        if (!s->rate_src[d]) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) D->rho[i] = 2 * D->rho[i] - D->rho0[i];
    }
    for (int d = 0; d < s->narrays; ++d) {
        if (!(s->step_on & (1u << d))) continue;
        const orc_array *D = &s->a[d];
        for (int64_t i = 0; i < D->n; ++i) {
            D->x[i] = 2 * D->x[i] - D->x0[i];
            D->y[i] = 2 * D->y[i] - D->y0[i];
            D->u[i] = 2 * D->u[i] - D->u0[i];
            D->v[i] = 2 * D->v[i] - D->v0[i];
            if (s->dim == 3) {
                D->z[i] = 2 * D->z[i] - D->z0[i];
                D->w[i] = 2 * D->w[i] - D->w0[i];
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* the other integrators (S/solver/integrator.py:420-609), each preceded  */
/* by the Solver's particles.update() like orc_pc_step                    */
/* ------------------------------------------------------------------ */
static void save_initial(const orc_system *s)
{
    for (int d = 0; d < s->narrays; ++d) {
        const orc_array *D = &s->a[d];
        size_t nb = sizeof(double) * (size_t)D->n;
        if (s->rate_src[d]) memcpy(D->rho0, D->rho, nb);
        if (!(s->step_on & (1u << d))) continue;
        memcpy(D->x0, D->x, nb);
        memcpy(D->y0, D->y, nb);
        memcpy(D->u0, D->u, nb);
        memcpy(D->v0, D->v, nb);
        if (s->dim == 3) {
            memcpy(D->z0, D->z, nb);
            memcpy(D->w0, D->w, nb);
        }
    }
}

/* the rates of every stepped property, in a fixed order: x y z u v w rho */
#define ORC_NRATES 7
static double *rate_ptr(const orc_system *s, int d, int r)
{
    const orc_array *D = &s->a[d];
    int stepped = (s->step_on >> d) & 1u;
    switch (r) {
    case 0: return stepped ? D->ax : NULL;
    case 1: return stepped ? D->ay : NULL;
    case 2: return stepped && s->dim == 3 ? D->az : NULL;
    case 3: return stepped ? D->au : NULL;
    case 4: return stepped ? D->av : NULL;
    case 5: return stepped && s->dim == 3 ? D->aw : NULL;
    default: return s->rate_src[d] ? D->arho : NULL;
    }
}
static double *prop_ptr(const orc_system *s, int d, int r, int initial)
{
    const orc_array *D = &s->a[d];
    double *p[ORC_NRATES] = {D->x, D->y, D->z, D->u, D->v, D->w, D->rho};
    double *p0[ORC_NRATES] = {D->x0, D->y0, D->z0, D->u0, D->v0, D->w0, D->rho0};
    return initial ? p0[r] : p[r];
}

/* kind 0: EulerIntegrator.integrate (:420-447); 1: RK2Integrator (:452-499);
 * 2: RK4Integrator (:504-609). */
int orc_integrate(orc_system *s, orc_nnps *c, double dt, int kind)
{
    uint32_t pm = pair_mask_of(s);
    int rc = orc_update(s, c, pm);
    if (rc) return rc;
    save_initial(s);
    if (kind == 0 || kind == 1) {
        reset_acc(s);
        rc = orc_eval(s, c);
        if (rc) return rc;
        half_step(s, kind == 0 ? dt : dt / 2);
        if (kind == 0) return 0;
        rc = orc_update(s, c, pm);
        if (rc) return rc;
        reset_acc(s);
        rc = orc_eval(s, c);
        if (rc) return rc;
        half_step(s, dt);
        return 0;
    }
    if (kind != 2) return -1;
    /* RK4: K1..K3 kept per stepped property */
    double *K[3][ORC_MAX_ARRAYS][ORC_NRATES];
    memset(K, 0, sizeof(K));
    for (int d = 0; d < s->narrays; ++d)
        for (int r = 0; r < ORC_NRATES; ++r)
            if (rate_ptr(s, d, r))
                for (int q = 0; q < 3; ++q)
                    K[q][d][r] = (double *)malloc(sizeof(double) * (size_t)(s->a[d].n + 1));
    const double h[3] = {dt / 2, dt / 2, dt};
    for (int q = 0; q < 4; ++q) {
        if (q > 0) {
            rc = orc_update(s, c, pm);
            if (rc) break;
        }
        reset_acc(s);
        rc = orc_eval(s, c);
        if (rc) break;
        if (q < 3) {
            for (int d = 0; d < s->narrays; ++d)
                for (int r = 0; r < ORC_NRATES; ++r)
                    if (K[q][d][r])
                        memcpy(K[q][d][r], rate_ptr(s, d, r), sizeof(double) * (size_t)s->a[d].n);
            half_step(s, h[q]);
            continue;
        }
        /* X = X0 + fac dt (K1 + 2 K2 + 2 K3 + K4), numpy's order */
        double fdt = (1.0 / 6.0) * dt;
        for (int d = 0; d < s->narrays; ++d)
            for (int r = 0; r < ORC_NRATES; ++r) {
                double *k4 = rate_ptr(s, d, r);
                if (!k4) continue;
                double *x = prop_ptr(s, d, r, 0), *x0 = prop_ptr(s, d, r, 1);
                for (int64_t i = 0; i < s->a[d].n; ++i) {
                    double t = K[0][d][r][i] + 2 * K[1][d][r][i];
                    t = t + 2 * K[2][d][r][i];
                    t = t + k4[i];
                    t = fdt * t;
                    x[i] = x0[i] + t;
                }
            }
    }
    for (int q = 0; q < 3; ++q)
        for (int d = 0; d < ORC_MAX_ARRAYS; ++d)
            for (int r = 0; r < ORC_NRATES; ++r) free(K[q][d][r]);
    return rc;
}
