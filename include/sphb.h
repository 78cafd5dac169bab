/*
 * sphb.h -- C ABI of the B200 (sm_100a) PySPH particle-update engine.
 *
 * Plain C: device pointers, sizes, a CUDA stream passed as void*, int status.
 * The library never allocates device memory: the caller owns every buffer,
 * including the scratch workspace whose size sphb_workspace_layout reports.
 * Calls are stream-ordered and asynchronous; concurrent use on different
 * streams is safe when the engines (and so their buffers) are distinct.
 *
 * Each entry point names the reference interface it replaces (paths in the
 * PySPH project, S/ = source/pysph/).  The reference binds its particle path
 * through OpenCL kernel signatures assembled by SPHFunction.set_cl_kernel_args
 * (S/sph/sph_func.pyx:295-351) plus the locator arguments of
 * RadixSortNeighborLocator (S/base/locator.py:576-600); here each of those
 * kernels is one entry point over an engine descriptor instead.
 *
 * Particle storage ("engine order"): all particles of all scenes in one SoA
 * set, grouped in segments (scene s, array a) at fixed offsets
 * seg_offset[s*A + a], and sorted by cell inside each segment after every
 * sphb_bin.  idx[k] maps engine position k back to the particle's index in
 * its ParticleArray.
 */
#ifndef SPHB_H
#define SPHB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPHB_MAX_ARRAYS 4
#define SPHB_ABI_VERSION 2

#if defined(__GNUC__)
#define SPHB_API __attribute__((visibility("default")))
#else
#define SPHB_API
#endif

/* return codes of every entry point */
enum {
    SPHB_OK = 0,
    SPHB_ERR_ARG = -1,          /* bad argument (NULL, size, mode) */
    SPHB_ERR_WORKSPACE = -2,    /* a buffer is smaller than required */
    SPHB_ERR_CUDA = -3,         /* a launch failed (sphb_last_cuda_error) */
    SPHB_ERR_UNSUPPORTED = -4   /* dim / precision / stencil not built */
};

/* device status word bits (sphb_engine.work.status); kernels OR them in */
enum {
    SPHB_ST_GRID_OVERFLOW = 1u << 0,  /* cells needed > cell_capacity */
    SPHB_ST_NONFINITE_POS = 1u << 1,  /* NaN/Inf position met while binning */
    SPHB_ST_OUT_OF_GRID = 1u << 2,    /* a particle fell outside its scene grid */
    SPHB_ST_NONFINITE_RHO = 1u << 3,  /* NaN/Inf density or pressure */
    SPHB_ST_NONFINITE_ACC = 1u << 4,  /* NaN/Inf acceleration */
    SPHB_ST_BAD_INDEX = 1u << 5,      /* an index failed its bounds check */
    SPHB_ST_NBR_CAPACITY = 1u << 6,   /* neighbour list output too small */
    SPHB_ST_STAGE_TIMEOUT = 1u << 7   /* a tiled pass's shared-memory staging
                                         did not complete in its wait limit
                                         (the block's dests were skipped) */
};

enum { SPHB_FP64 = 0, SPHB_FP32C = 1 };   /* plain FP64 / FP32 + Kahan */

/* Smoothing kernels, numbered as KernelBase.get_type (S/base/kernels.pyx:
 * 31-40).  The quintic spline (support 3h) and the Wendland quintic
 * (support 2h) are 2D only, as in the reference; 0 means the cubic. */
enum {
    SPHB_KERNEL_CUBIC = 1,      /* CubicSplineKernel, support 2h */
    SPHB_KERNEL_QUINTIC = 3,    /* QuinticSplineKernel */
    SPHB_KERNEL_WENDLAND = 4    /* WendlandQuinticSplineKernel */
};

/* Engine-wide configuration. */
typedef struct {
    int32_t dim;            /* 2 or 3 */
    int32_t precision;      /* SPHB_FP64 or SPHB_FP32C */
    int32_t num_scenes;     /* S >= 1 */
    int32_t num_arrays;     /* A, arrays per scene, 1..SPHB_MAX_ARRAYS */
    int32_t stencil;        /* R: cell size = support / R; 1 or 2 */
    int32_t lanes;          /* lanes per dest particle in pair kernels: 1,2,4,8 */
    int32_t pair_block;     /* threads per block of the pair kernels, 32..256 */
    int32_t num_particles;  /* total over all segments */
    int32_t cell_capacity;  /* cell table capacity (all scenes, all arrays) */
    int32_t list_batch;     /* list entries the FP32C force pass loads ahead
                               per thread: 2 or 4 (0: 4) */
    /* the scheme, per array index (identical for every scene):
     * SPHRho sources, MomentumEquation sources (bitmasks over arrays),
     * TaitEquation dests and integrated arrays (bitmasks) */
    uint32_t rho_src[SPHB_MAX_ARRAYS];
    uint32_t mom_src[SPHB_MAX_ARRAYS];
    uint32_t tait_on;
    uint32_t step_on;
    /* continuity-equation scheme (the reference's dam-break / FluidSolver
     * scheme): SPHDensityRate sources per dest array (its rho is integrated,
     * buf.rho / rho0 must be set) and XSPHCorrection sources per dest array
     * (added to the position rate of the integrated arrays); all zero for
     * the summation-density scheme */
    uint32_t rate_src[SPHB_MAX_ARRAYS];
    uint32_t xsph_src[SPHB_MAX_ARRAYS];
    int32_t kernel;         /* SPHB_KERNEL_*; scene.radius_scale must be its
                               support (3 for the quintic, else 2) */
    int32_t pair_mode;      /* how the pair passes find neighbours:
                               SPHB_PAIRS_LISTS (0): neighbour lists recorded
                               by sphb_density (f.nbr, list_cap slots) and
                               read back by later passes;
                               SPHB_PAIRS_TILED (1): every pass searches the
                               stencil cells of a block's dests from shared
                               memory, where the block stages their
                               particles' records (2D FP32C, fixed h per
                               pair (no variable_h / hks), summation
                               density scheme); no lists */
} sphb_config;

enum { SPHB_PAIRS_LISTS = 0, SPHB_PAIRS_TILED = 1 };

/* Per-scene constants, written by the host once. */
typedef struct {
    double cell_size;       /* radius_scale * max h / stencil */
    double radius_scale;    /* kernel support in units of h (2, cubic spline) */
    double h_min;           /* min h over the integrated arrays (CFL) */
    double c0, rho0, gamma, B;   /* TaitEquation, B = c0*c0*rho0/gamma */
    double alpha, beta, eta;     /* MomentumEquation */
    double g[3];                 /* GravityForce */
    double cfl, dt_initial;      /* ViscousAndForceBasedTimeStep */
    double static_lo[3];    /* bounds of the particles the integrator never */
    double static_hi[3];    /*   moves (+inf / -inf when there are none);
                               informative, every rebin measures all */
    int32_t use_cfl;        /* 0: dt kept as set; 1: viscous + force CFL rule;
                               2: viscous rule only (ViscousTimeStep) */
    int32_t uniform_h;      /* 1: every particle of the scene has the same h
                               (the FP32 pair passes then take h_ab, 1/h_ab
                               and the kernel normalisation from the dest) */
    double skin_max;        /* list skin: lists hold every pair within
                               (radius_scale h + skin_max)(1 + 1e-5) and
                               stay valid while no particle has moved
                               skin_max / 2 from where it was binned
                               (0: lists serve one stage only) */
    double xsph_eps;        /* XSPHCorrection eps */
    int32_t variable_h;     /* 1: symmetric neighbour lists, r < radius_scale
                               max(h_a, h_b) (VarHNbrParticleLocator,
                               S/base/nnps.pyx:691-786); 0: r < radius_scale
                               h_a (FixedDestNbrParticleLocator).  The cells
                               must cover radius_scale times the largest h */
    int32_t hks;            /* 1: every pair function averages its kernel over
                               h_a and h_b instead of using (h_a + h_b) / 2
                               (the functions' `hks` option) */
} sphb_scene;

/* Per-scene state, written by the kernels (host may seed dt, t, count). */
typedef struct {
    int32_t lo[3];          /* global cell coordinates of local cell (0,0,0) */
    int32_t n[3];           /* grid dimensions (n[2] == 1 in 2D) */
    int32_t cell_base;      /* first cell key of the scene */
    int32_t ncells;         /* cells per array of this scene */
    unsigned long long box[6];  /* order-encoded min xyz, max xyz of the
                                   particles at the last rebin */
    double dt;              /* time step used by the next integrator stage */
    double t;               /* simulated time */
    long long count;        /* completed steps */
    unsigned long long max_dtfac;  /* bits of max dt_fac (double, >= 0) */
    unsigned long long max_acc2;   /* bits of max |a|^2 (double, >= 0) */
    unsigned long long max_disp2;  /* bits of max |x - x_bin|^2 over the
                                      particles, from the last
                                      sphb_pc_stage (x_bin: position at the
                                      last rebin) */
} sphb_scene_state;

/* Contiguous particle range inside one segment; launch unit of every
 * particle kernel. */
typedef struct {
    int32_t seg;            /* s * A + a */
    int32_t begin, end;     /* engine positions [begin, end) */
    int32_t pad0;
} sphb_tile;

/* Double-buffered particle state (engine order, FP64 masters). */
typedef struct {
    double *x, *y, *z, *u, *v, *w;      /* z, w unused (may be NULL) in 2D */
    double *x0, *y0, *z0, *u0, *v0, *w0;
    double *m, *h;
    int32_t *idx;           /* index inside the particle's ParticleArray */
    int32_t *tag;           /* 0 == LocalReal (S/base/particle_array.pxd:20) */
    double *rho, *rho0;     /* integrated density and its stage-initial copy
                               (continuity scheme; may be NULL otherwise) */
    double *kx, *ky, *kz, *ku, *kv, *kw, *krho;
                            /* RK4's running sum K1 + 2 K2 + 2 K3 of each
                               integrated property (stage kinds 4-7; may be
                               NULL otherwise), carried by rebins with
                               SPHB_BIN_MOVE_INITIAL like x0 */
} sphb_buffers;

/* Fields recomputed every stage, in the current engine order.  Element type
 * T is double for SPHB_FP64, float for SPHB_FP32C. */
typedef struct {
    void *rho, *p, *cs;     /* T[N] (FP64 only; FP32C keeps them in thermo) */
    void *au, *av, *aw;     /* T[N]  _a_u_1, _a_v_1, _a_w_1 */
    void *dt_fac;           /* T[N]  MomentumEquation dt_fac */
    void *geo;              /* FP32C float4[N]: 2D {xr,yr,h,m}, 3D {xr,yr,zr,h} */
    void *mass;             /* FP32C 3D float[N]: m */
    void *vel;              /* FP32C: 2D float2 {u,v}, 3D float4 {u,v,w,0} */
    void *thermo;           /* FP32C float4[N]: {rho, p, cs, p/rho^2} */
    int32_t *cell;          /* local cell index of each particle */
    /* Neighbour lists of the last sphb_density pass (optional, may be
     * NULL): uint32 [list_cap][N] slot-major, entry = j | cell offsets
     * (SPHB_NBR_* packing), and int32 [lanes][N] entries per lane (-1 when
     * a lane overflowed its list_cap / lanes slots). */
    uint32_t *nbr;
    int32_t *nbr_cnt;
    /* Optional (NULL: no list reuse across stages): FP32 position of every
     * particle at its last rebin, relative to the origin of its cell; 2D
     * float2, 3D float4 {x, y, z, 0}.  sphb_pc_stage measures how far the
     * particles have moved from it. */
    void *anchor;
    /* continuity scheme outputs of sphb_momentum (T[N]; may be NULL
     * otherwise): _a_rho_1 of SPHDensityRate and the XSPHCorrection
     * velocity that sphb_pc_stage adds to the position rate */
    void *drho;
    void *xu, *xv, *xw;
    /* Optional (FP32C): the second copy of the pair records for the
     * integrator stage fused into sphb_momentum (SPHB_FORCE_STAGE): the
     * pass reads geo / vel and writes the moved particles' new records
     * here, so the caller swaps geo <-> geo_next and vel <-> vel_next after
     * it.  When set, the rebin and sphb_refresh write both copies. */
    void *geo_next, *vel_next;
    int32_t list_cap;       /* slots per particle, 0 = no lists */
    int32_t pad0;
} sphb_fields;

/* List entry packing: particle index in the low bits, each cell offset
 * (-2..2) + 2 in 3 bits above it.  2D: 26 index bits; 3D: 23. */
#define SPHB_NBR_IDX_BITS_2D 26
#define SPHB_NBR_IDX_BITS_3D 23

/* Scratch; carve it from one buffer with sphb_workspace_layout. */
typedef struct {
    int32_t *count;         /* [cell_capacity], zero between bins */
    int32_t *start;         /* [cell_capacity + 1] */
    int32_t *key;           /* [N] */
    int32_t *slot;          /* [N] */
    int32_t *perm;          /* [N] */
    int32_t *bsum;          /* [scan blocks + 1 + 64]: the scan's chunk totals,
                               then the rebin's grid-barrier word and the
                               arrival count of a launch that keeps the
                               cells (both zero when the workspace is first
                               used; the barrier word's low 31 bits and the
                               count return to zero after every launch) */
    int32_t *meta;          /* [8]  meta[0] = cells in use (all scenes);
                               meta[1] = 1 when the last rebin decision
                               rebinned; meta[2] = 1 when it kept the lists
                               (cleared by anything that moves particles);
                               meta[3] = 2 while the positions are those of
                               the last rebin; meta[4] = 1 when the lists
                               were recorded with the skin at them;
                               meta[5] = 1 after the host wrote positions or
                               velocities, until sphb_refresh has rebuilt the
                               records and measured the displacements */
    unsigned int *status;   /* [1]  SPHB_ST_* bits, cleared by the host */
    unsigned long long *pairs;  /* [4]  pairs evaluated: density, force;
                                   [2]: blocks of the tiled passes that read
                                   their records from global memory (their
                                   ranges exceeded the shared memory); [3]:
                                   rebins the device decisions ran
                                   (SPHB_BIN_IF_NEEDED) */
} sphb_work;

/* Everything the kernels see.  Tables are device pointers. */
typedef struct {
    sphb_config cfg;
    const int32_t *seg_offset;      /* [S*A + 1] */
    const sphb_scene *scene;        /* [S] */
    sphb_scene_state *sstate;       /* [S] */
    const sphb_tile *tiles;         /* elementwise tiles (256 particles) */
    const sphb_tile *pair_tiles;    /* pair-kernel tiles (pair_block/lanes) */
    int32_t num_tiles;
    int32_t num_pair_tiles;
    sphb_buffers buf[2];
    sphb_fields f;
    sphb_work work;
} sphb_engine;

/* ---- host-side helpers (no device work) ---------------------------- */

SPHB_API int sphb_abi_version(void);

/* Number of tiles of at most tile_size particles covering the segments
 * seg_offset[0..nseg]; writes them to `tiles` (host memory) when non-NULL. */
SPHB_API int sphb_make_tiles(const int32_t *seg_offset_host, int32_t nseg,
                    int32_t tile_size, sphb_tile *tiles, int32_t *num_tiles);

/* Byte offsets of the sphb_work members inside one workspace buffer
 * (offsets[0..8] in member order, 256-byte aligned) and its total size.
 * Replaces the buffer sizing of RadixSortManager._setup_buffers
 * (S/base/domain_manager.py:840-899). */
SPHB_API int sphb_workspace_layout(const sphb_config *cfg, size_t offsets[9],
                          size_t *total_bytes);

/* Last CUDA error string seen by this thread ("" when none). */
SPHB_API const char *sphb_last_cuda_error(void);

/* ---- device entry points ------------------------------------------ */

/* Bounding box of every particle of every scene into sstate[].box; run it
 * after the host writes positions.  Replaces DomainManager._find_bounds
 * (S/base/domain_manager.py:94-131). */
SPHB_API int sphb_box_init(const sphb_engine *e, int cur, void *stream);

/* Rebin: grid per scene from the accumulated box, cell key per particle,
 * counting sort (stable by engine position), per-cell start table, and the
 * gather of buf[cur] into buf[cur^1] plus the FP32 pair records.  Replaces
 * CellManager.update/_rebin_particles (S/base/cell.pyx:943-986, :1179-1300),
 * RadixSortManager._cl_update (S/base/domain_manager.py:901-972) and the
 * `bin` / `compute_cell_counts` kernels (S/base/radix_sort.cl:31-108).
 * Every rebin first measures each scene's box from all its particles.
 * flags: SPHB_BIN_MOVE_INITIAL carries x0..w0 too; SPHB_BIN_BOX is accepted
 * and has no further effect. */
#define SPHB_BIN_MOVE_INITIAL 1
#define SPHB_BIN_BOX 2
/* SPHB_BIN_IF_NEEDED (needs f.anchor): the device decides whether to
 * rebin.  It does not while the particles are where the last rebin put them
 * (work.meta[3] == 2); otherwise it rebins unless the lists were recorded
 * with the skin right after the last rebin (work.meta[4]) and no particle
 * has moved skin_max / 2 since (max_disp2 of the last sphb_pc_stage).  The
 * decision goes to work.meta[1] and [2].  A rebin then
 * gathers into buf[cur ^ 1] and copies the result back into buf[cur], so
 * the state stays in buf[cur] whatever the decision: the caller does not
 * flip cur, and one captured graph serves every step.  Between rebins the
 * lists, the cell tables and the cell of each particle stay those of the
 * last rebin; they remain complete because no pair can close from beyond
 * support + skin while every particle stays within skin / 2 of its binned
 * position.  Without the flag, sphb_bin always rebins into buf[cur ^ 1]. */
#define SPHB_BIN_IF_NEEDED 4
/* SPHB_BIN_STEP_BEGIN (with SPHB_BIN_IF_NEEDED only): the decision first
 * runs sphb_step_begin's prologue for every scene, in the same launch, so
 * that a step's first bin replaces the sphb_step_begin call. */
#define SPHB_BIN_STEP_BEGIN 8
SPHB_API int sphb_bin(const sphb_engine *e, int cur, int flags, void *stream);

/* Neighbour lists of every particle of the dest arrays in dest_mask among
 * the source arrays in src_mask, FP64 predicate r^2 < (radius_scale*h_dest)^2
 * on the master positions (FixedDestNbrParticleLocator._update_cache,
 * S/base/nnps.pyx:596-621).  counts[k] (engine order) always; when
 * nbr_offsets != NULL (exclusive prefix of counts, host computed) the engine
 * positions of the neighbours are written to nbr_index[nbr_offsets[k]..]. */
SPHB_API int sphb_neighbors(const sphb_engine *e, int cur, uint32_t dest_mask,
                   uint32_t src_mask, int32_t *counts,
                   const int64_t *nbr_offsets, int32_t *nbr_index,
                   int64_t nbr_capacity, void *stream);

/* Global integer cell coordinates floor(x / cell_size) of every particle
 * (int32[3*N], engine order); find_cell_id (S/base/cell.pyx:63-84). */
SPHB_API int sphb_cell_coords(const sphb_engine *e, int cur, int32_t *out, void *stream);

/* Summation density, optionally followed by the Tait EOS, over the dest
 * arrays in dest_mask.  Sources per dest array come from cfg.rho_src.
 * with_eos: p, cs from Tait for dest arrays in cfg.tait_on.  SPHRho
 * (S/sph/funcs/density_funcs.pyx:37-73, .clt:3-53) + TaitEquation
 * (S/sph/funcs/eos_funcs.pyx:88-129, .clt:36-65).  When f.list_cap > 0 the
 * pass also records every dest particle's neighbour list (the reference
 * caches one list per particle for all calcs of a stage,
 * FixedDestNbrParticleLocator._update_cache, S/base/nnps.pyx:596-621). */
SPHB_API int sphb_density(const sphb_engine *e, int cur, uint32_t dest_mask,
                 int with_eos, void *stream);
/* with_eos bits: SPHB_DENSITY_EOS applies Tait; SPHB_DENSITY_USE_LIST sums
 * over the lists of an earlier pass instead of searching cells (the caller
 * vouches that they are complete).  SPHB_DENSITY_LIST_IF_VALID is the list
 * reuse of the integrator: it reads the lists when the last
 * SPHB_BIN_IF_NEEDED kept them and nothing moved the particles since, and
 * otherwise searches cells and records lists with the skin
 * (radius_scale h + skin_max)(1 + 1e-5), which become reusable when
 * recorded right after a rebin.  A pass that records without it uses no
 * skin and withdraws the lists from reuse.  Every pass applies
 * the exact predicate r^2 < (radius_scale h)^2 to what it visits. */
#define SPHB_DENSITY_EOS 1
#define SPHB_DENSITY_USE_LIST 2
#define SPHB_DENSITY_LIST_IF_VALID 4
/* SPHB_DENSITY_LISTS_ONLY: no density, only the lists (continuity scheme,
 * where the density is integrated): recorded over every pair function's
 * sources when the pass would record, nothing otherwise. */
#define SPHB_DENSITY_LISTS_ONLY 8

/* Refresh the FP32 pair records (positions relative to each particle's
 * cell of the last bin, velocities) from the FP64 state without rebinning,
 * and, with f.anchor, measure every particle's displacement from its anchor
 * into the scenes' max_disp2, so that the next SPHB_BIN_IF_NEEDED decision
 * may keep the lists after positions or velocities written by the host
 * (work.meta[5]; without this call it rebins).
 * sphb_pc_stage refreshes them itself; this is for state written by other
 * means.  No-op for SPHB_FP64. */
SPHB_API int sphb_refresh(const sphb_engine *e, int cur, void *stream);

/* Tait EOS alone on the dest arrays in dest_mask (rho already set). */
SPHB_API int sphb_tait(const sphb_engine *e, int cur, uint32_t dest_mask, void *stream);

/* MomentumEquation (pressure gradient + Monaghan artificial viscosity,
 * dt_fac) over the dest arrays in dest_mask with sources cfg.mom_src,
 * then GravityForce when with_gravity; writes au/av/aw and dt_fac and the
 * per-scene max dt_fac and |a|^2.  S/sph/funcs/pressure_funcs.pyx:246-391,
 * .clt:69-157; S/sph/funcs/external_force.pyx:13-62.
 * mode: 0 = MomentumEquation, 1 = SPHPressureGradient (:62-161, no AV),
 * 2 = the split-form MonaghanArtificialViscosity alone
 * (S/sph/funcs/viscosity_funcs.pyx:19-157): a += -m_b Pi_ab grad W when
 * v_ab . r_ab < 0, with scene.eta as its eta (the reference's constructor
 * never sets it, so its callers pass 0), and dt_fac with 0.01 h_ab^2 in the
 * denominator whatever eta is.
 * mode | SPHB_FORCE_USE_LIST: iterate the lists of the last sphb_density
 * pass (same bin, same sources) instead of searching cells. */
#define SPHB_FORCE_USE_LIST 16
/* mode | SPHB_FORCE_NO_MAXIMA: leave the per-scene dt_fac / |a| maxima
 * alone (a predictor's pass, whose maxima the CFL rule does not read). */
#define SPHB_FORCE_NO_MAXIMA 32
/* mode | SPHB_FORCE_STAGE(kind), FP32C with f.geo_next / vel_next: the
 * sphb_pc_stage stage `kind` (0..7) of every dest particle in the pass's
 * epilogue, on the accelerations, density rate and XSPH velocity it has
 * just computed.  The new records go to geo_next / vel_next; every stepped
 * array (cfg.step_on) and density-rate dest must be a dest of the pass.
 * Unlike sphb_pc_stage, stage 0 does not clear the CFL maxima: give the
 * predictor's pass (and RK2's first, RK4's first three)
 * SPHB_FORCE_NO_MAXIMA instead. */
#define SPHB_FORCE_STAGE(kind) (((kind) + 1) << 8)
#define SPHB_FORCE_STAGE_MASK 0xF00
SPHB_API int sphb_momentum(const sphb_engine *e, int cur, uint32_t dest_mask,
                  int with_gravity, int mode, void *stream);

/* Integrator stage on the integrated arrays (cfg.step_on, and the density
 * of cfg.rate_src dests): stage 0 = predict (save X0, X = X0 + dt/2 F; also
 * RK2's first stage), stage 1 = correct and final (X = 2 (X0 + dt/2 F) -
 * X0), stage 2 = Euler (save X0, X = X0 + dt F;
 * EulerIntegrator.integrate, S/solver/integrator.py:420-447), stage 3 =
 * RK2's second stage (X = X0 + dt F; RK2Integrator, :452-499); stages 4-7
 * are RK4Integrator's four (:504-609), with buf.kx .. krho holding the
 * running sum S: 4 save X0, S = K1, X = X0 + dt/2 K1; 5 S = S + 2 K2,
 * X = X0 + dt/2 K2; 6 S = S + 2 K3, X = X0 + dt K3; 7 X = X0 + (dt/6)
 * (S + K4), in numpy's order of the reference's final_step.  Stages 0, 4,
 * 5 and 6 also clear the per-scene dt_fac / |a| maxima, so sphb_step_begin
 * sees the last stage's pass only.
 * Refreshes the FP32 pair records of the moved particles and, with
 * f.anchor, accumulates max_disp2 (cleared by the next SPHB_BIN_IF_NEEDED
 * decision).  PositionStepping
 * (S/sph/funcs/position_funcs.pyx:10-56) supplies F_x = u.
 * PredictorCorrectorIntegrator.integrate (S/solver/integrator.py:646-683),
 * step (:340-367), final_step (:632-644); integrator.cl step_array /
 * pc_final_step (S/solver/integrator.cl:1-24). */
SPHB_API int sphb_pc_stage(const sphb_engine *e, int cur, int stage, void *stream);

/* Per-step prologue of Solver.solve (S/solver/solver.py:546-566): for
 * every scene count += 1, then, for scenes with use_cfl, dt from
 * ViscousAndForceBasedTimeStep.compute_time_step
 * (S/solver/time_step_functions.py:8-57, Integrator.get_max_acceleration
 * S/solver/integrator.py:369-412) using the max dt_fac and |a| of the last
 * sphb_momentum; then t += dt, and the maxima restart for this step's
 * force passes. */
SPHB_API int sphb_step_begin(const sphb_engine *e, void *stream);

/* Gather (dir 0: user order -> engine order) or scatter (dir 1: engine ->
 * user order) one FP64 property of the particles in array `array`:
 * engine[k] <-> user[seg-local idx[k]], for every scene's segment of that
 * array, with user arrays concatenated over scenes (user_offset[s]).
 * `field` names the engine field: 0..5 x..w, 6..11 x0..w0, 12 m, 13 h,
 * 14 rho, 15 p, 16 cs, 17 au, 18 av, 19 aw, 20 dt_fac; continuity scheme:
 * 21 the integrated density (buf.rho), 22 its stage-initial copy, 23 its
 * rate _a_rho_1; 24..26 the XSPHCorrection velocity.  Fields 17..20 and
 * 23..26 are scatter-only.  Gathering m or h withdraws the lists: the next
 * SPHB_BIN_IF_NEEDED rebins, which also rebuilds the FP32 pair records.
 * Gathering x..w marks them unchecked (work.meta[5]): the next decision
 * rebins unless sphb_refresh has since measured that no particle left half
 * the skin around its anchor.  `user` and `user_offset` must not be NULL
 * (SPHB_ERR_ARG): an array without particles has nothing to exchange and
 * the call is simply not made. */
SPHB_API int sphb_exchange(const sphb_engine *e, int cur, int array, int field,
                  int dir, double *user, const int32_t *user_offset,
                  void *stream);

/* sphb_exchange of count (1..SPHB_EXCHANGE_MAX) fields of one array in one
 * launch: fields[i] <-> users[i], fields and users being host arrays read
 * during the call; each thread finds its particle's user position once for
 * all of them.  The same import marks as the single calls.  Used by the
 * integrators' imports of host-written x, y, u, v and by
 * ParticleArray.get of several properties (S/base/particle_array.pyx:
 * get(*args) returns each of them). */
#define SPHB_EXCHANGE_MAX 8
SPHB_API int sphb_exchange_many(const sphb_engine *e, int cur, int array, int dir,
                                int32_t count, const int32_t *fields, double *const *users,
                                const int32_t *user_offset, void *stream);

/* Same for the int32 tag field. */
SPHB_API int sphb_exchange_tag(const sphb_engine *e, int cur, int array, int dir,
                      int32_t *user, const int32_t *user_offset, void *stream);

/* Time step of the next sphb_pc_stage for every scene without use_cfl: the
 * dt argument of PredictorCorrectorIntegrator.integrate(dt)
 * (S/solver/integrator.py:646). */
SPHB_API int sphb_set_dt(const sphb_engine *e, double dt, void *stream);

/* Write identity idx (0..n-1 inside each segment) into buf[cur].idx. */
SPHB_API int sphb_init_index(const sphb_engine *e, int cur, void *stream);

/* Copy one FP64 per-particle array of array index `array` between the
 * caller's order (dir 0: user -> engine_buf; dir 1: engine_buf -> user)
 * and the engine order of buf[cur]; like sphb_exchange for arbitrary
 * buffers (adjoint vectors, ...). */
SPHB_API int sphb_permute(const sphb_engine *e, int cur, int array, int dir, double *user,
                          double *engine_buf, const int32_t *user_offset, void *stream);

/* ---- adjoint of the particle update ---------------------------------
 * The reference has no gradients; these are the reverse-mode kernels of the
 * differentiable rollout (FP64 engines only).  Vectors are SoA [dim][N] in
 * engine order.  Each needs the forward quantities of the stage (positions,
 * velocities, rho, p, cs from sphb_density) and its bin.  In a scene of
 * uniform h, the pair kernels walk the neighbour lists that sphb_density
 * recorded for that bin (every array with SPHRho sources, f.list_cap > 0);
 * otherwise they search the cells.  The pair kernels launch on the engine's
 * pair-pass shape (its pair tiles, pair_block threads, `lanes` lanes per
 * dest particle merged by warp shuffles), so an engine made for the
 * adjoint picks its own lanes (2 suits these kernels' FP64 pair work). */

/* Given lam_a, the adjoint of the MomentumEquation acceleration of the dest
 * arrays in dest_mask: lam_x += (da/dx)^T lam_a, lam_v += (da/dv)^T lam_a;
 * lam_rho, lam_p, lam_c = (da/drho, dp, dcs)^T lam_a. */
SPHB_API int sphb_force_vjp(const sphb_engine *e, int cur, uint32_t dest_mask,
                            const double *lam_a, double *lam_x, double *lam_v,
                            double *lam_rho, double *lam_p, double *lam_c, void *stream);

/* lam_rho += lam_p dp/drho + lam_c dcs/drho through the Tait EOS. */
SPHB_API int sphb_eos_vjp(const sphb_engine *e, int cur, double *lam_rho,
                          const double *lam_p, const double *lam_c, void *stream);

/* lam_x += (drho/dx)^T lam_rho through summation density. */
SPHB_API int sphb_density_vjp(const sphb_engine *e, int cur, uint32_t dest_mask,
                              const double *lam_rho, double *lam_x, void *stream);

/* ---- neighbour counts without caller scratch ------------------------ */

/* Largest particle set sphb_neighbor_counts_static accepts. */
#define SPHB_STATIC_MAX_PARTICLES (1 << 18)

/* Neighbour count of every particle of one particle set: counts[i] = number
 * of j (self included) with |x_i - x_j|^2 < (radius_scale * h_i)^2, the FP64
 * predicate of sphb_neighbors; -1 for a particle with a non-finite position
 * (which is then nobody's neighbour) or a non-finite smoothing length (the
 * others still count it: the predicate takes each particle's own h).
 * x, y, z (z may be NULL when dim == 2), h and counts are device arrays of n
 * elements in the caller's order.
 *
 * It has no counterpart in the reference.  It exists for callers that cannot
 * call cudaMalloc -- a host application whose own memory manager owns all
 * device memory and gives this library only the particle arrays, or code on
 * a latency-critical path where cudaMalloc's implicit device-wide
 * synchronisation is not acceptable -- and so cannot provide the workspace
 * the engine entry points take.  Its scratch is one file-scope device array
 * inside the library of about 7 MiB (cell tables for up to 2^19 cells plus
 * three int32 arrays of SPHB_STATIC_MAX_PARTICLES), which every GPU that
 * loads the library holds until the process exits.  n above
 * SPHB_STATIC_MAX_PARTICLES returns SPHB_ERR_WORKSPACE; the cell size grows
 * past radius_scale * max h when a grid would need more than 2^19 cells or
 * cell coordinates beyond 2^30 (particles far from the origin), which
 * lengthens the cell walks but not the counts.  Cost: one pass over the
 * particles per phase, and one block that scans the cell counts
 * serially (up to 512 cells per thread at the 2^19-cell maximum).
 * The call allocates nothing (no cudaMalloc, cudaFree or allocating library
 * routine).  Its first call on a device looks up the scratch array's device
 * address with that device current; make that first call before any stream
 * capture.  A cudaDeviceReset leaves that address stale: do not call it on
 * a device after resetting the device.  All calls share the one array, which keeps the last call's
 * contents, so calls that overlap on the GPU race: serialise them. */
SPHB_API int sphb_neighbor_counts_static(int32_t n, int32_t dim, const double *x,
                                         const double *y, const double *z,
                                         const double *h, double radius_scale,
                                         int32_t *counts, void *stream);


#ifdef __cplusplus
}
#endif
#endif /* SPHB_H */
