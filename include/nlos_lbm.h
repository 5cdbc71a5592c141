/*
 * nlos_lbm.h -- C-ABI of the B200 D3Q19 lattice-Boltzmann acoustic solver.
 *
 * The reference solver has no library interface: its entry points are the
 * public members of `LBMSolver` in 06_transient_localization_dx1.cpp (and the
 * identical family-B solvers 05/07/08), called from `main`.  Each function
 * below replaces one of those members; the comment names the reference
 * member it stands in for (file:line).  Plain C types only: pointers, sizes,
 * doubles.  The library owns all device memory; callers own host arrays.
 *
 * Error behaviour: every call returns an lbm_status.  0 is success, negative
 * values are errors (nothing was changed), positive values are warnings for
 * the cases the reference reports on stdout and then carries on (STL not
 * loaded, probe inside a solid).  No C++ exceptions cross this boundary.
 * A handle owns one CUDA stream and is not re-entrant: use one handle per
 * host thread.  (The library also runs some small kernels, such as the probe
 * record beside the step, on a second stream of the handle, joined back to
 * the handle's stream before anything reads their results or overwrites
 * their inputs, so work ordered on the handle's stream sees the same order.)
 *
 * Lattice: D3Q19 in the reference's family-B velocity order (06:21-31).
 * Populations are stored on the device as deviations g_q = f_q - w_q from the
 * rest equilibrium, in FP32 or (scaled) FP16, and collided in FP32.
 */
#ifndef NLOS_LBM_H
#define NLOS_LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbm_handle lbm_handle;

typedef enum lbm_status
{
    LBM_OK = 0,
    LBM_WARN_STL_NOT_LOADED = 1,   /* 06:397-410: geometry left empty, run continues */
    LBM_WARN_PROBE_IN_SOLID = 2,   /* 06:432-435: probe cell is SOLID, run continues */
    LBM_WARN_STL_TRUNCATED = 3,    /* the STL ends before its header's triangle count; the missing
                                      records read as zeros, as the reference's loader leaves them
                                      (06:82-85), and the run continues */
    LBM_ERR_INVALID_ARGUMENT = -1,
    LBM_ERR_BAD_CONFIG = -2,
    LBM_ERR_OUT_OF_MEMORY = -3,
    LBM_ERR_CUDA = -4,
    LBM_ERR_NAN = -5,              /* an owned probe read a non-finite value.  The probe kernel
                                      sets a device flag that lbm_step / lbm_run read at the end
                                      of each batch of steps (at most 4096 steps, usually the
                                      whole call): the call in which the value appeared returns
                                      this code, with the steps taken; the flag stays set, so
                                      every later lbm_step call returns it too.  Standalone
                                      lbm_record_probes calls are checked at the next lbm_step
                                      or lbm_get_probes.  A grid without probes is not checked
                                      (the reference checks nothing). */
    LBM_ERR_STATE = -6,            /* call out of order, e.g. step before init */
    LBM_ERR_CAPACITY = -7,         /* caller's output buffer too small */
    LBM_ERR_NO_DEVICE = -8,
    LBM_ERR_IO = -9,
    LBM_ERR_UNSUPPORTED = -10
} lbm_status;

/* Boundary treatment of one face of the box. */
enum
{
    LBM_BC_NSCBC = 0,  /* characteristic open boundary, zero incoming wave (06:684-835) */
    LBM_BC_REST = 1,   /* halo held at rest equilibrium w_q (06:677-682 with use_nscbc=false) */
    LBM_BC_WALL = 2,   /* SOLID halo: halfway bounce-back (ground plane, 06:520-531) */
    LBM_BC_COPY = 3,   /* zero-gradient halo, a copy of the nearest interior cell that then
                          collides like any cell (fill_halo_copy 03:175-237); scheme A only,
                          and then on all six faces */
    LBM_BC_PERIODIC = 4 /* periodic: the halo plane is the opposite interior plane (01:105-107,
                           exchanged with itself at one rank, 01:288-299); scheme A, both z
                           faces only */
};

/* Update scheme.  B is the family of 05-08 (06:906-972): pull, halfway
 * bounce-back, BGK with one tau and a sponge blend toward rest.  A is the
 * family of 01-04 (02:363-420, 03:402-441): every population arriving at a
 * cell is the post-collision value of the cell it left, relaxed with that
 * cell's own tau (a tau ramp is the sponge, 02:164-179, 03:148-160), while a
 * population arriving from a SOLID cell is the destination's own
 * pre-collision value of the opposite direction. */
enum { LBM_SCHEME_B = 0, LBM_SCHEME_A = 1 };
enum { LBM_FACE_XLO = 0, LBM_FACE_XHI, LBM_FACE_YLO, LBM_FACE_YHI, LBM_FACE_ZLO, LBM_FACE_ZHI };

enum { LBM_STORE_F32 = 0, LBM_STORE_F16 = 1 };

/* Source time functions. */
enum
{
    LBM_WAVE_GAUSS = 0,   /* amp*exp(-0.5*((t-t0)/sigma_t)^2)            (06:579-581) */
    LBM_WAVE_SINE = 1,    /* amp*sin(2*pi*freq*t)                         (08:543) */
    LBM_WAVE_RICKER = 2,  /* amp*(1-2a)exp(-a), a=(pi*freq*(t-t0))^2 */
    LBM_WAVE_TABLE = 3    /* amp*table[s], one sample per time step s */
};
/* Spatial injection stencils. */
enum
{
    LBM_INJECT_GAUSS = 0,     /* (2R+1)^3 Gaussian, fluid-normalised          (06:587-666) */
    LBM_INJECT_TRILINEAR = 1, /* 8 cells, trilinear weights, fluid-normalised */
    LBM_INJECT_FIELD = 2      /* scheme A: every cell, weight exp(-|x - s|^2 / (2 sigma^2)),
                                 sigma = sigma_cells * dx, not normalised (02:181, 03:166-169) */
};
/* How a LBM_INJECT_FIELD source enters a scheme-A step. */
enum
{
    LBM_FIELD_DST = 0,   /* w_q * weight(dst) * val(t) * dt added to every population streamed
                            from a fluid cell, after the collision (02:373, 02:405) */
    LBM_FIELD_FORCE = 1, /* forcing at the cell being collided: w_q * weight * val(t) * dt
                            * (1 + 3 c_q.flow) * (1 - 1/(2 tau)) (03:74-78, 03:424-435) */
    LBM_FIELD_PRE = 2    /* w_q * weight * val(t) * dt added to every population of every
                            fluid cell before the step at time t (apply_source 04:212-235);
                            val(0) must be 0 */
};

/* Solver configuration: the member fields of LBMSolver (06:244-268), the
 * constants of init_domain (06:455-458) and UnitConverter (06:195-204), plus
 * the boundary/sponge/storage choices the reference hard-codes. */
typedef struct lbm_config
{
    double x_min, x_max, y_min, y_max, z_min, z_max; /* 06:250-252 */
    double dx;                                       /* 06:253 DX */
    double c_phys;                                   /* 06:198 speed of sound (dt = cs*dx/c) */
    double tau;                                      /* 06:268 BGK relaxation time */
    int use_geometry;                                /* 06:248 */
    int face_bc[6];                                  /* LBM_BC_* per face, LBM_FACE_* order */
    unsigned sponge_faces;                           /* bit f set: sponge ramps in from face f (06:491-496) */
    double sponge_width;                             /* in cells (06:455: 20) */
    double sponge_strength;                          /* 06:456: 0.35 */
    double sky_z;                                    /* cells above this z are FLUID (06:458,489) */
    int storage;                                     /* LBM_STORE_F32 or LBM_STORE_F16 */
    double f16_scale;                                /* FP16 stores (f_q - w_q) * f16_scale; about
                                                        100 / (source density amplitude) keeps
                                                        far-field values out of FP16's subnormals */
    int device;                                      /* CUDA device ordinal */
    int use_graphs;                                  /* replay multi-step runs as CUDA graphs */
    int verbose;                                     /* print the reference's progress lines */
    /* scheme A (01-04 family); ignored by scheme B */
    int scheme;                                      /* LBM_SCHEME_B (default) or LBM_SCHEME_A */
    double tau_sponge_max;                           /* tau at the sponge faces: tau + (max - tau) r^2,
                                                        r = (width - d)/width, d = cells to the nearest
                                                        sponge face (02:164-179, 03:148-160); <= 0: none */
    double flow[3];                                  /* uniform background velocity, lattice units
                                                        (03:121 uz = Ma cs); initial state feq(1, flow) */
    double dt;                                       /* > 0: time step in seconds instead of cs*dx/c_phys
                                                        (02:36 uses the constant 0.577350269) */
    /* z-slab of a decomposed domain (scheme B): the handle holds interior
     * z-layers slab_k0 .. slab_k0 + slab_nz - 1 of the grid above; slab_nz = 0:
     * the whole grid.  Cuts between slabs have no boundary treatment: their
     * halo planes come from the neighbour slab (lbm_slab_exchange). */
    int slab_k0;
    int slab_nz;
    /* scheme A: 1 = the sponge is 01's blend at the destination (01:207-225,
     * 01:343-347): every population arriving from a fluid cell becomes
     * (1 - s) f + s w_q with s = sponge_strength ((w - d) / w)^2, d the
     * distance of the cell centre to the nearest sponge face and w =
     * sponge_width cells, where s > 1e-6; needs tau_sponge_max <= 0. */
    int sponge_blend;
} lbm_config;

/* One sound source: DroneSource (06:211-239) plus its time function. */
typedef struct lbm_source
{
    double sx, sy, sz;      /* path start  (06:213) */
    double ex, ey, ez;      /* path end    (06:214) */
    double speed;           /* units / time; 0 = stationary (06:225) */
    double amp;             /* 06:216 */
    double freq;            /* 06:217 (sine, Ricker peak frequency) */
    int waveform;           /* LBM_WAVE_* */
    double t0, sigma_t;     /* Gaussian centre/width (06:579-580); Ricker delay t0 */
    int injection;          /* LBM_INJECT_* */
    double gain;            /* 06:583 source_gain */
    double sigma_cells;     /* Gaussian stencil width in cells (06:588: 1.25) */
    int radius;             /* Gaussian stencil radius in cells (06:587: 2), 0..3 */
    const double* table;    /* LBM_WAVE_TABLE samples (copied at lbm_add_source) */
    int table_len;
    int field_mode;         /* LBM_FIELD_* for LBM_INJECT_FIELD */
} lbm_source;

/* Seeded synthetic city: axis-aligned box buildings written as triangles. */
typedef struct lbm_city_params
{
    int nx, ny;             /* plan extent in cells */
    double dx;              /* cell size (vertex coordinates are multiples of it) */
    uint64_t seed;
    int fp_min, fp_max;     /* footprint side, cells */
    int h_min, h_max;       /* building height, cells */
    double coverage;        /* target plan-area fraction */
    int street;             /* minimum gap between buildings, cells */
    int margin;             /* keep-out band along the plan border, cells */
} lbm_city_params;

/* ---- defaults ------------------------------------------------------------ */

/* Reference defaults: 06:250-268 fields, 06:455-458 sponge/sky constants,
 * NSCBC on x-,x+,y-,y+,z+ and ground bounce-back at z- (06:509-531). */
void lbm_config_default(lbm_config* cfg);
/* Reference defaults for a source: Gaussian pulse t0=0.05 s, sigma_t=0.005 s
 * (06:579-580), 5x5x5 Gaussian stencil R=2, sigma 1.25 cells (06:587-588). */
void lbm_source_default(lbm_source* src);
const char* lbm_status_string(int status);
/* Library version string and the CUDA architecture it was built for. */
const char* lbm_version(void);

/* ---- lifetime ------------------------------------------------------------ */

/* Validates the config and binds the device; no device memory yet.
 * Replaces constructing LBMSolver and setting its fields (06:1128-1166). */
int lbm_create(const lbm_config* cfg, lbm_handle** out);
/* Frees all device and host memory of the handle. */
int lbm_destroy(lbm_handle* h);
/* Last error message of this handle (NUL-terminated, may be empty). */
const char* lbm_last_error(lbm_handle* h);

/* ---- geometry / mask (LBMSolver::init 06:397-413, init_domain 06:453-532) ---- */

/* Binary STL file; vertices * scale + (sx,sy,sz) as GeometryEngine::load
 * (06:70-111).  Returns LBM_WARN_STL_NOT_LOADED and keeps an empty geometry
 * when the file cannot be read, as the reference does (06:397-410), and
 * LBM_WARN_STL_TRUNCATED when the file holds fewer records than its header
 * counts (the mask is the reference's: missing records are zero triangles).
 * The status is also returned by lbm_init when no probe warning replaces it. */
int lbm_set_geometry_stl(lbm_handle* h, const char* path, double scale, double sx, double sy, double sz);
/* Same, from memory: tris holds ntris * 9 floats (v1, v2, v3). */
int lbm_set_geometry_triangles(lbm_handle* h, const float* tris, int ntris, double scale, double sx,
                               double sy, double sz);
/* Override the voxelised mask: nx_t*ny_t*nz_t bytes (0 FLUID, 1 SOLID) in the
 * reference's halo-inclusive order i + j*nx_t + k*nx_t*ny_t (06:206-209). */
int lbm_set_mask(lbm_handle* h, const uint8_t* mask, int nx_t, int ny_t, int nz_t);
/* Scheme A, before lbm_init: per-column (x, y) fields that are the same at
 * every height, count = nx*ny, x fastest (both programs that use them are
 * z-invariant: 01 and 04).  Blend strengths s of the destination blend
 * (sponge_blend = 1; a cell takes the larger of this and the face profile;
 * s <= 1e-6 is no blend), e.g. 04's radial layer (04:177-209).  Weights of
 * the field source, replacing its Gaussian, e.g. 04's line source with its
 * cutoff (04:212-235). */
int lbm_set_blend_xy(lbm_handle* h, const double* s_xy, long count);
int lbm_set_field_weights_xy(lbm_handle* h, const double* w_xy, long count);

/* The mask lbm_init builds for this config and triangle set (init_domain
 * 06:453-532), computed on the host; needs no device.  n3_halo receives
 * nx_t, ny_t, nz_t; mask needs nx_t*ny_t*nz_t bytes. */
int lbm_voxelize(const lbm_config* cfg, const float* tris, int ntris, double scale, double sx, double sy, double sz,
                 uint8_t* mask, long capacity, int* n3_halo);

/* ---- sources and probes ------------------------------------------------- */

/* Adds a source (the reference has exactly one, LBMSolver::drone 06:246). */
int lbm_add_source(lbm_handle* h, const lbm_source* src);
int lbm_clear_sources(lbm_handle* h);
/* Probe positions xyz[3*n] in physical coordinates (LBMSolver::probes
 * 06:257-266); cell = floor((x - x_min)/dx) (06:417-419). */
int lbm_set_probes(lbm_handle* h, const double* xyz, int n);
/* Per probe: owned (inside the grid) and in_solid flags; either may be NULL. */
int lbm_probe_info(lbm_handle* h, int* owned, int* in_solid);

/* ---- set-up and stepping ------------------------------------------------- */

/* Builds the grid, mask, sponge and rest state on the device
 * (LBMSolver::init 06:299-450).  May return LBM_WARN_* codes. */
int lbm_init(lbm_handle* h);
/* Source injection at time t (LBMSolver::apply_source 06:576-667). */
int lbm_apply_source(lbm_handle* h, double t);
/* Open-boundary ghost fill (LBMSolver::exchange_halos 06:671-904, one rank). */
int lbm_exchange_halos(lbm_handle* h);
/* Fused pull-stream + bounce-back + BGK + sponge, then buffer swap
 * (LBMSolver::step_collision_bgk 06:906-972). */
int lbm_step_collision_bgk(lbm_handle* h);
/* Appends rho-1 at every owned probe for the last step (06:1085-1092). */
int lbm_record_probes(lbm_handle* h);
/* nsteps full time steps s, s+1, ...: apply_source(s*dt), exchange_halos,
 * step_collision_bgk, record_probes -- the body of LBMSolver::run
 * (06:1077-1092) without VTK output. */
int lbm_step(lbm_handle* h, int nsteps);
/* LBMSolver::run(T_total, Frames) (06:1064-1121): steps s = 0..round(T/dt)
 * inclusive.  Frames only sets the progress/frame interval (no VTK here). */
int lbm_run(lbm_handle* h, double T_total, int frames);
/* Waits for all work queued on the handle's stream. */
int lbm_synchronize(lbm_handle* h);

/* ---- results ------------------------------------------------------------ */

/* Grid size NXg, NYg, NZg (06:332-334) and halo-inclusive nx_t, ny_t, nz_t. */
int lbm_get_dims(lbm_handle* h, int* n3, int* n3_halo);
double lbm_get_dt(lbm_handle* h);
/* Number of time steps taken so far. */
long lbm_get_step(lbm_handle* h);
/* Probe series rho-1, layout [step][probe], FP64 (06:1090, 06:1106-1118);
 * unowned probes read NaN.  *nsteps receives the number of rows. */
int lbm_get_probes(lbm_handle* h, double* out, long capacity, long* nsteps);
/* Per-probe sum over recorded steps of (rho-1)^2, accumulated in FP64. */
int lbm_get_probe_energy(lbm_handle* h, double* out);
/* Interior field (float)(rho-1) of the last step, i fastest (06:979-985).
 * Before the first step it is 0 (rho starts at 1, 06:368), or, after
 * lbm_set_density, the initial pulse at FLUID cells (01:197). */
int lbm_get_rho(lbm_handle* h, float* out, long capacity);
/* Largest grid (interior cells) lbm_get_rho_noalloc accepts. */
#define LBM_NOALLOC_MAX_CELLS 8388608L

/* lbm_get_rho without allocating: no counterpart in the reference (its
 * rho field is a host vector, 06:281).  Some callers cannot allocate device
 * memory at the moment they read a field: a host application that owns the
 * GPU's memory through its own pool, where a direct cudaMalloc would bypass
 * or overrun that budget, or a frame loop that must not stall, since
 * cudaMalloc and cudaFree can synchronise the whole device.  This call
 * writes the same values as lbm_get_rho into `out`, but the device-side
 * field passes through one array of LBM_NOALLOC_MAX_CELLS floats (32 MiB)
 * reserved statically in the library: every GPU that loads the library
 * holds it until the process exits, and nothing is allocated per call.
 * Grids with more interior cells are rejected with LBM_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's address and keeps it for
 * the life of the process; make that first call before any CUDA stream
 * capture, and do not reset the device (cudaDeviceReset) while the library
 * is in use: the kept address, like every handle's memory, would be stale.  All handles on a device share the
 * array: calls that overlap on the GPU (handles used from different host
 * threads at the same time) race and may return each other's field, so
 * serialise them.  The array keeps the last call's contents; every call
 * overwrites all the cells it returns, so nothing needs clearing. */
int lbm_get_rho_noalloc(lbm_handle* h, float* out, long capacity);
/* Populations f_q (FP64, w_q + deviation) in the reference's AoS,
 * halo-inclusive layout f[idx*19+q] (06:366, 06:206-209).  In the ghost
 * cells of open faces only the 5 directions the interior pulls from them are
 * kept up to date (the reference fills all 19; the other 14 are never read). */
int lbm_get_f(lbm_handle* h, double* out, long capacity);
int lbm_set_f(lbm_handle* h, const double* in, long count);
/* Scheme A: initial state at rest with density 1 + rho_minus_1 at every
 * interior fluid cell (count = nx*ny*nz, x fastest), i.e. f = feq(1 + rho',
 * flow) (the pulse initial condition of 01:183-205); SOLID cells keep theirs,
 * the bounce-back slots next to them and zero-gradient (LBM_BC_COPY) halo
 * cells follow the new values, periodic halo planes repeat them.  After
 * lbm_init, before the first step (LBM_ERR_STATE otherwise). */
int lbm_set_density(lbm_handle* h, const double* rho_minus_1, long count);
/* Voxelised mask, halo-inclusive, 0 FLUID / 1 SOLID (06:469-531). */
int lbm_get_mask(lbm_handle* h, uint8_t* out, long capacity);

/* ---- adjoint ---------------------------------------------------------------- */

/* Gradient of the receiver misfit
 *     L = 1/2 sum_{s < nsteps} sum_p (p_s[p] - observed[s * nprobe + p])^2
 * of an nsteps-step run from the rest state, with respect to a rigid shift of
 * the source path (grad_pos[3], per metre) and to the source signal value at
 * every step (grad_signal[nsteps]: dL/dval_s, val_s = amp * waveform(t_s) as in
 * 06:579-581, so dL/dtable[s] = amp * grad_signal[s] for LBM_WAVE_TABLE).
 * No counterpart in the reference, which has no adjoint or inverse solver;
 * the forward model is exactly lbm_step's (same kernels, FP32 storage).
 * A reverse-time discrete adjoint of the fused step.  The backward pass needs
 * each step's forward data: the moments of the pulled populations (6 bytes a
 * cell) and those of the ghost cells.  The forward pass keeps them for a tail
 * of whole ckpt_outer-step segments (<= 0: 200) and a full-state checkpoint at
 * the start of every segment before that tail; those segments are recomputed,
 * with inner checkpoints every ckpt_inner steps, before they are run
 * backwards.  ckpt_inner <= 0 picks the largest inner interval, then the
 * longest tail, that fit in 90 % of the free device memory (NLOS_LBM_ADJ_BUDGET
 * caps it); when the whole run's forward data fits nothing is recomputed.  An
 * explicit ckpt_inner > 0 keeps no tail.  lbm_adjoint_plan gives the schedule
 * and its device bytes.  Requires FP32 storage, exactly one source and at least
 * one probe.  Observed entries that are NaN, probes outside the grid and the
 * probe rows of SOLID cells (which read 0 whatever the state) contribute no
 * gradient.  Starts from and returns to the rest state (step 0, empty probe
 * series); `predicted` (optional, nsteps * nprobe) receives the forward probe
 * series.  grad_pos, grad_signal and predicted may be NULL. */
int lbm_adjoint_grad(lbm_handle* h, int nsteps, const double* observed, int ckpt_outer, int ckpt_inner,
                     double* loss, double* grad_pos, double* grad_signal, double* predicted);
/* The schedule lbm_adjoint_grad would run with these arguments (no
 * counterpart in the reference): the effective outer and inner checkpoint
 * intervals, the device bytes it allocates and the number of forward steps
 * it runs, recomputation included (nsteps when nothing is recomputed).
 * Every output may be NULL. */
int lbm_adjoint_plan(lbm_handle* h, int nsteps, int ckpt_outer, int ckpt_inner, int* outer, int* inner,
                     long long* device_bytes, long long* forward_steps);
/* lbm_adjoint_grad keeps its device workspace in the handle so repeated
 * gradient evaluations (the iterations of a localisation) allocate nothing
 * after the first; this frees it now instead of at lbm_destroy.  No
 * counterpart in the reference. */
int lbm_adjoint_release(lbm_handle* h);

/* ---- z-slab decomposition --------------------------------------------------- */

/* Halo exchange between two z-slab handles of one process (the reference's
 * MPI decomposition exchanges every face through exchange_halos, 06:837-903,
 * all 19 populations of each face cell, 06:840-845).  `lower` holds the
 * layers just below `upper`.  Call it once per time step, after
 * lbm_apply_source and lbm_exchange_halos of both handles and before their
 * lbm_step_collision_bgk.  Only what the next step pulls across the cut
 * travels: the 5 populations with ez toward the neighbour of each slab's
 * boundary plane (its y-halo rows included) and the 2 of its x-face ghost rows
 * among them, as one message each way (lbm_slab_pack / lbm_slab_unpack).  The
 * copies run on the receiving handle's stream, ordered against both streams
 * with events, so the handles may live on different GPUs (a peer copy of the
 * message) or on the same one.  The handles keep their message buffers (4
 * messages each) until lbm_destroy. */
int lbm_slab_exchange(lbm_handle* lower, lbm_handle* upper);
/* Size in bytes of one cut's message of this z-slab handle: 5 directions x
 * (ny + 2) rows x ceil(nx / cells per line) lines of 128 B, plus 2 x (ny + 2)
 * floats of x-face ghosts.  0 for a handle that is not a z-slab. */
long lbm_slab_message_bytes(lbm_handle* h);
/* For one z-slab per process (a rank per GPU): pack, on the handle's stream,
 * the message toward the neighbour on `side` (0: below, the directions with
 * ez = -1 of the slab's first plane; 1: above, ez = +1 of its last plane) into
 * `msg`, 16-byte aligned device memory of the handle's GPU of
 * lbm_slab_message_bytes bytes.  Call after lbm_exchange_halos.  The caller
 * moves the message to the neighbour's GPU (for example an NCCL send/recv),
 * ordered after this call's work on the handle's stream (lbm_get_stream). */
int lbm_slab_pack(lbm_handle* h, int side, void* msg);
/* Unpack the neighbour's message on `side` (0: from the slab below, into halo
 * plane 0; 1: from the slab above, into halo plane nz + 1), on the handle's
 * stream, before lbm_step_collision_bgk.  The message must be complete in
 * device memory of this handle's GPU before the handle's stream reaches this
 * call (order the transfer's stream before it). */
int lbm_slab_unpack(lbm_handle* h, int side, const void* msg);

/* ---- measurement ---------------------------------------------------------- */

/* When enabled, every launch of the fused step kernel is bracketed by CUDA
 * events on the handle's stream; lbm_get_kernel_time returns the summed
 * device time (ms) and launch count since the last reset. */
int lbm_set_kernel_timing(lbm_handle* h, int enable);
int lbm_get_kernel_time(lbm_handle* h, double* total_ms, long* launches);
/* Number of CUDA kernels this handle has launched (graph replays counted
 * per kernel node). */
long lbm_get_launch_count(lbm_handle* h);
/* Bytes per cell update the fused step moves by algorithm: 2*19*sizeof(store). */
int lbm_bytes_per_cell(lbm_handle* h);
/* The handle's CUDA stream (a cudaStream_t), for callers that record their
 * own CUDA events around library calls. */
void* lbm_get_stream(lbm_handle* h);
/* Host<->device bytes the handle has copied since lbm_init (source
 * schedules, control blocks and uploads in; probe series and results out). */
int lbm_get_transfer_bytes(lbm_handle* h, long* h2d, long* d2h);

/* ---- bounds-checked build (liblbm_b200_check.so, compiled with -DLBM_CHECK) --
 * (no counterpart in the reference).  In that build every device access of
 * the step, source, ghost, probe, adjoint-step and scheme-A kernels that
 * could leave its array is tested first; a failing test records where (a
 * site code, csrc/check.cuh) and the offending index, and the access is
 * skipped, so the GPU never faults.  lbm_check_status synchronises the
 * handle's stream, returns the first recorded failure on the handle's device
 * (site 0: none) and clears it; the product build returns
 * LBM_ERR_UNSUPPORTED.  lbm_check_selftest launches a kernel that fails one
 * test on purpose (site 99, no memory access), to show the mechanism works. */
int lbm_check_status(lbm_handle* h, long long* site, long long* index);
int lbm_check_selftest(lbm_handle* h);

/* ---- synthetic geometry -------------------------------------------------- */

/* Fills tris (capacity triangles, 9 floats each) with the city's boxes
 * (12 triangles per building).  Returns LBM_ERR_CAPACITY with *ntris set to
 * the required count when tris is too small.  *coverage receives the plan
 * fraction achieved. */
int lbm_city_generate(const lbm_city_params* p, float* tris, int capacity, int* ntris, double* coverage);
/* Writes a binary STL file (80-byte header, uint32 count, 50-byte records;
 * the format GeometryEngine::load reads, 06:49-58, 06:70-111). */
int lbm_stl_write(const char* path, const float* tris, int ntris);

#ifdef __cplusplus
}
#endif

#endif /* NLOS_LBM_H */
