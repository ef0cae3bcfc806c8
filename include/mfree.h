/*
 * mfree.h -- C ABI of the B200-native SPH cutting step (libmfree.so).
 *
 * One call of mfree_step() is one call of leap_frog::step() of iwf_mfree_gpu_3d
 * (src/leap_frog.cu:121-195): blanking, cell-list hash + stable sort, predictor,
 * EOS + artificial stress, pair interactions (Gray/Monaghan stress divergence,
 * artificial viscosity, XSPH, CSPM, Brookshaw or PSE conduction), Jaumann rate,
 * continuity, momentum, advection, corrector, Johnson-Cook radial return, rigid
 * tool contact with friction, friction heating, boundary conditions and the
 * translation of tool particles.
 *
 * The reference has no library boundary: its driver links C++ classes and
 * writes process globals.  Every entry point below names the reference call it
 * stands in for.  Conventions:
 *   - every call returns an int status (MFREE_OK = 0, negative on error; the
 *     message is in mfree_last_error()); nothing calls exit();
 *   - a context owns its device memory and frees it in mfree_destroy();
 *   - host buffers are caller-owned and copied;
 *   - calls on one context are not thread-safe; separate contexts are
 *     independent (the reference keeps its state in process globals);
 *   - arrays are in the current (sorted) particle order, as in the reference,
 *     with the reference's per-field layout (particle_gpu.h:36-99).
 *
 * Units are the reference's cm-g-us system (stress in Mbar).
 */
#ifndef MFREE_H_
#define MFREE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MFREE_OK              0
#define MFREE_ERR_ARG        -1  /* bad argument or call order            */
#define MFREE_ERR_CUDA       -2  /* CUDA runtime error                    */
#define MFREE_ERR_OOM        -3  /* device allocation failed              */
#define MFREE_ERR_NUMERIC    -4  /* device-reported numerical failure     */
#define MFREE_ERR_IO         -5  /* scene file could not be read/parsed   */
#define MFREE_ERR_EMPTY      -6  /* every particle left the box: the
                                    reference prints and exit(0)s
                                    (grid_gpu_base.cu:159-163)            */
#define MFREE_ERR_BUDGET     -7  /* admitting the scene would exceed the
                                    batch's device-memory budget          */
#define MFREE_ERR_TIMEOUT    -8  /* a bounded device wait ran out (the
                                    pair kernel's staging): the step that
                                    reported it is incomplete             */

/* ---- constant records (constants_structs.h:25-92) ----------------------- */
typedef struct { float E, nu, rho0, K, G, mass; } mfree_phys;          /* phys_constants */
typedef struct { float cp, tq, k, alpha, T_init, eta; } mfree_trml;    /* trml_constants */
typedef struct { float wdeltap, stresseps, xspheps, alpha, beta, eta; } mfree_corr; /* corr_constants */
typedef struct { float A, B, C, n, m, Tmelt, Tref, eps_dot_ref, clamp_temp; } mfree_joco; /* joco_constants */

/* ---- switches that are #defines in the reference (types.h:32-108) ------- */
#define MFREE_COND_NONE      0
#define MFREE_COND_BROOKSHAW 1   /* Thermal_Conduction_Brookshaw (types.h:104) */
#define MFREE_COND_PSE       2   /* Thermal_Conduction_PSE (types.h:105)       */

typedef struct {
    int cspm;               /* CSPM kernel correction (types.h:102)                  */
    int conduction;         /* MFREE_COND_*                                            */
    int precision;          /* 0: FP32 state; 1: FP32 bulk + compensated hi/lo
                               position and velocity in predictor/corrector          */
    int max_secant_iter;    /* Johnson-Cook secant limit (plasticity.cuh:66: 100)     */
    int lanes_per_particle; /* pair-loop tiling: 8, 16 or 32 lanes of a warp per
                               particle; 0 picks the tuned default                   */
    int diagnostics;        /* 1: keep neighbour counts, half-step positions and
                               contact normals for mfree_get_field()                  */
    int friction_tool_vel;  /* 1: subtract the tool velocity in the friction slip
                               velocity.  The reference never uploads its tool_vel
                               constant (tool_3d_gpu.cu:26,528), so 0 matches it.    */
    int tile_depth;         /* pair-loop tiling: cells per tile along z, 1..8; 0 picks
                               the tuned default (6).  Results do not depend on it.   */
    int full_stencil;       /* 1: the pair loop visits every candidate of the 5x5x5
                               cell stencil and evaluates every term.  0 (default):
                               it skips the stencil cells that lie wholly beyond the
                               target's support radius -- with PSE conduction only on
                               tiles whose PSE sums are exactly zero (every
                               temperature their stencils reach equal), where it also
                               skips the PSE terms.  Results do not depend on it.     */
} mfree_options;

/* ---- fields for mfree_get_field / mfree_set_field ------------------------
 * element layout = the reference's particle_gpu member (float4 = 4 floats,
 * float3 = 3 floats, mat3x3 = 9 floats in GLM column-major order m[col][row]). */
enum mfree_field {
    MFREE_POS = 0,        /* float4 */
    MFREE_VEL,            /* float4 */
    MFREE_VEL_BC,         /* float4 */
    MFREE_H,              /* float  */
    MFREE_RHO,            /* float  */
    MFREE_P,              /* float  (pressure of the last half step)           */
    MFREE_S,              /* mat3x3 */
    MFREE_R,              /* mat3x3 (artificial stress of the last half step)  */
    MFREE_FC,             /* float3 */
    MFREE_FT,             /* float3 */
    MFREE_NRM,            /* float3 contact normal (diagnostics only)          */
    MFREE_FIXED,          /* float  */
    MFREE_BLANKED,        /* float  */
    MFREE_TOOL_PARTICLE,  /* float  */
    MFREE_EPS_PL,         /* float  */
    MFREE_EPS_PL_DOT,     /* float  */
    MFREE_T,              /* float  */
    MFREE_POS_T,          /* float3 */
    MFREE_VEL_T,          /* float3 */
    MFREE_RHO_T,          /* float  */
    MFREE_S_T,            /* mat3x3 */
    MFREE_T_T,            /* float  */
    MFREE_NUM_NBH,        /* int    (diagnostics only)                         */
    MFREE_IDX,            /* int    sort permutation of the last step           */
    MFREE_HASH,           /* int    sorted cell ids, INT_MAX = blanked          */
    MFREE_ID,             /* int    particle id = index at creation (new)      */
    MFREE_POS_HALF,       /* float4 half-step positions (diagnostics only)     */
    MFREE_NUM_FIELDS
};

/* ---- compact structure-of-arrays access ----------------------------------
 * The library's own particle arrays: n_init float4 entries each, current
 * sorted order, the deviatoric stress as its 6 independent components (no
 * counterpart in the reference, whose particle_gpu keeps one array per field;
 * one copy instead of a per-field conversion). */
enum mfree_array {
    MFREE_A_POS_H = 0,    /* (x, y, z, h)                                      */
    MFREE_A_VEL_RHO,      /* (vx, vy, vz, rho)                                 */
    MFREE_A_S_A,          /* (Sxx, Syy, Szz, Sxy)                              */
    MFREE_A_S_B,          /* (Sxz, Syz, T, eps_pl)                             */
    MFREE_A_POS_T,        /* (xdot, ydot, zdot, rho_t)                         */
    MFREE_A_VEL_T,        /* (vx_t, vy_t, vz_t, T_t)                           */
    MFREE_A_S_T_A,        /* (Sxx_t, Syy_t, Szz_t, Sxy_t)                      */
    MFREE_A_S_T_B,        /* (Sxz_t, Syz_t, eps_pl_dot, fixed)                 */
    MFREE_A_FC,           /* (fc.x, fc.y, fc.z, tool_particle)                 */
    MFREE_A_FT,           /* (ft.x, ft.y, ft.z, blanked)                       */
    MFREE_A_VEL_BC,       /* (vbc.x, vbc.y, vbc.z, id as int bits)             */
    MFREE_A_LO,           /* precision form: (x_lo, y_lo, z_lo, vx_lo)         */
    MFREE_A_LO_B,         /* precision form: (vy_lo, vz_lo, 0, 0)              */
    MFREE_NUM_ARRAYS
};

/* per-context counters of device-detected conditions */
typedef struct {
    int64_t steps;              /* steps taken                                          */
    int64_t secant_failures;    /* radial returns that hit the iteration limit
                                   (the reference printf's, actions_gpu.cu:415-418)     */
    int64_t out_of_grid;        /* non-blanked particles outside the cell grid; they are
                                   blanked (the reference prints ALARM and writes out of
                                   bounds, grid_gpu_green.cu:56-58)                     */
    int64_t contact_search_cap; /* contact shell searches stopped by the bound          */
    int64_t nan_blanked;        /* blanked particles with a NaN/Inf position or rate,
                                   summed over steps                                    */
    int64_t staging_timeouts;   /* pair-kernel staging waits that ran out (each makes
                                   the next call return MFREE_ERR_TIMEOUT)              */
    int64_t full_stencil_steps; /* steps whose pair loop fell back to the full 5x5x5
                                   stencil because a particle moved too far in the
                                   predictor (variants without PSE; see full_stencil) */
    int64_t bounds_errors;      /* bounds-checked library only: data-derived indices
                                   that fell outside their array (always 0 otherwise) */
    int64_t pse_zero_targets;   /* PSE conduction: targets whose PSE sum was exactly zero
                                   because every temperature their tile's stencils reach
                                   was equal (with finite positions and volumes); the
                                   pair loop skipped the PSE terms and pruned the stencil
                                   for them, with the same results, summed over steps */
} mfree_counters;

typedef struct mfree_ctx mfree_ctx;

/* ---- context ------------------------------------------------------------ */

/* particle_gpu(pos, vel, rho, T, h, fixed, tool_p, N) (particle_gpu.h:300-304,
 * particle_gpu.cu:20-117).  pos/vel: n float4; T, fixed, tool_p may be NULL
 * (zeros, as the shorter reference constructors).  stream: the cudaStream_t
 * every call of this context is ordered on, or NULL for a stream the context
 * creates (and destroys) itself. */
int mfree_create(int n, const float *pos4, const float *vel4, const float *rho,
                 const float *T, const float *h, const float *fixed,
                 const float *tool_p, void *stream, mfree_ctx **out);
int mfree_destroy(mfree_ctx *ctx);
const char *mfree_last_error(void);

/* actions_setup_physical_constants + interactions_setup_physical_constants
 * (actions_gpu.cu:659-665, interactions_gpu.cu:564-569) */
int mfree_set_physics(mfree_ctx *ctx, const mfree_phys *phys);
/* actions_/interactions_setup_corrector_constants (actions_gpu.cu:667-674,
 * interactions_gpu.cu:571-573) */
int mfree_set_correctors(mfree_ctx *ctx, const mfree_corr *corr);
/* actions_setup_johnson_cook_constants (actions_gpu.cu:676-679): switches
 * plasticity on */
int mfree_set_johnson_cook(mfree_ctx *ctx, const mfree_joco *joco);
/* actions_setup_thermal_constants_wp + interactions_setup_thermal_constants_workpiece
 * (actions_gpu.cu:681-698, interactions_gpu.cu:575-590) */
int mfree_set_thermal_workpiece(mfree_ctx *ctx, const mfree_trml *trml);
/* actions_setup_thermal_constants_tool + interactions_setup_thermal_constants_tool
 * (actions_gpu.cu:700-710, interactions_gpu.cu:592-608) */
int mfree_set_thermal_tool(mfree_ctx *ctx, const mfree_trml *trml);
int mfree_set_options(mfree_ctx *ctx, const mfree_options *opt);
int mfree_get_options(const mfree_ctx *ctx, mfree_options *opt);

/* grid_gpu_green(num_part, bbmin, bbmax, h): locked cell grid
 * (grid_gpu_green.cu:342-346, grid_gpu_base.cu:237-273) */
int mfree_set_grid(mfree_ctx *ctx, const float bbmin[3], const float bbmax[3], float h);
/* grid_base::set_bbox_vel (grid_gpu_base.cu:113-115): moving locked grid */
int mfree_set_grid_velocity(mfree_ctx *ctx, const float vel[3]);
/* grid_gpu_green(max_cell, num_part) (grid_gpu_green.cu:336-340,
 * grid_gpu_base.cu:275-278): the unlocked grid.  Before every step the grid
 * box becomes the bounding box of the active particles (+-1e-6) and the cell
 * edge their largest h (update_geometry, grid_gpu_base.cu:185-233); a grid of
 * max_cell cells or more fails the step with MFREE_ERR_ARG (the reference
 * asserts).  Each step reads the box back to the host, so steps of such a
 * context run eagerly (mfree_advance does not capture a graph) and the
 * context cannot join a batch.  mfree_set_grid locks the grid again. */
int mfree_set_grid_adaptive(mfree_ctx *ctx, long max_cell);
/* blanking(bbmin, bbmax, [bbvel,] max_vel) (blanking.cpp:29-33) */
int mfree_set_blanking(mfree_ctx *ctx, const float bbmin[3], const float bbmax[3],
                       const float *bbvel3, float max_vel);

/* global_time_dt / global_time_current / global_time_step (mfree_gpu_3d.cpp:45-48).
 * mfree_step() uses t_current and then adds dt to it, as main() does after each
 * loop iteration (mfree_gpu_3d.cpp:203-204). */
int mfree_set_time(mfree_ctx *ctx, float dt, float t_current);
int mfree_get_time(const mfree_ctx *ctx, float *dt, float *t_current);

/* ---- tools --------------------------------------------------------------- */
#define MFREE_CONTACT_HASHED     0  /* tool_3d_gpu::contact_algorithm::spatial_hashing */
#define MFREE_CONTACT_EXHAUSTIVE 1  /* tool_3d_gpu::contact_algorithm::exhaustive      */

/* mesh_compute_vertex_normals + mesh_average_edge_length + tool_3d(tris, pos, h)
 * + tool_3d_gpu(tool, vel, phys, alpha) + set_mu + set_algorithm_type
 * (surface_tri_mesh.cpp:410-584, tool_3d.cpp:294-360, tool_3d_gpu.cu:688-812).
 * verts: nv*3 floats; tris: nt*3 vertex indices of a closed manifold.
 * The contact mass is the particle mass of mfree_set_physics. */
int mfree_add_tool(mfree_ctx *ctx, const float *verts, int nv, const int *tris, int nt,
                   const float vel[3], float contact_alpha, float mu, int algorithm,
                   int *tool_index);
/* tool_3d_gpu::set_birth_death (tool_3d_gpu.cu:698-701) */
int mfree_tool_set_birth_death(mfree_ctx *ctx, int tool, float birth, float death);
/* tool_forces::get_forces_host (tool_3d_gpu.cu:34-38): 3 floats per tool,
 * summed over the particles in a fixed order (the reference uses atomicAdd) */
int mfree_get_tool_forces(mfree_ctx *ctx, float *out3);
/* tool geometry of the setup: boxed-triangle count, tri-grid cells and bbox */
int mfree_get_tool_info(mfree_ctx *ctx, int tool, int *num_tris, int *num_boxed,
                        int *grid_n3, float *bbmin3, float *bbmax3, float *cell_dx);
/* per-triangle normals after setup: face n, vertex np1..3, edge ne1..3 as
 * 7 float3 per triangle in input order (surface_tri_mesh.h:39-63) */
int mfree_get_tool_normals(mfree_ctx *ctx, int tool, float *out21);
/* triangle grid of the setup: cells = CSR offsets (grid cells + 1 entries) into
 * the boxed triangles, boxed_src = input index of each boxed triangle
 * (grid_cpu_tri::get_cells, grid_cpu_tri.cpp:96-175) */
int mfree_get_tool_cells(mfree_ctx *ctx, int tool, int *cells, int *boxed_src);

/* ---- stepping ------------------------------------------------------------ */
/* leap_frog::step(particles, grid, record_forces) (leap_frog.cu:121-195) */
int mfree_step(mfree_ctx *ctx, int record_forces);
/* nsteps calls of mfree_step; forces recorded every record_every steps
 * (0: never).  With use_graph != 0 the step is captured once into a CUDA graph
 * and replayed. */
int mfree_advance(mfree_ctx *ctx, int nsteps, int record_every, int use_graph);
/* block the host until the context's stream is idle */
int mfree_sync(mfree_ctx *ctx);

/* ---- state access -------------------------------------------------------- */
int mfree_get_counts(const mfree_ctx *ctx, int *n_active, int *n_init);
/* count elements of one particle's entry of a field (4 for float4 ...) */
int mfree_field_width(int field);
/* copy a whole field (n_init entries) to / from host memory.  When out is
 * page-locked (cudaMallocHost / cudaHostAlloc / cudaHostRegister) the state
 * fields are written into it by the device in one pass; otherwise they are
 * copied and converted on the host.  The values are the same either way. */
int mfree_get_field(mfree_ctx *ctx, int field, void *out);
int mfree_set_field(mfree_ctx *ctx, int field, const void *in);
/* the same in double: MFREE_POS and MFREE_VEL return hi + lo of the
 * compensated accumulation when options.precision = 1 */
int mfree_get_field_f64(mfree_ctx *ctx, int field, double *out);
/* the compact arrays (enum mfree_array): copy one array (4 * n_init floats)
 * to / from host memory */
int mfree_get_array(mfree_ctx *ctx, int array, float *out4);
int mfree_set_array(mfree_ctx *ctx, int array, const float *in4);
/* the device address of the array's current copy, for callers that read it
 * on the device in stream order; valid until the next step (each step writes
 * the other of two copies) */
int mfree_array_device_ptr(mfree_ctx *ctx, int array, void **dptr);
/* cell ranges in the reference format (cell_start/cell_end, -1 = empty;
 * grid_gpu_green.cu:24-70,277-278), num_cell entries each */
int mfree_get_cells(mfree_ctx *ctx, int *cell_start, int *cell_end);
/* grid geometry after set_geometry (grid_gpu_base.cu:237-273) */
int mfree_get_grid(const mfree_ctx *ctx, long *nx, long *ny, long *nz,
                   float *bbmin3, float *dx);
int mfree_get_counters(mfree_ctx *ctx, mfree_counters *out);
/* FP64 reductions over the active workpiece particles of the current state
 * (no counterpart in the reference, which steps with a fixed dt and reports
 * no energies): out[0] kinetic energy sum m|v|^2/2, out[1] deviatoric elastic
 * energy sum (m/rho) S:S/(4G), out[2] volumetric elastic energy sum
 * (m/rho) p^2/(2K) with p = c0^2 (rho - rho0), out[3] thermal energy
 * sum m cp (T - T_init), out[4] the CFL time-step bound min h/(c + |v|) with
 * c = sqrt(K/rho) (multiply by the CFL number).  In the precision form
 * (options.precision = 1) the velocity is hi + lo of the compensated
 * accumulation.  Computed in double on the device in a fixed order (the same
 * bits on every call for the same state). */
int mfree_get_energies(mfree_ctx *ctx, double out[5]);
/* 1 in the bounds-checked build of the library (libmfree_checked.so, a debug
 * stand-in for a memory checker; no counterpart in the reference), else 0 */
int mfree_bounds_checked(void);
/* Failure injection for tests (no reference counterpart).  MFREE_FAULT_STAGING_WAIT
 * raises the byte count the pair kernel's staging waits expect, so every wait
 * runs out after its bound (~0.5 s), the kernel counts it and leaves, and the
 * next call returns MFREE_ERR_TIMEOUT; nothing faults and the CUDA context
 * stays usable.  MFREE_FAULT_NONE switches it off. */
#define MFREE_FAULT_NONE         0
#define MFREE_FAULT_STAGING_WAIT 1
int mfree_inject_fault(mfree_ctx *ctx, int kind);

/* ---- measurement (no reference counterpart) --------------------------------
 * Per-kernel device time of eager mfree_step calls: when on, CUDA events
 * bracket every kernel of a step on the context's stream.  Kernel order:
 * clock, hash, scan_reduce, scan_top, scan_down, scatter, cell_fixup,
 * gather_predict, interact, finalize, force_final (MFREE_NUM_KERNELS). */
#define MFREE_NUM_KERNELS 11
int mfree_set_kernel_timing(mfree_ctx *ctx, int on);
/* accumulated milliseconds and launch counts per kernel since the last call;
 * synchronises the stream and resets the accumulators */
int mfree_get_kernel_times(mfree_ctx *ctx, double *ms, int *launches);
/* sustained FP32 FMA throughput of the current device in TFLOP/s */
int mfree_probe_fp32_peak(double *tflops);
/* device-timed region on the context's stream (CUDA events) */
int mfree_timer_start(mfree_ctx *ctx);
int mfree_timer_stop(mfree_ctx *ctx, double *ms);
/* select the CUDA device for the contexts created afterwards on this thread
 * (one process per GPU) */
int mfree_set_device(int device);

/* ---- cell-list build without allocation -----------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory while they run (a host whose device memory is
 * reserved up front by its own allocator, or code that cannot afford the
 * device synchronisation a cudaMalloc may cause).  It computes what the
 * step's cell-list build computes -- the cell id (int)((x - bbmin)/dx) of each
 * position, the stable sort by cell id and the cell ranges -- with its
 * scratch in a fixed-size __device__ array of the library instead of
 * allocated buffers, and calls no allocation routine.
 *   pos4:       device pointer, n float4 positions (w ignored)
 *   bbmin, dx, nx, ny, nz: the grid (mfree_get_grid)
 *   perm:       device pointer, n ints out: sorted position -> input index;
 *               positions outside the grid, and positions with a NaN or
 *               infinite coordinate, come last, in input order (as in the
 *               step's truncating hash, a coordinate less than one cell below
 *               the grid's lower corner still falls in cell 0 of its axis)
 *   cell_first: device pointer, nx*ny*nz + 1 ints out: index of the first
 *               sorted position of each cell; cell_first[nx*ny*nz] = number of
 *               positions inside the grid
 *   stream:     cudaStream_t, or NULL for the legacy default stream
 * Limits: n <= MFREE_STATIC_MAX_PARTICLES and nx*ny*nz <= MFREE_STATIC_MAX_CELLS,
 * else MFREE_ERR_ARG.  The array (about 3 MiB) is held on every GPU that loads
 * the library until the process exits.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: after cudaDeviceReset on a device, do not call this function on
 * that device again.  All calls share the array and it keeps the last
 * call's contents (the counters are cleared at the start of each call): calls
 * that overlap on the GPU race. */
#define MFREE_STATIC_MAX_PARTICLES 262144
#define MFREE_STATIC_MAX_CELLS     524288
int mfree_cell_list_static(const float *pos4, int n, const float bbmin[3], float dx, int nx, int ny, int nz,
                           int *perm, int *cell_first, void *stream);

/* ---- batches: many scenes stepped together ------------------------------
 * The reference runs one scene per process (main(), mfree_gpu_3d.cpp:75-218);
 * these calls have no counterpart there.  A batch holds independent scenes
 * of any sizes (each an mfree_ctx, configured as for mfree_step) and steps
 * all of them with one launch per kernel: every scene keeps its own state and
 * cell list, and a scene's results are the same alone and in a batch when the
 * pair-loop tiling is the same.  Scenes are admitted and retired between
 * steps (continuous batching): admission is bounded by a device-memory
 * budget, and a scene may be admitted with a step count after which it stops.
 * All scenes of a batch share the pair-kernel variant (cspm, conduction,
 * precision options) and the tiling (lanes per particle, tile depth). */
typedef struct mfree_batch mfree_batch;

/* hbm_budget: device bytes the admitted scenes may hold (0: no limit).
 * stream: cudaStream_t, or NULL for a stream of the batch's own. */
int mfree_batch_create(size_t hbm_budget, void *stream, mfree_batch **out);
/* destroys the batch and every context it still holds */
int mfree_batch_destroy(mfree_batch *b);
/* Admits a configured context; on success the batch owns it (its work moves to
 * the batch's stream and mfree_step/mfree_advance on it are refused until it
 * is retired).  steps > 0: the scene stops after that many batch steps
 * (status done); steps <= 0: it runs until retired.  MFREE_ERR_BUDGET: its
 * device memory does not fit the budget (the caller keeps the context).
 * MFREE_ERR_ARG: its pair-kernel variant differs from the batch's. */
int mfree_batch_admit(mfree_batch *b, mfree_ctx *ctx, long long steps, int *slot);
/* Advances every running scene by up to nsteps steps (a scene stops at its
 * step count; the others go on).  record_every > 0: tool forces are recorded
 * on steps whose index is a multiple of it.  use_graph: each step replays one
 * captured CUDA graph covering all scenes (re-captured when scenes join or
 * leave). */
int mfree_batch_step(mfree_batch *b, int nsteps, int record_every, int use_graph);
/* slot state: *done steps run, *target requested (<= 0: unbounded),
 * *status 0 running, 1 done, 2 free slot, < 0 the scene's error status */
int mfree_batch_query(mfree_batch *b, int slot, long long *done, long long *target, int *status);
/* the slot's context, for the field and force calls (the batch still owns it) */
int mfree_batch_context(mfree_batch *b, int slot, mfree_ctx **ctx);
/* Removes a scene.  ctx != NULL: ownership returns to the caller (on its
 * original stream); ctx == NULL: the context is destroyed. */
int mfree_batch_retire(mfree_batch *b, int slot, mfree_ctx **ctx);
/* scenes held, running scenes, device bytes held by them and the budget */
int mfree_batch_info(mfree_batch *b, int *scenes, int *running, size_t *bytes, size_t *budget);
/* Pair-loop tiling of the batch: lanes per particle (8, 16, 32) and tile depth
 * (1..8 cells); 0 keeps the current value. */
int mfree_batch_set_tiling(mfree_batch *b, int lanes_per_particle, int tile_depth);
int mfree_batch_get_tiling(mfree_batch *b, int *lanes_per_particle, int *tile_depth);
/* Autotuner: times every tiling (lanes per particle x tile depth 4..8) for
 * trial_steps steps on copies of the batch's running scenes (their own state
 * is untouched) and keeps the fastest.  The cell size stays the reference's
 * (the smoothing length), which the bit-exact cell ids and order require.
 * *ms_best: time per step of the chosen tiling (may be NULL). */
int mfree_batch_autotune(mfree_batch *b, int trial_steps, int *lanes_per_particle, int *tile_depth, double *ms_best);
/* waits for the batch's queued work; CUDA-event timer on the batch's stream
 * (device milliseconds between start and stop) */
int mfree_batch_sync(mfree_batch *b);
int mfree_batch_timer_start(mfree_batch *b);
int mfree_batch_timer_stop(mfree_batch *b, double *ms);
/* device bytes a context holds (state, scratch and tools) */
int mfree_device_bytes(const mfree_ctx *ctx, size_t *bytes);
/* device bytes mfree_create + mfree_set_grid will take for n particles and
 * num_cell grid cells, before tools: to check a budget before creating */
size_t mfree_scene_bytes(int n, long long num_cell);

/* ---- checkpoint and resume (no counterpart in the reference) ---------------
 * mfree_export_state writes the context's configuration, tools (as their input
 * meshes), device clock, last recorded tool forces and particle state into one
 * binary record; with buf NULL it only sets *size to the bytes needed.
 * mfree_import_state creates a context from such a record (stream NULL: a
 * stream of its own); stepping it continues bitwise as the exported context
 * would. */
int mfree_export_state(mfree_ctx *ctx, void *buf, size_t *size);
int mfree_import_state(const void *buf, size_t size, void *stream, mfree_ctx **out);

/* ---- output in the reference's formats ------------------------------------
 * Particles as legacy VTK, the reference's vtk_writer_write(particle_gpu*)
 * (vtk_writer.cpp:78-262): the unblanked particles in sorted order with density,
 * contact, Temperature, Fixed, Tool, EquivAccumPlasticStrain and Svm.  The state
 * is snapshot on the context's stream by device copies; the copy to the host
 * (on a stream of its own) and the file writing (on a host thread) overlap the
 * steps that follow.  One particle output per context is in flight: the next
 * call, mfree_output_wait and mfree_destroy wait for it; a failure of the
 * writing is returned by the next of those calls. */
int mfree_write_vtk(mfree_ctx *ctx, const char *path);
int mfree_output_wait(mfree_ctx *ctx);
/* tool meshes at the last step's time, one file for all tools with "id" and
 * "active" point data (vtk_writer_write_unified, vtk_writer.cpp:307-386) */
int mfree_write_vtk_tools(mfree_ctx *ctx, const char *path);
/* the blanking box at the last step's time (vtk_writer_write_blanking, vtk_writer.cpp:22-77) */
int mfree_write_vtk_blanking(mfree_ctx *ctx, const char *path);
/* appends one line of the tool-force log, "%.9g %.9g %.9g " per tool and a
 * newline (tool_forces::report, tool_3d_gpu.cu:53-69); the forces are those of
 * the last recorded step, summed in a fixed order */
int mfree_append_force_log(mfree_ctx *ctx, const char *path);

/* ---- scene files (the reference's setup readers) ------------------------- */
/* json_read_triangles (json_reader.cpp:108-117): MeshLab JSON */
int mfree_read_mesh_json(const char *path, float **verts, int *nv, int **tris, int *nt);
/* ldynak_read_triangles_from_tetmesh (ldynak_reader.cpp:371-434): LS-DYNA .k */
int mfree_read_mesh_ldynak(const char *path, float **verts, int *nv, int **tris, int *nt);
/* ldynak_read_triangles_from_quadmesh (ldynak_reader.cpp:308-369): LS-DYNA .k of
 * hexahedral solids; each boundary face gives two triangles */
int mfree_read_mesh_ldynak_quad(const char *path, float **verts, int *nv, int **tris, int *nt);
void mfree_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* MFREE_H_ */
