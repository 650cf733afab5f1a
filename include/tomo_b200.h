/*
 * tomo_b200 -- B200-native (sm_100a) hot path of 3D first-arrival traveltime tomography:
 * batched eikonal solve -> ray tracing into a sparse Frechet matrix -> CGLS -> model
 * update.  Plain C ABI: opaque context, plain pointers and sizes, int status codes.
 *
 * Conventions
 *  - Volumes are float32, z fastest, then x, then y: idx = z + x*nz + y*nx*nz, exactly
 *    the reference layout (src/eikonal/block_FIM/block_FIM.cpp:17, files written by
 *    numpy as (nz,nx,ny) Fortran order, src/utils/py_codes/functions.py:23-25).
 *  - Positions are metres from the model origin; shot i / receiver r order is the
 *    caller's (the reference's Geometry x/y/z arrays, src/geometry/geometry.hpp:21-24).
 *  - Every call returns TOMO_OK (0) or a negative TOMO_ERR_*; tomo_last_error(ctx) gives
 *    a message.  Nothing crosses the ABI as an exception and nothing calls exit().
 *  - Host buffers belong to the caller and are only read/written during the call.
 *    Device memory belongs to the context.  One host thread per context at a time.
 *  - All device work of a context runs on one CUDA stream (its own, or the one given to
 *    tomo_ctx_create_on_stream); calls return after that work completes.
 */
#ifndef TOMO_B200_H
#define TOMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOMO_OK                 0
#define TOMO_ERR_INVALID_ARG   -1  /* bad sizes, pointers, positions outside the model */
#define TOMO_ERR_OOM           -2  /* device allocation failed                          */
#define TOMO_ERR_CUDA          -3  /* CUDA runtime error (message has the detail)       */
#define TOMO_ERR_NOT_CONVERGED -4  /* eikonal round cap reached before the fixed point  */
#define TOMO_ERR_TIMEOUT       -5  /* a device-side wait hit its iteration limit        */
#define TOMO_ERR_STATE         -6  /* call order (no model / no solve / no Jacobian)    */
#define TOMO_ERR_IO            -7  /* file could not be opened / short read             */
#define TOMO_ERR_NO_DEVICE     -8  /* no CUDA device, or not sm_100                      */
#define TOMO_ERR_CAPACITY      -9  /* a fixed device capacity was exceeded              */

typedef struct tomo_ctx tomo_ctx;

/* Model grid: x_samples, y_samples, z_samples and x/y/z_spacing of parameters.txt
 * (run/parameters.txt:5-11). */
typedef struct {
    int nx, ny, nz;
    float dx, dy, dz;
} tomo_grid;

typedef struct {
    float x, y, z;
} tomo_point;

/* Lateral solve window of one shot: nodes [x0,x1) x [y0,y1), full depth, inside the model
 * and at least 2 x 2 nodes, at any origin.  Each windowed solve equals the reference solve
 * on the model cropped to that window.  Windows whose x0, y0 are multiples of 4 and whose
 * x1 (y1) is a multiple of 4 or nx (ny) read whole bricks of the device model; any other
 * window reads its slowness node by node from the same model (no copy). */
typedef struct {
    int x0, x1, y0, y1;
} tomo_window;

/* Local Godunov operator of the eikonal solve. */
#define TOMO_OP_JW  0  /* Jeong & Whitaker 2008 first-order update, isotropic h = dx, single
                          node source seed: Block_FIM (src/eikonal/block_FIM/cuda_kernel.cu:217-248) */
#define TOMO_OP_NGB 1  /* Noble, Gesret & Belayouni 2014 operator with dx, dy, dz and the 27-node
                          seed, run as the reference's 8 source-anchored + 8 full sweeps:
                          Accurate_FSM (src/eikonal/accurate_FSM/accurate_FSM.cpp:159-650),
                          reproduced bit for bit */

typedef struct {
    int op;          /* TOMO_OP_*                                                     */
    int max_inner;   /* cap of in-brick iterations per activation (0: default 16)     */
    int max_rounds;  /* cap of outer rounds (0: default 1<<20)                        */
    int brick;       /* brick shape of the JW solve: TOMO_BRICK_4 (4x4x4, one warp per
                        brick) or TOMO_BRICK_8 (8x8x8, one CTA of 8 warps per brick, each
                        warp on one of its 4x4x4 sub-bricks; rounds schedule, no time band);
                        0: the autotuned shape, if any, else 4x4x4                     */
    int block_warps; /* warps per CTA of the persistent kernel, 1-16 (0: default 16;
                        the asynchronous schedule uses at most 8)                     */
    int occupancy;   /* register budget of the kernel, in CTAs of 8 warps per SM, 1..6
                        (0: default 4, i.e. 64 registers)                             */
    float change_tol;/* a face value must drop by more than this (s) to re-queue the
                        neighbour brick.  0: default 1e-6 s, the reference's EPS
                        (cuda_kernel.cuh:8); < 0: any drop (exact FP32 fixed point) */
    float inner_tol; /* in-brick relaxation stops when no node drops by more than this
                        (s).  <= 0: exact (default)                                  */
    int ieee_sqrt;   /* 1: IEEE sqrtf in the local update; 0 (default): sqrt.approx  */
    int sweep_groups;/* TOMO_OP_NGB schedule.  0 (default): tile wavefront -- one warp
                        per 16x8x8 tile of a sweep in shared memory, tiles in diagonal
                        order behind their upwind tiles, one grid barrier per sweep;
                        batches with a source on the last node of its window along an
                        axis take the plane schedule.  > 0: the diagonal-plane schedule
                        (a barrier per plane) with that many independent block groups
                        sweeping their own shots.  Both are bit-exact with the reference
                        where every source lies off the far faces of its window.        */
    int schedule;    /* TOMO_OP_JW work schedule: TOMO_SCHED_DEFAULT, TOMO_SCHED_ROUNDS,
                        TOMO_SCHED_ASYNC                                              */
    float time_band; /* ROUNDS schedule, time-band ordering (s).  Every push carries the
                        smallest new time of the pushing brick; a queued brick whose key
                        is more than time_band above the smallest key its shot met in
                        the previous round waits for a later round, so late, too-high
                        arrivals (a slow path reaching a brick before a faster diving
                        path) do not start re-activation cascades.  0 (default): off.
                        Same fixed point either way.  Measured with 0.2 s: 2.3x faster
                        on the config-5 starting model (v = 1500 + z, 0.34 x the brick
                        activations), 1.18x on config 3, slower on the windowed config-2
                        batch.  0: the band tomo_eik_autotune chose on this context, if
                        any, else off; < 0: off.  Untuned banded solves default to 8
                        warps per CTA at occupancy 3 (80 registers).  Ignored by the warm-started solve and
                        the ASYNC schedule.                                           */
    unsigned long long spin_limit; /* polls (>= 32 ns each) a device-side wait -- the round
                        barrier of the persistent solve, the NGB sweep barriers, the
                        ASYNC schedule's queue waits -- makes before it gives up: the
                        solve then ends with TOMO_ERR_TIMEOUT and the context stays usable
                        (0: default 2^26, i.e. seconds).  Replaces the unbounded wait of
                        block_FIM_solver's outer loop (cuda_kernel.cu:91).              */
} tomo_eik_opts;

/* Brick shapes of the JW solve (tomo_eik_opts.brick; tomo_eik_brick_shapes lists them). */
#define TOMO_BRICK_4 1
#define TOMO_BRICK_8 2

/* Work schedules of the JW solve (same fixed point, different order of brick updates).
 * ROUNDS (default): bricks queued during a round are relaxed in the next one, rounds
 *   separated by a grid-wide barrier -- a wavefront order; max_rounds caps the rounds.
 * ASYNC: no rounds -- one work ring, a brick is relaxed as soon as a warp is free;
 *   max_rounds caps the activations at max_rounds x the batch's bricks.  Measured 2.5x
 *   slower than ROUNDS on the config-2 batch (bricks relaxed before their upwind
 *   neighbours settle are relaxed again: 1.8x the activations). */
#define TOMO_SCHED_DEFAULT 0
#define TOMO_SCHED_ROUNDS  1
#define TOMO_SCHED_ASYNC   2
/* PAIR: the ROUNDS schedule with two 4x4x4 bricks per warp (16 lanes each, a y-column of 4
 *   nodes per lane), sharing the item fetch and queueing.  DEFAULT runs it for banded
 *   solves (time_band > 0) and when the autotuner chose it; ROUNDS keeps one brick per
 *   warp. */
#define TOMO_SCHED_PAIR    3

typedef struct {
    long long rounds;            /* outer rounds of the persistent solve                  */
    long long activations;       /* brick activations (sum over shots)                    */
    long long inner_iterations;  /* sum over activations of in-brick iterations           */
    long long nodes_per_brick;   /* nodes of one brick                                    */
    long long idle_activations;  /* activations that lowered no node (JW)                 */
    float setup_ms;              /* device time of the pool reset + seeding kernels       */
    float solve_ms;              /* device time of the persistent solve kernel             */
    float total_ms;              /* device time of the whole call incl. copies             */
    long long deferred;          /* queued bricks put off to a later round (time_band)    */
} tomo_eik_stats;

/* ---------------------------------------------------------------- context ---------- */
/* Replaces Eikonal::set_parameters + prepare_volumes (src/eikonal/eikonal.hpp:48-49) for
 * the device side: binds device `device` (must be sm_100) and records the grid. */
int tomo_ctx_create(const tomo_grid *grid, int device, tomo_ctx **out);
/* Same, but all device work is enqueued on the caller's stream (a cudaStream_t). */
int tomo_ctx_create_on_stream(const tomo_grid *grid, int device, void *stream, tomo_ctx **out);
/* Replaces Eikonal::destroy_volumes (eikonal.hpp:57). */
int tomo_ctx_destroy(tomo_ctx *ctx);
/* Message of the last failed call on ctx; with ctx == NULL, of the last failed
 * context-free call (tomo_eik_solve_static) on this host thread. */
const char *tomo_last_error(const tomo_ctx *ctx);
const char *tomo_status_string(int status);
/* The cudaStream_t the context enqueues on. */
void *tomo_ctx_stream(tomo_ctx *ctx);

/* --------------------------------------------------------------- the model --------- */
/* Velocity model (m/s), host, nz*nx*ny; slowness = 1/v as Eikonal::set_parameters does
 * (block_FIM.cpp:85-91). */
int tomo_set_velocity(tomo_ctx *ctx, const float *velocity);
/* Slowness model (s/m), host, nz*nx*ny. */
int tomo_set_slowness(tomo_ctx *ctx, const float *slowness);
/* Copies the current slowness (after model updates) to the host. */
int tomo_get_slowness(tomo_ctx *ctx, float *slowness_out);
/* Staged velocity upload, for callers that solve one model after another.
 * tomo_stage_velocity starts copying the next velocity model (m/s, host, nz*nx*ny) into
 * device staging memory on the context's own copy stream and returns without waiting, so
 * the copy overlaps the work already queued on the context (a solve of the current model).
 * tomo_commit_velocity then makes the staged model the context's model (slowness = 1/v,
 * as tomo_set_velocity) once its copy has landed, without blocking the host.  The host
 * buffer must stay valid and unchanged until a blocking call on the context (a solve) has
 * returned after the commit; the copy overlaps only from page-locked host memory.
 * tomo_commit_velocity without a staged model returns TOMO_ERR_STATE. */
int tomo_stage_velocity(tomo_ctx *ctx, const float *velocity);
int tomo_commit_velocity(tomo_ctx *ctx);

/* ------------------------------------------------------------ eikonal solve --------- */
/* Solves nshots first-arrival traveltime fields in ONE persistent launch.
 * Replaces the per-shot loop of Eikonal::eikonal_equation + write_first_arrival
 * (src/eikonal/eikonal_main.cpp:31-39, src/tomography/least_squares/least_squares.cpp:172-183;
 * device part: block_FIM_solver, src/eikonal/block_FIM/cuda_kernel.cu:17-215).
 *   shots      nshots source positions (metres)
 *   windows    NULL (full model) or nshots windows
 *   receivers  nrec receiver positions (may be NULL if nrec == 0)
 *   t_recv     host nshots*nrec (row-major shot, receiver) receiver times by trilinear
 *              interpolation (block_FIM.cpp:228-262); NULL keeps them on the device only
 *   opts/stats may be NULL.
 * Traveltime fields stay on the device for tomo_eik_volume(s) and tomo_build_jacobian. */
int tomo_eik_solve(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows,
                   int nrec, const tomo_point *receivers, float *t_recv,
                   const tomo_eik_opts *opts, tomo_eik_stats *stats);

/* Copies the traveltime field of shot `shot` of the last solve to the host, cropped to
 * its window: wz*wx*wy floats (z fastest) -- Eikonal::travel_time after
 * eikonal_equation (block_FIM.cpp:59-69, 371-401). */
int tomo_eik_volume(tomo_ctx *ctx, int shot, float *t_out);

/* Window extents of shot `shot` of the last solve (nodes). */
int tomo_eik_window(tomo_ctx *ctx, int shot, tomo_window *out);

/* All traveltime fields of the last solve, device to device: shot s's window volume
 * (nz*wx*wy floats, z fastest) at offset sum_{r<s} nz*wx_r*wy_r of the DEVICE array dst. */
int tomo_eik_volumes(tomo_ctx *ctx, float *dst);

typedef struct {
    long long violations;              /* nodes below the update of their final neighbours
                                          by more than 5e-7 (relative)                       */
    float max_deficit;                 /* largest (update - time) / update over those nodes   */
    int shots_fallback;                /* shots solved again from INF (plain FIM)            */
    long long rounds_seeded;           /* outer rounds of the warm-started launch            */
    long long activations_seeded;      /* brick activations of the warm-started launch       */
    long long inner_iterations_seeded; /* in-brick iterations of the warm-started launch     */
    float seeded_ms;                   /* device time of the warm-started launch             */
    float verify_ms;                   /* device time of the check                           */
    float fallback_ms;                 /* device time of the fallback solves (0 if none)     */
    long long stuck;                   /* nodes that kept their ceiling value (never lowered) */
} tomo_seed_stats;

/* Warm-started batch solve: tomo_eik_solve (JW operator), but every window node starts at
 * ceiling x (1 + inflate) instead of INF, so that only updates that beat the ceiling
 * propagate.  No counterpart in the reference (its solvers always start from INF).
 *   ceiling  DEVICE array, all shots' window volumes back to back as tomo_eik_volumes
 *            writes them: predicted traveltimes (s).  Entries <= 0 or non-finite: no
 *            ceiling at that node.
 *   inflate  in [0, 1): margin that makes the prediction an upper bound
 * A ceiling below the true time would stay in the result, so every shot is checked after
 * the solve.  A shot is solved again from INF within the call (the plain solver is the
 * fallback) when any node (source node excepted) still holds its ceiling value, bit for
 * bit -- the solve never lowered it -- or lies below the local update of its final
 * neighbours.  Every node of a correct result is an update of its neighbours, and a
 * ceiling below the truth always leaves nodes that kept it (the wrong node of smallest
 * time has correct upwind neighbours), so the check catches smooth deficits of any size.
 * A ceiling is therefore accepted only where the solve lowered every node: use inflate
 * well above the solver's tolerances (0.02; an exact field with inflate 0 falls back).
 * stats counts both launches; seed_stats (may be NULL) splits them. */
int tomo_eik_solve_seeded(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows,
                          int nrec, const tomo_point *receivers, float *t_recv, const float *ceiling,
                          float inflate, const tomo_eik_opts *opts, tomo_eik_stats *stats,
                          tomo_seed_stats *seed_stats);

/* Brick shapes the solver supports, in TOMO_BRICK_* order (4x4x4, 8x8x8): writes up to
 * `cap` triples (bx,by,bz) of nodes and returns how many there are. */
int tomo_eik_brick_shapes(int *xyz_triples, int cap);

typedef struct {
    int trials;        /* launch shapes timed                                           */
    float best_ms;     /* device time of the persistent solve with the chosen shape      */
    float default_ms;  /* the same with the built-in default shape                      */
} tomo_tune_stats;

/* Autotuner of the JW solve (no counterpart in the reference, whose launch shape is fixed).
 * Solves this batch (no receivers) with every launch shape -- 4x4x4 bricks: warps per CTA
 * {16, 8, 4} x CTAs per SM {3, 4, 5, 6} x in-brick iteration cap {8, 16, 32}; two 4x4x4
 * bricks per warp (TOMO_SCHED_PAIR): warps {8, 4, 16} x CTAs per SM {3, 4} at the chosen
 * cap; 8x8x8 bricks: CTAs of 8 warps per SM {2, 3, 4, 5} x cap {16, 32} -- `repeats` times
 * each (0: 2), then,
 * at the fastest 4x4x4 shape, the time band at 3, 6, 9 and 12 times the slowest brick
 * crossing (4 dx s_max; none is the shape's own time) and, if a band wins, the warps x
 * CTAs-per-SM shapes again with it.
 * Keeps the fastest in the context and writes it to *best (may be NULL).  Later solves on this context use the tuned value for every tomo_eik_opts field
 * they leave 0.  The traveltime pool holds the last trial's fields afterwards. */
int tomo_eik_autotune(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows,
                      int repeats, tomo_eik_opts *best, tomo_tune_stats *stats);

/* Allocation-free single-shot solve, for callers that cannot call cudaMalloc (their
 * application already owns the GPU's memory through its own pool, or must stay within
 * a fixed device-memory budget).  No counterpart in the reference: it has no library
 * boundary, and its Block_FIM allocates and frees device memory for every shot.
 *   slowness  device pointer, nz*nx*ny floats (z fastest), read only
 *   t_out     device pointer, nz*nx*ny floats: the traveltime field, as tomo_eik_volume
 *   stream    cudaStream_t the work is enqueued on (NULL: default stream); the call
 *             returns after that work completes
 * Same operator, seed and tolerances as tomo_eik_solve.  The solver's working memory is a
 * fixed device array inside the library (about 34.6 MB, reserved on each GPU where the
 * library's code is loaded, until the process exits), so the grid is limited to
 * 4,194,304 nodes after padding each axis to a multiple of 4; larger grids return
 * TOMO_ERR_CAPACITY.  All calls on a device share that array: calls whose GPU work
 * overlaps race and must not be issued.  The first call on a device looks up the array's
 * address with that device current; make it before any stream capture.  Later calls
 * look the address up again unless their stream is capturing, so a call after
 * cudaDeviceReset finds the array where the reloaded module put it.  The call blocks
 * until its work on `stream` is done (it reads the solver's error word back).  Errors:
 * tomo_last_error(NULL). */
int tomo_eik_solve_static(const float *slowness, int nx, int ny, int nz, float dx, float dy, float dz, float sx,
                          float sy, float sz, float *t_out, void *stream);

/* ------------------------------------------------- ray tracing and the Jacobian ------- */
typedef struct {
    float dx, dy, dz;       /* inversion cell size: dx_tomo, dy_tomo, dz_tomo (parameters.txt)  */
    int tk_order;           /* Tikhonov order (tk_order)                                         */
    float tk_param;         /* lambda (tk_param)                                                 */
    int max_ray_steps;      /* step cap per ray (0: 20 x the grid diagonal in ray steps)         */
    int max_cells_per_ray;  /* distinct cells one ray may cross (0: 1024)                        */
    int illumination;       /* 1: accumulate the illumination volume (least_squares.cpp:234)     */
} tomo_jacobian_opts;

typedef struct {
    int nx, ny, nz;               /* inversion grid (least_squares.cpp:124-126)            */
    long long rows, cols;         /* N = n_data + n_model - tk_order, M = n_model          */
    long long nnz_rays, nnz;      /* non-zeros of G, of A = [G ; lambda L]                 */
    long long rays, rays_ok, rays_stalled, rays_capped, rays_nonfinite, rays_outside, rays_overflow;
    long long ray_steps;          /* total marching steps                                  */
    float ms;                     /* device time of ray tracing + matrix assembly          */
} tomo_jacobian_stats;

/* Traces one ray per (shot, receiver) of the last tomo_eik_solve back through its
 * traveltime field and assembles the sparse Frechet matrix G and the Tikhonov rows on the
 * device: Least_squares::ray_tracing + tk_reg_matrix + the COO assembly of optimization
 * (src/tomography/least_squares/least_squares.cpp:192-280, 358-422, 321-347).  Row
 * ray + shot*nrec, column = inversion cell, value = run-length path length.  Rays the
 * reference would trace forever (stalled next to the source, zero gradient, step cap) are
 * cut and counted in the stats. */
int tomo_build_jacobian(tomo_ctx *ctx, const tomo_jacobian_opts *opts, tomo_jacobian_stats *stats);
/* Copies A = [G ; lambda L] in CSR to the host: row_ptr (rows+1), cols/vals (nnz). */
int tomo_jacobian_copy(tomo_ctx *ctx, int *row_ptr, int *cols, float *vals);
/* Per-ray status (nshots*nrec): 0 ok, 1 stalled at the source, 2 step cap, 3 zero
 * gradient, 4 outside the grid/window, 5 too many cells. */
int tomo_ray_status(tomo_ctx *ctx, int *status);
/* Illumination volume (nz*nx*ny) of the last tomo_build_jacobian with illumination = 1. */
int tomo_illumination(tomo_ctx *ctx, float *out);

/* ------------------------------------------------------------- inversion ----------- */
/* Observed picks, n = nshots*nrec (row-major shot, receiver): Least_squares::import_obs_data
 * (least_squares.cpp:144-161).  n must match the survey of the solve they are used with. */
int tomo_set_observed(tomo_ctx *ctx, const float *dobs, int n);

/* ------------------------------------------------- parameters.txt helpers --------- */
/* catch_parameter (src/utils/file_manager/file_manager.cpp:74-120) with its quirks: writes
 * the value of `key` in the parameter file to out (NUL-terminated, at most cap bytes) and
 * returns its length, or TOMO_ERR_INVALID_ARG if it does not fit. */
int tomo_catch_parameter(const char *key, const char *parameter_file, char *out, int cap);
/* Builds the "shots" or "nodes" geometry of a parameter file like Regular/Circular
 * set_geometry (src/geometry/regular/regular.cpp:29-56, circular/circular.cpp:5-30), incl.
 * writing its xyz text file; type 0 regular, 1 circular.  Writes up to cap points (x,y,z)
 * and returns the number of points, or a negative status. */
int tomo_geometry(const char *parameter_file, const char *name, int type, float *xyz, int cap);
/* ||dobs - dcal||_2 in FP64 with dcal the receiver times of the last solve:
 * Least_squares::converged (least_squares.cpp:301-319). */
int tomo_data_residual(tomo_ctx *ctx, double *norm);

typedef struct {
    int iterations;     /* iterations run                                      */
    double rnorm0;      /* ||B||                                               */
    double rnorm;       /* ||B - A x|| after the last iteration                */
    float ms;           /* device time                                         */
} tomo_cgls_stats;

/* CGLS on A x = [dobs - dcal ; 0]: Least_squares::optimization + sparse_cgls
 * (least_squares.cpp:321-356, 424-496).  FP32 matrix; FP64 vectors, row sums, inner
 * products and step lengths (FP32 vectors drift ~10 % from the FP64 iterates after 30
 * iterations on these ill-conditioned systems); one persistent launch.  x_out (host, M floats) and history (host, ||B - A x||
 * per iteration) may be NULL; the solution stays on the device for tomo_model_update. */
int tomo_cgls(tomo_ctx *ctx, int iterations, float *x_out, double *history, tomo_cgls_stats *stats);

typedef struct {
    int smooth;                /* smooth (parameters.txt)                          */
    int filter_samples;        /* filter_samples (odd)                             */
    float standard_deviation;  /* standard_deviation                               */
    int use_reference_masks;   /* 1 (default behaviour): the reference's hard-coded
                                  interior masks (least_squares.cpp:520, 559);
                                  0: no mask                                      */
} tomo_update_opts;

/* Least_squares::model_update (least_squares.cpp:498-570): trilinear coarse-to-fine of the
 * CGLS solution, optional Gaussian smoothing (src/utils/smoothing/gaussian.cpp:5-73),
 * slowness += dm, velocity = 1/slowness.  The device model is updated in place (as the
 * reference updates Eikonal::slowness); velocity_out (host nz*nx*ny) may be NULL. */
int tomo_model_update(tomo_ctx *ctx, const tomo_update_opts *opts, float *velocity_out);

/* ---------------------------------------------------------- one whole iteration ------ */
typedef struct {
    tomo_jacobian_opts jacobian;  /* inversion grid, Tikhonov, ray caps                      */
    int cg_iterations;            /* CGLS iterations (>= 1)                                   */
    tomo_update_opts update;      /* model update                                             */
    tomo_eik_opts eik;            /* eikonal solve (TOMO_OP_JW)                               */
    int use_graph;                /* 1: capture the iteration in CUDA graphs once, then replay */
    float nnz_headroom;           /* Jacobian capacity / first non-zero count, >= 1 (else 1.25) */
} tomo_iteration_opts;

typedef struct {
    double residual;        /* ||dobs - dcal|| of this iteration's forward model            */
    double cg_rnorm;        /* ||B - A x|| after the last CGLS iteration                     */
    long long nnz;          /* non-zeros of A = [G; lambda L]                                 */
    long long activations;  /* brick activations of the eikonal solve                         */
    int replayed;           /* 1: ran as replays of graphs captured by an earlier call         */
    int captured;           /* 1: a graph was (re)captured in this call                        */
    float ms;               /* device time of the iteration                                   */
} tomo_iteration_stats;

/* One tomography iteration on the device: eikonal solve of the batch with receiver times,
 * ray tracing into A = [G; lambda L], CGLS on B = [dobs - dcal; 0], model update -- the
 * body of the reference's loop (src/tomography/tomography_main.cpp:19-30: forward_modeling,
 * import_cal_data, converged, optimization, model_update).  Needs tomo_set_observed with
 * nshots x nrec picks.  With use_graph the device work runs as two CUDA graphs captured on
 * the first call (the second sized by the Jacobian's non-zero count x headroom) and
 * replayed on later calls; the host only reads the non-zero count in between.  Afterwards
 * the context holds the new model, the fields, A and x as after the per-stage calls. */
int tomo_iteration(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
                   const tomo_point *receivers, const tomo_iteration_opts *opts, tomo_iteration_stats *stats);

/* The reference's GPU CGLS entry point, sparse_cgls_gpu (src/utils/cgls/cgls.cuh:47):
 * host COO (iA, jA, vA; rows need not be sorted), host B and x, N rows, M columns, NIT
 * iterations, stop when ||A'(B - A x)|| < TOL.  Self-contained (own device buffers);
 * returns a status instead of printing. */
int tomo_sparse_cgls_gpu(const int *iA, const int *jA, const float *vA, const float *B, float *x, int N, int M,
                         int NNZ, int NIT, float TOL);

/* ------------------------------------------------ learned warm start (surrogate) ------ */
/* No counterpart in the reference (it has no learned component).  A 3D U-Net (4 levels,
 * 16/32/48/64 channels, 3x3x3 convolutions, ReLU) predicts the factored traveltime
 * tau = T / (s_src |x - x_src|) of one source from the slowness around it; BF16 tensor-core
 * convolutions with FP32 accumulation, trained on the device by the library's own
 * backward kernels and Adam.  Its prediction feeds tomo_eik_solve_seeded. */
typedef struct tomo_net tomo_net;

typedef struct {
    const float *slow;          /* DEVICE: model slowness, nz*nx*ny, z fastest            */
    int model_nx, model_ny, nz; /* that model's size                                      */
    tomo_window window;         /* the sample: lateral window (any origin), full depth    */
    tomo_point source;          /* metres, model coordinates, inside the window           */
    const float *T;             /* DEVICE: the window's traveltimes (nz*wx*wy, z fastest);
                                   training targets, unused by tomo_net_predict            */
} tomo_net_sample;

int tomo_net_create(int device, void *stream, unsigned long long seed, tomo_net **out);
int tomo_net_destroy(tomo_net *net);
const char *tomo_net_last_error(const tomo_net *net);
long long tomo_net_param_count(const tomo_net *net);
/* FP32 parameters (host): per convolution w[cout][27][cin] then b[cout], then the head. */
int tomo_net_get_params(tomo_net *net, float *out);
int tomo_net_set_params(tomo_net *net, const float *in);  /* also resets the optimiser */
/* Loss (mean squared tau error over nodes at distance >= h from the source) and its
 * gradient w.r.t. every parameter (host, may be NULL), without an update. */
int tomo_net_gradients(tomo_net *net, int n, const tomo_net_sample *samples, float h, double *loss, float *grads);
/* One Adam step (lr) on a batch of n samples of equal padded size; returns the loss. */
int tomo_net_train_step(tomo_net *net, int n, const tomo_net_sample *samples, float h, float lr, double *loss);
int tomo_net_evaluate(tomo_net *net, int n, const tomo_net_sample *samples, float h, double *loss);
/* Predicted traveltimes tau x s_src x distance for n samples, written to the DEVICE array
 * t_pred back to back (sample i's window volume, z fastest) -- the layout of
 * tomo_eik_volumes and of the ceiling of tomo_eik_solve_seeded; 0 within h of the source.
 * ms (may be NULL): device time. */
int tomo_net_predict(tomo_net *net, int n, const tomo_net_sample *samples, float h, float *t_pred, float *ms);
/* The same on a coarse grid: the network sees every stride-th node of each window (the
 * distance channel normalised by 64 h stride, so large windows stay in the range of the
 * 64^3 training tiles) at 1/stride^3 of the cost, and tau is interpolated trilinearly back
 * to every window node before T = tau s_src distance.  stride 1..16; 1 is tomo_net_predict. */
int tomo_net_predict_strided(tomo_net *net, int n, const tomo_net_sample *samples, float h, int stride, float *t_pred,
                             float *ms);

/* Training data: fills ctx's model with seeded random tiles (tile x tile nodes laterally,
 * full depth): 3-6 dipping layers of 1500-4500 m/s and 0-12 Gaussian anomalies of up to
 * +-15 %.  nx and ny must be multiples of tile. */
int tomo_random_tiles(tomo_ctx *ctx, int tile, unsigned long long seed);
/* The context's current slowness model on the device (nz*nx*ny, z fastest). */
const float *tomo_ctx_slowness_device(tomo_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* TOMO_B200_H */
