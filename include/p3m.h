/*
 * p3m.h — C-ABI of the B200 (sm_100a) P3M gravity step.
 *
 * This library replaces the P3M seam of Gravity's Kotlin `GravityPipeline`
 * (src/main/kotlin/dev/gravity/GravityPipeline.kt). That class has no FFI of
 * its own: the seam is the set of private methods that dispatch the GLSL
 * compute shaders. Each entry point below names the reference method or shader
 * it stands in for. The intended caller is a JNI shim inside `GravityPipeline`
 * (JDK 18 toolchain: build.gradle.kts:39-41), so every signature uses plain C
 * types, host or device pointers and sizes.
 *
 * Conventions
 *  - Every function returns an int status: P3M_OK (0) or a negative
 *    p3m_status. Nothing throws across the ABI. p3m_last_error() gives a
 *    one-line message for the last failing call of a context.
 *  - The library owns every device buffer of a context; the caller owns host
 *    arrays. Host arrays are read or written before the call returns.
 *  - All work of a context is ordered on its own CUDA stream. A context is
 *    used from one host thread at a time, like the GL context thread the
 *    reference runs on.
 *  - Units follow the reference: positions in unit coordinates [0,1)^2,
 *    velocities in unit/s, accelerations in unit/s^2
 *    (GravityPipeline.kt:752-756). Bodies are float4 (x, y, vx, vy); materials
 *    are float4 (mass, friction, solid, block) (GravityPipeline.kt:183-192).
 */
#ifndef GRAVITY_P3M_H
#define GRAVITY_P3M_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P3M_ABI_VERSION 1

typedef enum p3m_status {
    P3M_OK = 0,
    P3M_ERR_INVALID_ARGUMENT = -1, /* Kotlin require() -> IllegalArgumentException */
    P3M_ERR_OUT_OF_MEMORY = -2,
    P3M_ERR_CUDA = -3,             /* a CUDA runtime call failed */
    P3M_ERR_TIMEOUT = -4,          /* a bounded device wait gave up */
    P3M_ERR_NON_FINITE = -5,       /* non-finite body state detected */
    P3M_ERR_CAPACITY = -6,         /* more bodies than the context holds */
    P3M_ERR_UNSUPPORTED = -7,      /* configuration outside the supported range */
    P3M_ERR_STATE = -8             /* Kotlin check() -> IllegalStateException */
} p3m_status;

/* Mass deposit arithmetic. U32 is the reference's uint32 fixed point with
 * massScale = clamp(4e9 / M_tot, 1, 65536) quanta per unit mass
 * (build_grid.comp:64-69, GravityPipeline.kt:1546-1547). I64 is the precision
 * form: int64 atomics with 2^-32 mass quanta, bit-reproducible at any size. */
typedef enum p3m_deposit_mode {
    P3M_DEPOSIT_U32 = 0,
    P3M_DEPOSIT_I64 = 1
} p3m_deposit_mode;

/* Gravity configuration; defaults from GravityFieldConfig
 * (GravityConfig.kt:641-654), CollisionConfig.timeStep / maximumSubsteps
 * (GravityConfig.kt:677-678) and ParticleConfig.spatialSortInterval
 * (GravityConfig.kt:621). Fill with p3m_config_default() first. */
typedef struct p3m_config {
    int32_t struct_size;                    /* sizeof(p3m_config) */
    int32_t viewport_width;                 /* domain width in px (aspect = w/h) */
    int32_t viewport_height;                /* domain height in px */
    int32_t grid_width;                     /* physical grid, power of two, 16..4096 */
    int32_t grid_height;                    /* physical grid, power of two, 16..4096 */
    float gravitational_constant;           /* 0.035 */
    float softening_cells;                  /* sigma in cells, 0.85 */
    float local_search_sigma_multiplier;    /* 3 */
    int32_t minimum_neighbor_radius_cells;  /* 1 */
    int32_t maximum_neighbor_radius_cells;  /* 6 */
    int32_t exact_neighbor_body_limit;      /* 2 */
    int32_t maximum_home_body_interactions; /* 8 */
    float minimum_distance_cell_fraction;   /* 0.05 */
    float minimum_assignment_window_power;  /* 0.08 */
    float time_step;                        /* 1/120 s */
    int32_t drift_substeps;                 /* 16 (collision substeps drift the bodies) */
    int32_t spatial_sort_interval;          /* 2; 0 disables the Morton reorder */
    int32_t capacity;                       /* bodies the context can hold */
    int32_t bounded;                        /* 0 torus, 1 walls (Hockney 2x mesh) */
    int32_t deposit_mode;                   /* p3m_deposit_mode */
    int32_t mutual_gravity;                 /* 1; 0 = uniform field only */
} p3m_config;

typedef struct p3m_ctx p3m_ctx;

/* Device buffers readable through p3m_debug_get / p3m_device_pointer. */
typedef enum p3m_buffer {
    P3M_BUF_BODIES = 0,       /* float4[n]  (x, y, vx, vy) */
    P3M_BUF_ACCELERATION = 1, /* float2[n]  last acceleration */
    P3M_BUF_MATERIALS = 2,    /* float4[n]  (mass, friction, solid, block) */
    P3M_BUF_CELL_KEYS = 3,    /* uint32[n]  home cell of each sorted entry */
    P3M_BUF_CELL_BODIES = 4,  /* int32[n]   body IDs sorted by (cell asc, ID desc) */
    P3M_BUF_CELL_START = 5,   /* int32[P]   first sorted entry of a cell (valid where count > 0) */
    P3M_BUF_CELL_COUNT = 6,   /* int32[P]   bodies per cell */
    P3M_BUF_CELL_MASS = 7,    /* uint32[P]  sum of round(mass * 256) per cell */
    P3M_BUF_DENSITY = 8,      /* uint32[M] (U32) or int64[M] (I64) fixed-point mesh */
    P3M_BUF_FORCE = 9,        /* float2[M]  long-range mesh force (fx, fy) */
    P3M_BUF_DESTINATIONS = 10,/* uint32[n]  new ID of every body after the last reorder */
    P3M_BUF_GREEN = 11,       /* float2[(MW/2+1)*MH] spectral multipliers (gx, gy) */
    P3M_BUF_COUNT_ = 12
} p3m_buffer;

/* ---- lifecycle ---------------------------------------------------------- */

/* Defaults of GravityFieldConfig / CollisionConfig / ParticleConfig for a
 * 2560x1440 domain and a 512x256 grid. */
int p3m_config_default(p3m_config* config);

/* Replaces the GravityPipeline constructor's P3M part: buffers
 * (GravityPipeline.kt:183-246), twiddles (initializeTwiddles, :1359-1371) and
 * the Green's-function spectra (initializeKernel, :1341-1357). Validation
 * mirrors GravityFieldConfig.init (GravityConfig.kt:655-673). */
int p3m_create(const p3m_config* config, p3m_ctx** out);

/* Replaces GravityPipeline.close (GravityPipeline.kt:1556-1620). */
int p3m_destroy(p3m_ctx* ctx);

/* Message of the last failing call of ctx (or of p3m_create when ctx is
 * NULL); never NULL. */
const char* p3m_last_error(const p3m_ctx* ctx);
const char* p3m_status_string(int status);

/* ---- state hand-off ----------------------------------------------------- */

/* Replaces seedBodies / glBufferSubData uploads (GravityPipeline.kt:724-770,
 * :1438-1481). Any pointer may be NULL to leave that buffer unchanged. State
 * pointers of these three calls may be host memory (pageable or page-locked)
 * or device memory of the context's device. */
int p3m_upload_state(p3m_ctx* ctx, const float* bodies4, const float* materials4,
                     const float* acceleration2, int32_t n);
/* Writes `count` bodies starting at slot `first` (first + count <= capacity),
 * leaving the other slots as they are: spawnProjectile / spawnBlock write new
 * bodies past the active ones with glBufferSubData at an offset
 * (GravityPipeline.kt:621-718). Slots beyond the active count keep their
 * contents across steps and reorders. */
int p3m_upload_range(p3m_ctx* ctx, int32_t first, int32_t count, const float* bodies4,
                     const float* materials4, const float* acceleration2);
/* Readback (the reference maps the SSBOs: GravityPipeline.kt:378-443).
 * Returns P3M_ERR_TIMEOUT, after writing the arrays, when a bounded
 * look-back wait gave up since the last report (see p3m_synchronize). */
int p3m_download_state(p3m_ctx* ctx, float* bodies4, float* materials4,
                       float* acceleration2, int32_t n);
/* Copy the first `bytes` of a buffer to host memory (at most its size). */
int p3m_debug_get(p3m_ctx* ctx, int32_t which, void* host, size_t bytes);
/* Device address and size of a buffer (for callers that share device memory,
 * e.g. a renderer); the pointer stays valid until p3m_destroy. */
int p3m_device_pointer(p3m_ctx* ctx, int32_t which, void** device, size_t* bytes);

/* ---- properties (GravityPipeline.kt:97-121) ----------------------------- */

/* `bounded` setter: walls need 2*max(grid) <= 4096 (GravityPipeline.kt:97-103). */
int p3m_set_bounded(p3m_ctx* ctx, int32_t bounded);
/* `fieldAccelerationX/Y` in px/s^2; stored as unit/s^2 like applyKick
 * (GravityPipeline.kt:1230-1234). */
int p3m_set_field_acceleration(p3m_ctx* ctx, float ax_px, float ay_px);
int p3m_set_mutual_gravity(p3m_ctx* ctx, int32_t enabled);
/* massExcess: mass of the active bodies minus their count (GravityPipeline.kt:213). */
int p3m_set_mass_excess(p3m_ctx* ctx, float mass_excess);

/* ---- the step (GravityPipeline.kt:366-370, :445-494) -------------------- */

/* initializeAcceleration(n): normalizeTo, buildForce, applyKick(initial). */
int p3m_initialize_acceleration(p3m_ctx* ctx, int32_t n);
/* step(n) repeated `steps` times, gravity only: Morton reorder every
 * spatial_sort_interval steps, half kick + drift substeps, buildForce,
 * applyKick. Collisions, liquid and sleep are not part of this path. */
int p3m_step(p3m_ctx* ctx, int32_t n, int32_t steps);

/* step(n) with its host I/O pipelined against the neighbouring steps:
 * host_bodies_in4 (may be NULL) becomes the first n bodies before the step,
 * as p3m_upload_state would make it, and the stepped bodies go to
 * host_bodies_out4 (may be NULL), as p3m_download_state would write them.
 * The call only enqueues: the copies run on the context's own copy streams
 * (one per direction) through device staging buffers (2 x 16 B per body of
 * capacity, allocated at the first call), so the next call's upload overlaps
 * this step and this step's download overlaps the next step. Both host
 * arrays should be page-locked (p3m_host_alloc) for the copies to be
 * asynchronous; they must stay valid, and host_bodies_in4 unchanged, until
 * p3m_synchronize returns, which waits for every queued copy and reports
 * device failures like a download. The reference re-uploads and reads back
 * its SSBOs synchronously (GravityPipeline.kt:720-770, :378-443). */
int p3m_step_io(p3m_ctx* ctx, int32_t n, const float* host_bodies_in4, float* host_bodies_out4);

/* Launch shapes (results do not depend on them): FFT lines per CTA of the
 * row, column and inverse kernels (0: automatic, else 1..16, clamped to what
 * shared memory holds) and the short-range block (64, 128 or 256 threads).
 * Drops the captured step graphs. */
int p3m_set_launch_shape(p3m_ctx* ctx, int32_t fft_lines, int32_t short_range_threads);
/* Autotuner of one context: times `trial_steps` steps of its n active bodies
 * (after one untimed step) under each FFT line count (automatic, 1, 2, 4,
 * 8), then each short-range block with the best count, keeps the fastest
 * and puts the bodies, materials, accelerations and step counter back.
 * Writes (fft_lines, short_range_threads) to chosen2 when it is not NULL.
 * The reference has no counterpart (its dispatch sizes are fixed). */
int p3m_autotune(p3m_ctx* ctx, int32_t n, int32_t trial_steps, int32_t* chosen2);

/* Separately callable stages, for parity tests and for a host that keeps its
 * own loop. */
int p3m_sort_bodies(p3m_ctx* ctx, int32_t n);                   /* sortBodies, :1269-1319 */
int p3m_drift(p3m_ctx* ctx, int32_t n, float kick_dt, float drift_dt); /* collision_build.comp:40-51 */
int p3m_build_force(p3m_ctx* ctx, int32_t n);                   /* buildForce, :907-973 */
int p3m_apply_kick(p3m_ctx* ctx, int32_t n, int32_t initial);   /* applyKick, :1213-1261 */
/* Cell keys, their sort and the cell lists only (the first part of
 * build_grid.comp, as CSR lists). The keys are 32-bit home cells written in
 * descending body ID; a stable LSD radix sort over the cell bits then gives
 * the reference's (cell, ~id) order. */
int p3m_build_cell_lists(p3m_ctx* ctx, int32_t n);

/* Steps run as CUDA graphs captured once per (body count, reorder step,
 * current buffer, uniforms) and replayed (default on); 0 launches kernels one
 * by one. Profiling (p3m_profile_enable) always launches one by one. */
int p3m_set_graphs(p3m_ctx* ctx, int32_t enabled);

/* Wait for the context's stream. Returns the first pending CUDA error, else
 * the first failure the device detected since the last report, each reported
 * once: P3M_ERR_TIMEOUT when a bounded look-back wait of a sort gave up (the
 * cell lists, and everything computed from them since, are invalid), then
 * P3M_ERR_NON_FINITE when the drift met bodies with non-finite state (the
 * reference counts these in measureCluster, GravityPipeline.kt:817-819).
 * The stepping calls are asynchronous like CUDA launches: a failure inside
 * them surfaces at the next p3m_synchronize (or, for a timeout, the next
 * p3m_download_state). */
int p3m_synchronize(p3m_ctx* ctx);

/* ---- profiling and diagnostics ----------------------------------------- */

/* Stages of the step, timed with CUDA events on the context's stream
 * (the reference's GpuProfiler stages, GpuTimer.kt:17-40). */
typedef enum p3m_stage {
    P3M_STAGE_SPATIAL_SORT = 0, /* Morton reorder (SPATIAL_SORT) */
    P3M_STAGE_DRIFT = 1,        /* half kick + drift substeps + cell keys */
    P3M_STAGE_CELL_LISTS = 2,   /* cell-key radix sort + list build */
    P3M_STAGE_DEPOSIT = 3,      /* CIC deposit (GRAVITY_GRID) */
    P3M_STAGE_FORWARD_FFT = 4,  /* row transform (FORWARD_FFT) */
    P3M_STAGE_SPECTRAL = 5,     /* column transforms + Green's multiply (CONVOLUTION) */
    P3M_STAGE_INVERSE_FFT = 6,  /* row inverse (INVERSE_FFT_X/Y) */
    P3M_STAGE_KICK = 7,         /* interpolation + half kick (GRAVITY_KICK) */
    P3M_STAGE_SHORT_RANGE = 8,  /* short-range correction (GRAVITY_KICK, near field) */
    P3M_STAGE_COUNT_ = 9
} p3m_stage;

/* Start (enabled != 0, accumulators cleared) or stop recording stage events. */
int p3m_profile_enable(p3m_ctx* ctx, int32_t enabled);
/* Synchronises, then returns accumulated device milliseconds and the number
 * of timed intervals per stage (arrays of P3M_STAGE_COUNT_ entries). */
int p3m_profile_read(p3m_ctx* ctx, double* total_ms, int64_t* intervals);

/* Kernels this library has launched in this process (all contexts). */
int64_t p3m_kernel_launches(void);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events after the library's. */
int p3m_get_stream(p3m_ctx* ctx, void** stream);

/* Page-locked host memory for fast hand-off (cudaHostAlloc / cudaFreeHost). */
int p3m_host_alloc(size_t bytes, void** host);
int p3m_host_free(void* host);

/* Non-finite bodies the drift has seen since the context was created
 * (the reference counts them in measureCluster, GravityPipeline.kt:817-819). */
int p3m_nonfinite_count(p3m_ctx* ctx, int64_t* count);

/* Bounded device-side waits that gave up since the context was created. The
 * cell and Morton sorts find each tile's output offsets by looking back at
 * the tiles before it; every such wait has a poll limit, so a kernel always
 * ends. A nonzero count means a wait ran out and the results since then
 * cannot be trusted; p3m_synchronize and p3m_download_state report the
 * growth as P3M_ERR_TIMEOUT. Expected to stay 0. No counterpart in the reference
 * (its sorts are the atomic pushes of build_grid.comp and
 * spatial_sort_scatter.comp). */
int p3m_wait_timeouts(p3m_ctx* ctx, int64_t* count);

/* Test hook of the timeout path; no counterpart in the reference. Sets how
 * many times a look-back wait polls before it gives up (1..; 200,000 by
 * default) and a tile index whose counts the sort never publishes (-1: none,
 * the default). With a tile withheld, the waits of the tiles after it run
 * out: they end, are counted (p3m_wait_timeouts) and p3m_synchronize returns
 * P3M_ERR_TIMEOUT. Nothing faults; the results of such a sort are wrong.
 * Restore (200000, -1) to return to normal operation. */
int p3m_set_lookback_fault(p3m_ctx* ctx, int32_t poll_limit, int32_t withheld_tile);

/* validateFft (GravityPipeline.kt:378-419): the density spectrum of the last
 * force build, as the FP32 path computes it, against an FP64 transform of
 * the same density mesh (value / massScale, or / 2^32 for the int64 form),
 * both on the device. out3 = {maximum absolute error, maximum absolute error
 * / maximum |reference component|, RMS error} over every real and imaginary
 * component of the full MW x MH spectrum (the half spectrum extended by its
 * Hermitian symmetry). Periodic mesh only: P3M_ERR_STATE inside walls, as
 * the reference's check(!bounded), and before any force build. Blocking;
 * allocates its FP64 work buffers for the call. */
int p3m_validate_fft(p3m_ctx* ctx, double* out3);

/* The FP32 density spectrum of the last force build (forward 2D real FFT of
 * the density / massScale): (MW/2 + 1) * MH complex float2 values, row ky
 * then column kx, i.e. numpy.fft.rfft2's layout of the (MH, MW) mesh.
 * `bytes` is the capacity of `spectrum2` (host memory). Walls: the 2x mesh.
 * P3M_ERR_STATE before any force build. Blocking. */
int p3m_density_spectrum(p3m_ctx* ctx, float* spectrum2, size_t bytes);

/* FP64 direct-sum acceleration (unit/s^2) of `n_targets` bodies (IDs in
 * `targets`, host array) from all n bodies: the law the P3M split
 * approximates, G*m*d / (M_tot * max(r^2, r_min^2)) with the minimum image on
 * the torus and the open sum inside walls. Writes 2*n_targets doubles to host
 * `out`. Diagnostic; no counterpart kernel in the reference. */
int p3m_direct_accel_f64(p3m_ctx* ctx, int32_t n, const int32_t* targets, int32_t n_targets,
                         double* out);

/* FP64 conservation diagnostics of the first n bodies, in px units:
 * out[0..1] momentum sum(m*v), out[2] kinetic energy sum(m*v^2/2),
 * out[3..4] centre of mass, out[5] total mass. Deterministic reduction. */
int p3m_diagnostics_f64(p3m_ctx* ctx, int32_t n, double* out6);

/* ---- batched form ------------------------------------------------------- */

/* Many independent simulations of uneven body counts and grid sizes — the
 * application's trajectory previews (trajectory.comp, GravityPipeline.kt:
 * 514-600) and ensembles — stepped together: each simulation is a full
 * context, and one batch step is one CUDA graph that forks to every
 * simulation's stream, runs its step and joins (captured once per set of body
 * counts, reorder phases, buffers and uniforms, then replayed). The
 * reference runs one simulation per GravityPipeline. */
typedef struct p3m_batch p3m_batch;

/* count configurations, one per simulation. */
int p3m_batch_create(const p3m_config* configs, int32_t count, p3m_batch** out);
int p3m_batch_destroy(p3m_batch* batch);
/* Message of the last failing batch call (or of p3m_batch_create when NULL). */
const char* p3m_batch_last_error(const p3m_batch* batch);
int p3m_batch_size(const p3m_batch* batch, int32_t* count);
/* The context of one simulation (for downloads, diagnostics, debug reads;
 * its stream is ordered after the batch's only through p3m_batch_synchronize). */
int p3m_batch_context(p3m_batch* batch, int32_t sim, p3m_ctx** ctx);
/* Upload n bodies (and materials, may be NULL) and make them simulation
 * sim's active bodies. */
int p3m_batch_upload(p3m_batch* batch, int32_t sim, const float* bodies4,
                     const float* materials4, int32_t n);
/* initializeAcceleration of every simulation. */
int p3m_batch_initialize_acceleration(p3m_batch* batch);
/* `steps` steps of every simulation, one graph launch per step. */
int p3m_batch_step(p3m_batch* batch, int32_t steps);
/* Autotuner. Fused form: times `trial_steps` whole batch steps (after four
 * untimed ones) under each candidate and keeps the fastest, by coordinate
 * descent: the form (one launch per stage, or one persistent launch), FFT
 * lines per CTA (automatic, 1, 2, 4, 8) for each distinct grid in turn, then
 * for the persistent form its CTAs per SM (as many as fit, 1, 2, 3); every
 * simulation's state is saved before and restored after (the choice of form
 * stays; p3m_batch_plan_info reports it). Other
 * form: for each distinct grid, times `trial_steps` steps of its largest
 * simulation under each FFT line count and short-range block (64, 128, 256
 * threads) and restores that simulation's state. Writes up to 64 rows of
 * (grid_width, grid_height, fft_lines, short_range_threads) to `chosen` when
 * it is not NULL. Results do not depend on the choices. */
int p3m_batch_autotune(p3m_batch* batch, int32_t trial_steps, int32_t* chosen);
/* Fused form (the default): the stages of a batch step run over all
 * simulations at once -- one launch per stage (the default), or ONE
 * persistent cooperative launch per step (p3m_batch_set_persistent) --
 * captured once per plan. Off: every simulation enqueues its own step (one graph over
 * the simulations' streams). All forms give the same bits. The fused form
 * needs every simulation at most 131,072 bodies; a batch with a larger one
 * runs the other form. */
int p3m_batch_set_fused(p3m_batch* batch, int32_t enabled);
/* One batch step with its host I/O pipelined against the neighbouring steps
 * (p3m_step_io for the whole batch): host_bodies_in4 (may be NULL) holds
 * every simulation's n bodies back to back, in simulation order, and becomes
 * their bodies before the step; the stepped bodies go to host_bodies_out4
 * (may be NULL) in the same layout. One copy per direction on the batch's
 * copy streams, through device staging buffers (2 x 16 B per body of the
 * simulations' capacities, allocated at the first call), and one row-copy
 * launch each way between the staging and the simulations: the next call's
 * upload overlaps this step and this step's download the next step. The
 * arrays should be page-locked (p3m_host_alloc) and must stay valid, the
 * input unchanged, until p3m_batch_synchronize returns. */
int p3m_batch_step_io(p3m_batch* batch, const float* host_bodies_in4, float* host_bodies_out4);
/* Persistent form of the fused step (default off; the autotuner picks the
 * faster form): one cooperative launch whose CTAs stay resident and run the
 * step's stages phase by phase, a bounded grid barrier between phases. Its
 * one register budget is the largest stage's (the radix scatter's), so it
 * keeps fewer warps per SM than the per-stage launches; it wins where the
 * launches' gaps outweigh that (many short stages). ctas_per_sm: CTAs per SM (0: as many
 * as stay resident; larger values are clamped to that). A batch with a
 * short-range stencil other than 3x3 cells (interaction radius), or whose
 * stages cannot stay resident, takes the per-stage launches instead. */
int p3m_batch_set_persistent(p3m_batch* batch, int32_t enabled, int32_t ctas_per_sm);
/* Test hook of the persistent form's grid barrier: each wait polls the
 * arrival counter at most poll_limit times (default 1 << 20, a few
 * milliseconds to a second), then gives up, counts the wait and ends its CTA;
 * withheld_cta (>= 0) never arrives at the barrier after phase `phase` (a
 * CTA that does not arrive). -1 / -1 clears it. P3M_ERR_INVALID_ARGUMENT for
 * poll_limit <= 0 or values below -1. */
int p3m_batch_set_barrier_fault(p3m_batch* batch, int32_t poll_limit, int32_t withheld_cta,
                                int32_t phase);
/* The plan of the last fused step: info4 = (persistent 0/1, kernel launches
 * per step, phases, CTAs of the persistent launch). All zero before one. */
int p3m_batch_plan_info(p3m_batch* batch, int32_t* info4);
/* Device time of each phase of the last persistent step (global-timer
 * stamps by CTA 0 as it leaves each phase's barrier), in milliseconds, up to
 * `capacity` values; *phases = the number of phases (0 when the last step was
 * not persistent). Synchronises the batch's stream. */
int p3m_batch_phase_times(p3m_batch* batch, double* ms, int32_t capacity, int32_t* phases);
/* Waits for the batch's stream. P3M_ERR_TIMEOUT (once per new occurrence)
 * when a grid barrier of a persistent step gave up: the simulations' state
 * is then incomplete and must be uploaded again. */
int p3m_batch_synchronize(p3m_batch* batch);
int p3m_batch_get_stream(p3m_batch* batch, void** stream);

/* ---- differentiated rollout ---------------------------------------------- */

/* A hand-written adjoint of the gravity-only step (GravityPipeline.kt:445-494
 * without collisions; the reference has no adjoint), as a forward/backward
 * pair: p3m_adjoint_forward runs `steps` plain steps from the current state,
 * saving bodies and accelerations every `interval` steps;
 * p3m_adjoint_backward takes the cotangents of the final state and returns
 * those of the initial state, recomputing each segment from its checkpoint.
 * The cell topology (monopole cells, summed list entries) is held fixed
 * where the positions are differentiated, and the fixed-point deposit is
 * taken as its real value. Torus only (walls: P3M_ERR_UNSUPPORTED), and the
 * context's spatial_sort_interval must be 0 (the rollout keeps body order).
 * State pointers may be host memory or device memory of the context's
 * device. Changing the state, the uniforms or the body count between the
 * two calls gives meaningless gradients. */
#define P3M_ADJOINT_INITIAL_ACCELERATION 1 /* a0 = initializeAcceleration(x0):
                                              the backward folds da0 into dx0 */
int p3m_adjoint_forward(p3m_ctx* ctx, int32_t n, int32_t steps, int32_t interval, int32_t flags);
/* seed_bodies4: dL/d(x, y, vx, vy) of the final state (unit coordinates);
 * seed_accel2: dL/d(final a), may be NULL (zero). Writes dL/d(initial
 * x, y, vx, vy) and, if grad_accel2 is not NULL, dL/d(initial a) (zero when
 * the forward computed a0 itself). Synchronous. Leaves the context in the
 * forward's final state. */
int p3m_adjoint_backward(p3m_ctx* ctx, const float* seed_bodies4, const float* seed_accel2,
                         float* grad_bodies4, float* grad_accel2);
/* Frees the checkpoints and recompute storage. */
int p3m_adjoint_release(p3m_ctx* ctx);

/* ---- aim previews --------------------------------------------------------- */

/* TrajectoryConfig (GravityConfig.kt:739-756) plus the collision
 * restitution the preview bounces off walls with (GravityConfig.kt:682). */
typedef struct p3m_trajectory_config {
    int32_t struct_size;                    /* sizeof(p3m_trajectory_config) */
    int32_t steps;                          /* 1..65536 (1024) */
    float maximum_time_step;                /* s (1) */
    float target_segment_pixels;            /* (6) */
    float maximum_path_viewport_diagonals;  /* (1) */
    float minimum_dash_pixels;              /* (3) */
    float restitution_coefficient;          /* [0, 1] (0) */
} p3m_trajectory_config;

int p3m_trajectory_config_default(p3m_trajectory_config* config);

/* updateTrajectory (GravityPipeline.kt:514-600, trajectory.comp) for `count`
 * previews at once, on the field of the last force build for n bodies (a
 * step or initializeAcceleration; P3M_ERR_STATE otherwise): origins and
 * launch velocities in px and px/s (count x 2 floats each); vertices: count x
 * steps x 6 (x, y, dash coordinate px, distance fraction or -1 when unused)
 * floats x 4, the reference's trajectory buffer per preview. Pointers may be
 * host or device memory. Synchronous. */
int p3m_trajectories(p3m_ctx* ctx, int32_t n, const p3m_trajectory_config* config, int32_t count,
                     const float* origins_px2, const float* velocities_px2, float* vertices4);

/* ---- cell lists without allocation ------------------------------------- */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory when they need cell lists — code running where allocation is
 * forbidden or would stall (inside a frame callback, a captured region), or a
 * host whose device memory is handed out by another runtime (a JVM, an
 * engine). Builds the same lists as p3m_build_cell_lists — keys of the home
 * cells, the stable sort of 32-bit cell keys written in descending ID, the
 * CSR lists — from caller-owned device
 * arrays into caller-owned device arrays, on `stream` (a cudaStream_t, NULL
 * for the default stream), without calling cudaMalloc, cudaFree or any
 * allocating routine.
 *
 * Inputs: bodies4 (float4[n]) and materials4 (float4[n]) on the current
 * device. Outputs: sorted_keys[n] (home cell per entry), sorted_ids[n] (body
 * IDs by cell ascending, ID descending), cell_start/cell_count/cell_mass of
 * grid_width*grid_height cells (start valid where count > 0; the entry point
 * zeroes all three first), entries4 (float4[n]: x, y, mass, ID bits).
 *
 * Limit: n <= P3M_CELL_LISTS_STATIC_MAX_BODIES; larger n returns
 * P3M_ERR_CAPACITY with a message in p3m_last_error(NULL). The working memory
 * is one array compiled into the library (about 16.3 MB held on every GPU that
 * loads it, until exit). The first call on each device looks up that array's
 * address (cudaGetSymbolAddress) with the device current; make that first call
 * before any stream capture. The address is kept for the life of the process:
 * after a cudaDeviceReset (or anything else that destroys the device's
 * primary context) it is stale, so do not call this entry point again in that
 * process. All calls share the array and it keeps the last
 * call's contents: calls whose work overlaps on the GPU race, so order them on
 * one stream. */
#define P3M_CELL_LISTS_STATIC_MAX_BODIES 1048576
int p3m_cell_lists_static(const float* bodies4, const float* materials4, int32_t n,
                          int32_t grid_width, int32_t grid_height, uint32_t* sorted_keys,
                          int32_t* sorted_ids, int32_t* cell_start, int32_t* cell_count,
                          uint32_t* cell_mass, float* entries4, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAVITY_P3M_H */
