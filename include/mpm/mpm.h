/*
 * mpm.h — C ABI of the B200 (sm_100a) MLS-MPM snow solver.
 *
 * This is the drop-in boundary for the reference's solver interface
 * (michal-sitarz2/MPM_Snow_Sim2D): the compile-time alias
 * `using Solver = GPUSolver | CPUSolver` (src/main.cpp:23-29) with
 *     Solver()                                  src/gpu/GPUSolver.cpp:7-51, src/cpu/CPUSolver.h:12-15
 *     void Step()                               src/gpu/GPUSolver.cpp:63-80, src/cpu/CPUSolver.h:16
 *     const std::vector<Vec>& GetParticlePositions()
 *                                               src/gpu/GPUSolver.cpp:276-295, src/cpu/CPUSolver.h:20-27
 * Knobs mirror src/shared/Parameters.h:6-84; particle arrays mirror the SSBO
 * contents built by GPUSolver::InitBuffers (src/gpu/GPUSolver.cpp:95-159).
 *
 * Units are the reference's grid units: cell size 1, node (i, j[, k]) at
 * x = (i, j[, k]), positions in [0, WIDTH] x [0, HEIGHT] (x [0, DEPTH]).
 *
 * Conventions
 *   - Every entry point returns an mpm_status; nothing throws across the ABI.
 *   - A solver owns its device memory (freed by mpm_destroy); the caller owns
 *     every host array it passes. Input arrays are copied before return.
 *   - Vectors are interleaved per particle (x, y[, z]) like std::vector<glm::vec2|3>;
 *     matrices are row-major dim x dim per particle.
 *   - A solver is bound to one device (the current one at mpm_create) and one
 *     CUDA stream; a handle must not be used from two threads at once.
 *   - mpm_step is asynchronous; every getter synchronises the solver's stream.
 *   - The product path has no CPU fallback: without a usable sm_100 device,
 *     mpm_create returns MPM_ERR_NO_DEVICE.
 */
#ifndef MPM_B200_MPM_H
#define MPM_B200_MPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(MPM_BUILDING_LIBRARY) && defined(__GNUC__)
#define MPM_API __attribute__((visibility("default")))
#else
#define MPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID_ARGUMENT = 1,
    MPM_ERR_CUDA = 2,
    MPM_ERR_OUT_OF_MEMORY = 3,
    MPM_ERR_NAN_STATE = 4,            /* a particle state became non-finite */
    MPM_ERR_FIXED_POINT_OVERFLOW = 5, /* a grid contribution exceeded the int64 fixed-point range */
    MPM_ERR_NO_DEVICE = 6,
    MPM_ERR_IO = 7,
    MPM_ERR_STATE_MISMATCH = 8,       /* checkpoint does not match this solver */
    MPM_ERR_TIMEOUT = 9,              /* a bounded device-side wait gave up */
    MPM_ERR_UNSUPPORTED = 10,
    MPM_ERR_CAPACITY = 11,            /* a buffer or fixed device capacity is too small */
    MPM_ERR_PARTICLE_OUT_OF_DOMAIN = 12 /* a particle's stencil reached outside the grid */
} mpm_status;

/* Device status word bits (mpm_get_status). Kernels set them with atomicOr
 * and never trap. */
enum {
    MPM_FLAG_NAN_STATE = 1u << 0,
    MPM_FLAG_FIXED_POINT_OVERFLOW = 1u << 1,
    MPM_FLAG_PARTICLE_OUT_OF_DOMAIN = 1u << 2, /* a stencil reached outside the grid */
    MPM_FLAG_SVD_FP64_FALLBACK = 1u << 3,      /* informational: the FP64 SVD branch ran */
    MPM_FLAG_TIMEOUT = 1u << 4                  /* a bounded device-side wait gave up: the TMA node-box
                                                   load of the fused transfer (MPM_BOX_LOAD=tma) did not
                                                   arrive; that step's results are invalid */
};

typedef enum mpm_formulation {
    MPM_FORMULATION_MLS = 0,           /* the reference GPU shaders (src/gpu/shaders/{2d,3d}) */
    MPM_FORMULATION_CLASSIC = 1,       /* the reference CPU path (src/cpu), 2D only */
    MPM_FORMULATION_MLS_QUADRATIC = 2  /* the MLS step on the quadratic B-spline stencil (3 nodes per
                                          axis, D^-1 = 4); no counterpart in the reference, which is cubic
                                          (src/gpu/shaders/2d/common.glsl:43-82) */
} mpm_formulation;

typedef enum mpm_boundary {
    MPM_BOUNDARY_FRICTION = 0, /* wall planes with separation + Coulomb friction (grid_update.glsl) */
    MPM_BOUNDARY_STICKY = 1    /* nodes within BORDER_MARGIN of a wall are held at rest */
} mpm_boundary;

typedef enum mpm_plasticity {
    MPM_PLASTIC_EXACT = 0, /* SVD return map (g2p.glsl:74-93) */
    MPM_PLASTIC_MLP = 1    /* learned surrogate with per-particle exact fallback */
} mpm_plasticity;

/* Simulation knobs: one field per src/shared/Parameters.h knob on the step
 * path, plus the solver's own choices. Fill with mpm_params_default(). */
typedef struct mpm_params {
    int32_t dim;           /* 2 or 3 (SIM_3D)                                   */
    int32_t width;         /* WIDTH: cells along x; nodes = WIDTH + 1           */
    int32_t height;        /* HEIGHT                                            */
    int32_t depth;         /* DEPTH (3D only)                                   */
    int32_t border_margin; /* BORDER_MARGIN (cells)                             */
    int32_t formulation;   /* mpm_formulation                                   */
    int32_t boundary;      /* mpm_boundary                                      */
    int32_t sort_period;   /* steps between particle re-binning; 0 = auto: each
                              period is 4..32 steps, the longest over which the
                              fastest particle (two periods earlier) moves at
                              most a quarter cell                              */
    float delta_time;      /* DELTA_TIME                                        */
    float gravity;         /* GRAVITY (along -y when negative), grid units/s^2  */
    float friction;        /* FRICTION (Coulomb coefficient at the walls)       */
    float theta_c;         /* THETA_C critical compression                      */
    float theta_s;         /* THETA_S critical stretch                          */
    float xi;              /* XI hardening coefficient                          */
    float nu;              /* NU Poisson ratio                                  */
    float youngs;          /* E Young's modulus                                 */
    float rho;             /* RHO: mass = volume * RHO / 100 when no mass given */
    int32_t fixed_point_log2_mass;     /* grid mass scale 2^k (0 = auto)        */
    int32_t fixed_point_log2_momentum; /* grid momentum scale 2^k (0 = auto)    */
    int32_t reserved[5];
} mpm_params;

/* Initial particles, as InitBuffers builds them (GPUSolver.cpp:95-159). */
typedef struct mpm_particles_init {
    int64_t count;
    const float* position; /* count * dim                                    */
    const float* velocity; /* count * dim (NULL = at rest)                   */
    const float* volume;   /* count                                          */
    const float* mass;     /* count, or NULL: volume * rho / 100 (Particles.cpp:18) */
} mpm_particles_init;

/* Host view of the particle state. Each pointer may be NULL (skipped). The
 * elastic gradient F_E and the plastic determinant J_p = det F_P are the
 * plastic state; the reference stores the full F_P but reads only its
 * determinant (p2g.glsl:46,52), so the solver stores J_p. */
typedef struct mpm_state_host {
    int64_t count;
    float* position;        /* count * dim                     */
    float* velocity;        /* count * dim                     */
    float* affine_b;        /* count * dim * dim (B_p)         */
    float* elastic_f;       /* count * dim * dim (F_E)         */
    float* plastic_det;     /* count (J_p)                     */
} mpm_state_host;

struct mpm_solver;
typedef struct mpm_solver mpm_solver;

/* Parameters.h defaults (WIDTH 200, HEIGHT 100, DEPTH 100, BORDER_MARGIN 2,
 * GRAVITY -9.81, FRICTION 0.3, DELTA_TIME 1e-3, THETA_C 2e-2, THETA_S 6e-3,
 * XI 10, NU 0.2, E 1.4e5, RHO 400), MLS formulation, friction walls.
 * Replaces the constants of src/shared/Parameters.h:29-84. */
MPM_API void mpm_params_default(mpm_params* out, int32_t dim);

/* Solver(): copies particles to the device and prepares the step.
 * Replaces GPUSolver::GPUSolver + InitBuffers (src/gpu/GPUSolver.cpp:7-51,83-202). */
MPM_API mpm_status mpm_create(const mpm_params* params, const mpm_particles_init* particles, mpm_solver** out);

/* ~Solver(): releases every device buffer (src/gpu/GPUSolver.cpp:53-60). */
MPM_API mpm_status mpm_destroy(mpm_solver* solver);

/* Step(): advances `nsteps` time steps of DELTA_TIME (P2G, grid update,
 * G2P with plasticity); asynchronous on the solver's stream.
 * Replaces GPUSolver::Step (src/gpu/GPUSolver.cpp:63-80) called nsteps times. */
MPM_API mpm_status mpm_step(mpm_solver* solver, int32_t nsteps);

/* GetParticlePositions(): copies `count * dim` floats into `out` (capacity
 * `cap_floats`), in the order the particles were given to mpm_create.
 * Replaces GPUSolver::GetParticlePositions (src/gpu/GPUSolver.cpp:276-295). */
MPM_API mpm_status mpm_get_positions(mpm_solver* solver, float* out, size_t cap_floats);

/* Number of particles and the dimension. */
MPM_API mpm_status mpm_get_info(const mpm_solver* solver, int64_t* count, int32_t* dim);

/* Particle re-binning sorts run so far and the current sort period (steps).
 * No counterpart in the reference (which does not sort its particles). */
MPM_API mpm_status mpm_get_sort_stats(const mpm_solver* solver, int64_t* sorts, int32_t* period);

/* Full particle state, host copies in creation order (the SSBO contents of
 * bindings 0-6, src/gpu/GPUSolver.cpp:166-172, minus mass/volume). */
MPM_API mpm_status mpm_get_state(mpm_solver* solver, mpm_state_host* state);

/* Overwrite the particle state (same layout as mpm_get_state; NULL fields keep
 * their values). */
MPM_API mpm_status mpm_set_state(mpm_solver* solver, const mpm_state_host* state);

/* One particle-to-grid pass on the current state without advancing time
 * (Grid::RasterizeToGrid, src/cpu/Grid.cpp:118-163; p2g.glsl): returns node
 * mass and momentum (MLS: momentum with the stress impulse folded in; CLASSIC:
 * momentum - DELTA_TIME * force) as doubles, `nodes` and `nodes * dim` values.
 * Optional raw int64 fixed-point sums in `raw` ((1 + dim) * nodes, component-major). */
MPM_API mpm_status mpm_rasterize(mpm_solver* solver, double* node_mass, double* node_momentum, int64_t* raw,
                         size_t nodes);

/* OR of every MPM_FLAG_* a kernel raised since creation (synchronises). */
MPM_API mpm_status mpm_get_status(mpm_solver* solver, uint32_t* flags);

/* The status word as an error code (synchronises): MPM_ERR_NAN_STATE,
 * MPM_ERR_FIXED_POINT_OVERFLOW, MPM_ERR_PARTICLE_OUT_OF_DOMAIN or
 * MPM_ERR_TIMEOUT for the first of those flags that is set, else MPM_OK (the informational FP64-SVD
 * flag is not an error); mpm_last_error names every flag set. This replaces
 * the reference's response to a non-finite stress, which prints and spins
 * forever (src/cpu/Particles.cpp:50-61): here the step completes, the flag
 * records what happened and the caller decides. */
MPM_API mpm_status mpm_check_status(mpm_solver* solver);

/* Launch work on this stream (a cudaStream_t) instead of the solver's own. */
MPM_API mpm_status mpm_set_stream(mpm_solver* solver, void* cuda_stream);

/* Checkpoint / resume: flat binary SoA with a header (dim, count, grid, params
 * hash, step). The reference has none; frames were PNGs (src/main.cpp:177-205). */
MPM_API mpm_status mpm_save_state(mpm_solver* solver, const char* path);
MPM_API mpm_status mpm_load_state(mpm_solver* solver, const char* path);

/* Steps taken since creation (or since the loaded checkpoint's step). */
MPM_API mpm_status mpm_get_step(const mpm_solver* solver, int64_t* step);

/* Human-readable description of the last error on this handle ("" if none).
 * Replaces CheckGLError's log line (src/gpu/GPUSolver.cpp:407-417). */
MPM_API const char* mpm_last_error(const mpm_solver* solver);

/* Text for a status code. */
MPM_API const char* mpm_status_string(mpm_status status);

/* Per-stage device timing: runs `nsteps` steps like mpm_step with a CUDA
 * event after every stage and adds each stage's device time in milliseconds to
 * stage_ms[s] for s < min(nstages, mpm_stage_count()). Synchronises. Stages:
 * "sort", "p2g", "grid_update", "g2p" (gather, APIC update and the in-band
 * return map) and "return_map" (the full return map of the particles whose
 * trial F left the elastic band, exact or learned). The reference has no
 * timers (src/main.cpp:11 includes <chrono> unused). */
MPM_API mpm_status mpm_step_profiled(mpm_solver* solver, int32_t nsteps, double* stage_ms, int32_t nstages);
MPM_API int32_t mpm_stage_count(const mpm_solver* solver);
MPM_API const char* mpm_stage_name(const mpm_solver* solver, int32_t stage);

/* Fixed-point scales in use (log2), for diagnostics. */
MPM_API mpm_status mpm_get_fixed_point(const mpm_solver* solver, int32_t* log2_mass, int32_t* log2_momentum);

/* ------------------------------------------------------------------------
 * Learned plasticity surrogate (no counterpart in the reference, which always
 * runs the SVD return map of g2p.glsl:74-104). A 10 -> 64 -> 64 -> 64 -> 10
 * GELU MLP, BF16 weights/activations, FP32 accumulation on the tensor cores,
 * FP32 master weights trained with AdamW on the GPU. Inputs: trial F_hat - I and
 * log J_p; outputs: F_E' - F_hat and log J_p' - log J_p (normalised per feature).
 * Used only for particles whose trial F is outside the elastic band; a
 * residual check with per-particle fallback to the exact SVD guards every
 * prediction. Pairs are rows of 20 floats: F_hat[9] J_p F_E'[9] J_p'. */
struct mpm_mlp;
typedef struct mpm_mlp mpm_mlp;

MPM_API int32_t mpm_mlp_param_count(void);
MPM_API mpm_status mpm_mlp_create(uint64_t seed, mpm_mlp** out);
MPM_API mpm_status mpm_mlp_destroy(mpm_mlp* mlp);
MPM_API const char* mpm_mlp_last_error(const mpm_mlp* mlp);
/* FP32 master parameters, layout W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64]
 * b3[64] W4[16][64] b4[16] (row-major W[out][in], padding zero). */
MPM_API mpm_status mpm_mlp_set_params(mpm_mlp* mlp, const float* params, size_t count);
MPM_API mpm_status mpm_mlp_get_params(mpm_mlp* mlp, float* out, size_t cap);
MPM_API mpm_status mpm_mlp_set_normalization(mpm_mlp* mlp, const float* in_mean, const float* in_std,
                                             const float* out_mean, const float* out_std);
/* Upload training pairs (n rows of 20 floats) to the device. */
MPM_API mpm_status mpm_mlp_load_pairs(mpm_mlp* mlp, const float* pairs, int64_t n);
/* `steps` AdamW steps on random batches of the loaded pairs (MSE on the
 * normalised outputs, cosine learning-rate decay); per-step loss into loss_out. */
MPM_API mpm_status mpm_mlp_train(mpm_mlp* mlp, int32_t steps, int32_t batch, float lr, float weight_decay,
                                 uint32_t seed, float* loss_out);
/* Mean-squared loss and its parameter gradient on the given pairs (no update). */
MPM_API mpm_status mpm_mlp_gradient(mpm_mlp* mlp, const float* pairs, int64_t n, float* grad_out, float* loss_out);
/* Denormalised outputs for rows whose first 10 floats are F_hat[9], J_p.
 * The network's device (current at mpm_mlp_create) must be current; any other
 * device returns MPM_ERR_INVALID_ARGUMENT before anything runs. */
MPM_API mpm_status mpm_mlp_predict(mpm_mlp* mlp, const float* inputs, int64_t n, int32_t stride, float* out);

/* mpm_mlp_predict without any device allocation (no counterpart in the
 * reference). Some callers cannot allocate device memory at the moment they
 * need an inference: a host process whose caching allocator has already
 * reserved the device's memory, or a loop with kernels in flight on other
 * streams, where cudaMalloc / cudaFree would fail or stall the whole device.
 * This entry point stages rows and results in a fixed scratch array that is
 * part of the library's device image (MPM_MLP_NOALLOC_MAX_ROWS rows, 5.2 MB
 * per device), so it allocates nothing. n above that limit returns
 * MPM_ERR_CAPACITY; split larger batches.
 * The first call on a device does a one-time set-up: it looks up the scratch
 * address, opts the kernel into its shared memory and creates a non-blocking
 * stream of its own for the copies and the launch (so calls neither wait for
 * nor hold up the legacy default stream). With CUDA's lazy module loading
 * (the default) that first call is also what loads this module onto the
 * device, scratch array included, which does take device memory: make one
 * warm-up call per device before the device's memory is reserved and before
 * any stream capture begins on it. A set-up that fails is not remembered; the
 * next call retries it. Nothing in the scratch has to start at zero: every
 * element a call reads was written earlier in the same call. Calls share the
 * scratch of their device, so two calls that overlap in time on the same
 * device (from two host threads) race: serialise them. Synchronous. The
 * network's device must be current (else MPM_ERR_INVALID_ARGUMENT). */
#define MPM_MLP_NOALLOC_MAX_ROWS 65536
MPM_API mpm_status mpm_mlp_predict_noalloc(mpm_mlp* mlp, const float* inputs, int64_t n, int32_t stride, float* out);

/* Return map of a solver: MPM_PLASTIC_EXACT, or MPM_PLASTIC_MLP with `mlp`
 * (3D MLS) and the residual-check tolerance (1e-3). The network must outlive
 * its use by the solver. */
MPM_API mpm_status mpm_set_plasticity(mpm_solver* solver, int32_t mode, mpm_mlp* mlp, float tolerance);
/* Particles the network handled (accepted) and those the residual check sent
 * to the exact SVD (rejected), since the mode was set. */
MPM_API mpm_status mpm_get_mlp_stats(mpm_solver* solver, uint64_t* accepted, uint64_t* rejected);
/* Log of exact return-map pairs for out-of-band particles (3D MLS); capacity 0
 * disables. Read copies up to cap_pairs logged pairs and restarts the log. */
MPM_API mpm_status mpm_pair_log_enable(mpm_solver* solver, int64_t capacity);
MPM_API mpm_status mpm_pair_log_read(mpm_solver* solver, float* out, int64_t cap_pairs, int64_t* n_pairs);

/* ---- Seeded shape sampling ---------------------------------------------
 * The reference fills each snow shape with Bridson's Poisson-disk sampling
 * seeded from std::random_device (PoissonDiskCircle / PoissonDiskSphere,
 * src/shared/Shapes.h:17-117,143-234): no two particles closer than min_dist,
 * not reproducible. mpm_sample_shapes does the same on the device in parallel
 * (grid-phase dart throwing, `rounds` candidates per background cell) and
 * deterministically for a given seed. Output: `count` positions (count * dim
 * floats, in background-cell order) and, if shape_of is not NULL, the first
 * shape containing each. With capacity too small it returns MPM_ERR_CAPACITY
 * and sets count to the number needed (call again with that capacity). */
typedef enum mpm_shape_kind {
    MPM_SHAPE_BALL = 0, /* SNOWBALL (Shapes.h:10-13): circle in 2D, sphere in 3D */
    MPM_SHAPE_BOX = 1   /* axis-aligned box (center +- half) */
} mpm_shape_kind;

typedef struct mpm_shape {
    int32_t kind;      /* mpm_shape_kind */
    float center[3];   /* grid units (z ignored in 2D) */
    float radius;      /* MPM_SHAPE_BALL */
    float half[3];     /* MPM_SHAPE_BOX half extents */
} mpm_shape;

MPM_API mpm_status mpm_sample_shapes(int32_t dim, const mpm_shape* shapes, int32_t nshapes, float min_dist,
                                     uint64_t seed, int32_t rounds, float* positions, int32_t* shape_of,
                                     int64_t capacity, int64_t* count);

/* ---- Headless frames ----------------------------------------------------
 * Visualize + saveFrame (src/main.cpp:51-205) without a window: particles as
 * white smoothed points of point_size pixels, the border at BORDER_MARGIN as
 * 2-pixel gray lines (2D rectangle; 3D wireframe box seen by the reference's
 * orbit camera: 45 deg perspective, angle / elevation / distance around the
 * grid centre), black background, nearest fragment wins. RGB8, rows top first
 * (what saveFrame writes to its PNG). */
typedef struct mpm_render_params {
    int32_t width, height; /* WINDOW_WIDTH, WINDOW_HEIGHT (1200 x 600) */
    float point_size;      /* PARTICLE_SIZE (1), pixels */
    float camera_angle;    /* 3D: degrees around y (0) */
    float camera_elevation;/* 3D: degrees (30) */
    float camera_distance; /* 3D: grid units from the grid centre (300) */
    float fov_degrees;     /* 3D: vertical field of view (45) */
    int32_t reserved[5];
} mpm_render_params;

MPM_API void mpm_render_params_default(mpm_render_params* params);
/* Writes width * height * 3 bytes into rgb (cap_bytes at least that). Synchronises. */
MPM_API mpm_status mpm_render(mpm_solver* solver, const mpm_render_params* params, uint8_t* rgb, size_t cap_bytes);

/* ---- Batched scenes (2D MLS) -------------------------------------------
 * Many independent scenes, each a full solver in the sense of mpm_create
 * (the reference constructs one Solver per process, src/main.cpp:164-174),
 * stepped together: every scene's grid lives in the shared memory of a
 * cluster of 1-8 CTAs, and one persistent launch per cluster size runs all
 * scenes from a work queue. Scenes: dim 2, MLS, at most 8 x 9,600 grid nodes
 * ((W+1)(H+1) <= ~76,000, e.g. 257 x 257 cells); larger or 3D scenes return
 * MPM_ERR_CAPACITY / MPM_ERR_UNSUPPORTED. */
struct mpm_batch;
typedef struct mpm_batch mpm_batch;

typedef struct mpm_batch_config {
    int32_t threads;           /* threads per CTA: 256, 512 or 1024 */
    int32_t particles_per_cta; /* spread a scene over more CTAs while it has more particles per CTA than this
                                  (0: only as many CTAs as its grid needs) */
    int32_t max_cluster;       /* largest cluster: 1, 2, 4 or 8 */
    int32_t sort_period;       /* steps between re-sorts of a multi-CTA scene's particles by row (0: 16) */
    int32_t reserved[4];
} mpm_batch_config;

/* Scene s uses params[s] (each validated as by mpm_create) and init[s]. */
MPM_API mpm_status mpm_batch_create(const mpm_params* params, const mpm_particles_init* init, int32_t nscenes,
                                    mpm_batch** batch);
MPM_API mpm_status mpm_batch_destroy(mpm_batch* batch);
MPM_API const char* mpm_batch_last_error(const mpm_batch* batch);
MPM_API mpm_status mpm_batch_info(const mpm_batch* batch, int32_t* nscenes, int64_t* total_particles);
/* Advance every scene by nsteps (asynchronous on the batch's stream; one CUDA
 * graph per nsteps value, replayed). */
MPM_API mpm_status mpm_batch_step(mpm_batch* batch, int32_t nsteps);
MPM_API mpm_status mpm_batch_set_stream(mpm_batch* batch, void* cuda_stream);
/* Per-scene state, host copies in the scene's creation order (as mpm_get_state). */
MPM_API mpm_status mpm_batch_get_state(mpm_batch* batch, int32_t scene, mpm_state_host* state);
MPM_API mpm_status mpm_batch_set_state(mpm_batch* batch, int32_t scene, const mpm_state_host* state);
MPM_API mpm_status mpm_batch_get_positions(mpm_batch* batch, int32_t scene, float* out, size_t cap_floats);
MPM_API mpm_status mpm_batch_get_status(mpm_batch* batch, int32_t scene, uint32_t* flags);
/* Device timestamps (ns) of the last mpm_batch_step call: for each scene, its
 * start and the end of each of its steps, [scene][nsteps + 1]; *nsteps gets the
 * call's step count. Synchronises. */
MPM_API mpm_status mpm_batch_step_times(mpm_batch* batch, uint64_t* out, size_t cap, int32_t* nsteps);
MPM_API mpm_status mpm_batch_get_config(const mpm_batch* batch, mpm_batch_config* config);
MPM_API mpm_status mpm_batch_set_config(mpm_batch* batch, const mpm_batch_config* config);
/* Autotuner: times trial_steps steps of the batch under each candidate
 * configuration (threads {256, 512, 1024} x particles per CTA {grid-limited,
 * 16k, 8k, 4k}), keeps the fastest, and restores
 * the particle state, so the batch continues as if untuned. *best_ms gets the
 * chosen configuration's time for the trial. Synchronises. */
MPM_API mpm_status mpm_batch_tune(mpm_batch* batch, int32_t trial_steps, mpm_batch_config* chosen, double* best_ms);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MPM_B200_MPM_H */
