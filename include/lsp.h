/*
 * lsp.h -- C ABI of liquidsimulation_b200, the B200 (sm_100a) implementation of
 * LiquidPhysics' per-step SPH / PCISPH particle pipeline.
 *
 * The reference exposes its solver as C++ classes (LiquidPhysics/include/SPHSolver.h,
 * PCISPHSolver.h, PhysicSolver.h) over a device seam (Parallelization/
 * ParallelComputationInterface.h). This header replaces both with a handle-based
 * C ABI: plain pointers and sizes, caller-owned host buffers, solver-owned device
 * memory. One handle = one scene = one CUDA stream; a handle is not re-entrant.
 *
 * Every call returns an int status: LSP_OK (0) or a negative LSP_ERR_* code.
 * lsp_last_error() gives a message for the last failing call on this thread.
 *
 * Particle order: every array passed in or out is in CALLER order (the order
 * particles were added). The device keeps particles sorted by grid cell; the
 * library maps back, so callers never see the device order (the reference's
 * OpenCL path instead hands back sorted data, SPHSolver.cpp:412-422).
 */
#ifndef LSP_H
#define LSP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSP_ABI_VERSION 1

/* ---- status codes ---- */
#define LSP_OK                   0
#define LSP_ERR_INVALID         -1   /* bad argument (null pointer, size, value out of range) */
#define LSP_ERR_CUDA            -2   /* a CUDA runtime call failed */
#define LSP_ERR_NO_DEVICE       -3   /* no CUDA device / wrong architecture */
#define LSP_ERR_DEVICE_STATUS   -4   /* the device raised an error flag (NaN, index out of range) */
#define LSP_ERR_NOT_CONVERGED   -5   /* PCISPH hit max iterations above eta (only if strict_convergence) */
#define LSP_ERR_TIMEOUT         -6   /* a bounded device-side wait gave up */
#define LSP_ERR_CAPACITY        -7   /* a size exceeds a fixed limit */
#define LSP_ERR_STATE           -8   /* call not valid in the current state */

/* ---- solver kinds (SPHSolver / PCISPHSolver) ---- */
#define LSP_SOLVER_SPH     0
#define LSP_SOLVER_PCISPH  1

/* ---- collider kinds (StaticCollisionObjectType, Collision/StaticCollisionObject.h:6-9) ---- */
#define LSP_OBSTACLE  0
#define LSP_BOUNDARY  1

/* ---- warm start of the PCISPH pressure ---- */
#define LSP_WARM_ZERO      0   /* reference: p = 0, F_p = 0 (PCISPHSolver.cpp:58-62) */
#define LSP_WARM_MLP       1   /* learned per-particle MLP guess, rejected if it raises the error */
/* Zero start (bit-identical to LSP_WARM_ZERO) until a step needs more than
 * warm_auto_iterations iterations or ends above eta; from the next step on, the learned
 * guess of LSP_WARM_MLP. The learned guess costs iterations while plain PCISPH converges
 * quickly and keeps a deep column converged once the plain loop starts running away, so
 * this mode uses it only after the plain loop has shown trouble. It stays on until the
 * parameters are set again (or a state file is loaded). No counterpart in the reference. */
#define LSP_WARM_AUTO      2

/* ---- PCISPH loop execution (results are identical) ---- */
#define LSP_LOOP_PERSISTENT 0   /* one cooperative kernel, convergence decided on the device */
#define LSP_LOOP_HOST       1   /* one launch per phase, convergence read back every iteration */

/*
 * Solver parameters. Field meaning and defaults follow SPHSolver::SPHSolver
 * (SPHSolver.cpp:11-23) and PCISPHSolver::PCISPHSolver (PCISPHSolver.cpp:6-7);
 * lsp_params_default() fills exactly those values.
 */
typedef struct lsp_params {
    float gravity[3];                  /* m_gravity, default (0,-9.81,0) */
    float particle_radius;             /* m_particleRadius, default 0.017 */
    float kernel_radius_factor;        /* m_kernelRadiusFactor, default 2.688; h = factor * radius */
    float rest_density;                /* m_restDensity, default 998.29 */
    float viscosity;                   /* m_viscosityCoefficient, default 3.5 */
    float stiffness;                   /* m_pressureStiffnessCoefficient, default 3 */
    float negative_pressure_factor;    /* m_negativePressureFactor, default 0 */
    float surface_tension;             /* m_surfaceTensionCoefficient, default 0.0728 */
    float surface_tension_threshold;   /* m_surfaceTensionThreshold, default 7.065 */
    float restitution;                 /* m_restitutionCoefficient, default 0.5 */
    float friction;                    /* m_frictionCoefficient, default 1 */
    float mass_override;               /* <= 0: mass derived as in SPHSolver::recalcParticleMass */
    int32_t solver;                    /* LSP_SOLVER_SPH or LSP_SOLVER_PCISPH */
    int32_t pci_max_iterations;        /* the reference's m_minIterations, which bounds the loop from above; default 4 */
    int32_t pci_min_iterations;        /* extension: no convergence exit before this many; default 1 (= reference) */
    float pci_eta;                     /* m_maxDensityErrorRatio, default 0.1 */
    int32_t warm_start;                /* LSP_WARM_*; default LSP_WARM_ZERO */
    int32_t strict_convergence;        /* 1: lsp_step returns LSP_ERR_NOT_CONVERGED at max iterations */
    int32_t keep_initial_velocity;     /* 1: skip the reference's first-step velocity wipe in PCISPH (Delta 5) */
    int32_t loop_mode;                 /* LSP_LOOP_*: how the PCISPH loop runs; default LSP_LOOP_PERSISTENT */
    int32_t warm_auto_iterations;      /* LSP_WARM_AUTO switch point (iterations); 0 = max(12, pci_max_iterations / 2) */
    int32_t reserved[5];
} lsp_params;

/* Per-step statistics, filled by lsp_step when non-NULL. */
typedef struct lsp_step_stats {
    int32_t iterations;               /* PCISPH predict-correct iterations this step (0 for SPH) */
    int32_t converged;                /* 1 if max density error ratio < eta at exit */
    double max_density_error_ratio;   /* max |rho* - rho0| / rho0 of the last iteration (compression only when negative_pressure_factor = 0) */
    int32_t max_neighbors;            /* largest neighbour count this step */
    int32_t escaped;                  /* particles outside the grid box (clamped into edge cells) */
    int32_t warm_start_used;          /* 1 if the warm-start guess was kept */
    int32_t warm_start_tried;         /* 1 if the step started from the learned guess (kept or not) */
} lsp_step_stats;

/* Fields for lsp_read_field. Vector fields are float[3*n], scalars float[n]. */
#define LSP_FIELD_POSITION            0
#define LSP_FIELD_VELOCITY            1
#define LSP_FIELD_HALF_VELOCITY       2
#define LSP_FIELD_DENSITY             3
#define LSP_FIELD_PRESSURE            4
#define LSP_FIELD_FIRST_STEP          5   /* 1.0 / 0.0 */
#define LSP_FIELD_PRED_DENSITY        6
#define LSP_FIELD_DENSITY_ERROR       7
#define LSP_FIELD_PRED_POSITION       8
#define LSP_FIELD_PRED_HALF_VELOCITY  9
#define LSP_FIELD_PRED_PRESSURE_FORCE 10
#define LSP_FIELD_OLD_HALF_VELOCITY   11
#define LSP_FIELD_NEIGHBOR_COUNT      12  /* float[n] holding integer counts */
#define LSP_FIELD_SPEED_SQUARED       13  /* |v|^2, the colour source of SPHParticleDrawable.cpp:10-27 */

typedef struct lsp_solver lsp_solver;

/* ---- lifecycle ---- */
void lsp_params_default(lsp_params* p);
const char* lsp_last_error(void);
int lsp_device_info(int* sm_count, int* cc_major, int* cc_minor);
/* Check of the bounded wait in the persistent loops' grid barrier (no counterpart in the
 * reference): on `device` (< 0: current), one barrier round with `blocks` blocks (1..8)
 * waiting for `parties` arrivals (1..16) and a short spin limit. completed = blocks that
 * passed; error_flags gets bit 4 (timeout) when a block gave up waiting. With fewer blocks
 * than parties the round cannot complete: the waits end with the timeout bit instead of a
 * hang, and the device stays usable. */
int lsp_barrier_probe(int device, int blocks, int parties, int32_t* completed, uint32_t* error_flags);

/* SPHSolver::SPHSolver / PCISPHSolver::PCISPHSolver (SPHSolver.cpp:9-86). device < 0 = current. */
int lsp_create(const lsp_params* params, int device, lsp_solver** out);
int lsp_destroy(lsp_solver* s);

/* Setters/getters of SPHSolver.h:79-109 and PCISPHSolver.h:16-20, all at once. */
int lsp_set_params(lsp_solver* s, const lsp_params* params);
int lsp_get_params(const lsp_solver* s, lsp_params* out);
int lsp_particle_mass(const lsp_solver* s, float* mass);          /* getParticleMass */
int lsp_kernel_radius(const lsp_solver* s, float* h);             /* getKernelRadius */
int lsp_particle_count(const lsp_solver* s, int64_t* n);          /* getParticleCount */
int lsp_pcisph_delta(const lsp_solver* s, float dt, float* delta);/* PCISPHSolver::calcDelta (PCISPHSolver.cpp:286-328) */
/* The 5 x 1001 lookup tables (poly6 W, poly6 dW, poly6 d2W, spiky dW, viscosity d2W),
 * SPHKernel::recalcCachedWeights (SPHKernel.cpp:113-132). out: float[5*1001]. */
int lsp_kernel_tables(const lsp_solver* s, float* out, int capacity);

/* ---- scene ---- */
/* SPHSolver::addParticle (SPHSolver.cpp:129-135), n at a time. vel may be NULL (zero).
 * New particles start with half-velocity 0 and the first-step flag set (SPHParticle.cpp:4-14). */
int lsp_add_particles(lsp_solver* s, const float* xyz, const float* vel, int64_t n);
int lsp_remove_particles(lsp_solver* s);                           /* SPHSolver::removeParticles */
/* SPHSolver::addStaticCollisionObject with StaticCollisionBox / StaticCollisionSphere.
 * Colliders act in insertion order, as the CPU solver does (SPHSolver.cpp:376-379). */
int lsp_add_box(lsp_solver* s, const float center[3], const float half_extent[3], int kind);
int lsp_add_sphere(lsp_solver* s, const float center[3], float radius, int kind);
int lsp_remove_colliders(lsp_solver* s);                           /* removeStaticCollisionObjects */
/* Moves/resizes collider `index` (insertion order); setHasCollisionObjectDataChanged. */
int lsp_update_box(lsp_solver* s, int index, const float center[3], const float half_extent[3]);
int lsp_update_sphere(lsp_solver* s, int index, const float center[3], float radius);
/* Optional grid box. Without it the grid covers the union of boundary boxes, or the
 * particle bounds at the first step plus a margin. Particles outside are clamped. */
int lsp_set_domain(lsp_solver* s, const float lo[3], const float hi[3]);

/* ---- stepping ---- */
/* PhysicSolver::update(dt) (PhysicSolver.cpp:12-21): one full step. */
int lsp_step(lsp_solver* s, float dt, lsp_step_stats* stats);
/* n steps in one call, stats of the last. Each step still reads its status word back before
 * the next is queued (a step whose neighbour lists overflow is redone with larger lists), so
 * this saves the per-call overhead, not the per-step synchronisation. */
int lsp_step_many(lsp_solver* s, float dt, int steps, lsp_step_stats* stats);
int lsp_synchronize(lsp_solver* s);

/* ---- read-back / state (caller order) ---- */
/* Replaces SPHSolver::onEndUpdate's sorted read-back (SPHSolver.cpp:400-427). */
int lsp_read_particles(lsp_solver* s, float* xyz, float* vel, int64_t n);
int lsp_read_field(lsp_solver* s, int field, float* out, int64_t n);
/* Full persistent state: x, v, v_half, v_half_old (float[3n] each) and first-step flags. */
int lsp_read_state(lsp_solver* s, float* x, float* v, float* half, float* old_half, int32_t* first, int64_t n);
int lsp_write_state(lsp_solver* s, const float* x, const float* v, const float* half, const float* old_half, const int32_t* first, int64_t n);

/* Start-of-step neighbour lists of the last step, caller order, in the reference's
 * order (SPHSpatialGrid::findNeighborParticles, SPHSpatialGrid.cpp:39-76). Like the grid
 * read-back and lsp_mlp_train, refused with LSP_ERR_STATE until a step has run on the current
 * particles (after lsp_add_particles or lsp_remove_particles, until the next step).
 * offsets: int64[n+1]; index: int32[offsets[n]] (pass index=NULL to get offsets only). */
int lsp_read_neighbors(lsp_solver* s, int64_t* offsets, int32_t* index, int64_t n, int64_t capacity);

/* Grid build of the last step, device order, for parity tests:
 * cell key and caller id per sorted slot, and the dense cell table (cells+1 entries). */
int lsp_grid_info(lsp_solver* s, int32_t dims[3], int32_t origin[3], int64_t* cells);
int lsp_read_grid(lsp_solver* s, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start, int64_t cells_plus_one);

/* ---- learned warm start (warm_start = LSP_WARM_MLP) ----
 * A per-particle MLP (8 features -> 32 -> 32 -> 1, SiLU, BF16 tensor-core MMA with FP32
 * accumulation) guesses each particle's PCISPH pressure; the loop then iterates to the
 * same eta. If the guess raises the maximum density error of the first correction, the
 * step restarts from zero pressure and ends bit-identical to the plain solver.
 * No counterpart in the reference. Parameters: FP32 vector of LSP_MLP_PARAMS floats,
 * W1[8][32], b1[32], W2[32][32], b2[32], W3[32], b3. */
#define LSP_MLP_PARAMS 1377
#define LSP_MLP_FEATURES 8
int lsp_mlp_reset(lsp_solver* s, uint64_t seed);                   /* random init, Adam state cleared */
int lsp_mlp_set_weights(lsp_solver* s, const float* w, int n);
int lsp_mlp_get_weights(lsp_solver* s, float* w, int n);
/* Records the 8 features of every particle at iteration 0 of each PCISPH step. */
int lsp_mlp_record(lsp_solver* s, int enable);
/* Sets params.warm_start (LSP_WARM_ZERO / LSP_WARM_MLP / LSP_WARM_AUTO) alone, without the
 * table rebuild of lsp_set_params, for callers that switch the warm start between steps
 * (online retraining with the zero start as fallback). LSP_WARM_AUTO restarts from the zero
 * start. No counterpart in the reference. */
int lsp_set_warm_start(lsp_solver* s, int mode);
/* Training loss 1/(2n) sum w r^2, r = guess - target, w = over_weight when r > 0
 * (default 1, plain MSE). PCISPH with a zero negative-pressure factor only adds pressure
 * within a step, so over-estimates cost iterations that under-estimates do not. */
int lsp_mlp_set_loss_asymmetry(lsp_solver* s, float over_weight);
/* Adam steps on the last recorded step: features -> final pressure (normalised).
 * Each iteration draws `batch` random particles. loss (may be NULL): mean 0.5 (y - t)^2. */
int lsp_mlp_train(lsp_solver* s, int iterations, int batch, float learning_rate, uint64_t seed, float* loss);
/* Network output for n feature rows (host arrays float[8n] -> float[n]). */
int lsp_mlp_forward(lsp_solver* s, const float* features, int64_t n, float* out);
/* Gradient of 1/(2n) sum (y - t)^2 at the current weights (host arrays); no update. */
int lsp_mlp_gradient(lsp_solver* s, const float* features, const float* targets, int64_t n, float* grad, float* loss);
/* Features of the last recorded step, caller order, float[8n]. */
int lsp_read_features(lsp_solver* s, float* out, int64_t n);

/* Allocation-free variant of lsp_mlp_gradient for callers that may not allocate device
 * memory while they run: every pointer is caller-owned DEVICE memory (features float[8n],
 * targets float[n], grad float[LSP_MLP_PARAMS], loss float[1], the mean 0.5 r^2), and the
 * per-warp partial sums use a fixed scratch array inside the library (2.7 MiB on each
 * device that loads it, kept until the process exits). n <= 16777216 (LSP_ERR_CAPACITY
 * beyond). The buffers must belong to the solver's GPU (or be managed memory).
 * Work is queued on the solver's stream and is not ordered after work on any other stream:
 * the inputs must be complete before the call (synchronise the stream that wrote them), and
 * the outputs may be read only after lsp_synchronize. The scratch address is looked up, and
 * the module holding it loaded, when the solver is created (lsp_create), so a call itself
 * allocates nothing. Calls that overlap on the GPU share the scratch and race.
 * No counterpart in the reference. */
int lsp_mlp_gradient_static(lsp_solver* s, const float* features, const float* targets, int64_t n,
                            float* grad, float* loss);

/* ---- measurement ---- */
/* CUDA events on the solver's stream: mark records event `slot` (0..15); elapsed waits for
 * slot_b and returns the device time between the two marks in milliseconds. */
int lsp_timer_mark(lsp_solver* s, int slot);
int lsp_timer_elapsed(lsp_solver* s, int slot_a, int slot_b, float* ms);
/* Per-kernel-class device time: with profiling on, every launch is bracketed by events on
 * the solver's stream. read: ms[k] and launches[k] for k < LSP_PROF_COUNT. */
#define LSP_PROF_GRID_SORT     0   /* cell keys and histogram (batches: the whole grid build) */
#define LSP_PROF_NEIGHBORS     1
#define LSP_PROF_DENSITY       2
#define LSP_PROF_NONPRESSURE   3
#define LSP_PROF_SPH_PRESSURE  4
#define LSP_PROF_PCI_PREDICT   5
#define LSP_PROF_PCI_DENSITY   6
#define LSP_PROF_PCI_FORCE     7
#define LSP_PROF_INTEGRATE     8
#define LSP_PROF_PCI_LOOP      9   /* the persistent predict-correct kernel */
#define LSP_PROF_WARM_START    10
#define LSP_PROF_GRID_SCAN     11  /* scan of the histogram into the dense cell table */
#define LSP_PROF_GRID_SCATTER  12  /* particle -> cell start + slot */
#define LSP_PROF_GRID_GATHER   13  /* rank inside each cell and gather of the persistent state */
#define LSP_PROF_COUNT         14
int lsp_profile(lsp_solver* s, int enable);
int lsp_profile_read(lsp_solver* s, double* ms, int64_t* launches, int capacity);
/* Kernels this solver has launched since creation. */
int lsp_launch_count(const lsp_solver* s, int64_t* launches);
/* ---- state files: save / resume, golden files ----
 * One binary file per scene: parameters, colliders, grid box, the caller-order state
 * (x, v, v_half, v_half_old, first-step flags), the warm-start pressure history when it
 * exists and the MLP weights (layout at the top of csrc/state_io.cpp). Loading replaces
 * the handle's parameters, particles, colliders and grid box; a resumed run continues
 * bit-identically to the run that was saved (the optimiser's Adam moments are not saved).
 * `seed` is the caller's label of the scene, stored as given. No counterpart in the
 * reference (it has no persistence). */
int lsp_save_state(lsp_solver* s, const char* path, uint64_t seed);
int lsp_load_state(lsp_solver* s, const char* path);
/* Reads only the header (no device needed): any output may be NULL. */
int lsp_state_file_info(const char* path, lsp_params* params, int64_t* n, int32_t* colliders, uint64_t* seed);

/* Page-locked host memory for asynchronous copies (cudaMallocHost / cudaFreeHost). */
int lsp_host_alloc(size_t bytes, void** out);
int lsp_host_free(void* p);

/*
 * ---- batches of independent scenes ----
 *
 * A batch steps many scenes together on one device: what the reference does with one
 * SPHSolver / PCISPHSolver object per scene, each updated in turn by its
 * PhysicSolver::update (PhysicSolver.cpp:12-21). Each scene keeps its own parameters,
 * particles (caller order within the scene), colliders and grid, and its results are
 * bit-identical to a single-scene handle given the same inputs. All scenes of a batch use
 * the same solver kind and step with the same dt. The whole step of all scenes runs as one
 * CUDA graph with one persistent kernel for the PCISPH loops of all scenes, each scene
 * converging on its own. Scenes and colliders are added before the first step; colliders
 * can be moved at any time. No counterpart in the reference (it has no batching).
 */
typedef struct lsp_batch lsp_batch;

typedef struct lsp_batch_tuning {
    int32_t threads;        /* chosen particles per block of the per-particle kernels */
    int32_t loop_blocks;    /* chosen blocks of the persistent PCISPH kernel */
    int32_t candidates;     /* configurations timed (<= 16) */
    int32_t reserved;
    int32_t cand_threads[16];
    int32_t cand_loop_blocks[16];
    float cand_ms[16];      /* best device time of one step, per configuration */
} lsp_batch_tuning;

/* device < 0: the current device. */
int lsp_batch_create(int device, lsp_batch** out);
int lsp_batch_destroy(lsp_batch* b);
/* Adds a scene: n >= 1 particles in caller order (vel may be NULL = zero). domain_lo/hi
 * (both or neither) fix the grid box like lsp_set_domain; without them it is the union of
 * the scene's boundary colliders at its first step, else the particle bounds plus a margin.
 * Writes the scene index (0, 1, ...). */
int lsp_batch_add_scene(lsp_batch* b, const lsp_params* params, const float* xyz, const float* vel, int64_t n,
                        const float* domain_lo, const float* domain_hi, int32_t* scene);
int lsp_batch_add_box(lsp_batch* b, int32_t scene, const float center[3], const float half_extent[3], int kind);
int lsp_batch_add_sphere(lsp_batch* b, int32_t scene, const float center[3], float radius, int kind);
/* Moves collider `index` of a scene (its kind and shape stay). */
int lsp_batch_update_box(lsp_batch* b, int32_t scene, int32_t index, const float center[3],
                         const float half_extent[3]);
int lsp_batch_update_sphere(lsp_batch* b, int32_t scene, int32_t index, const float center[3], float radius);
int lsp_batch_info(const lsp_batch* b, int32_t* scenes, int64_t* particles);
int lsp_batch_scene_count(const lsp_batch* b, int32_t scene, int64_t* n);
int lsp_batch_particle_mass(const lsp_batch* b, int32_t scene, float* mass);
/* One step of every scene. stats: NULL or an array of one lsp_step_stats per scene. */
int lsp_batch_step(lsp_batch* b, float dt, lsp_step_stats* stats);
/* Per-scene read-back in the scene's caller order (n = the scene's particle count). */
int lsp_batch_read_particles(lsp_batch* b, int32_t scene, float* xyz, float* vel, int64_t n);
int lsp_batch_read_field(lsp_batch* b, int32_t scene, int field, float* out, int64_t n);
int lsp_batch_read_neighbors(lsp_batch* b, int32_t scene, int64_t* offsets, int32_t* index, int64_t n,
                             int64_t capacity);
int lsp_batch_grid_info(const lsp_batch* b, int32_t scene, int32_t dims[3], int32_t origin[3], int64_t* cells);
int lsp_batch_read_grid(lsp_batch* b, int32_t scene, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start,
                        int64_t cells_plus_one);
/* The whole batch's state, scenes concatenated in index order, each in caller order
 * (n = total particles; same arrays as lsp_read_state / lsp_write_state). */
int lsp_batch_read_state(lsp_batch* b, float* x, float* v, float* v_half, float* v_half_old, int32_t* first_step,
                         int64_t n);
int lsp_batch_write_state(lsp_batch* b, const float* x, const float* v, const float* v_half,
                          const float* v_half_old, const int32_t* first_step, int64_t n);
/* Launch shape: use_graph (0/1), threads (128, 256, 512 or 1024 particles per block), loop_blocks
 * (blocks of the persistent kernel, 0 = all that fit). get also reports whether the step
 * currently runs as a captured graph. */
int lsp_batch_set_launch(lsp_batch* b, int use_graph, int threads, int loop_blocks);
int lsp_batch_get_launch(const lsp_batch* b, int* use_graph, int* threads, int* loop_blocks, int* graph_active);
/* Autotuner: runs the next step under each candidate launch shape (particles per block x
 * persistent-kernel blocks), re-running that same step from the same state `repeats` times
 * per candidate, keeps the fastest shape, and leaves the batch advanced by exactly that one
 * step (results do not depend on the shape). result and stats may be NULL. */
int lsp_batch_autotune(lsp_batch* b, float dt, int repeats, lsp_batch_tuning* result, lsp_step_stats* stats);
/* Learned warm start for the scenes of a PCISPH batch (LSP_WARM_ZERO, LSP_WARM_MLP or
 * LSP_WARM_AUTO; AUTO switches each scene on by itself, at that scene's
 * warm_auto_iterations): one network for the batch, features normalised per scene, the
 * guess checked and rejected per scene exactly as lsp_step does. The lsp_mlp_* counterparts below act on the batch's
 * network; train uses the features and final pressures of the last recorded step of all
 * scenes. No counterpart in the reference. */
int lsp_batch_set_warm_start(lsp_batch* b, int mode);
int lsp_batch_mlp_reset(lsp_batch* b, uint64_t seed);
int lsp_batch_mlp_set_weights(lsp_batch* b, const float* w, int n);
int lsp_batch_mlp_get_weights(lsp_batch* b, float* w, int n);
int lsp_batch_mlp_record(lsp_batch* b, int on);
int lsp_batch_mlp_set_loss_asymmetry(lsp_batch* b, float over_weight);
int lsp_batch_mlp_train(lsp_batch* b, int iterations, int batch, float lr, uint64_t seed, float* loss);
int lsp_batch_read_features(lsp_batch* b, int32_t scene, float* out, int64_t n);
int lsp_batch_timer_mark(lsp_batch* b, int slot);
int lsp_batch_timer_elapsed(lsp_batch* b, int slot_a, int slot_b, float* ms);
int lsp_batch_launch_count(const lsp_batch* b, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* LSP_H */
