/*
 * pawan_gpu.h - C ABI of the B200 vortex-particle backend.
 *
 * This is the boundary a PAWAN build binds to replace the CPU solve of its
 * __interaction / __parallel backend and the stage loop of its __rk3 / __rk4
 * integrators.  Plain C types only (no CUDA or torch types); every entry point
 * returns PGPU_OK (0) or a negative PGPU_E* code, and pgpu_last_error() gives
 * the message of the last failure on a context.
 *
 * Units and layouts follow PAWAN's __wake (src/wake/wake.h:49-54): positions
 * and strengths are row-major (n, 3) FP64 host arrays, radii and volumes (n).
 *
 * A context owns all device memory and one CUDA stream; it is used from one
 * host thread at a time (PAWAN calls its solver from one thread).
 * pgpu_create (and pgpu_mlp_create) make the new object's device current, as
 * cudaSetDevice does; every later call that works on the device makes that
 * object's device current for its duration and then restores the caller's, so
 * contexts on several GPUs can be driven from one thread.  Wakes are
 * grouped into systems: the wakes of one system all interact with one another,
 * exactly as the wakes held by one PAWAN __interaction do
 * (src/interaction/interaction.cpp:196-210); different systems are independent
 * and are advanced together in one persistent launch per stage.
 */
#ifndef PAWAN_GPU_H_
#define PAWAN_GPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGPU_OK 0
#define PGPU_EINVAL (-1)   /* bad argument or call order */
#define PGPU_ENOMEM (-2)   /* device or host allocation failed */
#define PGPU_ECUDA (-3)    /* a CUDA call failed */
#define PGPU_ETIMEOUT (-4) /* a bounded device wait expired */
#define PGPU_ENUMERIC (-5) /* a non-finite value was produced */

#define PGPU_FP32C 0 /* FP32 pair terms, compensated per-target sums, FP64 state */
#define PGPU_FP64 1  /* FP64 throughout */

/* Regularisation kernel.  PAWAN picks one at compile time with the
 * HIGHORDER / GAUSSIAN macros of src/interaction/interaction_utils.h:13-20;
 * here it is a per-context setting. */
#define PGPU_KERNEL_GAUSSIAN 0  /* src/interaction/gaussian.h (PAWAN's default) */
#define PGPU_KERNEL_HIGHORDER 1 /* src/interaction/highorder.h, high-order algebraic */

#define PGPU_EULER 0
#define PGPU_RK3 1
#define PGPU_RK4 2

typedef struct pgpu_ctx pgpu_ctx;

typedef struct pgpu_config {
  int precision;   /* PGPU_FP32C or PGPU_FP64 */
  int device;      /* CUDA device ordinal */
  double nu;       /* kinematic viscosity (PAWAN's protected __interaction::_nu, interaction.h:25) */
  double vinf[3];  /* uniform inflow added after each step, x += vinf dt
                      (__wake::updateVinfEffect, wake.cpp:564-577, called from integration.cpp:172) */
  int block;       /* pair-kernel threads per CTA; 0 = default (Gaussian: 128; high-order: 256) until pgpu_autotune */
  int tpt;         /* pair-kernel targets per thread; 0 = default (Gaussian FP32C: 2, FP64: 1; high-order: 1) */
  int chunks;      /* source chunks per system (1..16); 0 = automatic */
  int use_graphs;  /* capture each time step in a CUDA graph (default 1) */
  int kernel;      /* PGPU_KERNEL_GAUSSIAN (default) or PGPU_KERNEL_HIGHORDER; rates,
                      diagnostics (enstrophy and enstrophyF are non-zero only for the
                      high-order kernel, as in PAWAN), probes and the vorticity field all
                      use it.  The far-field surrogate supports the Gaussian kernel only. */
  int split_positions; /* FP32C with the Gaussian kernel: keep each position as its FP32 value plus the
                          FP32 residual of the FP64 state, and form the differences of nearby pairs
                          (tiles with a pair at rho^2 < 50 sigma^2) from both, so that dense filaments,
                          whose pair distances are a few hundred FP32 ulps of the coordinates, keep
                          FP64-quality differences.  Costs 16 B per particle and a few operations per
                          near pair; not supported with target ranges.  Default 0. */
} pgpu_config;

/* Fills cfg with defaults (FP32C, device 0, nu = 1.56e-5 as __interaction(),
 * interaction.cpp:15, no inflow, tuned tiles, graphs on). */
void pgpu_config_default(pgpu_config *cfg);

/* Replaces: constructing a backend, `new pawan::__parallel(W)` (src/pawan.cpp:48,
 * src/interaction/parallel.cpp:11-12).  On failure *ctx is NULL and
 * pgpu_last_error(NULL) gives the reason (per calling thread). */
int pgpu_create(pgpu_ctx **ctx, const pgpu_config *cfg);
/* Replaces: the backend destructor (interaction.cpp:37-42). */
int pgpu_destroy(pgpu_ctx *ctx);

/* Replaces: __interaction::addWake (interaction.h:198, interaction.cpp:44-52).
 * Reserves `capacity` particle slots for a wake of system `system`.  Wakes must
 * be added before the first particle upload.  Within a system every wake but
 * the last must be full (n == capacity) when the system is solved; the last
 * wake may grow up to its capacity (pgpu_append_particles). */
int pgpu_add_wake(pgpu_ctx *ctx, int32_t system, int64_t capacity, int32_t *wake_id);

/* Replaces: filling __wake::_position/_vorticity/_radius/_volume
 * (wake.h:49-54) - uploads n particles (host buffers) into a wake. */
int pgpu_set_particles(pgpu_ctx *ctx, int32_t wake, int64_t n, const double *pos, const double *alpha,
                       const double *sigma, const double *vol);
/* Replaces: __wake::addParticles (wake.cpp:179-531 in the coupled run) for a
 * synthetic shedder - appends m particles to the last wake of a system. */
int pgpu_append_particles(pgpu_ctx *ctx, int32_t wake, int64_t m, const double *pos, const double *alpha,
                          const double *sigma, const double *vol);
int pgpu_get_num_particles(pgpu_ctx *ctx, int32_t wake, int64_t *n);

/* Replaces: __interaction::getStates (interaction.cpp:357-365) restricted to
 * one wake: downloads positions and strengths (n, 3) each. */
int pgpu_get_state(pgpu_ctx *ctx, int32_t wake, double *pos, double *alpha);

/* Replaces: __interaction::setStates / getStates on PAWAN's flat state vector
 * (interaction.cpp:337-365; per wake [x (maxN x 3) ; alpha (maxN x 3)] at an
 * offset of sum 6 maxN, wake.cpp:856-893).  `maxn` lists each wake's PAWAN
 * capacity (__wake::_maxnumParticles), in wake-id order. */
int pgpu_set_states_flat(pgpu_ctx *ctx, const double *state, const int64_t *maxn, int32_t nwakes);
int pgpu_get_states_flat(pgpu_ctx *ctx, double *state, const int64_t *maxn, int32_t nwakes);
/* Replaces: __interaction::getRates (interaction.cpp:347-355): the flat rate
 * vector [velocity ; dalpha/dt] of the last evaluation. */
int pgpu_get_rates_flat(pgpu_ctx *ctx, double *rate, const int64_t *maxn, int32_t nwakes);

/* Replaces: __interaction::solve (interaction.cpp:54-57) with the OpenMP pair
 * loops of __parallel::interact (parallel.cpp:14-86): one rate evaluation of
 * every system at its current state. */
int pgpu_solve(pgpu_ctx *ctx);
/* Replaces: __interaction::getRates restricted to one wake: velocity and
 * dalpha/dt of the last evaluation, (n, 3) each. */
int pgpu_get_rates(pgpu_ctx *ctx, int32_t wake, double *vel, double *dalpha);

/* Replaces: the time loop body of __integration::integrate
 * (integration.cpp:112-116) with __rk4::step (rk4.cpp:12-77), __rk3::step
 * (rk3.cpp:12-65) or the Euler step (integration.cpp:198-208): advances every
 * system nsteps steps on the device; the config's vinf is applied after each
 * step.  The state stays on the device. */
int pgpu_step(pgpu_ctx *ctx, int scheme, double dt, int32_t nsteps);

/* ---------------------------------------------------------------------------
 * One system over several GPUs (no PAWAN counterpart: PAWAN runs on one host).
 * Each GPU's context holds the whole system and owns a contiguous range of
 * its targets; all particles stay sources.  A step then runs stage by stage:
 * pgpu_stage evaluates the owned targets' rates from the current source
 * records of all particles and updates the owned particles (state and
 * records); before the next stage the caller copies the other GPUs' owned
 * records into this context's record arrays (an all-gather), ordered on the
 * context's stream (pgpu_get_stream).
 *
 * pgpu_set_target_range: targets [first, first + count) of the system (in
 * the order of its wakes' particles); count < 0 restores all targets.  While
 * any system has a range, pgpu_step and pgpu_diagnose refuse (the state of
 * the other targets is not advanced here; pgpu_diagnose_partial gives this
 * context's share of the diagnostics).  With the surrogate enabled, every
 * context builds the octree of the whole system from its (exchanged) records,
 * evaluates only the tree's work items that hold owned targets, and draws its
 * sampled check targets from the owned ones; its fallback is the direct sum
 * over the owned targets.
 * pgpu_stage: stage 0..3 (RK4), 0..2 (RK3) or 0 (Euler) of one step of every
 * system; the last stage finishes the step (and applies vinf).
 * pgpu_records: device pointers to the system's source records, one per
 * particle in system order: FP32C float4 (x, y, z, sigma^2/2) and
 * (alpha_x, alpha_y, alpha_z, vol); FP64 mode double4. */
int pgpu_set_target_range(pgpu_ctx *ctx, int32_t system, int64_t first, int64_t count);
int pgpu_stage(pgpu_ctx *ctx, int scheme, int stage, double dt);
int pgpu_records(pgpu_ctx *ctx, int32_t system, void **P, void **Q);

/* Replaces: __interaction::influence (interaction.cpp:212-260, with
 * INFLUENCE / SELFINFLUENCE, interaction_utils.h:626-703), which
 * __interaction::resolve (interaction.cpp:59-62) calls: the vorticity field
 * k_t = sum_s zeta(rho_ts, sigma_ts) alpha_s at every particle, from every
 * particle of its system (the particle itself included).  Always in FP64,
 * from the FP64 state, in both precision modes: PAWAN's strength solve
 * (__resolve::rebuild, resolve.cpp:12-63) LU-solves a matrix of these fields
 * and needs their digits.  pgpu_get_vorticity_field then copies one wake's
 * rows (n x 3, row-major) to the host (PAWAN: the wake's _vorticityfield). */
int pgpu_influence(pgpu_ctx *ctx);
int pgpu_get_vorticity_field(pgpu_ctx *ctx, int32_t wake, double *field);

/* Replaces: __wake::merge (wake.cpp:112-159), the O(N^2) half of
 * __wake::relax (wake.cpp:161-165, called per wake by __interaction::relax,
 * interaction.cpp:367-371, in the coupled time loop, integration.cpp:87), on
 * the device state of one wake.  PAWAN's loop visits the particles i whose age
 * passes `stepnum - _active[i] > 45` up to the first that fails; the caller
 * passes the length of that prefix as n_elig (it holds the ages).  A particle
 * j > i within 0.125 (r_i + r_j) of i, with non-zero, non-aligned strength
 * (1 - cos >= 1e-4), is merged into i: x_i moves to the strength-weighted
 * mean, alpha_i += alpha_j, alpha_j and vol_j become zero.  The candidate
 * search runs on the device; the sequential loop, whose every decision
 * depends on the earlier merges, is replayed on the host over the candidates
 * in PAWAN's order and arithmetic, and the changed rows are written back.
 * *nmerged (may be NULL) receives the number of merges.  Wakes of fewer than
 * 2^31 particles. */
int pgpu_merge(pgpu_ctx *ctx, int32_t wake, int64_t n_elig, int64_t *nmerged);

/* Replaces: reading __wake::_position, _vorticity, _radius, _volume
 * (wake.h:49-54) - downloads one wake's particles; any pointer may be NULL. */
int pgpu_get_particles(pgpu_ctx *ctx, int32_t wake, double *pos, double *alpha, double *sigma, double *vol);

/* Replaces: __interaction::diagnose (interaction.cpp:64-194) for one system.
 * out[15] = total vorticity(3), linear impulse(3), angular impulse(3),
 * helicity, enstrophy, enstrophyF, kinetic energy, kinetic energyF, Zc - the
 * record of writediagnosis (interaction.cpp:325-335); vbi[3] = velocity
 * induced at the origin (may be NULL).  Enstrophy terms are identically zero
 * for the Gaussian kernel (gaussian.h:69-92) and follow ENST / ENSTF
 * (highorder.h:71-110) for the high-order kernel.  Zc follows PAWAN: the last wake
 * with non-zero weight wins, else the previous value is kept. */
int pgpu_diagnose(pgpu_ctx *ctx, int32_t system, double *out, double *vbi);

/* The two halves of pgpu_diagnose, for a system split over several contexts
 * by target ranges (no PAWAN counterpart; PAWAN sums on one host,
 * parallel.cpp:140-401 and interaction.cpp:92-132).
 *
 * pgpu_diagnose_partial: PGPU_DIAG_FIELDS FP64 sums per wake of the system
 * (fields[k * PGPU_DIAG_FIELDS + m] for the k-th wake of the system, in the
 * order added) over this context's owned targets, every target if it has no
 * range.  The O(N^2) terms (helicity, kinetic energies, enstrophies) are
 * summed over the unordered pairs whose lower index is an owned target, so
 * the sum of the contexts' fields over a partition of the targets is the
 * whole system's: in FP32C from the source records, which the contexts
 * share after each exchange; the O(N) terms from the owned FP64 state.
 * Layout: 0-2 sum alpha, 3-5 sum x x alpha, 6-8 sum x x (x x alpha), 9-10 the
 * numerator and denominator of Zc, 11-13 the velocity at the origin, 14
 * helicity, 15-16 pair terms of KE and KEF, 17-18 their self terms, 19-20
 * pair terms of the enstrophies, 21-22 their self terms.
 *
 * pgpu_diagnose_combine (host only, no device work): the 15-value record of
 * pgpu_diagnose and vbi from fields summed over the contexts (an all-reduce
 * of nwakes x PGPU_DIAG_FIELDS doubles); zc_prev is the previous Zc, kept if
 * no wake has weight, and *zc_out (may be NULL) receives the new one. */
#define PGPU_DIAG_FIELDS 23
int pgpu_diagnose_partial(pgpu_ctx *ctx, int32_t system, double *fields);
int pgpu_diagnose_combine(const double *fields, int32_t nwakes, double zc_prev, double *out, double *vbi,
                          double *zc_out);

/* Replaces: __interaction::getVi (interaction.cpp:453-477) and the airstation
 * loop of getInflow (:399-451): velocity induced at npts points (row-major
 * (npts, 3)) by every particle of a system, using each particle's own radius. */
int pgpu_probe(pgpu_ctx *ctx, int32_t system, int64_t npts, const double *pts, double *vel);

/* Asynchronous state download for per-step output: the .wake record that
 * PAWAN's offline loop writes after every step (__integration::integrate,
 * integration.cpp:42-50, through __interaction::write, interaction.cpp:304-319,
 * and __wake::write, wake.cpp:832-841).
 *
 * pgpu_snapshot_begin queues on the context's stream, after the work queued so
 * far, a gather of every wake's positions and strengths into device buffer
 * `slot` (0 or 1), then a device-to-host copy of that buffer into a pinned
 * host buffer owned by the context, on a second stream, and returns without
 * waiting.  Work queued afterwards (the next step) runs while the copy is in
 * flight.  Before the gather overwrites a slot, the device waits for that
 * slot's previous copy; the caller must have finished reading the slot's host
 * buffer before it begins the slot again.
 *
 * pgpu_snapshot_wait blocks until the slot's copy has landed (PGPU_ETIMEOUT
 * after `seconds`, the copy left running; seconds <= 0 waits without limit)
 * and returns the host buffer in *state.  Wake w of the snapshot (in creation
 * order) holds n[w] positions, row-major (n[w], 3), at *state + 6 * off[w],
 * followed by its n[w] strengths, row-major (n[w], 3).  off and n receive up
 * to `nwakes` entries (either may be NULL).  The buffer stays valid until the
 * slot's next pgpu_snapshot_begin or pgpu_destroy.  Under a target range
 * (pgpu_set_target_range) only the owned rows of the state are advanced by
 * this context, and only those rows of a snapshot are current.
 * Buffers: 6 * (total capacity) doubles per slot, on the device and pinned on
 * the host, allocated by the slot's first begin.
 * Threads: pgpu_snapshot_wait may run on another thread than the one queueing
 * work on the context (a file writer), as long as no pgpu_snapshot_begin of
 * the same slot runs at the same time; every other call on a context belongs
 * to one thread at a time.  pgpu_last_error gives the message of whichever
 * call failed last. */
int pgpu_snapshot_begin(pgpu_ctx *ctx, int32_t slot);
int pgpu_snapshot_wait(pgpu_ctx *ctx, int32_t slot, double seconds, const double **state, int64_t *off, int64_t *n,
                       int32_t nwakes);

/* Waits for all queued work; reports PGPU_ENUMERIC if a step produced a
 * non-finite state. */
int pgpu_sync(pgpu_ctx *ctx);
/* Pair-kernel timing (pgpu_pair_kernel_time) is on by default.  Reading the
 * CUDA-event times makes pgpu_solve / pgpu_step / pgpu_stage wait for their
 * pair kernels; with timing off (on = 0) those calls only queue work, and
 * pgpu_sync or pgpu_sync_timeout waits.  No PAWAN counterpart. */
int pgpu_set_timing(pgpu_ctx *ctx, int on);
/* pgpu_sync with a host watchdog: returns PGPU_ETIMEOUT if the queued work has
 * not finished after `seconds` (the work is left running; a later pgpu_sync
 * waits for it), else as pgpu_sync.  No PAWAN counterpart. */
int pgpu_sync_timeout(pgpu_ctx *ctx, double seconds);

/* Device time in milliseconds of the pair kernel launches since the last call
 * (CUDA events on the context stream), and the number of them. */
int pgpu_pair_kernel_time(pgpu_ctx *ctx, double *ms, int64_t *launches);

/* Ordered pair interactions (self pairs excluded) evaluated by the pair
 * kernel since the last call, and how many of them took the full formula;
 * with the Gaussian kernel the rest took the far-field limit (FP32C:
 * rho^2 >= 50 sigma^2, where erf rounds to 1 and exp(-rho^2/2sigma^2) <
 * 1.4e-11; FP64: rho^2 >= 100 sigma^2, where the limit equals the closed form
 * to double rounding).  The high-order kernel counts every pair as full.
 * Resets both counts.  No PAWAN counterpart (PAWAN has no counters). */
int pgpu_pair_counts(pgpu_ctx *ctx, int64_t *pairs, int64_t *full_pairs);

/* Kernel launches issued since context creation (all kernels of this library). */
int64_t pgpu_launch_count(pgpu_ctx *ctx);

/* Times every compiled pair-kernel shape on the current particles (`reps`
 * launches each) and selects the fastest for subsequent solves and steps.
 * block/tpt receive the choice; ms_per_launch (may be NULL) receives the
 * time of each candidate in the order of pgpu_kernel_shapes. */
int pgpu_autotune(pgpu_ctx *ctx, int reps, int *block, int *tpt, double *ms_per_launch);
/* Number of compiled pair-kernel shapes and their (block, tpt). */
int pgpu_kernel_shapes(int *block, int *tpt, int max);

/* Autotuning per size class (no PAWAN counterpart: PAWAN's OpenMP loops,
 * parallel.cpp:14-86, have no tiles to choose).  The systems of a context are
 * grouped by particle count into classes (class 0: n < 4096; class k >= 1:
 * 1024 4^k <= n < 1024 4^(k+1)); every compiled shape is timed on each class's
 * systems alone (`reps` launches after one untimed).  If one shape is within
 * 2% of each class's fastest, every system uses it (one pair launch per
 * evaluation); otherwise each class uses its fastest shape, and an evaluation
 * is one pair launch per distinct shape, each over its classes' systems.
 * With cache_path set, a class already recorded there for this GPU name,
 * precision and kernel takes its recorded times instead of being timed, and
 * newly timed classes are appended, one JSON object per line:
 *   {"gpu": .., "precision": "fp32c"|"fp64", "kernel": "gaussian"|"highorder",
 *    "class": k, "nmin": .., "nmax": .., "block": .., "tpt": .., "ms": [one per shape]}
 * classes[i] (up to max_classes) describes the i-th class present, by
 * increasing size; *per_class = 1 if the classes launch separately.  The
 * rates of the current state are recomputed with the chosen launches.  A
 * cache file that cannot be appended to gives PGPU_EINVAL after the choice
 * is in place and the outputs are filled. */
typedef struct pgpu_tune_class {
  int32_t size_class;        /* class index k */
  int32_t systems;           /* systems of the context in the class */
  int64_t nmin, nmax;        /* particle counts [nmin, nmax) of the class */
  int32_t block, tpt;        /* fastest shape of the class */
  int32_t single_block, single_tpt;  /* the one shape with the least total time over all classes */
  int32_t from_cache;        /* 1: times read from the cache file */
  int32_t pad;
  double ms[8];              /* one pair launch over the class's systems, per shape (pgpu_kernel_shapes order) */
} pgpu_tune_class;
int pgpu_autotune_classes(pgpu_ctx *ctx, int reps, const char *cache_path, pgpu_tune_class *classes, int max_classes,
                          int *nclasses, int *per_class);

/* ---------------------------------------------------------------------------
 * Far-field surrogate (no PAWAN counterpart: PAWAN only has the O(N^2) sum).
 *
 * With the surrogate enabled, every rate evaluation of the context's single
 * system uses an octree: each target leaf's near field (cells closer than
 * near_widths cube widths, or with a particle within sqrt(far_u) sigma_ij of the leaf's)
 * is summed exactly with the direct kernel's terms,
 * and farther cells act through their multipole moments (order 0/1/2/3),
 * optionally corrected by the learned model of pgpu_surrogate_set_mlp.  After
 * every evaluation, check_targets sampled targets are recomputed by the direct
 * sum; if the max-norm relative error of the velocity or of dalpha/dt
 * exceeds `tolerance`, the evaluation is redone by the direct sum (the
 * surrogate never returns an unchecked result when check_targets > 0). */
typedef struct pgpu_surrogate_config {
  int leaf_size;       /* particles per octree leaf, 1..512 (default 256) */
  double near_widths;  /* near field: cells closer than this many cube widths (default 5) */
  int order;           /* far-field expansion: 0 monopole, 1 + dipole, 2 + quadrupole (default), 3 + octupole */
  int use_mlp;         /* add the learned correction to the far field of `order` (pgpu_surrogate_set_mlp) */
  double tolerance;    /* maximum relative error of the velocity and of dalpha/dt on the sampled targets
                          (default 1e-4) */
  int check_targets;   /* targets re-checked by the direct sum per evaluation (default 4096, 0 = off) */
  int seed;            /* seed of the sampled targets */
  double far_u;        /* a far cell's particles are all at rho^2 >= far_u sigma_ij^2 from the leaf's
                          (default 16, 0 = no test): the expansion is of the singular kernel, and the
                          Gaussian core it leaves out decays as exp(-far_u / 2) */
} pgpu_surrogate_config;

typedef struct pgpu_surrogate_stats {
  int64_t evaluations;     /* surrogate evaluations since enable */
  int64_t fallbacks;       /* evaluations redone by the direct sum */
  double last_err_vel;     /* sampled max-norm relative velocity error of the last evaluation */
  double last_err_dalpha;  /* same for dalpha/dt */
  double max_err_vel;      /* largest sampled velocity error seen */
  double ms_tree, ms_eval, ms_check, ms_fallback;  /* device time of the last evaluation's phases */
  int64_t cells, leaves;   /* octree of the last evaluation */
  int64_t far_entries, near_entries;  /* interaction-list lengths summed over leaves */
  double max_err_dalpha;   /* largest sampled dalpha/dt error seen */
} pgpu_surrogate_stats;

void pgpu_surrogate_config_default(pgpu_surrogate_config *cfg);
/* Enables the surrogate for `system`, which must be the context's only system.
 * Refused (PGPU_EINVAL) for a context with the high-order kernel. */
int pgpu_surrogate_enable(pgpu_ctx *ctx, int32_t system, const pgpu_surrogate_config *cfg);
int pgpu_surrogate_disable(pgpu_ctx *ctx);
int pgpu_surrogate_get_stats(pgpu_ctx *ctx, pgpu_surrogate_stats *stats);
/* Copies the octree of the last surrogate evaluation to host buffers (for
 * inspection and tests): idx[n] maps sorted position to particle index;
 * cell[4 ncells] = (start, end, first_child, nchild) per cell; leaves[nleaves]
 * are cell indices; counts[2 nleaves] = far- then near-list lengths.  Any
 * buffer may be NULL; a buffer smaller than needed is left untouched. */
int pgpu_surrogate_tree(pgpu_ctx *ctx, int *idx, int64_t idx_cap, int *cell, int64_t cell_cap, int *leaves,
                        int *counts, int64_t leaf_cap, int64_t *n, int64_t *ncells, int64_t *nleaves);

/* ---------------------------------------------------------------------------
 * Far-field correction network (no PAWAN counterpart).  A 24-128-128-128-6
 * GELU MLP whose products run on the tensor cores in BF16 with FP32
 * accumulation (forward, backward and Adam are this library's kernels:
 * training and pgpu_mlp_forward on the tcgen05 tensor cores with TMEM
 * accumulators, the far field's fused per-warp path on mma.sync).  It
 * predicts, per (target, far cell) pair, the residual of the multipole
 * expansion of the order it was trained against, from the cell's moments and
 * the target offset; the features and output scales are documented in
 * pawan_b200/csrc/treeeval.cuh.  Parameters
 * are pgpu_mlp_num_params() floats: W1[32][128] (rows 24..31 zero), b1[128],
 * W2[128][128], b2[128], W3[128][128], b3[128], W4[128][8] (columns 6, 7
 * zero), b4[8]; a row times W is the layer's pre-activation. */
typedef struct pgpu_mlp pgpu_mlp;
int pgpu_mlp_num_params(void);
int pgpu_mlp_create(pgpu_mlp **mlp, int device, int seed);  /* Glorot-uniform weights from `seed` */
int pgpu_mlp_destroy(pgpu_mlp *mlp);
const char *pgpu_mlp_last_error(pgpu_mlp *mlp);
int pgpu_mlp_get_params(pgpu_mlp *mlp, float *params);
int pgpu_mlp_set_params(pgpu_mlp *mlp, const float *params);  /* also resets the Adam state */
/* Outputs (rows x 6) for host feature rows (rows x 24). */
int pgpu_mlp_forward(pgpu_mlp *mlp, const float *x, int64_t rows, float *y);
/* The same outputs through the fused warp-level path of the far field
 * (packed BF16 weights, activations in registers, tanh.approx GELU). */
int pgpu_mlp_forward_fused(pgpu_mlp *mlp, const float *x, int64_t rows, float *y);
/* Mean-squared-error loss over the rows and its gradient (params layout). */
int pgpu_mlp_gradient(pgpu_mlp *mlp, const float *x, const float *t, int64_t rows, float *grad, double *loss);
/* Training set: replace with host rows, or append rows drawn from the octree
 * of a context's last surrogate evaluation (targets are the exact direct-sum
 * contribution of the cell minus its expansion to the context's surrogate
 * order, scaled).  The network and the context must be on the same device
 * (PGPU_EINVAL otherwise), here and in pgpu_surrogate_set_mlp. */
int pgpu_mlp_set_dataset(pgpu_mlp *mlp, const float *x, const float *t, int64_t rows);
int pgpu_mlp_add_samples(pgpu_mlp *mlp, pgpu_ctx *ctx, int64_t nsamples, int seed);
int64_t pgpu_mlp_dataset_rows(pgpu_mlp *mlp);
int pgpu_mlp_get_dataset(pgpu_mlp *mlp, float *x, float *t, int64_t max_rows);
/* Adam (beta 0.9 / 0.999) on random minibatches; loss_history[steps] may be NULL. */
int pgpu_mlp_train(pgpu_mlp *mlp, int steps, int batch, double lr, int seed, float *loss_history);
/* Uses a snapshot of the network's current weights for the surrogate's far
 * field (expansion to the configured order + correction) when use_mlp is set;
 * the network should have been trained on samples drawn at that order. */
int pgpu_surrogate_set_mlp(pgpu_ctx *ctx, pgpu_mlp *mlp);

/* The context's CUDA stream (a cudaStream_t), so a caller can order its own
 * work or timing events with the library's launches.  No PAWAN counterpart. */
int pgpu_get_stream(pgpu_ctx *ctx, void **stream);

/* Measures the device's sustained FP32 FMA throughput (TFLOP/s, an FMA
 * counted as 2 flops) with register-resident FMA loops on every SM, for
 * roofline denominators: scalar FFMA and the packed two-wide FFMA2 of sm_100.
 * pgpu_fp32_peak gives the larger of the two (ms is set to 0).  No PAWAN
 * counterpart. */
int pgpu_fp32_peaks(int device, double *ffma_tflops, double *ffma2_tflops);
int pgpu_fp32_peak(int device, double *tflops, double *ms);
/* The same measurement for the FP64 pipe (DFMA register loop), the bound of
 * the FP64 mode's pair kernel.  No PAWAN counterpart. */
int pgpu_fp64_peak(int device, double *tflops);

/* Largest system pgpu_rates_noalloc accepts (its fixed scratch: ~13.6 MB of
 * device memory per GPU, held from library load until process exit). */
#define PGPU_NOALLOC_MAX_N 32768

/* Velocity and dalpha/dt of one system of n <= PGPU_NOALLOC_MAX_N particles,
 * FP32C pair terms as pgpu_solve computes them (no freestream added), for
 * callers that must not allocate device memory: a host whose own pool owns
 * all of the GPU's memory, or a real-time loop where cudaMalloc would
 * synchronise the device.  No counterpart in PAWAN, which has no device code.
 *
 * All arrays are DEVICE pointers, row-major FP64: pos, alpha, vel, dalpha
 * (n, 3); sigma, vol (n).  Work is queued on `stream` (a cudaStream_t, NULL
 * for the legacy default stream); the call does not wait for it.  It never
 * calls cudaMalloc or cudaFree: its intermediates live in one static device
 * array.  The first call on each device looks up that array's address and
 * clears its work counters (an asynchronous memset on `stream`, ordered
 * before that call's kernels), so make it before any stream capture.  Calls
 * share the array: calls that overlap on the GPU (different streams, or host
 * threads without ordering) race and must not be issued.
 * n > PGPU_NOALLOC_MAX_N is rejected with PGPU_EINVAL; the reason is in
 * pgpu_noalloc_last_error(). */
int pgpu_rates_noalloc(const double *pos, const double *alpha, const double *sigma, const double *vol, int64_t n,
                       double nu, double *vel, double *dalpha, void *stream);
/* Message for the last pgpu_rates_noalloc failure on the calling thread ("" after a success). */
const char *pgpu_noalloc_last_error(void);

/* Message of the last failure on ctx; with ctx NULL, of the calling thread's
 * last pgpu_create ("" after a success). */
const char *pgpu_last_error(pgpu_ctx *ctx);
const char *pgpu_version(void);

#ifdef __cplusplus
}
#endif
#endif
