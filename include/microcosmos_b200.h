/*
 * microcosmos_b200 — C ABI of the B200 (sm_100a) physics hot path of microcosmos.
 *
 * One rollout = the reference's `simulate(nodes, edges, fields, dt, num_steps,
 * solver_config)` (src/microcosmos/simulate.py:15-35) with the PBD constraint plugin
 * (src/microcosmos/solver/pbd.py:14-91), the IB + D2Q9 TRT lattice-Boltzmann fluid
 * (src/microcosmos/solver/fluid.py:202-386) and the FFT steric field
 * (src/microcosmos/forces.py:41-118).  A batch is a set of rollouts of any sizes that
 * step together; the single-instance path is a batch of one.
 *
 * Conventions
 *   - All array arguments of mc_state / mc_actuation / mc_record are DEVICE pointers
 *     (float32 or int32, C-contiguous, the reference's layouts: positions (N,2) as
 *     (x, y), f_grid (9,H,W), fluid_velocity (2,H,W), steric (H,W)).  Topology
 *     (pairs, bending_pairs) is passed as HOST arrays at plan creation.
 *   - The library never allocates device memory: the caller provides one workspace of
 *     mc_plan_workspace_bytes() bytes (256-byte aligned).  Host memory for the plan
 *     object itself is allocated by mc_plan_create and released by mc_plan_destroy.
 *   - Work is stream-ordered on the caller's stream; calls return after enqueueing.
 *     A plan is not thread-safe; distinct plans are independent.
 *   - Errors are returned as mc_status; nothing aborts, traps or exits.
 *     Numerical faults (non-finite node state) are recorded per rollout on the device
 *     and read back with mc_plan_read_flags().
 */
#ifndef MICROCOSMOS_B200_H
#define MICROCOSMOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mc_status {
  MC_OK = 0,
  MC_ERR_INVALID = 1,      /* bad argument: shape, index out of range, null pointer */
  MC_ERR_CUDA = 2,         /* a CUDA runtime call failed (mc_last_error() has the text) */
  MC_ERR_WORKSPACE = 3,    /* workspace missing, too small or misaligned */
  MC_ERR_UNSUPPORTED = 4,  /* configuration outside what the kernels implement */
  MC_ERR_NOT_BOUND = 5     /* plan used before mc_plan_bind() */
} mc_status;

/* Per-rollout flag bits reported by mc_plan_read_flags(). */
#define MC_FLAG_NONFINITE 1u /* a node position/velocity became NaN/Inf */
#define MC_FLAG_TIMEOUT 2u   /* a bounded device-side wait gave up; the step's results are invalid */

/* Scalar fields of ConstraintSolverConfig (src/microcosmos/solver/config.py:9-72).  The
 * callable `bending_constraint` plugin slot is selected by solver_type:
 * MC_SOLVER_PBD = pbd_rod_constraint (solver/pbd.py:14-91), MC_SOLVER_COSSERAT =
 * stable_cosserat_constraint (solver/stable_cosserat.py:13-119, inertia weight
 * 1/solver_dt^2 where solver_dt is the config's own `dt` field).
 * `cycles_per_constraint` is never read by the reference. */
#define MC_SOLVER_PBD 0
#define MC_SOLVER_COSSERAT 1
typedef struct mc_config {
  int32_t cycles_per_step;
  float stiffness_stretch;
  float stiffness_shear;
  float damping;
  int32_t enable_fluid;
  double viscosity;           /* a Python float: omega+ = 1/(3 viscosity + 0.5) is taken in double */
  double max_fluid_velocity;  /* a Python float: the velocity caps are max_fluid_velocity times the
                               * mean grid scale, taken in double and rounded once to float32 */
  int32_t ibm_iterations;
  float synthetic_node_width; /* >= 0; > 0 puts a pair of IB points at +- width along the chain normal */
  int32_t ibm_kernel_size;    /* 1..8 */
  float ibm_relaxation;
  float node_mass;
  float lambda_trt;
  int32_t enable_force_clamp;
  int32_t enable_steric;
  float steric_strength;
  double steric_sigma;        /* a Python float: 2 sigma^2 etc. are taken in double */
  int32_t steric_neighbor_skip;
  float steric_scatter_value;
  int32_t solver_type;        /* MC_SOLVER_PBD or MC_SOLVER_COSSERAT */
  double solver_dt;           /* ConstraintSolverConfig.dt (a Python float; Cosserat inertia weight), > 0 */
} mc_config;

/* Sizes of one rollout.  H, W: grid_shape, the domain grid of positions and of the steric
 * field.  fluid_H, fluid_W: the lattice of f_grid (src/microcosmos/solver/fluid.py:221-235:
 * IB points at position * (fluid_W / H, fluid_H / W), velocities and the velocity clamp
 * scaled to match); 0 = the domain grid. */
typedef struct mc_dims {
  int32_t H, W;
  int32_t N; /* nodes */
  int32_t E; /* edges (pairs) */
  int32_t B; /* bending pairs */
  int32_t fluid_H, fluid_W;
} mc_dims;

/* Device state of one rollout (Nodes / Edges / Fields of src/microcosmos/structs/*.py).
 * Read at the start of a rollout call and written back at its end. */
typedef struct mc_state {
  float* position;            /* (N,2) in/out */
  float* velocity;            /* (N,2) in/out */
  float* theta;               /* (E,)  in/out */
  const float* rest_lengths;  /* (E,)  in */
  float* bending_rest_angles; /* (B,)  in/out (overwritten by the actuation, if any) */
  const float* bending_stiffness; /* (B,) in */
  float* steric;              /* (H,W) in/out */
  float* fluid_velocity;      /* (2,fluid_H,fluid_W) in/out (u* of the last step) */
  float* f_grid;              /* (9,fluid_H,fluid_W) in/out */
} mc_state;

/* Optional caller-side curvature actuation, evaluated on the device before every step:
 *   rest[b](t) = c[b] + amp[b] * sin(omega[b] * t + phase[b]),  t = t0 + step index.
 * Replaces the reference's control_fn that rewrites edges.bending_rest_angles before
 * each step (experiments/swim_sweep/swimmers/worm.py:60-74). All arrays (B,), device. */
typedef struct mc_actuation {
  const float* c;
  const float* amp;
  const float* omega;
  const float* phase;
  int32_t t0;
} mc_actuation;

/* Optional per-step recording, the reference's scan outputs (simulate.py:21-34).
 * Entry k (0-based) is written after step (k+1)*every - 1.  Any pointer may be NULL. */
typedef struct mc_record {
  float* position;       /* (T,N,2) */
  float* velocity;       /* (T,N,2) */
  float* steric;         /* (T,H,W) */
  float* fluid_velocity; /* (T,2,H,W): u* on the domain grid, linearly resized from the
                          * fluid grid when the two differ (simulate.py:24-29) */
  int32_t every;         /* >= 1 */
} mc_record;

typedef struct mc_plan mc_plan;

/* Build a plan for `n` rollouts.  dims/cfg/dt/pairs/bending_pairs are arrays of length
 * n; pairs[r] is (E_r,2) and bending_pairs[r] is (B_r,2) int32 HOST memory.  The
 * topology is validated (indices in range) and turned into gather lists that keep the
 * reference's scatter-add order.  Replaces the jit-static arguments of
 * simulate()/step() (src/microcosmos/simulate.py:15,37). */
mc_status mc_plan_create(int32_t n, const mc_dims* dims, const mc_config* cfg, const float* dt,
                         const int32_t* const* pairs, const int32_t* const* bending_pairs,
                         mc_plan** out);
void mc_plan_destroy(mc_plan* plan);

/* Tile shape of the dense stream+collide pass: each CTA covers 32 * cells_per_lane columns
 * (1, 2 or 4 cells per thread, vector loads and stores; it must divide every rollout's
 * lattice width) by rows_per_cta rows (2, 4, 8, 16 or 32; up to 4 warps per CTA, each
 * looping over rows_per_cta / 4 rows).  The default is 4 cells per lane by 16 rows for plans
 * of at least 4 M lattice cells and 2 cells per lane by 4 rows below (fewer cells per lane
 * when a width needs it).  0 keeps the current value.  Results do not depend on the shape.
 * Only before mc_plan_bind(); microcosmos_b200.autotune picks it by timing.
 * No counterpart in the reference (XLA chooses its own fusion tiling). */
mc_status mc_plan_set_lbm_shape(mc_plan* plan, int32_t cells_per_lane, int32_t rows_per_cta);
mc_status mc_plan_get_lbm_shape(const mc_plan* plan, int32_t* cells_per_lane, int32_t* rows_per_cta);

/* Staged dense pass: stages = 2..6 runs the stream+collide pass as a persistent kernel whose
 * CTAs copy bands of whole lattice rows (about 1024 cells) of the 9 population planes into
 * shared memory with bulk asynchronous copies, `stages` bands in flight per CTA, and collide
 * them from there; 0 selects the tiled kernel of mc_plan_set_lbm_shape (which also selects
 * it).  Needs every fluid lattice width to be a multiple of 4 and at most 1024
 * (MC_ERR_UNSUPPORTED otherwise).  Results do not depend on the choice.  Only before
 * mc_plan_bind(); mc_plan_lbm_staging returns the current value (-1 for a null plan).
 * No counterpart in the reference (XLA chooses its own fusion tiling). */
mc_status mc_plan_set_lbm_staging(mc_plan* plan, int32_t stages);
int32_t mc_plan_lbm_staging(const mc_plan* plan);

/* How the steric potential's spectral Gaussian (src/microcosmos/utils.py:35-49) is applied:
 * 1 = FFT along rows, then columns (H, W with prime factors <= 13, at most 4096): the
 *     reference's operator, to float32 rounding;
 * 2 = direct circular convolution with the filter's periodic kernel kept to radius 24 (one
 *     32 x 32 tile per CTA; needs 2 * 24 + 1 <= H, W).  The Nyquist cut-off of the spectral
 *     Gaussian leaves a ~1e-6 tail in that kernel beyond the Gaussian core, which this
 *     drops: the field differs from the FFT's by ~6e-7 rel-L2 (sigma = 1.5);
 * 0 = per rollout, the FFT where it exists, else the direct form (the default).
 * Only before mc_plan_bind().  mc_plan_steric_method returns 1 (all FFT), 2 (all direct),
 * 3 (mixed) or 0 (no steric rollout). */
mc_status mc_plan_set_steric_method(mc_plan* plan, int32_t method);
int32_t mc_plan_steric_method(const mc_plan* plan);

/* Values each thread holds in registers in the FFT kernels of power-of-two sides (4, 8 or
 * 16; 0 = the library's choice from the plan's total size).  More values per thread take
 * fewer instructions per value, fewer give more threads: small single rollouts want 4,
 * large batches 16.  Results do not depend on it beyond float32 rounding of the transform
 * order.  Only before mc_plan_bind(); microcosmos_b200.autotune picks it by timing.  No
 * counterpart in the reference. */
mc_status mc_plan_set_fft_values_per_thread(mc_plan* plan, int32_t values);
int32_t mc_plan_fft_values_per_thread(const mc_plan* plan);

/* Threads per CTA of the tile kernel that sorts the IB and cloud-in-cell contributions of
 * each touched 16 x 16 tile (64, 128 or 256; 0 = 128).  Sparse tiles favour small CTAs.
 * Results do not depend on it.  Only before mc_plan_bind().  No counterpart in the
 * reference. */
mc_status mc_plan_set_bin_threads(mc_plan* plan, int32_t threads);
int32_t mc_plan_bin_threads(const mc_plan* plan);

/* Contributions a touched tile may hold to be sorted in shared memory (a power of two in
 * 256..8192, capped by the plan's bin capacity; 0 = 2048).  Denser tiles sort in a global
 * arena.  Smaller capacities keep more CTAs resident.  Results do not depend on it.  Only
 * before mc_plan_bind().  No counterpart in the reference. */
mc_status mc_plan_set_bin_sort_capacity(mc_plan* plan, int32_t entries);
int32_t mc_plan_bin_sort_capacity(const mc_plan* plan);

/* Bytes of device workspace the plan needs (all rollouts). */
size_t mc_plan_workspace_bytes(const mc_plan* plan);

/* Attach a caller-allocated device workspace and upload the plan's tables on `stream`. */
mc_status mc_plan_bind(mc_plan* plan, void* workspace, size_t bytes, void* stream);

/* Run `num_steps` steps of every rollout of the plan: the device-side equivalent of
 * simulate() (src/microcosmos/simulate.py:15-35) / repeated step() (:37-100).
 * states[r], act[r] (NULL = none), rec[r] (NULL = none) per rollout; act and rec may
 * themselves be NULL.  use_graph != 0 captures the per-step launch sequence in a CUDA
 * graph on first use and replays it. */
mc_status mc_rollout(mc_plan* plan, const mc_state* states, int32_t num_steps,
                     const mc_actuation* const* act, const mc_record* const* rec,
                     int32_t use_graph, void* stream);

/* The three phases of mc_rollout, for callers that interleave their own work between
 * steps (timing, L2 flushes, host control).  begin: bind states/actuation/recording and
 * convert fields.f_grid to the internal layout; advance: run num_steps more steps
 * (last != 0: the final one of them writes fields.fluid_velocity and the call returns with
 * that step complete -- none of the next step is started -- so the caller may change the
 * state's positions, velocities, rest lengths or rest angles before a further advance; the
 * advance before end must pass last != 0); end: write fields.f_grid back.
 * mc_rollout(...) == begin + advance(num_steps, last=1) + end. */
mc_status mc_rollout_begin(mc_plan* plan, const mc_state* states, const mc_actuation* const* act,
                           const mc_record* const* rec, void* stream);
mc_status mc_rollout_advance(mc_plan* plan, int32_t num_steps, int32_t use_graph, int32_t last, void* stream);
mc_status mc_rollout_end(mc_plan* plan, void* stream);

/* One step: mc_rollout with num_steps = 1 (src/microcosmos/simulate.py:37-100). */
mc_status mc_step(mc_plan* plan, const mc_state* states, void* stream);

/* Copy the per-rollout MC_FLAG_* words to host `flags` (n entries); synchronises
 * `stream`.  clear != 0 resets them afterwards. */
mc_status mc_plan_read_flags(mc_plan* plan, uint32_t* flags, int32_t clear, void* stream);

/* Number of kernel launches the last mc_rollout() enqueued (graph replays count the
 * kernels inside the graph). */
int64_t mc_plan_last_launch_count(const mc_plan* plan);

/* The multi-direct forcing iterations run either as separate interpolate / spread launches
 * (the default) or, with enable != 0, as one cooperative kernel with bounded device-side
 * barriers (used only when all of its CTAs fit on the GPU at once).  Both give identical
 * results.  Call after mc_plan_bind, outside a rollout. */
mc_status mc_plan_set_fused_ib(mc_plan* plan, int32_t enable);
int32_t mc_plan_uses_fused_ib(const mc_plan* plan);

/* The multi-direct forcing iterations and the body force of each rollout in one
 * thread-block cluster of `ctas` CTAs (1..16; 0 = separate launches, the default), phases
 * separated by the hardware cluster barrier instead of kernel boundaries.  Same arithmetic
 * and order, identical results.  Pays off when a plan holds many rollouts with few IB
 * points each (their iterations then run side by side with no launch per phase); a single
 * large rollout keeps more threads in flight with the separate launches.  Call after
 * mc_plan_bind, outside a rollout; microcosmos_b200.autotune picks it by timing.
 * No counterpart in the reference (its iterations are a lax.scan of dense grid ops,
 * solver/fluid.py:292-316). */
mc_status mc_plan_set_ib_cluster(mc_plan* plan, int32_t ctas);
int32_t mc_plan_ib_cluster(const mc_plan* plan);

/* Per-kernel CUDA-event timing.  While enabled, steps are launched directly (no graph)
 * and each kernel launch is bracketed by two events; mc_plan_profile_read() returns the
 * accumulated milliseconds and launch count of one kernel (names from
 * mc_profile_kernel_names(), comma-separated) and synchronises on pending events. */
mc_status mc_plan_profile(mc_plan* plan, int32_t enable);
mc_status mc_plan_profile_read(mc_plan* plan, const char* kernel, double* total_ms, int64_t* launches);
mc_status mc_plan_profile_reset(mc_plan* plan);
const char* mc_profile_kernel_names(void);

/* Steric potential field of N node positions without any device allocation.
 *
 * No counterpart in the reference: it computes the same field as the reference's
 * update_steric_potential (cloud-in-cell deposit of the wrapped positions followed by the
 * spectral Gaussian of width sigma) and as fields.steric after a step from these positions
 * with zero velocity, but for callers that cannot call cudaMalloc — e.g. a custom call
 * inside a framework that owns all device memory and gave it no workspace buffer, or a
 * host loop that must not allocate once it is running.  position (N,2) and steric_out
 * (H,W) are caller-owned device arrays; nothing else is passed in.
 *
 * Limits: 1 <= N <= MC_NOALLOC_MAX_NODES, 4 <= H, W <= MC_NOALLOC_MAX_GRID (prime factors
 * <= 13); larger sizes return MC_ERR_INVALID.  The scratch (about 6.6 MB) is one
 * file-scope __device__ array that every GPU loading this library keeps until the process
 * exits.  The first call made on a device looks up that array's device address (set-up);
 * make that first call before any stream capture.  The address is kept per device together
 * with the id of the context it belongs to, so the first call after that context is torn
 * down (cudaDeviceReset) repeats the set-up.  Each call enqueues one set-up kernel that
 * receives the call's tables and descriptor as its by-value parameter, writes them into the
 * array and clears what must start at zero, then the deposit and filter kernels.  All calls
 * share the array, so calls that overlap on the GPU (different streams, no ordering between
 * them) race and must not be issued. */
#define MC_NOALLOC_MAX_GRID 512
#define MC_NOALLOC_MAX_NODES 16384
mc_status mc_steric_potential_noalloc(const float* position, int32_t N, int32_t H, int32_t W, float sigma,
                                      float scatter_value, float* steric_out, void* stream);

/* ------------------------------------------------------------------ gradients
 * Reverse-mode derivative of a rollout of ONE instance, with the derivative conventions
 * jax.grad applies to the reference's simulate() (src/microcosmos/simulate.py:15-35):
 * the IB stencil positions are stop_gradient-ed (src/microcosmos/solver/fluid.py:239),
 * floor has derivative 0, mod derivative 1, max/min split ties evenly.  It replaces the
 * jax.grad / jax.value_and_grad calls on simulate() in the reference's
 * tests/test_differentiability.py:45,65 (there through XLA's autodiff; here through
 * hand-written adjoint kernels of stream+collide, IB, PBD / stable Cosserat and steric).
 *
 * mc_grad_forward runs the rollout with the same kernels as mc_rollout, keeping a
 * checkpoint of (position, velocity, theta, f_grid) every `checkpoint_every` steps
 * (<= 0: ceil(sqrt(num_steps))).  mc_grad_backward recomputes each segment's step inputs
 * from its checkpoint and runs the adjoint steps in reverse: device memory is
 * O(sqrt(T)) states, compute about three forward rollouts plus the adjoint.
 * Cotangents of the outputs steric and fluid_velocity are taken as zero.
 * Actuation, if given to mc_grad_forward, must have t0 = 0.  Both rod solvers (MC_SOLVER_PBD, MC_SOLVER_COSSERAT) are
 * differentiated, with or without synthetic IB pairs, the force clamp and a fluid lattice
 * other than the domain grid (dims->fluid_H/fluid_W; f_grid arrays and cotangents are then
 * (9, fluid_H, fluid_W)). */
typedef struct mc_state_cot {
  float* position; /* (N,2) */
  float* velocity; /* (N,2) */
  float* theta;    /* (E,)  */
  float* f_grid;   /* (9,H,W) */
} mc_state_cot;

/* Gradient outputs, any may be NULL.  rest_angles: the static bending_rest_angles (used
 * when mc_grad_forward had no actuation); act_c/act_amp/act_phase/act_omega: the actuation
 * arrays. */
typedef struct mc_param_grads {
  float* rest_angles;       /* (B,) */
  float* act_c;             /* (B,) */
  float* act_amp;           /* (B,) */
  float* act_phase;         /* (B,) */
  float* rest_lengths;      /* (E,) */
  float* bending_stiffness; /* (B,) */
  float* act_omega;         /* (B,) */
} mc_param_grads;

typedef struct mc_grad_plan mc_grad_plan;

mc_status mc_grad_plan_create(const mc_dims* dims, const mc_config* cfg, float dt, const int32_t* pairs,
                              const int32_t* bending_pairs, int32_t num_steps, int32_t checkpoint_every,
                              mc_grad_plan** out);
void mc_grad_plan_destroy(mc_grad_plan* plan);
size_t mc_grad_plan_workspace_bytes(const mc_grad_plan* plan);
int32_t mc_grad_plan_checkpoint_every(const mc_grad_plan* plan);
mc_status mc_grad_plan_bind(mc_grad_plan* plan, void* workspace, size_t bytes, void* stream);
/* Forward rollout of num_steps steps; the state is read and overwritten with the final
 * state (all mc_state arrays as in mc_rollout). */
mc_status mc_grad_forward(mc_grad_plan* plan, const mc_state* state, const mc_actuation* act, void* stream);
/* Given the cotangent of the final state (NULL arrays = zero), write the cotangent of the
 * initial state and the parameter gradients.  final_cot and initial_cot may alias. */
mc_status mc_grad_backward(mc_grad_plan* plan, const mc_state_cot* final_cot, mc_state_cot* initial_cot,
                           mc_param_grads* grads, void* stream);

/* ------------------------------------------------------------------ gym environments
 * The device work of the reference's gym Environment.step around one rollout step
 * (src/microcosmos/gym/base.py:173-196), for a table of environments (the reference
 * batches environments with jax.vmap): mc_env_act writes the step's rest lengths and
 * rest angles from the episode's base values plus the action (base.py:177-182; then
 * mc_rollout runs the step on the same buffers), mc_env_observe walks the energy source
 * (base.py:187-190), writes the observation (base.py:112-121) and the reward (base.py:123-124;
 * per node range for several creatures, multi_agent.py:201-212), advances the step counter
 * and sets done = time >= max_steps (base.py:192-195).  All pointers are device pointers. */
typedef struct mc_env {
  int32_t N, E, B;                        /* nodes, edges, bending pairs */
  int32_t H, W;                           /* grid_shape */
  const float* base_rest_lengths;         /* (E,) the episode's rest lengths */
  const float* base_bending_rest_angles;  /* (B,) */
  const float* d_rest_length;             /* (E,) action; NULL = zero */
  const float* d_bending_angle;           /* (B,) action; NULL = zero */
  float* rest_lengths;                    /* (E,) out: the buffers the step reads */
  float* bending_rest_angles;             /* (B,) out */
  const float* position;                  /* (N,2) the state after the step */
  const float* velocity;                  /* (N,2) */
  float* energy_center;                   /* (2,) in/out */
  const float* noise;                     /* (2,) standard-normal draws of this step; NULL = no walk */
  float energy_walk_std;
  float energy_amplitude;
  float energy_two_size_sq;               /* float32 of 2 * energy_size^2 */
  int32_t max_steps;
  int32_t* time;                          /* () in/out */
  int32_t* done;                          /* () out */
  float* observation;                     /* (5N,) out: positions - mean (2N), velocities (2N), energy (N) */
  float* reward;                          /* () out */
  int32_t num_segments;                   /* node ranges ("creatures"), 0 or 1 = one */
  const int32_t* segment_offsets;         /* (num_segments+1,) node offsets; NULL with one range */
  float* segment_fitness;                 /* (num_segments,) out, may be NULL */
} mc_env;

/* Device bytes of a table of n environments; mc_env_table_upload copies the host structs
 * into such a caller-owned device buffer (stream-ordered; the host array may be freed on
 * return). */
size_t mc_env_table_bytes(int32_t n);
mc_status mc_env_table_upload(const mc_env* envs, int32_t n, void* table, void* stream);
mc_status mc_env_act(const void* table, int32_t n, void* stream);
/* advance = 0: the observation, reward and fitness of the current state only (reset,
 * base.py:140-149); the energy source, step counter and done flag are left alone. */
mc_status mc_env_observe(const void* table, int32_t n, int32_t advance, void* stream);

/* ------------------------------------------------------------------ frames
 * The reference's render() of a recorded rollout (src/microcosmos/rendering.py:20-80)
 * into a caller-owned device buffer, no display or graphics API involved.  Inputs (device):
 * position and debug_vector (T,N,2) (debug_vector may be NULL = zero), color_bend (N,)
 * (the first frame's colours; NULL = 0), steric (T,H,W).  Output frames
 * (T, size*H/max(H,W), size*W/max(H,W), 3) uint8 RGB.  scratch: mc_render_scratch_bytes
 * (T,H,W) bytes of device memory (unused when render_particles == 0). */
size_t mc_render_scratch_bytes(int32_t T, int32_t H, int32_t W);
mc_status mc_render_frames(const float* position, const float* debug_vector, const float* color_bend,
                           const float* steric, int32_t T, int32_t N, int32_t H, int32_t W, int32_t size,
                           int32_t render_particles, int32_t uniform_color, int32_t* scratch, uint8_t* frames,
                           void* stream);

/* Text of the last error of this thread ("" if none). */
const char* mc_last_error(void);

/* Library version string. */
const char* mc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MICROCOSMOS_B200_H */
