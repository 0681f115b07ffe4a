/*
 * snow_gpu.h -- C ABI of the B200 explicit-MPM snow step.
 *
 * This is the boundary between the C++20 drop-in API (the headers under include/snow/, the
 * reference solver's own function signatures) and the sm_100a CUDA kernels.
 * Only plain C types cross it: pointers, sizes, doubles and small structs.
 * Every entry point returns 0 on success or a negative SNOW_E* code; the text
 * of the last error on the calling thread is available from
 * snow_gpu_last_error().  A `stream` argument is a cudaStream_t (NULL = the
 * legacy default stream); calls are stream-ordered and, unless stated
 * otherwise, return once their work has completed.
 *
 * Particles cross the boundary as records of 26 doubles (208 bytes) in the
 * order of the reference's struct Particle (include/snow/particle.hpp:5-28 in
 * the reference tree): x_p[3], v_p[3], m_p, V_p0, F_P[9], F_E[9], the 3x3
 * matrices column-major as in Eigen::Matrix3d.
 *
 * Reference interfaces replaced (reference tree paths):
 *   snow_gpu_setup            setup(std::vector<Particle>&, double)          include/snow/grid.hpp:96, src/grid.cpp:340
 *   snow_gpu_step             step(particles, colliders, stencils, gravity, dt, dx, mu_0,
 *                             lambda_0, xi, theta_c, theta_s, alpha, timings)  include/snow/grid.hpp:97, src/grid.cpp:359
 *   snow_gpu_make_plane       make_plane(point, normal, friction)             include/snow/collision.hpp:14, src/collision.cpp:5
 *   snow_step_timings         struct StepTimings                              include/snow/debug.hpp:3-15
 *   snow_gpu_stage_*          the per-stage functions of include/snow/grid.hpp:75-95
 *                             (P2G, calculate_volume, force_calculation,
 *                             grid_velocity, grid_collisions, stress_update,
 *                             G2P, particle_collisions, position_update)
 *   snow_gpu_batch_*          no reference counterpart: many independent scenes
 *                             advanced by one launch per stage
 */
#ifndef SNOW_GPU_H
#define SNOW_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNOW_GPU_ABI_VERSION 2
#define SNOW_RECORD_DOUBLES 26

enum {
  SNOW_OK = 0,
  SNOW_E_ARG = -1,        /* invalid argument */
  SNOW_E_CUDA = -2,       /* CUDA runtime error (no device, out of memory, ...) */
  SNOW_E_CAPACITY = -3,   /* grid block / hash capacity exceeded during a step */
  SNOW_E_NONFINITE = -4,  /* a particle position became NaN or infinite */
  SNOW_E_KEYRANGE = -5,   /* scene extent too large for the 32-bit block keys */
  SNOW_E_STATE = -6       /* call out of order (e.g. unknown scene id) */
};

/* Precision of a batch. */
enum {
  SNOW_FP64 = 0,  /* every quantity in double: the drop-in path */
  SNOW_MIXED = 1  /* x, v, m, V_p0, F_E, grid and transfers in float; F_P, its
                     determinant and the hardening exponential in double */
};

/* Collider kinds. */
enum { SNOW_COLLIDER_PLANE = 0, SNOW_COLLIDER_SPHERE = 1, SNOW_COLLIDER_BOX = 2 };

/* A collider (CollisionBody, include/snow/collision.hpp:6-12; the reference
 * takes any phi / normal / velocity functions and defines make_plane,
 * src/collision.cpp:5-27).  A plane is the half-space
 * phi(x) = normal . (x - point) <= 0 with unit `normal`; a sphere (kind 1) is
 * the solid ball |x - point| <= param[0] with normal (x - point)/|x - point|.
 * A box (kind 2) is the solid oriented box centred at `point` with orthonormal
 * axes u = `normal`, w = `axis` and u x w, and half extents `extent` along
 * them: with l = (u.d, w.d, (u x w).d) for d = x - point and q_k = |l_k| -
 * extent[k], phi = |max(q, 0)| + min(max_k q_k, 0) (the exact signed
 * distance), and inside the box (phi <= 0, where collisions act) the normal is
 * the outward normal sign(l_k) e_k of the face k with the largest q_k (the
 * first such k on a tie, sign +1 at l_k = 0), in world axes.  Every kind moves
 * with constant `velocity` (zero for make_plane). */
typedef struct snow_collider {
  int32_t kind;
  int32_t reserved;
  double point[3];
  double normal[3];
  double velocity[3];
  double friction;
  double param[2];
  double axis[3];    /* box: second axis (unit, orthogonal to normal) */
  double extent[3];  /* box: half extents along normal, axis, normal x axis */
} snow_collider;

/* Arguments 4-12 of step() (src/grid.cpp:359). */
typedef struct snow_step_params {
  double gravity[3];
  double time_step;
  double grid_spacing;
  double mu_0;
  double lambda_0;
  double hardening_coefficient;
  double max_compression;
  double max_stretch;
  double alpha;
} snow_step_params;

/* StepTimings (include/snow/debug.hpp:3-15), milliseconds, accumulated.
 * The fused kernels report their time under the first stage they contain:
 * stencil = key/sort/block build, p2g = P2G + constitutive + force scatter,
 * grid_velocity = grid update + collisions, stress_update = elastoplastic
 * update + G2P + particle collisions + advection; the other fields stay 0. */
typedef struct snow_step_timings {
  double stencil, p2g, forces_constitutive, forces_accumulative, grid_velocity, grid_collisions,
      stress_update, g2p, particle_collisions, position_update;
} snow_step_timings;

typedef struct snow_gpu_batch snow_gpu_batch;

/* ---- process ---------------------------------------------------------- */
int snow_gpu_init(int device);
const char* snow_gpu_last_error(void);
int snow_gpu_abi_version(void);

/* make_plane (src/collision.cpp:5-27): unit normal = normal / |normal|
 * (a zero normal is kept as is), zero velocity. */
int snow_gpu_make_plane(const double point[3], const double normal[3], double friction,
                        snow_collider* out);

/* ---- batches of scenes -------------------------------------------------- */
int snow_gpu_batch_create(snow_gpu_batch** out, int precision);
int snow_gpu_batch_destroy(snow_gpu_batch* batch);

/* Adds a scene: uploads n particle records (host memory), its step
 * parameters and colliders.  The scene id is written to *scene_id. */
int snow_gpu_batch_add_scene(snow_gpu_batch* batch, const double* records, int64_t n,
                             const snow_step_params* params, const snow_collider* colliders,
                             int n_colliders, int32_t* scene_id, void* stream);
int snow_gpu_batch_remove_scene(snow_gpu_batch* batch, int32_t scene_id);
int snow_gpu_batch_set_params(snow_gpu_batch* batch, int32_t scene_id,
                              const snow_step_params* params, const snow_collider* colliders,
                              int n_colliders);
/* Replaces the particle state of a scene (same particle count). */
int snow_gpu_batch_upload(snow_gpu_batch* batch, int32_t scene_id, const double* records,
                          int64_t n, void* stream);
/* Copies a scene's particles back in their original order. */
int snow_gpu_batch_download(snow_gpu_batch* batch, int32_t scene_id, double* records, int64_t n,
                            void* stream);
/* Copies only a scene's particle positions back, x y z per particle in their
 * original order (n x 3 doubles): what a frame export (export_particles,
 * src/export.cpp:10-22) reads, an eighth of the records' bytes. */
int snow_gpu_batch_download_positions(snow_gpu_batch* batch, int32_t scene_id, double* xyz, int64_t n,
                                      void* stream);
/* A device copy of a scene's particle state (one per scene, replaced by the
 * next call), and putting it back so the scene continues from there: for
 * pre-empting or retrying served work.  No reference counterpart (the
 * reference keeps no state between steps). */
int snow_gpu_batch_snapshot(snow_gpu_batch* batch, int32_t scene_id, void* stream);
int snow_gpu_batch_restore(snow_gpu_batch* batch, int32_t scene_id, void* stream);
/* setup() for one scene: V_p0 = m_p / (sum_i m_i w_ip / dx^3) from a mass-only P2G. */
int snow_gpu_batch_setup(snow_gpu_batch* batch, int32_t scene_id, double grid_spacing,
                         void* stream);
/* Advances every scene of the batch by n_steps explicit steps (one launch per
 * stage for all scenes; replayed from a CUDA graph when timings == NULL).
 * Returns after the steps complete and reports overflow/NaN status. */
int snow_gpu_batch_step(snow_gpu_batch* batch, int n_steps, snow_step_timings* timings,
                        void* stream);
int snow_gpu_batch_scene_count(snow_gpu_batch* batch);
int64_t snow_gpu_batch_particles(snow_gpu_batch* batch);
/* Device bytes held by the batch (particles, sort, grid). */
int64_t snow_gpu_batch_device_bytes(snow_gpu_batch* batch);
/* Last status word (bit set of overflow / NaN conditions) and the grid blocks
 * used by the last step. */
int snow_gpu_batch_status(snow_gpu_batch* batch, uint32_t* status, int64_t* blocks_used,
                          int64_t* blocks_capacity);
/* Use (1) or bypass (0) CUDA-graph replay for timing-free steps. */
int snow_gpu_batch_set_graphs(snow_gpu_batch* batch, int enable);
/* Mixed form: particles whose plastic projection was redone in double in the
 * last step (a singular value within 1e-5 of a clamp bound, or a clamp acting
 * with two singular values within 1e-5 of each other).  0 for an FP64 batch. */
int64_t snow_gpu_batch_fp64_projections(snow_gpu_batch* batch);
/* Particles per P2G/G2P work item (power of two in [32, 1024]).  Until set
 * (or chosen by snow_gpu_batch_autotune) it follows the batch's particle
 * count: the largest power of two in [256, 1024] that leaves about four work
 * items per resident CTA of the particle kernels (2 per SM in FP64, 3 in the
 * mixed form). */
int snow_gpu_batch_set_chunk(snow_gpu_batch* batch, int chunk);
/* The work-item size the last step used (or will use), or SNOW_E_ARG. */
int snow_gpu_batch_chunk(snow_gpu_batch* batch);
/* Particle ordering: 1 (default) a counting sort over dense per-cell key bins
 * with direct block lookup, used while the scenes' key boxes need at most
 * 2^26 bins; 0 the radix sort with the block hash table.  Both give the same
 * step up to the order of floating-point sums.  No reference counterpart. */
int snow_gpu_batch_set_dense(snow_gpu_batch* batch, int enable);
/* Kernels launched by one replay of the batch's captured step graph (0 until
 * a step was captured: the batch's first step runs eagerly, later steps, one
 * per call or several, are captured and replayed).  No reference counterpart. */
int snow_gpu_batch_graph_kernels(snow_gpu_batch* batch);
/* Particle ordering in use: 1 counting sort over dense key bins, 0 radix sort
 * (set by set_dense, the autotuner, or the size of the key boxes).  No
 * reference counterpart. */
int snow_gpu_batch_sort_mode(snow_gpu_batch* batch);

/* Autotuner: times `trial_steps` steps of the batch for each work-item size
 * (particles per P2G/G2P CTA work item: 64 ... 1024) and each particle
 * ordering (counting sort over dense key bins, or the radix sort with the
 * block hash table, unless set_dense(0) ruled the former out) on a snapshot of
 * the current state, restores the state, keeps the fastest pair and reports
 * the size in *chosen (and its ms per step in *ms_per_step).  No reference
 * counterpart. */
int snow_gpu_batch_autotune(snow_gpu_batch* batch, int trial_steps, int* chosen, double* ms_per_step,
                            void* stream);

/* Semi-implicit velocity update (Stomakhin et al. 2013, eq. 9).  The
 * reference declares its pieces -- constitutive_differential, index_nodes,
 * deformation_differential, force_differential, apply_A and
 * Conjugate_residual (include/snow/grid.hpp:76,80,88-92) -- and defines none.
 * beta = 0 (the default) is the reference's explicit step.  With beta in
 * (0, 1], after the grid update and collisions the velocities of the nodes
 * with mass solve (I + beta dt^2 M^-1 H) v = v*, H the Hessian of the elastic
 * energy (F_P held fixed), by conjugate residuals in the mass-weighted inner
 * product until the residual falls below `tolerance` relative to v*, or
 * `max_iterations`.  Steps then run kernel by kernel (the solve reads its dot
 * products back), not from a CUDA graph. */
int snow_gpu_batch_set_implicit(snow_gpu_batch* batch, double beta, double tolerance, int max_iterations);
/* Iterations and relative residual of the last step's solve. */
int snow_gpu_batch_implicit_stats(snow_gpu_batch* batch, int* iterations, double* residual);

/* ---- serving: continuous batching of independent scenes -----------------
 * No reference counterpart.  Requests are queued with an arrival time (seconds
 * on the server's clock, which starts when run() starts; a negative arrival_s
 * stamps the request with the current time on that clock); run() admits each
 * one once it has arrived and the device-memory budget and scene slots allow,
 * runs setup() on it, advances all admitted scenes together (at most
 * max_steps_per_tick steps per tick, never past a scene's end), and retires
 * finished scenes, until every request is done or rejected (a request larger
 * than the whole budget).  Latency = completion - arrival.
 *
 * submit, result and stats may be called from any thread, also while run()
 * loops on another.  With streaming on (set_streaming(1) before or during
 * run()), run() does not return when it runs out of work but waits for more
 * submissions, until close() has been called and every request is done;
 * submit after close() fails with SNOW_E_STATE.  result() returns
 * SNOW_E_STATE until the request is complete.  Device buffers are reserved
 * when run() starts for the requests queued then, and grown between ticks,
 * with 2x headroom, when later requests need more (stats.reservations counts
 * the reservations of the last run). */
typedef struct snow_gpu_server snow_gpu_server;
typedef struct snow_server_stats {
  int64_t completed, rejected, peak_scenes, peak_bytes, ticks, particle_steps;
  double wall_s, p50_s, p99_s, mean_s, particle_steps_per_s;
  /* host wall time of the loop's phases: admission (upload + setup),
   * stepping (batched steps, including graph capture after a change of
   * membership), retirement (download + release) */
  double admit_s, step_s, retire_s;
  int64_t reservations;
} snow_server_stats;
int snow_gpu_server_create(snow_gpu_server** out, int precision, int64_t hbm_budget_bytes,
                           int max_scenes, int max_steps_per_tick);
int snow_gpu_server_destroy(snow_gpu_server* server);
int snow_gpu_server_submit(snow_gpu_server* server, const double* records, int64_t n,
                           const snow_step_params* params, const snow_collider* colliders,
                           int n_colliders, int64_t steps, double arrival_s, int64_t* request_id);
int snow_gpu_server_run(snow_gpu_server* server, void* stream);
int snow_gpu_server_result(snow_gpu_server* server, int64_t request_id, double* records, int64_t n,
                           double* latency_s);
int snow_gpu_server_stats(snow_gpu_server* server, snow_server_stats* stats);
int snow_gpu_server_set_streaming(snow_gpu_server* server, int on);
int snow_gpu_server_close(snow_gpu_server* server);
/* One tick of the last run(): host times on the server's clock (launch of the
 * tick's steps, and the moment the host saw them complete), the device span of
 * the steps (CUDA events on the run's stream, seconds after the first tick's
 * start event), steps, live scenes and particles, and the scenes admitted into
 * and retired from the live batch after it.  *count = ticks recorded; at most
 * `capacity` are copied. */
/* Particles per P2G/G2P work item of the live batch: 0 (the default) chooses
 * it in run() from the particles of all admissible requests, by the rule of
 * snow_gpu_batch_set_chunk, else a power of two in [32, 1024].  Results do not depend on it beyond the
 * order of atomic sums.  No reference counterpart. */
int snow_gpu_server_set_work_item(snow_gpu_server* server, int particles);
/* One tick of run(): host and device seconds on the server clock, steps,
 * live scenes and particles, the scenes that joined the live batch just before
 * it and those that finish with it. */
typedef struct snow_server_tick {
  double host_start_s, host_end_s, device_start_s, device_end_s;
  int64_t steps, scenes, particles, admitted, retired;
} snow_server_tick;
int snow_gpu_server_ticks(snow_gpu_server* server, snow_server_tick* out, int64_t capacity, int64_t* count);

/* ---- one scene: setup() / step() of the reference ------------------------ */
/* setup() on host records: records[i].V_p0 is overwritten. */
int snow_gpu_setup(double* records, int64_t n, double grid_spacing);
/* n_steps of step() on host records, in place (upload, steps, download).  A
 * call on as many records as the last completed call places them in the
 * block-sorted order that call's step left, so its first step reads sorted
 * particles; the results do not depend on it. */
int snow_gpu_step(double* records, int64_t n, const snow_step_params* params,
                  const snow_collider* colliders, int n_colliders, int n_steps,
                  snow_step_timings* timings);

/* Same as snow_gpu_step (FP64, host records in place) but allocates nothing:
 * for callers that cannot call cudaMalloc (a plugin inside an application that
 * owns the GPU's memory pool, or a loop that cannot afford an allocation's
 * implicit synchronisation).  No counterpart in the reference solver.  All
 * device scratch lives in one fixed file-scope device array (about 26 MB,
 * held on every GPU that loads the library until exit), which limits a call
 * to 16,384 particles, 2,048 grid blocks and 16 colliders; larger inputs
 * return SNOW_E_ARG, a scene that outgrows the blocks SNOW_E_CAPACITY; on any
 * error the records are left unchanged.  The first call on a device looks up
 * the array's address, which (with lazy module loading) is when the driver
 * reserves it; a call with n = 0 does only that set-up.  The call synchronises
 * its stream, so it must not be made while that stream is being captured.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Returns after the steps complete. */
int snow_gpu_step_noalloc(double* records, int64_t n, const snow_step_params* params,
                          const snow_collider* colliders, int n_colliders, int n_steps,
                          void* stream);

/* ---- single stages (the reference's per-stage functions) ----------------
 * Grids cross as node lists: ijk[n][3] (int32) and fields[n][10] (double) =
 * mass, momentum[3], velocity[3], force[3].  Stage entry points run the same
 * device code as the fused step.  The *_p2g and *_force entries return the
 * contributions of the particles on an empty grid: every node of the grid
 * blocks the particles' stencils touch (capacity cap_nodes; the count is
 * written to *n_nodes). */
int snow_gpu_stage_p2g(const double* records, int64_t n, double grid_spacing, int32_t* ijk,
                       double* fields, int64_t cap_nodes, int64_t* n_nodes);
int snow_gpu_stage_force(const double* records, int64_t n, double grid_spacing, double mu_0,
                         double lambda_0, double hardening_coefficient, int32_t* ijk,
                         double* fields, int64_t cap_nodes, int64_t* n_nodes);
/* The kernels' own stencil weights along one axis (the branch-free form of
 * N and N_dash, src/grid.cpp:24-58, that P2G and G2P evaluate): for each
 * coordinate x[i], base[i] = floor(x / dx) - 1 and, for the nodes base + k,
 * k = 0..3, w[4 i + k] = N(base + k, x / dx) and dw[4 i + k] =
 * N_dash(base + k, x / dx) / dx, computed on the device in double
 * (precision SNOW_FP64) or in float (SNOW_MIXED, results widened). */
int snow_gpu_stage_weights(const double* x, int64_t n, double grid_spacing, int precision, int32_t* base,
                           double* w, double* dw);
/* P2G with a caller's stencil (src/grid.cpp:119-129): for each particle and
 * each of its 64 stencil weights, the mass and momentum contributions
 * out[n][64][4] = (m w, m v w); the caller adds them to the stencil's nodes. */
int snow_gpu_stage_p2g_stencil(const double* records, int64_t n, const double* weights,
                               double* out);
/* force_constitutive (src/grid.cpp:162-172): the first Piola-Kirchhoff stress
 * P of each particle, P_out[n][9] column-major. */
int snow_gpu_stage_stress(const double* records, int64_t n, double mu_0, double lambda_0,
                          double hardening_coefficient, double* P_out);
/* force_grid_accumulation (src/grid.cpp:174-182): for each particle and each
 * of its 64 stencil entries, the force (-V_p0 P F_E^T) grad w.  P[n][9]
 * column-major, gradients[n][64][3] as build_stencil stores them; the result
 * forces[n][64][3] is added to the stencil's nodes by the caller. */
int snow_gpu_stage_force_scatter(const double* records, int64_t n, const double* P,
                                 const double* gradients, double* forces);
/* The implicit update's differentials (Stomakhin et al. 2013; declared and not
 * defined by the reference, include/snow/grid.hpp:76,88): per particle,
 * dP[n][9] = the differential of the fixed-corotated stress at F_E for
 * dF[n][9], and dF[n][9] = dt (sum_e delta_v[n][e] gradients[n][e]^T) F_E over
 * the 64 stencil entries (delta_v, gradients: [n][64][3]).  Column-major. */
int snow_gpu_stage_constitutive_differential(const double* records, int64_t n, const double* dF, double mu_0,
                                             double lambda_0, double hardening_coefficient, double* dP);
int snow_gpu_stage_deformation_differential(const double* records, int64_t n, double time_step,
                                            const double* gradients, const double* delta_v, double* dF);
/* apply_A and Conjugate_residual (declared at include/snow/grid.hpp:90-91 of
 * the reference, defined nowhere there) on a host grid: nodes ijk[n][3] and
 * fields[n][10] as above, the particles whose stencils the operator couples,
 * and the step's parameters.  The unknowns are the nodes with mass.  With q
 * (n_nodes x 3): out = A q = q - beta dt delta f(q) / m at nodes with mass and
 * q elsewhere.  With q NULL: out = the solution of A v = velocity by conjugate
 * residuals in the mass-weighted inner product, from v = velocity, until
 * <r, r>_M <= squared_tolerance <velocity, velocity>_M or max_iterations
 * (*iterations gets the count); massless nodes keep their velocity. */
int snow_gpu_stage_implicit(const int32_t* ijk, const double* fields, int64_t n_nodes,
                            const double* records, int64_t n, double grid_spacing, double time_step,
                            double mu_0, double lambda_0, double hardening_coefficient, double beta,
                            double squared_tolerance, int max_iterations, const double* q, double* out,
                            int* iterations);
int snow_gpu_stage_grid_velocity(double* fields, int64_t n_nodes, const double gravity[3],
                                 double time_step);
int snow_gpu_stage_grid_collisions(const int32_t* ijk, double* fields, int64_t n_nodes,
                                   const snow_collider* colliders, int n_colliders,
                                   double grid_spacing);
/* calculate_volume / stress_update / G2P of particles against a given grid. */
int snow_gpu_stage_volume(const int32_t* ijk, const double* fields, int64_t n_nodes,
                          double* records, int64_t n, double grid_spacing);
int snow_gpu_stage_stress_update(const int32_t* ijk, const double* fields, int64_t n_nodes,
                                 double* records, int64_t n, double grid_spacing,
                                 double time_step, double max_compression, double max_stretch);
int snow_gpu_stage_g2p(const int32_t* ijk, const double* fields, int64_t n_nodes,
                       double* records, int64_t n, double grid_spacing, double alpha);
int snow_gpu_stage_particle_collisions(double* records, int64_t n,
                                       const snow_collider* colliders, int n_colliders);
int snow_gpu_stage_position_update(double* records, int64_t n, double time_step);

/* ---- measured arithmetic peaks (roofline denominators) ------------------
 * No counterpart in the reference.  Runs a fused multiply-add loop on every SM
 * of the current device for at least 20 ms at the clocks the GPU runs (no clock
 * or power setting is changed) and returns the sustained rate in FLOP/s (two
 * per FMA): kind SNOW_PEAK_FP64 (double FMA), SNOW_PEAK_FP32 (float FMA) or
 * SNOW_PEAK_FP32X2 (packed two-wide float FMA).  *ms (optional) receives the
 * timed run's duration.  The roofline of the particle kernels, which do 3x3
 * algebra and stencil sums, is the larger of their HBM and FMA-pipe fractions. */
enum { SNOW_PEAK_FP64 = 0, SNOW_PEAK_FP32 = 1, SNOW_PEAK_FP32X2 = 2 };
int snow_gpu_measure_fma_peak(int kind, double* flops_per_s, double* ms, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SNOW_GPU_H */
