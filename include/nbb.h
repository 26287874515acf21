/*
 * nbb.h -- C ABI of the B200-native Barnes-Hut step (libnbb.so).
 *
 * The entry points replace the public interface of sytrams/AMSC-Nbody's
 * hot path; each cites the reference interface it stands in for (paths
 * relative to that project's root).  Plain C types only: sizes, status codes
 * and raw host or device pointers.  A header-only C++ layer with the
 * reference's own class and function names sits on top of this ABI
 * (amsc-nbody_b200/cpp/nbb_simulation.hpp).
 *
 * Status convention: every function returns an nbb_status; on failure
 * nbb_last_error_message() describes the error in the words the reference
 * would have thrown with, and nbb_last_error_code() carries the stage/device
 * code.  A simulation handle that reported an error other than
 * NBB_ERR_INVALID_ARGUMENT / NBB_ERR_LOGIC on a step is unusable afterwards,
 * as the reference's Simulation enters State::failed
 * (src/simulation.cpp:100-119).
 *
 * Threading: a handle is not thread-safe; distinct handles are independent.
 */
#ifndef NBB_H
#define NBB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBB_API_VERSION 1

typedef enum {
  NBB_OK = 0,
  NBB_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
  NBB_ERR_DOMAIN = 2,           /* reference: std::domain_error (non-finite) */
  NBB_ERR_LOGIC = 3,            /* reference: std::logic_error (call order) */
  NBB_ERR_CUDA = 4,             /* CUDA runtime failure (runtime_error) */
  NBB_ERR_DEVICE = 5,           /* device stage error code (runtime_error) */
  NBB_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up */
  NBB_ERR_OVERFLOW = 7,         /* reference: std::overflow_error */
  NBB_ERR_NO_DEVICE = 8         /* no CUDA device / kernel image */
} nbb_status;

/* Traversal arithmetic.  FP64 is the reference's plain form
 * (gpu/cuda_kernels/barnes_hut.cu:164-322): per-target acceptance test and
 * interaction sets, FP64 throughout.  MIXED evaluates the interaction bulk in
 * FP32 (offsets formed in FP64 and rounded, rsqrtf + one Newton step,
 * Kahan-compensated partial sums) over interaction lists shared by a warp
 * group of Morton-consecutive targets whose acceptance test is the
 * reference's d > s/theta + delta measured from the group's bounding box. */
typedef enum { NBB_PRECISION_FP64 = 0, NBB_PRECISION_MIXED = 1 } nbb_precision;

/* SimulationConfig{timeStep, theta, softening} (src/simulation.hpp:18-22)
 * plus BarnesHutParameters::gravitationalConstant (src/barnes_hut.hpp:8-13),
 * which the reference's Simulation fixes to the SI value. */
typedef struct {
  double time_step;
  double theta;
  double softening;
  double gravitational_constant;
  int precision;  /* nbb_precision */
  int group_size; /* MIXED: targets per warp group, 32/64/128; 0 = tuned */
  int use_graph;  /* capture each step into a CUDA graph (default 1) */
  int device;     /* CUDA device ordinal (default 0) */
  int cache_depth; /* MIXED: tree levels below the root staged in shared memory
                      per block: -1 = tuned (default), 0, 1 or 2 */
} nbb_config;

/* Defaults of BarnesHutParameters (theta 0.5, softening 1e-6, G = SI);
 * time_step 0 must be set by the caller. */
void nbb_config_default(nbb_config *cfg);

typedef struct nbb_sim nbb_sim;

/* Simulation(Particles, SimulationConfig) (src/simulation.cpp:70-74):
 * validates the configuration and copies the planar state in (host pointers
 * when on_device == 0, device pointers otherwise).  type may be NULL. */
int nbb_sim_create(const nbb_config *cfg, size_t n, const double *mass,
                   const double *x, const double *y, const double *z,
                   const double *vx, const double *vy, const double *vz,
                   const uint8_t *type, int on_device, nbb_sim **out);

/* No counterpart in the reference (it steps one system per Simulation):
 * n_systems independent systems stored back to back -- system k owns
 * particles [offsets[k], offsets[k+1]) -- advanced together, one launch per
 * stage.  Each system has its own bounding box, Morton keys, octree and
 * softening (softening[k]; NULL uses cfg->softening), and never feels the
 * others: its result equals stepping it alone.  At most 512 systems and
 * 2^25 particles.  The handle accepts every nbb_sim_* call. */
int nbb_ensemble_create(const nbb_config *cfg, int n_systems,
                        const int64_t *offsets, const double *softening,
                        const double *mass, const double *x, const double *y,
                        const double *z, const double *vx, const double *vy,
                        const double *vz, int on_device, nbb_sim **out);

/* Simulation::initialize (src/simulation.cpp:78-98): first spatial build
 * and acceleration; NBB_ERR_LOGIC when called twice. */
int nbb_sim_initialize(nbb_sim *sim);

/* Simulation::step / run (src/simulation.cpp:100-127): KD, rebuild, force,
 * K.  No host synchronisation inside a step; the call synchronises once at
 * its end to report device errors. */
int nbb_sim_step(nbb_sim *sim);
int nbb_sim_run(nbb_sim *sim, uint64_t steps);

/* Simulation::time / stepNumber (src/simulation.cpp:129-131) */
double nbb_sim_time(const nbb_sim *sim);
uint64_t nbb_sim_step_number(const nbb_sim *sim);

/* Simulation::particles() -> DeviceParticlesView (src/particle.hpp:85-96):
 * non-owning device pointers, valid until nbb_sim_destroy.  ax/ay/az hold
 * the acceleration of the current state. */
typedef struct {
  size_t count;
  double *mass, *x, *y, *z, *vx, *vy, *vz;
  uint8_t *type;
  double *ax, *ay, *az;
} nbb_state_view;
int nbb_sim_state(nbb_sim *sim, nbb_state_view *view);

/* Host <-> device state transfer (positions and velocities; mass too on
 * upload when mass != NULL).  Pinned host memory gives asynchronous copies
 * on the simulation stream; the call returns after the copy is enqueued
 * (upload) or complete (download). */
int nbb_sim_upload(nbb_sim *sim, const double *mass, const double *x,
                   const double *y, const double *z, const double *vx,
                   const double *vy, const double *vz);
int nbb_sim_download(nbb_sim *sim, double *x, double *y, double *z,
                     double *vx, double *vy, double *vz);
/* Accelerations of the current state to host memory. */
int nbb_sim_download_accel(nbb_sim *sim, double *ax, double *ay, double *az);

/* One step with the state in host memory: nbb_sim_upload + nbb_sim_step +
 * nbb_sim_download in one call, with the same result bit for bit.  The
 * reference copies host buffers to the device only when it loads particles
 * (thrust::copy per block, src/particle.hpp:172-192) and hands out device
 * views after that (Simulation::particles, src/simulation.cpp:133-134);
 * this call serves a host that owns the state between steps.  Any input may
 * be NULL (that array is not uploaded), and so may any output.  The masses
 * are first read after the sort, so their upload overlaps the kick-drift
 * and the sort on a second stream; the positions are final after the drift,
 * so their copy to the host overlaps the rebuild and the walk; the
 * velocities follow the closing kick.  Returns when every copy is
 * complete. */
int nbb_sim_step_host(nbb_sim *sim, const double *mass, const double *x,
                      const double *y, const double *z, const double *vx,
                      const double *vy, const double *vz, double *out_x,
                      double *out_y, double *out_z, double *out_vx,
                      double *out_vy, double *out_vz);

/* Stream control: all work of the handle goes to this stream (a
 * cudaStream_t; NULL = the handle's own stream). */
int nbb_sim_set_stream(nbb_sim *sim, void *stream);
int nbb_sim_synchronize(nbb_sim *sim);
int nbb_sim_destroy(nbb_sim *sim);

/* Counters of the last force evaluation. */
typedef struct {
  int n_groups;         /* unique Morton keys G */
  int n_octree_nodes;   /* M */
  int64_t interactions; /* monopole + leaf-pair interactions evaluated */
  int64_t mac_tests;    /* acceptance tests evaluated */
  int group_size;       /* MIXED: warp target group size in use (32, 64 or 128) */
  int64_t stack_overflow; /* MIXED: nodes accepted because the walk's stack was
                             full (their children would not fit).  The stack's
                             global extension is sized for any walk, so this is
                             0; a nonzero count also fails the call or step with
                             NBB_ERR_DEVICE */
  int cache_depth;      /* MIXED: tree levels below the root the walk stages in
                           shared memory per block (0, 1 or 2; autotuned) */
} nbb_stats;
int nbb_sim_stats(nbb_sim *sim, nbb_stats *stats);

/* Diagnostic: recompute the force of the current state (no kick, no drift,
 * state unchanged) outside the step graph, with CUDA events between the
 * stages.  stage_ms receives NBB_PROFILE_STAGES durations in milliseconds:
 * reset, bounding box, Morton + sort + groups, tree build, traversal. */
#define NBB_PROFILE_STAGES 5
int nbb_sim_profile(nbb_sim *sim, float *stage_ms, nbb_stats *stats);

/* Every intermediate of the last spatial build, for bit-exact comparison
 * with the reference's MortonKeys / MortonLeafGroups / Tree /
 * RadixToOctreePlan / Octree structures.  The caller provides host buffers
 * (any may be NULL) with capacities: n for keys/idx/groups, n-1 for radix
 * internal arrays, 2n-1 for radix-node arrays, m_capacity octree nodes
 * (children 8*m_capacity).  Sizes are returned in n_groups / n_octree. */
typedef struct {
  double box[4];                                  /* Bbox centre + side */
  uint32_t *keys, *idx;                           /* MortonKeys */
  uint32_t *uniq;                                 /* MortonLeafGroups */
  int *gfirst, *gcount;
  int *left, *right, *rfirst, *rlast, *plen;      /* Tree (G-1) */
  int *rparent;                                   /* Tree (2G-1) */
  int *plan_level, *plan_count, *plan_offset;     /* RadixToOctreePlan */
  int m_capacity;
  int *children, *oparent, *olevel;               /* Octree topology */
  uint32_t *oprefix;
  int *ofirst, *ocount, *child_count;
  double *cx, *cy, *cz, *half;                    /* Octree geometry */
  double *mass, *comx, *comy, *comz;              /* Octree physics */
  int n_groups, n_octree;
} nbb_tree_export;
int nbb_sim_export(nbb_sim *sim, nbb_tree_export *out);

/* ---------------------------------------------------- function level ---- */

/* One spatial build + Barnes-Hut evaluation on caller particles, the
 * sequence Bbox -> MortonKeys -> allocate/build{MortonLeafGroups, Tree,
 * RadixToOctreePlan, Octree, geometry, physics} ->
 * computeBarnesHutAcceleration (src/simulation.cpp:137-198,
 * gpu/cuda_kernels/barnes_hut.cu:325-391).  Accelerations are written at the
 * original particle index.  Pointers are host (on_device == 0) or device.
 * export_out and stats may be NULL. */
int nbb_accel(size_t n, const double *mass, const double *x, const double *y,
              const double *z, double theta, double softening, double g,
              int precision, double *ax, double *ay, double *az,
              int on_device, nbb_tree_export *export_out, nbb_stats *stats);

/* FP64 direct summation (the theta-error oracle of
 * tests/integration/cuda/barnes_hut_accuracy_test.cu:101-172) for the
 * n_targets particle indices in targets (NULL: all n).  Output k belongs to
 * targets[k]. */
int nbb_accel_direct(size_t n, const double *mass, const double *x,
                     const double *y, const double *z, int n_targets,
                     const int *targets, double g, double softening,
                     double *ax, double *ay, double *az, int on_device);

/* computeBarnesHutAcceleration on a caller-built octree
 * (gpu/cuda_kernels/barnes_hut.cu:325-391), FP64 plain form.  Octree arrays
 * follow src/octree_types.hpp:73-104 (children node-major, 8 per node; root
 * 0).  particle_order: 0 = original, 1 = morton (BarnesHutParticleOrder). */
typedef struct {
  int n_nodes, n_particles;
  const int *children, *parent, *first, *count;
  const double *mass, *comx, *comy, *comz;
  const double *cx, *cy, *cz, *half;
} nbb_octree_view;
int nbb_accel_octree(const nbb_octree_view *octree, const uint32_t *idx,
                     const double *mass, const double *x, const double *y,
                     const double *z, double *ax, double *ay, double *az,
                     double theta, double softening, double g,
                     int particle_order, int on_device);

/* leapfrogKickDrift / leapfrogKick (src/integrator.hpp:5-7).  Pointers are
 * device pointers, as in the reference; dt must be finite and positive. */
int nbb_kick_drift(double *x, double *y, double *z, double *vx, double *vy,
                   double *vz, const double *ax, const double *ay,
                   const double *az, size_t n, double dt, void *stream);
int nbb_kick(double *vx, double *vy, double *vz, const double *ax,
             const double *ay, const double *az, size_t n, double dt,
             void *stream);

/* buildMortonLeafGroups -> buildTreeFromMortonGroups ->
 * buildRadixToOctreePlan -> buildSparseOctreeTopology on caller sorted keys
 * (src/morton_leaf_groups.hpp:43-47, src/tree_builder.hpp:5-13,
 * src/radix_to_octree.hpp:67-70, src/octree_builder.hpp:7-11).  Host
 * pointers; outputs into out (geometry/physics fields are left untouched). */
int nbb_octree_from_keys(const uint32_t *sorted_keys, int n,
                         nbb_tree_export *out);

/* buildTree on caller keys (src/tree_builder.hpp:9), any 32-bit keys,
 * duplicates allowed.  Host pointers; left..plen n-1 entries, parent 2n-1. */
int nbb_radix_tree(const uint32_t *keys, int n, int *left, int *right,
                   int *rfirst, int *rlast, int *plen, int *parent);

/* ----------------------------------------- function-level build stages ----
 * One entry point per build function of the reference, on caller DEVICE
 * arrays laid out as the reference's structures (src/morton.hpp,
 * src/morton_leaf_groups.hpp:8-41, src/tree_types.hpp:48-109,
 * src/radix_to_octree.hpp:31-65, src/octree_types.hpp:73-178).  Each call is
 * synchronous on the default stream, as the reference's are, and reports the
 * reference's errors (messages and exception classes of the same stage). */

/* Bbox::compute_box (gpu/cuda_kernels/globalbounding.cu:94-144): box receives
 * {centre x, y, z, side} in device memory. */
int nbb_bbox(const double *x, const double *y, const double *z, size_t n,
             double *box);

/* MortonKeys::build (gpu/cuda_kernels/morton.cu:160-225): keys of the
 * positions against the device box and their stable ascending sort with the
 * particle indices. */
int nbb_morton_keys(const double *x, const double *y, const double *z,
                    size_t n, const double *box, uint32_t *keys,
                    uint32_t *idx);

/* buildMortonLeafGroups (gpu/cuda_kernels/morton_leaf_groups.cu:58-103):
 * unique keys, first sorted index and size of every run of equal keys;
 * *n_groups (host) receives G. */
int nbb_leaf_groups(const uint32_t *sorted_keys, int n, uint32_t *unique_keys,
                    int *first, int *count, int *n_groups);

/* buildTree (gpu/cuda_kernels/tree_builder.cu:303-352) on device keys:
 * left..plen n-1 entries (NULL allowed for n = 1), parent 2n-1. */
int nbb_radix_tree_device(const uint32_t *keys, int n, int *left, int *right,
                          int *rfirst, int *rlast, int *plen, int *parent);

/* buildRadixToOctreePlan (gpu/cuda_kernels/radix_to_octree.cu:174-244) for a
 * tree over n_groups unique keys: level, count and offset per radix node
 * (2 n_groups - 1); *n_octree_nodes (host) receives M. */
int nbb_octree_plan(const uint32_t *unique_keys, int n_groups, const int *plen,
                    const int *parent, int *level, int *count, int *offset,
                    int *n_octree_nodes);

/* buildSparseOctreeTopology (gpu/cuda_kernels/octree_builder.cu:254-362):
 * the M-node octree of a radix tree, its leaf groups and plan. */
int nbb_octree_topology(const uint32_t *unique_keys, const int *group_first,
                        const int *group_count, int n_groups,
                        const int *rfirst, const int *parent,
                        const int *plan_level, const int *plan_count,
                        const int *plan_offset, int n_nodes, int *children,
                        int *octree_parent, int *octree_level,
                        uint32_t *octree_prefix, int *first, int *count);

/* computeOctreeGeometry (gpu/cuda_kernels/octree_geometry.cu:137-173): cell
 * centre and half size of every node from its level and Morton prefix and
 * the device box. */
int nbb_octree_geometry(int n_nodes, const int *level, const uint32_t *prefix,
                        const double *box, double *cx, double *cy, double *cz,
                        double *half);

/* computeOctreeMassAndCenterOfMass (gpu/cuda_kernels/octree_physics.cu:
 * 283-337): child counts, and mass and centre of mass of every node -- leaves
 * over their particles in sorted order, internal nodes over their children in
 * octant order -- for n_particles particles reached through sorted_indices. */
int nbb_octree_mass(int n_nodes, int n_particles, const int *children,
                    const int *level, const int *first, const int *count,
                    const uint32_t *sorted_indices, const double *mass,
                    const double *x, const double *y, const double *z,
                    int *child_count, double *node_mass, double *comx,
                    double *comy, double *comz);

/* Device memory for the C++ layer's buffers (cudaMalloc / cudaFree /
 * cudaMemcpy; kind 0 host to device, 1 device to host, 2 device to device). */
int nbb_device_alloc(void **ptr, size_t bytes);
int nbb_device_free(void *ptr);
int nbb_memcpy(void *dst, const void *src, size_t bytes, int kind);

/* Diagnostic: measured SIMT FMA throughput of the current device in TFLOP/s
 * (precision NBB_PRECISION_FP64, NBB_PRECISION_MIXED = scalar FP32, or 2 =
 * packed two-wide FP32), the roofline denominators of the traversal kernels. */
int nbb_measure_fma_tflops(int precision, double *tflops);

/* ------------------------------------------------- allocation-free ---- */

/* No counterpart in the reference.  Bounding box, Morton keys and their
 * stable sorted permutation (the MortonKeys result) for callers that cannot
 * allocate device memory: a host that owns all device memory through its own
 * pool or budget and forbids libraries to call cudaMalloc/cudaFree.  This call
 * allocates nothing: its scratch is one file-scope device array sized for
 * NBB_NOALLOC_MAX_PARTICLES particles (about 4.3 MB), held by every GPU that
 * loads the library's device code until the process exits (with lazy module
 * loading, CUDA's default, it is placed when the module loads, at the first
 * call of the library on that device).  x, y, z, keys and idx are device
 * pointers of n elements; larger n is rejected with
 * NBB_ERR_INVALID_ARGUMENT.  Every call looks up the array's device address
 * in the current context (cudaGetSymbolAddress; nothing is cached, so a reset
 * device or another context is served by its own copy).  The call reads its
 * error word back and synchronises the given stream before it returns, so it
 * cannot be captured in a CUDA graph: on a capturing stream it returns
 * NBB_ERR_INVALID_ARGUMENT without touching the capture.  Every call shares
 * the array: calls that overlap on the GPU (other streams, other threads)
 * race and give wrong results.  Its errors are reported by
 * nbb_noalloc_last_error_message(). */
#define NBB_NOALLOC_MAX_PARTICLES (1 << 18)
int nbb_morton_sort_noalloc(const double *x, const double *y, const double *z,
                            size_t n, uint32_t *keys, uint32_t *idx,
                            void *stream);
const char *nbb_noalloc_last_error_message(void);

/* Self-test of failure detection: runs a device look-back whose predecessor
 * never publishes.  The bounded spin gives up (about a second) and the call
 * returns NBB_ERR_TIMEOUT with the CUDA context intact; any other status is a
 * failure of the detection itself. */
int nbb_selftest_bounded_wait(void);

/* ---------------------------------------------------------------------------
 * Frame capture (src/streaming/device_capture.hpp:12-35 DeviceFrameWriter and
 * src/streaming/frame.cpp:341-470 writeQuantizedPositions): a quantized
 * snapshot of the current positions as one byte buffer in the reference's
 * version-3 frame layout -- 128-byte little-endian header ("NBSNAP01",
 * version, header size, sequence, step, time, source and sample counts,
 * scalar bytes 2, components 3, payload bytes, bounds min/max, type bytes),
 * then 3 x uint16 per sample, then one uint8 particle type per sample (0 when
 * the simulation has no types).  max_particles 0 (or >= count) samples every
 * particle, otherwise sample i is particle (i * count) / max_particles.
 * nbb_frame_bytes gives the buffer size needed.  Errors as the reference:
 * NBB_ERR_DOMAIN for a non-finite sampled position, NBB_ERR_INVALID_ARGUMENT
 * for an invalid type or a buffer that is too small.  The frame is built on
 * the device; `out` is host memory unless on_device. */
size_t nbb_frame_bytes(const nbb_sim *sim, size_t max_particles);
int nbb_sim_capture_frame(nbb_sim *sim, size_t max_particles, uint64_t sequence, void *out, size_t capacity,
                          size_t *written, int on_device);

/* ---------------------------------------------------------------------------
 * Conserved-quantity monitor (the reference lists total energy, linear and
 * angular momentum monitoring as planned work, README.md:766-774): sums over
 * the current state, each in a fixed order (repeatable bit for bit).  The
 * potential energy 1/2 sum m_i phi_i is optional: NBB_POTENTIAL_TREE
 * evaluates phi with the Barnes-Hut acceptance test of the plain form on a
 * tree rebuilt at the current positions (the cost of one FP64 force
 * evaluation), NBB_POTENTIAL_DIRECT by all pairs (O(N^2); not for
 * ensembles).  For an ensemble the sums run over all systems. */
enum { NBB_POTENTIAL_NONE = 0, NBB_POTENTIAL_TREE = 1, NBB_POTENTIAL_DIRECT = 2 };
typedef struct nbb_diagnostics {
  double mass;
  double center_of_mass[3];
  double momentum[3];          /* sum m v */
  double angular_momentum[3];  /* sum m x cross v, about the origin */
  double kinetic_energy;       /* sum 1/2 m |v|^2 */
  double potential_energy;     /* 0 unless requested */
  double total_energy;
  int potential;               /* the mode used */
} nbb_diagnostics;
int nbb_sim_diagnostics(nbb_sim *sim, int potential, nbb_diagnostics *out);

/* ---------------------------------------------------------------------------
 * Differentiable rollout.  No counterpart in the reference (which has no
 * derivative of its step); the force differentiated is the plain FP64
 * Barnes-Hut force of gpu/cuda_kernels/barnes_hut.cu:164-322 with the tree
 * topology and every target's accepted-node and opened-leaf sets held fixed
 * at the positions of each step.
 *
 * nbb_sim_rollout advances an initialized simulation by `steps` steps (as
 * nbb_sim_run) and keeps (x, v, a) every `checkpoint_every` steps on the
 * device.  nbb_sim_backward then returns the gradient of a scalar loss of the
 * final state with respect to the rollout's initial masses, positions and
 * velocities, given dL/d(final positions) and, optionally (all three or none),
 * dL/d(final velocities).  It recomputes each checkpoint segment forward with
 * the handle's own step (so a mixed-precision rollout is differentiated along
 * its own trajectory), rebuilds the tree at every stored position and applies
 * the hand-written vector-Jacobian product of the force and of the leapfrog
 * kick-drift-kick.  The handle's state is restored to the rollout's final
 * state before returning.  Output pointers may be null (not copied); on_device
 * says whether every array argument is a device pointer.
 * ------------------------------------------------------------------------- */
int nbb_sim_rollout(nbb_sim *sim, uint64_t steps, uint64_t checkpoint_every);
int nbb_sim_backward(nbb_sim *sim, const double *gx, const double *gy, const double *gz, const double *gvx,
                     const double *gvy, const double *gvz, double *gm, double *gx0, double *gy0, double *gz0,
                     double *gvx0, double *gvy0, double *gvz0, int on_device);

/* Frozen-structure replay, for finite differences of the differentiated
 * function: the unperturbed system (m, x, y, z, vx, vy, vz; FP64 plain
 * stepping) advances `steps` steps, and alongside it `copies` perturbed
 * copies (copy q at offset q*n of each c* array; cmass may be null for the
 * unperturbed masses) advance with forces evaluated on the unperturbed
 * system's tree, acceptance decisions and leaf sets of the same step.  Writes
 * each copy's final positions / velocities at offset q*n. */
int nbb_frozen_rollout(const nbb_config *cfg, size_t n, const double *mass, const double *x, const double *y,
                       const double *z, const double *vx, const double *vy, const double *vz, size_t copies,
                       const double *cmass, const double *cx, const double *cy, const double *cz,
                       const double *cvx, const double *cvy, const double *cvz, uint64_t steps, double *ox,
                       double *oy, double *oz, double *ovx, double *ovy, double *ovz, int on_device);

/* FP64 direct-summation rollout and its adjoint (the theta-error oracle of
 * the tree adjoint): `steps` leapfrog steps with all-pairs forces (softening
 * and G from cfg; theta, precision and group size ignored), final state into
 * o* (each may be null), and the gradient with respect to the initial state
 * for the final-state cotangents, as nbb_sim_backward.  Stores every step's
 * positions (refused above 16 GiB). */
int nbb_direct_rollout_adjoint(const nbb_config *cfg, size_t n, const double *mass, const double *x,
                               const double *y, const double *z, const double *vx, const double *vy,
                               const double *vz, uint64_t steps, const double *gx, const double *gy,
                               const double *gz, const double *gvx, const double *gvy, const double *gvz,
                               double *ox, double *oy, double *oz, double *ovx, double *ovy, double *ovz,
                               double *gm, double *gx0, double *gy0, double *gz0, double *gvx0, double *gvy0,
                               double *gvz0, int on_device);

/* Last error of the calling thread. */
const char *nbb_last_error_message(void);
int nbb_last_error_code(void);

/* Number of kernels this library launched in the calling process. */
uint64_t nbb_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
