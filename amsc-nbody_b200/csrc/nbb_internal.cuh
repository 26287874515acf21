// nbb_internal.cuh -- device workspace, error words and small device helpers
// shared by the build, traversal and C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace nbb {

// src/radix_to_octree.hpp:10-19
constexpr int kDims = 3;
constexpr int kSpatialBits = 30;
constexpr int kPaddingBits = 2;
constexpr int kMaxLevel = 10;
constexpr uint32_t kSpatialMask = 0x3FFFFFFFu;

// Device error word: stage * 100 + code.  Codes 1..8 are the reference's own
// device error codes of that stage; the rest are this library's.
enum Stage : int {
  kStageBbox = 1,       // code 1 non-finite position, 2 invalid box
  kStageSort = 2,       // code 99 bounded look-back wait gave up
  kStageGroups = 3,     // code 99 bounded look-back wait gave up
  kStagePlan = 4,       // radix_to_octree.cu:32-51 codes 1..4; 90 overflow
  kStageOctree = 5,     // octree_builder.cu:18-46 codes 1..7
  kStageGeometry = 6,   // octree_geometry.cu:21-34 codes 1..2
  kStagePhysics = 7,    // octree_physics.cu:18-46 codes 1..7
  kStageTraversal = 8,  // barnes_hut.cu:21-52 codes 1..8
  kStageLayout = 9      // code 1 inconsistent preorder walk
};
constexpr int kCodeTimeout = 99;
constexpr int kCodeOverflow = 90;

// Per-workspace device scalars; one block reset at the start of each step.
struct DevScalars {
  unsigned long long bb_min[3];  // order-preserving encoded extrema
  unsigned long long bb_max[3];
  double box[4];                 // centre x, y, z, side (Bbox layout)
  int nonfinite;
  int n_groups;                  // G
  int n_nodes;                   // M
  int error;                     // sticky first error (not reset per step)
  unsigned int ticket_bbox;
  unsigned int ticket_encode;
  unsigned int tile_counter[9];  // dynamic tile ids: sort passes, then scans
  unsigned int work_counter;     // traversal work queue
  int n_tgroups;                 // traversal target groups
  unsigned int stack_overflow;   // mixed traversal nodes accepted on overflow
  unsigned long long interactions;
  unsigned long long mac_tests;
  int level_count[16];           // octree nodes per level (kMaxLevels)
  int level_base[18];            // level-order index of each level's first node (kMaxLevels + 2)
};

// Sort tiling (onesweep LSD radix sort of packed (key << 32 | index)).
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 pairs
constexpr int kSortPasses = 4;     // 8-bit digits over a single system's 30-bit keys
constexpr int kMaxSortPasses = 5;  // ensemble keys: up to 9 system bits + 30 Morton bits
constexpr int kMaxLevels = 16;     // octree levels: 10 spatial + up to 3 above the system roots

// Largest target group supported (two targets per lane of a warp).
constexpr int kGroupMaxLimit = 128;
// Shallowest cell depth (below the system's root) whose particles may form
// one target group; a group spanning a larger cell has a box so wide that its
// walk opens most of the tree (sparse outskirts).
#ifndef NBB_GROUP_DEPTH
#define NBB_GROUP_DEPTH 3
#endif
constexpr int kGroupDepth = NBB_GROUP_DEPTH;
// Largest ensemble: 3 octree levels of system id.
constexpr int kMaxSystems = 512;

// Dynamic tile-id counters (DevScalars::tile_counter): one per sort pass,
// then one per single-pass scan kernel.
constexpr int kTileGroups = kMaxSortPasses;      // 5
constexpr int kTilePlan = kMaxSortPasses + 1;    // 6
constexpr int kTileTargetGroups = kMaxSortPasses + 2;  // 7
constexpr int kTileEnds = kMaxSortPasses + 3;          // 8
constexpr int kTileCounters = kMaxSortPasses + 4;      // 9

// Single-pass scan tiling.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// The mixed walk's record of one node (48 bytes, two 32-byte sectors):
// centre of mass and mass, the squared acceptance radius for a target box
// rounded up to FP32, and the node's particle range and child count.
struct __align__(16) MixedNode {
  double4 a;   // com x, y, z, mass
  float cr2;   // (max(crit, sqrt(3) h + |com - centre|) (1 + 2^-40))^2 (1 + 2^-18), rounded up
  int first;   // first particle of an occupied leaf, -1 otherwise
  int count;   // particles of an occupied leaf, 0 otherwise
  int nchild;  // children
};
static_assert(sizeof(MixedNode) == 48, "two 32-byte sectors per node");

// A node of the level-order octree (the step's build): the same octree as
// the reference's, numbered level by level with each level in ascending key
// order, so that a node's children are consecutive entries of the next level.
struct __align__(16) LevelNode {
  double4 a;  // com x, y, z, mass
  int pre;    // depth-first preorder index (children visited octant 7 -> 0)
  int np;     // particles in the subtree
  int first;  // first particle of the subtree (sorted order)
  int leaf;   // 1 for an occupied leaf
};
static_assert(sizeof(LevelNode) == 48, "two 32-byte sectors per node");

// The top levels of the level-order octree (levels 0..kTopDepth: at most
// 1 + 8 + 64 cells, in level order), the table the mixed walk's shared-memory
// node cache is loaded from: each cell's record, its children's preorder
// indices (visit order) and, for a cell whose children are cached too, their
// place in the table (first child, count).
constexpr int kTopDepth = 2;
constexpr int kTopMax = 73;
struct __align__(16) TopNode {
  MixedNode rec;
  int kids[8];
  int first_child;  // level-order index of the first child
  int nchild;
  int level;
  int pad;
};
static_assert(sizeof(TopNode) == 96, "record, child list, child range");

// Per-tile counts of the level-order build (tiles of kScanTile groups): the
// cells started per octree level, then the cells ended (kMaxLevels); the
// rest pad a warp.
constexpr int kLevelOrderChannels = 32;

// Traversal records a build writes: the plain FP64 walk's (node_a, node_b,
// node_c, node_meta) and the mixed walk's (node_m); child lists always.
constexpr int kRecordsFp64 = 1;
constexpr int kRecordsMixed = 2;

// Everything a spatial rebuild and a traversal touch, sized for capacity n.
struct Workspace {
  int n = 0;            // particle count
  int cap_nodes = 0;    // octree node capacity (sum over levels of min(8^L, n))
  int num_sms = 0;
  int fp64_grid = 0;    // persistent traversal grids (blocks)
  int mixed_grid[2][3] = {{0, 0, 0}, {0, 0, 0}};  // [track source][1, 2 or 4 targets per lane]
  int vjp_grid = 0;     // the mixed walk's adjoint form
  int walk_warps = 0;     // warps of the largest mixed-walk grid
  int walk_ext_cap = 0;   // entries per warp of the mixed walk's stack extension
  int group_max = 32;   // largest octree target group: 32, 64 or 128 (32 x target slots per lane)
  int group_depth = kGroupDepth;  // shallowest cell (levels below its system's root) a group may span

  // key layout: an ensemble's system id sits above the 30 Morton bits and
  // adds sys_levels octree levels above the system roots
  int n_systems = 1;
  int sys_levels = 0;    // ceil(log8(n_systems)), at most 3
  int key_bits = 30;     // 30 + 3 * sys_levels
  int max_level = 10;    // key_bits / 3
  int pack_shift = 34;   // sort pairs: key << pack_shift | particle index
  int sort_passes = 4;   // ceil(key_bits / 8)

  // particle state, original order (SoA, FP64)
  double *m = nullptr, *x = nullptr, *y = nullptr, *z = nullptr;
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *ax = nullptr, *ay = nullptr, *az = nullptr;
  uint8_t *type = nullptr;
  int *sys_of = nullptr;       // ensemble: system of each particle (original order)

  DevScalars *sc = nullptr;
  unsigned long long *sys_bb = nullptr;  // 6 per system: encoded min xyz, max xyz
  double *sys_box = nullptr;             // 4 per system: centre xyz, side
  double *sys_eps = nullptr;             // ensemble: softening per system
  int *root_pre = nullptr;               // preorder index of each system's root

  // sort
  unsigned long long *pairs_a = nullptr, *pairs_b = nullptr;  // n each
  uint32_t *digit_hist = nullptr;    // kSortPasses * 256 (counts -> offsets)
  uint32_t *sort_status = nullptr;   // kSortPasses * tiles * 256
  int sort_tiles = 0;
  unsigned long long *scan_status = nullptr;  // scan tiles: groups, plan, target groups
  int scan_tiles_n = 0;   // tiles over n
  int scan_tiles_r = 0;   // tiles over 2n-1

  // Morton keys / permutation (reference MortonKeys layout; keys hold the low
  // 32 bits of the full key)
  uint32_t *keys = nullptr, *idx = nullptr;
  int *psys = nullptr;     // system of each sorted particle
  double4 *pm4 = nullptr;  // Morton-ordered particles {x, y, z, m}

  // leaf groups (MortonLeafGroups)
  unsigned long long *ukey = nullptr;  // full unique keys
  uint32_t *uniq = nullptr;            // their low 32 bits (reference layout)
  int *gfirst = nullptr, *gcount = nullptr, *glast = nullptr;

  // radix tree (Tree): internal n-1, all nodes 2n-1
  int *left = nullptr, *right = nullptr, *rfirst = nullptr, *rlast = nullptr,
      *plen = nullptr, *rparent = nullptr;

  // plan (RadixToOctreePlan), 2n-1
  int *plevel = nullptr, *pcount = nullptr, *poffset = nullptr;

  // octree, reference numbering (Octree), cap_nodes
  int *children = nullptr, *oparent = nullptr, *olevel = nullptr;
  unsigned long long *oprefix = nullptr;
  int *ofirst = nullptr, *ocount = nullptr, *child_count = nullptr,
      *pre_of = nullptr;    // preorder index by octree id
  int *by_level = nullptr;  // octree ids binned by level (fixed region per level)
  double *cx = nullptr, *cy = nullptr, *cz = nullptr, *half = nullptr;
  double *mass = nullptr, *comx = nullptr, *comy = nullptr, *comz = nullptr;
  int *subtree = nullptr, *preoff = nullptr;
  int *psub = nullptr, *pfirst = nullptr;  // particles in a subtree / its first
  int *pends = nullptr;   // n: octree nodes whose particle range ends at each sorted index, then their exclusive scan

  // traversal target groups: contiguous Morton ranges of <= kGroupMax
  // particles inside one parent cell
  unsigned char *tflag = nullptr;  // n, 1 where a target group starts
  int *tstart = nullptr;           // n, start of each target group

  // traversal layout: depth-first preorder, children visited octant 7 -> 0
  double4 *node_a = nullptr;  // com x, y, z, mass
  double4 *node_b = nullptr;  // centre x, y, z, half size
  double4 *node_c = nullptr;  // crit, crit^2 lower/upper band, mixed walk's squared box radius
  int4 *node_meta = nullptr;  // skip, first particle, particle count, nchild
  int *node_kids = nullptr;   // 8 per node, preorder ids in visit order
  MixedNode *node_m = nullptr;  // the mixed walk's records, preorder

  // level-order build (simulation steps): the octree numbered level by level
  int level_order = 0;          // host: 1 when steps build the level-order octree
  int *gspan = nullptr;         // n: per group (delta + 1) | lambda << 8 | (delta_next + 1) << 16
  int4 *lo_first = nullptr;     // cap: first particle, first child, subtree end (preorder), parent
  int *lo_arrive = nullptr;     // cap: children finished (arrival counters of the upward pass)
  int4 *lo_last = nullptr;      // cap: particle end, preorder index, key (low, high 32 bits)
  int2 *lo_gleaf = nullptr;     // n: per group, its leaf's level-order index and S(g)
  double4 *pos4 = nullptr;      // n: {x, y, z, -} in original order, written by the kick-drift pass
  LevelNode *lo_node = nullptr;  // cap: mass, centre of mass, preorder index, particles
  int *lo_tiles = nullptr;      // scan_tiles_n * kLevelOrderChannels: per-tile counts, then their prefixes
  int records = kRecordsFp64 | kRecordsMixed;  // host: the records the level-order build writes
  TopNode *top = nullptr;       // kTopMax: the top levels, for the mixed walk's node cache
  int *walk_ext = nullptr;    // walk_warps x walk_ext_cap: the mixed walk's stack below shared memory
};

// ------------------------------------------------------------ helpers ---

__device__ __forceinline__ void record_error(DevScalars *sc, int stage,
                                             int code) {
  atomicCAS(&sc->error, 0, stage * 100 + code);
}

// A relaxed load: for a word that carries its own flag and value (look-back
// status), no ordering against other memory is needed, and several such
// loads can be in flight at once.
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(
    const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p,
                                               unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Arrival counter increment with acquire-release ordering at GPU scope: the
// caller's earlier writes are visible to whoever sees the new count, and the
// caller sees every write released by earlier arrivals.
__device__ __forceinline__ int arrive_acq_rel(int *counter) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
  return old;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Order-preserving map of a double onto unsigned 64-bit integers.
__device__ __forceinline__ unsigned long long order_bits(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double order_value(unsigned long long k) {
  const unsigned long long b =
      (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
  return __longlong_as_double((long long)b);
}

// Spin limit of every bounded device wait (look-back).  Far above any wait
// that a live predecessor can cause; reaching it records kCodeTimeout.
constexpr int kSpinLimit = 1 << 22;

}  // namespace nbb

// Host-side entry points of the build and traversal translation units.
namespace nbb {

struct TraversalParams {
  double theta = 0.5;
  double soft = 0.0;
  double g = 1.0;
  double half_dt = 0.0;  // second half kick fused into the epilogue when kick
  int kick = 0;
  int precision = 0;     // 0 FP64 plain, 1 mixed
  int group_size = 32;
  // warp target sets: 0 = fixed slices of 32 consecutive Morton-ordered
  // particles, 1 = octree target groups (contiguous, inside one parent cell)
  int group_mode = 0;
  // mixed walk: tree levels below the root staged in shared memory per block
  // (0: none; 1 or 2: the top 9 or 73 cells; level-order builds of a single
  // system only)
  int cache_depth = 0;
};

// Launch-count bookkeeping (kernels launched by this library).
void count_launches(uint64_t k);
uint64_t launch_count();

// Reset per-step device scalars (sticky error untouched) and status arrays.
cudaError_t launch_step_reset(Workspace &ws, cudaStream_t s);
// Kick-drift (optional) fused with the global bounding-box reduction.
cudaError_t launch_kd_bbox(Workspace &ws, double dt, int do_kd, cudaStream_t s);
// Morton encode + digit histograms, onesweep sort, groups + gather.
// part: 0 all, 1 Morton encode + sort only, 2 leaf groups + gather only
cudaError_t launch_morton_sort_groups(Workspace &ws, cudaStream_t s, int part = 0);
// Karras tree, plan + scan, octree materialisation, geometry, physics,
// preorder layout.
cudaError_t launch_tree(Workspace &ws, double theta, cudaStream_t s);
// The same octree built level by level from the sorted unique keys (no radix
// tree), with the same traversal records and target groups; needs the
// level-order arrays of the workspace.
cudaError_t launch_level_order_tree(Workspace &ws, double theta, cudaStream_t s);
// launch_level_order_tree when ws.level_order, else launch_tree.
cudaError_t launch_octree(Workspace &ws, double theta, cudaStream_t s);
// The reference-numbered octree (Karras .. layout, no target groups) over the
// current leaf groups, after a level-order build of the same step (export).
cudaError_t launch_reference_octree(Workspace &ws, double theta, cudaStream_t s);
// Rebuild the octree target groups for ws.group_max on the current tree and
// reset the traversal counters (used by the group-size autotuner).
cudaError_t launch_retarget(Workspace &ws, cudaStream_t s);
// Bounded-wait self-test: a look-back whose predecessor never publishes.
cudaError_t launch_lookback_probe(unsigned long long *status, DevScalars *sc, cudaStream_t s);
// Traversal (+ optional fused second half kick).
cudaError_t launch_traversal(Workspace &ws, const TraversalParams &p,
                             cudaStream_t s);
// Diagnostic SIMT FMA throughput, TFLOP/s (precision 0 FP64, 1 FP32).
cudaError_t measure_fma_tflops(int precision, double *tflops);
// Plain kick / kick-drift over n particles.
cudaError_t launch_kick(double *vx, double *vy, double *vz, const double *ax,
                        const double *ay, const double *az, size_t n,
                        double dt, cudaStream_t s);
cudaError_t launch_kick_drift(double *x, double *y, double *z, double *vx,
                              double *vy, double *vz, const double *ax,
                              const double *ay, const double *az, size_t n,
                              double dt, cudaStream_t s);
// FP64 direct sum for a target list.
// Source chunks the direct sum uses for n sources and n_targets targets (1:
// each target's sum in one pass in index order, bit for bit the sequential
// sum; more: partial sums of consecutive source ranges added in range order,
// for few targets over many sources).  part holds chunks * 3 * n_targets.
int direct_chunks(size_t n, int n_targets);
cudaError_t launch_direct(size_t n, const double *m, const double *x,
                          const double *y, const double *z, int n_targets,
                          const int *targets, double g, double soft,
                          double *ax, double *ay, double *az, double *part,
                          cudaStream_t s);
// Traversal on a caller octree in the reference numbering (FP64 plain).
struct RefOctree {
  int n_nodes, n_particles;
  const int *children, *parent, *first, *count;
  const double *mass, *comx, *comy, *comz, *cx, *cy, *cz, *half;
};
cudaError_t launch_ref_octree_traversal(const RefOctree &o, const uint32_t *idx,
                                        const double *m, const double *x,
                                        const double *y, const double *z,
                                        double *ax, double *ay, double *az,
                                        double theta, double soft, double g,
                                        int morton_order, int *err,
                                        cudaStream_t s);
// Karras tree alone over caller keys (any 32-bit keys, duplicates allowed).
cudaError_t launch_radix_tree_only(const uint32_t *keys, int n, int *left,
                                   int *right, int *rfirst, int *rlast,
                                   int *plen, int *parent, cudaStream_t s);
// Bounding box, Morton keys and the stable (key, index) sort alone, on a
// workspace holding only positions, scalars, digit histograms, sort status
// and the two pair buffers; writes the caller's key and index arrays.
cudaError_t launch_morton_sort_only(Workspace &ws, uint32_t *keys, uint32_t *idx, cudaStream_t s);
// Leaf groups from caller sorted keys (no particles): fills uniq / gfirst /
// gcount / glast and n_groups.
cudaError_t launch_groups_from_keys(Workspace &ws, const uint32_t *sorted_keys,
                                    cudaStream_t s);
// Topology stages only (Karras .. materialise) for caller keys.
cudaError_t launch_topology(Workspace &ws, cudaStream_t s);

// Function-level stages (one reference build function each) on workspaces
// whose arrays alias the caller's: the box alone; keys and the sort against
// the box in ws.sys_box; leaf groups of caller keys (with their sizes); the
// plan of g groups; the octree of g groups and m nodes; cell geometry of m
// nodes; child counts, leaf and internal mass / centre of mass of m nodes
// from particles gathered by idx.
cudaError_t launch_bbox_only(Workspace &ws, cudaStream_t s);
cudaError_t launch_morton_sort_box(Workspace &ws, uint32_t *keys, uint32_t *idx, cudaStream_t s);
cudaError_t launch_leaf_groups(Workspace &ws, const uint32_t *sorted_keys, cudaStream_t s);
cudaError_t launch_plan_only(Workspace &ws, int g, cudaStream_t s);
cudaError_t launch_octree_only(Workspace &ws, int g, int m, cudaStream_t s);
cudaError_t launch_geometry_only(Workspace &ws, int m, cudaStream_t s);
cudaError_t launch_mass_only(Workspace &ws, const uint32_t *idx, int m, cudaStream_t s);
cudaError_t launch_widen_u32(const uint32_t *in, int n, unsigned long long *out, cudaStream_t s);
cudaError_t launch_narrow_u64(const unsigned long long *in, int n, uint32_t *out, cudaStream_t s);

// Reverse-mode buffers of one frozen-structure force evaluation.  The
// accelerations cotangent is coef * (gvx, gvy, gvz); gx / gy / gz / gm
// accumulate; gv += dt_v * gx afterwards when dt_v != 0.
struct AdjointBuffers {
  double *gvx = nullptr, *gvy = nullptr, *gvz = nullptr;
  double coef = 0.0;
  double dt_v = 0.0;
  double *gx = nullptr, *gy = nullptr, *gz = nullptr, *gm = nullptr;
  double4 *node_g = nullptr;  // per preorder node (cap_nodes)
  double4 *part_g = nullptr;  // per Morton slot
  double4 *tgt_g = nullptr;   // per Morton slot
  int *pparent = nullptr;     // per preorder node
  int2 *prange = nullptr;     // per preorder node
};
// Perturbed copies of the particles: field arrays of copies * n values,
// copy q at offset q * n (original order), plus per-copy scratch.
struct FrozenBatch {
  int copies = 0;
  double *m = nullptr, *x = nullptr, *y = nullptr, *z = nullptr;
  double *vx = nullptr, *vy = nullptr, *vz = nullptr;
  double *ax = nullptr, *ay = nullptr, *az = nullptr;
  double4 *pm4q = nullptr;     // copies * n, Morton order of the unperturbed tree
  double4 *aq_oct = nullptr;   // copies * cap_nodes, by octree id
  double4 *node_aq = nullptr;  // copies * cap_nodes, by preorder id
  int *pre_of = nullptr;       // cap_nodes
  int *pparent = nullptr;      // cap_nodes
  int2 *prange = nullptr;      // cap_nodes
};
// Frame capture (capture.cu): device scalars and header fields.
constexpr unsigned long long kFrameHeaderBytes = 128;  // version-3 header
struct FrameScalars {
  unsigned long long lo[3], hi[3];  // order-preserving encoded extrema
  int nonfinite;                    // a sampled position is not finite
  int bad_type;                     // a sampled type is outside 0..4
};
struct FrameHeaderFields {
  unsigned long long sequence = 0, step = 0, source_count = 0, sample_count = 0;
  double time = 0.0;
};
// Sample s of n particles ((i * n) / s), bounds, quantized payload and
// header into `frame` (kFrameHeaderBytes + 7 s bytes); flags in f.
cudaError_t launch_frame_capture(const double *x, const double *y, const double *z, const uint8_t *type, size_t n,
                                 size_t s, FrameScalars *f, const FrameHeaderFields &h, unsigned char *frame,
                                 cudaStream_t st);

// Conserved quantities (diagnostics.cu): 12 sums -- m, m x (3), m v (3),
// m x cross v (3), kinetic energy, 1/2 m phi -- over n particles (phi may be
// null), block partials then one fixed-order final sum into out[12].
cudaError_t launch_moments(const double *m, const double *x, const double *y, const double *z, const double *vx,
                           const double *vy, const double *vz, const double *phi, size_t n, double *partials,
                           int blocks, double *out, cudaStream_t s);
// Potential of every particle (original order) from the current tree, with
// the plain walk's acceptance test; and by direct summation.
cudaError_t launch_potential_tree(Workspace &ws, const TraversalParams &p, double *phi, cudaStream_t s);
cudaError_t launch_potential_direct(const double *m, const double *x, const double *y, const double *z, int n,
                                    double g, double soft, double *phi, cudaStream_t s);

// VJP of the force on the current tree (built from the positions in the
// workspace): the plain FP64 form's (p.precision 0) or the mixed form's (1,
// on the mixed walk's interaction lists); accumulates into ab.gx / gy / gz / gm.
cudaError_t launch_adjoint_force(Workspace &ws, const TraversalParams &p, const AdjointBuffers &ab,
                                 cudaStream_t s);
// The mixed walk evaluating the VJP (node / particle / target cotangents into
// ab.node_g, ab.part_g, ab.tgt_g).
cudaError_t launch_adjoint_mixed(Workspace &ws, const TraversalParams &p, const AdjointBuffers &ab,
                                 cudaStream_t s);
// Forces on every perturbed copy with the current tree's structure
// (accelerations into fb.ax / ay / az).
cudaError_t launch_frozen_force(Workspace &ws, const TraversalParams &p, const FrozenBatch &fb, cudaStream_t s);
// Adjoint of the FP64 direct sum (accumulating).
cudaError_t launch_direct_vjp(size_t n, const double *m, const double *x, const double *y, const double *z,
                              const double *gvx, const double *gvy, const double *gvz, double coef, double g,
                              double soft, double *gx, double *gy, double *gz, double *gm, cudaStream_t s);
// y += a x on three arrays.
cudaError_t launch_axpy3(double *yx, double *yy, double *yz, const double *xx, const double *xy, const double *xz,
                         double a, size_t n, cudaStream_t s);

}  // namespace nbb
