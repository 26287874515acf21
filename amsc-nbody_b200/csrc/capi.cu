// capi.cu -- the C ABI of include/nbb.h over the build and traversal kernels.
//
// Ownership and error behaviour follow the reference's Simulation
// (src/simulation.cpp, paths relative to the sytrams/AMSC-Nbody project
// root): the handle owns every device buffer, all of them allocated once at
// creation; a step allocates nothing, never synchronises with the host
// inside, and is captured once into a CUDA graph that later steps replay.
#include "nbb.h"
#include "nbb_internal.cuh"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace nbb {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

cudaError_t configure_traversal(Workspace &ws);

}  // namespace nbb

using namespace nbb;

namespace {

thread_local std::string t_message;
thread_local int t_code = 0;

int fail(int status, const std::string &msg, int code = 0) {
  t_message = msg;
  t_code = code;
  return status;
}

int ok() {
  t_message.clear();
  t_code = 0;
  return NBB_OK;
}

int cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
    return fail(NBB_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e), (int)e);
  return fail(NBB_ERR_CUDA, std::string(what) + " failed: " + cudaGetErrorString(e), (int)e);
}

#define NBB_CUDA(call, what)                 \
  do {                                       \
    cudaError_t _e = (call);                 \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

// Messages of the reference's device error codes, by stage.
const char *device_message(int stage, int code) {
  if (code == kCodeTimeout) {
    switch (stage) {
      case kStageSort: return "A bounded device-side wait gave up in the radix sort look-back";
      case kStageGroups: return "A bounded device-side wait gave up in a leaf/target group scan look-back";
      case kStagePlan: return "A bounded device-side wait gave up in the radix-to-octree plan scan look-back";
      default: return "A bounded device-side wait gave up";
    }
  }
  switch (stage) {
    case kStageBbox:
      return code == 1 ? "Particle positions must be finite to compute a bounding box."
                       : "Morton bounding box is not valid";
    case kStagePlan:  // radix_to_octree.cu:32-51
      switch (code) {
        case 1: return "A Morton key uses bits outside the configured 30-bit spatial layout";
        case 2: return "A radix node has an invalid parent";
        case 3: return "A radix child has an octree level smaller than its parent";
        case 4: return "A radix internal node has an invalid prefix length";
        case kCodeOverflow: return "The computed octree node count exceeds the node capacity";
        default: return "Unknown radix-to-octree planning error";
      }
    case kStageOctree:  // octree_builder.cu:18-46
      switch (code) {
        case 1: return "Invalid radix edge metadata";
        case 2: return "Invalid radix ancestor while constructing octree";
        case 3: return "Could not find the correct octree parent level";
        case 4: return "Two octree nodes attempted to occupy the same parent octant";
        case 5: return "A radix leaf terminates at an invalid octree level";
        case 6: return "Generated octree node ID is outside the allocated range";
        case 7: return "Invalid representative Morton key";
        default: return "Unknown sparse-octree construction error";
      }
    case kStageGeometry:  // octree_geometry.cu:21-34
      return code == 1 ? "Octree node has an invalid level"
                       : code == 2 ? "Octree node has an invalid Morton prefix" : "Unknown octree geometry error";
    case kStagePhysics:  // octree_physics.cu:18-46
      switch (code) {
        case 1: return "Octree contains an invalid child ID";
        case 2: return "Occupied octree leaf has invalid particle range";
        case 3: return "Sorted particle index is outside the particle array";
        case 4: return "Occupied octree leaf has children";
        case 5: return "Invalid octree parent during bottom-up propagation";
        case 6: return "Invalid octree child count";
        case 7: return "An octree parent was signalled too many times";
        default: return "Unknown octree physics error";
      }
    case kStageTraversal:  // barnes_hut.cu:21-52
      switch (code) {
        case 1: return "Barnes-Hut traversal found an invalid child node";
        case 2: return "Barnes-Hut traversal found an invalid leaf particle range";
        case 3: return "Sorted particle index is outside the particle array";
        case 4: return "Barnes-Hut traversal found inconsistent parent-child topology";
        case 5: return "Barnes-Hut traversal found an empty terminal node";
        case 6: return "Singular gravitational interaction; use positive softening";
        case 7: return "Occupied octree leaf unexpectedly has children";
        case 8: return "Octree node has invalid geometry";
        case 9: return "Mixed-precision traversal ran out of stack space; nodes were accepted untested";
        default: return "Unknown Barnes-Hut traversal error";
      }
    case kStageLayout:
      return "Octree preorder layout found an inconsistent parent chain";
    default:
      return "Unknown device error";
  }
}

int device_status(int word) {
  const int stage = word / 100, code = word % 100;
  const int status = (code == kCodeTimeout) ? NBB_ERR_TIMEOUT
                     : (stage == kStageBbox && code == 1) ? NBB_ERR_DOMAIN
                     : (stage == kStagePlan && code == kCodeOverflow) ? NBB_ERR_OVERFLOW
                                                                      : NBB_ERR_DEVICE;
  return fail(status, device_message(stage, code), word);
}

// Octree node capacity: every level L holds at most min(8^L, G) nodes and
// G <= n, over levels 0..max_level.
int node_capacity(int n, int max_level) {
  long long cap = 1;
  long long width = 1;
  for (int level = 0; level <= max_level; ++level) {
    cap += (width < n) ? width : n;
    if (width < (1ll << 40)) width *= 8;
  }
  return cap > INT_MAX ? INT_MAX : (int)cap;
}

struct Allocation {
  std::vector<void *> ptrs;
  ~Allocation() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t get(T *&out, size_t count) {
    void *p = nullptr;
    const cudaError_t e = cudaMalloc(&p, (count > 0 ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    ptrs.push_back(p);
    out = static_cast<T *>(p);
    return cudaSuccess;
  }
};

// Allocate every buffer of a workspace for n particles (state included when
// with_state).  All device memory is taken here; nothing is allocated later.
cudaError_t alloc_workspace(Workspace &ws, Allocation &al, int n, bool with_state, int n_systems = 1,
                            bool level_order = false) {
  ws = Workspace{};
  ws.n = n;
  ws.n_systems = n_systems;
  ws.sys_levels = 0;
  while ((1 << (3 * ws.sys_levels)) < n_systems) ++ws.sys_levels;
  ws.key_bits = kSpatialBits + kDims * ws.sys_levels;
  ws.max_level = ws.key_bits / kDims;
  ws.pack_shift = 64 - ws.key_bits;
  ws.sort_passes = (ws.key_bits + 7) / 8;
  ws.cap_nodes = node_capacity(n, ws.max_level);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&ws.num_sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t N = (size_t)n, C = (size_t)ws.cap_nodes;
  cudaError_t e = cudaSuccess;
#define GET(ptr, cnt) \
  if ((e = al.get(ptr, cnt)) != cudaSuccess) return e
  if (with_state) {
    GET(ws.m, N); GET(ws.x, N); GET(ws.y, N); GET(ws.z, N);
    GET(ws.vx, N); GET(ws.vy, N); GET(ws.vz, N);
    GET(ws.ax, N); GET(ws.ay, N); GET(ws.az, N);
    GET(ws.type, N);
  }
  const size_t S = (size_t)n_systems;
  if (n_systems > 1) {
    GET(ws.sys_of, N);
    GET(ws.sys_eps, S);
  }
  GET(ws.sc, 1);
  GET(ws.sys_bb, 6 * S); GET(ws.sys_box, 4 * S); GET(ws.root_pre, S);
  GET(ws.pairs_a, N); GET(ws.pairs_b, N);
  GET(ws.digit_hist, (size_t)kMaxSortPasses * 256);
  ws.sort_tiles = (n + kSortTile - 1) / kSortTile;
  GET(ws.sort_status, (size_t)ws.sort_passes * ws.sort_tiles * 256);
  ws.scan_tiles_n = (n + kScanTile - 1) / kScanTile;
  ws.scan_tiles_r = (2 * n - 1 + kScanTile - 1) / kScanTile;
  GET(ws.scan_status, (size_t)(3 * ws.scan_tiles_n + ws.scan_tiles_r));
  GET(ws.keys, N); GET(ws.idx, N); GET(ws.pm4, N); GET(ws.psys, N);
  GET(ws.ukey, N); GET(ws.uniq, N); GET(ws.gfirst, N); GET(ws.gcount, N); GET(ws.glast, N);
  GET(ws.left, N); GET(ws.right, N); GET(ws.rfirst, N); GET(ws.rlast, N); GET(ws.plen, N);
  GET(ws.rparent, 2 * N);
  GET(ws.plevel, 2 * N); GET(ws.pcount, 2 * N); GET(ws.poffset, 2 * N);
  GET(ws.children, 8 * C);
  GET(ws.oparent, C); GET(ws.olevel, C); GET(ws.oprefix, C); GET(ws.ofirst, C); GET(ws.ocount, C);
  GET(ws.child_count, C); GET(ws.pre_of, C); GET(ws.by_level, C); GET(ws.subtree, C); GET(ws.preoff, C);
  GET(ws.psub, C); GET(ws.pfirst, C); GET(ws.pends, N);
  GET(ws.tflag, N); GET(ws.tstart, N);
  GET(ws.cx, C); GET(ws.cy, C); GET(ws.cz, C); GET(ws.half, C);
  GET(ws.mass, C); GET(ws.comx, C); GET(ws.comy, C); GET(ws.comz, C);
  GET(ws.node_a, C); GET(ws.node_b, C); GET(ws.node_c, C); GET(ws.node_meta, C);
  GET(ws.node_kids, 8 * C);
  GET(ws.node_m, C);
  if (level_order) {
    ws.level_order = 1;
    GET(ws.gspan, N);
    GET(ws.lo_first, C); GET(ws.lo_arrive, C); GET(ws.lo_last, C); GET(ws.lo_node, C); GET(ws.lo_gleaf, N);
    GET(ws.pos4, N);
    GET(ws.lo_tiles, (size_t)ws.scan_tiles_n * kLevelOrderChannels);
    GET(ws.top, (size_t)kTopMax);
  }
#undef GET
  e = cudaMemset(ws.sc, 0, sizeof(DevScalars));
  if (e != cudaSuccess) return e;
  e = cudaMemset(ws.root_pre, 0, S * sizeof(int));
  if (e != cudaSuccess) return e;
  e = configure_traversal(ws);
  if (e != cudaSuccess) return e;
  return al.get(ws.walk_ext, (size_t)ws.walk_warps * ws.walk_ext_cap);
}

bool finite_nonneg(double v) { return std::isfinite(v) && v >= 0.0; }

// The plain walk's per-lane acceptance test tolerates wide warps and prefers
// full ones (fixed 32-particle slices); the mixed walk shares one acceptance
// test per warp and needs compact octree target groups.
int default_group_mode(int precision) { return precision == NBB_PRECISION_MIXED ? 1 : 0; }

template <typename T>
cudaError_t d2h_opt(T *dst, const T *src, size_t count, cudaStream_t s) {
  if (dst == nullptr || count == 0) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s);
}

// Copy every intermediate of the last build into caller buffers.
int export_workspace(const Workspace &ws, nbb_tree_export *o, cudaStream_t s, bool particles) {
  DevScalars sc;
  NBB_CUDA(cudaMemcpyAsync(&sc, ws.sc, sizeof(sc), cudaMemcpyDeviceToHost, s), "copy device scalars");
  NBB_CUDA(cudaStreamSynchronize(s), "export synchronisation");
  const int n = ws.n, g = sc.n_groups, m = sc.n_nodes;
  o->n_groups = g;
  o->n_octree = m;
  for (int a = 0; a < 4; ++a) o->box[a] = sc.box[a];
  if (m > o->m_capacity && (o->children || o->oparent || o->olevel || o->oprefix || o->ofirst ||
                            o->ocount || o->child_count || o->cx || o->mass))
    return fail(NBB_ERR_INVALID_ARGUMENT, "export m_capacity is smaller than the octree node count");
  if (ws.key_bits > 32 && (o->keys || o->uniq || o->oprefix))
    return fail(NBB_ERR_INVALID_ARGUMENT,
                "keys of an ensemble with more than 4 systems exceed 32 bits; pass null keys, uniq and oprefix");
  const size_t G = (size_t)g, R = g > 0 ? (size_t)(2 * g - 1) : 0, I = g > 1 ? (size_t)(g - 1) : 0;
  const size_t M = (size_t)m;
  NBB_CUDA(d2h_opt(o->keys, ws.keys, (size_t)n, s), "export keys");
  NBB_CUDA(d2h_opt(o->idx, ws.idx, (size_t)n, s), "export idx");
  NBB_CUDA(d2h_opt(o->uniq, ws.uniq, G, s), "export groups");
  NBB_CUDA(d2h_opt(o->gfirst, ws.gfirst, G, s), "export groups");
  NBB_CUDA(d2h_opt(o->gcount, ws.gcount, G, s), "export groups");
  NBB_CUDA(d2h_opt(o->left, ws.left, I, s), "export tree");
  NBB_CUDA(d2h_opt(o->right, ws.right, I, s), "export tree");
  NBB_CUDA(d2h_opt(o->rfirst, ws.rfirst, I, s), "export tree");
  NBB_CUDA(d2h_opt(o->rlast, ws.rlast, I, s), "export tree");
  NBB_CUDA(d2h_opt(o->plen, ws.plen, I, s), "export tree");
  NBB_CUDA(d2h_opt(o->rparent, ws.rparent, R, s), "export tree");
  NBB_CUDA(d2h_opt(o->plan_level, ws.plevel, R, s), "export plan");
  NBB_CUDA(d2h_opt(o->plan_count, ws.pcount, R, s), "export plan");
  NBB_CUDA(d2h_opt(o->plan_offset, ws.poffset, R, s), "export plan");
  NBB_CUDA(d2h_opt(o->children, ws.children, 8 * M, s), "export octree");
  NBB_CUDA(d2h_opt(o->oparent, ws.oparent, M, s), "export octree");
  NBB_CUDA(d2h_opt(o->olevel, ws.olevel, M, s), "export octree");
  if (o->oprefix && M) {
    std::vector<unsigned long long> wide(M);
    NBB_CUDA(cudaMemcpyAsync(wide.data(), ws.oprefix, M * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
             "export octree");
    NBB_CUDA(cudaStreamSynchronize(s), "export synchronisation");
    for (size_t k = 0; k < M; ++k) o->oprefix[k] = (uint32_t)wide[k];
  }
  NBB_CUDA(d2h_opt(o->ofirst, ws.ofirst, M, s), "export octree");
  NBB_CUDA(d2h_opt(o->ocount, ws.ocount, M, s), "export octree");
  if (particles) {
    NBB_CUDA(d2h_opt(o->child_count, ws.child_count, M, s), "export octree");
    NBB_CUDA(d2h_opt(o->cx, ws.cx, M, s), "export geometry");
    NBB_CUDA(d2h_opt(o->cy, ws.cy, M, s), "export geometry");
    NBB_CUDA(d2h_opt(o->cz, ws.cz, M, s), "export geometry");
    NBB_CUDA(d2h_opt(o->half, ws.half, M, s), "export geometry");
    NBB_CUDA(d2h_opt(o->mass, ws.mass, M, s), "export physics");
    NBB_CUDA(d2h_opt(o->comx, ws.comx, M, s), "export physics");
    NBB_CUDA(d2h_opt(o->comy, ws.comy, M, s), "export physics");
    NBB_CUDA(d2h_opt(o->comz, ws.comz, M, s), "export physics");
  }
  NBB_CUDA(cudaStreamSynchronize(s), "export synchronisation");
  return ok();
}

// Read the sticky device error word (one small copy + stream sync).
int check_device(const Workspace &ws, cudaStream_t s) {
  int word = 0;
  NBB_CUDA(cudaMemcpyAsync(&word, &ws.sc->error, sizeof(int), cudaMemcpyDeviceToHost, s), "copy error word");
  NBB_CUDA(cudaStreamSynchronize(s), "device synchronisation");
  if (word != 0) return device_status(word);
  return ok();
}

// Rebuild + force on the workspace state (kd: first half kick + drift before
// the rebuild; kick: second half kick fused into the traversal).
// part: 0 the whole step; or one of its three parts: 1 reset and
// kick-drift + box (the last writes of the positions), 2 Morton encode and
// sort, 3 leaf groups with the gather (the first read of the masses), tree,
// walk + kick.
cudaError_t enqueue_rebuild_force(Workspace &ws, const TraversalParams &tp, double dt, int kd,
                                  cudaStream_t s, int part = 0) {
  ws.group_max = (tp.group_mode && tp.group_size > 32) ? (tp.group_size > 64 ? 128 : 64) : 32;
  // the level-order build writes only the records of this walk
  ws.records = tp.precision == NBB_PRECISION_MIXED ? kRecordsMixed : kRecordsFp64;
  cudaError_t e = cudaSuccess;
  if (part == 0 || part == 1) {
    e = launch_step_reset(ws, s);
    if (e == cudaSuccess) e = launch_kd_bbox(ws, dt, kd, s);
  }
  if (e == cudaSuccess && part != 1) e = launch_morton_sort_groups(ws, s, part == 0 ? 0 : part - 1);
  if (part == 1 || part == 2) return e;
  if (e == cudaSuccess) e = launch_octree(ws, tp.theta, s);
  if (e == cudaSuccess) e = launch_traversal(ws, tp, s);
  return e;
}

template <typename T>
cudaError_t stage_in(const T *src, size_t count, bool on_device, Allocation &al, const T *&dst,
                            cudaStream_t s) {
  if (src == nullptr || on_device) {
    dst = src;
    return cudaSuccess;
  }
  T *d = nullptr;
  cudaError_t e = al.get(d, count);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
  dst = d;
  return e;
}

}  // namespace

// -------------------------------------------------------------- handle ---

// Device storage of a recorded rollout: (x, v, a) every `every` steps, the
// final state, one segment of recomputed positions and the reverse-mode
// buffers.  Taken when the rollout starts, released with the handle or by
// the next rollout.
struct RolloutRecord {
  Allocation al;
  uint64_t steps = 0, every = 0, slots = 0;
  double *ckpt = nullptr;         // slots x 9 x n: x y z vx vy vz ax ay az
  double *final_state = nullptr;  // 9 x n
  double *seg = nullptr;          // (every - 1) x 3 x n recomputed positions
  double *g = nullptr;            // 7 x n: gx gy gz gvx gvy gvz gm
  double4 *node_g = nullptr, *part_g = nullptr, *tgt_g = nullptr;
  int *pparent = nullptr;
  int2 *prange = nullptr;
};

// Device buffers of frame capture, taken at the first capture.
struct FrameBuffers {
  Allocation al;
  size_t bytes = 0;
  unsigned char *frame = nullptr;
  FrameScalars *scalars = nullptr;
};

// A step with host state in and out (nbb_sim_step_host): the step split
// into three graphs (enqueue_rebuild_force's parts) so that a second stream
// uploads the masses while the positions are sorted and copies the drifted
// positions to the host while the tree is rebuilt and walked.  Taken at the
// first such step.
struct HostStep {
  static constexpr int kParts = 3;
  cudaGraphExec_t exec[kParts] = {};
  cudaGraph_t def[kParts] = {};
  uint64_t kernels[kParts] = {};
  cudaStream_t copy = nullptr;
  cudaEvent_t state_in = nullptr, mass_in = nullptr, drifted = nullptr, copied = nullptr;
  ~HostStep() {
    if (copy) cudaStreamSynchronize(copy);
    for (int k = 0; k < kParts; ++k) {
      if (exec[k]) cudaGraphExecDestroy(exec[k]);
      if (def[k]) cudaGraphDestroy(def[k]);
    }
    for (cudaEvent_t ev : {state_in, mass_in, drifted, copied})
      if (ev) cudaEventDestroy(ev);
    if (copy) cudaStreamDestroy(copy);
  }
};

// Device buffers of the conserved-quantity monitor, taken at its first use.
struct DiagBuffers {
  static constexpr int kBlocks = 592;  // fixed: the sums' order never changes
  Allocation al;
  double *partials = nullptr, *out = nullptr, *phi = nullptr;
};

struct nbb_sim {
  nbb_config cfg{};
  Workspace ws{};
  Allocation alloc;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  enum class State { created, ready, failed } state = State::created;
  double time = 0.0;
  uint64_t steps = 0;
  cudaGraphExec_t step_graph = nullptr;
  cudaGraph_t step_graph_def = nullptr;
  uint64_t graph_kernels = 0;
  int tuned_group_size = 0;
  int tuned_cache_depth = -1;     // mixed walk's node-cache depth; -1 untuned
  int tuned_fp64_grouping = -1;  // plain walk: 0 Morton slices, 1 octree groups; -1 untuned
  double min_softening = 0.0;  // ensembles: smallest per-system softening
  std::unique_ptr<RolloutRecord> rollout;
  std::unique_ptr<FrameBuffers> frames;
  std::unique_ptr<DiagBuffers> diag;
  std::unique_ptr<HostStep> host_step;
};

extern "C" {

void nbb_config_default(nbb_config *cfg) {
  if (!cfg) return;
  cfg->time_step = 0.0;
  cfg->theta = 0.5;                        // barnes_hut.hpp:10
  cfg->softening = 1.0e-6;                 // barnes_hut.hpp:11
  cfg->gravitational_constant = 6.67430e-11;  // barnes_hut.hpp:12
  cfg->precision = NBB_PRECISION_FP64;
  cfg->group_size = 0;
  cfg->use_graph = 1;
  cfg->device = 0;
  cfg->cache_depth = -1;
}

int nbb_selftest_bounded_wait(void) {
  Allocation al;
  cudaStream_t s = nullptr;
  NBB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  DevScalars *sc = nullptr;
  unsigned long long *status = nullptr;
  cudaError_t e = al.get(sc, 1);
  if (e == cudaSuccess) e = al.get(status, 2);
  if (e == cudaSuccess) e = cudaMemsetAsync(sc, 0, sizeof(DevScalars), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, 2 * sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = launch_lookback_probe(status, sc, s);
  int word = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&word, &sc->error, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return cuda_fail(e, "bounded-wait self-test");
  if (word == 0) return fail(NBB_ERR_DEVICE, "bounded-wait self-test: the wait did not report a timeout");
  return device_status(word);
}

int nbb_measure_fma_tflops(int precision, double *tflops) {
  if (!tflops) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  if (precision < 0 || precision > 2) return fail(NBB_ERR_INVALID_ARGUMENT, "precision must be 0, 1 or 2");
  NBB_CUDA(measure_fma_tflops(precision, tflops), "FMA throughput kernel");
  return ok();
}

const char *nbb_last_error_message(void) { return t_message.c_str(); }
int nbb_last_error_code(void) { return t_code; }
uint64_t nbb_kernel_launch_count(void) { return nbb::launch_count(); }

static int validate_config(const nbb_config *c) {
  // simulation.cpp:21-33, barnes_hut.cu:355-363
  if (!std::isfinite(c->time_step) || c->time_step <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Simulation timeStep must be finite and positive");
  if (!finite_nonneg(c->theta))
    return fail(NBB_ERR_INVALID_ARGUMENT, "Simulation theta must be finite and non-negative");
  if (!finite_nonneg(c->softening))
    return fail(NBB_ERR_INVALID_ARGUMENT, "Simulation softening must be finite and non-negative");
  if (!std::isfinite(c->gravitational_constant) || c->gravitational_constant <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Gravitational constant must be finite and positive");
  if (c->precision != NBB_PRECISION_FP64 && c->precision != NBB_PRECISION_MIXED)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Unknown traversal precision");
  if (c->group_size != 0 && c->group_size != 32 && c->group_size != 64 && c->group_size != 128)
    return fail(NBB_ERR_INVALID_ARGUMENT, "group_size must be 0 (tuned), 32, 64 or 128");
  if (c->cache_depth < -1 || c->cache_depth > kTopDepth)
    return fail(NBB_ERR_INVALID_ARGUMENT, "cache_depth must be -1 (tuned), 0, 1 or 2");
  return NBB_OK;
}

static int create_sim(const nbb_config *cfg, size_t n, int n_systems, const int64_t *offsets,
                      const double *softening, const double *mass, const double *x, const double *y,
                      const double *z, const double *vx, const double *vy, const double *vz,
                      const uint8_t *type, int on_device, nbb_sim **out) {
  if (!cfg || !out) return fail(NBB_ERR_INVALID_ARGUMENT, "nbb_sim_create: null argument");
  *out = nullptr;
  int st = validate_config(cfg);
  if (st) return st;
  if (n == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Simulation requires at least one particle");
  if (n > (size_t)(INT_MAX / 2))
    return fail(NBB_ERR_OVERFLOW, "Particle count exceeds the tree representation");
  if (!mass || !x || !y || !z || !vx || !vy || !vz)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Particle arrays must not be null");
  std::vector<int> sys_of;
  std::vector<double> eps;
  double min_eps = cfg->softening;
  if (n_systems > 1) {
    if (n_systems > kMaxSystems)
      return fail(NBB_ERR_INVALID_ARGUMENT, "An ensemble holds at most " + std::to_string(kMaxSystems) + " systems");
    if (!offsets || offsets[0] != 0 || offsets[n_systems] != (int64_t)n)
      return fail(NBB_ERR_INVALID_ARGUMENT, "Ensemble offsets must start at 0 and end at the particle count");
    const int key_bits = kSpatialBits + kDims * 3;
    if ((unsigned long long)n >= (1ull << (64 - key_bits)))
      return fail(NBB_ERR_OVERFLOW, "Ensemble particle count exceeds the sort key layout");
    sys_of.resize(n);
    eps.resize((size_t)n_systems);
    min_eps = INFINITY;
    for (int k = 0; k < n_systems; ++k) {
      if (offsets[k + 1] <= offsets[k])
        return fail(NBB_ERR_INVALID_ARGUMENT, "Every ensemble system needs at least one particle");
      eps[k] = softening ? softening[k] : cfg->softening;
      if (!finite_nonneg(eps[k]))
        return fail(NBB_ERR_INVALID_ARGUMENT, "Simulation softening must be finite and non-negative");
      min_eps = std::min(min_eps, eps[k]);
      for (int64_t i = offsets[k]; i < offsets[k + 1]; ++i) sys_of[(size_t)i] = k;
    }
  }
  NBB_CUDA(cudaSetDevice(cfg->device), "cudaSetDevice");
  nbb_sim *sim = new (std::nothrow) nbb_sim();
  if (!sim) return fail(NBB_ERR_CUDA, "host allocation failed");
  sim->cfg = *cfg;
  sim->min_softening = min_eps;
  cudaError_t e = cudaStreamCreateWithFlags(&sim->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = alloc_workspace(sim->ws, sim->alloc, (int)n, true, n_systems > 1 ? n_systems : 1, true);
  if (e != cudaSuccess) {
    if (sim->own_stream) cudaStreamDestroy(sim->own_stream);
    delete sim;
    return cuda_fail(e, "allocate simulation state");
  }
  sim->stream = sim->own_stream;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t bytes = n * sizeof(double);
  Workspace &ws = sim->ws;
  const double *src[7] = {mass, x, y, z, vx, vy, vz};
  double *dst[7] = {ws.m, ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz};
  for (int k = 0; k < 7 && e == cudaSuccess; ++k) e = cudaMemcpyAsync(dst[k], src[k], bytes, kind, sim->stream);
  if (e == cudaSuccess) e = type ? cudaMemcpyAsync(ws.type, type, n, kind, sim->stream)
                                 : cudaMemsetAsync(ws.type, 0, n, sim->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.ax, 0, bytes, sim->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.ay, 0, bytes, sim->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws.az, 0, bytes, sim->stream);
  if (e == cudaSuccess && n_systems > 1) {
    e = cudaMemcpyAsync(ws.sys_of, sys_of.data(), n * sizeof(int), cudaMemcpyHostToDevice, sim->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ws.sys_eps, eps.data(), eps.size() * sizeof(double), cudaMemcpyHostToDevice, sim->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(sim->stream);
  if (e != cudaSuccess) {
    nbb_sim_destroy(sim);
    return cuda_fail(e, "copy particle state");
  }
  *out = sim;
  return ok();
}

int nbb_sim_create(const nbb_config *cfg, size_t n, const double *mass, const double *x,
                   const double *y, const double *z, const double *vx, const double *vy,
                   const double *vz, const uint8_t *type, int on_device, nbb_sim **out) {
  return create_sim(cfg, n, 1, nullptr, nullptr, mass, x, y, z, vx, vy, vz, type, on_device, out);
}

int nbb_ensemble_create(const nbb_config *cfg, int n_systems, const int64_t *offsets,
                        const double *softening, const double *mass, const double *x, const double *y,
                        const double *z, const double *vx, const double *vy, const double *vz,
                        int on_device, nbb_sim **out) {
  if (n_systems <= 0 || !offsets) return fail(NBB_ERR_INVALID_ARGUMENT, "An ensemble needs at least one system");
  const size_t n = (size_t)offsets[n_systems];
  if (n_systems == 1) {
    nbb_config c = *cfg;
    if (softening) c.softening = softening[0];
    return create_sim(&c, n, 1, nullptr, nullptr, mass, x, y, z, vx, vy, vz, nullptr, on_device, out);
  }
  return create_sim(cfg, n, n_systems, offsets, softening, mass, x, y, z, vx, vy, vz, nullptr, on_device, out);
}

static TraversalParams traversal_params(const nbb_sim *sim, int kick) {
  TraversalParams tp;
  tp.theta = sim->cfg.theta;
  tp.soft = sim->cfg.softening;
  tp.g = sim->cfg.gravitational_constant;
  tp.half_dt = 0.5 * sim->cfg.time_step;
  tp.kick = kick;
  tp.precision = sim->cfg.precision;
  tp.group_size = sim->cfg.group_size > 0 ? sim->cfg.group_size
                                          : (sim->tuned_group_size > 0 ? sim->tuned_group_size : 32);
  tp.group_mode = default_group_mode(tp.precision);
  if (tp.precision == NBB_PRECISION_MIXED && sim->ws.top && sim->ws.n_systems == 1)
    tp.cache_depth = sim->cfg.cache_depth >= 0 ? sim->cfg.cache_depth
                                               : (sim->tuned_cache_depth > 0 ? sim->tuned_cache_depth : 0);
  if (tp.precision == NBB_PRECISION_FP64 && sim->tuned_fp64_grouping >= 0) tp.group_mode = sim->tuned_fp64_grouping;
  if (sim->ws.n_systems > 1) {
    tp.group_mode = 1;  // a warp's targets must share a system
    tp.soft = sim->min_softening;
  }
  return tp;
}

// Autotuner of the mixed walk: on the tree of the first force evaluation,
// time the traversal (CUDA events, best of three rounds) for each candidate warp group
// size (32, 64 or 128 targets: 1, 2 or 4 per lane; only the configured one
// when nbb_config.group_size pins it) and each node-cache depth (0, 1 or 2
// levels below the root staged in shared memory; single systems), and keep
// the fastest pair.  Results do not depend on the cache depth.  The choice is
// cached per process for the particle count's power-of-two bucket and the
// pinned group size, so every simulation of that size in the process uses
// the same setting.
struct MixedTuning {
  int bucket, pinned, pinned_depth, group_size, cache_depth;
};
static std::mutex g_tune_lock;
static std::vector<MixedTuning> g_tuned;

static int autotune_mixed_walk(nbb_sim *sim) {
  Workspace &ws = sim->ws;
  int bucket = 0;
  while ((1 << bucket) < ws.n && bucket < 31) ++bucket;
  const int pinned = sim->cfg.group_size;
  bool found = false;
  {
    std::lock_guard<std::mutex> g(g_tune_lock);
    for (const auto &t : g_tuned)
      if (t.bucket == bucket && t.pinned == pinned && t.pinned_depth == sim->cfg.cache_depth) {
        if (!pinned) sim->tuned_group_size = t.group_size;
        sim->tuned_cache_depth = t.cache_depth;
        found = true;
        break;
      }
  }
  if (!found) {
    cudaStream_t s = sim->stream;
    cudaEvent_t e0, e1;
    NBB_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
    NBB_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
    const int sizes[3] = {32, 64, 128};
    const int n_sizes = pinned ? 1 : 3;
    const int pinned_depth = sim->cfg.cache_depth;
    const bool cacheable = ws.top && ws.n_systems == 1;
    const int n_depths = (pinned_depth >= 0 || !cacheable) ? 1 : kTopDepth + 1;
    // candidates timed round-robin (three rounds, best time of each) after
    // one untimed walk, so that clock ramp-up and cache warm-up fall on no
    // single candidate
    float cand_ms[3][kTopDepth + 1];
    for (auto &row : cand_ms)
      for (float &v : row) v = 1e30f;
    cudaError_t e = cudaSuccess;
    for (int round = -1; round < 3 && e == cudaSuccess; ++round) {
      for (int c = 0; c < n_sizes && e == cudaSuccess; ++c) {
        TraversalParams tp = traversal_params(sim, 0);
        tp.group_size = pinned ? pinned : sizes[c];
        ws.group_max = tp.group_size;
        for (int d = 0; d < n_depths && e == cudaSuccess; ++d) {
          tp.cache_depth = cacheable ? (pinned_depth >= 0 ? pinned_depth : d) : 0;
          e = launch_retarget(ws, s);
          if (e == cudaSuccess) e = cudaEventRecord(e0, s);
          if (e == cudaSuccess) e = launch_traversal(ws, tp, s);
          if (e == cudaSuccess) e = cudaEventRecord(e1, s);
          if (e == cudaSuccess) e = cudaEventSynchronize(e1);
          float ms = 0.f;
          if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
          if (e == cudaSuccess && round >= 0 && ms < cand_ms[c][d]) cand_ms[c][d] = ms;
          if (round < 0) break;  // the warm-up walk: one candidate
        }
        if (round < 0) break;
      }
    }
    float best = 1e30f;
    int best_size = pinned ? pinned : 32, best_depth = 0;
    for (int c = 0; c < n_sizes; ++c)
      for (int d = 0; d < n_depths; ++d)
        if (cand_ms[c][d] < best) {
          best = cand_ms[c][d];
          best_size = pinned ? pinned : sizes[c];
          best_depth = cacheable ? (pinned_depth >= 0 ? pinned_depth : d) : 0;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "mixed walk autotuning");
    if (!pinned) sim->tuned_group_size = best_size;
    sim->tuned_cache_depth = best_depth;
    std::lock_guard<std::mutex> g(g_tune_lock);
    g_tuned.push_back({bucket, pinned, sim->cfg.cache_depth, best_size, best_depth});
  }
  // the initial acceleration comes from the chosen setting
  TraversalParams tp = traversal_params(sim, 0);
  ws.group_max = tp.group_size;
  NBB_CUDA(launch_retarget(ws, sim->stream), "retarget");
  NBB_CUDA(launch_traversal(ws, tp, sim->stream), "traversal");
  return check_device(ws, sim->stream);
}

// Grouping autotuner of the plain FP64 walk: every lane follows its own
// target's node sequence, so results do not depend on which targets share a
// warp, only the time does -- fixed slices of 32 Morton-consecutive targets
// (short runs, best for large systems) or octree target groups of at most 32
// (compact, best where few warps must fill the GPU).  Timed on the tree of
// the first force evaluation (best of two each), cached per process and
// power-of-two size bucket.
static std::vector<std::pair<int, int>> g_tuned_fp64;  // (log2 bucket, grouping)

static int autotune_fp64_grouping(nbb_sim *sim) {
  Workspace &ws = sim->ws;
  int bucket = 0;
  while ((1 << bucket) < ws.n && bucket < 31) ++bucket;
  {
    std::lock_guard<std::mutex> g(g_tune_lock);
    for (const auto &kv : g_tuned_fp64)
      if (kv.first == bucket) {
        sim->tuned_fp64_grouping = kv.second;
        return ok();
      }
  }
  cudaStream_t s = sim->stream;
  cudaEvent_t e0, e1;
  NBB_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
  NBB_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
  float best = 1e30f;
  int best_mode = 0;
  cudaError_t e = cudaSuccess;
  for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
    TraversalParams tp = traversal_params(sim, 0);
    tp.group_mode = mode;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
      e = launch_retarget(ws, s);
      if (e == cudaSuccess) e = cudaEventRecord(e0, s);
      if (e == cudaSuccess) e = launch_traversal(ws, tp, s);
      if (e == cudaSuccess) e = cudaEventRecord(e1, s);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e == cudaSuccess && ms < best) {
        best = ms;
        best_mode = mode;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "walk grouping autotuning");
  sim->tuned_fp64_grouping = best_mode;
  std::lock_guard<std::mutex> g(g_tune_lock);
  g_tuned_fp64.emplace_back(bucket, best_mode);
  return check_device(ws, s);
}

int nbb_sim_initialize(nbb_sim *sim) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (sim->state != nbb_sim::State::created)
    return fail(NBB_ERR_LOGIC, "Simulation can only be initialized once");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  Workspace &ws = sim->ws;
  cudaError_t e = enqueue_rebuild_force(ws, traversal_params(sim, 0), sim->cfg.time_step, 0, sim->stream);
  if (e != cudaSuccess) {
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "initialize");
  }
  int st = check_device(ws, sim->stream);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  if (sim->cfg.precision == NBB_PRECISION_MIXED) {
    st = autotune_mixed_walk(sim);
    if (st) {
      sim->state = nbb_sim::State::failed;
      return st;
    }
  }
  if (sim->cfg.precision == NBB_PRECISION_FP64 && ws.n_systems == 1) {
    st = autotune_fp64_grouping(sim);
    if (st) {
      sim->state = nbb_sim::State::failed;
      return st;
    }
  }
  sim->state = nbb_sim::State::ready;
  return ok();
}

// Capture one step (reset, KD + bbox, Morton + sort + groups, tree,
// traversal + K) into a graph on the handle's own stream.
static cudaError_t capture_step(nbb_sim *sim) {
  Workspace &ws = sim->ws;
  const uint64_t before = nbb::launch_count();
  cudaError_t e = cudaStreamBeginCapture(sim->own_stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t body = enqueue_rebuild_force(ws, traversal_params(sim, 1), sim->cfg.time_step, 1, sim->own_stream);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(sim->own_stream, &graph);
  sim->graph_kernels = nbb::launch_count() - before;
  // kernels recorded during capture did not run; count them per replay
  nbb::count_launches((uint64_t)0 - sim->graph_kernels);
  if (body != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return body;
  }
  if (e != cudaSuccess) return e;
  e = cudaGraphInstantiate(&sim->step_graph, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return e;
  }
  sim->step_graph_def = graph;
  return cudaSuccess;
}

// One step on the handle's stream: the captured graph, or the same kernels.
static cudaError_t enqueue_step(nbb_sim *sim) {
  if (sim->step_graph) {
    nbb::count_launches(sim->graph_kernels);
    return cudaGraphLaunch(sim->step_graph, sim->stream);
  }
  return enqueue_rebuild_force(sim->ws, traversal_params(sim, 1), sim->cfg.time_step, 1, sim->stream);
}

static int run_steps(nbb_sim *sim, uint64_t steps, const char *what) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (sim->state != nbb_sim::State::ready) return fail(NBB_ERR_LOGIC, what);
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  Workspace &ws = sim->ws;
  cudaError_t e = cudaSuccess;
  if (steps > 0 && sim->cfg.use_graph && !sim->step_graph) e = capture_step(sim);
  for (uint64_t k = 0; k < steps && e == cudaSuccess; ++k) e = enqueue_step(sim);
  if (e != cudaSuccess) {
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "step");
  }
  const int st = check_device(ws, sim->stream);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  sim->time += sim->cfg.time_step * (double)steps;
  sim->steps += steps;
  return ok();
}

int nbb_sim_step(nbb_sim *sim) { return run_steps(sim, 1, "Simulation must be initialized before stepping"); }

int nbb_sim_run(nbb_sim *sim, uint64_t steps) {
  return run_steps(sim, steps, "Simulation must be initialized before running");
}

// Capture one part (1..3) of the step into a graph.
static cudaError_t capture_part(nbb_sim *sim, int part, cudaGraph_t &def, cudaGraphExec_t &exec,
                                uint64_t &kernels) {
  const uint64_t before = nbb::launch_count();
  cudaError_t e = cudaStreamBeginCapture(sim->own_stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t body =
      enqueue_rebuild_force(sim->ws, traversal_params(sim, 1), sim->cfg.time_step, 1, sim->own_stream, part);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(sim->own_stream, &graph);
  kernels = nbb::launch_count() - before;
  nbb::count_launches((uint64_t)0 - kernels);
  if (body != cudaSuccess || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return body != cudaSuccess ? body : e;
  }
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return e;
  }
  def = graph;
  return cudaSuccess;
}

static cudaError_t host_step_setup(nbb_sim *sim) {
  if (sim->host_step) return cudaSuccess;
  auto hs = std::make_unique<HostStep>();
  cudaError_t e = cudaStreamCreateWithFlags(&hs->copy, cudaStreamNonBlocking);
  for (cudaEvent_t *ev : {&hs->state_in, &hs->mass_in, &hs->drifted, &hs->copied})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  for (int k = 0; k < HostStep::kParts && e == cudaSuccess && sim->cfg.use_graph; ++k)
    e = capture_part(sim, k + 1, hs->def[k], hs->exec[k], hs->kernels[k]);
  if (e == cudaSuccess) sim->host_step = std::move(hs);
  return e;
}

static cudaError_t enqueue_part(nbb_sim *sim, int part) {
  HostStep &hs = *sim->host_step;
  if (hs.exec[part - 1]) {
    nbb::count_launches(hs.kernels[part - 1]);
    return cudaGraphLaunch(hs.exec[part - 1], sim->stream);
  }
  return enqueue_rebuild_force(sim->ws, traversal_params(sim, 1), sim->cfg.time_step, 1, sim->stream, part);
}

int nbb_sim_step_host(nbb_sim *sim, const double *mass, const double *x, const double *y, const double *z,
                      const double *vx, const double *vy, const double *vz, double *out_x, double *out_y,
                      double *out_z, double *out_vx, double *out_vy, double *out_vz) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (sim->state != nbb_sim::State::ready)
    return fail(NBB_ERR_LOGIC, "Simulation must be initialized before stepping");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  Workspace &ws = sim->ws;
  const size_t bytes = (size_t)ws.n * sizeof(double);
  cudaError_t e = host_step_setup(sim);
  if (e != cudaSuccess) return cuda_fail(e, "host step setup");
  HostStep &hs = *sim->host_step;
  cudaStream_t s = sim->stream;
  // positions and velocities first: the kick-drift needs them
  const double *src[6] = {x, y, z, vx, vy, vz};
  double *dev[6] = {ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz};
  for (int k = 0; k < 6 && e == cudaSuccess; ++k)
    if (src[k]) e = cudaMemcpyAsync(dev[k], src[k], bytes, cudaMemcpyHostToDevice, s);
  // the masses follow on the second stream, under the kick-drift and sort
  if (e == cudaSuccess) e = cudaEventRecord(hs.state_in, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(hs.copy, hs.state_in, 0);
  if (e == cudaSuccess && mass) e = cudaMemcpyAsync(ws.m, mass, bytes, cudaMemcpyHostToDevice, hs.copy);
  if (e == cudaSuccess) e = cudaEventRecord(hs.mass_in, hs.copy);
  if (e == cudaSuccess) e = enqueue_part(sim, 1);
  if (e == cudaSuccess) e = cudaEventRecord(hs.drifted, s);
  if (e == cudaSuccess) e = enqueue_part(sim, 2);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, hs.mass_in, 0);
  // the rest is queued before the positions' copy: a copy to pageable
  // memory returns only when it is done
  if (e == cudaSuccess) e = enqueue_part(sim, 3);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(hs.copy, hs.drifted, 0);
  double *pos[3] = {out_x, out_y, out_z};
  const double *dpos[3] = {ws.x, ws.y, ws.z};
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    if (pos[k]) e = cudaMemcpyAsync(pos[k], dpos[k], bytes, cudaMemcpyDeviceToHost, hs.copy);
  if (e == cudaSuccess) e = cudaEventRecord(hs.copied, hs.copy);
  double *vel[3] = {out_vx, out_vy, out_vz};
  const double *dvel[3] = {ws.vx, ws.vy, ws.vz};
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    if (vel[k]) e = cudaMemcpyAsync(vel[k], dvel[k], bytes, cudaMemcpyDeviceToHost, s);
  // the handle's stream ends after both streams' copies
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, hs.copied, 0);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(hs.copy);
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "host step");
  }
  const int st = check_device(ws, s);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  sim->time += sim->cfg.time_step;
  sim->steps += 1;
  return ok();
}

double nbb_sim_time(const nbb_sim *sim) { return sim ? sim->time : 0.0; }
uint64_t nbb_sim_step_number(const nbb_sim *sim) { return sim ? sim->steps : 0; }

int nbb_sim_state(nbb_sim *sim, nbb_state_view *v) {
  if (!sim || !v) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  const Workspace &ws = sim->ws;
  v->count = (size_t)ws.n;
  v->mass = ws.m; v->x = ws.x; v->y = ws.y; v->z = ws.z;
  v->vx = ws.vx; v->vy = ws.vy; v->vz = ws.vz;
  v->type = ws.type;
  v->ax = ws.ax; v->ay = ws.ay; v->az = ws.az;
  return ok();
}

int nbb_sim_upload(nbb_sim *sim, const double *mass, const double *x, const double *y, const double *z,
                   const double *vx, const double *vy, const double *vz) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  Workspace &ws = sim->ws;
  const size_t bytes = (size_t)ws.n * sizeof(double);
  const double *src[7] = {mass, x, y, z, vx, vy, vz};
  double *dst[7] = {ws.m, ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz};
  for (int k = 0; k < 7; ++k)
    if (src[k]) NBB_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyHostToDevice, sim->stream), "upload");
  return ok();
}

int nbb_sim_download(nbb_sim *sim, double *x, double *y, double *z, double *vx, double *vy, double *vz) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  Workspace &ws = sim->ws;
  const size_t bytes = (size_t)ws.n * sizeof(double);
  double *dst[6] = {x, y, z, vx, vy, vz};
  const double *src[6] = {ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) NBB_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToHost, sim->stream), "download");
  NBB_CUDA(cudaStreamSynchronize(sim->stream), "download synchronisation");
  return ok();
}

int nbb_sim_download_accel(nbb_sim *sim, double *ax, double *ay, double *az) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  Workspace &ws = sim->ws;
  const size_t bytes = (size_t)ws.n * sizeof(double);
  double *dst[3] = {ax, ay, az};
  const double *src[3] = {ws.ax, ws.ay, ws.az};
  for (int k = 0; k < 3; ++k)
    if (dst[k]) NBB_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyDeviceToHost, sim->stream), "download");
  NBB_CUDA(cudaStreamSynchronize(sim->stream), "download synchronisation");
  return ok();
}

int nbb_sim_set_stream(nbb_sim *sim, void *stream) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  sim->stream = stream ? (cudaStream_t)stream : sim->own_stream;
  return ok();
}

int nbb_sim_synchronize(nbb_sim *sim) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  NBB_CUDA(cudaStreamSynchronize(sim->stream), "synchronise");
  return ok();
}

int nbb_sim_destroy(nbb_sim *sim) {
  if (!sim) return ok();
  cudaSetDevice(sim->cfg.device);
  if (sim->stream) cudaStreamSynchronize(sim->stream);
  if (sim->step_graph) cudaGraphExecDestroy(sim->step_graph);
  if (sim->step_graph_def) cudaGraphDestroy(sim->step_graph_def);
  sim->host_step.reset();
  cudaStream_t s = sim->own_stream;
  delete sim;  // frees every device buffer
  if (s) cudaStreamDestroy(s);
  return ok();
}

int nbb_sim_stats(nbb_sim *sim, nbb_stats *stats) {
  if (!sim || !stats) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  DevScalars sc;
  NBB_CUDA(cudaMemcpyAsync(&sc, sim->ws.sc, sizeof(sc), cudaMemcpyDeviceToHost, sim->stream), "stats");
  NBB_CUDA(cudaStreamSynchronize(sim->stream), "stats");
  stats->n_groups = sc.n_groups;
  stats->n_octree_nodes = sc.n_nodes;
  stats->interactions = (int64_t)sc.interactions;
  stats->mac_tests = (int64_t)sc.mac_tests;
  stats->group_size = sim->cfg.precision == NBB_PRECISION_MIXED ? traversal_params(sim, 0).group_size : 0;
  stats->stack_overflow = (int64_t)sc.stack_overflow;
  stats->cache_depth = sim->cfg.precision == NBB_PRECISION_MIXED ? traversal_params(sim, 0).cache_depth : 0;
  return ok();
}

int nbb_sim_profile(nbb_sim *sim, float *stage_ms, nbb_stats *stats) {
  if (!sim || !stage_ms) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  if (sim->state != nbb_sim::State::ready)
    return fail(NBB_ERR_LOGIC, "Simulation must be initialized before profiling");
  Workspace &ws = sim->ws;
  cudaStream_t s = sim->stream;
  cudaEvent_t ev[NBB_PROFILE_STAGES + 1] = {};
  for (auto &e : ev) NBB_CUDA(cudaEventCreate(&e), "cudaEventCreate");
  const TraversalParams tp = traversal_params(sim, 0);
  cudaError_t e = cudaEventRecord(ev[0], s);
  if (e == cudaSuccess) e = launch_step_reset(ws, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev[1], s);
  if (e == cudaSuccess) e = launch_kd_bbox(ws, sim->cfg.time_step, 0, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev[2], s);
  if (e == cudaSuccess) e = launch_morton_sort_groups(ws, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev[3], s);
  if (e == cudaSuccess) e = launch_octree(ws, tp.theta, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev[4], s);
  if (e == cudaSuccess) e = launch_traversal(ws, tp, s);
  if (e == cudaSuccess) e = cudaEventRecord(ev[5], s);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[5]);
  for (int k = 0; k < NBB_PROFILE_STAGES && e == cudaSuccess; ++k) e = cudaEventElapsedTime(&stage_ms[k], ev[k], ev[k + 1]);
  for (auto &x : ev) cudaEventDestroy(x);
  if (e != cudaSuccess) {
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "profile");
  }
  int st = check_device(ws, s);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  if (stats) return nbb_sim_stats(sim, stats);
  return ok();
}

int nbb_sim_export(nbb_sim *sim, nbb_tree_export *out) {
  if (!sim || !out) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  if (sim->state == nbb_sim::State::created)
    return fail(NBB_ERR_LOGIC, "Simulation spatial/device state is not available");
  if (sim->ws.level_order && sim->state == nbb_sim::State::ready) {
    // the steps build the level-order octree: the reference-numbered arrays
    // of the exported tree are rebuilt from the last build's leaf groups
    NBB_CUDA(launch_reference_octree(sim->ws, traversal_params(sim, 0).theta, sim->stream), "tree export");
    const int st = check_device(sim->ws, sim->stream);
    if (st) return st;
  }
  return export_workspace(sim->ws, out, sim->stream, true);
}

// ------------------------------------------------------- function level ---

// A temporary workspace on its own stream for the one-shot entry points.
struct Scratch {
  Workspace ws{};
  Allocation al;
  cudaStream_t s = nullptr;
  ~Scratch() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

int nbb_accel(size_t n, const double *mass, const double *x, const double *y, const double *z, double theta,
              double softening, double g, int precision, double *ax, double *ay, double *az, int on_device,
              nbb_tree_export *export_out, nbb_stats *stats) {
  if (n == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Cannot compute a bounding box for an empty particle set.");
  if (n > (size_t)(INT_MAX / 2)) return fail(NBB_ERR_OVERFLOW, "Particle count exceeds the tree representation");
  if (!mass || !x || !y || !z) return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut particle arrays must not be null");
  if (!finite_nonneg(theta)) return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut theta must be finite and non-negative");
  if (!finite_nonneg(softening))
    return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut softening must be finite and non-negative");
  if (!std::isfinite(g) || g <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Gravitational constant must be finite and positive");
  if (precision != NBB_PRECISION_FP64 && precision != NBB_PRECISION_MIXED)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Unknown traversal precision");
  Scratch sc;
  NBB_CUDA(cudaStreamCreateWithFlags(&sc.s, cudaStreamNonBlocking), "create stream");
  NBB_CUDA(alloc_workspace(sc.ws, sc.al, (int)n, true), "allocate workspace");
  Workspace &ws = sc.ws;
  const cudaMemcpyKind in = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t bytes = n * sizeof(double);
  NBB_CUDA(cudaMemcpyAsync(ws.m, mass, bytes, in, sc.s), "copy mass");
  NBB_CUDA(cudaMemcpyAsync(ws.x, x, bytes, in, sc.s), "copy x");
  NBB_CUDA(cudaMemcpyAsync(ws.y, y, bytes, in, sc.s), "copy y");
  NBB_CUDA(cudaMemcpyAsync(ws.z, z, bytes, in, sc.s), "copy z");
  TraversalParams tp;
  tp.theta = theta;
  tp.soft = softening;
  tp.g = g;
  tp.precision = precision;
  tp.group_mode = default_group_mode(precision);
  NBB_CUDA(enqueue_rebuild_force(ws, tp, 0.0, 0, sc.s), "Barnes-Hut evaluation");
  int st = check_device(ws, sc.s);
  if (st) return st;
  if (ax || ay || az) {
    const cudaMemcpyKind outk = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (ax) NBB_CUDA(cudaMemcpyAsync(ax, ws.ax, bytes, outk, sc.s), "copy ax");
    if (ay) NBB_CUDA(cudaMemcpyAsync(ay, ws.ay, bytes, outk, sc.s), "copy ay");
    if (az) NBB_CUDA(cudaMemcpyAsync(az, ws.az, bytes, outk, sc.s), "copy az");
  }
  if (stats) {
    DevScalars d;
    NBB_CUDA(cudaMemcpyAsync(&d, ws.sc, sizeof(d), cudaMemcpyDeviceToHost, sc.s), "stats");
    NBB_CUDA(cudaStreamSynchronize(sc.s), "stats");
    stats->n_groups = d.n_groups;
    stats->n_octree_nodes = d.n_nodes;
    stats->interactions = (int64_t)d.interactions;
    stats->mac_tests = (int64_t)d.mac_tests;
    stats->group_size = precision == NBB_PRECISION_MIXED ? tp.group_size : 0;
    stats->stack_overflow = (int64_t)d.stack_overflow;
    stats->cache_depth = 0;
  }
  if (export_out) {
    st = export_workspace(ws, export_out, sc.s, true);
    if (st) return st;
  }
  NBB_CUDA(cudaStreamSynchronize(sc.s), "Barnes-Hut evaluation");
  return ok();
}

int nbb_accel_direct(size_t n, const double *mass, const double *x, const double *y, const double *z,
                     int n_targets, const int *targets, double g, double softening, double *ax, double *ay,
                     double *az, int on_device) {
  if (n == 0 || n > (size_t)INT_MAX) return fail(NBB_ERR_INVALID_ARGUMENT, "invalid particle count");
  if (!mass || !x || !y || !z || !ax || !ay || !az) return fail(NBB_ERR_INVALID_ARGUMENT, "null array");
  if (!targets) n_targets = (int)n;
  if (n_targets <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "invalid target count");
  Allocation al;
  cudaStream_t s = nullptr;
  NBB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  const double *dm, *dx, *dy, *dz;
  const int *dt = nullptr;
  cudaError_t e = stage_in(mass, n, on_device, al, dm, s);
  if (e == cudaSuccess) e = stage_in(x, n, on_device, al, dx, s);
  if (e == cudaSuccess) e = stage_in(y, n, on_device, al, dy, s);
  if (e == cudaSuccess) e = stage_in(z, n, on_device, al, dz, s);
  if (e == cudaSuccess && targets) e = stage_in(targets, (size_t)n_targets, on_device, al, dt, s);
  double *oa[3] = {ax, ay, az};
  double *da[3] = {ax, ay, az};
  for (int k = 0; k < 3 && e == cudaSuccess && !on_device; ++k) e = al.get(da[k], (size_t)n_targets);
  double *part = nullptr;
  const int chunks = direct_chunks(n, n_targets);
  if (e == cudaSuccess && chunks > 1) e = al.get(part, (size_t)chunks * 3 * n_targets);
  if (e == cudaSuccess)
    e = launch_direct(n, dm, dx, dy, dz, n_targets, dt, g, softening, da[0], da[1], da[2], part, s);
  for (int k = 0; k < 3 && e == cudaSuccess && !on_device; ++k)
    e = cudaMemcpyAsync(oa[k], da[k], (size_t)n_targets * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return cuda_fail(e, "direct summation");
  return ok();
}

int nbb_accel_octree(const nbb_octree_view *o, const uint32_t *idx, const double *mass, const double *x,
                     const double *y, const double *z, double *ax, double *ay, double *az, double theta,
                     double softening, double g, int particle_order, int on_device) {
  // barnes_hut.cu:325-391 validation
  if (!o || o->n_particles <= 0 || o->n_nodes <= 0)
    return fail(NBB_ERR_LOGIC, "Octree is not valid for Barnes-Hut traversal");
  if (!o->children || !o->parent || !o->first || !o->count)
    return fail(NBB_ERR_LOGIC, "Octree topology arrays required for traversal are not allocated");
  if (!o->mass || !o->comx || !o->comy || !o->comz) return fail(NBB_ERR_LOGIC, "Octree physical data is not allocated");
  if (!o->cx || !o->cy || !o->cz || !o->half) return fail(NBB_ERR_LOGIC, "Octree geometry is not allocated");
  if (!idx || !mass || !x || !y || !z)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut particle arrays must not be null");
  if (!ax || !ay || !az) return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut acceleration arrays must not be null");
  if (!finite_nonneg(theta)) return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut theta must be finite and non-negative");
  if (!finite_nonneg(softening))
    return fail(NBB_ERR_INVALID_ARGUMENT, "Barnes-Hut softening must be finite and non-negative");
  if (!std::isfinite(g) || g <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Gravitational constant must be finite and positive");
  if (particle_order != 0 && particle_order != 1) return fail(NBB_ERR_INVALID_ARGUMENT, "Unknown Barnes-Hut particle order");
  Allocation al;
  cudaStream_t s = nullptr;
  NBB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  const size_t M = (size_t)o->n_nodes, N = (size_t)o->n_particles;
  RefOctree d{};
  d.n_nodes = o->n_nodes;
  d.n_particles = o->n_particles;
  const bool dev = on_device != 0;
  cudaError_t e = stage_in(o->children, 8 * M, dev, al, d.children, s);
  if (e == cudaSuccess) e = stage_in(o->parent, M, dev, al, d.parent, s);
  if (e == cudaSuccess) e = stage_in(o->first, M, dev, al, d.first, s);
  if (e == cudaSuccess) e = stage_in(o->count, M, dev, al, d.count, s);
  if (e == cudaSuccess) e = stage_in(o->mass, M, dev, al, d.mass, s);
  if (e == cudaSuccess) e = stage_in(o->comx, M, dev, al, d.comx, s);
  if (e == cudaSuccess) e = stage_in(o->comy, M, dev, al, d.comy, s);
  if (e == cudaSuccess) e = stage_in(o->comz, M, dev, al, d.comz, s);
  if (e == cudaSuccess) e = stage_in(o->cx, M, dev, al, d.cx, s);
  if (e == cudaSuccess) e = stage_in(o->cy, M, dev, al, d.cy, s);
  if (e == cudaSuccess) e = stage_in(o->cz, M, dev, al, d.cz, s);
  if (e == cudaSuccess) e = stage_in(o->half, M, dev, al, d.half, s);
  const uint32_t *di = nullptr;
  const double *dm = nullptr, *dx = nullptr, *dy = nullptr, *dz = nullptr;
  if (e == cudaSuccess) e = stage_in(idx, N, dev, al, di, s);
  if (e == cudaSuccess) e = stage_in(mass, N, dev, al, dm, s);
  if (e == cudaSuccess) e = stage_in(x, N, dev, al, dx, s);
  if (e == cudaSuccess) e = stage_in(y, N, dev, al, dy, s);
  if (e == cudaSuccess) e = stage_in(z, N, dev, al, dz, s);
  double *oa[3] = {ax, ay, az};
  double *da[3] = {ax, ay, az};
  for (int k = 0; k < 3 && e == cudaSuccess && !dev; ++k) e = al.get(da[k], N);
  int *derr = nullptr;
  if (e == cudaSuccess) e = al.get(derr, 1);
  if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(int), s);
  if (e == cudaSuccess)
    e = launch_ref_octree_traversal(d, di, dm, dx, dy, dz, da[0], da[1], da[2], theta, softening, g,
                                    particle_order, derr, s);
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
  for (int k = 0; k < 3 && e == cudaSuccess && !dev; ++k)
    e = cudaMemcpyAsync(oa[k], da[k], N * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return cuda_fail(e, "computeBarnesHutAccelerationKernel execution");
  if (herr) return fail(NBB_ERR_DEVICE, device_message(kStageTraversal, herr), kStageTraversal * 100 + herr);
  return ok();
}

int nbb_kick_drift(double *x, double *y, double *z, double *vx, double *vy, double *vz, const double *ax,
                   const double *ay, const double *az, size_t n, double dt, void *stream) {
  // integrator.cu:109-126
  if (!std::isfinite(dt) || dt <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog timestep must be finite and positive");
  if (n == 0) return ok();
  if (!x || !y || !z) return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog position arrays must not be null");
  if (!vx || !vy || !vz) return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog velocity arrays must not be null");
  if (!ax || !ay || !az) return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog acceleration arrays must not be null");
  cudaStream_t s = (cudaStream_t)stream;
  NBB_CUDA(launch_kick_drift(x, y, z, vx, vy, vz, ax, ay, az, n, dt, s), "leapfrogKickDriftKernel launch");
  NBB_CUDA(cudaStreamSynchronize(s), "leapfrogKickDriftKernel execution");
  return ok();
}

int nbb_kick(double *vx, double *vy, double *vz, const double *ax, const double *ay, const double *az, size_t n,
             double dt, void *stream) {
  // integrator.cu:129-145
  if (!std::isfinite(dt) || dt <= 0.0)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog timestep must be finite and positive");
  if (n == 0) return ok();
  if (!vx || !vy || !vz) return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog velocity arrays must not be null");
  if (!ax || !ay || !az) return fail(NBB_ERR_INVALID_ARGUMENT, "Leapfrog acceleration arrays must not be null");
  cudaStream_t s = (cudaStream_t)stream;
  NBB_CUDA(launch_kick(vx, vy, vz, ax, ay, az, n, dt, s), "leapfrogKickKernel launch");
  NBB_CUDA(cudaStreamSynchronize(s), "leapfrogKickKernel execution");
  return ok();
}

int nbb_octree_from_keys(const uint32_t *sorted_keys, int n, nbb_tree_export *out) {
  if (n <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "buildMortonLeafGroups requires nParticles >= 1");
  if (!sorted_keys || !out) return fail(NBB_ERR_INVALID_ARGUMENT, "d_sortedKeys must not be null");
  Scratch sc;
  NBB_CUDA(cudaStreamCreateWithFlags(&sc.s, cudaStreamNonBlocking), "create stream");
  NBB_CUDA(alloc_workspace(sc.ws, sc.al, n, false), "allocate workspace");
  sc.ws.pack_shift = 32;  // caller keys may use all 32 bits (rejected by the plan)
  uint32_t *dk = nullptr;
  NBB_CUDA(sc.al.get(dk, (size_t)n), "allocate keys");
  NBB_CUDA(cudaMemcpyAsync(dk, sorted_keys, (size_t)n * 4, cudaMemcpyHostToDevice, sc.s), "copy keys");
  NBB_CUDA(launch_step_reset(sc.ws, sc.s), "reset");
  NBB_CUDA(launch_groups_from_keys(sc.ws, dk, sc.s), "buildMortonLeafGroups");
  NBB_CUDA(launch_topology(sc.ws, sc.s), "octree topology");
  const int st = check_device(sc.ws, sc.s);
  if (st) return st;
  return export_workspace(sc.ws, out, sc.s, false);
}

int nbb_radix_tree(const uint32_t *keys, int n, int *left, int *right, int *rfirst, int *rlast, int *plen,
                   int *parent) {
  if (n <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "buildTree requires N >= 1");
  if (!keys) return fail(NBB_ERR_INVALID_ARGUMENT, "d_sortedKeys must not be null");
  Allocation al;
  cudaStream_t s = nullptr;
  NBB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  uint32_t *dk = nullptr;
  int *dl = nullptr, *dr = nullptr, *df = nullptr, *dla = nullptr, *dp = nullptr, *dpar = nullptr;
  const size_t ni = n > 1 ? (size_t)(n - 1) : 1;
  cudaError_t e = al.get(dk, (size_t)n);
  if (e == cudaSuccess) e = al.get(dl, ni);
  if (e == cudaSuccess) e = al.get(dr, ni);
  if (e == cudaSuccess) e = al.get(df, ni);
  if (e == cudaSuccess) e = al.get(dla, ni);
  if (e == cudaSuccess) e = al.get(dp, ni);
  if (e == cudaSuccess) e = al.get(dpar, (size_t)(2 * n - 1));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys, (size_t)n * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_radix_tree_only(dk, n, dl, dr, df, dla, dp, dpar, s);
  const size_t ib = (size_t)(n - 1) * sizeof(int);
  if (n > 1) {
    if (e == cudaSuccess && left) e = cudaMemcpyAsync(left, dl, ib, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && right) e = cudaMemcpyAsync(right, dr, ib, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && rfirst) e = cudaMemcpyAsync(rfirst, df, ib, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && rlast) e = cudaMemcpyAsync(rlast, dla, ib, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && plen) e = cudaMemcpyAsync(plen, dp, ib, cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess && parent)
    e = cudaMemcpyAsync(parent, dpar, (size_t)(2 * n - 1) * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return cuda_fail(e, "buildTreeKernel execution");
  return ok();
}


}  // extern "C"

// ------------------------------------------- function-level build stages ---

namespace {

// A workspace for one function-level stage: device scalars (zeroed), the
// default stream, every other array aliased to the caller's or taken here.
struct StageRun {
  Workspace ws{};
  Allocation al;
  cudaStream_t s = nullptr;  // the default stream: synchronous as the reference
  cudaError_t init(int n) {
    ws.n = n;
    ws.n_systems = 1;
    ws.sys_levels = 0;
    ws.key_bits = kSpatialBits;
    ws.max_level = kMaxLevel;
    ws.pack_shift = 64 - kSpatialBits;
    ws.sort_passes = kSortPasses;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&ws.num_sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = al.get(ws.sc, 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws.sc, 0, sizeof(DevScalars), s);
    return e;
  }
};

int read_box(const double *box, double out[4]) {
  NBB_CUDA(cudaMemcpy(out, box, 4 * sizeof(double), cudaMemcpyDeviceToHost), "copy bounding box");
  return ok();
}

bool box_valid(const double b[4]) {
  return std::isfinite(b[0]) && std::isfinite(b[1]) && std::isfinite(b[2]) && std::isfinite(b[3]) && b[3] > 0.0;
}

int read_scalar(const int *p, int *out) {
  NBB_CUDA(cudaMemcpy(out, p, sizeof(int), cudaMemcpyDeviceToHost), "copy device count");
  return ok();
}

}  // namespace

extern "C" {

int nbb_bbox(const double *x, const double *y, const double *z, size_t n, double *box) {
  if (n == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Cannot compute a bounding box for an empty particle set.");
  if (n > (size_t)INT_MAX) return fail(NBB_ERR_OVERFLOW, "Particle count exceeds the tree representation");
  if (!x || !y || !z || !box) return fail(NBB_ERR_INVALID_ARGUMENT, "Bounding box device pointers must not be null");
  StageRun st;
  NBB_CUDA(st.init((int)n), "bounding box set-up");
  Workspace &ws = st.ws;
  ws.x = const_cast<double *>(x);
  ws.y = const_cast<double *>(y);
  ws.z = const_cast<double *>(z);
  NBB_CUDA(st.al.get(ws.sys_bb, 6), "bounding box set-up");
  ws.sys_box = box;
  NBB_CUDA(launch_bbox_only(ws, st.s), "Bbox::compute_box");
  return check_device(ws, st.s);
}

int nbb_morton_keys(const double *x, const double *y, const double *z, size_t n, const double *box,
                    uint32_t *keys, uint32_t *idx) {
  // morton.cu:34-60 and :167-170
  if (n == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Cannot compute Morton keys for an empty particle set");
  if (!x || !y || !z) return fail(NBB_ERR_INVALID_ARGUMENT, "Morton coordinate device pointers must not be null");
  if (n > (size_t)INT_MAX) return fail(NBB_ERR_OVERFLOW, "Particle count exceeds the Morton index representation");
  if (!box || !keys || !idx) return fail(NBB_ERR_INVALID_ARGUMENT, "Morton box and output device pointers must not be null");
  double b[4];
  int r = read_box(box, b);
  if (r) return r;
  if (!box_valid(b)) return fail(NBB_ERR_INVALID_ARGUMENT, "Morton bounding box is not valid");
  StageRun st;
  NBB_CUDA(st.init((int)n), "Morton set-up");
  Workspace &ws = st.ws;
  ws.x = const_cast<double *>(x);
  ws.y = const_cast<double *>(y);
  ws.z = const_cast<double *>(z);
  ws.sys_box = const_cast<double *>(box);
  ws.sort_tiles = ((int)n + kSortTile - 1) / kSortTile;
  NBB_CUDA(st.al.get(ws.digit_hist, (size_t)kMaxSortPasses * 256), "Morton set-up");
  NBB_CUDA(st.al.get(ws.sort_status, (size_t)ws.sort_passes * ws.sort_tiles * 256), "Morton set-up");
  NBB_CUDA(st.al.get(ws.pairs_a, n), "Morton set-up");
  NBB_CUDA(st.al.get(ws.pairs_b, n), "Morton set-up");
  NBB_CUDA(launch_morton_sort_box(ws, keys, idx, st.s), "MortonKeys::build");
  return check_device(ws, st.s);
}

int nbb_leaf_groups(const uint32_t *sorted_keys, int n, uint32_t *unique_keys, int *first, int *count,
                    int *n_groups) {
  // morton_leaf_groups.cu:60-70
  if (n <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "buildMortonLeafGroups requires nParticles >= 1");
  if (!sorted_keys) return fail(NBB_ERR_INVALID_ARGUMENT, "d_sortedKeys must not be null");
  if (!unique_keys || !first || !count || !n_groups)
    return fail(NBB_ERR_LOGIC, "MortonLeafGroups memory has not been allocated");
  StageRun st;
  NBB_CUDA(st.init(n), "leaf-group set-up");
  Workspace &ws = st.ws;
  ws.pack_shift = 32;  // caller keys may use all 32 bits
  ws.scan_tiles_n = (n + kScanTile - 1) / kScanTile;
  const size_t N = (size_t)n;
  NBB_CUDA(st.al.get(ws.pairs_a, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.ukey, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.glast, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.keys, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.idx, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.psys, N), "leaf-group set-up");
  NBB_CUDA(st.al.get(ws.scan_status, (size_t)ws.scan_tiles_n), "leaf-group set-up");
  ws.uniq = unique_keys;
  ws.gfirst = first;
  ws.gcount = count;
  NBB_CUDA(launch_leaf_groups(ws, sorted_keys, st.s), "buildMortonLeafGroups");
  int r = check_device(ws, st.s);
  if (r) return r;
  r = read_scalar(&ws.sc->n_groups, n_groups);
  if (r) return r;
  if (*n_groups <= 0 || *n_groups > n)
    return fail(NBB_ERR_DEVICE, "DeviceRunLengthEncode produced an invalid group count");
  return ok();
}

int nbb_radix_tree_device(const uint32_t *keys, int n, int *left, int *right, int *rfirst, int *rlast, int *plen,
                          int *parent) {
  // tree_builder.cu:305-324
  if (n <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "buildTree requires N >= 1");
  if (!parent || (n > 1 && (!left || !right || !rfirst || !rlast || !plen)))
    return fail(NBB_ERR_LOGIC, "Tree memory has not been allocated");
  if (!keys) return fail(NBB_ERR_INVALID_ARGUMENT, "d_sortedKeys must not be null");
  NBB_CUDA(launch_radix_tree_only(keys, n, left, right, rfirst, rlast, plen, parent, nullptr), "buildTreeKernel launch");
  NBB_CUDA(cudaStreamSynchronize(nullptr), "buildTreeKernel execution");
  return ok();
}

int nbb_octree_plan(const uint32_t *unique_keys, int n_groups, const int *plen, const int *parent, int *level,
                    int *count, int *offset, int *n_octree_nodes) {
  // radix_to_octree.cu:176-197
  if (n_groups <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "The radix tree has no leaves");
  if (!unique_keys) return fail(NBB_ERR_LOGIC, "Morton unique keys are not allocated");
  if (!parent) return fail(NBB_ERR_LOGIC, "Radix-tree parent array is not allocated");
  if (!plen && n_groups > 1) return fail(NBB_ERR_LOGIC, "Radix-tree prefix metadata is not allocated");
  if (!level || !count || !offset || !n_octree_nodes)
    return fail(NBB_ERR_LOGIC, "RadixToOctreePlan memory is not allocated");
  StageRun st;
  NBB_CUDA(st.init(n_groups), "plan set-up");
  Workspace &ws = st.ws;
  ws.cap_nodes = INT_MAX;  // the reference's bound: the count must fit in int
  ws.scan_tiles_n = (n_groups + kScanTile - 1) / kScanTile;
  ws.scan_tiles_r = (2 * n_groups - 1 + kScanTile - 1) / kScanTile;
  NBB_CUDA(st.al.get(ws.ukey, (size_t)n_groups), "plan set-up");
  NBB_CUDA(st.al.get(ws.scan_status, (size_t)(ws.scan_tiles_n + ws.scan_tiles_r)), "plan set-up");
  NBB_CUDA(launch_widen_u32(unique_keys, n_groups, ws.ukey, st.s), "plan set-up");
  ws.plen = const_cast<int *>(plen);
  ws.rparent = const_cast<int *>(parent);
  ws.plevel = level;
  ws.pcount = count;
  ws.poffset = offset;
  NBB_CUDA(launch_plan_only(ws, n_groups, st.s), "computeRadixToOctreePlanKernel");
  int r = check_device(ws, st.s);
  if (r) return r;
  return read_scalar(&ws.sc->n_nodes, n_octree_nodes);
}

int nbb_octree_topology(const uint32_t *unique_keys, const int *group_first, const int *group_count, int n_groups,
                        const int *rfirst, const int *parent, const int *plan_level, const int *plan_count,
                        const int *plan_offset, int n_nodes, int *children, int *octree_parent, int *octree_level,
                        uint32_t *octree_prefix, int *first, int *count) {
  // octree_builder.cu:256-286
  if (n_groups <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Morton groups are empty");
  if (!unique_keys || !group_first || !group_count) return fail(NBB_ERR_LOGIC, "Morton group arrays are not allocated");
  if (n_nodes <= 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Radix-to-octree plan has no octree nodes");
  if (!children || !octree_parent || !octree_level || !octree_prefix || !first || !count)
    return fail(NBB_ERR_LOGIC, "Octree topology memory is not allocated");
  if (!parent) return fail(NBB_ERR_LOGIC, "Radix parent array is not allocated");
  if (!rfirst && n_groups > 1) return fail(NBB_ERR_LOGIC, "Radix metadata is incomplete");
  if (!plan_level || !plan_count || !plan_offset) return fail(NBB_ERR_LOGIC, "Radix-to-octree plan arrays are not allocated");
  StageRun st;
  NBB_CUDA(st.init(n_groups), "octree set-up");
  Workspace &ws = st.ws;
  const size_t M = (size_t)n_nodes;
  ws.cap_nodes = n_nodes;
  NBB_CUDA(st.al.get(ws.ukey, (size_t)n_groups), "octree set-up");
  NBB_CUDA(st.al.get(ws.oprefix, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.child_count, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.subtree, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.preoff, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.psub, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.pfirst, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.mass, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.comx, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.comy, M), "octree set-up");
  NBB_CUDA(st.al.get(ws.comz, M), "octree set-up");
  NBB_CUDA(launch_widen_u32(unique_keys, n_groups, ws.ukey, st.s), "octree set-up");
  ws.gfirst = const_cast<int *>(group_first);
  ws.gcount = const_cast<int *>(group_count);
  ws.rfirst = const_cast<int *>(rfirst);
  ws.rparent = const_cast<int *>(parent);
  ws.plevel = const_cast<int *>(plan_level);
  ws.pcount = const_cast<int *>(plan_count);
  ws.poffset = const_cast<int *>(plan_offset);
  ws.children = children;
  ws.oparent = octree_parent;
  ws.olevel = octree_level;
  ws.ofirst = first;
  ws.ocount = count;
  NBB_CUDA(launch_octree_only(ws, n_groups, n_nodes, st.s), "materializeSparseOctreeKernel");
  NBB_CUDA(launch_narrow_u64(ws.oprefix, n_nodes, octree_prefix, st.s), "octree prefixes");
  return check_device(ws, st.s);
}

int nbb_octree_geometry(int n_nodes, const int *level, const uint32_t *prefix, const double *box, double *cx,
                        double *cy, double *cz, double *half) {
  // octree_geometry.cu:139-152
  if (n_nodes <= 0) return fail(NBB_ERR_LOGIC, "Octree topology is not valid");
  if (!level || !prefix) return fail(NBB_ERR_LOGIC, "Octree topology arrays required for geometry are not allocated");
  if (!cx || !cy || !cz || !half) return fail(NBB_ERR_LOGIC, "Octree geometry arrays are not allocated");
  if (!box) return fail(NBB_ERR_INVALID_ARGUMENT, "Bounding box geometry is not valid");
  double b[4];
  int r = read_box(box, b);
  if (r) return r;
  if (!box_valid(b)) return fail(NBB_ERR_INVALID_ARGUMENT, "Bounding box geometry is not valid");
  StageRun st;
  NBB_CUDA(st.init(n_nodes), "geometry set-up");
  Workspace &ws = st.ws;
  NBB_CUDA(st.al.get(ws.oprefix, (size_t)n_nodes), "geometry set-up");
  NBB_CUDA(launch_widen_u32(prefix, n_nodes, ws.oprefix, st.s), "geometry set-up");
  ws.olevel = const_cast<int *>(level);
  ws.sys_box = const_cast<double *>(box);
  ws.cx = cx;
  ws.cy = cy;
  ws.cz = cz;
  ws.half = half;
  NBB_CUDA(launch_geometry_only(ws, n_nodes, st.s), "computeOctreeGeometryKernel");
  return check_device(ws, st.s);
}

int nbb_octree_mass(int n_nodes, int n_particles, const int *children, const int *level, const int *first,
                    const int *count, const uint32_t *sorted_indices, const double *mass, const double *x,
                    const double *y, const double *z, int *child_count, double *node_mass, double *comx,
                    double *comy, double *comz) {
  // octree_physics.cu:283-314
  if (n_nodes <= 0 || n_particles <= 0) return fail(NBB_ERR_LOGIC, "Octree topology is not valid");
  if (!children || !level || !first || !count) return fail(NBB_ERR_LOGIC, "Octree topology arrays are not allocated");
  if (!child_count || !node_mass || !comx || !comy || !comz)
    return fail(NBB_ERR_LOGIC, "Octree physical arrays are not allocated");
  if (!sorted_indices) return fail(NBB_ERR_INVALID_ARGUMENT, "d_sortedIndices must not be null");
  if (!mass || !x || !y || !z) return fail(NBB_ERR_INVALID_ARGUMENT, "Particle arrays must not be null");
  StageRun st;
  NBB_CUDA(st.init(n_particles), "mass set-up");
  Workspace &ws = st.ws;
  const size_t M = (size_t)n_nodes;
  ws.cap_nodes = node_capacity(n_particles, kMaxLevel);
  NBB_CUDA(st.al.get(ws.pm4, (size_t)n_particles), "mass set-up");
  NBB_CUDA(st.al.get(ws.subtree, M), "mass set-up");
  NBB_CUDA(st.al.get(ws.preoff, M), "mass set-up");
  NBB_CUDA(st.al.get(ws.psub, M), "mass set-up");
  NBB_CUDA(st.al.get(ws.pfirst, M), "mass set-up");
  NBB_CUDA(st.al.get(ws.by_level, (size_t)ws.cap_nodes), "mass set-up");
  NBB_CUDA(cudaMemsetAsync(ws.subtree, 0, M * sizeof(int), st.s), "mass set-up");
  NBB_CUDA(cudaMemsetAsync(ws.psub, 0, M * sizeof(int), st.s), "mass set-up");
  NBB_CUDA(cudaMemsetAsync(ws.pfirst, 0x7F, M * sizeof(int), st.s), "mass set-up");
  // octree_physics.cu:302-310: node masses and centres of mass start at zero
  NBB_CUDA(cudaMemsetAsync(node_mass, 0, M * sizeof(double), st.s), "clear octree.mass");
  NBB_CUDA(cudaMemsetAsync(comx, 0, M * sizeof(double), st.s), "clear octree.comX");
  NBB_CUDA(cudaMemsetAsync(comy, 0, M * sizeof(double), st.s), "clear octree.comY");
  NBB_CUDA(cudaMemsetAsync(comz, 0, M * sizeof(double), st.s), "clear octree.comZ");
  NBB_CUDA(cudaMemsetAsync(child_count, 0, M * sizeof(int), st.s), "clear octree.childCount");
  ws.m = const_cast<double *>(mass);
  ws.x = const_cast<double *>(x);
  ws.y = const_cast<double *>(y);
  ws.z = const_cast<double *>(z);
  ws.children = const_cast<int *>(children);
  ws.olevel = const_cast<int *>(level);
  ws.ofirst = const_cast<int *>(first);
  ws.ocount = const_cast<int *>(count);
  ws.child_count = child_count;
  ws.mass = node_mass;
  ws.comx = comx;
  ws.comy = comy;
  ws.comz = comz;
  NBB_CUDA(launch_mass_only(ws, sorted_indices, n_nodes, st.s), "computeOctreeMassAndCenterOfMass");
  return check_device(ws, st.s);
}

int nbb_device_alloc(void **ptr, size_t bytes) {
  if (!ptr) return fail(NBB_ERR_INVALID_ARGUMENT, "nbb_device_alloc: null output pointer");
  *ptr = nullptr;
  if (bytes == 0) return ok();
  NBB_CUDA(cudaMalloc(ptr, bytes), "cudaMalloc");
  return ok();
}

int nbb_device_free(void *ptr) {
  if (ptr) NBB_CUDA(cudaFree(ptr), "cudaFree");
  return ok();
}

int nbb_memcpy(void *dst, const void *src, size_t bytes, int kind) {
  if (bytes == 0) return ok();
  if (!dst || !src) return fail(NBB_ERR_INVALID_ARGUMENT, "nbb_memcpy: null pointer");
  const cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                           : kind == 1 ? cudaMemcpyDeviceToHost
                           : kind == 2 ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault;
  if (kind < 0 || kind > 2) return fail(NBB_ERR_INVALID_ARGUMENT, "nbb_memcpy: kind must be 0, 1 or 2");
  NBB_CUDA(cudaMemcpy(dst, src, bytes, k), "cudaMemcpy");
  return ok();
}

}  // extern "C"

// ---------------------------------------------------------- adjoint ----

namespace {

constexpr int kStateArrays = 9;

double *const *state_arrays(Workspace &ws, double *(&arr)[kStateArrays]) {
  double *a[kStateArrays] = {ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz, ws.ax, ws.ay, ws.az};
  for (int k = 0; k < kStateArrays; ++k) arr[k] = a[k];
  return arr;
}

// Copy the first `count` state arrays between the workspace and a slot of
// contiguous n-arrays (save: workspace -> slot).
cudaError_t copy_state(nbb_sim *sim, double *slot, int count, bool save) {
  Workspace &ws = sim->ws;
  double *arr[kStateArrays];
  state_arrays(ws, arr);
  const size_t n = (size_t)ws.n, bytes = n * sizeof(double);
  for (int k = 0; k < count; ++k) {
    double *dst = save ? slot + k * n : arr[k];
    const double *src = save ? arr[k] : slot + k * n;
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, sim->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Rebuild the tree on the workspace positions and add the VJP of the plain
// FP64 force there to the cotangents.
cudaError_t enqueue_vjp(nbb_sim *sim, const TraversalParams &tpa, const AdjointBuffers &ab) {
  Workspace &ws = sim->ws;
  cudaStream_t s = sim->stream;
  const int group_max = ws.group_max;
  ws.group_max = 32;  // target groups of one warp (kernels take the workspace by value)
  cudaError_t e = launch_step_reset(ws, s);
  if (e == cudaSuccess) e = launch_kd_bbox(ws, 0.0, 0, s);
  if (e == cudaSuccess) e = launch_morton_sort_groups(ws, s);
  if (e == cudaSuccess) e = launch_tree(ws, tpa.theta, s);
  if (e == cudaSuccess) e = launch_adjoint_force(ws, tpa, ab, s);
  ws.group_max = group_max;
  return e;
}

cudaMemcpyKind copy_kind(int on_device, bool to_device) {
  if (on_device) return cudaMemcpyDeviceToDevice;
  return to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
}

}  // namespace

extern "C" {

int nbb_sim_rollout(nbb_sim *sim, uint64_t steps, uint64_t checkpoint_every) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (sim->state != nbb_sim::State::ready)
    return fail(NBB_ERR_LOGIC, "Simulation must be initialized before a rollout");
  if (checkpoint_every == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "checkpoint interval must be positive");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  Workspace &ws = sim->ws;
  const size_t n = (size_t)ws.n;
  const uint64_t slots = steps == 0 ? 1 : (steps - 1) / checkpoint_every + 1;
  const uint64_t seg = std::min<uint64_t>(checkpoint_every, steps > 0 ? steps : 1) - 1;
  const double need = 8.0 * (double)n * (kStateArrays * (double)(slots + 1) + 3.0 * (double)seg + 7.0);
  if (need > 0x1p46) return fail(NBB_ERR_INVALID_ARGUMENT, "rollout checkpoints exceed device memory");
  sim->rollout.reset();
  auto rec = std::make_unique<RolloutRecord>();
  Allocation &al = rec->al;
  cudaError_t e = al.get(rec->ckpt, (size_t)slots * kStateArrays * n);
  if (e == cudaSuccess) e = al.get(rec->final_state, kStateArrays * n);
  if (e == cudaSuccess) e = al.get(rec->seg, (size_t)(seg > 0 ? seg : 1) * 3 * n);
  if (e == cudaSuccess) e = al.get(rec->g, 7 * n);
  if (e == cudaSuccess) e = al.get(rec->node_g, (size_t)ws.cap_nodes);
  if (e == cudaSuccess) e = al.get(rec->part_g, n);
  if (e == cudaSuccess) e = al.get(rec->tgt_g, n);
  if (e == cudaSuccess) e = al.get(rec->pparent, (size_t)ws.cap_nodes);
  if (e == cudaSuccess) e = al.get(rec->prange, (size_t)ws.cap_nodes);
  if (e != cudaSuccess) return cuda_fail(e, "rollout checkpoint allocation");
  if (steps > 0 && sim->cfg.use_graph && !sim->step_graph) e = capture_step(sim);
  if (e == cudaSuccess) e = copy_state(sim, rec->ckpt, kStateArrays, true);
  for (uint64_t k = 0; k < steps && e == cudaSuccess; ++k) {
    e = enqueue_step(sim);
    if (e == cudaSuccess && (k + 1) % checkpoint_every == 0 && k + 1 < steps)
      e = copy_state(sim, rec->ckpt + (size_t)((k + 1) / checkpoint_every) * kStateArrays * n, kStateArrays,
                     true);
  }
  if (e != cudaSuccess) {
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "rollout");
  }
  const int st = check_device(ws, sim->stream);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  rec->steps = steps;
  rec->every = checkpoint_every;
  rec->slots = slots;
  sim->rollout = std::move(rec);
  sim->time += sim->cfg.time_step * (double)steps;
  sim->steps += steps;
  return ok();
}

int nbb_sim_backward(nbb_sim *sim, const double *gx, const double *gy, const double *gz, const double *gvx,
                     const double *gvy, const double *gvz, double *gm, double *gx0, double *gy0, double *gz0,
                     double *gvx0, double *gvy0, double *gvz0, int on_device) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (sim->state != nbb_sim::State::ready)
    return fail(NBB_ERR_LOGIC, "Simulation must be initialized before a backward pass");
  if (!sim->rollout) return fail(NBB_ERR_LOGIC, "backward pass without a recorded rollout");
  if (!gx || !gy || !gz) return fail(NBB_ERR_INVALID_ARGUMENT, "final-position cotangents are required");
  if ((gvx || gvy || gvz) && !(gvx && gvy && gvz))
    return fail(NBB_ERR_INVALID_ARGUMENT, "velocity cotangents must be all given or all null");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  Workspace &ws = sim->ws;
  RolloutRecord &rec = *sim->rollout;
  cudaStream_t s = sim->stream;
  const size_t n = (size_t)ws.n, bytes = n * sizeof(double);
  double *G[7];
  for (int k = 0; k < 7; ++k) G[k] = rec.g + k * n;
  const double *gin[6] = {gx, gy, gz, gvx, gvy, gvz};
  for (int k = 0; k < 6; ++k) {
    if (gin[k]) {
      NBB_CUDA(cudaMemcpyAsync(G[k], gin[k], bytes, copy_kind(on_device, true), s), "copy cotangents");
    } else {
      NBB_CUDA(cudaMemsetAsync(G[k], 0, bytes, s), "clear cotangents");
    }
  }
  NBB_CUDA(cudaMemsetAsync(G[6], 0, bytes, s), "clear cotangents");
  const uint64_t S = rec.steps, K = rec.every;
  const double dt = sim->cfg.time_step;
  AdjointBuffers ab;
  ab.gx = G[0];
  ab.gy = G[1];
  ab.gz = G[2];
  ab.gvx = G[3];
  ab.gvy = G[4];
  ab.gvz = G[5];
  ab.gm = G[6];
  ab.node_g = rec.node_g;
  ab.part_g = rec.part_g;
  ab.tgt_g = rec.tgt_g;
  ab.pparent = rec.pparent;
  ab.prange = rec.prange;
  // the VJP of the force the rollout ran: the plain form's, or the mixed
  // form's on its own interaction lists (32-target groups)
  TraversalParams tpa = traversal_params(sim, 0);
  tpa.precision = sim->cfg.precision == NBB_PRECISION_MIXED ? 1 : 0;
  tpa.kick = 0;
  tpa.group_mode = 1;  // compact warps; the plain form's sums do not depend on it
  tpa.group_size = 32;
  tpa.cache_depth = 0;
  cudaError_t e = cudaSuccess;
  if (S > 0) {
    // the step s -> s+1 is undone by the VJP at x_{s+1} with accelerations
    // cotangent (1/2 dt at the last step, dt inside) times gv, then gv += dt gx
    e = copy_state(sim, rec.final_state, kStateArrays, true);
    for (uint64_t j = rec.slots; j-- > 0 && e == cudaSuccess;) {
      const uint64_t lo = j * K, hi = std::min(lo + K, S);
      e = copy_state(sim, rec.ckpt + (size_t)j * kStateArrays * n, kStateArrays, false);
      for (uint64_t t = lo + 1; t < hi && e == cudaSuccess; ++t) {
        e = enqueue_step(sim);
        if (e == cudaSuccess) e = copy_state(sim, rec.seg + (size_t)(t - lo - 1) * 3 * n, 3, true);
      }
      for (uint64_t t = hi; t > lo && e == cudaSuccess; --t) {
        double *pos = (t < hi) ? rec.seg + (size_t)(t - lo - 1) * 3 * n
                               : (hi == S ? rec.final_state : rec.ckpt + (size_t)(j + 1) * kStateArrays * n);
        e = copy_state(sim, pos, 3, false);
        ab.coef = (t == S) ? 0.5 * dt : dt;
        ab.dt_v = dt;
        if (e == cudaSuccess) e = enqueue_vjp(sim, tpa, ab);
      }
    }
    if (e == cudaSuccess) e = copy_state(sim, rec.ckpt, 3, false);
    ab.coef = 0.5 * dt;  // a_0 = F(x_0) enters through the first half kick only
    ab.dt_v = 0.0;
    if (e == cudaSuccess) e = enqueue_vjp(sim, tpa, ab);
    if (e == cudaSuccess) e = copy_state(sim, rec.final_state, kStateArrays, false);
  }
  if (e != cudaSuccess) {
    sim->state = nbb_sim::State::failed;
    return cuda_fail(e, "backward pass");
  }
  const int st = check_device(ws, s);
  if (st) {
    sim->state = nbb_sim::State::failed;
    return st;
  }
  double *outs[7] = {gx0, gy0, gz0, gvx0, gvy0, gvz0, gm};
  for (int k = 0; k < 7; ++k)
    if (outs[k]) NBB_CUDA(cudaMemcpyAsync(outs[k], G[k], bytes, copy_kind(on_device, false), s), "copy gradients");
  NBB_CUDA(cudaStreamSynchronize(s), "backward synchronisation");
  return ok();
}

int nbb_frozen_rollout(const nbb_config *cfg, size_t n, const double *mass, const double *x, const double *y,
                       const double *z, const double *vx, const double *vy, const double *vz, size_t copies,
                       const double *cmass, const double *cx, const double *cy, const double *cz,
                       const double *cvx, const double *cvy, const double *cvz, uint64_t steps, double *ox,
                       double *oy, double *oz, double *ovx, double *ovy, double *ovz, int on_device) {
  if (!cfg) return fail(NBB_ERR_INVALID_ARGUMENT, "null configuration");
  if (copies == 0 || copies > 4096) return fail(NBB_ERR_INVALID_ARGUMENT, "copies must be in [1, 4096]");
  if (!cx || !cy || !cz || !cvx || !cvy || !cvz)
    return fail(NBB_ERR_INVALID_ARGUMENT, "perturbed positions and velocities are required");
  nbb_config c2 = *cfg;
  c2.precision = NBB_PRECISION_FP64;
  c2.use_graph = 0;
  nbb_sim *sim = nullptr;
  int st = create_sim(&c2, n, 1, nullptr, nullptr, mass, x, y, z, vx, vy, vz, nullptr, on_device, &sim);
  if (st) return st;
  std::unique_ptr<nbb_sim, int (*)(nbb_sim *)> guard(sim, nbb_sim_destroy);
  // the frozen walk reads the octree in the reference numbering
  sim->ws.level_order = 0;
  st = nbb_sim_initialize(sim);
  if (st) return st;
  Workspace &ws = sim->ws;
  cudaStream_t s = sim->stream;
  const size_t bytes = n * sizeof(double), qn = copies * n, qcap = copies * (size_t)ws.cap_nodes;
  Allocation al;
  FrozenBatch fb;
  fb.copies = (int)copies;
  double **fields[10] = {&fb.m, &fb.x, &fb.y, &fb.z, &fb.vx, &fb.vy, &fb.vz, &fb.ax, &fb.ay, &fb.az};
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 10 && e == cudaSuccess; ++k) e = al.get(*fields[k], qn);
  if (e == cudaSuccess) e = al.get(fb.pm4q, qn);
  if (e == cudaSuccess) e = al.get(fb.aq_oct, qcap);
  if (e == cudaSuccess) e = al.get(fb.node_aq, qcap);
  if (e == cudaSuccess) e = al.get(fb.pre_of, (size_t)ws.cap_nodes);
  if (e == cudaSuccess) e = al.get(fb.pparent, (size_t)ws.cap_nodes);
  if (e == cudaSuccess) e = al.get(fb.prange, (size_t)ws.cap_nodes);
  const double *src[7] = {cmass, cx, cy, cz, cvx, cvy, cvz};
  for (int k = 0; k < 7 && e == cudaSuccess; ++k) {
    if (src[k]) {
      e = cudaMemcpyAsync(*fields[k], src[k], copies * bytes, copy_kind(on_device, true), s);
    } else {
      for (size_t q = 0; q < copies && e == cudaSuccess; ++q)
        e = cudaMemcpyAsync(*fields[k] + q * n, ws.m, bytes, cudaMemcpyDeviceToDevice, s);
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "frozen rollout setup");
  const TraversalParams tp = traversal_params(sim, 0);
  const double dt = c2.time_step;
  e = launch_frozen_force(ws, tp, fb, s);
  for (uint64_t k = 0; k < steps && e == cudaSuccess; ++k) {
    e = launch_kick_drift(fb.x, fb.y, fb.z, fb.vx, fb.vy, fb.vz, fb.ax, fb.ay, fb.az, qn, dt, s);
    if (e == cudaSuccess) e = enqueue_rebuild_force(ws, traversal_params(sim, 1), dt, 1, s);
    if (e == cudaSuccess) e = launch_frozen_force(ws, tp, fb, s);
    if (e == cudaSuccess) e = launch_kick(fb.vx, fb.vy, fb.vz, fb.ax, fb.ay, fb.az, qn, dt, s);
  }
  if (e != cudaSuccess) return cuda_fail(e, "frozen rollout");
  st = check_device(ws, s);
  if (st) return st;
  double *outs[6] = {ox, oy, oz, ovx, ovy, ovz};
  const double *from[6] = {fb.x, fb.y, fb.z, fb.vx, fb.vy, fb.vz};
  for (int k = 0; k < 6; ++k)
    if (outs[k])
      NBB_CUDA(cudaMemcpyAsync(outs[k], from[k], copies * bytes, copy_kind(on_device, false), s),
               "copy frozen rollout state");
  NBB_CUDA(cudaStreamSynchronize(s), "frozen rollout synchronisation");
  return ok();
}

int nbb_direct_rollout_adjoint(const nbb_config *cfg, size_t n, const double *mass, const double *x,
                               const double *y, const double *z, const double *vx, const double *vy,
                               const double *vz, uint64_t steps, const double *gx, const double *gy,
                               const double *gz, const double *gvx, const double *gvy, const double *gvz,
                               double *ox, double *oy, double *oz, double *ovx, double *ovy, double *ovz,
                               double *gm, double *gx0, double *gy0, double *gz0, double *gvx0, double *gvy0,
                               double *gvz0, int on_device) {
  if (!cfg) return fail(NBB_ERR_INVALID_ARGUMENT, "null configuration");
  int st = validate_config(cfg);
  if (st) return st;
  if (n == 0 || n > (size_t)INT_MAX) return fail(NBB_ERR_INVALID_ARGUMENT, "particle count out of range");
  if (!mass || !x || !y || !z || !vx || !vy || !vz || !gx || !gy || !gz)
    return fail(NBB_ERR_INVALID_ARGUMENT, "state and final-position cotangents are required");
  if ((gvx || gvy || gvz) && !(gvx && gvy && gvz))
    return fail(NBB_ERR_INVALID_ARGUMENT, "velocity cotangents must be all given or all null");
  const double need = 8.0 * (double)n * (3.0 * (double)(steps + 1) + 17.0);
  if (need > 0x1p34) return fail(NBB_ERR_INVALID_ARGUMENT, "the direct adjoint's stored trajectory exceeds 16 GiB");
  NBB_CUDA(cudaSetDevice(cfg->device), "cudaSetDevice");
  cudaStream_t s = nullptr;
  NBB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  std::unique_ptr<CUstream_st, cudaError_t (*)(cudaStream_t)> sguard(s, cudaStreamDestroy);
  Allocation al;
  const size_t bytes = n * sizeof(double);
  double *traj = nullptr, *st10 = nullptr, *g = nullptr;
  cudaError_t e = al.get(traj, (size_t)(steps + 1) * 3 * n);
  if (e == cudaSuccess) e = al.get(st10, 10 * n);
  if (e == cudaSuccess) e = al.get(g, 7 * n);
  if (e != cudaSuccess) return cuda_fail(e, "direct adjoint allocation");
  double *M = st10, *X = st10 + n, *Y = st10 + 2 * n, *Z = st10 + 3 * n, *VX = st10 + 4 * n,
         *VY = st10 + 5 * n, *VZ = st10 + 6 * n, *AX = st10 + 7 * n, *AY = st10 + 8 * n, *AZ = st10 + 9 * n;
  const double *in[7] = {mass, x, y, z, vx, vy, vz};
  double *dst[7] = {M, X, Y, Z, VX, VY, VZ};
  for (int k = 0; k < 7; ++k)
    NBB_CUDA(cudaMemcpyAsync(dst[k], in[k], bytes, copy_kind(on_device, true), s), "copy state");
  const double dt = cfg->time_step, G = cfg->gravitational_constant, eps = cfg->softening;
  auto store = [&](uint64_t t) -> cudaError_t {
    double *slot = traj + (size_t)t * 3 * n;
    cudaError_t r = cudaMemcpyAsync(slot, X, bytes, cudaMemcpyDeviceToDevice, s);
    if (r == cudaSuccess) r = cudaMemcpyAsync(slot + n, Y, bytes, cudaMemcpyDeviceToDevice, s);
    if (r == cudaSuccess) r = cudaMemcpyAsync(slot + 2 * n, Z, bytes, cudaMemcpyDeviceToDevice, s);
    return r;
  };
  e = store(0);
  if (e == cudaSuccess) e = launch_direct(n, M, X, Y, Z, (int)n, nullptr, G, eps, AX, AY, AZ, nullptr, s);
  for (uint64_t t = 1; t <= steps && e == cudaSuccess; ++t) {
    e = launch_kick_drift(X, Y, Z, VX, VY, VZ, AX, AY, AZ, n, dt, s);
    if (e == cudaSuccess) e = launch_direct(n, M, X, Y, Z, (int)n, nullptr, G, eps, AX, AY, AZ, nullptr, s);
    if (e == cudaSuccess) e = launch_kick(VX, VY, VZ, AX, AY, AZ, n, dt, s);
    if (e == cudaSuccess) e = store(t);
  }
  double *Gc[7];
  for (int k = 0; k < 7; ++k) Gc[k] = g + k * n;
  const double *gin[6] = {gx, gy, gz, gvx, gvy, gvz};
  for (int k = 0; k < 6 && e == cudaSuccess; ++k)
    e = gin[k] ? cudaMemcpyAsync(Gc[k], gin[k], bytes, copy_kind(on_device, true), s)
               : cudaMemsetAsync(Gc[k], 0, bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(Gc[6], 0, bytes, s);
  for (uint64_t t = steps; t >= 1 && e == cudaSuccess; --t) {
    const double *slot = traj + (size_t)t * 3 * n;
    e = launch_direct_vjp(n, M, slot, slot + n, slot + 2 * n, Gc[3], Gc[4], Gc[5], t == steps ? 0.5 * dt : dt, G,
                          eps, Gc[0], Gc[1], Gc[2], Gc[6], s);
    if (e == cudaSuccess) e = launch_axpy3(Gc[3], Gc[4], Gc[5], Gc[0], Gc[1], Gc[2], dt, n, s);
  }
  if (steps > 0 && e == cudaSuccess)
    e = launch_direct_vjp(n, M, traj, traj + n, traj + 2 * n, Gc[3], Gc[4], Gc[5], 0.5 * dt, G, eps, Gc[0], Gc[1],
                          Gc[2], Gc[6], s);
  double *outs[13] = {ox, oy, oz, ovx, ovy, ovz, gx0, gy0, gz0, gvx0, gvy0, gvz0, gm};
  const double *from[13] = {X, Y, Z, VX, VY, VZ, Gc[0], Gc[1], Gc[2], Gc[3], Gc[4], Gc[5], Gc[6]};
  for (int k = 0; k < 13 && e == cudaSuccess; ++k)
    if (outs[k]) e = cudaMemcpyAsync(outs[k], from[k], bytes, copy_kind(on_device, false), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "direct adjoint");
  return ok();
}

}  // extern "C"

// ------------------------------------------------------ frame capture ----

namespace {

size_t frame_samples(size_t n, size_t max_particles) {
  return (max_particles == 0 || max_particles > n) ? n : max_particles;
}

}  // namespace

extern "C" {

size_t nbb_frame_bytes(const nbb_sim *sim, size_t max_particles) {
  if (!sim) return 0;
  return (size_t)kFrameHeaderBytes + 7 * frame_samples((size_t)sim->ws.n, max_particles);
}

int nbb_sim_capture_frame(nbb_sim *sim, size_t max_particles, uint64_t sequence, void *out, size_t capacity,
                          size_t *written, int on_device) {
  if (!sim) return fail(NBB_ERR_INVALID_ARGUMENT, "null simulation");
  if (!out) return fail(NBB_ERR_INVALID_ARGUMENT, "null frame buffer");
  if (sim->state == nbb_sim::State::failed) return fail(NBB_ERR_LOGIC, "Simulation is in a failed state");
  if (!std::isfinite(sim->time) || sim->time < 0.0) return fail(NBB_ERR_INVALID_ARGUMENT, "Frame simulation time is invalid");
  const size_t n = (size_t)sim->ws.n;
  const size_t s = frame_samples(n, max_particles);
  const size_t bytes = (size_t)kFrameHeaderBytes + 7 * s;
  if (capacity < bytes) return fail(NBB_ERR_INVALID_ARGUMENT, "frame buffer is smaller than nbb_frame_bytes()");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  if (!sim->frames || sim->frames->bytes < bytes) {
    auto fb = std::make_unique<FrameBuffers>();
    NBB_CUDA(fb->al.get(fb->frame, bytes), "Could not allocate the quantized sampling buffer");
    NBB_CUDA(fb->al.get(fb->scalars, 1), "Could not allocate the sampling bounds buffer");
    fb->bytes = bytes;
    sim->frames = std::move(fb);
  }
  FrameBuffers &fb = *sim->frames;
  const Workspace &ws = sim->ws;
  cudaStream_t st = sim->stream;
  FrameHeaderFields h;
  h.sequence = sequence;
  h.step = sim->steps;
  h.time = sim->time;
  h.source_count = n;
  h.sample_count = s;
  NBB_CUDA(launch_frame_capture(ws.x, ws.y, ws.z, ws.type, n, s, fb.scalars, h, fb.frame, st),
           "Could not launch the graphical quantization kernel");
  FrameScalars f;
  NBB_CUDA(cudaMemcpyAsync(&f, fb.scalars, sizeof(f), cudaMemcpyDeviceToHost, st), "Could not validate graphical samples");
  NBB_CUDA(cudaStreamSynchronize(st), "Could not validate graphical samples");
  if (f.nonfinite) return fail(NBB_ERR_DOMAIN, "Cannot quantize a graphical frame with non-finite positions");
  if (f.bad_type) return fail(NBB_ERR_INVALID_ARGUMENT, "Cannot capture a frame with invalid particle types");
  for (int a = 0; a < 3; ++a) {
    double lo, hi;
    const unsigned long long bl = f.lo[a], bh = f.hi[a];
    // decode the order-preserving encoding (the inverse of order_bits)
    const unsigned long long rl = (bl >> 63) ? (bl & 0x7FFFFFFFFFFFFFFFull) : ~bl;
    const unsigned long long rh = (bh >> 63) ? (bh & 0x7FFFFFFFFFFFFFFFull) : ~bh;
    std::memcpy(&lo, &rl, sizeof(lo));
    std::memcpy(&hi, &rh, sizeof(hi));
    if (!std::isfinite(lo) || !std::isfinite(hi) || lo > hi || !std::isfinite(hi - lo))
      return fail(NBB_ERR_INVALID_ARGUMENT, "Position frame bounds must be finite and ordered");
  }
  NBB_CUDA(cudaMemcpyAsync(out, fb.frame, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st),
           "Could not copy quantized samples to the frame writer");
  NBB_CUDA(cudaStreamSynchronize(st), "Could not copy quantized samples to the frame writer");
  if (written) *written = bytes;
  return ok();
}

}  // extern "C"

// -------------------------------------------------- conserved quantities --

extern "C" {

int nbb_sim_diagnostics(nbb_sim *sim, int potential, nbb_diagnostics *d) {
  if (!sim || !d) return fail(NBB_ERR_INVALID_ARGUMENT, "null argument");
  if (potential < NBB_POTENTIAL_NONE || potential > NBB_POTENTIAL_DIRECT)
    return fail(NBB_ERR_INVALID_ARGUMENT, "unknown potential mode");
  if (sim->state == nbb_sim::State::failed) return fail(NBB_ERR_LOGIC, "Simulation is in a failed state");
  Workspace &ws = sim->ws;
  if (potential == NBB_POTENTIAL_DIRECT && ws.n_systems > 1)
    return fail(NBB_ERR_INVALID_ARGUMENT, "direct potential of an ensemble is not defined; use the tree potential");
  NBB_CUDA(cudaSetDevice(sim->cfg.device), "cudaSetDevice");
  const size_t n = (size_t)ws.n;
  if (!sim->diag) {
    auto db = std::make_unique<DiagBuffers>();
    NBB_CUDA(db->al.get(db->partials, (size_t)DiagBuffers::kBlocks * 12), "diagnostics allocation");
    NBB_CUDA(db->al.get(db->out, 12), "diagnostics allocation");
    NBB_CUDA(db->al.get(db->phi, n), "diagnostics allocation");
    sim->diag = std::move(db);
  }
  DiagBuffers &db = *sim->diag;
  cudaStream_t s = sim->stream;
  const double *phi = nullptr;
  if (potential == NBB_POTENTIAL_TREE) {
    // the tree of the current positions (the handle's last tree may belong
    // to other positions, e.g. after a backward pass)
    TraversalParams tp = traversal_params(sim, 0);
    tp.precision = 0;
    tp.group_mode = 1;
    const int group_max = ws.group_max;
    ws.group_max = 32;  // target groups of one warp
    cudaError_t e = launch_step_reset(ws, s);
    if (e == cudaSuccess) e = launch_kd_bbox(ws, 0.0, 0, s);
    if (e == cudaSuccess) e = launch_morton_sort_groups(ws, s);
    if (e == cudaSuccess) e = launch_tree(ws, tp.theta, s);
    if (e == cudaSuccess) e = launch_potential_tree(ws, tp, db.phi, s);
    ws.group_max = group_max;
    NBB_CUDA(e, "potential evaluation");
    phi = db.phi;
  } else if (potential == NBB_POTENTIAL_DIRECT) {
    NBB_CUDA(launch_potential_direct(ws.m, ws.x, ws.y, ws.z, (int)n, sim->cfg.gravitational_constant,
                                     sim->cfg.softening, db.phi, s),
             "potential evaluation");
    phi = db.phi;
  }
  NBB_CUDA(launch_moments(ws.m, ws.x, ws.y, ws.z, ws.vx, ws.vy, ws.vz, phi, n, db.partials, DiagBuffers::kBlocks,
                          db.out, s),
           "moments");
  double h[12];
  NBB_CUDA(cudaMemcpyAsync(h, db.out, sizeof(h), cudaMemcpyDeviceToHost, s), "copy diagnostics");
  const int st = check_device(ws, s);
  if (st) return st;
  d->mass = h[0];
  for (int a = 0; a < 3; ++a) {
    d->center_of_mass[a] = h[0] != 0.0 ? h[1 + a] / h[0] : 0.0;
    d->momentum[a] = h[4 + a];
    d->angular_momentum[a] = h[7 + a];
  }
  d->kinetic_energy = h[10];
  d->potential_energy = potential ? h[11] : 0.0;
  d->total_energy = d->kinetic_energy + d->potential_energy;
  d->potential = potential;
  return ok();
}

}  // extern "C"
