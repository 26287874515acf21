// traverse.cu -- Barnes-Hut force evaluation on sm_100a.
//
//  traverse_fp64_kernel   plain form of barnes_hut.cu:164-322 (paths relative
//                         to the sytrams/AMSC-Nbody project root): per-target
//                         acceptance test and interaction order identical to
//                         the reference, FP64 throughout.
//  traverse_mixed_kernel  mixed form: warp-group acceptance test, shared
//                         interaction lists evaluated in FP32.
//  direct_kernel          FP64 direct summation (theta-error oracle).
//  ref_octree_kernel      traversal of a caller octree in the reference's own
//                         node numbering (function-level API).
//  kick / kick_drift      integrator.cu:51-106.
#include "nbb_internal.cuh"
#include "walk_fp64.cuh"

#include <algorithm>
#include <climits>
#include <cmath>

namespace nbb {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ long long warp_sum_ll(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Plain FP64 traversal, one warp per 32 Morton-consecutive targets.
//
// The tree is laid out in depth-first preorder with children visited octant
// 7 -> 0, so the reference's per-thread stackless walk (barnes_hut.cu:90-162)
// becomes: a target opened at node i continues at i + 1, a target done with
// node i (accepted, zero mass, or a leaf) continues at skip(i).  Each lane
// keeps its own resume index and the warp always visits the smallest one, so
// every lane sees exactly its own node sequence -- the reference's
// interaction set in the reference's order -- while node records are fetched
// once per warp (broadcast loads) instead of once per thread.
__global__ void __launch_bounds__(256) traverse_fp64_kernel(Workspace ws, TraversalParams p) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int lane = threadIdx.x & 31;
  const int n = ws.n;
  const int m = sc->n_nodes;
  const int n_groups = p.group_mode ? sc->n_tgroups : (n + 31) >> 5;
  const double g = p.g;
  long long inter = 0, tests = 0;
  bool singular = false;
  while (true) {
    int grp = 0;
    if (lane == 0) grp = (int)atomicAdd(&sc->work_counter, 1u);
    grp = __shfl_sync(kFull, grp, 0);
    if (grp >= n_groups) break;
    const int g0 = p.group_mode ? ws.tstart[grp] : grp * 32;
    const int g1 = p.group_mode ? ((grp + 1 < n_groups) ? ws.tstart[grp + 1] : n) : min(g0 + 32, n);
    // a group larger than a warp is walked 32 targets at a time
    for (int c0 = g0; c0 < g1; c0 += 32) {
      const int c1 = min(c0 + 32, g1);
      const int s = c0 + lane;
      const bool valid = s < c1 && s < n;
      double4 t = make_double4(0.0, 0.0, 0.0, 0.0);
      if (valid) t = ws.pm4[s];
      // a warp's targets belong to one system: walk that system's subtree
      const int sys = ws.n_systems > 1 ? ws.psys[g0] : 0;
      const int root = ws.root_pre[sys];
      const int end = (root >= 0 && root < m) ? min(ws.node_meta[root].x, m) : 0;
      const double soft = ws.sys_eps ? ws.sys_eps[sys] : p.soft;
      const double soft2 = __dmul_rn(soft, soft);
      double ax = 0.0, ay = 0.0, az = 0.0;
      int resume = valid ? root : INT_MAX;
      int node = __reduce_min_sync(kFull, resume);
      while (node < end) {
        // every record of the node in one round trip (warp-uniform address:
        // one broadcast transaction each)
        const int4 meta = ws.node_meta[node];
        const double4 a = ws.node_a[node];
        const double4 c = ws.node_c[node];
        if (resume == node) {
          if (meta.z > 0) {
            // occupied leaf: exact sum over its particles, self excluded
            // (barnes_hut.cu:204-257).  Two particles at a time: their square
            // roots and divisions are independent and overlap; the sums
            // still take them in the reference's order.
            int k = 0;
            for (; k + 1 < meta.z; k += 2) {
              const int s0 = meta.y + k, s1 = s0 + 1;
              const double4 q0 = ws.pm4[s0], q1 = ws.pm4[s1];
              const double dx0 = __dsub_rn(q0.x, t.x), dy0 = __dsub_rn(q0.y, t.y), dz0 = __dsub_rn(q0.z, t.z);
              const double dx1 = __dsub_rn(q1.x, t.x), dy1 = __dsub_rn(q1.y, t.y), dz1 = __dsub_rn(q1.z, t.z);
              double f0, f1;
              const bool ok0 = point_mass_factor(sqdist(dx0, dy0, dz0), q0.w, g, soft2, f0);
              const bool ok1 = point_mass_factor(sqdist(dx1, dy1, dz1), q1.w, g, soft2, f1);
              if (s0 != s && q0.w != 0.0) {
                singular |= !ok0;
                if (ok0) {
                  ax = __fma_rn(f0, dx0, ax);
                  ay = __fma_rn(f0, dy0, ay);
                  az = __fma_rn(f0, dz0, az);
                }
                ++inter;
              }
              if (s1 != s && q1.w != 0.0) {
                singular |= !ok1;
                if (ok1) {
                  ax = __fma_rn(f1, dx1, ax);
                  ay = __fma_rn(f1, dy1, ay);
                  az = __fma_rn(f1, dz1, az);
                }
                ++inter;
              }
            }
            if (k < meta.z) {
              const int sp = meta.y + k;
              const double4 q = ws.pm4[sp];
              if (sp != s && q.w != 0.0) {
                const double dx = __dsub_rn(q.x, t.x), dy = __dsub_rn(q.y, t.y), dz = __dsub_rn(q.z, t.z);
                singular |= !point_mass_fp64(dx, dy, dz, sqdist(dx, dy, dz), q.w, g, soft2, ax, ay, az);
                ++inter;
              }
            }
            resume = meta.x;
          } else if (a.w == 0.0) {
            resume = meta.x;  // zero-mass node (barnes_hut.cu:259-271)
          } else {
            double dx, dy, dz, d2;
            const bool accept = accept_fp64(a, ws.node_b + node, c, t, dx, dy, dz, d2);
            ++tests;
            if (accept) {
              singular |= !point_mass_fp64(dx, dy, dz, d2, a.w, g, soft2, ax, ay, az);
              ++inter;
              resume = meta.x;
            } else {
              resume = node + 1;
            }
          }
        }
        // a lane's resume index always moves forward (skip > node); this keeps
        // the walk finite whatever the node records hold
        if (resume <= node) resume = node + 1;
        node = __reduce_min_sync(kFull, resume);
      }
      if (valid) {
        const uint32_t ti = ws.idx[s];
        ws.ax[ti] = ax;
        ws.ay[ti] = ay;
        ws.az[ti] = az;
        if (p.kick) {
          // second half kick, integrator.cu:86-106
          ws.vx[ti] = __fma_rn(p.half_dt, ax, ws.vx[ti]);
          ws.vy[ti] = __fma_rn(p.half_dt, ay, ws.vy[ti]);
          ws.vz[ti] = __fma_rn(p.half_dt, az, ws.vz[ti]);
        }
      }
    }
  }
  if (__any_sync(kFull, singular) && lane == 0) record_error(sc, kStageTraversal, 6);
  inter = warp_sum_ll(inter);
  tests = warp_sum_ll(tests);
  if (lane == 0) {
    atomicAdd(&sc->interactions, (unsigned long long)inter);
    atomicAdd(&sc->mac_tests, (unsigned long long)tests);
  }
}

// ------------------------------------------------------------ mixed ----

// Compile-time tuning of the mixed walk (warps per block, minimum resident
// blocks per SM for the register budget).
#ifndef NBB_MIXED_WARPS
#define NBB_MIXED_WARPS 2
#endif
#ifndef NBB_MIXED_MINBLOCKS
#define NBB_MIXED_MINBLOCKS 10
#endif
// resident blocks per SM for the two- and four-targets-per-lane instances
// (more registers per thread for the targets' sums)
#ifndef NBB_MIXED_MINBLOCKS2
#define NBB_MIXED_MINBLOCKS2 10
#endif
#ifndef NBB_MIXED_MINBLOCKS4
#define NBB_MIXED_MINBLOCKS4 7
#endif
constexpr int kMixedWarps = NBB_MIXED_WARPS;
constexpr int kWalkPop = 64;     // nodes per round: two per lane
constexpr int kStackCap = 1024;  // shared-memory part of a warp's stack
constexpr int kSpill = 512;      // entries moved to / from the global extension at once
// A spill starts above kStackCap - 7 kWalkPop entries and moves the bottom
// kSpill of them, so that threshold must hold at least kSpill entries (and
// the moved-down rest must end below kSpill, where the sources start).
static_assert(kStackCap - 7 * kWalkPop >= kSpill && kStackCap <= 2 * kSpill, "stack spill bounds");
// Entries per evaluated batch of the force walk: the list is evaluated when it
// holds this many, so each batch's set-up and compensated addition are paid
// once per kEvalBatch entries.  The walks that track sources (zero softening,
// the adjoint) keep 32-entry batches and the smaller list, whose shared
// memory keeps 10 blocks per SM.
#ifndef NBB_EVAL_BATCH
#define NBB_EVAL_BATCH 64
#endif
constexpr int kEvalBatch = NBB_EVAL_BATCH;
static_assert(kEvalBatch % 32 == 0 && kEvalBatch >= 32 && kEvalBatch <= 128, "batch of whole warps");
template <bool kTrackSource>
__host__ __device__ constexpr int batch_of() {
  return kTrackSource ? 32 : kEvalBatch;
}
// list capacity: < batch left over + 64 cells + up to 96 leaf particles
template <bool kTrackSource>
__host__ __device__ constexpr int list_cap_of() {
  return batch_of<kTrackSource>() + 160;
}

// The interaction list keeps entries in pairs so that packed two-wide FP32
// instructions (sm_100's FADD2 / FMUL2 / FFMA2) evaluate two entries at once
// from one 16-byte load per half: pair p holds entries 2p and 2p + 1 as
// a = {x0, x1, y0, y1} and b = {z0, z1, m0, m1}.
struct PairList {
  float4 *a, *b;
  __device__ __forceinline__ void put(int j, float x, float y, float z, float m) const {
    float *pa = reinterpret_cast<float *>(a + (j >> 1));
    float *pb = reinterpret_cast<float *>(b + (j >> 1));
    const int h = j & 1;
    pa[h] = x;
    pa[2 + h] = y;
    pb[h] = z;
    pb[2 + h] = m;
  }
};

template <bool kTrackSource>
struct MixedShared {
  double gbox[kMixedWarps][9];  // group box lo (3), hi (3), centre (3)
  float ghalf[kMixedWarps][4];  // group box half extents, rounded up to FP32
  int stack[kMixedWarps][kStackCap];
  float4 la[kMixedWarps][list_cap_of<kTrackSource>() / 2];
  float4 lb[kMixedWarps][list_cap_of<kTrackSource>() / 2];
  int src[kMixedWarps][kTrackSource ? list_cap_of<kTrackSource>() : 1];
};

// Hardware approximate reciprocal square root (MUFU), subnormal inputs and
// results flushed to zero: r^2 + eps^2 of a force evaluation is never
// subnormal where it matters, and the flush saves the range fix-up that
// rsqrtf adds around the same instruction.
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Evaluate `count` list entries (rounded up to a whole pair; an odd count
// has a zero-mass pad after it) for this lane's kTPL targets: FP32 offsets,
// approximate rsqrt (no refinement), two-wide FP32 partial sums over
// the batch, then one Kahan-compensated addition of each batch partial into
// its running sum.
//
// With positive softening a target's own entry (a leaf particle equal to the
// target) has offset exactly (0, 0, 0) -- both offsets are rounded from the
// same FP64 difference -- and contributes exactly zero, so no source index is
// needed.  With zero softening the source index excludes self and detects
// the reference's singular interaction (returns true).
// Pairs per unrolled block of the evaluation loop, by the walk's target
// slots per lane (its register budget): 8 for one or two slots, 4 for four
// (8 spills there).
#ifndef NBB_EVAL_UNROLL
#define NBB_EVAL_UNROLL 8
#endif
#ifndef NBB_EVAL_UNROLL4
#define NBB_EVAL_UNROLL4 4
#endif
template <int kSlots>
__host__ __device__ constexpr int eval_unroll() {
  return kSlots >= 4 ? NBB_EVAL_UNROLL4 : NBB_EVAL_UNROLL;
}

template <bool kTrackSource, int kTPL, int kUnroll>
__device__ __forceinline__ bool eval_batch(const PairList &list, const int *src, int count, const int *self,
                                           const float2 *ntx, const float2 *nty, const float2 *ntz, float2 eps2,
                                           float3 *sum, float3 *comp) {
  float2 px[kTPL], py[kTPL], pz[kTPL];
#pragma unroll
  for (int q = 0; q < kTPL; ++q) px[q] = py[q] = pz[q] = make_float2(0.f, 0.f);
  bool singular = false;
  const int pairs = (count + 1) >> 1;
#pragma unroll kUnroll
  for (int pr = 0; pr < pairs; ++pr) {
    const float4 ea = list.a[pr], eb = list.b[pr];
    const float2 ex = make_float2(ea.x, ea.y), ey = make_float2(ea.z, ea.w);
    const float2 ez = make_float2(eb.x, eb.y), em = make_float2(eb.z, eb.w);
#pragma unroll
    for (int q = 0; q < kTPL; ++q) {
      const float2 dx = __fadd2_rn(ex, ntx[q]), dy = __fadd2_rn(ey, nty[q]), dz = __fadd2_rn(ez, ntz[q]);
      const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
      const float2 r = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
      // m r^-3 straight from the hardware estimate: its relative error (a few
      // 1e-7 on r^-3) sits far below the Barnes-Hut truncation error this
      // form is held to, and a Newton step would add 3 packed FP32 operations
      // to the 12 of a pair of entries
      const float2 rr = __fmul2_rn(r, r);
      float2 f = __fmul2_rn(__fmul2_rn(em, r), rr);
      if (kTrackSource) {
        const bool o0 = src[2 * pr] != self[q], o1 = src[2 * pr + 1] != self[q];
        singular |= (o0 && !(r2.x > 0.f) && em.x != 0.f) || (o1 && !(r2.y > 0.f) && em.y != 0.f);
        f.x = (o0 && r2.x > 0.f) ? f.x : 0.f;
        f.y = (o1 && r2.y > 0.f) ? f.y : 0.f;
      }
      px[q] = __ffma2_rn(f, dx, px[q]);
      py[q] = __ffma2_rn(f, dy, py[q]);
      pz[q] = __ffma2_rn(f, dz, pz[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < kTPL; ++q) {
    float y, t;
    y = (px[q].x + px[q].y) - comp[q].x; t = sum[q].x + y; comp[q].x = (t - sum[q].x) - y; sum[q].x = t;
    y = (py[q].x + py[q].y) - comp[q].y; t = sum[q].y + y; comp[q].y = (t - sum[q].y) - y; sum[q].y = t;
    y = (pz[q].x + pz[q].y) - comp[q].z; t = sum[q].z + y; comp[q].z = (t - sum[q].z) - y; sum[q].z = t;
  }
  return singular;
}

// A child entry the mixed walk may push: a node's children come after it in
// preorder; a cached cell's children are cached cells after it or any node.
__device__ __forceinline__ bool valid_child(int kid, int node, int m, int mc) {
  return node < m ? (kid > node && kid < m) : ((kid > node && kid < mc) || (kid >= 0 && kid < m));
}

// Per-lane target state of the mixed walk: negated target offsets from the
// group centre, each duplicated into both halves of a pair.
template <int kTPL>
struct LaneTargets {
  int s[kTPL];
  bool valid[kTPL];
  float2 ntx[kTPL], nty[kTPL], ntz[kTPL];
  float3 sum[kTPL], comp[kTPL];
  long long inter = 0;
  bool singular = false;
};

// Evaluate `count` entries for the first nq (warp-uniform) of the lane's
// kTPL target slots: a group of g targets fills ceil(g / 32) slots, and the
// empty ones cost nothing (the branch is taken once per batch, outside the
// entry loop).
template <bool kTrackSource, int kTPL>
__device__ __forceinline__ bool eval_slots(const PairList &list, const int *src, int count, int nq,
                                           LaneTargets<kTPL> &t, float2 eps2) {
  if (kTPL >= 4 && nq >= 4)
    return eval_batch<kTrackSource, (kTPL >= 4 ? 4 : 1), eval_unroll<kTPL>()>(list, src, count, t.s, t.ntx, t.nty, t.ntz, eps2, t.sum,
                                                         t.comp);
  if (kTPL >= 3 && nq == 3)
    return eval_batch<kTrackSource, (kTPL >= 3 ? 3 : 1), eval_unroll<kTPL>()>(list, src, count, t.s, t.ntx, t.nty, t.ntz, eps2, t.sum,
                                                         t.comp);
  if (kTPL >= 2 && nq == 2)
    return eval_batch<kTrackSource, (kTPL >= 2 ? 2 : 1), eval_unroll<kTPL>()>(list, src, count, t.s, t.ntx, t.nty, t.ntz, eps2, t.sum,
                                                         t.comp);
  return eval_batch<kTrackSource, 1, eval_unroll<kTPL>()>(list, src, count, t.s, t.ntx, t.nty, t.ntz, eps2, t.sum, t.comp);
}

// ------------------------------------------------- mixed adjoint walk ----
//
// Vector-Jacobian product of the mixed form's force, on the mixed walk's own
// interaction lists (group-box acceptance, FP32 offsets from the group
// centre).  For target i, entry s (mass mu, offset r = Y_s - x_i) and the
// accelerations cotangent c_i (see adjoint.cu's file comment):
//   u = G mu (inv3 c_i - 3 inv5 (r . c_i) r),  d/dx_i -= u,  d/dY_s += u,
//   d/dmu_s += G inv3 (r . c_i),
// in FP32 with the hardware reciprocal square root.  A source's u is summed
// over the warp's targets before it is added (FP64 atomics) to the cell's or
// particle's cotangent; the list names each entry's source: a particle by its
// Morton slot, a cell by -3 - its preorder index.

// Cotangent state of the adjoint walk's target (one per lane).
struct LaneVjp {
  float cx = 0.f, cy = 0.f, cz = 0.f;  // accelerations cotangent
  double gx = 0.0, gy = 0.0, gz = 0.0;  // position cotangent (running)
};

// Sum over the warp of 8 per-lane values, transposed: lane l ends with the
// total of value ((l >> 4) & 1) * 4 + ((l >> 3) & 1) * 2 + ((l >> 2) & 1)
// (the four lanes of a quad hold the same total) -- 9 shuffles for 8 sums.
__device__ __forceinline__ float warp_sum8_transposed(float (&v)[8], int lane) {
  const bool u16 = lane & 16, u8 = lane & 8, u4 = lane & 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float send = u16 ? v[i] : v[i + 4];
    const float keep = u16 ? v[i + 4] : v[i];
    v[i] = keep + __shfl_xor_sync(kFull, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float send = u8 ? v[i] : v[i + 2];
    const float keep = u8 ? v[i + 2] : v[i];
    v[i] = keep + __shfl_xor_sync(kFull, send, 8);
  }
  const float send = u4 ? v[0] : v[1];
  float x = (u4 ? v[1] : v[0]) + __shfl_xor_sync(kFull, send, 4);
  x += __shfl_xor_sync(kFull, x, 2);
  x += __shfl_xor_sync(kFull, x, 1);
  return x;
}

// VJP of `count` list entries (zero-mass pads contribute nothing) for the
// lane's target; returns true on a singular pair.
__device__ bool vjp_entries(const PairList &list, const int *src, int count, int self, bool valid, float ntx,
                            float nty, float ntz, LaneVjp &v, float eps2, float g, const AdjointBuffers &ab) {
  const int lane = threadIdx.x & 31;
  bool singular = false;
  float gx = 0.f, gy = 0.f, gz = 0.f;
  for (int e0 = 0; e0 < count; e0 += 8) {
    float ux[8], uy[8], uz[8], uw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      ux[k] = uy[k] = uz[k] = uw[k] = 0.f;
      const int e = e0 + k;
      if (e >= count) continue;  // warp-uniform
      const float4 ea = list.a[e >> 1], eb = list.b[e >> 1];
      const bool hi = e & 1;
      const float ex = hi ? ea.y : ea.x, ey = hi ? ea.w : ea.z, ez = hi ? eb.y : eb.x, mu = hi ? eb.w : eb.z;
      const float dx = ex + ntx, dy = ey + nty, dz = ez + ntz;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
      if (!valid || src[e] == self || mu == 0.f) continue;
      if (!(r2 > 0.f)) {
        singular = true;
        continue;
      }
      const float r = rsqrt_approx(r2);
      const float rr = r * r;
      const float gi3 = g * rr * r;
      const float rc = fmaf(dx, v.cx, fmaf(dy, v.cy, dz * v.cz));
      const float f = gi3 * mu;
      const float h = 3.f * f * rr * rc;
      ux[k] = fmaf(f, v.cx, -h * dx);
      uy[k] = fmaf(f, v.cy, -h * dy);
      uz[k] = fmaf(f, v.cz, -h * dz);
      uw[k] = gi3 * rc;
      gx -= ux[k];
      gy -= uy[k];
      gz -= uz[k];
    }
    const float sx = warp_sum8_transposed(ux, lane);
    const float sy = warp_sum8_transposed(uy, lane);
    const float sz = warp_sum8_transposed(uz, lane);
    const float sw = warp_sum8_transposed(uw, lane);
    const int e = e0 + ((((lane >> 4) & 1) << 2) | (((lane >> 3) & 1) << 1) | ((lane >> 2) & 1));
    const int comp = lane & 3;
    const float val = comp == 0 ? sx : (comp == 1 ? sy : (comp == 2 ? sz : sw));
    if (e < count && val != 0.f) {
      const int sr = src[e];
      double *dst = nullptr;
      if (sr >= 0) dst = reinterpret_cast<double *>(ab.part_g + sr);
      else if (sr <= -3) dst = reinterpret_cast<double *>(ab.node_g + (-3 - sr));
      if (dst) atomicAdd(dst + comp, (double)val);
    }
  }
  v.gx += gx;
  v.gy += gy;
  v.gz += gz;
  return singular;
}

template <bool kTrackSource, int kTPL, bool kVjp>
__device__ __forceinline__ void flush_full(const PairList &list, int *src, int &ls, LaneTargets<kTPL> &lt_,
                                           LaneVjp &vj, float2 eps2, int nq, float g, const AdjointBuffers &ab) {
  constexpr int kBatch = batch_of<kTrackSource>();
  const int lane = threadIdx.x & 31;
  int done = 0;
  while (ls - done >= kBatch) {
    const PairList part{list.a + done / 2, list.b + done / 2};
    bool sg;
    if constexpr (kVjp)
      sg = vjp_entries(part, src + done, kBatch, lt_.s[0], lt_.valid[0], lt_.ntx[0].x, lt_.nty[0].x, lt_.ntz[0].x,
                       vj, eps2.x, g, ab);
    else
      sg = eval_slots<kTrackSource, kTPL>(part, src + (kTrackSource ? done : 0), kBatch, nq, lt_, eps2);
#pragma unroll
    for (int q = 0; q < kTPL; ++q)
      if (lt_.valid[q]) {
        lt_.inter += kBatch;
        lt_.singular |= sg;
      }
    done += kBatch;
  }
  if (done) {
    __syncwarp();
    // fewer than kBatch entries left; the sources start at done >= kBatch,
    // past the destinations
    const int rest = ls - done;
    for (int i = lane; i < (rest + 1) / 2; i += 32) {
      list.a[i] = list.a[done / 2 + i];
      list.b[i] = list.b[done / 2 + i];
    }
    if (kTrackSource)
      for (int i = lane; i < rest; i += 32) src[i] = src[done + i];
    ls = rest;
    __syncwarp();
  }
}

// Exclusive prefix sum over the warp of a small count v in [0, 2^kBits):
// one ballot per bit, no chain of dependent shuffles.  `total` receives the
// warp's sum (one warp reduction instead of a population count per bit: the
// XU pipe that counts bits also runs the walk's reciprocal square roots).
template <int kBits>
__device__ __forceinline__ int warp_prefix_small(int v, unsigned lt, int &total) {
  int excl = 0;
#pragma unroll
  for (int b = 0; b < kBits; ++b) {
    const unsigned m = __ballot_sync(kFull, (v >> b) & 1);
    excl += __popc(m & lt) << b;
  }
  total = __reduce_add_sync(kFull, v);
  return excl;
}

// The group-box acceptance test of the mixed walk, in FP32.  The node's
// centre of mass is taken relative to the group centre in FP64 and rounded
// (the list entry's offset, returned in e); the squared distance from the
// box (half extents rounded up) to that point is computed in FP32 and shrunk
// by 2^-20 so that it never exceeds the exact FP64 distance, and cr2 is the
// exact squared radius rounded up with a 2^-18 margin.  An accepted node is
// therefore accepted by the exact test for every target in the box; a node
// within the margins is opened instead (more work, never less accuracy).
__device__ __forceinline__ bool accept_box(const double4 &a, const double *gbox, const float *ghalf, float cr2,
                                           float4 &e) {
  const float ox = (float)(a.x - gbox[6]), oy = (float)(a.y - gbox[7]), oz = (float)(a.z - gbox[8]);
  constexpr float kShrink = 1.0f - 0x1p-20f;
  const float ex = fmaxf(0.f, fmaf(fabsf(ox), kShrink, -ghalf[0]));
  const float ey = fmaxf(0.f, fmaf(fabsf(oy), kShrink, -ghalf[1]));
  const float ez = fmaxf(0.f, fmaf(fabsf(oz), kShrink, -ghalf[2]));
  const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex)) * kShrink;
  e = make_float4(ox, oy, oz, (float)a.w);
  return d2 > cr2;
}

// Mixed-precision traversal, one warp per target group of at most 32 x kTPL
// Morton-consecutive targets inside one parent cell (kTPL targets per lane).
// The group's bounding box (FP64) replaces the target in the reference's
// acceptance test: a node is accepted for the whole group when the
// box-to-centre-of-mass distance exceeds max(crit, sqrt(3) h + |com -
// centre|) (crit = side/theta + |com - centre|, h the cell's half side),
// tested conservatively in FP32 (accept_box).  Every target in the box is
// then farther than crit from the centre of mass and outside the cell, so
// the reference's test accepts the node for each of them.  Nodes are
// examined 64 at a time (two per lane) from a warp-private stack in shared
// memory, each lane fetching both nodes' 48-byte records (MixedNode) in one
// round trip and the child lists of the nodes that open; a full stack spills
// its bottom half to a global extension sized for any walk, so every node
// gets the acceptance test.  Accepted nodes and the particles of reached leaves go to
// a shared interaction list as FP32 offsets from the group centre (formed in
// FP64, then rounded) and are evaluated by all lanes in batches of 32.
// With kVjp (one target per lane, sources tracked) the same walk evaluates
// the vector-Jacobian product above instead of the force.
template <bool kTrackSource, int kTPL, bool kVjp = false>
__global__ void __launch_bounds__(kMixedWarps * 32,
                                   kTPL >= 4 ? NBB_MIXED_MINBLOCKS4 : (kTPL == 2 ? NBB_MIXED_MINBLOCKS2 : NBB_MIXED_MINBLOCKS))
    traverse_mixed_kernel(Workspace ws, TraversalParams p, AdjointBuffers ab) {
  static_assert(!kVjp || (kTrackSource && kTPL == 1), "the adjoint walk tracks sources, one target per lane");
  __shared__ MixedShared<kTrackSource> sh;
  // node cache: the top cache_depth levels below the root, loaded once per
  // block from the step's table; stack entry m + q names cached cell q
  __shared__ MixedNode c_rec[kTopMax];
  __shared__ int4 c_kids[kTopMax][2];
  __shared__ int s_ccount;
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  int *stack = sh.stack[wid];
  const PairList list{sh.la[wid], sh.lb[wid]};
  int *src = sh.src[wid];
  const int n = ws.n;
  const int m = sc->n_nodes;
  const int n_groups = p.group_mode ? sc->n_tgroups : (n + 32 * kTPL - 1) / (32 * kTPL);
  const unsigned lt = lanemask_lt();
  int ccount = 0;
  if (p.cache_depth > 0 && ws.top && ws.n_systems == 1) {
    if (threadIdx.x == 0) {
      s_ccount = min(sc->level_base[min(p.cache_depth, kTopDepth) + 1], kTopMax);
    }
    __syncthreads();
    ccount = s_ccount;
    for (int q = threadIdx.x; q < ccount; q += blockDim.x) {
      const TopNode &t = ws.top[q];
      c_rec[q] = t.rec;
      int kk[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        // children in visit order (descending level order); cached ones by slot
        const int slot = t.first_child + t.nchild - 1 - j;
        kk[j] = (t.level < p.cache_depth && j < t.nchild && slot < ccount) ? m + slot : t.kids[j];
      }
      c_kids[q][0] = make_int4(kk[0], kk[1], kk[2], kk[3]);
      c_kids[q][1] = make_int4(kk[4], kk[5], kk[6], kk[7]);
    }
    __syncthreads();
  }
  const int mc = m + ccount;  // stack entries in [m, mc) are cached cells
  long long tests = 0;
  unsigned overflow = 0;
  long long inter_total = 0;
  bool singular_any = false;
  while (true) {
    int grp = 0;
    if (lane == 0) grp = (int)atomicAdd(&sc->work_counter, 1u);
    grp = __shfl_sync(kFull, grp, 0);
    if (grp >= n_groups) break;
    const int g0 = p.group_mode ? ws.tstart[grp] : grp * 32 * kTPL;
    const int g1 = p.group_mode ? ((grp + 1 < n_groups) ? ws.tstart[grp + 1] : n) : min(g0 + 32 * kTPL, n);
    const int nq = min(kTPL, max(1, (g1 - g0 + 31) >> 5));  // occupied target slots
    LaneTargets<kTPL> T;
    LaneVjp V;
    double4 tp[kTPL];
    double lo[3], hi[3];
#pragma unroll
    for (int q = 0; q < kTPL; ++q) {
      T.s[q] = g0 + lane + 32 * q;
      T.valid[q] = T.s[q] < g1 && T.s[q] < n;
      tp[q] = ws.pm4[T.valid[q] ? T.s[q] : g0];
      T.sum[q] = make_float3(0.f, 0.f, 0.f);
      T.comp[q] = make_float3(0.f, 0.f, 0.f);
    }
    if (kVjp && T.valid[0]) {
      const uint32_t ti = ws.idx[T.s[0]];
      V.cx = (float)(ab.coef * ab.gvx[ti]);
      V.cy = (float)(ab.coef * ab.gvy[ti]);
      V.cz = (float)(ab.coef * ab.gvz[ti]);
    }
    lo[0] = hi[0] = tp[0].x;
    lo[1] = hi[1] = tp[0].y;
    lo[2] = hi[2] = tp[0].z;
#pragma unroll
    for (int q = 1; q < kTPL; ++q) {
      lo[0] = fmin(lo[0], tp[q].x); hi[0] = fmax(hi[0], tp[q].x);
      lo[1] = fmin(lo[1], tp[q].y); hi[1] = fmax(hi[1], tp[q].y);
      lo[2] = fmin(lo[2], tp[q].z); hi[2] = fmax(hi[2], tp[q].z);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      for (int o = 16; o > 0; o >>= 1) {
        lo[a] = fmin(lo[a], __shfl_xor_sync(kFull, lo[a], o));
        hi[a] = fmax(hi[a], __shfl_xor_sync(kFull, hi[a], o));
      }
    }
    {
      // the box and centre live in shared memory while the walk runs, so
      // they hold no registers through the evaluation
      volatile double *gb = sh.gbox[wid];
      if (lane == 0) {
        for (int a = 0; a < 3; ++a) {
          gb[a] = lo[a];
          gb[3 + a] = hi[a];
          gb[6 + a] = 0.5 * (lo[a] + hi[a]);
          sh.ghalf[wid][a] = __double2float_ru(0.5 * (hi[a] - lo[a]));
        }
      }
      __syncwarp();
    }
    const double *gbox = sh.gbox[wid];
    const double gcx = 0.5 * (lo[0] + hi[0]), gcy = 0.5 * (lo[1] + hi[1]),
                 gcz = 0.5 * (lo[2] + hi[2]);
    {
      float tx[kTPL], ty[kTPL], tz[kTPL];
#pragma unroll
      for (int q = 0; q < kTPL; ++q) {
        tx[q] = -(float)(tp[q].x - gcx);
        ty[q] = -(float)(tp[q].y - gcy);
        tz[q] = -(float)(tp[q].z - gcz);
      }
#pragma unroll
      for (int q = 0; q < kTPL; ++q) {
        T.ntx[q] = make_float2(tx[q], tx[q]);
        T.nty[q] = make_float2(ty[q], ty[q]);
        T.ntz[q] = make_float2(tz[q], tz[q]);
      }
    }
    // a group's targets belong to one system: walk that system's subtree
    const int sys = ws.n_systems > 1 ? ws.psys[g0] : 0;
    const int root = ws.root_pre[sys];
    const double soft = ws.sys_eps ? ws.sys_eps[sys] : p.soft;
    const float eps2f = (float)(soft * soft);
    const float2 eps2 = make_float2(eps2f, eps2f);
    int ls = 0;
    if (lane == 0) stack[0] = ccount > 0 ? m : root;
    int sp = (m > 0 && root >= 0 && root < m) ? 1 : 0;
    __syncwarp();
    // this warp's stack extension in global memory: when the shared part
    // fills, its bottom half moves there (the combined stack keeps its
    // order) and comes back when the shared part runs low
    int *ext = nullptr;
    int esp = 0;
    {
      const int gw = blockIdx.x * kMixedWarps + wid;
      if (ws.walk_ext && gw < ws.walk_warps) ext = ws.walk_ext + (size_t)gw * ws.walk_ext_cap;
    }
    while (sp > 0 || esp > 0) {
      if (sp > kStackCap - 7 * kWalkPop && ext && esp + kSpill <= ws.walk_ext_cap) {
        for (int i = lane; i < kSpill; i += 32) ext[esp + i] = stack[i];
        __syncwarp();
        // the destination ends below kSpill, where the sources start
        for (int i = lane; i < sp - kSpill; i += 32) stack[i] = stack[kSpill + i];
        esp += kSpill;
        sp -= kSpill;
        __syncwarp();
      } else if (sp < kWalkPop && esp > 0) {
        const int r = min(esp, kSpill);
        const int v0 = (lane < sp) ? stack[lane] : 0, v1 = (lane + 32 < sp) ? stack[lane + 32] : 0;
        __syncwarp();
        if (lane < sp) stack[r + lane] = v0;
        if (lane + 32 < sp) stack[r + lane + 32] = v1;
        for (int i = lane; i < r; i += 32) stack[i] = ext[esp - r + i];
        sp += r;
        esp -= r;
        __syncwarp();
      }
      // up to 64 nodes per round, two per lane, fetched in one round trip
      int k = sp < kWalkPop ? sp : kWalkPop;
      const int room = (kStackCap - sp) / 7;
      if (k > room) k = room > 0 ? room : 1;
      const int n0 = (lane < k) ? stack[sp - k + lane] : -1;
      const int n1 = (lane + 32 < k) ? stack[sp - k + 32 + lane] : -1;
      sp -= k;
      __syncwarp();
      int4 m0 = make_int4(0, 0, 0, 0), m1 = m0;
      int4 k00 = make_int4(-1, -1, -1, -1), k01 = k00, k10 = k00, k11 = k00;
      double4 a0 = make_double4(0.0, 0.0, 0.0, 0.0), a1 = a0;
      float cr0 = 0.f, cr1 = 0.f;  // squared acceptance radius for a target box
      if (n0 >= m) {
        const MixedNode &rec = c_rec[n0 - m];
        a0 = rec.a;
        const int4 meta = *reinterpret_cast<const int4 *>(&rec.cr2);
        cr0 = __int_as_float(meta.x);
        m0 = make_int4(0, meta.y, meta.z, meta.w);
      } else if (n0 >= 0) {
        const MixedNode &rec = ws.node_m[n0];
        a0 = rec.a;
        const int4 meta = *reinterpret_cast<const int4 *>(&rec.cr2);
        cr0 = __int_as_float(meta.x);
        m0 = make_int4(0, meta.y, meta.z, meta.w);
      }
      if (n1 >= m) {
        const MixedNode &rec = c_rec[n1 - m];
        a1 = rec.a;
        const int4 meta = *reinterpret_cast<const int4 *>(&rec.cr2);
        cr1 = __int_as_float(meta.x);
        m1 = make_int4(0, meta.y, meta.z, meta.w);
      } else if (n1 >= 0) {
        const MixedNode &rec = ws.node_m[n1];
        a1 = rec.a;
        const int4 meta = *reinterpret_cast<const int4 *>(&rec.cr2);
        cr1 = __int_as_float(meta.x);
        m1 = make_int4(0, meta.y, meta.z, meta.w);
      }
      // 0 nothing, 1 accepted cell, 2 leaf, 3 open; the cell's list entry
      // (centre of mass offset from the group centre, mass) in FP32
      int cat0 = 0, cat1 = 0;
      float4 e0 = make_float4(0.f, 0.f, 0.f, 0.f), e1 = e0;
      {
        const double4 a = a0;
        if (n0 >= 0) {
          if (m0.z > 0) {
            cat0 = 2;
          } else if (a.w != 0.0) {
            ++tests;
            cat0 = accept_box(a, gbox, sh.ghalf[wid], cr0, e0) ? 1 : 3;
          }
        }
      }
      {
        const double4 a = a1;
        if (n1 >= 0) {
          if (m1.z > 0) {
            cat1 = 2;
          } else if (a.w != 0.0) {
            ++tests;
            cat1 = accept_box(a, gbox, sh.ghalf[wid], cr1, e1) ? 1 : 3;
          }
        }
      }
      // opened nodes push their children (node 0's, then node 1's); a push
      // that would end past the stack accepts the node instead
      int nc0 = (cat0 == 3) ? min(max(m0.w, 0), 8) : 0;
      int nc1 = (cat1 == 3) ? min(max(m1.w, 0), 8) : 0;
      // child lists only of the nodes that open; their loads overlap the
      // prefix sums below
      if (nc0 > 0) {
        if (n0 >= m) {
          k00 = c_kids[n0 - m][0];
          k01 = c_kids[n0 - m][1];
        } else {
          const int4 *kids = reinterpret_cast<const int4 *>(ws.node_kids + (size_t)n0 * 8);
          k00 = kids[0];
          if (nc0 > 4) k01 = kids[1];
        }
      }
      if (nc1 > 0) {
        if (n1 >= m) {
          k10 = c_kids[n1 - m][0];
          k11 = c_kids[n1 - m][1];
        } else {
          const int4 *kids = reinterpret_cast<const int4 *>(ws.node_kids + (size_t)n1 * 8);
          k10 = kids[0];
          if (nc1 > 4) k11 = kids[1];
        }
      }
      int all_children;
      const int excl = warp_prefix_small<5>(nc0 + nc1, lt, all_children);
      int pushed = all_children;
      if (sp + all_children > kStackCap) {
        if (nc0 > 0 && sp + excl + nc0 > kStackCap) {
          cat0 = 1;
          nc0 = 0;
          ++overflow;
        }
        if (nc1 > 0 && sp + excl + nc0 + nc1 > kStackCap) {
          cat1 = 1;
          nc1 = 0;
          ++overflow;
        }
        pushed = __reduce_max_sync(kFull, (nc0 + nc1 > 0) ? excl + nc0 + nc1 : 0);
      }
      {
        const int kid[8] = {k00.x, k00.y, k00.z, k00.w, k01.x, k01.y, k01.z, k01.w};
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (j < nc0) stack[sp + excl + j] = valid_child(kid[j], n0, m, mc) ? kid[j] : -1;
      }
      {
        const int kid[8] = {k10.x, k10.y, k10.z, k10.w, k11.x, k11.y, k11.z, k11.w};
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (j < nc1) stack[sp + excl + nc0 + j] = valid_child(kid[j], n1, m, mc) ? kid[j] : -1;
      }
      sp += pushed;
      // accepted cells -> interaction list (fewer than 32 entries before,
      // at most 64 more)
      const unsigned cm0 = __ballot_sync(kFull, cat0 == 1);
      const unsigned cm1 = __ballot_sync(kFull, cat1 == 1);
      if (cat0 == 1) {
        const int pos = ls + __popc(cm0 & lt);
        list.put(pos, e0.x, e0.y, e0.z, e0.w);
        if (kTrackSource) src[pos] = kVjp ? -3 - n0 : -1;
      }
      if (cat1 == 1) {
        const int pos = ls + __popc(cm0) + __popc(cm1 & lt);
        list.put(pos, e1.x, e1.y, e1.z, e1.w);
        if (kTrackSource) src[pos] = kVjp ? -3 - n1 : -1;
      }
      ls += __popc(cm0) + __popc(cm1);
      // reached leaves -> their particles: all at once when they fit
      const int lc0 = (cat0 == 2) ? m0.z : 0;
      const int lc1 = (cat1 == 2) ? m1.z : 0;
      int lexcl, ltotal;
      if (__all_sync(kFull, lc0 < 16 && lc1 < 16)) {
        lexcl = warp_prefix_small<5>(lc0 + lc1, lt, ltotal);
      } else {
        int linc = lc0 + lc1;
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(kFull, linc, o);
          if (lane >= o) linc += v;
        }
        ltotal = __shfl_sync(kFull, linc, 31);
        lexcl = linc - lc0 - lc1;
      }
      if (ls + ltotal <= list_cap_of<kTrackSource>()) {
        const int base = ls + lexcl;
        double4 q0 = make_double4(0.0, 0.0, 0.0, 0.0), q1 = q0;
        if (lc0 > 0) q0 = ws.pm4[m0.y];
        if (lc1 > 0) q1 = ws.pm4[m1.y];
        if (lc0 > 0) {
          list.put(base, (float)(q0.x - gbox[6]), (float)(q0.y - gbox[7]), (float)(q0.z - gbox[8]), (float)q0.w);
          if (kTrackSource) src[base] = m0.y;
        }
        if (lc1 > 0) {
          list.put(base + lc0, (float)(q1.x - gbox[6]), (float)(q1.y - gbox[7]), (float)(q1.z - gbox[8]),
                   (float)q1.w);
          if (kTrackSource) src[base + lc0] = m1.y;
        }
        for (int j = 1; j < lc0; ++j) {
          const double4 q = ws.pm4[m0.y + j];
          list.put(base + j, (float)(q.x - gbox[6]), (float)(q.y - gbox[7]), (float)(q.z - gbox[8]), (float)q.w);
          if (kTrackSource) src[base + j] = m0.y + j;
        }
        for (int j = 1; j < lc1; ++j) {
          const double4 q = ws.pm4[m1.y + j];
          list.put(base + lc0 + j, (float)(q.x - gbox[6]), (float)(q.y - gbox[7]), (float)(q.z - gbox[8]),
                   (float)q.w);
          if (kTrackSource) src[base + lc0 + j] = m1.y + j;
        }
        ls += ltotal;
        __syncwarp();
        flush_full<kTrackSource, kTPL, kVjp>(list, src, ls, T, V, eps2, nq, (float)p.g, ab);
      } else {
        // rare: the leaves' particles do not fit behind the list; their
        // ranges stay in registers through the flush
        __syncwarp();
        flush_full<kTrackSource, kTPL, kVjp>(list, src, ls, T, V, eps2, nq, (float)p.g, ab);
        for (int h = 0; h < 2; ++h) {
          unsigned lm = __ballot_sync(kFull, (h == 0 ? lc0 : lc1) > 0);
          while (lm) {
            const int l = __ffs(lm) - 1;
            lm &= lm - 1;
            const int first = __shfl_sync(kFull, h == 0 ? m0.y : m1.y, l);
            const int cnt = __shfl_sync(kFull, h == 0 ? lc0 : lc1, l);
            for (int b0 = 0; b0 < cnt; b0 += 32) {
              const int j = b0 + lane;
              if (j < cnt) {
                const double4 q = ws.pm4[first + j];
                list.put(ls + lane, (float)(q.x - gbox[6]), (float)(q.y - gbox[7]), (float)(q.z - gbox[8]),
                         (float)q.w);
                if (kTrackSource) src[ls + lane] = first + j;
              }
              ls += (cnt - b0 < 32) ? (cnt - b0) : 32;
              __syncwarp();
              flush_full<kTrackSource, kTPL, kVjp>(list, src, ls, T, V, eps2, nq, (float)p.g, ab);
            }
          }
        }
      }
    }
    if (ls > 0) {
      if (ls & 1) {
        // complete the last pair with a zero-mass entry far away (its
        // offset squared stays finite in FP32 and it contributes exactly 0)
        if (lane == 0) {
          list.put(ls, 1.0e18f, 1.0e18f, 1.0e18f, 0.f);
          if (kTrackSource) src[ls] = -2;
        }
        __syncwarp();
      }
      bool sg;
      if constexpr (kVjp)
        sg = vjp_entries(list, src, ls + (ls & 1), T.s[0], T.valid[0], T.ntx[0].x, T.nty[0].x, T.ntz[0].x, V, eps2.x,
                         (float)p.g, ab);
      else
        sg = eval_slots<kTrackSource, kTPL>(list, src, ls, nq, T, eps2);
#pragma unroll
      for (int q = 0; q < kTPL; ++q)
        if (T.valid[q]) {
          T.inter += ls;
          T.singular |= sg;
        }
    }
    __syncwarp();
    if constexpr (kVjp) {
      if (T.valid[0]) ab.tgt_g[T.s[0]] = make_double4(V.gx, V.gy, V.gz, 0.0);
    }
#pragma unroll
    for (int q = 0; q < kTPL; ++q) {
      if (kVjp || !T.valid[q]) continue;
      const double ax = p.g * ((double)T.sum[q].x - (double)T.comp[q].x);
      const double ay = p.g * ((double)T.sum[q].y - (double)T.comp[q].y);
      const double az = p.g * ((double)T.sum[q].z - (double)T.comp[q].z);
      const uint32_t ti = ws.idx[T.s[q]];
      ws.ax[ti] = ax;
      ws.ay[ti] = ay;
      ws.az[ti] = az;
      if (p.kick) {
        ws.vx[ti] = __fma_rn(p.half_dt, ax, ws.vx[ti]);
        ws.vy[ti] = __fma_rn(p.half_dt, ay, ws.vy[ti]);
        ws.vz[ti] = __fma_rn(p.half_dt, az, ws.vz[ti]);
      }
    }
    inter_total += T.inter;
    singular_any |= T.singular;
  }
  if (__any_sync(kFull, singular_any) && lane == 0) record_error(sc, kStageTraversal, 6);
  inter_total = warp_sum_ll(inter_total);
  tests = warp_sum_ll(tests);
  unsigned ov = overflow;
  for (int o = 16; o > 0; o >>= 1) ov += __shfl_xor_sync(kFull, ov, o);
  if (lane == 0) {
    atomicAdd(&sc->interactions, (unsigned long long)inter_total);
    atomicAdd(&sc->mac_tests, (unsigned long long)tests);
    if (ov) {
      // the extension is sized for any walk, so this is a broken invariant:
      // the accepted nodes skipped their acceptance test, and the call fails
      atomicAdd(&sc->stack_overflow, ov);
      record_error(sc, kStageTraversal, 9);
    }
  }
}

// ------------------------------------------------------------ direct ----

constexpr int kDirectThreads = 128;

// barnes_hut_accuracy_test.cu:101-172: each thread sums every other particle
// in index order; sources are staged through shared memory in tiles.  With
// chunked sources (blockIdx.y of gridDim.y chunks, partial sums to
// part[chunk][3][n_targets]) few targets still fill the GPU; the partials are
// then added in chunk order by direct_combine_kernel.
__global__ void __launch_bounds__(kDirectThreads)
    direct_kernel(int n, const double *__restrict__ m, const double *__restrict__ x,
                  const double *__restrict__ y, const double *__restrict__ z, int n_targets,
                  const int *__restrict__ targets, double g, double soft2, double *ax, double *ay,
                  double *az, double *part) {
  __shared__ double4 tile[kDirectThreads];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int chunks = gridDim.y;
  const long long span = ((long long)n + chunks - 1) / chunks;
  const int j0 = (int)min((long long)n, span * blockIdx.y);
  const int j1 = (int)min((long long)n, span * (blockIdx.y + 1));
  int t = (k < n_targets) ? (targets ? targets[k] : k) : 0;
  const bool active = k < n_targets && t >= 0 && t < n;
  if (!active) t = 0;
  const double tx = active ? x[t] : 0.0, ty = active ? y[t] : 0.0, tz = active ? z[t] : 0.0;
  double rx = 0.0, ry = 0.0, rz = 0.0;
  for (int base = j0; base < j1; base += kDirectThreads) {
    const int j = base + threadIdx.x;
    tile[threadIdx.x] = (j < j1) ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int lim = (j1 - base < kDirectThreads) ? j1 - base : kDirectThreads;
    if (active) {
      for (int q = 0; q < lim; ++q) {
        if (base + q == t) continue;
        const double4 s = tile[q];
        const double dx = __dsub_rn(s.x, tx), dy = __dsub_rn(s.y, ty), dz = __dsub_rn(s.z, tz);
        const double d2 = __dadd_rn(sqdist(dx, dy, dz), soft2);
        const double inv = __drcp_rn(__dsqrt_rn(d2));
        const double f = __dmul_rn(__dmul_rn(g, s.w), __dmul_rn(__dmul_rn(inv, inv), inv));
        rx = __fma_rn(f, dx, rx);
        ry = __fma_rn(f, dy, ry);
        rz = __fma_rn(f, dz, rz);
      }
    }
    __syncthreads();
  }
  if (k < n_targets) {
    if (chunks == 1) {
      ax[k] = active ? rx : NAN;
      ay[k] = active ? ry : NAN;
      az[k] = active ? rz : NAN;
    } else {
      double *pc = part + (size_t)blockIdx.y * 3 * n_targets;
      pc[k] = active ? rx : NAN;
      pc[n_targets + k] = active ? ry : NAN;
      pc[2 * (size_t)n_targets + k] = active ? rz : NAN;
    }
  }
}

__global__ void __launch_bounds__(kDirectThreads)
    direct_combine_kernel(const double *__restrict__ part, int chunks, int n_targets, double *ax, double *ay,
                          double *az) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_targets) return;
  double rx = 0.0, ry = 0.0, rz = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const double *pc = part + (size_t)c * 3 * n_targets;
    rx = __dadd_rn(rx, pc[k]);
    ry = __dadd_rn(ry, pc[n_targets + k]);
    rz = __dadd_rn(rz, pc[2 * (size_t)n_targets + k]);
  }
  ax[k] = rx;
  ay[k] = ry;
  az[k] = rz;
}

// ------------------------------------------- reference-layout octree ----

// barnes_hut.cu:90-162 on a caller octree in the reference numbering.
__device__ int ref_first_child(const RefOctree &o, int node, int &err) {
  for (int oc = 7; oc >= 0; --oc) {
    const int c = o.children[node * 8 + oc];
    if (c == -1) continue;
    if (c <= 0 || c >= o.n_nodes) {
      err = 1;
      return -2;
    }
    return c;
  }
  err = 5;
  return -2;
}

__device__ int ref_next(const RefOctree &o, int node, int &err) {
  int climbs = 0;
  while (node != 0) {
    if (++climbs > o.n_nodes) {
      err = 4;
      return -2;
    }
    const int par = o.parent[node];
    if (par < 0 || par >= o.n_nodes) {
      err = 4;
      return -2;
    }
    bool found = false;
    for (int oc = 7; oc >= 0; --oc) {
      const int c = o.children[par * 8 + oc];
      if (c == -1) continue;
      if (c <= 0 || c >= o.n_nodes) {
        err = 1;
        return -2;
      }
      if (found) return c;
      if (c == node) found = true;
    }
    if (!found) {
      err = 4;
      return -2;
    }
    node = par;
  }
  return -1;
}

__global__ void ref_octree_kernel(RefOctree o, const uint32_t *idx, const double *pm,
                                  const double *px, const double *py, const double *pz, double *ax,
                                  double *ay, double *az, double theta, double soft2, double g,
                                  int morton, int *err_out) {
  const int st = blockIdx.x * blockDim.x + threadIdx.x;
  if (st >= o.n_particles) return;
  int err = 0;
  const uint32_t tu = idx[st];
  if (tu >= (uint32_t)o.n_particles) {
    atomicCAS(err_out, 0, 3);
    return;
  }
  const int target = (int)tu;
  const int ti = morton ? st : target;
  const double tx = px[ti], ty = py[ti], tz = pz[ti];
  double rx = 0.0, ry = 0.0, rz = 0.0;
  int node = 0;
  long long visits = 0;
  const long long max_visits = 2ll * o.n_nodes + 8;
  while (node >= 0) {
    if (++visits > max_visits) {  // a cyclic caller octree never ends
      atomicCAS(err_out, 0, 4);
      return;
    }
    const double h = o.half[node];
    if (h <= 0.0) {
      atomicCAS(err_out, 0, 8);
      return;
    }
    const int cnt = o.count[node];
    if (cnt > 0) {
      for (int oc = 0; oc < 8; ++oc)
        if (o.children[node * 8 + oc] != -1) {
          atomicCAS(err_out, 0, 7);
          return;
        }
      const int f = o.first[node];
      if (f < 0 || cnt > o.n_particles || f > o.n_particles - cnt) {
        atomicCAS(err_out, 0, 2);
        return;
      }
      for (int k = 0; k < cnt; ++k) {
        const int sp = f + k;
        const uint32_t su = idx[sp];
        if (su >= (uint32_t)o.n_particles) {
          atomicCAS(err_out, 0, 3);
          return;
        }
        if (su == tu) continue;
        const int si = morton ? sp : (int)su;
        if (pm[si] == 0.0) continue;
        const double dx = __dsub_rn(px[si], tx), dy = __dsub_rn(py[si], ty), dz = __dsub_rn(pz[si], tz);
        if (!point_mass_fp64(dx, dy, dz, sqdist(dx, dy, dz), pm[si], g, soft2, rx, ry, rz)) {
          atomicCAS(err_out, 0, 6);
          return;
        }
      }
      node = ref_next(o, node, err);
      if (node == -2) {
        atomicCAS(err_out, 0, err);
        return;
      }
      continue;
    }
    const double nm = o.mass[node];
    if (nm == 0.0) {
      node = ref_next(o, node, err);
      if (node == -2) {
        atomicCAS(err_out, 0, err);
        return;
      }
      continue;
    }
    const double dx = __dsub_rn(o.comx[node], tx), dy = __dsub_rn(o.comy[node], ty),
                 dz = __dsub_rn(o.comz[node], tz);
    const double d2 = sqdist(dx, dy, dz);
    const bool contains = fabs(__dsub_rn(tx, o.cx[node])) <= h && fabs(__dsub_rn(ty, o.cy[node])) <= h &&
                          fabs(__dsub_rn(tz, o.cz[node])) <= h;
    bool accept = false;
    if (!contains && d2 > 0.0 && theta > 0.0) {
      const double ox = __dsub_rn(o.comx[node], o.cx[node]), oy = __dsub_rn(o.comy[node], o.cy[node]),
                   oz = __dsub_rn(o.comz[node], o.cz[node]);
      const double crit = __dadd_rn(__ddiv_rn(__dmul_rn(2.0, h), theta), __dsqrt_rn(sqdist(ox, oy, oz)));
      accept = __dsqrt_rn(d2) > crit;
    }
    if (accept) {
      if (!point_mass_fp64(dx, dy, dz, d2, nm, g, soft2, rx, ry, rz)) {
        atomicCAS(err_out, 0, 6);
        return;
      }
      node = ref_next(o, node, err);
    } else {
      node = ref_first_child(o, node, err);
    }
    if (node == -2) {
      atomicCAS(err_out, 0, err);
      return;
    }
  }
  ax[target] = rx;
  ay[target] = ry;
  az[target] = rz;
}

// ---------------------------------------------------------- integrator --

__global__ void kick_drift_kernel(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                                  const double *ax, const double *ay, const double *az, size_t n,
                                  double dt) {
  const double hdt = 0.5 * dt;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double nvx = __fma_rn(hdt, ax[i], vx[i]);
    const double nvy = __fma_rn(hdt, ay[i], vy[i]);
    const double nvz = __fma_rn(hdt, az[i], vz[i]);
    vx[i] = nvx;
    vy[i] = nvy;
    vz[i] = nvz;
    x[i] = __fma_rn(dt, nvx, x[i]);
    y[i] = __fma_rn(dt, nvy, y[i]);
    z[i] = __fma_rn(dt, nvz, z[i]);
  }
}

__global__ void kick_kernel(double *vx, double *vy, double *vz, const double *ax, const double *ay,
                            const double *az, size_t n, double dt) {
  const double hdt = 0.5 * dt;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    vx[i] = __fma_rn(hdt, ax[i], vx[i]);
    vy[i] = __fma_rn(hdt, ay[i], vy[i]);
    vz[i] = __fma_rn(hdt, az[i], vz[i]);
  }
}

// Diagnostic: SIMT FMA throughput (8 independent chains per thread).
template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x * (T)1e-3, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-12345) out[threadIdx.x] = s;
}

// Packed two-wide FP32 variant (sm_100 FFMA2): 8 independent float2 chains.
__global__ void __launch_bounds__(256) fma2_peak_kernel(float *out, int iters, float a, float b) {
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
  float2 x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = make_float2(threadIdx.x * 1e-3f + k, threadIdx.x * 1e-3f - k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = __ffma2_rn(x[k], a2, b2);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k].x + x[k].y;
  if (s == -12345.f) out[threadIdx.x] = s;
}

inline int stream_grid(size_t n, int num_sms) {
  size_t b = (n + 255) / 256;
  const size_t cap = (size_t)(num_sms > 0 ? num_sms : 148) * 8;
  if (b > cap) b = cap;
  return b < 1 ? 1 : (int)b;
}

int device_sms() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

// Persistent grids: as many resident blocks as the occupancy calculator
// allows on every SM; warps then pull target groups from a work counter.
template <typename K>
static cudaError_t grid_of(K kernel, int threads, int sms, int &grid) {
  int per_sm = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  grid = sms * (per_sm > 0 ? per_sm : 1);
  return e;
}

cudaError_t configure_traversal(Workspace &ws) {
  const int sms = ws.num_sms > 0 ? ws.num_sms : 148;
  cudaError_t e = grid_of(traverse_fp64_kernel, 256, sms, ws.fp64_grid);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<false, 1>, kMixedWarps * 32, sms, ws.mixed_grid[0][0]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<true, 1>, kMixedWarps * 32, sms, ws.mixed_grid[1][0]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<false, 2>, kMixedWarps * 32, sms, ws.mixed_grid[0][1]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<true, 2>, kMixedWarps * 32, sms, ws.mixed_grid[1][1]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<false, 4>, kMixedWarps * 32, sms, ws.mixed_grid[0][2]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<true, 4>, kMixedWarps * 32, sms, ws.mixed_grid[1][2]);
  if (e == cudaSuccess) e = grid_of(traverse_mixed_kernel<true, 1, true>, kMixedWarps * 32, sms, ws.vjp_grid);
  // The stack extension holds a whole walk: the stack stays sorted by tree
  // level (a round pops the top and pushes children one level deeper), and
  // a level's entries are pushed only after every older entry of that level
  // has been popped, so at most 8 x kWalkPop entries per level are pending;
  // and a walk pushes each node at most once, so never more than the tree's
  // node capacity either (small systems take a small extension).
  int blocks = 148;
  for (int t = 0; t < 2; ++t)
    for (int q = 0; q < 3; ++q) blocks = std::max(blocks, ws.mixed_grid[t][q]);
  ws.walk_warps = blocks * kMixedWarps;
  ws.walk_ext_cap = std::min(8 * kWalkPop * (ws.max_level + 1), std::max(ws.cap_nodes, 1));
  return e;
}

cudaError_t launch_traversal(Workspace &ws, const TraversalParams &p, cudaStream_t s) {
  // target slots per lane: 1, 2 or 4 for groups of at most 32, 64 or 128
  const int slot = !p.group_mode ? 0 : (p.group_size > 64 ? 2 : (p.group_size > 32 ? 1 : 0));
  const int track = p.soft > 0.0 ? 0 : 1;
  const int grid = ws.mixed_grid[track][slot] > 0 ? ws.mixed_grid[track][slot] : 148;
  if (p.precision == 0)
    traverse_fp64_kernel<<<ws.fp64_grid > 0 ? ws.fp64_grid : 148, 256, 0, s>>>(ws, p);
  else if (slot == 0)
    (track ? traverse_mixed_kernel<true, 1> : traverse_mixed_kernel<false, 1>)<<<grid, kMixedWarps * 32, 0, s>>>(
        ws, p, AdjointBuffers{});
  else if (slot == 1)
    (track ? traverse_mixed_kernel<true, 2> : traverse_mixed_kernel<false, 2>)<<<grid, kMixedWarps * 32, 0, s>>>(
        ws, p, AdjointBuffers{});
  else
    (track ? traverse_mixed_kernel<true, 4> : traverse_mixed_kernel<false, 4>)<<<grid, kMixedWarps * 32, 0, s>>>(
        ws, p, AdjointBuffers{});
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_mixed(Workspace &ws, const TraversalParams &p, const AdjointBuffers &ab,
                                 cudaStream_t s) {
  // the stack extension is sized for the largest mixed grid
  int grid = ws.vjp_grid > 0 ? ws.vjp_grid : 148;
  if (ws.walk_warps > 0 && grid * kMixedWarps > ws.walk_warps) grid = ws.walk_warps / kMixedWarps;
  TraversalParams q = p;
  q.cache_depth = 0;  // cached cells carry no preorder index
  traverse_mixed_kernel<true, 1, true><<<grid, kMixedWarps * 32, 0, s>>>(ws, q, ab);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t measure_fma_tflops(int precision, double *tflops) {
  const int sms = device_sms();
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  void *out = nullptr;
  cudaError_t e = cudaMalloc(&out, 256 * sizeof(double));
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    cudaEventRecord(e0);
    if (precision == 0)
      fma_peak_kernel<double><<<blocks, threads>>>((double *)out, iters, 0.9999999, 1e-9);
    else if (precision == 1)
      fma_peak_kernel<float><<<blocks, threads>>>((float *)out, iters * 2, 0.9999f, 1e-6f);
    else
      fma2_peak_kernel<<<blocks, threads>>>((float *)out, iters, 0.9999f, 1e-6f);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  count_launches(4);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return e;
  // FP64: iters x 8 FMAs; FP32: 2 iters x 8; packed: iters x 8 x 2 lanes
  const double flops = 2.0 * 8.0 * (double)iters * (precision == 0 ? 1.0 : 2.0) * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return cudaSuccess;
}

cudaError_t launch_kick(double *vx, double *vy, double *vz, const double *ax, const double *ay,
                        const double *az, size_t n, double dt, cudaStream_t s) {
  kick_kernel<<<stream_grid(n, device_sms()), 256, 0, s>>>(vx, vy, vz, ax, ay, az, n, dt);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_kick_drift(double *x, double *y, double *z, double *vx, double *vy, double *vz,
                              const double *ax, const double *ay, const double *az, size_t n,
                              double dt, cudaStream_t s) {
  kick_drift_kernel<<<stream_grid(n, device_sms()), 256, 0, s>>>(x, y, z, vx, vy, vz, ax, ay, az, n, dt);
  count_launches(1);
  return cudaGetLastError();
}

int direct_chunks(size_t n, int n_targets) {
  const int blocks = (n_targets + kDirectThreads - 1) / kDirectThreads;
  const int want = device_sms() * 8;  // blocks that keep every SM busy
  if (blocks >= want || n < 65536) return 1;
  const long long c = std::min<long long>((want + blocks - 1) / blocks, (long long)(n / 4096));
  return (int)std::max(1ll, std::min(c, 256ll));
}

cudaError_t launch_direct(size_t n, const double *m, const double *x, const double *y, const double *z,
                          int n_targets, const int *targets, double g, double soft, double *ax,
                          double *ay, double *az, double *part, cudaStream_t s) {
  const int blocks = std::max(1, (n_targets + kDirectThreads - 1) / kDirectThreads);
  const int chunks = part ? direct_chunks(n, n_targets) : 1;
  direct_kernel<<<dim3(blocks, chunks), kDirectThreads, 0, s>>>((int)n, m, x, y, z, n_targets, targets, g,
                                                                soft * soft, ax, ay, az, part);
  if (chunks > 1) direct_combine_kernel<<<blocks, kDirectThreads, 0, s>>>(part, chunks, n_targets, ax, ay, az);
  count_launches(chunks > 1 ? 2 : 1);
  return cudaGetLastError();
}

cudaError_t launch_ref_octree_traversal(const RefOctree &o, const uint32_t *idx, const double *m,
                                        const double *x, const double *y, const double *z, double *ax,
                                        double *ay, double *az, double theta, double soft, double g,
                                        int morton_order, int *err, cudaStream_t s) {
  const int blocks = (o.n_particles + 127) / 128;
  ref_octree_kernel<<<blocks > 0 ? blocks : 1, 128, 0, s>>>(o, idx, m, x, y, z, ax, ay, az, theta,
                                                            soft * soft, g, morton_order, err);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace nbb
