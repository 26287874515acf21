// adjoint.cu -- reverse-mode derivative of the Barnes-Hut force with the tree
// frozen, a frozen-structure replay for finite differences, and the FP64
// direct-sum adjoint.  None of this has a counterpart in sytrams/AMSC-Nbody;
// the force being differentiated is the plain form of barnes_hut.cu:164-322.
//
// Force with frozen structure.  For target i with accepted-node set A_i and
// opened-leaf particle set L_i (both decided by the reference's acceptance
// test on the positions the tree was built from),
//
//   a_i = G sum_{s in A_i u L_i} mu_s phi(Y_s - x_i),  phi(r) = r (|r|^2 + eps^2)^-3/2
//
// with (mu, Y) = (M_c, X_c) for a node (mass, centre of mass) and (m_j, x_j)
// for a particle.  For an accelerations cotangent c_i and r = Y_s - x_i,
//
//   u = G mu (inv3 c_i - 3 inv5 (r . c_i) r),  inv3 = (|r|^2+eps^2)^-3/2, inv5 = inv3 / (|r|^2+eps^2)
//   d/dx_i  -= u,   d/dY_s += u,   d/dmu_s += G inv3 (r . c_i).
//
// A node's (M_c, X_c) is a function of its particles: M_c = sum m_j,
// X_c = sum m_j x_j / M_c, so with P_c = gX_c / M_c and Q_c = gM_c - X_c . P_c
// a particle j receives  m_j sum P_c  and  sum Q_c + x_j . sum P_c  over every
// node c on its root path -- a prefix sum down the tree instead of a scatter
// over each node's particles.
//
//   adj_topology_kernel  preorder parent and Morton particle range per node
//   adjoint_walk_kernel  the plain walk's visit order, vector-Jacobian products;
//                        node / particle cotangents reduced across the warp
//                        (all lanes at a node share it) and added atomically
//   adj_node_kernel      (gX, gM) -> (P, Q) per node
//   adj_leaf_kernel      root-path sums, per-particle totals, velocity update
//   frozen_*             the force on perturbed copies of the particles with
//                        the tree, acceptance decisions and leaf sets of the
//                        unperturbed particles (all copies in one launch per
//                        stage; node masses bottom-up, one launch per level)
//   direct_vjp_kernel    adjoint of the FP64 direct sum (all pairs)
#include "nbb_internal.cuh"
#include "walk_fp64.cuh"

#include <climits>
#include <cmath>

namespace nbb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlock = 256;
constexpr int kDirectVjpThreads = 128;

inline int grid_of_ws(const Workspace &ws, int per_sm) {
  return (ws.num_sms > 0 ? ws.num_sms : 148) * per_sm;
}

// u and the mass term of one interaction (see the file comment).
__device__ __forceinline__ bool vjp_pair(double dx, double dy, double dz, double d2, double mu, double g,
                                         double soft2, double cx, double cy, double cz, double &ux,
                                         double &uy, double &uz, double &uw) {
  const double r2 = d2 + soft2;
  if (!(r2 > 0.0)) {
    ux = uy = uz = uw = 0.0;
    return false;
  }
  const double inv = 1.0 / sqrt(r2);
  const double inv2 = inv * inv;
  const double gi3 = g * inv2 * inv;
  const double rc = dx * cx + dy * cy + dz * cz;
  const double f = gi3 * mu;
  const double h = 3.0 * f * inv2 * rc;
  ux = f * cx - h * dx;
  uy = f * cy - h * dy;
  uz = f * cz - h * dz;
  uw = gi3 * rc;
  return true;
}

// Add (ux, uy, uz, uw) of the lanes in `who` (warp-uniform ballot; other
// lanes hold zeros) to dst: one lane's values directly, otherwise a butterfly
// sum and lanes 0..3 each add one component.
__device__ __forceinline__ void scatter4(double4 *dst, unsigned who, int lane, double ux, double uy,
                                         double uz, double uw) {
  double *d = reinterpret_cast<double *>(dst);
  if (__popc(who) == 1) {
    if (lane == __ffs(who) - 1) {
      atomicAdd(d + 0, ux);
      atomicAdd(d + 1, uy);
      atomicAdd(d + 2, uz);
      atomicAdd(d + 3, uw);
    }
    return;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ux += __shfl_xor_sync(kFull, ux, o);
    uy += __shfl_xor_sync(kFull, uy, o);
    uz += __shfl_xor_sync(kFull, uz, o);
    uw += __shfl_xor_sync(kFull, uw, o);
  }
  const double v = (lane == 0) ? ux : (lane == 1) ? uy : (lane == 2) ? uz : uw;
  if (lane < 4) atomicAdd(d + lane, v);
}

__global__ void adj_reset_kernel(DevScalars *sc) {
  if (threadIdx.x == 0) sc->work_counter = 0;
}

// Preorder parent and Morton-order particle range of every octree node
// (pre = sum of preorder offsets up the parent chain, as the layout does).
__global__ void __launch_bounds__(kBlock) adj_topology_kernel(Workspace ws, int *pparent, int2 *prange,
                                                              int *pre_of) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    int pre = 0, u = v, guard = 0;
    while (u != 0) {
      pre += ws.preoff[u];
      u = ws.oparent[u];
      if (u < 0 || ++guard > ws.max_level + 1) break;
    }
    if (u != 0 || pre < 0 || pre >= m) {
      record_error(sc, kStageLayout, 1);
      continue;
    }
    if (pre_of) pre_of[v] = pre;
    pparent[pre] = (v == 0) ? -1 : pre - ws.preoff[v];
    const bool leaf = ws.child_count[v] == 0;
    const int cnt = leaf ? max(ws.ocount[v], 0) : ws.psub[v];
    const int first = leaf ? ws.ofirst[v] : ws.pfirst[v];
    prange[pre] = (cnt > 0 && first >= 0 && first + cnt <= ws.n) ? make_int2(first, cnt) : make_int2(0, 0);
  }
}

// Vector-Jacobian product of the frozen-structure force: the plain walk's
// node sequence per lane (same records, same acceptance test), with the
// accelerations cotangent coef * gv of each target.
__global__ void __launch_bounds__(256) adjoint_walk_kernel(Workspace ws, TraversalParams p, AdjointBuffers ab) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int lane = threadIdx.x & 31;
  const int n = ws.n;
  const int m = sc->n_nodes;
  const int n_groups = p.group_mode ? sc->n_tgroups : (n + 31) >> 5;
  const double g = p.g;
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
      double cx = 0.0, cy = 0.0, cz = 0.0;
      if (valid) {
        t = ws.pm4[s];
        const uint32_t ti = ws.idx[s];
        cx = ab.coef * ab.gvx[ti];
        cy = ab.coef * ab.gvy[ti];
        cz = ab.coef * ab.gvz[ti];
      }
      const int sys = ws.n_systems > 1 ? ws.psys[g0] : 0;
      const int root = ws.root_pre[sys];
      const int end = (root >= 0 && root < m) ? min(ws.node_meta[root].x, m) : 0;
      const double soft = ws.sys_eps ? ws.sys_eps[sys] : p.soft;
      const double soft2 = __dmul_rn(soft, soft);
      double gtx = 0.0, gty = 0.0, gtz = 0.0;
      int resume = valid ? root : INT_MAX;
      int node = __reduce_min_sync(kFull, resume);
      while (node < end) {
        const int4 meta = ws.node_meta[node];
        const double4 a = ws.node_a[node];
        const bool here = resume == node;
        if (meta.z > 0) {
          // two particles at a time: both products are formed (independent
          // square roots and divisions) before they are added and scattered
          // in particle order
          int k = 0;
          for (; k + 1 < meta.z; k += 2) {
            const int s0 = meta.y + k, s1 = s0 + 1;
            const double4 q0 = ws.pm4[s0], q1 = ws.pm4[s1];
            const bool act0 = here && s0 != s && q0.w != 0.0;
            const bool act1 = here && s1 != s && q1.w != 0.0;
            double u0x = 0.0, u0y = 0.0, u0z = 0.0, u0w = 0.0, u1x = 0.0, u1y = 0.0, u1z = 0.0, u1w = 0.0;
            if (act0) {
              const double dx = __dsub_rn(q0.x, t.x), dy = __dsub_rn(q0.y, t.y), dz = __dsub_rn(q0.z, t.z);
              singular |= !vjp_pair(dx, dy, dz, sqdist(dx, dy, dz), q0.w, g, soft2, cx, cy, cz, u0x, u0y, u0z, u0w);
            }
            if (act1) {
              const double dx = __dsub_rn(q1.x, t.x), dy = __dsub_rn(q1.y, t.y), dz = __dsub_rn(q1.z, t.z);
              singular |= !vjp_pair(dx, dy, dz, sqdist(dx, dy, dz), q1.w, g, soft2, cx, cy, cz, u1x, u1y, u1z, u1w);
            }
            if (act0) {
              gtx -= u0x;
              gty -= u0y;
              gtz -= u0z;
            }
            const unsigned who0 = __ballot_sync(kFull, act0);
            if (who0) scatter4(ab.part_g + s0, who0, lane, u0x, u0y, u0z, u0w);
            if (act1) {
              gtx -= u1x;
              gty -= u1y;
              gtz -= u1z;
            }
            const unsigned who1 = __ballot_sync(kFull, act1);
            if (who1) scatter4(ab.part_g + s1, who1, lane, u1x, u1y, u1z, u1w);
          }
          if (k < meta.z) {
            const int sp = meta.y + k;
            const double4 q = ws.pm4[sp];
            const bool act = here && sp != s && q.w != 0.0;
            double ux = 0.0, uy = 0.0, uz = 0.0, uw = 0.0;
            if (act) {
              const double dx = __dsub_rn(q.x, t.x), dy = __dsub_rn(q.y, t.y), dz = __dsub_rn(q.z, t.z);
              singular |= !vjp_pair(dx, dy, dz, sqdist(dx, dy, dz), q.w, g, soft2, cx, cy, cz, ux, uy, uz, uw);
              gtx -= ux;
              gty -= uy;
              gtz -= uz;
            }
            const unsigned who = __ballot_sync(kFull, act);
            if (who) scatter4(ab.part_g + sp, who, lane, ux, uy, uz, uw);
          }
          if (here) resume = meta.x;
        } else if (a.w == 0.0) {
          if (here) resume = meta.x;
        } else {
          const double4 c = ws.node_c[node];
          bool acc = false;
          double ux = 0.0, uy = 0.0, uz = 0.0, uw = 0.0;
          if (here) {
            double dx, dy, dz, d2;
            acc = accept_fp64(a, ws.node_b + node, c, t, dx, dy, dz, d2);
            if (acc) {
              singular |= !vjp_pair(dx, dy, dz, d2, a.w, g, soft2, cx, cy, cz, ux, uy, uz, uw);
              gtx -= ux;
              gty -= uy;
              gtz -= uz;
            }
            resume = acc ? meta.x : node + 1;
          }
          const unsigned who = __ballot_sync(kFull, acc);
          if (who) scatter4(ab.node_g + node, who, lane, ux, uy, uz, uw);
        }
        if (resume <= node) resume = node + 1;
        node = __reduce_min_sync(kFull, resume);
      }
      if (valid) ab.tgt_g[s] = make_double4(gtx, gty, gtz, 0.0);
    }
  }
  if (__any_sync(kFull, singular) && lane == 0) record_error(sc, kStageTraversal, 6);
}

// (gX, gM) of a node -> (P, Q) = (gX / M, gM - X . gX / M).
__global__ void __launch_bounds__(kBlock) adj_node_kernel(Workspace ws, AdjointBuffers ab) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int pre = blockIdx.x * blockDim.x + threadIdx.x; pre < m; pre += gridDim.x * blockDim.x) {
    const double4 gg = ab.node_g[pre];
    const double4 a = ws.node_a[pre];
    double px = 0.0, py = 0.0, pz = 0.0, q = gg.w;
    if (a.w > 0.0) {
      const double inv = 1.0 / a.w;
      px = gg.x * inv;
      py = gg.y * inv;
      pz = gg.z * inv;
      q = gg.w - (a.x * px + a.y * py + a.z * pz);
    }
    ab.node_g[pre] = make_double4(px, py, pz, q);
  }
}

// Per occupied leaf: sums of (P, Q) along the root path, then each of its
// particles' total position / mass cotangent of this force evaluation; adds
// them to the running cotangents and, when dt_v != 0, carries the position
// cotangent into the velocity cotangent (gv += dt gx, the drift's adjoint).
__global__ void __launch_bounds__(kBlock) adj_leaf_kernel(Workspace ws, AdjointBuffers ab) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int pre = blockIdx.x * blockDim.x + threadIdx.x; pre < m; pre += gridDim.x * blockDim.x) {
    const int4 meta = ws.node_meta[pre];
    if (meta.z <= 0) continue;
    double px = 0.0, py = 0.0, pz = 0.0, q = 0.0;
    int v = pre, guard = 0;
    while (v >= 0) {
      if (v >= m || ++guard > ws.max_level + 2) {
        record_error(sc, kStageLayout, 2);
        break;
      }
      const double4 pq = ab.node_g[v];
      px += pq.x;
      py += pq.y;
      pz += pq.z;
      q += pq.w;
      v = ab.pparent[v];
    }
    for (int k = 0; k < meta.z; ++k) {
      const int sp = meta.y + k;
      if (sp < 0 || sp >= ws.n) break;
      const uint32_t j = ws.idx[sp];
      const double4 pt = ws.pm4[sp];
      const double4 tg = ab.tgt_g[sp];
      const double4 pg = ab.part_g[sp];
      const double gx = ab.gx[j] + (tg.x + pg.x + pt.w * px);
      const double gy = ab.gy[j] + (tg.y + pg.y + pt.w * py);
      const double gz = ab.gz[j] + (tg.z + pg.z + pt.w * pz);
      ab.gx[j] = gx;
      ab.gy[j] = gy;
      ab.gz[j] = gz;
      ab.gm[j] += pg.w + q + (pt.x * px + pt.y * py + pt.z * pz);
      if (ab.dt_v != 0.0) {
        ab.gvx[j] += ab.dt_v * gx;
        ab.gvy[j] += ab.dt_v * gy;
        ab.gvz[j] += ab.dt_v * gz;
      }
    }
  }
}

// ------------------------------------------------------------ frozen ----

// Perturbed copies in the unperturbed Morton order (copy q at q * n).
__global__ void frozen_gather_kernel(Workspace ws, FrozenBatch fb) {
  const size_t n = (size_t)ws.n, total = n * (size_t)fb.copies;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const size_t q = k / n, sp = k - q * n;
    const size_t j = q * n + ws.idx[sp];
    fb.pm4q[k] = make_double4(fb.x[j], fb.y[j], fb.z[j], fb.m[j]);
  }
}

// Mass and centre of mass of every copy's particles in each node of one
// octree level (deepest level first): leaves sum their particles in Morton
// order, internal nodes combine their children in octant order 0..7.  Values
// are kept by octree id (for the parents) and written at the preorder id.
__global__ void __launch_bounds__(kBlock) frozen_level_kernel(Workspace ws, FrozenBatch fb, int level) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const size_t m = (size_t)sc->n_nodes, cap = (size_t)ws.cap_nodes, n = (size_t)ws.n;
  const size_t total = m * (size_t)fb.copies;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const size_t q = k / m;
    const int v = (int)(k - q * m);
    if (ws.olevel[v] != level) continue;
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    if (ws.child_count[v] == 0) {
      const int f = ws.ofirst[v], c = ws.ocount[v];
      if (c > 0 && f >= 0 && (size_t)(f + c) <= n) {
        const double4 *pq = fb.pm4q + q * n + f;
        for (int i = 0; i < c; ++i) {
          const double4 t = pq[i];
          tm += t.w;
          wx = fma(t.w, t.x, wx);
          wy = fma(t.w, t.y, wy);
          wz = fma(t.w, t.z, wz);
        }
      }
    } else {
      for (int o = 0; o < 8; ++o) {
        const int c = ws.children[(size_t)v * 8 + o];
        if (c <= 0 || (size_t)c >= m) continue;
        const double4 t = fb.aq_oct[q * cap + c];
        tm += t.w;
        wx = fma(t.w, t.x, wx);
        wy = fma(t.w, t.y, wy);
        wz = fma(t.w, t.z, wz);
      }
    }
    const double4 r = (tm > 0.0) ? make_double4(wx / tm, wy / tm, wz / tm, tm) : make_double4(0.0, 0.0, 0.0, 0.0);
    fb.aq_oct[q * cap + v] = r;
    const int pre = fb.pre_of[v];
    if (pre >= 0 && (size_t)pre < m) fb.node_aq[q * cap + pre] = r;
  }
}

// Force on each perturbed copy: visit order, acceptance decisions, zero-mass
// skips and self exclusion from the unperturbed tree and targets; offsets,
// masses and centres of mass from the copy.  Work items are (copy, target
// group) pairs taken from one counter, so every copy's walk shares the grid.
__global__ void __launch_bounds__(256) frozen_walk_kernel(Workspace ws, TraversalParams p, FrozenBatch fb) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int lane = threadIdx.x & 31;
  const int n = ws.n;
  const int m = sc->n_nodes;
  const size_t cap = (size_t)ws.cap_nodes;
  const int n_groups = p.group_mode ? sc->n_tgroups : (n + 31) >> 5;
  const unsigned items = (unsigned)n_groups * (unsigned)fb.copies;
  const double g = p.g;
  bool singular = false;
  while (true) {
    unsigned item = 0;
    if (lane == 0) item = atomicAdd(&sc->work_counter, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= items) break;
    const int q = (int)(item / (unsigned)n_groups);
    const int grp = (int)(item - (unsigned)q * (unsigned)n_groups);
    const double4 *pm4q = fb.pm4q + (size_t)q * n;
    const double4 *node_aq = fb.node_aq + (size_t)q * cap;
    const int g0 = p.group_mode ? ws.tstart[grp] : grp * 32;
    const int g1 = p.group_mode ? ((grp + 1 < n_groups) ? ws.tstart[grp + 1] : n) : min(g0 + 32, n);
    // a group larger than a warp is walked 32 targets at a time
    for (int c0 = g0; c0 < g1; c0 += 32) {
      const int c1 = min(c0 + 32, g1);
      const int s = c0 + lane;
      const bool valid = s < c1 && s < n;
      double4 t = make_double4(0.0, 0.0, 0.0, 0.0), tq = t;
      if (valid) {
        t = ws.pm4[s];
        tq = pm4q[s];
      }
      const int sys = ws.n_systems > 1 ? ws.psys[g0] : 0;
      const int root = ws.root_pre[sys];
      const int end = (root >= 0 && root < m) ? min(ws.node_meta[root].x, m) : 0;
      const double soft = ws.sys_eps ? ws.sys_eps[sys] : p.soft;
      const double soft2 = __dmul_rn(soft, soft);
      double ax = 0.0, ay = 0.0, az = 0.0;
      int resume = valid ? root : INT_MAX;
      int node = __reduce_min_sync(kFull, resume);
      while (node < end) {
        const int4 meta = ws.node_meta[node];
        const double4 a = ws.node_a[node];
        const double4 c = ws.node_c[node];
        if (resume == node) {
          if (meta.z > 0) {
            for (int k = 0; k < meta.z; ++k) {
              const int sp = meta.y + k;
              if (sp == s) continue;
              if (ws.pm4[sp].w == 0.0) continue;
              const double4 u = pm4q[sp];
              const double dx = __dsub_rn(u.x, tq.x), dy = __dsub_rn(u.y, tq.y), dz = __dsub_rn(u.z, tq.z);
              singular |= !point_mass_fp64(dx, dy, dz, sqdist(dx, dy, dz), u.w, g, soft2, ax, ay, az);
            }
            resume = meta.x;
          } else if (a.w == 0.0) {
            resume = meta.x;
          } else {
            double dx, dy, dz, d2;
            if (accept_fp64(a, ws.node_b + node, c, t, dx, dy, dz, d2)) {
              const double4 aq = node_aq[node];
              const double ex = __dsub_rn(aq.x, tq.x), ey = __dsub_rn(aq.y, tq.y), ez = __dsub_rn(aq.z, tq.z);
              singular |= !point_mass_fp64(ex, ey, ez, sqdist(ex, ey, ez), aq.w, g, soft2, ax, ay, az);
              resume = meta.x;
            } else {
              resume = node + 1;
            }
          }
        }
        if (resume <= node) resume = node + 1;
        node = __reduce_min_sync(kFull, resume);
      }
      if (valid) {
        const size_t ti = (size_t)q * n + ws.idx[s];
        fb.ax[ti] = ax;
        fb.ay[ti] = ay;
        fb.az[ti] = az;
      }
    }
  }
  if (__any_sync(kFull, singular) && lane == 0) record_error(sc, kStageTraversal, 6);
}

// ------------------------------------------------------------ direct ----

// Adjoint of a_i = G sum_{j != i} m_j phi(x_j - x_i) for the cotangent
// c = coef * gv: with r = x_j - x_k and w = m_k c_j - m_j c_k,
//   gx_k += G sum_j (inv3 w - 3 inv5 (r . w) r),   gm_k -= G sum_j inv3 (r . c_j).
__global__ void __launch_bounds__(kDirectVjpThreads)
    direct_vjp_kernel(int n, const double *__restrict__ m, const double *__restrict__ x,
                      const double *__restrict__ y, const double *__restrict__ z,
                      const double *__restrict__ gvx, const double *__restrict__ gvy,
                      const double *__restrict__ gvz, double coef, double g, double soft2, double *gx,
                      double *gy, double *gz, double *gm) {
  __shared__ double4 tp[kDirectVjpThreads];
  __shared__ double4 tc[kDirectVjpThreads];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < n;
  const int kk = active ? k : 0;
  const double xk = x[kk], yk = y[kk], zk = z[kk], mk = m[kk];
  const double ckx = coef * gvx[kk], cky = coef * gvy[kk], ckz = coef * gvz[kk];
  double ax = 0.0, ay = 0.0, az = 0.0, am = 0.0;
  for (int base = 0; base < n; base += kDirectVjpThreads) {
    const int j = base + threadIdx.x;
    tp[threadIdx.x] = (j < n) ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    tc[threadIdx.x] = (j < n) ? make_double4(coef * gvx[j], coef * gvy[j], coef * gvz[j], 0.0)
                              : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int lim = (n - base < kDirectVjpThreads) ? n - base : kDirectVjpThreads;
    if (active) {
      for (int q = 0; q < lim; ++q) {
        if (base + q == k) continue;
        const double4 s = tp[q];
        const double4 cj = tc[q];
        const double rx = s.x - xk, ry = s.y - yk, rz = s.z - zk;
        const double r2 = rx * rx + ry * ry + rz * rz + soft2;
        if (!(r2 > 0.0)) continue;
        const double inv = 1.0 / sqrt(r2);
        const double inv2 = inv * inv;
        const double gi3 = g * inv2 * inv;
        const double wx = mk * cj.x - s.w * ckx, wy = mk * cj.y - s.w * cky, wz = mk * cj.z - s.w * ckz;
        const double h = 3.0 * gi3 * inv2 * (rx * wx + ry * wy + rz * wz);
        ax += gi3 * wx - h * rx;
        ay += gi3 * wy - h * ry;
        az += gi3 * wz - h * rz;
        am -= gi3 * (rx * cj.x + ry * cj.y + rz * cj.z);
      }
    }
    __syncthreads();
  }
  if (active) {
    gx[k] += ax;
    gy[k] += ay;
    gz[k] += az;
    gm[k] += am;
  }
}

// y += a x over three arrays.
__global__ void axpy3_kernel(double *yx, double *yy, double *yz, const double *xx, const double *xy,
                             const double *xz, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    yx[i] += a * xx[i];
    yy[i] += a * xy[i];
    yz[i] += a * xz[i];
  }
}

}  // namespace

// ------------------------------------------------------------ launches ---

cudaError_t launch_adjoint_force(Workspace &ws, const TraversalParams &p, const AdjointBuffers &ab,
                                 cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(ab.node_g, 0, sizeof(double4) * (size_t)ws.cap_nodes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ab.part_g, 0, sizeof(double4) * (size_t)ws.n, s);
  if (e != cudaSuccess) return e;
  const int grid = grid_of_ws(ws, 8);
  adj_reset_kernel<<<1, 32, 0, s>>>(ws.sc);
  adj_topology_kernel<<<grid, kBlock, 0, s>>>(ws, ab.pparent, ab.prange, nullptr);
  if (p.precision == 1) {
    e = launch_adjoint_mixed(ws, p, ab, s);
    if (e != cudaSuccess) return e;
  } else {
    adjoint_walk_kernel<<<grid_of_ws(ws, 8), 256, 0, s>>>(ws, p, ab);
  }
  adj_node_kernel<<<grid, kBlock, 0, s>>>(ws, ab);
  adj_leaf_kernel<<<grid, kBlock, 0, s>>>(ws, ab);
  count_launches(p.precision == 1 ? 4 : 5);
  return cudaGetLastError();
}

cudaError_t launch_frozen_force(Workspace &ws, const TraversalParams &p, const FrozenBatch &fb, cudaStream_t s) {
  const int grid = grid_of_ws(ws, 8);
  adj_reset_kernel<<<1, 32, 0, s>>>(ws.sc);
  adj_topology_kernel<<<grid, kBlock, 0, s>>>(ws, fb.pparent, fb.prange, fb.pre_of);
  frozen_gather_kernel<<<grid, kBlock, 0, s>>>(ws, fb);
  for (int level = ws.max_level; level >= 0; --level) frozen_level_kernel<<<grid, kBlock, 0, s>>>(ws, fb, level);
  frozen_walk_kernel<<<grid, 256, 0, s>>>(ws, p, fb);
  count_launches(5 + ws.max_level);
  return cudaGetLastError();
}

cudaError_t launch_direct_vjp(size_t n, const double *m, const double *x, const double *y, const double *z,
                              const double *gvx, const double *gvy, const double *gvz, double coef, double g,
                              double soft, double *gx, double *gy, double *gz, double *gm, cudaStream_t s) {
  const int blocks = (int)((n + kDirectVjpThreads - 1) / kDirectVjpThreads);
  direct_vjp_kernel<<<blocks > 0 ? blocks : 1, kDirectVjpThreads, 0, s>>>(
      (int)n, m, x, y, z, gvx, gvy, gvz, coef, g, soft * soft, gx, gy, gz, gm);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_axpy3(double *yx, double *yy, double *yz, const double *xx, const double *xy, const double *xz,
                         double a, size_t n, cudaStream_t s) {
  size_t blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  axpy3_kernel<<<blocks > 0 ? (int)blocks : 1, 256, 0, s>>>(yx, yy, yz, xx, xy, xz, a, n);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace nbb
