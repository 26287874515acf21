// diagnostics.cu -- conserved quantities of the particle state: mass, centre
// of mass, linear and angular momentum, kinetic energy, and optionally the
// potential energy (Barnes-Hut with the plain form's acceptance test, or all
// pairs).  The reference lists these monitors as planned work
// (README.md:766-774 of sytrams/AMSC-Nbody); nothing here changes the state.
//
//   moments_kernel / moments_final_kernel
//       one pass over m, x, v into per-block partial sums, then one block
//       adds the partials in block order: deterministic for a given grid
//   potential_tree_kernel
//       phi_i = -G sum mu / sqrt(d^2 + eps^2) over the nodes and leaf
//       particles the plain walk would use for target i
//   potential_direct_kernel
//       phi_i over all j != i
#include "nbb_internal.cuh"
#include "walk_fp64.cuh"

#include <climits>
#include <cmath>

namespace nbb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kDirectThreads = 128;

// m, m x, m y, m z, m vx, m vy, m vz, Lx, Ly, Lz, kinetic, potential
constexpr int kQ = 12;

__device__ __forceinline__ void block_sum(double (&v)[kQ], double *shared) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kQ; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(kFull, v[q], o);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kQ; ++q) shared[warp * kQ + q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
#pragma unroll
      for (int q = 0; q < kQ; ++q) v[q] += shared[w * kQ + q];
  }
}

__global__ void __launch_bounds__(kThreads) moments_kernel(const double *m, const double *x, const double *y,
                                                           const double *z, const double *vx, const double *vy,
                                                           const double *vz, const double *phi, size_t n,
                                                           double *partials) {
  __shared__ double shared[(kThreads / 32) * kQ];
  double v[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) v[q] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double mi = m[i], px = x[i], py = y[i], pz = z[i], ux = vx[i], uy = vy[i], uz = vz[i];
    v[0] += mi;
    v[1] += mi * px;
    v[2] += mi * py;
    v[3] += mi * pz;
    v[4] += mi * ux;
    v[5] += mi * uy;
    v[6] += mi * uz;
    v[7] += mi * (py * uz - pz * uy);
    v[8] += mi * (pz * ux - px * uz);
    v[9] += mi * (px * uy - py * ux);
    v[10] += 0.5 * mi * (ux * ux + uy * uy + uz * uz);
    if (phi) v[11] += 0.5 * mi * phi[i];
  }
  block_sum(v, shared);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kQ; ++q) partials[blockIdx.x * kQ + q] = v[q];
}

__global__ void moments_final_kernel(const double *partials, int blocks, double *out) {
  if (threadIdx.x < kQ) {
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += partials[b * kQ + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

// The plain walk's node sequence for each target (Morton slot s), summing
// the potential instead of the acceleration.
__global__ void __launch_bounds__(256) potential_tree_kernel(Workspace ws, TraversalParams p, double *phi) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int lane = threadIdx.x & 31;
  const int n = ws.n;
  const int m = sc->n_nodes;
  const int n_groups = p.group_mode ? sc->n_tgroups : (n + 31) >> 5;
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
      const int sys = ws.n_systems > 1 ? ws.psys[g0] : 0;
      const int root = ws.root_pre[sys];
      const int end = (root >= 0 && root < m) ? min(ws.node_meta[root].x, m) : 0;
      const double soft = ws.sys_eps ? ws.sys_eps[sys] : p.soft;
      const double soft2 = soft * soft;
      double acc = 0.0;
      int resume = valid ? root : INT_MAX;
      int node = __reduce_min_sync(kFull, resume);
      while (node < end) {
        const int4 meta = ws.node_meta[node];
        const double4 a = ws.node_a[node];
        const double4 c = ws.node_c[node];
        if (resume == node) {
          if (meta.z > 0) {
            // two particles at a time (independent square roots and
            // divisions), added in order
            int k = 0;
            for (; k + 1 < meta.z; k += 2) {
              const int s0 = meta.y + k, s1 = s0 + 1;
              const double4 q0 = ws.pm4[s0], q1 = ws.pm4[s1];
              const double dx0 = q0.x - t.x, dy0 = q0.y - t.y, dz0 = q0.z - t.z;
              const double dx1 = q1.x - t.x, dy1 = q1.y - t.y, dz1 = q1.z - t.z;
              const double r20 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0 + soft2;
              const double r21 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1 + soft2;
              const double e0 = q0.w / sqrt(r20), e1 = q1.w / sqrt(r21);
              if (s0 != s && q0.w != 0.0 && r20 > 0.0) acc += e0;
              if (s1 != s && q1.w != 0.0 && r21 > 0.0) acc += e1;
            }
            if (k < meta.z) {
              const int sp = meta.y + k;
              const double4 q = ws.pm4[sp];
              if (sp != s && q.w != 0.0) {
                const double dx = q.x - t.x, dy = q.y - t.y, dz = q.z - t.z;
                const double r2 = dx * dx + dy * dy + dz * dz + soft2;
                if (r2 > 0.0) acc += q.w / sqrt(r2);
              }
            }
            resume = meta.x;
          } else if (a.w == 0.0) {
            resume = meta.x;
          } else {
            double dx, dy, dz, d2;
            if (accept_fp64(a, ws.node_b + node, c, t, dx, dy, dz, d2)) {
              const double r2 = d2 + soft2;
              if (r2 > 0.0) acc += a.w / sqrt(r2);
              resume = meta.x;
            } else {
              resume = node + 1;
            }
          }
        }
        if (resume <= node) resume = node + 1;
        node = __reduce_min_sync(kFull, resume);
      }
      if (valid) phi[ws.idx[s]] = -p.g * acc;
    }
  }
}

__global__ void __launch_bounds__(kDirectThreads) potential_direct_kernel(const double *m, const double *x,
                                                                          const double *y, const double *z, int n,
                                                                          double g, double soft2, double *phi) {
  __shared__ double4 tile[kDirectThreads];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < n;
  const int kk = active ? k : 0;
  const double tx = x[kk], ty = y[kk], tz = z[kk];
  double acc = 0.0;
  for (int base = 0; base < n; base += kDirectThreads) {
    const int j = base + threadIdx.x;
    tile[threadIdx.x] = (j < n) ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int lim = min(n - base, kDirectThreads);
    if (active)
      for (int q = 0; q < lim; ++q) {
        if (base + q == k) continue;
        const double4 s = tile[q];
        const double dx = s.x - tx, dy = s.y - ty, dz = s.z - tz;
        const double r2 = dx * dx + dy * dy + dz * dz + soft2;
        if (r2 > 0.0) acc += s.w / sqrt(r2);
      }
    __syncthreads();
  }
  if (active) phi[k] = -g * acc;
}

}  // namespace

cudaError_t launch_moments(const double *m, const double *x, const double *y, const double *z, const double *vx,
                           const double *vy, const double *vz, const double *phi, size_t n, double *partials,
                           int blocks, double *out, cudaStream_t s) {
  moments_kernel<<<blocks, kThreads, 0, s>>>(m, x, y, z, vx, vy, vz, phi, n, partials);
  moments_final_kernel<<<1, 32, 0, s>>>(partials, blocks, out);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_potential_tree(Workspace &ws, const TraversalParams &p, double *phi, cudaStream_t s) {
  // the walk takes work from the traversal counter; the build's reset
  // zeroed it
  potential_tree_kernel<<<ws.fp64_grid > 0 ? ws.fp64_grid : 148, 256, 0, s>>>(ws, p, phi);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_potential_direct(const double *m, const double *x, const double *y, const double *z, int n,
                                    double g, double soft, double *phi, cudaStream_t s) {
  const int blocks = (n + kDirectThreads - 1) / kDirectThreads;
  potential_direct_kernel<<<blocks > 0 ? blocks : 1, kDirectThreads, 0, s>>>(m, x, y, z, n, g, soft * soft, phi);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace nbb
