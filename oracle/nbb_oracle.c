/*
 * nbb_oracle.c -- CPU restatement of the AMSC-Nbody Barnes-Hut step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * nbb_oracle.h.  Each function cites the reference statements it restates
 * (paths relative to the sytrams/AMSC-Nbody project root).  Parity of this
 * restatement is pinned by tests/test_oracle_golden.py against the known
 * answers of the reference's own test-suite and against fixtures produced by
 * the reference itself (tests/golden/make_golden.py).
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off -mfma).
 */
#include "nbb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* radix_to_octree.hpp:10-19 */
#define MORTON_DIMS 3
#define MORTON_BITS_PER_AXIS 10
#define MORTON_SPATIAL_BITS 30
#define MORTON_PADDING_BITS 2
#define OCTREE_MAX_LEVEL 10
#define MORTON_SPATIAL_MASK 0x3FFFFFFFu

static void set_threads(int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
}

/* ---------------------------------------------------------------- bbox -- */

int orc_bbox(size_t n, const double *x, const double *y, const double *z,
             double out[4]) {
  /* globalbounding.cu:96-99: empty input is rejected. */
  if (n == 0) return ORC_EINVAL;
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  int non_finite = 0;
  /* globalbounding.cu:17-56: per-particle degenerate box, component-wise
   * fmin/fmax combine, non-finite flag OR-ed. */
  for (size_t i = 0; i < n; ++i) {
    const double p[3] = {x[i], y[i], z[i]};
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) non_finite = 1;
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], p[a]);
      hi[a] = fmax(hi[a], p[a]);
    }
  }
  /* globalbounding.cu:117-120 */
  if (non_finite) return ORC_EDOMAIN;
  /* globalbounding.cu:122-136 */
  out[0] = (lo[0] + hi[0]) * 0.5;
  out[1] = (lo[1] + hi[1]) * 0.5;
  out[2] = (lo[2] + hi[2]) * 0.5;
  double ext = hi[0] - lo[0];
  if (hi[1] - lo[1] > ext) ext = hi[1] - lo[1];
  if (hi[2] - lo[2] > ext) ext = hi[2] - lo[2];
  double side = 1.1 * ext;
  if (side == 0.0) side = 1.0;
  out[3] = side;
  return ORC_OK;
}

/* -------------------------------------------------------------- morton -- */

/* morton.cu:119-128 */
static uint32_t expand_bits(uint32_t v) {
  uint32_t x = v & 0x000003FFu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

/* morton.cu:98-117: normalise against the cube, scale by the 1024-cell
 * grid, clamp to [0, 1023] and truncate. */
static uint32_t quantise(double a, double centre, double side) {
  const double lower = centre - side / 2.0;
  const double normalised = (a - lower) / side;
  const double scaled = normalised * 1024.0;
  const double clamped = fmin(fmax(scaled, 0.0), 1023.0);
  return (uint32_t)clamped;
}

/* Stable LSD radix sort of (key, value) pairs over all 32 key bits: the
 * result equals std::stable_sort / thrust::stable_sort_by_key
 * (morton.cu:221-224). */
static void stable_sort_pairs(size_t n, uint32_t *keys, uint32_t *vals) {
  uint32_t *k2 = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *v2 = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *ks = keys, *vs = vals, *kd = k2, *vd = v2;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t hist[257];
    memset(hist, 0, sizeof(hist));
    for (size_t i = 0; i < n; ++i) hist[((ks[i] >> shift) & 255u) + 1]++;
    for (int d = 0; d < 256; ++d) hist[d + 1] += hist[d];
    for (size_t i = 0; i < n; ++i) {
      const size_t pos = hist[(ks[i] >> shift) & 255u]++;
      kd[pos] = ks[i];
      vd[pos] = vs[i];
    }
    uint32_t *t = ks; ks = kd; kd = t;
    t = vs; vs = vd; vd = t;
  }
  /* four passes: the data is back in the caller's arrays */
  free(k2);
  free(v2);
}

int orc_morton(size_t n, const double *x, const double *y, const double *z,
               const double box[4], uint32_t *keys, uint32_t *idx) {
  /* morton.cu:34-60 */
  if (n == 0 || !x || !y || !z) return ORC_EINVAL;
  /* morton.cu:167-170 */
  if (!isfinite(box[0]) || !isfinite(box[1]) || !isfinite(box[2]) ||
      !isfinite(box[3]) || box[3] <= 0.0)
    return ORC_EINVAL;
  for (size_t i = 0; i < n; ++i) {
    const uint32_t qx = quantise(x[i], box[0], box[3]);
    const uint32_t qy = quantise(y[i], box[1], box[3]);
    const uint32_t qz = quantise(z[i], box[2], box[3]);
    /* morton.cu:130-139 */
    keys[i] = (expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz);
    idx[i] = (uint32_t)i; /* morton.cu:165 */
  }
  stable_sort_pairs(n, keys, idx);
  return ORC_OK;
}

/* --------------------------------------------------------- leaf groups -- */

int orc_leaf_groups(int n, const uint32_t *sorted_keys, uint32_t *uniq,
                    int *first, int *count) {
  /* morton_leaf_groups.cu:60-70 */
  if (n <= 0 || !sorted_keys) return ORC_EINVAL;
  /* cub::DeviceRunLengthEncode::Encode + cub::DeviceScan::ExclusiveSum
   * (morton_leaf_groups.cu:76-98). */
  int g = 0;
  for (int i = 0; i < n; ++i) {
    if (i == 0 || sorted_keys[i] != sorted_keys[i - 1]) {
      uniq[g] = sorted_keys[i];
      count[g] = 0;
      ++g;
    }
    count[g - 1]++;
  }
  int running = 0;
  for (int j = 0; j < g; ++j) {
    first[j] = running;
    running += count[j];
  }
  return g;
}

/* ------------------------------------------------------------- karras -- */

static int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

/* tree_builder.cu:9-24 */
static int lcp(const uint32_t *keys, int i, int j, int n) {
  if (j < 0 || j >= n) return -1;
  if (i == j) return 64;
  const uint32_t a = keys[i], b = keys[j];
  if (a != b) return clz32(a ^ b);
  return 32 + clz32((uint32_t)(i ^ j));
}

/* tree_builder.cu:30-62 */
static void determine_range(const uint32_t *keys, int i, int n, int *first,
                            int *last) {
  const int dright = lcp(keys, i, i + 1, n);
  const int dleft = lcp(keys, i, i - 1, n);
  const int dir = (dright > dleft) ? 1 : -1;
  const int dmin = lcp(keys, i, i - dir, n);
  int length = 2;
  while (lcp(keys, i, i + length * dir, n) > dmin) length *= 2;
  int l = 0;
  for (int t = length / 2; t >= 1; t /= 2)
    if (lcp(keys, i, i + (l + t) * dir, n) > dmin) l += t;
  const int j = i + l * dir;
  *first = (i < j) ? i : j;
  *last = (i > j) ? i : j;
}

/* tree_builder.cu:64-84 (note the `candidate < last` guard) */
static int find_split(const uint32_t *keys, int first, int last, int n) {
  if (first >= last) return first;
  const int node_prefix = lcp(keys, first, last, n);
  int split = first;
  int step = last - first;
  do {
    step = (step + 1) >> 1;
    const int candidate = split + step;
    if (candidate < last && lcp(keys, first, candidate, n) > node_prefix)
      split = candidate;
  } while (step > 1);
  return split;
}

int orc_radix_tree(int n, const uint32_t *keys, int *left, int *right,
                   int *rfirst, int *rlast, int *plen, int *parent) {
  if (n <= 0 || !keys) return ORC_EINVAL; /* tree_builder.cu:305-324 */
  /* tree_builder.cu:328: parent initialised to -1 */
  for (int i = 0; i < 2 * n - 1; ++i) parent[i] = -1;
  /* tree_builder.cu:87-113 */
  for (int i = 0; i < n - 1; ++i) {
    int first, last;
    determine_range(keys, i, n, &first, &last);
    rfirst[i] = first;
    rlast[i] = last;
    plen[i] = lcp(keys, first, last, n);
    const int split = find_split(keys, first, last, n);
    const int lc = (split == first) ? split : n + split;
    const int rc = (split + 1 == last) ? split + 1 : n + split + 1;
    left[i] = lc;
    right[i] = rc;
    parent[lc] = n + i;
    parent[rc] = n + i;
  }
  return ORC_OK;
}

/* --------------------------------------------------------------- plan -- */

/* radix_to_octree.cu:54-68 */
static int octree_level_of(int n_leaves, const int *plen, int r) {
  const int prefix = (r < n_leaves) ? MORTON_SPATIAL_BITS
                                    : plen[r - n_leaves] - MORTON_PADDING_BITS;
  return prefix / MORTON_DIMS;
}

int orc_octree_plan(int n_leaves, const uint32_t *uniq, const int *parent,
                    const int *plen, int *level, int *count, int *offset,
                    int *n_octree) {
  const int nr = 2 * n_leaves - 1;
  int err = 0;
#define PLAN_FAIL(code)                \
  do {                                 \
    if (err == 0) err = (code);        \
    level[r] = 0;                      \
    count[r] = 0;                      \
    continue;                          \
  } while (0)
  /* radix_to_octree.cu:70-145 */
  for (int r = 0; r < nr; ++r) {
    if (r < n_leaves) {
      if ((uniq[r] & ~MORTON_SPATIAL_MASK) != 0u) PLAN_FAIL(1);
    } else {
      const int sp = plen[r - n_leaves] - MORTON_PADDING_BITS;
      if (sp < 0 || sp >= MORTON_SPATIAL_BITS) PLAN_FAIL(4);
    }
    const int p = parent[r];
    int parent_level = 0;
    if (p != -1) {
      if (p < n_leaves || p >= nr) PLAN_FAIL(2);
      parent_level = octree_level_of(n_leaves, plen, p);
    }
    const int node_level = (r < n_leaves) ? parent_level + 1
                                          : octree_level_of(n_leaves, plen, r);
    if (node_level < 0 || node_level > OCTREE_MAX_LEVEL) PLAN_FAIL(3);
    if (node_level < parent_level) PLAN_FAIL(3);
    level[r] = node_level;
    count[r] = node_level - parent_level;
  }
#undef PLAN_FAIL
  if (err) return err;
  /* radix_to_octree.cu:221-243 */
  long long running = 0;
  for (int r = 0; r < nr; ++r) {
    offset[r] = (int)running;
    running += count[r];
  }
  *n_octree = 1 + (int)running;
  return 0;
}

/* ------------------------------------------------------------ octree -- */

/* octree_builder.cu:49-85 */
static uint32_t prefix_at_level(uint32_t key, int lvl) {
  if (lvl == 0) return 0u;
  const int rem = MORTON_SPATIAL_BITS - lvl * MORTON_DIMS;
  return key & (MORTON_SPATIAL_MASK & (~0u << rem));
}
static int octant_at_level(uint32_t key, int lvl) {
  return (int)((key >> (MORTON_SPATIAL_BITS - lvl * MORTON_DIMS)) & 7u);
}

int orc_octree_build(int n_leaves, const uint32_t *uniq, const int *gfirst,
                     const int *gcount, const int *rparent, const int *rfirst,
                     const int *plan_level, const int *plan_count,
                     const int *plan_offset, int m, int *children, int *parent,
                     int *level, uint32_t *prefix, int *first, int *count) {
  const int nr = 2 * n_leaves - 1;
  if (m <= 0) return ORC_EINVAL;
  /* octree_builder.cu:288-321 */
  for (int i = 0; i < 8 * m; ++i) children[i] = -1;
  for (int i = 0; i < m; ++i) {
    parent[i] = -1;
    level[i] = -1;
    prefix[i] = 0u;
    first[i] = -1;
    count[i] = 0;
  }
  level[0] = 0;
  prefix[0] = 0u;
  int err = 0;
#define OCT_FAIL(code)          \
  do {                          \
    if (err == 0) err = (code); \
    goto next_radix;            \
  } while (0)
  /* octree_builder.cu:87-224 */
  for (int r = 0; r < nr; ++r) {
    const int cnt = plan_count[r];
    const int node_level = plan_level[r];
    if (cnt < 0 || node_level < 0 || node_level > OCTREE_MAX_LEVEL) OCT_FAIL(1);
    if (cnt == 0) {
      if (r < n_leaves) OCT_FAIL(5);
      continue;
    }
    const int parent_level = node_level - cnt;
    if (parent_level < 0) OCT_FAIL(1);
    uint32_t key;
    if (r < n_leaves) {
      key = uniq[r];
    } else {
      const int f = rfirst[r - n_leaves];
      if (f < 0 || f >= n_leaves) OCT_FAIL(7);
      key = uniq[f];
    }
    int parent_node = 0;
    int anc = rparent[r];
    int iters = 0;
    while (anc != -1) {
      if (anc < 0 || anc >= nr) OCT_FAIL(2);
      const int ac = plan_count[anc];
      if (ac > 0) {
        if (plan_level[anc] != parent_level) OCT_FAIL(3);
        parent_node = 1 + plan_offset[anc] + ac - 1;
        break;
      }
      anc = rparent[anc];
      if (++iters > nr) OCT_FAIL(2);
    }
    if (anc == -1 && parent_level != 0) OCT_FAIL(3);
    {
      const int first_node = 1 + plan_offset[r];
      for (int local = 0; local < cnt; ++local) {
        const int node = first_node + local;
        if (node <= 0 || node >= m) OCT_FAIL(6);
        const int lvl = parent_level + local + 1;
        const int par = (local == 0) ? parent_node : node - 1;
        level[node] = lvl;
        prefix[node] = prefix_at_level(key, lvl);
        parent[node] = par;
        const int oct = octant_at_level(key, lvl);
        int *slot = &children[par * 8 + oct];
        if (*slot != -1 && *slot != node) OCT_FAIL(4);
        *slot = node;
      }
      if (r < n_leaves) {
        const int leaf = first_node + cnt - 1;
        const int ll = level[leaf];
        if (ll <= 0 || ll > OCTREE_MAX_LEVEL) OCT_FAIL(5);
        first[leaf] = gfirst[r];
        count[leaf] = gcount[r];
      }
    }
  next_radix:;
  }
#undef OCT_FAIL
  return err;
}

/* ---------------------------------------------------------- geometry -- */

int orc_octree_geometry(int m, const int *level, const uint32_t *prefix,
                        const double box[4], double *cx, double *cy,
                        double *cz, double *half) {
  /* octree_geometry.cu:151-152 */
  if (!isfinite(box[0]) || !isfinite(box[1]) || !isfinite(box[2]) ||
      !isfinite(box[3]) || box[3] <= 0.0)
    return ORC_EINVAL;
  int err = 0;
  for (int node = 0; node < m; ++node) {
    /* octree_geometry.cu:56-102 */
    const int lvl = level[node];
    if (lvl < 0 || lvl > OCTREE_MAX_LEVEL) {
      if (!err) err = 1;
      continue;
    }
    const uint32_t p = prefix[node];
    int valid = (p & ~MORTON_SPATIAL_MASK) == 0u;
    if (valid) {
      if (lvl == 0) {
        valid = p == 0u;
      } else {
        const int rem = MORTON_SPATIAL_BITS - lvl * MORTON_DIMS;
        const uint32_t mask = MORTON_SPATIAL_MASK & (~0u << rem);
        valid = (p & ~mask) == 0u;
      }
    }
    if (!valid) {
      if (!err) err = 2;
      continue;
    }
    double x = box[0], y = box[1], z = box[2], h = box[3] * 0.5;
    for (int d = 1; d <= lvl; ++d) {
      const int oct = (int)((p >> (MORTON_SPATIAL_BITS - d * MORTON_DIMS)) & 7u);
      const double ch = h * 0.5;
      x += (oct & 4) ? ch : -ch;
      y += (oct & 2) ? ch : -ch;
      z += (oct & 1) ? ch : -ch;
      h = ch;
    }
    cx[node] = x;
    cy[node] = y;
    cz[node] = z;
    half[node] = h;
  }
  return err;
}

/* ----------------------------------------------------------- physics -- */

int orc_octree_mass(int m, int n, const int *children, const int *parent,
                    const int *first, const int *count, const uint32_t *idx,
                    const double *pm, const double *px, const double *py,
                    const double *pz, double *mass, double *comx,
                    double *comy, double *comz, int *child_count) {
  (void)parent;
  /* octree_physics.cu:302-310: cleared first */
  for (int i = 0; i < m; ++i) {
    mass[i] = comx[i] = comy[i] = comz[i] = 0.0;
    child_count[i] = 0;
  }
  /* octree_physics.cu:64-93 */
  int err = 0;
  for (int node = 0; node < m; ++node) {
    int c = 0;
    for (int o = 0; o < 8; ++o) {
      const int ch = children[node * 8 + o];
      if (ch == -1) continue;
      if (ch <= 0 || ch >= m) {
        if (!err) err = 1;
        c = -1;
        break;
      }
      ++c;
    }
    if (c < 0) continue;
    child_count[node] = c;
    if (count[node] > 0 && c != 0 && !err) err = 4;
  }
  if (err) return err;
  /* octree_physics.cu:95-154: occupied leaves summed in sorted order */
  for (int node = 0; node < m; ++node) {
    const int cnt = count[node];
    if (cnt <= 0) continue;
    const int f = first[node];
    if (f < 0 || f + cnt > n) return 2;
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int k = 0; k < cnt; ++k) {
      const uint32_t p = idx[f + k];
      if (p >= (uint32_t)n) return 3;
      const double mm = pm[p];
      tm = tm + mm;
      wx = fma(mm, px[p], wx);
      wy = fma(mm, py[p], wy);
      wz = fma(mm, pz[p], wz);
    }
    mass[node] = tm;
    if (tm > 0.0) {
      const double inv = 1.0 / tm;
      comx[node] = wx * inv;
      comy[node] = wy * inv;
      comz[node] = wz * inv;
    }
  }
  /* octree_physics.cu:156-245: the last arriving child sums the children in
   * octant order 0..7, so a parent is combined only after every child.  A
   * reversed breadth-first order from the root gives the same dependency
   * order on the CPU. */
  int *order = (int *)malloc((size_t)m * sizeof(int));
  int head = 0, tail = 0;
  order[tail++] = 0;
  while (head < tail) {
    const int node = order[head++];
    for (int o = 0; o < 8; ++o) {
      const int ch = children[node * 8 + o];
      if (ch > 0 && ch < m && tail < m) order[tail++] = ch;
    }
  }
  for (int k = tail - 1; k >= 0; --k) {
    const int node = order[k];
    if (child_count[node] == 0) continue;
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int o = 0; o < 8; ++o) {
      const int ch = children[node * 8 + o];
      if (ch == -1) continue;
      const double cm = mass[ch];
      tm = tm + cm;
      wx = fma(cm, comx[ch], wx);
      wy = fma(cm, comy[ch], wy);
      wz = fma(cm, comz[ch], wz);
    }
    mass[node] = tm;
    if (tm > 0.0) {
      const double inv = 1.0 / tm;
      comx[node] = wx * inv;
      comy[node] = wy * inv;
      comz[node] = wz * inv;
    } else {
      comx[node] = comy[node] = comz[node] = 0.0;
    }
  }
  free(order);
  return 0;
}

/* --------------------------------------------------------- traversal -- */

typedef struct {
  int m, n;
  const int *children, *parent, *first, *count;
  const double *mass, *comx, *comy, *comz, *cx, *cy, *cz, *half;
} octree_view;

/* barnes_hut.cu:56-80: returns 0 on success, 6 on a singular interaction. */
static int point_mass(double tx, double ty, double tz, double sx, double sy,
                      double sz, double sm, double g, double soft2, double *ax,
                      double *ay, double *az) {
  if (sm == 0.0) return 0;
  const double dx = sx - tx, dy = sy - ty, dz = sz - tz;
  const double d2 = fma(dz, dz, fma(dy, dy, dx * dx)) + soft2;
  if (d2 <= 0.0) return 6;
  const double inv = 1.0 / sqrt(d2);
  const double inv3 = inv * inv * inv;
  const double f = g * sm * inv3;
  *ax = fma(f, dx, *ax);
  *ay = fma(f, dy, *ay);
  *az = fma(f, dz, *az);
  return 0;
}

/* barnes_hut.cu:90-112 */
static int first_child(const octree_view *t, int node, int *err) {
  for (int o = 7; o >= 0; --o) {
    const int c = t->children[node * 8 + o];
    if (c == -1) continue;
    if (c <= 0 || c >= t->m) {
      *err = 1;
      return -2;
    }
    return c;
  }
  *err = 5;
  return -2;
}

/* barnes_hut.cu:115-162 */
static int next_node(const octree_view *t, int node, int *err) {
  while (node != 0) {
    const int p = t->parent[node];
    if (p < 0 || p >= t->m) {
      *err = 4;
      return -2;
    }
    int found = 0;
    for (int o = 7; o >= 0; --o) {
      const int c = t->children[p * 8 + o];
      if (c == -1) continue;
      if (c <= 0 || c >= t->m) {
        *err = 1;
        return -2;
      }
      if (found) return c;
      if (c == node) found = 1;
    }
    if (!found) {
      *err = 4;
      return -2;
    }
    node = p;
  }
  return -1;
}

/* barnes_hut.cu:164-322, one target. Returns the device error code (0 ok). */
static int traverse_one(const octree_view *t, const uint32_t *idx,
                        const double *pm, const double *px, const double *py,
                        const double *pz, int morton_ordered, int sorted_target,
                        double theta, double soft2, double g, double *ax,
                        double *ay, double *az, int64_t *n_inter) {
  const uint32_t target_u = idx[sorted_target];
  if (target_u >= (uint32_t)t->n) return 3;
  const int target = (int)target_u;
  const int ti = morton_ordered ? sorted_target : target;
  const double tx = px[ti], ty = py[ti], tz = pz[ti];
  double rx = 0.0, ry = 0.0, rz = 0.0;
  int64_t inter = 0;
  int err = 0;
  int node = 0;
  while (node >= 0) {
    const double h = t->half[node];
    if (h <= 0.0) return 8;
    const int cnt = t->count[node];
    if (cnt > 0) {
      for (int o = 0; o < 8; ++o)
        if (t->children[node * 8 + o] != -1) return 7;
      const int f = t->first[node];
      if (f < 0 || cnt > t->n || f > t->n - cnt) return 2;
      for (int k = 0; k < cnt; ++k) {
        const int sp = f + k;
        const uint32_t src = idx[sp];
        if (src >= (uint32_t)t->n) return 3;
        if (src == (uint32_t)target) continue;
        const int si = morton_ordered ? sp : (int)src;
        if (point_mass(tx, ty, tz, px[si], py[si], pz[si], pm[si], g, soft2, &rx,
                       &ry, &rz))
          return 6;
        ++inter;
      }
      node = next_node(t, node, &err);
      if (node == -2) return err;
      continue;
    }
    const double nm = t->mass[node];
    if (nm == 0.0) {
      node = next_node(t, node, &err);
      if (node == -2) return err;
      continue;
    }
    const double dx = t->comx[node] - tx;
    const double dy = t->comy[node] - ty;
    const double dz = t->comz[node] - tz;
    const double d2 = fma(dz, dz, fma(dy, dy, dx * dx));
    const double side = 2.0 * h;
    const int contains = fabs(tx - t->cx[node]) <= h &&
                         fabs(ty - t->cy[node]) <= h &&
                         fabs(tz - t->cz[node]) <= h;
    int accept = 0;
    if (!contains && d2 > 0.0 && theta > 0.0) {
      const double ox = t->comx[node] - t->cx[node];
      const double oy = t->comy[node] - t->cy[node];
      const double oz = t->comz[node] - t->cz[node];
      const double o2 = fma(oz, oz, fma(oy, oy, ox * ox));
      const double crit = side / theta + sqrt(o2);
      accept = sqrt(d2) > crit;
    }
    if (accept) {
      if (point_mass(tx, ty, tz, t->comx[node], t->comy[node], t->comz[node], nm,
                     g, soft2, &rx, &ry, &rz))
        return 6;
      ++inter;
      node = next_node(t, node, &err);
      if (node == -2) return err;
      continue;
    }
    node = first_child(t, node, &err);
    if (node == -2) return err;
  }
  ax[target] = rx;
  ay[target] = ry;
  az[target] = rz;
  *n_inter = inter;
  return 0;
}

int orc_bh_accel(int m, int n, const int *children, const int *parent,
                 const int *first, const int *count, const double *mass,
                 const double *comx, const double *comy, const double *comz,
                 const double *cx, const double *cy, const double *cz,
                 const double *half, const uint32_t *idx, const double *pm,
                 const double *px, const double *py, const double *pz,
                 int morton_ordered, double theta, double soft, double g,
                 double *ax, double *ay, double *az, int n_threads,
                 int64_t *interactions) {
  /* barnes_hut.cu:325-391 */
  if (n <= 0 || m <= 0) return ORC_EINVAL;
  if (!isfinite(theta) || theta < 0.0) return ORC_EINVAL;
  if (!isfinite(soft) || soft < 0.0) return ORC_EINVAL;
  if (!isfinite(g) || g <= 0.0) return ORC_EINVAL;
  const double soft2 = soft * soft;
  const octree_view t = {m, n, children, parent, first, count, mass, comx,
                         comy, comz, cx, cy, cz, half};
  int err = 0;
  int64_t total = 0;
  set_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int s = 0; s < n; ++s) {
    int64_t k = 0;
    const int e = traverse_one(&t, idx, pm, px, py, pz, morton_ordered, s,
                               theta, soft2, g, ax, ay, az, &k);
    total += k;
    if (e) {
#pragma omp critical
      if (!err) err = e;
    }
  }
  if (interactions) *interactions = total;
  return err;
}

/* ---------------------------------------------------------- direct sum -- */

void orc_direct_accel(int n, const double *pm, const double *px,
                      const double *py, const double *pz, int n_targets,
                      const int *targets, double g, double soft, double *ax,
                      double *ay, double *az, int n_threads) {
  const double soft2 = soft * soft;
  set_threads(n_threads);
  /* barnes_hut_accuracy_test.cu:101-172 */
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < n_targets; ++k) {
    const int t = targets ? targets[k] : k;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    for (int s = 0; s < n; ++s) {
      if (s == t) continue;
      const double dx = px[s] - px[t], dy = py[s] - py[t], dz = pz[s] - pz[t];
      const double d2 = fma(dz, dz, fma(dy, dy, dx * dx)) + soft2;
      const double inv = 1.0 / sqrt(d2);
      const double f = g * pm[s] * (inv * inv * inv);
      rx = fma(f, dx, rx);
      ry = fma(f, dy, ry);
      rz = fma(f, dz, rz);
    }
    ax[k] = rx;
    ay[k] = ry;
    az[k] = rz;
  }
}

/* --------------------------------------------------------- integrator -- */

void orc_kick_drift(size_t n, double *x, double *y, double *z, double *vx,
                    double *vy, double *vz, const double *ax, const double *ay,
                    const double *az, double dt) {
  const double hdt = 0.5 * dt; /* integrator.cu:58 */
  for (size_t i = 0; i < n; ++i) {
    vx[i] = fma(hdt, ax[i], vx[i]);
    vy[i] = fma(hdt, ay[i], vy[i]);
    vz[i] = fma(hdt, az[i], vz[i]);
    x[i] = fma(dt, vx[i], x[i]);
    y[i] = fma(dt, vy[i], y[i]);
    z[i] = fma(dt, vz[i], z[i]);
  }
}

void orc_kick(size_t n, double *vx, double *vy, double *vz, const double *ax,
              const double *ay, const double *az, double dt) {
  const double hdt = 0.5 * dt; /* integrator.cu:93 */
  for (size_t i = 0; i < n; ++i) {
    vx[i] = fma(hdt, ax[i], vx[i]);
    vy[i] = fma(hdt, ay[i], vy[i]);
    vz[i] = fma(hdt, az[i], vz[i]);
  }
}

/* ----------------------------------------------------------- pipeline -- */

int orc_pipeline(size_t n, const double *m, const double *x, const double *y,
                 const double *z, double theta, double soft, double g,
                 int n_threads, orc_pipeline_out *o) {
  if (n == 0 || n > 0x7fffffff) return ORC_EINVAL;
  int st = orc_bbox(n, x, y, z, o->box);
  if (st) return st;
  st = orc_morton(n, x, y, z, o->box, o->keys, o->idx);
  if (st) return st;
  const int nn = (int)n;
  const int gcnt = orc_leaf_groups(nn, o->keys, o->uniq, o->gfirst, o->gcount);
  if (gcnt <= 0) return ORC_EINVAL;
  o->n_groups = gcnt;
  st = orc_radix_tree(gcnt, o->uniq, o->left, o->right, o->rfirst, o->rlast,
                      o->plen, o->rparent);
  if (st) return st;
  int mo = 0;
  st = orc_octree_plan(gcnt, o->uniq, o->rparent, o->plen, o->plan_level,
                       o->plan_count, o->plan_offset, &mo);
  if (st) return 100 + st;
  if (mo > o->m_capacity) return ORC_ECAP;
  o->n_octree = mo;
  st = orc_octree_build(gcnt, o->uniq, o->gfirst, o->gcount, o->rparent,
                        o->rfirst, o->plan_level, o->plan_count, o->plan_offset,
                        mo, o->children, o->oparent, o->olevel, o->oprefix,
                        o->ofirst, o->ocount);
  if (st) return 200 + st;
  st = orc_octree_geometry(mo, o->olevel, o->oprefix, o->box, o->cx, o->cy,
                           o->cz, o->half);
  if (st) return 300 + st;
  st = orc_octree_mass(mo, nn, o->children, o->oparent, o->ofirst, o->ocount,
                       o->idx, m, x, y, z, o->mass, o->comx, o->comy, o->comz,
                       o->child_count);
  if (st) return 400 + st;
  if (!o->ax) return 0;
  /* simulation.cu:34-58: gather into Morton order, then traverse with
   * BarnesHutParticleOrder::morton (simulation.cpp:182-198). */
  double *gm = (double *)malloc(4 * n * sizeof(double));
  double *gx = gm + n, *gy = gm + 2 * n, *gz = gm + 3 * n;
  for (size_t s = 0; s < n; ++s) {
    const uint32_t p = o->idx[s];
    gm[s] = m[p];
    gx[s] = x[p];
    gy[s] = y[p];
    gz[s] = z[p];
  }
  st = orc_bh_accel(mo, nn, o->children, o->oparent, o->ofirst, o->ocount,
                    o->mass, o->comx, o->comy, o->comz, o->cx, o->cy, o->cz,
                    o->half, o->idx, gm, gx, gy, gz, 1, theta, soft, g, o->ax,
                    o->ay, o->az, n_threads, &o->interactions);
  free(gm);
  if (st > 0) return 500 + st;
  return st;
}

typedef struct {
  orc_pipeline_out o;
  void *block;
} pipeline_buffers;

static int alloc_pipeline(size_t n, pipeline_buffers *b) {
  const size_t mcap = 10 * n + 1;
  const size_t ints = 2 * n + 2 * n + 5 * n + 2 * n + 3 * (2 * n) + 8 * mcap +
                      6 * mcap;
  const size_t dbls = 8 * mcap;
  b->block = malloc(ints * 4 + dbls * 8 + 64);
  if (!b->block) return ORC_ECAP;
  double *d = (double *)b->block;
  orc_pipeline_out *o = &b->o;
  o->cx = d; d += mcap;
  o->cy = d; d += mcap;
  o->cz = d; d += mcap;
  o->half = d; d += mcap;
  o->mass = d; d += mcap;
  o->comx = d; d += mcap;
  o->comy = d; d += mcap;
  o->comz = d; d += mcap;
  int *p = (int *)d;
  o->keys = (uint32_t *)p; p += n;
  o->idx = (uint32_t *)p; p += n;
  o->uniq = (uint32_t *)p; p += n;
  o->gfirst = p; p += n;
  o->gcount = p; p += n;
  o->left = p; p += n;
  o->right = p; p += n;
  o->rfirst = p; p += n;
  o->rlast = p; p += n;
  o->plen = p; p += n;
  o->rparent = p; p += 2 * n;
  o->plan_level = p; p += 2 * n;
  o->plan_count = p; p += 2 * n;
  o->plan_offset = p; p += 2 * n;
  o->children = p; p += 8 * mcap;
  o->oparent = p; p += mcap;
  o->olevel = p; p += mcap;
  o->oprefix = (uint32_t *)p; p += mcap;
  o->ofirst = p; p += mcap;
  o->ocount = p; p += mcap;
  o->child_count = p; p += mcap;
  o->m_capacity = (int)mcap;
  return 0;
}

int orc_simulate(size_t n, const double *m, double *x, double *y, double *z,
                 double *vx, double *vy, double *vz, double *ax, double *ay,
                 double *az, double dt, double theta, double soft, double g,
                 int steps, int n_threads) {
  /* simulation.cpp:21-33 */
  if (!isfinite(dt) || dt <= 0.0) return ORC_EINVAL;
  if (!isfinite(theta) || theta < 0.0) return ORC_EINVAL;
  if (!isfinite(soft) || soft < 0.0) return ORC_EINVAL;
  pipeline_buffers b;
  if (alloc_pipeline(n, &b)) return ORC_ECAP;
  b.o.ax = ax;
  b.o.ay = ay;
  b.o.az = az;
  /* initialize(): rebuild, force into the current acceleration */
  int st = orc_pipeline(n, m, x, y, z, theta, soft, g, n_threads, &b.o);
  for (int s = 0; s < steps && st == 0; ++s) {
    /* step(): KD, rebuild + force (next a), K, swap */
    orc_kick_drift(n, x, y, z, vx, vy, vz, ax, ay, az, dt);
    st = orc_pipeline(n, m, x, y, z, theta, soft, g, n_threads, &b.o);
    if (st) break;
    orc_kick(n, vx, vy, vz, ax, ay, az, dt);
  }
  free(b.block);
  return st;
}

/* ------------------------------------------------------- frame capture */

static unsigned char *put_le(unsigned char *p, uint64_t v, int bytes) {
  for (int b = 0; b < bytes; ++b) p[b] = (unsigned char)((v >> (8 * b)) & 0xffu);
  return p + bytes;
}

static unsigned char *put_f64(unsigned char *p, double v) {
  uint64_t bits;
  memcpy(&bits, &v, sizeof(bits));
  return put_le(p, bits, 8);
}

/* device_capture.cu:118-126 as nvcc compiles it (the product plus one half
 * is a fused multiply-add). */
static uint16_t frame_quantize(double p, double lo, double hi) {
  if (hi == lo) return 0;
  double u = (p - lo) / (hi - lo);
  u = fmin(1.0, fmax(0.0, u));
  return (uint16_t)fma(u, 65535.0, 0.5);
}

long long orc_frame_capture(size_t n, const double *x, const double *y, const double *z,
                            const uint8_t *type, size_t max_particles, uint64_t sequence,
                            uint64_t step, double time, unsigned char *out, size_t cap) {
  if (n == 0 || !x || !y || !z || !out || !isfinite(time) || time < 0.0) return -1;
  const size_t s = (max_particles == 0 || max_particles > n) ? n : max_particles;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  const double *c[3] = {x, y, z};
  for (size_t i = 0; i < s; ++i) {
    const size_t src = (size_t)(((unsigned long long)i * n) / s);
    const double v[3] = {x[src], y[src], z[src]};
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) return -2;
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], v[a]);
      hi[a] = fmax(hi[a], v[a]);
    }
  }
  for (int a = 0; a < 3; ++a)
    if (!isfinite(lo[a]) || !isfinite(hi[a]) || lo[a] > hi[a] || !isfinite(hi[a] - lo[a])) return -4;
  if (type)
    for (size_t i = 0; i < s; ++i)
      if (type[(size_t)(((unsigned long long)i * n) / s)] > 4) return -3;
  const size_t header = type ? 128 : 120;
  const size_t type_bytes = type ? s : 0;
  const size_t total = header + 6 * s + type_bytes;
  if (cap < total) return -5;
  unsigned char *p = out;
  memcpy(p, "NBSNAP01", 8);
  p += 8;
  p = put_le(p, type ? 3u : 2u, 4);
  p = put_le(p, header, 4);
  p = put_le(p, sequence, 8);
  p = put_le(p, step, 8);
  p = put_f64(p, time);
  p = put_le(p, n, 8);
  p = put_le(p, s, 8);
  p = put_le(p, 2, 4);
  p = put_le(p, 3, 4);
  p = put_le(p, 6 * s + type_bytes, 8);
  for (int a = 0; a < 3; ++a) p = put_f64(p, lo[a]);
  for (int a = 0; a < 3; ++a) p = put_f64(p, hi[a]);
  if (type) p = put_le(p, type_bytes, 8);
  for (size_t i = 0; i < s; ++i) {
    const size_t src = (size_t)(((unsigned long long)i * n) / s);
    for (int a = 0; a < 3; ++a) p = put_le(p, frame_quantize(c[a][src], lo[a], hi[a]), 2);
  }
  if (type)
    for (size_t i = 0; i < s; ++i) *p++ = type[(size_t)(((unsigned long long)i * n) / s)];
  return (long long)total;
}
