// build.cu -- the spatial rebuild of one Barnes-Hut step on sm_100a.
//
// Stage map (reference file:line each kernel replaces, paths relative to the
// sytrams/AMSC-Nbody project root):
//   kd_bbox_kernel        integrator.cu:51-83 (KD) fused with
//                         globalbounding.cu:94-144 (Bbox)
//   encode_kernel         morton.cu:98-139,160-219 (normalise/quantise/interleave)
//                         + the digit histograms of the radix sort
//   onesweep_kernel       morton.cu:221-224 (stable_sort_by_key), in-house
//                         LSD radix sort with decoupled look-back
//   groups_kernel         morton_leaf_groups.cu:58-103 (RLE + scan) fused
//                         with simulation.cu:34-58 (Morton-order gather)
//   karras_kernel         tree_builder.cu:9-113
//   plan_kernel           radix_to_octree.cu:70-145 + its exclusive scan
//   octree_clear_kernel   octree_builder.cu:288-321 (initialisation)
//   materialize_kernel    octree_builder.cu:87-224
//   node_init_kernel      octree_geometry.cu:56-102 + octree_physics.cu:64-154
//   level_bin_kernel      octree nodes binned by level
//   propagate_level_kernel octree_physics.cu:156-245 (+ subtree sizes), one
//                         level per launch, deepest first
//   ends_hist_kernel, ends_scan_kernel, preorder_kernel
//                         preorder indices in closed form
//   layout_kernel         traversal records in depth-first preorder
//
// No kernel synchronises with the host: data-dependent sizes (G, M) live in
// device memory and every later kernel bounds its grid-stride loop by them.
#include "nbb_internal.cuh"

#include <cfloat>
#include <climits>
#include <cmath>

namespace nbb {

namespace {

constexpr int kBlock = 256;

inline int grid_for(const Workspace &ws, int per_sm = 8) {
  return ws.num_sms > 0 ? ws.num_sms * per_sm : 1184;
}

// Blocks for one octree level: enough for the most nodes a level can hold
// (min(8^L, n)), at most grid_for().
inline int level_grid(const Workspace &ws, int level) {
  long long width = 1;
  for (int l = 0; l < level && width < (1ll << 40); ++l) width *= 8;
  const long long nodes = width < ws.n ? width : ws.n;
  const long long blocks = (nodes + kBlock - 1) / kBlock;
  const int cap = grid_for(ws, 8);
  return blocks < 1 ? 1 : (blocks > cap ? cap : (int)blocks);
}

// ------------------------------------------------------------- reset ----

__global__ void reset_sys_kernel(unsigned long long *bb, int n_systems) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 6 * n_systems; k += gridDim.x * blockDim.x)
    bb[k] = (k % 6 < 3) ? ~0ull : 0ull;
}

__global__ void reset_scalars_kernel(DevScalars *sc) {
  if (threadIdx.x == 0) {
    for (int a = 0; a < 3; ++a) {
      sc->bb_min[a] = ~0ull;
      sc->bb_max[a] = 0ull;
    }
    sc->nonfinite = 0;
    sc->n_groups = 0;
    sc->n_nodes = 0;
    sc->ticket_bbox = 0;
    sc->ticket_encode = 0;
    for (int k = 0; k < kTileCounters; ++k) sc->tile_counter[k] = 0;
    sc->work_counter = 0;
    sc->n_tgroups = 0;
    sc->stack_overflow = 0;
    sc->interactions = 0;
    sc->mac_tests = 0;
    for (int l = 0; l < kMaxLevels; ++l) sc->level_count[l] = 0;
    for (int l = 0; l < kMaxLevels + 2; ++l) sc->level_base[l] = 0;
  }
}

// --------------------------------------------------------- KD + bbox ----

template <typename T>
__device__ __forceinline__ T warp_reduce_min(T v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_reduce_max(T v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Box of one system from its encoded extrema (globalbounding.cu:122-136):
// centre = (min + max) * 0.5, side = 1.1 * longest extent, 1 when that is 0.
__device__ void finish_box(const unsigned long long *mn, const unsigned long long *mx, double *box) {
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = order_value(mn[a]);
    hi[a] = order_value(mx[a]);
  }
  for (int a = 0; a < 3; ++a) box[a] = __dmul_rn(__dadd_rn(lo[a], hi[a]), 0.5);
  double ext = __dsub_rn(hi[0], lo[0]);
  const double ey = __dsub_rn(hi[1], lo[1]);
  const double ez = __dsub_rn(hi[2], lo[2]);
  if (ey > ext) ext = ey;
  if (ez > ext) ext = ez;
  double side = __dmul_rn(1.1, ext);
  if (side == 0.0) side = 1.0;
  box[3] = side;
}

// One pass over the state: optional first half kick + drift
// (integrator.cu:51-83), then the extrema of the new positions and a
// non-finite flag (globalbounding.cu:17-56), per system.  The last block to
// finish forms every system's box.  A single system reduces through shared
// memory with one set of atomics per block; an ensemble (systems stored
// contiguously) reduces per warp when the warp's particles share a system
// and per particle otherwise.
__global__ void __launch_bounds__(kBlock) kd_bbox_kernel(Workspace ws, double dt,
                                                         int do_kd) {
  __shared__ double s_lo[3][kBlock / 32], s_hi[3][kBlock / 32];
  __shared__ int s_nf[kBlock / 32];
  __shared__ bool s_last;
  const int n = ws.n;
  const bool multi = ws.n_systems > 1;
  const double hdt = 0.5 * dt;
  double lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY;
  double hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
  int nf = 0;
  DevScalars *sc = ws.sc;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const bool in = i < n;
    double px = 0.0, py = 0.0, pz = 0.0;
    if (in) {
      px = ws.x[i];
      py = ws.y[i];
      pz = ws.z[i];
      if (do_kd) {
        const double vx = __fma_rn(hdt, ws.ax[i], ws.vx[i]);
        const double vy = __fma_rn(hdt, ws.ay[i], ws.vy[i]);
        const double vz = __fma_rn(hdt, ws.az[i], ws.vz[i]);
        ws.vx[i] = vx;
        ws.vy[i] = vy;
        ws.vz[i] = vz;
        px = __fma_rn(dt, vx, px);
        py = __fma_rn(dt, vy, py);
        pz = __fma_rn(dt, vz, pz);
        ws.x[i] = px;
        ws.y[i] = py;
        ws.z[i] = pz;
      }
      // one 32-byte record per particle for the Morton-order gather
      if (ws.pos4) ws.pos4[i] = make_double4(px, py, pz, 0.0);
      nf |= !(isfinite(px) && isfinite(py) && isfinite(pz));
    }
    if (!multi) {
      if (in) {
        lo0 = fmin(lo0, px); hi0 = fmax(hi0, px);
        lo1 = fmin(lo1, py); hi1 = fmax(hi1, py);
        lo2 = fmin(lo2, pz); hi2 = fmax(hi2, pz);
      }
      continue;
    }
    // ensemble: per-system extrema
    const int sys = in ? ws.sys_of[i] : -1;
    const int sys0 = __shfl_sync(0xffffffffu, sys, 0);
    const bool uniform = __all_sync(0xffffffffu, !in || sys == sys0) && sys0 >= 0;
    double l0 = in ? px : INFINITY, l1 = in ? py : INFINITY, l2 = in ? pz : INFINITY;
    double h0 = in ? px : -INFINITY, h1 = in ? py : -INFINITY, h2 = in ? pz : -INFINITY;
    if (uniform) {
      l0 = warp_reduce_min(l0); l1 = warp_reduce_min(l1); l2 = warp_reduce_min(l2);
      h0 = warp_reduce_max(h0); h1 = warp_reduce_max(h1); h2 = warp_reduce_max(h2);
    }
    if (in && (!uniform || lane == 0)) {
      unsigned long long *b = ws.sys_bb + 6 * (size_t)sys;
      atomicMin(b + 0, order_bits(l0)); atomicMax(b + 3, order_bits(h0));
      atomicMin(b + 1, order_bits(l1)); atomicMax(b + 4, order_bits(h1));
      atomicMin(b + 2, order_bits(l2)); atomicMax(b + 5, order_bits(h2));
    }
  }
  nf = __any_sync(0xffffffffu, nf);
  const int warp = threadIdx.x >> 5;
  if (!multi) {
    lo0 = warp_reduce_min(lo0); lo1 = warp_reduce_min(lo1); lo2 = warp_reduce_min(lo2);
    hi0 = warp_reduce_max(hi0); hi1 = warp_reduce_max(hi1); hi2 = warp_reduce_max(hi2);
    if (lane == 0) {
      s_lo[0][warp] = lo0; s_lo[1][warp] = lo1; s_lo[2][warp] = lo2;
      s_hi[0][warp] = hi0; s_hi[1][warp] = hi1; s_hi[2][warp] = hi2;
    }
  }
  if (lane == 0) s_nf[warp] = nf;
  __syncthreads();
  if (threadIdx.x == 0) {
    int anynf = 0;
    if (!multi) {
      for (int a = 0; a < 3; ++a) {
        double lo = INFINITY, hi = -INFINITY;
        for (int w = 0; w < kBlock / 32; ++w) {
          lo = fmin(lo, s_lo[a][w]);
          hi = fmax(hi, s_hi[a][w]);
        }
        if (lo <= hi) {
          atomicMin(&ws.sys_bb[a], order_bits(lo));
          atomicMax(&ws.sys_bb[3 + a], order_bits(hi));
        }
      }
    }
    for (int w = 0; w < kBlock / 32; ++w) anynf |= s_nf[w];
    if (anynf) atomicOr(&sc->nonfinite, 1);
    __threadfence();
    const unsigned t = atomicAdd(&sc->ticket_bbox, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    if (threadIdx.x == 0 && atomicAdd(&sc->nonfinite, 0)) record_error(sc, kStageBbox, 1);
    for (int sys = threadIdx.x; sys < ws.n_systems; sys += blockDim.x) {
      unsigned long long mn[3], mx[3];
      for (int a = 0; a < 3; ++a) {
        mn[a] = atomicAdd(&ws.sys_bb[6 * (size_t)sys + a], 0ull);
        mx[a] = atomicAdd(&ws.sys_bb[6 * (size_t)sys + 3 + a], 0ull);
      }
      finish_box(mn, mx, ws.sys_box + 4 * (size_t)sys);
      if (sys == 0)
        for (int a = 0; a < 4; ++a) sc->box[a] = ws.sys_box[a];
    }
  }
}

// ---------------------------------------------------- Morton encode ----

// morton.cu:119-128
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  uint32_t x = v & 0x000003FFu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// morton.cu:98-117 with explicitly rounded operations: the normalised
// coordinate is a true division, then scaled by the 1024-cell grid, clamped
// to [0, 1023] and truncated.
__device__ __forceinline__ uint32_t quantise(double a, double lower, double side) {
  const double normalised = __ddiv_rn(__dsub_rn(a, lower), side);
  const double scaled = __dmul_rn(normalised, 1024.0);
  const double clamped = fmin(fmax(scaled, 0.0), 1023.0);
  return (uint32_t)clamped;
}

// Keys and packed (key << pack_shift | index) pairs, plus the digit
// histograms of the sort passes; the last block turns the histograms into
// exclusive digit offsets.  An ensemble's key carries the system id above the
// 30 Morton bits, each system quantised against its own box.
__global__ void __launch_bounds__(kBlock) encode_kernel(Workspace ws) {
  __shared__ uint32_t hist[kMaxSortPasses][256];
  __shared__ bool s_last;
  const int passes = ws.sort_passes;
  for (int k = threadIdx.x; k < kMaxSortPasses * 256; k += blockDim.x) (&hist[0][0])[k] = 0;
  __syncthreads();
  DevScalars *sc = ws.sc;
  const int n = ws.n;
  const bool multi = ws.n_systems > 1;
  if (blockIdx.x == 0) {
    // morton.cu:167-170, every system's box
    for (int sys = threadIdx.x; sys < ws.n_systems; sys += blockDim.x) {
      const double *b = ws.sys_box + 4 * (size_t)sys;
      if (!isfinite(b[0]) || !isfinite(b[1]) || !isfinite(b[2]) || !isfinite(b[3]) || b[3] <= 0.0)
        record_error(sc, kStageBbox, 2);
    }
  }
  int cur = -1;
  double lx = 0.0, ly = 0.0, lz = 0.0, side = 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int sys = multi ? ws.sys_of[i] : 0;
    if (sys != cur) {
      const double *b = ws.sys_box + 4 * (size_t)sys;
      side = b[3];
      const double half_side = __dmul_rn(side, 0.5);  // side / 2.0, exact
      lx = __dsub_rn(b[0], half_side);
      ly = __dsub_rn(b[1], half_side);
      lz = __dsub_rn(b[2], half_side);
      cur = sys;
    }
    const uint32_t qx = quantise(ws.x[i], lx, side);
    const uint32_t qy = quantise(ws.y[i], ly, side);
    const uint32_t qz = quantise(ws.z[i], lz, side);
    const unsigned long long key = ((unsigned long long)sys << kSpatialBits) |
                                   ((expand_bits(qx) << 2) | (expand_bits(qy) << 1) | expand_bits(qz));
    ws.pairs_a[i] = (key << ws.pack_shift) | (unsigned long long)i;
    for (int p = 0; p < passes; ++p) atomicAdd(&hist[p][(key >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < passes * 256; k += blockDim.x) {
    const uint32_t c = (&hist[0][0])[k];
    if (c) atomicAdd(&ws.digit_hist[k], c);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&sc->ticket_encode, 1u) == gridDim.x - 1);
  __syncthreads();
  if (s_last) {
    // digit counts -> exclusive digit offsets, one thread per digit (the
    // counts were added at L2 by every block before its ticket)
    __threadfence();
    static_assert(kBlock == 256, "one thread per digit");
    __shared__ uint32_t warp_tot[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int p = 0; p < passes; ++p) {
      uint32_t *h = ws.digit_hist + p * 256;
      const uint32_t c = __ldcg(h + threadIdx.x);
      uint32_t inc = c;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
      }
      if (lane == 31) warp_tot[warp] = inc;
      __syncthreads();
      uint32_t base = 0;
      for (int w = 0; w < warp; ++w) base += warp_tot[w];
      h[threadIdx.x] = base + inc - c;
      __syncthreads();
    }
  }
}

// ------------------------------------------------------ onesweep pass ----

constexpr uint32_t kDigitFlagA = 1u << 30;  // tile aggregate published
constexpr uint32_t kDigitFlagP = 2u << 30;  // inclusive prefix published
constexpr uint32_t kDigitMask = (1u << 30) - 1u;

// One stable LSD pass over 8 key bits.  A tile's items are ranked warp by
// warp and round by round in input order (the lanes holding the same digit in
// a round are found with one ballot per digit bit, a cost that does not grow
// with the number of distinct digits), so equal digits keep their input
// order: the result is the stable order of thrust::stable_sort_by_key.  Tile
// prefixes per digit come from a decoupled look-back over the tiles launched
// before it (tile ids are taken from an atomic counter, so every predecessor
// is already running), reading 16 predecessors' status words at once.  The
// ranked tile is first placed in shared memory in digit order, then written
// out by consecutive threads: a digit's items of one tile land at consecutive
// addresses, so the stores go out as runs instead of one scattered 8-byte
// store per item.
__global__ void __launch_bounds__(kSortThreads)
    onesweep_kernel(const unsigned long long *__restrict__ in,
                    unsigned long long *__restrict__ out, int n, int pass, int shift,
                    const uint32_t *__restrict__ digit_offsets,
                    uint32_t *status, DevScalars *sc) {
  constexpr int kWarps = kSortThreads / 32;
  static_assert(kSortThreads == 256, "one thread per digit");
  __shared__ uint32_t whist[kWarps][256];
  __shared__ uint32_t tile_excl[256];   // digit's first slot in the staged tile
  __shared__ uint32_t digit_base[256];  // digit's first output position of this tile
  __shared__ uint32_t warp_tot[kWarps];
  __shared__ unsigned long long stage[kSortTile];
  __shared__ int s_tile;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_tile = (int)atomicAdd(&sc->tile_counter[pass], 1u);
  for (int k = tid; k < kWarps * 256; k += kSortThreads) (&whist[0][0])[k] = 0;
  __syncthreads();
  const int tile = s_tile;
  const int start = tile * kSortTile + warp * (32 * kSortItems);
  unsigned long long key[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int i = start + it * 32 + lane;
    key[it] = (i < n) ? in[i] : ~0ull;
  }
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int i = start + it * 32 + lane;
    const bool valid = i < n;
    const uint32_t dig = (uint32_t)(key[it] >> shift) & 255u;
    // lanes with the same digit (bit 8 marks the items past the end)
    const uint32_t code = valid ? dig : 256u;
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; ++b) {
      const bool bit = (code >> b) & 1u;
      const unsigned on = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? on : ~on;
    }
    uint32_t base = 0;
    if (valid) base = whist[warp][dig];
    __syncwarp();
    if (valid) {
      rank[it] = base + __popc(peers & lt);
      if ((peers & lt) == 0) whist[warp][dig] = base + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // digit tid: offsets of the warps' runs, the tile's count (published at
  // once), its place in the staged tile (exclusive scan over digits)
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const uint32_t c = whist[w][tid];
    whist[w][tid] = run;
    run += c;
  }
  uint32_t *my = status + (size_t)tile * 256 + tid;
  st_release_u32(my, (tile == 0 ? kDigitFlagP : kDigitFlagA) | run);
  {
    uint32_t inc = run;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    tile_excl[tid] = wbase + inc - run;
  }
  __syncthreads();
  // the tile in digit order in shared memory, while the predecessors publish
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const int i = start + it * 32 + lane;
    if (i < n) {
      const uint32_t dig = (uint32_t)(key[it] >> shift) & 255u;
      const uint32_t local = tile_excl[dig] + whist[warp][dig] + rank[it];
      if (local < (uint32_t)kSortTile) stage[local] = key[it];
    }
  }
  {
    // digit tid: the tile's output base from the look-back
    uint32_t prefix = 0;
    if (tile > 0) {
      // predecessors j, j-1, ..., read kLookWindow at a time: aggregates are
      // added until an inclusive prefix (added too); an unpublished word
      // ends the window and is read again
      constexpr int kLookWindow = 32;
      int j = tile - 1;
      int spins = 0;
      bool done = false;
      while (!done) {
        uint32_t st[kLookWindow];
#pragma unroll
        for (int w = 0; w < kLookWindow; ++w)
          st[w] = (j - w >= 0) ? ld_relaxed_u32(status + (size_t)(j - w) * 256 + tid) : kDigitFlagP;
        int used = 0;
        bool stop = false;
#pragma unroll
        for (int w = 0; w < kLookWindow; ++w) {
          if (stop) continue;
          const uint32_t flag = st[w] & ~kDigitMask;
          if (flag == 0u) {
            stop = true;
          } else {
            prefix += st[w] & kDigitMask;
            ++used;
            if (flag == kDigitFlagP) stop = done = true;
          }
        }
        j -= used;
        if (!done && used == 0 && ++spins > kSpinLimit) {
          record_error(sc, kStageSort, kCodeTimeout);
          break;
        }
      }
      st_release_u32(my, kDigitFlagP | (prefix + run));
    }
    digit_base[tid] = digit_offsets[pass * 256 + tid] + prefix;
  }
  __syncthreads();
  const int count = min(kSortTile, n - tile * kSortTile);
  for (int j = tid; j < count; j += kSortThreads) {
    const unsigned long long k = stage[j];
    const uint32_t dig = (uint32_t)(k >> shift) & 255u;
    const uint32_t pos = digit_base[dig] + ((uint32_t)j - tile_excl[dig]);
    if (pos < (uint32_t)n) {
      out[pos] = k;
    } else {
      record_error(sc, kStageSort, 1);
    }
  }
}

// ------------------------------------------- single-pass scan helpers ----

constexpr unsigned long long kScanFlagA = 1ull << 62;
constexpr unsigned long long kScanFlagP = 2ull << 62;
constexpr unsigned long long kScanMask = (1ull << 62) - 1ull;

// Decoupled look-back by one full warp: publishes this tile's aggregate,
// accumulates predecessors until one with an inclusive prefix, publishes the
// inclusive prefix and returns the exclusive one.
__device__ unsigned long long warp_lookback(unsigned long long *status, int tile,
                                            unsigned long long aggregate,
                                            DevScalars *sc, int stage) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_release_u64(status, kScanFlagP | aggregate);
    return 0ull;
  }
  if (lane == 0) st_release_u64(status + tile, kScanFlagA | aggregate);
  unsigned long long excl = 0;
  int j = tile - 1;
  while (true) {
    const int idx = j - lane;
    unsigned long long s = kScanFlagP;
    if (idx >= 0) {
      s = ld_acquire_u64(status + idx);
      int spins = 0;
      while ((s >> 62) == 0ull) {
        if (++spins > kSpinLimit) {
          record_error(sc, stage, kCodeTimeout);
          s = kScanFlagP;
          break;
        }
        s = ld_acquire_u64(status + idx);
      }
    }
    const unsigned pmask = __ballot_sync(0xffffffffu, (s >> 62) == 2ull);
    unsigned long long v = s & kScanMask;
    if (pmask) {
      const int stop = __ffs(pmask) - 1;
      if (lane > stop) v = 0;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      excl += v;
      break;
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    j -= 32;
  }
  if (lane == 0) st_release_u64(status + tile, kScanFlagP | (excl + aggregate));
  return excl;
}

// Block-wide exclusive scan of ITEMS rows of 0/1 or small int values laid
// out row-major (element (k, tid) precedes (k, tid+1) and (k+1, 0)).  Each
// thread passes its values; returns per-row exclusive offsets in `excl` and
// the block total.  `row_warp` is shared scratch of ITEMS * warps ints.
template <int ITEMS, int THREADS>
__device__ unsigned long long block_scan_rows(const int (&val)[ITEMS], int (&excl)[ITEMS],
                                              unsigned long long *row_warp,
                                              unsigned long long *s_total) {
  constexpr int kWarps = THREADS / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    int v = val[k];
    // warp inclusive scan
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    excl[k] = v - val[k];
    if (lane == 31) row_warp[k * kWarps + warp] = (unsigned long long)v;
  }
  __syncthreads();
  if (warp == 0) {
    constexpr int kCount = ITEMS * kWarps;
    static_assert(kCount % 32 == 0, "scan rows must fill whole warps");
    unsigned long long carry = 0;
    for (int base = 0; base < kCount; base += 32) {
      unsigned long long v = row_warp[base + lane];
      unsigned long long inc = v;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      row_warp[base + lane] = carry + inc - v;
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) *s_total = carry;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) excl[k] += (int)row_warp[k * kWarps + warp];
  return *s_total;
}

// ------------------------------------------------------------ groups ----

// Run-length encoding of the sorted keys as a scan of "key differs from its
// predecessor" flags: a group starts where the flag is set; its id is the
// number of flags before it.  Also splits the packed pairs into the
// reference's key / index arrays and gathers {x, y, z, m} into Morton order.
__global__ void __launch_bounds__(kScanThreads) groups_kernel(Workspace ws,
                                                              const unsigned long long *pairs,
                                                              int gather) {
  __shared__ unsigned long long row_warp[kScanItems * (kScanThreads / 32)];
  __shared__ unsigned long long s_total, s_prefix;
  __shared__ int s_tile;
  DevScalars *sc = ws.sc;
  const int n = ws.n;
  const int shift = ws.pack_shift;
  const unsigned long long imask = (1ull << shift) - 1ull;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(&sc->tile_counter[kTileGroups], 1u);
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kScanTile;
  if (base >= n) return;
  int flag[kScanItems], excl[kScanItems];
  unsigned long long key[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    flag[k] = 0;
    key[k] = 0;
    if (i < n) {
      key[k] = pairs[i] >> shift;
      flag[k] = (i == 0) || (key[k] != (pairs[i - 1] >> shift));
    }
  }
  const unsigned long long total = block_scan_rows<kScanItems, kScanThreads>(flag, excl, row_warp, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long p = warp_lookback(ws.scan_status, tile, total, sc, kStageGroups);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  const int prefix = (int)s_prefix;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    if (i >= n) continue;
    const int g = prefix + excl[k] + flag[k] - 1;
    const unsigned long long pr = pairs[i];
    const unsigned long long id = pr & imask;
    if (g < 0 || g >= n || id >= (unsigned long long)n) {
      record_error(sc, kStageGroups, 1);
      continue;
    }
    if (flag[k]) {
      ws.ukey[g] = key[k];
      ws.uniq[g] = (uint32_t)key[k];
      ws.gfirst[g] = i;
    }
    const bool last = (i == n - 1) || ((pairs[i + 1] >> shift) != key[k]);
    if (last) ws.glast[g] = i;
    ws.keys[i] = (uint32_t)key[k];
    ws.idx[i] = (uint32_t)id;
    ws.psys[i] = (int)(key[k] >> kSpatialBits);
    if (gather) ws.pm4[i] = make_double4(ws.x[id], ws.y[id], ws.z[id], ws.m[id]);
  }
  if (base + kScanTile >= n && threadIdx.x == 0) sc->n_groups = prefix + (int)total;
}

// ------------------------------------------------------------ Karras ----

// tree_builder.cu:9-24, for 32-bit keys (the reference's) and for 64-bit
// keys; the 64-bit frame is the 32-bit one plus 32 for keys below 2^32.
template <typename K>
__device__ __forceinline__ int lcp(const K *keys, int i, int j, int n) {
  if (j < 0 || j >= n) return -1;
  if (i == j) return 8 * (int)sizeof(K) + 32;
  const K a = keys[i], b = keys[j];
  if (a != b) return (sizeof(K) == 8) ? __clzll((long long)(a ^ b)) : __clz((unsigned)(a ^ b));
  return 8 * (int)sizeof(K) + __clz((uint32_t)(i ^ j));
}

// tree_builder.cu:30-113 for internal node i of a tree over n keys.  The
// stored prefix length is in the reference's 32-bit frame.
template <typename K>
__device__ void karras_node(const K *keys, int n, int i, int *left, int *right,
                            int *rfirst, int *rlast, int *plen, int *parent) {
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
  const int first = (i < j) ? i : j;
  const int last = (i > j) ? i : j;
  rfirst[i] = first;
  rlast[i] = last;
  const int node_prefix = lcp(keys, first, last, n);
  plen[i] = node_prefix - (8 * (int)sizeof(K) - 32);
  // findSplit (tree_builder.cu:64-84), including the candidate < last guard
  int split = first;
  if (first < last) {
    int step = last - first;
    do {
      step = (step + 1) >> 1;
      const int candidate = split + step;
      if (candidate < last && lcp(keys, first, candidate, n) > node_prefix) split = candidate;
    } while (step > 1);
  }
  const int lc = (split == first) ? split : n + split;
  const int rc = (split + 1 == last) ? split + 1 : n + split + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = n + i;
  parent[rc] = n + i;
}

// Karras tree over the G unique keys; also finishes the group counts.  The
// root (internal node 0, id G) keeps parent -1; every other node's parent is
// written by exactly one thread, which equals the reference's memset + write.
__global__ void __launch_bounds__(kBlock) karras_kernel(Workspace ws) {
  if (ws.sc->error) return;
  const int g = ws.sc->n_groups;
  if (g <= 0 || g > ws.n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) record_error(ws.sc, kStageGroups, 2);
    return;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g; i += gridDim.x * blockDim.x) {
    ws.gcount[i] = ws.glast[i] - ws.gfirst[i] + 1;
    if (i == 0) ws.rparent[g == 1 ? 0 : g] = -1;
    if (i < g - 1)
      karras_node(ws.ukey, g, i, ws.left, ws.right, ws.rfirst, ws.rlast, ws.plen, ws.rparent);
  }
}

__global__ void __launch_bounds__(kBlock)
    karras_only_kernel(const uint32_t *keys, int n, int *left, int *right, int *rfirst,
                       int *rlast, int *plen, int *parent) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i == 0) parent[n == 1 ? 0 : n] = -1;
    if (i < n - 1) karras_node(keys, n, i, left, right, rfirst, rlast, plen, parent);
  }
}

// -------------------------------------------------------------- plan ----

// radix_to_octree.cu:54-68.  Spatial prefix bits = prefix length in the
// reference's 32-bit frame minus (32 - key bits); for a single system (30-bit
// keys) that is the reference's plen - 2.
__device__ __forceinline__ int octree_level_of(const Workspace &ws, int n_leaves, int r) {
  const int prefix = (r < n_leaves) ? ws.key_bits : ws.plen[r - n_leaves] - (32 - ws.key_bits);
  return prefix / kDims;
}

// radix_to_octree.cu:70-145 for radix node r; returns the edge node count.
__device__ int plan_node(const Workspace &ws, int g, int r) {
  const int nr = 2 * g - 1;
  DevScalars *sc = ws.sc;
  auto fail = [&](int code) {
    record_error(sc, kStagePlan, code);
    ws.plevel[r] = 0;
    ws.pcount[r] = 0;
    return 0;
  };
  if (r < g) {
    if ((ws.ukey[r] >> ws.key_bits) != 0ull) return fail(1);
  } else {
    const int sp = ws.plen[r - g] - (32 - ws.key_bits);
    if (sp < 0 || sp >= ws.key_bits) return fail(4);
  }
  const int p = ws.rparent[r];
  int parent_level = 0;
  if (p != -1) {
    if (p < g || p >= nr) return fail(2);
    parent_level = octree_level_of(ws, g, p);
  }
  const int node_level = (r < g) ? parent_level + 1 : octree_level_of(ws, g, r);
  if (node_level < 0 || node_level > ws.max_level) return fail(3);
  if (node_level < parent_level) return fail(3);
  ws.plevel[r] = node_level;
  ws.pcount[r] = node_level - parent_level;
  return node_level - parent_level;
}

// Plan values + their exclusive scan in one pass; the last tile sets
// M = 1 + sum (radix_to_octree.cu:221-243), bounded by the node capacity.
__global__ void __launch_bounds__(kScanThreads) plan_kernel(Workspace ws) {
  __shared__ unsigned long long row_warp[kScanItems * (kScanThreads / 32)];
  __shared__ unsigned long long s_total, s_prefix;
  __shared__ int s_tile;
  DevScalars *sc = ws.sc;
  const int g = sc->n_groups;
  if (g <= 0 || g > ws.n || sc->error) return;
  const int nr = 2 * g - 1;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(&sc->tile_counter[kTilePlan], 1u);
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kScanTile;
  if (base >= nr) return;
  int val[kScanItems], excl[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int r = base + k * kScanThreads + threadIdx.x;
    val[k] = (r < nr) ? plan_node(ws, g, r) : 0;
  }
  const unsigned long long total = block_scan_rows<kScanItems, kScanThreads>(val, excl, row_warp, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long p =
        warp_lookback(ws.scan_status + ws.scan_tiles_n, tile, total, sc, kStagePlan);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  const long long prefix = (long long)s_prefix;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int r = base + k * kScanThreads + threadIdx.x;
    if (r < nr) ws.poffset[r] = (int)(prefix + excl[k]);
  }
  if (base + kScanTile >= nr && threadIdx.x == 0) {
    const long long m = 1 + prefix + (long long)total;
    if (m > ws.cap_nodes) {
      record_error(sc, kStagePlan, kCodeOverflow);
      sc->n_nodes = 0;
    } else {
      sc->n_nodes = (int)m;
    }
  }
}

// ------------------------------------------------------------ octree ----

// octree_builder.cu:288-321: empty child slots and parents -1, root level 0.
__global__ void __launch_bounds__(kBlock) octree_clear_kernel(Workspace ws) {
  const int m = ws.sc->n_nodes;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    int4 *c = reinterpret_cast<int4 *>(ws.children + (size_t)i * 8);
    c[0] = make_int4(-1, -1, -1, -1);
    c[1] = make_int4(-1, -1, -1, -1);
    ws.oparent[i] = -1;
    ws.olevel[i] = (i == 0) ? 0 : -1;
    ws.oprefix[i] = 0ull;
    ws.ofirst[i] = -1;
    ws.ocount[i] = 0;
    ws.child_count[i] = 0;
    ws.subtree[i] = 0;
    ws.preoff[i] = 0;
    ws.psub[i] = 0;
    ws.pfirst[i] = INT_MAX;
    ws.mass[i] = 0.0;
    ws.comx[i] = 0.0;
    ws.comy[i] = 0.0;
    ws.comz[i] = 0.0;
  }
}

// octree_builder.cu:49-85 for keys of key_bits bits.
__device__ __forceinline__ unsigned long long prefix_at_level(unsigned long long key, int level, int key_bits) {
  if (level == 0) return 0ull;
  const int rem = key_bits - level * kDims;
  return (key >> rem) << rem;
}
__device__ __forceinline__ int octant_at_level(unsigned long long key, int level, int key_bits) {
  return (int)((key >> (key_bits - level * kDims)) & 7ull);
}

// octree_builder.cu:87-224: each radix edge emits its chain of octree nodes
// at ids 1 + edgeNodeOffset[r] + k; children slots are claimed with
// atomicCAS so a collision is detected as the reference does.
__global__ void __launch_bounds__(kBlock) materialize_kernel(Workspace ws) {
  DevScalars *sc = ws.sc;
  const int g = sc->n_groups;
  const int m = sc->n_nodes;
  if (g <= 0 || g > ws.n || m <= 0 || sc->error) return;
  const int nr = 2 * g - 1;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nr; r += gridDim.x * blockDim.x) {
    const int count = ws.pcount[r];
    const int node_level = ws.plevel[r];
    if (count < 0 || node_level < 0 || node_level > ws.max_level) {
      record_error(sc, kStageOctree, 1);
      continue;
    }
    if (count == 0) {
      if (r < g) record_error(sc, kStageOctree, 5);
      continue;
    }
    const int parent_level = node_level - count;
    if (parent_level < 0) {
      record_error(sc, kStageOctree, 1);
      continue;
    }
    unsigned long long key;
    if (r < g) {
      key = ws.ukey[r];
    } else {
      const int f = ws.rfirst[r - g];
      if (f < 0 || f >= g) {
        record_error(sc, kStageOctree, 7);
        continue;
      }
      key = ws.ukey[f];
    }
    int parent_node = 0;
    int anc = ws.rparent[r];
    int iters = 0;
    bool bad = false;
    while (anc != -1) {
      if (anc < 0 || anc >= nr) {
        record_error(sc, kStageOctree, 2);
        bad = true;
        break;
      }
      const int ac = ws.pcount[anc];
      if (ac > 0) {
        if (ws.plevel[anc] != parent_level) {
          record_error(sc, kStageOctree, 3);
          bad = true;
          break;
        }
        parent_node = 1 + ws.poffset[anc] + ac - 1;
        break;
      }
      anc = ws.rparent[anc];
      if (++iters > nr) {
        record_error(sc, kStageOctree, 2);
        bad = true;
        break;
      }
    }
    if (bad) continue;
    if (anc == -1 && parent_level != 0) {
      record_error(sc, kStageOctree, 3);
      continue;
    }
    if (parent_node < 0 || parent_node >= m) {
      record_error(sc, kStageOctree, 6);
      continue;
    }
    const int first_node = 1 + ws.poffset[r];
    for (int local = 0; local < count; ++local) {
      const int node = first_node + local;
      if (node <= 0 || node >= m) {
        record_error(sc, kStageOctree, 6);
        bad = true;
        break;
      }
      const int level = parent_level + local + 1;
      const int par = (local == 0) ? parent_node : node - 1;
      ws.olevel[node] = level;
      ws.oprefix[node] = prefix_at_level(key, level, ws.key_bits);
      ws.oparent[node] = par;
      const int prev = atomicCAS(&ws.children[(size_t)par * 8 + octant_at_level(key, level, ws.key_bits)], -1, node);
      if (prev != -1 && prev != node) {
        record_error(sc, kStageOctree, 4);
        bad = true;
        break;
      }
    }
    if (bad) continue;
    if (r < g) {
      const int leaf = first_node + count - 1;
      const int ll = parent_level + count;
      if (ll <= 0 || ll > ws.max_level) {
        record_error(sc, kStageOctree, 5);
        continue;
      }
      ws.ofirst[leaf] = ws.gfirst[r];
      ws.ocount[leaf] = ws.gcount[r];
    }
  }
}

// -------------------------------------------- geometry + leaf physics ----

// Per node: cell centre / half size from the Morton prefix path
// (octree_geometry.cu:56-102), child count (octree_physics.cu:64-93) and,
// for occupied leaves, mass and centre of mass summed over the group's
// particles in sorted order (octree_physics.cu:95-154).  The step runs both
// parts in one pass; the function-level entry points (computeOctreeGeometry,
// computeOctreeMassAndCenterOfMass) run one each.
template <bool kGeometry, bool kPhysics>
__global__ void __launch_bounds__(kBlock) node_init_kernel(Workspace ws) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < m; node += gridDim.x * blockDim.x) {
    if (kGeometry) {
      const int level = ws.olevel[node];
      if (level < 0 || level > ws.max_level) {
        record_error(sc, kStageGeometry, 1);
      } else {
        const unsigned long long prefix = ws.oprefix[node];
        const int kb = ws.key_bits;
        bool valid = (prefix >> kb) == 0ull;
        if (valid) {
          if (level == 0) {
            valid = prefix == 0ull;
          } else {
            const int rem = kb - level * kDims;
            valid = (prefix & ((1ull << rem) - 1ull)) == 0ull;
          }
        }
        if (!valid) {
          record_error(sc, kStageGeometry, 2);
        } else if (level < ws.sys_levels) {
          // above the system roots of an ensemble: no cell, never visited
          ws.cx[node] = 0.0;
          ws.cy[node] = 0.0;
          ws.cz[node] = 0.0;
          ws.half[node] = 0.0;
        } else {
          const double *box = ws.sys_box + 4 * (size_t)(prefix >> kSpatialBits);
          double cx = box[0], cy = box[1], cz = box[2], h = __dmul_rn(box[3], 0.5);
          for (int d = ws.sys_levels + 1; d <= level; ++d) {
            const int oct = (int)((prefix >> (kb - d * kDims)) & 7ull);
            const double ch = __dmul_rn(h, 0.5);
            cx = __dadd_rn(cx, (oct & 4) ? ch : -ch);
            cy = __dadd_rn(cy, (oct & 2) ? ch : -ch);
            cz = __dadd_rn(cz, (oct & 1) ? ch : -ch);
            h = ch;
          }
          ws.cx[node] = cx;
          ws.cy[node] = cy;
          ws.cz[node] = cz;
          ws.half[node] = h;
        }
      }
    }
    if (!kPhysics) continue;
    const int4 *c4 = reinterpret_cast<const int4 *>(ws.children + (size_t)node * 8);
    const int4 a = c4[0], b = c4[1];
    const int ch[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    int cnt = 0;
    bool bad = false;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      if (ch[o] == -1) continue;
      if (ch[o] <= 0 || ch[o] >= m) bad = true;
      ++cnt;
    }
    if (bad) {
      record_error(sc, kStagePhysics, 1);
      continue;
    }
    ws.child_count[node] = cnt;
    const int pc = ws.ocount[node];
    if (pc > 0 && cnt != 0) record_error(sc, kStagePhysics, 4);
    if (node == 0) ws.preoff[0] = 0;
    if (pc <= 0) continue;
    const int f = ws.ofirst[node];
    if (f < 0 || f + pc > ws.n) {
      record_error(sc, kStagePhysics, 2);
      continue;
    }
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    for (int k = 0; k < pc; ++k) {
      const double4 p = ws.pm4[f + k];
      tm = __dadd_rn(tm, p.w);
      wx = __fma_rn(p.w, p.x, wx);
      wy = __fma_rn(p.w, p.y, wy);
      wz = __fma_rn(p.w, p.z, wz);
    }
    ws.mass[node] = tm;
    if (tm > 0.0) {
      const double inv = __drcp_rn(tm);
      ws.comx[node] = __dmul_rn(wx, inv);
      ws.comy[node] = __dmul_rn(wy, inv);
      ws.comz[node] = __dmul_rn(wz, inv);
    }
    ws.subtree[node] = 1;
    ws.psub[node] = pc;
    ws.pfirst[node] = f;
  }
}

// Octree nodes binned by level: level L owns the fixed region
// [level_base(L), level_base(L) + min(8^L, n)) of by_level (no octree level
// holds more nodes than that), filled in any order.
__device__ __forceinline__ int level_base(const Workspace &ws, int level) {
  long long base = 0, width = 1;
  for (int l = 0; l < level; ++l) {
    base += (width < ws.n) ? width : ws.n;
    if (width < (1ll << 40)) width *= 8;
  }
  return (int)base;
}
__device__ __forceinline__ int level_cap(const Workspace &ws, int level) {
  long long width = 1;
  for (int l = 0; l < level && width < (1ll << 40); ++l) width *= 8;
  return (int)((width < ws.n) ? width : ws.n);
}

__global__ void __launch_bounds__(kBlock) level_bin_kernel(Workspace ws) {
  __shared__ int s_cnt[kMaxLevels], s_base[kMaxLevels];
  __shared__ int s_m;
  DevScalars *sc = ws.sc;
  if (threadIdx.x == 0) s_m = sc->error ? 0 : sc->n_nodes;
  __syncthreads();
  const int m = s_m;  // block-uniform trip count below
  for (int b0 = blockIdx.x * blockDim.x; b0 < m; b0 += gridDim.x * blockDim.x) {
    if (threadIdx.x < kMaxLevels) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int v = b0 + threadIdx.x;
    int level = -1, slot = 0;
    if (v < m) {
      level = ws.olevel[v];
      if (level < 0 || level > ws.max_level || level >= kMaxLevels) {
        record_error(sc, kStagePhysics, 5);
        level = -1;
      } else {
        slot = atomicAdd(&s_cnt[level], 1);
      }
    }
    __syncthreads();
    if (threadIdx.x < kMaxLevels && s_cnt[threadIdx.x] > 0)
      s_base[threadIdx.x] = atomicAdd(&sc->level_count[threadIdx.x], s_cnt[threadIdx.x]);
    __syncthreads();
    if (level >= 0) {
      const int pos = s_base[level] + slot;
      if (pos < level_cap(ws, level))
        ws.by_level[level_base(ws, level) + pos] = v;
      else
        record_error(sc, kStagePhysics, 5);
    }
    __syncthreads();
  }
}

// octree_physics.cu:156-245, one octree level per launch, deepest first:
// every internal node of the level combines its (finished) children in
// octant order 0..7 -- the reference's deterministic order, so mass and
// centre of mass are bit-identical -- and also sums its subtree size,
// particle count and first particle and assigns each child its offset
// within the node's depth-first preorder range (children visited 7 -> 0).
// The device scalars a level launch needs, read once per block (every
// thread reading the same word would queue at one L2 slice).
struct LevelScalars {
  int m, count;
};
__device__ __forceinline__ LevelScalars level_scalars(const Workspace &ws, int level) {
  __shared__ LevelScalars s;
  if (threadIdx.x == 0) {
    const DevScalars *sc = ws.sc;
    s.m = sc->error ? 0 : sc->n_nodes;
    s.count = sc->error ? 0 : min(sc->level_count[level], level_cap(ws, level));
  }
  __syncthreads();
  return s;
}

__global__ void __launch_bounds__(kBlock) propagate_level_kernel(Workspace ws, int level) {
  DevScalars *sc = ws.sc;
  const LevelScalars ls = level_scalars(ws, level);
  const int m = ls.m, count = ls.count;
  const int base = level_base(ws, level);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int node = ws.by_level[base + i];
    if (node < 0 || node >= m || ws.child_count[node] == 0) continue;  // leaves: node_init_kernel
    const int4 *c4 = reinterpret_cast<const int4 *>(ws.children + (size_t)node * 8);
    const int4 a = c4[0], b = c4[1];
    const int ch[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
    int size = 1, nparticles = 0, firstp = INT_MAX;
    int sub[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      sub[o] = 0;
      const int c = ch[o];
      if (c <= 0 || c >= m) continue;
      if (ws.olevel[c] <= level) {
        record_error(sc, kStagePhysics, 5);
        continue;
      }
      const double cm = ws.mass[c];
      tm = __dadd_rn(tm, cm);
      wx = __fma_rn(cm, ws.comx[c], wx);
      wy = __fma_rn(cm, ws.comy[c], wy);
      wz = __fma_rn(cm, ws.comz[c], wz);
      sub[o] = ws.subtree[c];
      size += sub[o];
      nparticles += ws.psub[c];
      firstp = min(firstp, ws.pfirst[c]);
    }
    ws.mass[node] = tm;
    if (tm > 0.0) {
      const double inv = __drcp_rn(tm);
      ws.comx[node] = __dmul_rn(wx, inv);
      ws.comy[node] = __dmul_rn(wy, inv);
      ws.comz[node] = __dmul_rn(wz, inv);
    } else {
      ws.comx[node] = 0.0;
      ws.comy[node] = 0.0;
      ws.comz[node] = 0.0;
    }
    int run = 1;
#pragma unroll
    for (int o = 7; o >= 0; --o) {
      if (ch[o] <= 0 || ch[o] >= m) continue;
      ws.preoff[ch[o]] = run;
      run += sub[o];
    }
    ws.subtree[node] = size;
    ws.psub[node] = nparticles;
    ws.pfirst[node] = firstp;
  }
}

// --------------------------------------------------------------- layout --

// Traversal records in depth-first preorder with children visited octant
// 7 -> 0 (the reference's traversal order, barnes_hut.cu:90-162).  Preorder
// indices go top-down, one octree level per launch: node n sits at
// pre(n) = pre(parent) + its offset within the parent's range; then one
// launch over all nodes writes the records.  Its
// subtree ends at pre(n) + size(n) ("skip"), and its children are listed in
// visit order.  The acceptance radius crit = side/theta + |com - centre|
// (barnes_hut.cu:283-293) is precomputed once per node, with a +-2^-44 band
// around crit^2 inside which the traversal falls back to the exact
// sqrt(d^2) > crit comparison.
// Preorder indices in closed form.  In a depth-first preorder that visits
// children in octant order 7 -> 0 (descending Morton order), the nodes before
// n are its ancestors and the nodes lying wholly after n in Morton order, so
// with M nodes, size(n) the nodes of n's subtree and before(n) the nodes
// lying wholly before it (their particle range ends before n's first
// particle), pre(n) = M - size(n) - before(n).  before() is a count of range
// ends per sorted particle index, scanned: two passes over the particles
// instead of one launch per octree level.
__global__ void __launch_bounds__(kBlock) ends_hist_kernel(Workspace ws) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < m; node += gridDim.x * blockDim.x) {
    const int last = ws.pfirst[node] + ws.psub[node] - 1;
    if (ws.psub[node] < 1 || ws.pfirst[node] < 0 || last >= ws.n) {
      record_error(sc, kStageLayout, 1);
      continue;
    }
    atomicAdd(&ws.pends[last], 1);
  }
}

__global__ void __launch_bounds__(kScanThreads) ends_scan_kernel(Workspace ws) {
  __shared__ unsigned long long row_warp[kScanItems * (kScanThreads / 32)];
  __shared__ unsigned long long s_total, s_prefix;
  __shared__ int s_tile;
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int n = ws.n;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(&sc->tile_counter[kTileEnds], 1u);
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kScanTile;
  if (base >= n) return;
  int val[kScanItems], excl[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    val[k] = (i < n) ? ws.pends[i] : 0;
  }
  const unsigned long long total = block_scan_rows<kScanItems, kScanThreads>(val, excl, row_warp, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long p =
        warp_lookback(ws.scan_status + 2 * ws.scan_tiles_n + ws.scan_tiles_r, tile, total, sc, kStageLayout);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  const int prefix = (int)s_prefix;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    if (i < n) ws.pends[i] = prefix + excl[k];
  }
}

__global__ void __launch_bounds__(kBlock) preorder_kernel(Workspace ws) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < m; node += gridDim.x * blockDim.x) {
    const int f = ws.pfirst[node];
    const int pre = (f >= 0 && f < ws.n) ? m - ws.subtree[node] - ws.pends[f] : -1;
    if (pre < 0 || pre >= m) {
      record_error(sc, kStageLayout, 1);
      continue;
    }
    ws.pre_of[node] = pre;
  }
}

__global__ void __launch_bounds__(kBlock) layout_kernel(Workspace ws, double theta) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < m; node += gridDim.x * blockDim.x) {
    const int pre = ws.pre_of[node];
    const double h = ws.half[node];
    const int lvl = ws.olevel[node];
    if (lvl == ws.sys_levels) ws.root_pre[ws.oprefix[node] >> kSpatialBits] = pre;
    if (!(h > 0.0) && lvl >= ws.sys_levels) record_error(sc, kStageTraversal, 8);
    int pc = ws.ocount[node];
    const int cnt = ws.child_count[node];
    const int f = ws.ofirst[node];
    if (pc > 0 && (f < 0 || f + pc > ws.n)) {
      record_error(sc, kStageTraversal, 2);
      pc = 0;
    }
    int size = (pc > 0) ? 1 : ws.subtree[node];
    if (size < 1 || pre + size > m) {
      record_error(sc, kStageLayout, 1);
      size = 1;
    }
    if (pc > 0 && cnt != 0) record_error(sc, kStageTraversal, 7);
    const double mass = ws.mass[node];
    if (pc <= 0 && cnt == 0 && mass != 0.0) record_error(sc, kStageTraversal, 5);
    const double comx = ws.comx[node], comy = ws.comy[node], comz = ws.comz[node];
    const double cx = ws.cx[node], cy = ws.cy[node], cz = ws.cz[node];
    ws.node_a[pre] = make_double4(comx, comy, comz, mass);
    ws.node_b[pre] = make_double4(cx, cy, cz, h);
    const double side = __dmul_rn(2.0, h);
    const double ox = __dsub_rn(comx, cx), oy = __dsub_rn(comy, cy), oz = __dsub_rn(comz, cz);
    const double o2 = __fma_rn(oz, oz, __fma_rn(oy, oy, __dmul_rn(ox, ox)));
    const double crit = (theta > 0.0) ? __dadd_rn(__ddiv_rn(side, theta), __dsqrt_rn(o2)) : INFINITY;
    const double c2 = __dmul_rn(crit, crit);
    // the mixed walk's squared acceptance radius for a target box: crit, or
    // the farthest a point of the cell lies from the centre of mass
    // (sqrt(3) h + |com - centre|) when that is larger, widened by 2^-40 for
    // rounding.  A box farther than this from the centre of mass touches no
    // point of the cell, so no overlap test is needed.
    const double inner = __fma_rn(1.7320508075688774, h, __dsqrt_rn(o2));
    const double cm = fmax(crit, inner) * (1.0 + 0x1p-40);
    ws.node_c[pre] = make_double4(crit, c2 * (1.0 - 0x1p-44), c2 * (1.0 + 0x1p-44), cm * cm);
    int j = 0;
    int *kids = ws.node_kids + (size_t)pre * 8;
    for (int o = 7; o >= 0; --o) {
      const int c = ws.children[(size_t)node * 8 + o];
      if (c <= 0 || c >= m) continue;
      kids[j++] = pre + ws.preoff[c];
    }
    ws.node_meta[pre] = make_int4(pre + size, pc > 0 ? f : -1, pc > 0 ? pc : 0, j);
    if (ws.node_m) {
      MixedNode rec;
      rec.a = make_double4(comx, comy, comz, mass);
      rec.cr2 = __double2float_ru(cm * cm * (1.0 + 0x1p-18));
      rec.first = pc > 0 ? f : -1;
      rec.count = pc > 0 ? pc : 0;
      rec.nchild = j;
      ws.node_m[pre] = rec;
    }
    for (; j < 8; ++j) kids[j] = -1;
  }
}

// ------------------------------------------------------ target groups ---

// Target groups for the traversal.  A subtree is a group candidate when it
// holds at most group_max particles and is compact: a leaf, a single
// particle, or a cell at least group_depth levels below its system's root.
// Every other node splits: a node split only for its count packs its
// candidate children, in octant (= Morton) order, greedily into runs of at
// most group_max particles, one group per run; a node split for its size
// makes each candidate child a group of its own (merging siblings would span
// the wide cell again).  Groups are contiguous ranges of the sorted
// particles, never larger than group_max, so a warp's targets stay spatially
// compact (fixed 32-particle slices of the Morton order can straddle the
// whole system where the curve jumps; a sparse outer cell holding a few dozen
// scattered particles gives a box so wide that its walk opens most of the
// tree).
__device__ __forceinline__ bool group_compact(const Workspace &ws, int node, int np) {
  return ws.ocount[node] > 0 || np <= 1 || ws.olevel[node] - ws.sys_levels >= ws.group_depth;
}

__global__ void __launch_bounds__(kBlock) group_mark_kernel(Workspace ws) {
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int m = sc->n_nodes;
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < m; node += gridDim.x * blockDim.x) {
    const int gmax = ws.group_max;
    const int np = ws.psub[node];
    const bool virt = ws.olevel[node] < ws.sys_levels;  // children are other systems
    const bool compact = !virt && group_compact(ws, node, np);
    if (!virt && np <= gmax && compact) {
      // a whole system that is one group
      if (ws.olevel[node] == ws.sys_levels && np > 0) ws.tflag[ws.pfirst[node]] = 1;
      continue;
    }
    if (ws.ocount[node] > 0) {
      // an occupied leaf with more than group_max coincident-key particles:
      // consecutive slices of group_max
      const int f = ws.pfirst[node];
      for (int k = 0; k < np; k += gmax)
        if (f + k >= 0 && f + k < ws.n) ws.tflag[f + k] = 1;
      continue;
    }
    const bool merge = compact;  // split for its count only
    int run = 0;
    for (int o = 0; o < 8; ++o) {
      const int c = ws.children[(size_t)node * 8 + o];
      if (c <= 0 || c >= m) continue;
      const int cp = ws.psub[c];
      if (virt) run = 0;
      if (cp > gmax || !group_compact(ws, c, cp)) {
        // the child splits itself
        run = 0;
        continue;
      }
      if (!merge || run == 0 || run + cp > gmax) {
        const int f = ws.pfirst[c];
        if (f >= 0 && f < ws.n) ws.tflag[f] = 1;
        run = 0;
      }
      run += cp;
    }
  }
}

// Compaction of the group-start flags into the list of group starts.
__global__ void __launch_bounds__(kScanThreads) group_scan_kernel(Workspace ws) {
  __shared__ unsigned long long row_warp[kScanItems * (kScanThreads / 32)];
  __shared__ unsigned long long s_total, s_prefix;
  __shared__ int s_tile;
  DevScalars *sc = ws.sc;
  if (sc->error) return;
  const int n = ws.n;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(&sc->tile_counter[kTileTargetGroups], 1u);
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kScanTile;
  if (base >= n) return;
  int flag[kScanItems], excl[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    flag[k] = (i < n) ? (int)ws.tflag[i] : 0;
  }
  const unsigned long long total = block_scan_rows<kScanItems, kScanThreads>(flag, excl, row_warp, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long p = warp_lookback(ws.scan_status + ws.scan_tiles_n + ws.scan_tiles_r, tile,
                                               total, sc, kStageGroups);
    if (threadIdx.x == 0) s_prefix = p;
  }
  __syncthreads();
  const int prefix = (int)s_prefix;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int i = base + k * kScanThreads + threadIdx.x;
    if (i < n && flag[k]) {
      const int g = prefix + excl[k];
      if (g >= 0 && g < n) ws.tstart[g] = i;
    }
  }
  if (base + kScanTile >= n && threadIdx.x == 0) sc->n_tgroups = prefix + (int)total;
}

// ------------------------------------------------- level-order build ----
//
// The step's octree, built from the sorted unique keys without the radix
// tree.  The octree the reference derives from the Karras tree
// (radix_to_octree.cu:70-145, octree_builder.cu:87-224) holds, for every leaf
// group g of the G sorted unique keys u[0..G), the cells of u[g]'s prefixes
// from the root down to level lambda_g = 1 + max(0, delta_g, delta_{g+1}),
// where delta_g is the number of octree levels u[g-1] and u[g] share (-1 past
// either end): a leaf sits one level below its radix parent, whose prefix is
// the longer of the leaf's two common prefixes.  Group g is the first group
// of its cells at levels (delta_g, lambda_g] and the last group of its cells
// at levels (delta_{g+1}, lambda_g].
//
// Numbered level by level, each level in ascending key order, the children of
// a cell (octants 0..7) are consecutive entries of the next level.  A
// depth-first preorder that visits children octant 7 -> 0 meets the groups in
// descending key order, group g adding its cells at levels (delta_{g+1},
// lambda_g] top-down; with S(g) the number of cells added by the groups >= g,
// the cell at level L whose last group is g has preorder index
// S(g) - lambda_g + L - 1, and a cell's subtree ends at S(its first group).
// One scan over the groups numbers every cell and gives its first child and
// its preorder range; mass and centre of mass are then combined level by
// level, deepest first, from the consecutive child records in octant order
// (octree_physics.cu:156-245), and the traversal records are written at the
// preorder index in the same pass.

// Octree levels two distinct keys of key_bits bits share.
__device__ __forceinline__ int common_levels(unsigned long long a, unsigned long long b, int key_bits) {
  return (__clzll((long long)(a ^ b)) - (64 - key_bits)) / kDims;
}

// Per group: the level span (delta, lambda, delta of the next group) and the
// particle count; per tile of kScanTile groups: the cells its groups start at
// each level and the cells they end.
__global__ void __launch_bounds__(kScanThreads) lo_span_kernel(Workspace ws) {
  __shared__ int s_cnt[kLevelOrderChannels];
  __shared__ int s_g;
  constexpr int kEnded = kMaxLevels;  // channel of the ended cells
  DevScalars *sc = ws.sc;
  if (threadIdx.x == 0) {
    const int g = sc->n_groups;
    const bool ok = g > 0 && g <= ws.n;
    if (!ok && blockIdx.x == 0) record_error(sc, kStageGroups, 2);
    s_g = ok ? g : 0;
  }
  if (threadIdx.x < kLevelOrderChannels) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int G = s_g, kb = ws.key_bits;
  const int base = blockIdx.x * kScanTile;
#pragma unroll 1
  for (int k = 0; k < kScanItems; ++k) {
    const int g = base + k * kScanThreads + threadIdx.x;
    if (g >= G) break;
    ws.gcount[g] = ws.glast[g] - ws.gfirst[g] + 1;
    const unsigned long long key = ws.ukey[g];
    int d = -1, dn = -1;
    bool bad = (key >> kb) != 0ull;
    if (g > 0) {
      const unsigned long long kp = ws.ukey[g - 1];
      if (kp >= key) bad = true;
      else d = common_levels(kp, key, kb);
    }
    if (g + 1 < G) {
      const unsigned long long kn = ws.ukey[g + 1];
      if (kn <= key) bad = true;
      else dn = common_levels(key, kn, kb);
    }
    const int lam = 1 + max(0, max(d, dn));
    if (bad || lam > ws.max_level) {
      record_error(sc, kStagePlan, bad ? 1 : 3);
      continue;
    }
    ws.gspan[g] = (d + 1) | (lam << 8) | ((dn + 1) << 16);
    for (int l = d + 1; l <= lam; ++l) atomicAdd(&s_cnt[l], 1);
    atomicAdd(&s_cnt[kEnded], lam - dn);
  }
  __syncthreads();
  if (threadIdx.x < kLevelOrderChannels)
    ws.lo_tiles[(size_t)blockIdx.x * kLevelOrderChannels + threadIdx.x] = s_cnt[threadIdx.x];
}

// Exclusive prefixes of the per-tile counts, in place, through shared memory:
// chunks of tiles are loaded with coalesced reads, each warp scans one
// channel of the chunk (a lane holds 8 consecutive tiles), and the chunk is
// written back coalesced.  The totals give the cells per level and M (the
// node count).
__global__ void __launch_bounds__(32 * kLevelOrderChannels) lo_tile_scan_kernel(Workspace ws) {
  constexpr int kEnded = kMaxLevels;
  constexpr int kPerLane = 8;
  constexpr int kChunk = 32 * kPerLane;  // tiles per chunk
  __shared__ int s_cnt[kChunk][kLevelOrderChannels + 1];
  __shared__ long long s_total[kLevelOrderChannels];
  DevScalars *sc = ws.sc;
  const int g = sc->n_groups;
  const int G = (g > 0 && g <= ws.n) ? g : 0;
  const int tiles = (G + kScanTile - 1) / kScanTile;
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int inc = 0;  // running total of channel c
  for (int t0 = 0; t0 < tiles; t0 += kChunk) {
    const int nt = min(kChunk, tiles - t0);
    const int *src = ws.lo_tiles + (size_t)t0 * kLevelOrderChannels;
    for (int i = threadIdx.x; i < nt * kLevelOrderChannels; i += blockDim.x)
      s_cnt[i / kLevelOrderChannels][i % kLevelOrderChannels] = src[i];
    __syncthreads();
    int v[kPerLane], sum = 0;
#pragma unroll
    for (int j = 0; j < kPerLane; ++j) {
      const int t = lane * kPerLane + j;
      v[j] = (t < nt) ? s_cnt[t][c] : 0;
      sum += v[j];
    }
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    int acc = inc + x - sum;
#pragma unroll
    for (int j = 0; j < kPerLane; ++j) {
      const int t = lane * kPerLane + j;
      if (t < nt) s_cnt[t][c] = acc;
      acc += v[j];
    }
    inc += __shfl_sync(0xffffffffu, x, 31);
    __syncthreads();
    int *dst = ws.lo_tiles + (size_t)t0 * kLevelOrderChannels;
    for (int i = threadIdx.x; i < nt * kLevelOrderChannels; i += blockDim.x)
      dst[i] = s_cnt[i / kLevelOrderChannels][i % kLevelOrderChannels];
    __syncthreads();
  }
  if (lane == 0) s_total[c] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long m = 0;
    for (int l = 0; l < kMaxLevels; ++l) {
      sc->level_count[l] = (int)s_total[l];
      sc->level_base[l] = (int)m;
      m += s_total[l];
    }
    sc->level_base[kMaxLevels] = sc->level_base[kMaxLevels + 1] = (int)m;
    if (G == 0 || m != s_total[kEnded] || m > ws.cap_nodes) {
      if (G > 0) record_error(sc, m > ws.cap_nodes ? kStagePlan : kStageLayout, m > ws.cap_nodes ? kCodeOverflow : 1);
      sc->n_nodes = 0;
    } else {
      sc->n_nodes = (int)m;
    }
  }
}

// A finished cell of the upward pass whose traversal records are still to
// be written: its mass and centre of mass and what the records need.
struct LoCell {
  double4 a;  // centre of mass, mass
  unsigned long long key;
  int level, pre, skip, pf, pe, nk;
  bool leaf;
};

// One cell's mass and centre of mass from its sums, and the LevelNode its
// parent reads (the only record another thread of the upward pass needs).
__device__ __forceinline__ void lo_emit_node(const Workspace &ws, int b, double tm, double wx, double wy, double wz,
                                             LoCell &c) {
  double comx = 0.0, comy = 0.0, comz = 0.0;
  if (tm > 0.0) {
    const double inv = __drcp_rn(tm);
    comx = __dmul_rn(wx, inv);
    comy = __dmul_rn(wy, inv);
    comz = __dmul_rn(wz, inv);
  }
  c.a = make_double4(comx, comy, comz, tm);
  LevelNode rec;
  rec.a = c.a;
  rec.pre = c.pre;
  rec.np = c.pe - c.pf;
  rec.first = c.pf;
  rec.leaf = c.leaf ? 1 : 0;
  ws.lo_node[b] = rec;
}

// A finished cell's geometry from the key prefix (octree_geometry.cu:56-102)
// and its traversal records at the preorder index (as layout_kernel writes
// them).  The child list is the caller's.  Neither walk applies the
// acceptance test to an occupied leaf (its particles are summed), so a leaf
// gets no geometry and no acceptance radius.  Returns false on an invalid
// system id.
template <int kRecords>
__device__ __forceinline__ bool lo_emit_records(const Workspace &ws, double theta, const LoCell &c) {
  const int level = c.level, pre = c.pre;
  const bool leaf = c.leaf;
  const double4 a = c.a;
  double cx = 0.0, cy = 0.0, cz = 0.0, h = 0.0;
  if (level >= ws.sys_levels) {
    const unsigned long long sys = c.key >> kSpatialBits;
    if (sys >= (unsigned long long)ws.n_systems) return false;
    if (level == ws.sys_levels) ws.root_pre[sys] = pre;
  }
  if (level >= ws.sys_levels && !leaf) {
    const unsigned long long sys = c.key >> kSpatialBits;
    const double *box = ws.sys_box + 4 * (size_t)sys;
    cx = box[0];
    cy = box[1];
    cz = box[2];
    h = __dmul_rn(box[3], 0.5);
    const int kb = ws.key_bits;
    for (int d = ws.sys_levels + 1; d <= level; ++d) {
      const int oct = (int)((c.key >> (kb - d * kDims)) & 7ull);
      const double ch = __dmul_rn(h, 0.5);
      cx = __dadd_rn(cx, (oct & 4) ? ch : -ch);
      cy = __dadd_rn(cy, (oct & 2) ? ch : -ch);
      cz = __dadd_rn(cz, (oct & 1) ? ch : -ch);
      h = ch;
    }
    if (!(h > 0.0)) record_error(ws.sc, kStageTraversal, 8);
  }
  double crit = 0.0, c2 = 0.0, cm = 0.0;
  if (!leaf) {
    const double side = __dmul_rn(2.0, h);
    const double ox = __dsub_rn(a.x, cx), oy = __dsub_rn(a.y, cy), oz = __dsub_rn(a.z, cz);
    const double o2 = __fma_rn(oz, oz, __fma_rn(oy, oy, __dmul_rn(ox, ox)));
    crit = (theta > 0.0) ? __dadd_rn(__ddiv_rn(side, theta), __dsqrt_rn(o2)) : INFINITY;
    c2 = __dmul_rn(crit, crit);
    const double inner = __fma_rn(1.7320508075688774, h, __dsqrt_rn(o2));
    cm = fmax(crit, inner) * (1.0 + 0x1p-40);
  }
  if (kRecords & kRecordsFp64) {
    ws.node_a[pre] = a;
    if (!leaf) {
      ws.node_b[pre] = make_double4(cx, cy, cz, h);
      ws.node_c[pre] = make_double4(crit, c2 * (1.0 - 0x1p-44), c2 * (1.0 + 0x1p-44), cm * cm);
    }
    ws.node_meta[pre] = make_int4(c.skip, leaf ? c.pf : -1, leaf ? c.pe - c.pf : 0, c.nk);
  }
  if (kRecords & kRecordsMixed) {
    MixedNode mrec;
    mrec.a = a;
    mrec.cr2 = leaf ? 0.f : __double2float_ru(cm * cm * (1.0 + 0x1p-18));
    mrec.first = leaf ? c.pf : -1;
    mrec.count = leaf ? c.pe - c.pf : 0;
    mrec.nchild = c.nk;
    ws.node_m[pre] = mrec;
  }
  return true;
}

// Cell numbers: per tile, the cells started by the groups before it (the
// tile prefixes) plus the ranks inside the tile.  Writes each cell's first
// particle, first child, subtree end and parent, and zeroes its arrival
// counter (by its first group), and
// its particle end, preorder index and key (by its last group; every group of
// a cell carries the cell's prefix), and per group its leaf's level-order
// index and S(g) (the leaf sits at level lambda, preorder index S(g) - 1).
template <int kRecords>
__global__ void __launch_bounds__(kScanThreads) lo_rank_kernel(Workspace ws, double theta) {
  constexpr int kWarps = kScanThreads / 32;
  constexpr int kNodes = kMaxLevels;  // channel of the ended cells (the node count S)
  static_assert(kNodes < kLevelOrderChannels, "one warp holds every channel");
  __shared__ int s_warp[kWarps][kLevelOrderChannels];
  __shared__ int s_prefix[kLevelOrderChannels];
  __shared__ int s_base[kMaxLevels + 2];
  __shared__ int s_span[kScanItems][kScanThreads];
  __shared__ int s_g, s_m;
  DevScalars *sc = ws.sc;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  // the level bases, one load per thread (a serial loop of dependent
  // additions over the level counts would cost a memory round trip each)
  if (tid < kMaxLevels + 2) s_base[tid] = sc->level_base[tid];
  if (tid == 0) {
    const int g = sc->n_groups, m = sc->n_nodes;
    s_g = (g > 0 && g <= ws.n && m > 0) ? g : 0;
    s_m = m;
  }
  if (tid < kLevelOrderChannels) s_prefix[tid] = ws.lo_tiles[(size_t)tile * kLevelOrderChannels + tid];
  __syncthreads();
  const int G = s_g, M = s_m;
  const int base = tile * kScanTile;
  if (G == 0 || base >= G) return;
  const int max_level = ws.max_level;
  // each warp owns 32 * kScanItems consecutive groups, item k at g0 + 32 k;
  // a group's cells: started at levels (delta, lambda], ended at (delta_next, lambda]
  const int g0 = base + warp * (32 * kScanItems) + lane;
  auto masks = [&](int sp, unsigned &smask, unsigned &lmask, int &lam) {
    smask = lmask = 0u;
    lam = 0;
    if (sp < 0) return;
    const int d = (sp & 255) - 1, l = (sp >> 8) & 255, dn = ((sp >> 16) & 255) - 1;
    if (l < 1 || l > max_level || d >= l || dn >= l) {
      record_error(sc, kStagePlan, 3);
      return;
    }
    const unsigned upto = (2u << l) - 1u;  // levels 0..lambda
    smask = upto & ~((1u << (d + 1)) - 1u);
    lmask = upto & ~((1u << (dn + 1)) - 1u);
    lam = l;
  };
  // the spans, all loads in flight at once; kept in shared memory for the
  // second pass
  int span[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int g = g0 + 32 * k;
    span[k] = (g < G) ? ws.gspan[g] : -1;
  }
  // this warp's cells per level (lane l) and node count (lane kNodes)
  int cnt[kMaxLevels];
#pragma unroll
  for (int l = 0; l < kMaxLevels; ++l) cnt[l] = 0;
  int e = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_span[k][tid] = span[k];
    unsigned sm, lm;
    int lam;
    masks(span[k], sm, lm, lam);
#pragma unroll
    for (int l = 0; l < kMaxLevels; ++l) cnt[l] += (int)((sm >> l) & 1u);
    e += __popc(lm);
  }
  // the warp's level range: ranks are formed only where its groups have
  // cells, and at the level above (the parent of a group's shallowest cell)
  int wlo = kMaxLevels, whi = -1;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (span[k] < 0) continue;
    const int d = (span[k] & 255) - 1, l = (span[k] >> 8) & 255, dn = ((span[k] >> 16) & 255) - 1;
    wlo = min(wlo, max(0, min(d, dn)));
    whi = max(whi, l + 1);
  }
  wlo = __reduce_min_sync(0xffffffffu, wlo);
  whi = min(__reduce_max_sync(0xffffffffu, whi), kMaxLevels);
  int mine = __reduce_add_sync(0xffffffffu, e);
  mine = (lane == kNodes) ? mine : 0;
#pragma unroll
  for (int l = 0; l < kMaxLevels; ++l) {
    const int c = __reduce_add_sync(0xffffffffu, cnt[l]);
    if (lane == l) mine = c;
  }
  s_warp[warp][lane] = mine;
  __syncthreads();
  if (warp == 0) {
    // channel `lane`: the warps' exclusive offsets inside the tile
    int tot = 0;
    for (int w = 0; w < kWarps; ++w) {
      const int v = s_warp[w][lane];
      s_warp[w][lane] = tot;
      tot += v;
    }
  }
  __syncthreads();
  const unsigned lt = lanemask_lt();
  int run[kMaxLevels];
#pragma unroll
  for (int l = 0; l < kMaxLevels; ++l) run[l] = s_prefix[l] + s_warp[warp][l];
  int nrun = s_prefix[kNodes] + s_warp[warp][kNodes];
#pragma unroll 1
  for (int k = 0; k < kScanItems; ++k) {
    const int g = g0 + 32 * k;
    const int sp = s_span[k][tid];
    // the cell payloads (read before the ranks are formed)
    int pf = 0, pe = 0;
    unsigned long long key = 0ull;
    if (sp >= 0) {
      pf = ws.gfirst[g];
      pe = ws.glast[g] + 1;
      key = ws.ukey[g];
    }
    unsigned sm, lm;
    int lam;
    masks(sp, sm, lm, lam);
    const int ek = __popc(lm);
    int inc = ek;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    const int s_from = M - (nrun + inc - ek);  // S(g): cells added by groups >= g
    nrun += __shfl_sync(0xffffffffu, inc, 31);
    int excl[kMaxLevels + 1];
#pragma unroll
    for (int l = 0; l < kMaxLevels; ++l) {
      excl[l] = 0;
      if (l < wlo || l > whi) continue;  // warp-uniform
      const unsigned bal = __ballot_sync(0xffffffffu, (sm >> l) & 1u);
      excl[l] = run[l] + __popc(bal & lt);
      run[l] += __popc(bal);
    }
    excl[kMaxLevels] = 0;
    if (lam == 0) continue;
    int bleaf = -1;
    const int delta = (sp & 255) - 1;
#pragma unroll
    for (int l = 0; l < kMaxLevels; ++l) {
      if (l < wlo || l > whi) continue;
      const int started = (int)((sm >> l) & 1u);
      if (started) {
        const int b = s_base[l] + excl[l];
        // the parent: started by this group too, or (one level below the
        // common levels) the last cell started before it at level delta
        const int parent = (l == 0) ? -1 : s_base[l - 1] + excl[l - 1] - (l - 1 == delta ? 1 : 0);
        if (b < s_base[l + 1]) {
          ws.lo_first[b] = make_int4(pf, s_base[l + 1] + excl[l + 1], s_from, parent);
          ws.lo_arrive[b] = 0;
        } else {
          record_error(sc, kStageLayout, 1);
        }
        if (l == lam) bleaf = b;
      }
      if (((lm >> l) & 1u) && l < lam) {
        const int b = s_base[l] + excl[l] + started - 1;
        const int pre = s_from - lam + l - 1;
        if (b >= s_base[l] && b < s_base[l + 1] && pre >= 0 && pre < M)
          ws.lo_last[b] = make_int4(pe, pre, (int)(unsigned)key, (int)(unsigned)(key >> 32));
        else
          record_error(sc, kStageLayout, 1);
      }
    }
    // the leaf (level lambda, preorder index S(g) - 1), finished by lo_upsweep_kernel
    if (bleaf < 0 || s_from < 1 || s_from > M) {
      record_error(sc, kStageLayout, 1);
      continue;
    }
    ws.lo_gleaf[g] = make_int2(bleaf, s_from);
  }
}

// The target-group rule (group_mark_kernel) for one cell of the level-order
// octree: whether the cell is one group by itself (then it marks its first
// particle only as a whole system); otherwise an occupied leaf marks slices
// of group_max and any other cell the starts of its children's runs
// (children in octant order, packed greedily when the cell is compact).
__device__ __forceinline__ bool lo_whole_group(const Workspace &ws, int level, int np, bool leaf) {
  const bool virt = level < ws.sys_levels;  // children are other systems
  const bool compact = !virt && (leaf || np <= 1 || level - ws.sys_levels >= ws.group_depth);
  return !virt && np <= ws.group_max && compact;
}

// The occupied leaf of group g: mass and centre of mass of the group's
// particles in sorted order (octree_physics.cu:95-154), its LevelNode and its
// target-group marks; the traversal records (at preorder index S(g) - 1, no
// child list: neither walk reads one for an occupied leaf) are the caller's
// (lo_emit_records with c).  Returns the leaf's level-order index, or false
// on inconsistent input.
__device__ __forceinline__ bool lo_leaf_cell(const Workspace &ws, int g, int M, int &bleaf, LoCell &c) {
  DevScalars *sc = ws.sc;
  const int2 lf = ws.lo_gleaf[g];
  const int pf = ws.gfirst[g], pe = ws.glast[g] + 1;
  c.key = ws.ukey[g];
  c.level = (ws.gspan[g] >> 8) & 255;
  bleaf = lf.x;
  c.skip = lf.y;
  c.pre = c.skip - 1;
  c.pf = pf;
  c.pe = pe;
  c.nk = 0;
  c.leaf = true;
  if (bleaf < 0 || bleaf >= M || c.pre < 0 || c.pre >= M || pf < 0 || pe <= pf || pe > ws.n || c.level < 1 ||
      c.level > ws.max_level) {
    record_error(sc, kStageLayout, 1);
    return false;
  }
  double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
  for (int i = pf; i < pe; ++i) {
    const double4 q = ws.pm4[i];
    tm = __dadd_rn(tm, q.w);
    wx = __fma_rn(q.w, q.x, wx);
    wy = __fma_rn(q.w, q.y, wy);
    wz = __fma_rn(q.w, q.z, wz);
  }
  lo_emit_node(ws, bleaf, tm, wx, wy, wz, c);
  const int np = pe - pf;
  if (lo_whole_group(ws, c.level, np, true)) {
    if (c.level == ws.sys_levels) ws.tflag[pf] = 1;
  } else {
    for (int k = 0; k < np; k += ws.group_max) ws.tflag[pf + k] = 1;
  }
  return true;
}

// A child's LevelNode, written earlier in the same kernel by another thread
// of the upward pass: read from L2 (ld.global.cg), never from a stale L1 line.
__device__ __forceinline__ LevelNode ld_level_node_cg(const LevelNode *p) {
  const double2 *d = reinterpret_cast<const double2 *>(p);
  const double2 lo = __ldcg(d), hi = __ldcg(d + 1);
  const int4 t = __ldcg(reinterpret_cast<const int4 *>(p) + 2);
  LevelNode r;
  r.a = make_double4(lo.x, lo.y, hi.x, hi.y);
  r.pre = t.x;
  r.np = t.y;
  r.first = t.z;
  r.leaf = t.w;
  return r;
}

// One internal cell b of a level (children in the next level's range
// [hi, end); f, q its lo_first and lo_last entries): mass and centre of mass
// from the children's records in octant order (octree_physics.cu:156-245),
// the child list, the target-group marks and its LevelNode; the traversal
// records are the caller's (lo_emit_records with c).  Returns false on
// inconsistent input.
__device__ __forceinline__ bool lo_level_cell(const Workspace &ws, int level, int b, int hi, int end, int M,
                                              const int4 &f, const int4 &q, int next_first_child, LoCell &c) {
  DevScalars *sc = ws.sc;
  const int c0 = f.y;
  const int c1 = (b + 1 < hi) ? next_first_child : end;
  const int pf = f.x, skip = f.z, pe = q.x, pre = q.y;
  if (pre < 0 || pre >= M || skip <= pre + 1 || skip > M || c0 < hi || c1 <= c0 || c1 > end || c1 - c0 > 8 ||
      pf < 0 || pe <= pf || pe > ws.n) {
    record_error(sc, kStageLayout, 1);
    return false;
  }
  const int nk = c1 - c0;
  c.level = level;
  c.pre = pre;
  c.skip = skip;
  c.pf = pf;
  c.pe = pe;
  c.nk = nk;
  c.leaf = false;
  c.key = (unsigned long long)(unsigned)q.z | ((unsigned long long)(unsigned)q.w << 32);
  // children in visit order: octant 7 -> 0, the children in descending key order
  int *kids = ws.node_kids + (size_t)pre * 8;
  // target groups (group_mark_kernel's rule): a whole system that is one
  // group, else the starts of the children's runs
  const int np = pe - pf;
  const bool whole = lo_whole_group(ws, level, np, false);
  if (whole && level == ws.sys_levels) ws.tflag[pf] = 1;
  const bool virt = level < ws.sys_levels;
  const bool merge = !virt && (np <= 1 || level - ws.sys_levels >= ws.group_depth);
  const bool child_compact_level = level + 1 - ws.sys_levels >= ws.group_depth;
  int run = 0;
  double tm = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (c0 + j < c1) {
      const LevelNode ch = ld_level_node_cg(ws.lo_node + c0 + j);
      const double cm = ch.a.w;
      tm = __dadd_rn(tm, cm);
      wx = __fma_rn(cm, ch.a.x, wx);
      wy = __fma_rn(cm, ch.a.y, wy);
      wz = __fma_rn(cm, ch.a.z, wz);
      kids[nk - 1 - j] = ch.pre;
      if (!whole) {
        if (virt) run = 0;
        const int cp = ch.np;
        if (cp > ws.group_max || !(ch.leaf || cp <= 1 || child_compact_level)) {
          run = 0;  // the child splits itself
        } else {
          if (!merge || run == 0 || run + cp > ws.group_max) {
            if (ch.first >= 0 && ch.first < ws.n) ws.tflag[ch.first] = 1;
            run = 0;
          }
          run += cp;
        }
      }
    }
  }
  for (int j = nk; j < 8; ++j) kids[j] = -1;
  lo_emit_node(ws, b, tm, wx, wy, wz, c);
  return true;
}

// Atomic addition with acquire-release semantics at GPU scope: the adding
// thread's earlier writes are visible to any thread that later observes the
// sum, and this thread's later reads see what the earlier adders wrote.
__device__ __forceinline__ unsigned atomic_add_acq_rel(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// A cell's arrival at its parent p.  The children of p are the consecutive
// cells [c0, c1) of the next level; child c adds 1, plus c if it is the first
// child (the cell before it has another parent) and 2^31 - (c + 1) if it is
// the last.  The counter (zeroed by lo_rank) reaches 2^31 exactly when every
// child has added, (c1 - c0) + c0 + 2^31 - c1, and stays below it before, so
// the child count is not needed to detect the last arrival.  Returns whether
// this cell arrived last.
__device__ __forceinline__ bool lo_arrive_last(const Workspace &ws, int c, int p, int left_parent, int right_parent,
                                               bool &bad) {
  constexpr unsigned kDone = 0x80000000u;
  const unsigned add = 1u + (left_parent != p ? (unsigned)c : 0u) + (right_parent != p ? kDone - (unsigned)(c + 1) : 0u);
  const unsigned sum = atomic_add_acq_rel(reinterpret_cast<unsigned *>(ws.lo_arrive) + p, add) + add;
  bad = sum > kDone;
  return sum == kDone;
}

// The whole upward pass in one launch, with arrival counters instead of one
// launch per level: a thread finishes the leaf of group g, then climbs.  At
// each parent it counts itself in (lo_arrive_last: an acquire-release atomic
// publishes the child's LevelNode); the child that arrives last finishes the
// parent from its children's records and climbs on, the others stop.  Every
// cell is finished exactly once, after all of its children, with the same
// arithmetic in the same child order as a level-by-level pass.  No thread
// ever waits: a climb ends at the root, at a parent that other children
// still owe, or at the first inconsistency.  What keeps the climb short: a
// cell's traversal records (geometry, acceptance radius, the scattered
// writes at the preorder index) are written after its arrival, not before;
// the parent's entries are read before the arrival; and a block is one warp
// (32 resident per SM, 64 registers), so a warp whose lanes climb far holds
// no other warp's slot.  Measured at 2^20 particles (kernel time, cold):
// 174 us before these three changes, 152 us after (blocks of 64: 156 us,
// of 256: 170 us; one-warp blocks at 78 registers, 26 per SM: 163 us).
constexpr int kUpsweepBlock = 32;

template <int kRecords>
__global__ void __launch_bounds__(kUpsweepBlock, 32) lo_upsweep_kernel(Workspace ws, double theta) {
  __shared__ int s_g, s_m;
  __shared__ int s_base[kMaxLevels + 2];
  DevScalars *sc = ws.sc;
  if (threadIdx.x < kMaxLevels + 2) s_base[threadIdx.x] = sc->level_base[threadIdx.x];
  if (threadIdx.x == 0) {
    const int g = sc->n_groups, m = sc->n_nodes;
    s_g = (!sc->error && g > 0 && g <= ws.n && m > 0) ? g : 0;
    s_m = m;
  }
  __syncthreads();
  const int G = s_g, M = s_m;
  if (G > 0 && s_base[kMaxLevels] != M) {
    if (threadIdx.x == 0) record_error(sc, kStageLayout, 1);
    return;
  }
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    int cell;
    LoCell c;
    if (!lo_leaf_cell(ws, g, M, cell, c)) continue;
    // the cell's parent and its neighbours' (which children are first and last)
    int level = c.level;
    int p = ws.lo_first[cell].w;
    int pl = cell > s_base[level] ? ws.lo_first[cell - 1].w : -1;
    int pr = cell + 1 < s_base[level + 1] ? ws.lo_first[cell + 1].w : -1;
    while (true) {
      if (level == 0) {
        if (!lo_emit_records<kRecords>(ws, theta, c)) record_error(sc, kStageGeometry, 2);
        break;
      }
      const int lv = level - 1;
      const int lo = s_base[lv], hi = s_base[lv + 1], end = s_base[lv + 2];
      if (p < lo || p >= hi) {
        record_error(sc, kStageLayout, 1);
        break;
      }
      // the parent's entries, its successor's first child and the parents of
      // its neighbours: read-only here, loaded before the arrival
      const int4 f = ws.lo_first[p];
      const int4 q = ws.lo_last[p];
      const int4 fr = (p + 1 < hi) ? ws.lo_first[p + 1] : make_int4(0, end, 0, -1);
      const int npl = p > lo ? ws.lo_first[p - 1].w : -1;
      bool bad;
      const bool last = lo_arrive_last(ws, cell, p, pl, pr, bad);
      if (!lo_emit_records<kRecords>(ws, theta, c)) record_error(sc, kStageGeometry, 2);
      if (!last) {
        if (bad) record_error(sc, kStageLayout, 1);
        break;
      }
      if (!lo_level_cell(ws, lv, p, hi, end, M, f, q, fr.y, c)) break;
      cell = p;
      level = lv;
      p = f.w;
      pl = npl;
      pr = fr.w;
    }
  }
}

// Target-group starts on the level-order octree: group_mark_kernel's rule
// with the children read as consecutive entries of the next level.
__global__ void __launch_bounds__(kBlock) lo_group_mark_kernel(Workspace ws) {
  __shared__ int s_base[kMaxLevels + 2];
  __shared__ int s_m;
  DevScalars *sc = ws.sc;
  if (threadIdx.x < kMaxLevels + 2) s_base[threadIdx.x] = sc->level_base[threadIdx.x];
  if (threadIdx.x == 0) {
    const int m = sc->n_nodes;
    s_m = (sc->error || m != sc->level_base[kMaxLevels]) ? 0 : m;
  }
  __syncthreads();
  const int M = s_m, gmax = ws.group_max, n = ws.n;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < M; b += gridDim.x * blockDim.x) {
    int level = 0;
    while (level + 1 < kMaxLevels && b >= s_base[level + 1]) ++level;
    const LevelNode nd = ws.lo_node[b];
    const int np = nd.np;
    const bool virt = level < ws.sys_levels;  // children are other systems
    const bool compact = !virt && (nd.leaf || np <= 1 || level - ws.sys_levels >= ws.group_depth);
    if (!virt && np <= gmax && compact) {
      // a whole system that is one group
      if (level == ws.sys_levels && np > 0 && nd.first >= 0 && nd.first < n) ws.tflag[nd.first] = 1;
      continue;
    }
    if (nd.leaf) {
      // an occupied leaf with more than group_max coincident-key particles
      for (int k = 0; k < np; k += gmax)
        if (nd.first + k >= 0 && nd.first + k < n) ws.tflag[nd.first + k] = 1;
      continue;
    }
    const int hi = s_base[level + 1], end = s_base[level + 2];
    const int c0 = ws.lo_first[b].y;
    const int c1 = (b + 1 < hi) ? ws.lo_first[b + 1].y : end;
    if (c0 < hi || c1 < c0 || c1 > end || c1 - c0 > 8) {
      record_error(sc, kStageLayout, 1);
      continue;
    }
    const bool merge = compact;  // split for its count only
    int run = 0;
    for (int c = c0; c < c1; ++c) {
      const LevelNode ch = ws.lo_node[c];
      const int cp = ch.np;
      if (virt) run = 0;
      const bool ccompact = ch.leaf || cp <= 1 || level + 1 - ws.sys_levels >= ws.group_depth;
      if (cp > gmax || !ccompact) {
        // the child splits itself
        run = 0;
        continue;
      }
      if (!merge || run == 0 || run + cp > gmax) {
        if (ch.first >= 0 && ch.first < n) ws.tflag[ch.first] = 1;
        run = 0;
      }
      run += cp;
    }
  }
}

// The node-cache table: the cells of levels 0..kTopDepth with their mixed
// records and child lists (read back from the step's records).
__global__ void __launch_bounds__(128) lo_top_kernel(Workspace ws) {
  __shared__ int s_base[kTopDepth + 3];
  __shared__ int s_ok;
  DevScalars *sc = ws.sc;
  if (threadIdx.x < kTopDepth + 3) s_base[threadIdx.x] = sc->level_base[threadIdx.x];
  if (threadIdx.x == 0) {
    const int m = sc->n_nodes;
    s_ok = !sc->error && m > 0 && sc->level_base[kTopDepth + 2] <= m;
  }
  __syncthreads();
  if (!s_ok) return;
  const int count = min(s_base[kTopDepth + 1], kTopMax);
  for (int q = threadIdx.x; q < count; q += blockDim.x) {
    const int level = (q < s_base[1]) ? 0 : (q < s_base[2] ? 1 : 2);
    const LevelNode nd = ws.lo_node[q];
    const int c0 = ws.lo_first[q].y;
    const int c1 = (q + 1 < s_base[level + 1]) ? ws.lo_first[q + 1].y : s_base[level + 2];
    TopNode t;
    t.rec = ws.node_m[nd.pre];
    const int4 *k = reinterpret_cast<const int4 *>(ws.node_kids + (size_t)nd.pre * 8);
    const int4 k0 = k[0], k1 = k[1];
    t.kids[0] = k0.x; t.kids[1] = k0.y; t.kids[2] = k0.z; t.kids[3] = k0.w;
    t.kids[4] = k1.x; t.kids[5] = k1.y; t.kids[6] = k1.z; t.kids[7] = k1.w;
    t.first_child = c0;
    t.nchild = nd.leaf ? 0 : min(max(c1 - c0, 0), 8);
    t.level = level;
    t.pad = 0;
    ws.top[q] = t;
  }
}

// Reset of the counters the reference-numbered octree build uses, so that it
// can run after a level-order build of the same step (tree export).
__global__ void reference_octree_reset_kernel(DevScalars *sc) {
  if (threadIdx.x == 0) {
    sc->tile_counter[kTilePlan] = 0;
    sc->tile_counter[kTileEnds] = 0;
    for (int l = 0; l < kMaxLevels; ++l) sc->level_count[l] = 0;
  }
}

// Reset the traversal counters and target-group scan state so the groups can
// be rebuilt with another group size on an unchanged tree.
__global__ void retarget_reset_kernel(DevScalars *sc) {
  if (threadIdx.x == 0) {
    sc->work_counter = 0;
    sc->n_tgroups = 0;
    sc->tile_counter[kTileTargetGroups] = 0;
    sc->interactions = 0;
    sc->mac_tests = 0;
    sc->stack_overflow = 0;
  }
}

// Self-test of the bounded waits: one warp looks back from tile 1 while tile
// 0 never publishes; the spin limit must end the wait and record the
// timeout code instead of hanging.
__global__ void lookback_probe_kernel(unsigned long long *status, DevScalars *sc) {
  if (threadIdx.x < 32) (void)warp_lookback(status, 1, 1ull, sc, kStageGroups);
}

// Sorted packed pairs -> caller key / index arrays (sort-only entry point).
__global__ void __launch_bounds__(kBlock) split_pairs_kernel(const unsigned long long *pairs, int n, int shift,
                                                             uint32_t *keys, uint32_t *idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long pr = pairs[i];
    keys[i] = (uint32_t)(pr >> shift);
    idx[i] = (uint32_t)(pr & ((1ull << shift) - 1ull));
  }
}

// Reference-layout keys only (no particles): used by the function-level
// topology entry points.
// --------------------------------------- function-level stage helpers ---

// 32-bit keys or prefixes to the workspace's 64-bit layout and back.
__global__ void __launch_bounds__(kBlock) widen_u32_kernel(const uint32_t *in, int n, unsigned long long *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i];
}
__global__ void __launch_bounds__(kBlock) narrow_u64_kernel(const unsigned long long *in, int n, uint32_t *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (uint32_t)in[i];
}
// Group sizes from the first and last sorted index of each group.
__global__ void __launch_bounds__(kBlock) group_counts_kernel(Workspace ws) {
  const int g = ws.sc->error ? 0 : ws.sc->n_groups;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g; i += gridDim.x * blockDim.x)
    ws.gcount[i] = ws.glast[i] - ws.gfirst[i] + 1;
}
// Sizes a stage works on, known to the caller (G groups, M octree nodes).
__global__ void set_counts_kernel(DevScalars *sc, int g, int m) {
  if (threadIdx.x == 0) {
    sc->n_groups = g;
    sc->n_nodes = m;
  }
}
// Particle data gathered by the sorted indices, as octree_physics.cu:95-154
// reads it (an index outside the particle array is its error 3).
__global__ void __launch_bounds__(kBlock) gather_sorted_kernel(Workspace ws, const uint32_t *idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ws.n; i += gridDim.x * blockDim.x) {
    const uint32_t k = idx[i];
    if (k >= (uint32_t)ws.n) {
      record_error(ws.sc, kStagePhysics, 3);
      continue;
    }
    ws.pm4[i] = make_double4(ws.x[k], ws.y[k], ws.z[k], ws.m[k]);
  }
}

// The same gather from the kick-drift pass's {x, y, z} records: two reads
// per particle instead of four (random reads are what this gather waits on).
__global__ void __launch_bounds__(kBlock) gather_pos4_kernel(Workspace ws) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ws.n; i += gridDim.x * blockDim.x) {
    const uint32_t k = ws.idx[i];
    if (k >= (uint32_t)ws.n) {
      record_error(ws.sc, kStagePhysics, 3);
      continue;
    }
    const double4 q = ws.pos4[k];
    ws.pm4[i] = make_double4(q.x, q.y, q.z, ws.m[k]);
  }
}

__global__ void __launch_bounds__(kBlock) pack_keys_kernel(Workspace ws, const uint32_t *keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ws.n; i += gridDim.x * blockDim.x)
    ws.pairs_a[i] = ((unsigned long long)keys[i] << ws.pack_shift) | (unsigned)i;
}

}  // namespace

// ------------------------------------------------------------ launches ---

cudaError_t launch_step_reset(Workspace &ws, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  reset_sys_kernel<<<(6 * ws.n_systems + 255) / 256, 256, 0, s>>>(ws.sys_bb, ws.n_systems);
  count_launches(2);
  cudaError_t e = cudaMemsetAsync(ws.digit_hist, 0, sizeof(uint32_t) * kMaxSortPasses * 256, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.sort_status, 0, sizeof(uint32_t) * (size_t)ws.sort_passes * ws.sort_tiles * 256, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.scan_status, 0,
                      sizeof(unsigned long long) * (size_t)(3 * ws.scan_tiles_n + ws.scan_tiles_r), s);
  if (e != cudaSuccess) return e;
  if (ws.tflag) {
    e = cudaMemsetAsync(ws.tflag, 0, (size_t)ws.n, s);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t launch_kd_bbox(Workspace &ws, double dt, int do_kd, cudaStream_t s) {
  int blocks = (ws.n + kBlock - 1) / kBlock;
  const int cap = grid_for(ws, 4);
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  kd_bbox_kernel<<<blocks, kBlock, 0, s>>>(ws, dt, do_kd);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_morton_sort_groups(Workspace &ws, cudaStream_t s, int part) {
  // the passes alternate between the two pair buffers
  unsigned long long *sorted = (ws.sort_passes & 1) ? ws.pairs_b : ws.pairs_a;
  if (part != 2) {
    int blocks = (ws.n + kBlock - 1) / kBlock;
    const int cap = grid_for(ws, 4);
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    encode_kernel<<<blocks, kBlock, 0, s>>>(ws);
    unsigned long long *src = ws.pairs_a, *dst = ws.pairs_b;
    for (int p = 0; p < ws.sort_passes; ++p) {
      onesweep_kernel<<<ws.sort_tiles, kSortThreads, 0, s>>>(
          src, dst, ws.n, p, ws.pack_shift + 8 * p, ws.digit_hist,
          ws.sort_status + (size_t)p * ws.sort_tiles * 256, ws.sc);
      unsigned long long *t = src;
      src = dst;
      dst = t;
    }
    count_launches(1 + ws.sort_passes);
  }
  if (part != 1) {
    groups_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws, sorted, 0);
    // the first reader of the masses: the Morton-order gather, one particle
    // per thread so that every thread's four loads are in flight at once
    const int blocks = (ws.n + kBlock - 1) / kBlock > 0 ? (ws.n + kBlock - 1) / kBlock : 1;
    if (ws.pos4)
      gather_pos4_kernel<<<blocks, kBlock, 0, s>>>(ws);
    else
      gather_sorted_kernel<<<blocks, kBlock, 0, s>>>(ws, ws.idx);
    count_launches(2);
  }
  return cudaGetLastError();
}

// Karras tree .. traversal layout in the reference's octree numbering.
static cudaError_t launch_reference_body(Workspace &ws, double theta, cudaStream_t s) {
  const int grid = grid_for(ws, 8);
  karras_kernel<<<grid, kBlock, 0, s>>>(ws);
  plan_kernel<<<ws.scan_tiles_r, kScanThreads, 0, s>>>(ws);
  octree_clear_kernel<<<grid, kBlock, 0, s>>>(ws);
  materialize_kernel<<<grid, kBlock, 0, s>>>(ws);
  node_init_kernel<true, true><<<grid, kBlock, 0, s>>>(ws);
  level_bin_kernel<<<grid, kBlock, 0, s>>>(ws);
  for (int level = ws.max_level; level >= 0; --level)
    propagate_level_kernel<<<level_grid(ws, level), kBlock, 0, s>>>(ws, level);
  cudaError_t e = cudaMemsetAsync(ws.pends, 0, sizeof(int) * (size_t)ws.n, s);
  if (e != cudaSuccess) return e;
  ends_hist_kernel<<<grid, kBlock, 0, s>>>(ws);
  ends_scan_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws);
  preorder_kernel<<<grid, kBlock, 0, s>>>(ws);
  layout_kernel<<<grid, kBlock, 0, s>>>(ws, theta);
  count_launches(10 + (ws.max_level + 1));
  return cudaGetLastError();
}

cudaError_t launch_tree(Workspace &ws, double theta, cudaStream_t s) {
  cudaError_t e = launch_reference_body(ws, theta, s);
  if (e != cudaSuccess) return e;
  const int grid = grid_for(ws, 8);
  group_mark_kernel<<<grid, kBlock, 0, s>>>(ws);
  group_scan_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_level_order_tree(Workspace &ws, double theta, cudaStream_t s) {
  if (!ws.lo_tiles) return cudaErrorInvalidValue;
  lo_span_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws);
  lo_tile_scan_kernel<<<1, 32 * kLevelOrderChannels, 0, s>>>(ws);
  if (ws.records == kRecordsMixed)
    lo_rank_kernel<kRecordsMixed><<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws, theta);
  else if (ws.records == kRecordsFp64)
    lo_rank_kernel<kRecordsFp64><<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws, theta);
  else
    lo_rank_kernel<kRecordsFp64 | kRecordsMixed><<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws, theta);
  // leaves and every internal cell in one launch (arrival counters), one
  // thread per group in one-warp blocks (a resident grid taking groups
  // grid-stride measured slower: 267 against 174 us at 2^20 particles)
  const int want = (ws.n + kUpsweepBlock - 1) / kUpsweepBlock;
  const int up_grid = want > 0 ? want : 1;
  if (ws.records == kRecordsMixed)
    lo_upsweep_kernel<kRecordsMixed><<<up_grid, kUpsweepBlock, 0, s>>>(ws, theta);
  else if (ws.records == kRecordsFp64)
    lo_upsweep_kernel<kRecordsFp64><<<up_grid, kUpsweepBlock, 0, s>>>(ws, theta);
  else
    lo_upsweep_kernel<kRecordsFp64 | kRecordsMixed><<<up_grid, kUpsweepBlock, 0, s>>>(ws, theta);
  if (ws.top && (ws.records & kRecordsMixed) && ws.n_systems == 1) {
    lo_top_kernel<<<1, 128, 0, s>>>(ws);
    count_launches(1);
  }
  // target-group marks were set by the upward pass
  group_scan_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws);
  count_launches(5);
  return cudaGetLastError();
}

cudaError_t launch_octree(Workspace &ws, double theta, cudaStream_t s) {
  return ws.level_order ? launch_level_order_tree(ws, theta, s) : launch_tree(ws, theta, s);
}

cudaError_t launch_reference_octree(Workspace &ws, double theta, cudaStream_t s) {
  reference_octree_reset_kernel<<<1, 32, 0, s>>>(ws.sc);
  count_launches(1);
  cudaError_t e = cudaMemsetAsync(ws.scan_status + ws.scan_tiles_n, 0,
                                  sizeof(unsigned long long) * (size_t)ws.scan_tiles_r, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.scan_status + 2 * ws.scan_tiles_n + ws.scan_tiles_r, 0,
                      sizeof(unsigned long long) * (size_t)ws.scan_tiles_n, s);
  if (e != cudaSuccess) return e;
  return launch_reference_body(ws, theta, s);
}

cudaError_t launch_morton_sort_only(Workspace &ws, uint32_t *keys, uint32_t *idx, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  reset_sys_kernel<<<1, 32, 0, s>>>(ws.sys_bb, ws.n_systems);
  cudaError_t e = cudaMemsetAsync(ws.digit_hist, 0, sizeof(uint32_t) * kMaxSortPasses * 256, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.sort_status, 0, sizeof(uint32_t) * (size_t)ws.sort_passes * ws.sort_tiles * 256, s);
  if (e != cudaSuccess) return e;
  int blocks = (ws.n + kBlock - 1) / kBlock;
  const int cap = grid_for(ws, 4);
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  kd_bbox_kernel<<<blocks, kBlock, 0, s>>>(ws, 0.0, 0);
  encode_kernel<<<blocks, kBlock, 0, s>>>(ws);
  unsigned long long *src = ws.pairs_a, *dst = ws.pairs_b;
  for (int p = 0; p < ws.sort_passes; ++p) {
    onesweep_kernel<<<ws.sort_tiles, kSortThreads, 0, s>>>(
        src, dst, ws.n, p, ws.pack_shift + 8 * p, ws.digit_hist,
        ws.sort_status + (size_t)p * ws.sort_tiles * 256, ws.sc);
    unsigned long long *t = src;
    src = dst;
    dst = t;
  }
  split_pairs_kernel<<<blocks, kBlock, 0, s>>>(src, ws.n, ws.pack_shift, keys, idx);
  count_launches(4 + ws.sort_passes);
  return cudaGetLastError();
}

cudaError_t launch_lookback_probe(unsigned long long *status, DevScalars *sc, cudaStream_t s) {
  lookback_probe_kernel<<<1, 32, 0, s>>>(status, sc);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_retarget(Workspace &ws, cudaStream_t s) {
  retarget_reset_kernel<<<1, 32, 0, s>>>(ws.sc);
  cudaError_t e = cudaMemsetAsync(ws.tflag, 0, (size_t)ws.n, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.scan_status + ws.scan_tiles_n + ws.scan_tiles_r, 0,
                      sizeof(unsigned long long) * (size_t)ws.scan_tiles_n, s);
  if (e != cudaSuccess) return e;
  const int grid = grid_for(ws, 8);
  if (ws.level_order)
    lo_group_mark_kernel<<<grid, kBlock, 0, s>>>(ws);
  else
    group_mark_kernel<<<grid, kBlock, 0, s>>>(ws);
  group_scan_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws);
  count_launches(3);
  return cudaGetLastError();
}

cudaError_t launch_groups_from_keys(Workspace &ws, const uint32_t *sorted_keys, cudaStream_t s) {
  pack_keys_kernel<<<grid_for(ws, 4), kBlock, 0, s>>>(ws, sorted_keys);
  groups_kernel<<<ws.scan_tiles_n, kScanThreads, 0, s>>>(ws, ws.pairs_a, 0);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_topology(Workspace &ws, cudaStream_t s) {
  const int grid = grid_for(ws, 8);
  karras_kernel<<<grid, kBlock, 0, s>>>(ws);
  plan_kernel<<<ws.scan_tiles_r, kScanThreads, 0, s>>>(ws);
  octree_clear_kernel<<<grid, kBlock, 0, s>>>(ws);
  materialize_kernel<<<grid, kBlock, 0, s>>>(ws);
  count_launches(4);
  return cudaGetLastError();
}

// ------------------------------------------- function-level stages ----
// Each runs one stage of the build on a workspace whose arrays alias the
// caller's (see the C ABI's function-level entry points).

cudaError_t launch_bbox_only(Workspace &ws, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  reset_sys_kernel<<<1, 32, 0, s>>>(ws.sys_bb, ws.n_systems);
  count_launches(2);
  return launch_kd_bbox(ws, 0.0, 0, s);
}

cudaError_t launch_morton_sort_box(Workspace &ws, uint32_t *keys, uint32_t *idx, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  cudaError_t e = cudaMemsetAsync(ws.digit_hist, 0, sizeof(uint32_t) * kMaxSortPasses * 256, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(ws.sort_status, 0, sizeof(uint32_t) * (size_t)ws.sort_passes * ws.sort_tiles * 256, s);
  if (e != cudaSuccess) return e;
  e = launch_morton_sort_groups(ws, s, 1);
  if (e != cudaSuccess) return e;
  const unsigned long long *sorted = (ws.sort_passes & 1) ? ws.pairs_b : ws.pairs_a;
  split_pairs_kernel<<<grid_for(ws, 4), kBlock, 0, s>>>(sorted, ws.n, ws.pack_shift, keys, idx);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_leaf_groups(Workspace &ws, const uint32_t *sorted_keys, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  cudaError_t e = cudaMemsetAsync(ws.scan_status, 0, sizeof(unsigned long long) * (size_t)ws.scan_tiles_n, s);
  if (e != cudaSuccess) return e;
  e = launch_groups_from_keys(ws, sorted_keys, s);
  if (e != cudaSuccess) return e;
  group_counts_kernel<<<grid_for(ws, 4), kBlock, 0, s>>>(ws);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_plan_only(Workspace &ws, int g, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  set_counts_kernel<<<1, 32, 0, s>>>(ws.sc, g, 0);
  cudaError_t e = cudaMemsetAsync(ws.scan_status, 0,
                                  sizeof(unsigned long long) * (size_t)(ws.scan_tiles_n + ws.scan_tiles_r), s);
  if (e != cudaSuccess) return e;
  plan_kernel<<<ws.scan_tiles_r, kScanThreads, 0, s>>>(ws);
  count_launches(3);
  return cudaGetLastError();
}

cudaError_t launch_octree_only(Workspace &ws, int g, int m, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  set_counts_kernel<<<1, 32, 0, s>>>(ws.sc, g, m);
  const int grid = grid_for(ws, 8);
  octree_clear_kernel<<<grid, kBlock, 0, s>>>(ws);
  materialize_kernel<<<grid, kBlock, 0, s>>>(ws);
  count_launches(4);
  return cudaGetLastError();
}

cudaError_t launch_geometry_only(Workspace &ws, int m, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  set_counts_kernel<<<1, 32, 0, s>>>(ws.sc, 0, m);
  node_init_kernel<true, false><<<grid_for(ws, 8), kBlock, 0, s>>>(ws);
  count_launches(3);
  return cudaGetLastError();
}

cudaError_t launch_mass_only(Workspace &ws, const uint32_t *idx, int m, cudaStream_t s) {
  reset_scalars_kernel<<<1, 32, 0, s>>>(ws.sc);
  set_counts_kernel<<<1, 32, 0, s>>>(ws.sc, 0, m);
  const int grid = grid_for(ws, 8);
  gather_sorted_kernel<<<grid_for(ws, 4), kBlock, 0, s>>>(ws, idx);
  node_init_kernel<false, true><<<grid, kBlock, 0, s>>>(ws);
  level_bin_kernel<<<grid, kBlock, 0, s>>>(ws);
  for (int level = ws.max_level; level >= 0; --level)
    propagate_level_kernel<<<level_grid(ws, level), kBlock, 0, s>>>(ws, level);
  count_launches(6 + ws.max_level + 1);
  return cudaGetLastError();
}

cudaError_t launch_widen_u32(const uint32_t *in, int n, unsigned long long *out, cudaStream_t s) {
  int blocks = (n + kBlock - 1) / kBlock;
  blocks = blocks < 1 ? 1 : (blocks > 4096 ? 4096 : blocks);
  widen_u32_kernel<<<blocks, kBlock, 0, s>>>(in, n, out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_narrow_u64(const unsigned long long *in, int n, uint32_t *out, cudaStream_t s) {
  int blocks = (n + kBlock - 1) / kBlock;
  blocks = blocks < 1 ? 1 : (blocks > 4096 ? 4096 : blocks);
  narrow_u64_kernel<<<blocks, kBlock, 0, s>>>(in, n, out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_radix_tree_only(const uint32_t *keys, int n, int *left, int *right, int *rfirst,
                                   int *rlast, int *plen, int *parent, cudaStream_t s) {
  int blocks = (n + kBlock - 1) / kBlock;
  if (blocks < 1) blocks = 1;
  if (blocks > 4096) blocks = 4096;
  karras_only_kernel<<<blocks, kBlock, 0, s>>>(keys, n, left, right, rfirst, rlast, plen, parent);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace nbb
