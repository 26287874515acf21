/*
 * nbb_oracle.h -- CPU restatement of the AMSC-Nbody Barnes-Hut step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg (and
 * its reference arm) may load it.  The product library never links it and has
 * no CPU fallback.
 *
 * Every function restates one stage of the reference pipeline statement by
 * statement; the reference file:line each follows is cited beside it (paths
 * are relative to the sytrams/AMSC-Nbody project root).
 *
 * Floating-point convention shared with the CUDA plain-FP64 path: products
 * that the reference accumulates into a sum are fused explicitly with fma(),
 * every other operation is a separately rounded IEEE operation (the library
 * is compiled with -ffp-contract=off), sqrt and division are correctly
 * rounded.  With identical summation order this makes the CPU and GPU plain
 * paths bit-identical.
 */
#ifndef NBB_ORACLE_H
#define NBB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: 0 ok; negative = host-side validation error (the reference
 * throws std::invalid_argument / std::domain_error); positive = the
 * reference's device error code of the failing stage. */
enum {
  ORC_OK = 0,
  ORC_EINVAL = -1,   /* std::invalid_argument */
  ORC_EDOMAIN = -2,  /* std::domain_error (non-finite positions) */
  ORC_ECAP = -3      /* caller buffer too small */
};

/* globalbounding.cu:94-144 -- out = {centre_x, centre_y, centre_z, side}. */
int orc_bbox(size_t n, const double *x, const double *y, const double *z,
             double out[4]);

/* morton.cu:98-139,160-219 + 160-225 -- keys and the stable (key, index) sort. */
int orc_morton(size_t n, const double *x, const double *y, const double *z,
               const double box[4], uint32_t *keys, uint32_t *idx);

/* morton_leaf_groups.cu:58-103 -- run-length encode + exclusive scan.
 * Returns G (>0) or a negative status. */
int orc_leaf_groups(int n, const uint32_t *sorted_keys, uint32_t *uniq,
                    int *first, int *count);

/* tree_builder.cu:9-113 + 303-352 -- Karras radix tree over n keys.
 * left/right/rfirst/rlast/plen have n-1 entries, parent 2n-1. */
int orc_radix_tree(int n, const uint32_t *keys, int *left, int *right,
                   int *rfirst, int *rlast, int *plen, int *parent);

/* radix_to_octree.cu:54-145 + 174-243 -- per radix node octree level, edge
 * node count and their exclusive scan.  *n_octree receives 1 + sum.
 * Returns 0 or the reference's plan error code (1..4). */
int orc_octree_plan(int n_leaves, const uint32_t *uniq, const int *parent,
                    const int *plen, int *level, int *count, int *offset,
                    int *n_octree);

/* octree_builder.cu:49-362 + 254-362 -- materialise the sparse octree.
 * children has 8*m entries. Returns 0 or construction error code (1..7). */
int orc_octree_build(int n_leaves, const uint32_t *uniq, const int *gfirst,
                     const int *gcount, const int *rparent, const int *rfirst,
                     const int *plan_level, const int *plan_count,
                     const int *plan_offset, int m, int *children, int *parent,
                     int *level, uint32_t *prefix, int *first, int *count);

/* octree_geometry.cu:39-102 -- cell centre and half size from the prefix. */
int orc_octree_geometry(int m, const int *level, const uint32_t *prefix,
                        const double box[4], double *cx, double *cy,
                        double *cz, double *half);

/* octree_physics.cu:64-337 -- childCount, leaf mass/COM in sorted order,
 * internal mass/COM summed in octant order 0..7. */
int orc_octree_mass(int m, int n, const int *children, const int *parent,
                    const int *first, const int *count, const uint32_t *idx,
                    const double *pm, const double *px, const double *py,
                    const double *pz, double *mass, double *comx,
                    double *comy, double *comz, int *child_count);

/* barnes_hut.cu:56-322 -- per-target stackless traversal, children visited
 * 7 -> 0.  Particle arrays are in original order (morton_ordered = 0) or
 * already gathered into Morton order (morton_ordered = 1); accelerations are
 * written at the original index.  theta/soft/g validated as
 * barnes_hut.cu:355-363.  n_threads <= 0 uses every available core.
 * interactions (may be NULL) receives the total count of monopole and
 * leaf-pair interactions. */
int orc_bh_accel(int m, int n, const int *children, const int *parent,
                 const int *first, const int *count, const double *mass,
                 const double *comx, const double *comy, const double *comz,
                 const double *cx, const double *cy, const double *cz,
                 const double *half, const uint32_t *idx, const double *pm,
                 const double *px, const double *py, const double *pz,
                 int morton_ordered, double theta, double soft, double g,
                 double *ax, double *ay, double *az, int n_threads,
                 int64_t *interactions);

/* barnes_hut_accuracy_test.cu:101-172 -- FP64 direct summation for the
 * targets listed in `targets` (all n when targets == NULL, n_targets = n).
 * Output i belongs to targets[i]. */
void orc_direct_accel(int n, const double *pm, const double *px,
                      const double *py, const double *pz, int n_targets,
                      const int *targets, double g, double soft, double *ax,
                      double *ay, double *az, int n_threads);

/* integrator.cu:51-106 */
void orc_kick_drift(size_t n, double *x, double *y, double *z, double *vx,
                    double *vy, double *vz, const double *ax, const double *ay,
                    const double *az, double dt);
void orc_kick(size_t n, double *vx, double *vy, double *vz, const double *ax,
              const double *ay, const double *az, double dt);

/* Every intermediate of one spatial rebuild + force evaluation, sized by the
 * caller: n particles, G <= n groups, M <= 10*n+1 octree nodes. */
typedef struct {
  double box[4];
  uint32_t *keys, *idx;                              /* n */
  uint32_t *uniq; int *gfirst, *gcount;              /* n (G used) */
  int *left, *right, *rfirst, *rlast, *plen;         /* n-1 */
  int *rparent;                                      /* 2n-1 */
  int *plan_level, *plan_count, *plan_offset;        /* 2n-1 */
  int m_capacity;
  int *children;                                     /* 8*M */
  int *oparent, *olevel; uint32_t *oprefix;          /* M */
  int *ofirst, *ocount, *child_count;                /* M */
  double *cx, *cy, *cz, *half;                       /* M */
  double *mass, *comx, *comy, *comz;                 /* M */
  double *ax, *ay, *az;                              /* n (may be NULL) */
  int n_groups, n_octree;
  int64_t interactions;
} orc_pipeline_out;

/* simulation.cpp:137-198 -- rebuild the spatial structure from positions and
 * (if ax != NULL) evaluate Barnes-Hut accelerations with Morton-gathered
 * particle data.  Returns 0 or a status (negative host error, or 100*stage +
 * device code with stage 1 plan, 2 octree, 3 geometry, 4 physics,
 * 5 traversal). */
int orc_pipeline(size_t n, const double *m, const double *x, const double *y,
                 const double *z, double theta, double soft, double g,
                 int n_threads, orc_pipeline_out *out);

/* simulation.cpp:78-127 -- initialize() then `steps` calls of step():
 * KD, rebuild, force, K.  State arrays are updated in place; a (3n) holds the
 * last accelerations on return. */
int orc_simulate(size_t n, const double *m, double *x, double *y, double *z,
                 double *vx, double *vy, double *vz, double *ax, double *ay,
                 double *az, double dt, double theta, double soft, double g,
                 int steps, int n_threads);

/* Quantized position frame of the current state (src/streaming/
 * device_capture.cu:27-330 for sampling, bounds and quantization;
 * src/streaming/frame.cpp:68-95, 341-470 for the byte layout).  Samples
 * s = max_particles (0 or more than n: all) particles at source indices
 * (i * n) / s; writes the frame -- a 128-byte (types given) or 120-byte
 * header, 3 x uint16 per sample, then one uint8 type per sample -- into out
 * (capacity cap bytes) and returns its size, or a negative status: -1
 * argument, -2 non-finite sampled position, -3 invalid particle type,
 * -4 bounds not finite, -5 capacity too small. */
long long orc_frame_capture(size_t n, const double *x, const double *y, const double *z,
                            const uint8_t *type, size_t max_particles, uint64_t sequence,
                            uint64_t step, double time, unsigned char *out, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
