// ref_harness.cu -- drives the UNMODIFIED AMSC-Nbody CUDA sources through
// their own public function-level API, for parity fixtures and for timing the
// reference on the same GPU.
//
// TEST INFRASTRUCTURE ONLY: compiled by oracle/Makefile (target `ref`) from
// the reference's sources where they lie, together with this file, into
// oracle/_ref/libnbody_ref.so.  Only tests/golden/make_golden.py, the GPU
// tests and bench.py's reference arm load it.
//
// The call sequence replays the reference's own pipeline:
//   Simulation::rebuildSpatialStructure   (src/simulation.cpp:137-180)
//   Simulation::computeAccelerations      (src/simulation.cpp:182-198)
//   Simulation::initialize / step         (src/simulation.cpp:78-119)
// with an explicit gravitational constant, as the reference's accuracy test
// does (tests/integration/cuda/barnes_hut_accuracy_test.cu:404-711), because
// Simulation itself hard-codes the SI value (src/simulation.cpp:196).
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "barnes_hut.hpp"
#include "globalbounding.hpp"
#include "integrator.hpp"
#include "morton.hpp"
#include "morton_leaf_groups.hpp"
#include "octree_builder.hpp"
#include "octree_geometry.hpp"
#include "octree_physics.hpp"
#include "radix_to_octree.hpp"
#include "simulation_cuda.hpp"
#include "tree_builder.hpp"

namespace {

thread_local std::string g_message;

template <typename T>
void d2h(T *dst, const T *src, std::size_t count) {
  if (dst == nullptr || count == 0) return;
  const cudaError_t e =
      cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

double *raw(thrust::device_vector<double> &v) {
  return thrust::raw_pointer_cast(v.data());
}

struct Spatial {
  MortonLeafGroups groups{};
  Tree tree{};
  RadixToOctreePlan plan{};
  Octree octree{};
  ~Spatial() {
    freeOctree(octree);
    freeRadixToOctreePlan(plan);
    freeTree(tree);
    freeMortonLeafGroups(groups);
  }
};

// src/simulation.cpp:137-165
void rebuild(Spatial &s, const Bbox &box, const MortonKeys &morton,
             const double *dm, const double *dx, const double *dy,
             const double *dz, int n) {
  allocateMortonLeafGroups(s.groups, n);
  buildMortonLeafGroups(s.groups, morton.keys_device_data(), n);
  allocateTreeTopology(s.tree, s.groups.nGroups);
  buildTreeFromMortonGroups(s.tree, s.groups);
  allocateRadixToOctreePlan(s.plan, 2 * s.groups.nGroups - 1);
  buildRadixToOctreePlan(s.plan, s.tree, s.groups);
  allocateOctreeTopology(s.octree, s.plan.nOctreeNodes);
  buildSparseOctreeTopology(s.octree, s.tree, s.groups, s.plan);
  allocateOctreeGeometry(s.octree);
  computeOctreeGeometry(s.octree, box);
  allocateOctreePhysicalData(s.octree);
  computeOctreeMassAndCenterOfMass(s.octree, morton.indices_device_data(), dm,
                                   dx, dy, dz);
}

// src/simulation.cpp:182-198 with an explicit G.
void accelerations(nbody::detail::SimulationDeviceState &state,
                   const Octree &octree, const MortonKeys &morton,
                   const double *dm, const double *dx, const double *dy,
                   const double *dz, std::size_t n, double theta, double soft,
                   double g) {
  nbody::detail::gatherMortonOrderedParticleData(
      state, morton.indices_device_data(), dm, dx, dy, dz, n);
  const auto mp = nbody::detail::mortonOrderedParticles(state);
  const auto out = nbody::detail::nextAcceleration(state);
  computeBarnesHutAcceleration(octree, morton.indices_device_data(), mp.mass,
                               mp.x, mp.y, mp.z, out.x, out.y, out.z, n,
                               BarnesHutParameters{theta, soft, g},
                               BarnesHutParticleOrder::morton);
}

} // namespace

extern "C" {

// Host output buffers, all optional (NULL skips the copy).  Capacities: n
// for per-particle and per-group arrays, 2n for per-radix-node arrays, and
// m_capacity for octree arrays (children: 8*m_capacity).
struct ref_out {
  double box[4];
  uint32_t *keys, *idx;
  uint32_t *uniq;
  int *gfirst, *gcount;
  int *left, *right, *rfirst, *rlast, *plen, *rparent;
  int *plan_level, *plan_count, *plan_offset;
  int m_capacity;
  int *children, *oparent, *olevel;
  uint32_t *oprefix;
  int *ofirst, *ocount, *child_count;
  double *cx, *cy, *cz, *half;
  double *mass, *comx, *comy, *comz;
  double *ax, *ay, *az;
  int n_groups, n_octree;
};

const char *ref_last_error(void) { return g_message.c_str(); }

// One rebuild + force evaluation, every intermediate copied to the host.
int ref_pipeline(std::size_t n, const double *m, const double *x,
                 const double *y, const double *z, double theta, double soft,
                 double g, ref_out *o) {
  try {
    thrust::device_vector<double> dm(m, m + n), dx(x, x + n), dy(y, y + n),
        dz(z, z + n);
    const Bbox box(raw(dx), raw(dy), raw(dz), n);
    const BboxValues bv = box.values();
    o->box[0] = bv.center_x;
    o->box[1] = bv.center_y;
    o->box[2] = bv.center_z;
    o->box[3] = bv.side;
    const MortonKeys morton(raw(dx), raw(dy), raw(dz), n, box);
    Spatial s;
    rebuild(s, box, morton, raw(dm), raw(dx), raw(dy), raw(dz),
            static_cast<int>(n));
    const int gcount = s.groups.nGroups;
    const int mcount = s.octree.nNodes;
    o->n_groups = gcount;
    o->n_octree = mcount;
    if (mcount > o->m_capacity) throw std::runtime_error("m_capacity too small");
    d2h(o->keys, morton.keys_device_data(), n);
    d2h(o->idx, morton.indices_device_data(), n);
    d2h(o->uniq, s.groups.uniqueKeys.data(), gcount);
    d2h(o->gfirst, s.groups.firstParticle.data(), gcount);
    d2h(o->gcount, s.groups.particleCount.data(), gcount);
    if (gcount > 1) {
      d2h(o->left, s.tree.left.data(), gcount - 1);
      d2h(o->right, s.tree.right.data(), gcount - 1);
      d2h(o->rfirst, s.tree.rangeFirst.data(), gcount - 1);
      d2h(o->rlast, s.tree.rangeLast.data(), gcount - 1);
      d2h(o->plen, s.tree.prefixLength.data(), gcount - 1);
    }
    d2h(o->rparent, s.tree.parent.data(), 2 * gcount - 1);
    d2h(o->plan_level, s.plan.radixLevel.data(), 2 * gcount - 1);
    d2h(o->plan_count, s.plan.edgeNodeCount.data(), 2 * gcount - 1);
    d2h(o->plan_offset, s.plan.edgeNodeOffset.data(), 2 * gcount - 1);
    d2h(o->children, s.octree.children.data(), 8 * (std::size_t)mcount);
    d2h(o->oparent, s.octree.parent.data(), mcount);
    d2h(o->olevel, s.octree.level.data(), mcount);
    d2h(o->oprefix, s.octree.prefix.data(), mcount);
    d2h(o->ofirst, s.octree.firstParticle.data(), mcount);
    d2h(o->ocount, s.octree.particleCount.data(), mcount);
    d2h(o->child_count, s.octree.childCount.data(), mcount);
    d2h(o->cx, s.octree.centerX.data(), mcount);
    d2h(o->cy, s.octree.centerY.data(), mcount);
    d2h(o->cz, s.octree.centerZ.data(), mcount);
    d2h(o->half, s.octree.halfSize.data(), mcount);
    d2h(o->mass, s.octree.mass.data(), mcount);
    d2h(o->comx, s.octree.comX.data(), mcount);
    d2h(o->comy, s.octree.comY.data(), mcount);
    d2h(o->comz, s.octree.comZ.data(), mcount);
    if (o->ax != nullptr) {
      nbody::detail::SimulationDeviceState *state =
          nbody::detail::createSimulationDeviceState(n);
      try {
        accelerations(*state, s.octree, morton, raw(dm), raw(dx), raw(dy),
                      raw(dz), n, theta, soft, g);
        const auto a = nbody::detail::nextAcceleration(*state);
        d2h(o->ax, a.x, n);
        d2h(o->ay, a.y, n);
        d2h(o->az, a.z, n);
      } catch (...) {
        nbody::detail::destroySimulationDeviceState(state);
        throw;
      }
      nbody::detail::destroySimulationDeviceState(state);
    }
    return 0;
  } catch (const std::exception &e) {
    g_message = e.what();
    return 1;
  }
}

// initialize() then `steps` x step() of src/simulation.cpp:78-119 with an
// explicit G.  State is updated in place; a receives the last acceleration.
// step_ms (optional, `steps` entries) receives each step's CUDA-event time.
int ref_simulate(std::size_t n, const double *m, double *x, double *y,
                 double *z, double *vx, double *vy, double *vz, double *ax,
                 double *ay, double *az, double dt, double theta, double soft,
                 double g, int steps, float *step_ms) {
  nbody::detail::SimulationDeviceState *state = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    thrust::device_vector<double> dm(m, m + n), dx(x, x + n), dy(y, y + n),
        dz(z, z + n), dvx(vx, vx + n), dvy(vy, vy + n), dvz(vz, vz + n);
    state = nbody::detail::createSimulationDeviceState(n);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto rebuild_and_force = [&]() {
      const Bbox box(raw(dx), raw(dy), raw(dz), n);
      const MortonKeys morton(raw(dx), raw(dy), raw(dz), n, box);
      Spatial s;
      rebuild(s, box, morton, raw(dm), raw(dx), raw(dy), raw(dz),
              static_cast<int>(n));
      accelerations(*state, s.octree, morton, raw(dm), raw(dx), raw(dy),
                    raw(dz), n, theta, soft, g);
    };
    rebuild_and_force();
    nbody::detail::swapAccelerationBuffers(*state);
    for (int s = 0; s < steps; ++s) {
      cudaEventRecord(e0);
      const auto cur = nbody::detail::currentAcceleration(*state);
      leapfrogKickDrift(raw(dx), raw(dy), raw(dz), raw(dvx), raw(dvy),
                        raw(dvz), cur.x, cur.y, cur.z, n, dt);
      rebuild_and_force();
      const auto nxt = nbody::detail::nextAcceleration(*state);
      leapfrogKick(raw(dvx), raw(dvy), raw(dvz), nxt.x, nxt.y, nxt.z, n, dt);
      nbody::detail::swapAccelerationBuffers(*state);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      if (step_ms != nullptr) cudaEventElapsedTime(&step_ms[s], e0, e1);
    }
    d2h(x, raw(dx), n);
    d2h(y, raw(dy), n);
    d2h(z, raw(dz), n);
    d2h(vx, raw(dvx), n);
    d2h(vy, raw(dvy), n);
    d2h(vz, raw(dvz), n);
    const auto cur = nbody::detail::currentAcceleration(*state);
    d2h(ax, cur.x, n);
    d2h(ay, cur.y, n);
    d2h(az, cur.z, n);
    nbody::detail::destroySimulationDeviceState(state);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
  } catch (const std::exception &e) {
    g_message = e.what();
    if (state != nullptr) nbody::detail::destroySimulationDeviceState(state);
    if (e0 != nullptr) cudaEventDestroy(e0);
    if (e1 != nullptr) cudaEventDestroy(e1);
    return 1;
  }
}

// Karras tree over caller keys (tree_builder.cu:303-352), for the reference's
// own known-answer inputs.
int ref_radix_tree(int n, const uint32_t *keys, int *left, int *right,
                   int *rfirst, int *rlast, int *plen, int *parent) {
  try {
    thrust::device_vector<uint32_t> dk(keys, keys + n);
    Tree tree{};
    allocateTreeTopology(tree, n);
    buildTree(tree, thrust::raw_pointer_cast(dk.data()), n);
    if (n > 1) {
      d2h(left, tree.left.data(), n - 1);
      d2h(right, tree.right.data(), n - 1);
      d2h(rfirst, tree.rangeFirst.data(), n - 1);
      d2h(rlast, tree.rangeLast.data(), n - 1);
      d2h(plen, tree.prefixLength.data(), n - 1);
    }
    d2h(parent, tree.parent.data(), 2 * n - 1);
    freeTree(tree);
    return 0;
  } catch (const std::exception &e) {
    g_message = e.what();
    return 1;
  }
}

} // extern "C"
