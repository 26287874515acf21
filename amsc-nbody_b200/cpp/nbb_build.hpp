// nbb_build.hpp -- the reference's function-level build API with its own
// names, over the C ABI of libnbb.so (include/nbb.h).
//
// A translation unit written against sytrams/AMSC-Nbody's build headers --
// include/globalbounding.hpp (Bbox), src/morton.hpp (MortonKeys),
// src/morton_leaf_groups.hpp, src/tree_types.hpp + src/tree_builder.hpp,
// src/radix_to_octree.hpp, src/octree_types.hpp + src/octree_builder.hpp,
// src/octree_geometry.hpp, src/octree_physics.hpp, src/barnes_hut.hpp and
// src/device_buffer.hpp -- includes this header instead and keeps its calls:
//
//   Bbox box(d_x, d_y, d_z, n);
//   MortonKeys morton(d_x, d_y, d_z, n, box);
//   allocateMortonLeafGroups(groups, n);
//   buildMortonLeafGroups(groups, morton.keys_device_data(), n);
//   allocateTree(tree, groups.nGroups);
//   buildTreeFromMortonGroups(tree, groups);
//   allocateRadixToOctreePlan(plan, 2 * groups.nGroups - 1);
//   buildRadixToOctreePlan(plan, tree, groups);
//   allocateOctreeTopology(octree, plan.nOctreeNodes);
//   buildSparseOctreeTopology(octree, tree, groups, plan);
//   allocateOctreeGeometry(octree);        computeOctreeGeometry(octree, box);
//   allocateOctreePhysicalData(octree);    computeOctreeMassAndCenterOfMass(...);
//   computeBarnesHutAcceleration(octree, morton.indices_device_data(), ...);
//
// Every buffer is device memory owned by a DeviceBuffer, every call is
// synchronous and throws the reference's exception classes with its messages
// (through nbb::throwStatus).  Results equal the reference's bit for bit.
// Not provided: the radix tree's own centre-of-mass kernels
// (computeCenterOfMass / computeGroupedCenterOfMass), which the reference's
// step does not use; allocateTree allocates their arrays all the same.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>

#include "nbb.h"
#include "nbb_simulation.hpp"

// src/device_buffer.hpp:12-123: an owning device array.
template <typename T>
class DeviceBuffer {
 public:
  DeviceBuffer() noexcept = default;
  explicit DeviceBuffer(std::size_t count) { allocate(count); }
  ~DeviceBuffer() noexcept { reset(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&other) noexcept
      : data_(std::exchange(other.data_, nullptr)), size_(std::exchange(other.size_, 0)) {}
  DeviceBuffer &operator=(DeviceBuffer &&other) noexcept {
    if (this == &other) return *this;
    reset();
    data_ = std::exchange(other.data_, nullptr);
    size_ = std::exchange(other.size_, 0);
    return *this;
  }
  void allocate(std::size_t count) {
    if (data_ != nullptr) throw std::logic_error("DeviceBuffer is already allocated");
    if (count == 0) return;
    if (count > std::numeric_limits<std::size_t>::max() / sizeof(T))
      throw std::overflow_error("DeviceBuffer allocation size overflows");
    void *p = nullptr;
    if (nbb_device_alloc(&p, count * sizeof(T)) != NBB_OK)
      throw std::runtime_error(std::string("DeviceBuffer cudaMalloc failed: ") + nbb_last_error_message());
    data_ = static_cast<T *>(p);
    size_ = count;
  }
  void reset() noexcept {
    if (data_ != nullptr) (void)nbb_device_free(data_);
    data_ = nullptr;
    size_ = 0;
  }
  [[nodiscard]] T *data() noexcept { return data_; }
  [[nodiscard]] const T *data() const noexcept { return data_; }
  [[nodiscard]] std::size_t size() const noexcept { return size_; }
  [[nodiscard]] bool empty() const noexcept { return size_ == 0; }
  void swap(DeviceBuffer &other) noexcept {
    std::swap(data_, other.data_);
    std::swap(size_, other.size_);
  }

 private:
  T *data_ = nullptr;
  std::size_t size_ = 0;
};

// include/globalbounding.hpp:7-36: the cube {centre, side} around the
// particles, kept on the device.
struct BboxValues {
  double center_x;
  double center_y;
  double center_z;
  double side;
};

class Bbox {
 public:
  static constexpr std::size_t value_count = 4;
  Bbox() : centre_and_side_(value_count) {
    // a negative side marks a box that was never computed
    const double init[value_count] = {0.0, 0.0, 0.0, -1.0};
    nbb::throwStatus(nbb_memcpy(centre_and_side_.data(), init, sizeof(init), 0));
  }
  Bbox(const double *d_x, const double *d_y, const double *d_z, std::size_t count) : Bbox() {
    recompute(d_x, d_y, d_z, count);
  }
  void recompute(const double *d_x, const double *d_y, const double *d_z, std::size_t count) {
    nbb::throwStatus(nbb_bbox(d_x, d_y, d_z, count, centre_and_side_.data()));
  }
  [[nodiscard]] BboxValues values() const {
    double v[value_count];
    nbb::throwStatus(nbb_memcpy(v, centre_and_side_.data(), sizeof(v), 1));
    return {v[0], v[1], v[2], v[3]};
  }
  [[nodiscard]] const double *device_data() const noexcept { return centre_and_side_.data(); }
  [[nodiscard]] double *device_data() noexcept { return centre_and_side_.data(); }

 private:
  DeviceBuffer<double> centre_and_side_;
};

// src/morton.hpp: 30-bit Morton keys of the positions against a box, sorted
// ascending with their particle indices (stable).
using MortonKey = std::uint32_t;
using QuantisedCoordinate = std::uint32_t;
using ParticleIndex = std::uint32_t;

class MortonKeys {
 public:
  MortonKeys(const double *x, const double *y, const double *z, std::size_t count) {
    validate(x, y, z, count);
    const Bbox boundingBox(x, y, z, count);
    build(x, y, z, count, boundingBox);
  }
  MortonKeys(const double *x, const double *y, const double *z, std::size_t count, const Bbox &boundingBox) {
    validate(x, y, z, count);
    build(x, y, z, count, boundingBox);
  }
  [[nodiscard]] const MortonKey *keys_device_data() const noexcept { return keys_.data(); }
  [[nodiscard]] MortonKey *keys_device_data() noexcept { return keys_.data(); }
  [[nodiscard]] const ParticleIndex *indices_device_data() const noexcept { return indices_.data(); }
  [[nodiscard]] ParticleIndex *indices_device_data() noexcept { return indices_.data(); }
  [[nodiscard]] std::size_t size() const noexcept { return keys_.size(); }

 private:
  // gpu/cuda_kernels/morton.cu:34-60
  static void validate(const double *x, const double *y, const double *z, std::size_t count) {
    if (count == 0) throw std::invalid_argument("Cannot compute Morton keys for an empty particle set");
    if (x == nullptr || y == nullptr || z == nullptr)
      throw std::invalid_argument("Morton coordinate device pointers must not be null");
    if (count > std::numeric_limits<ParticleIndex>::max())
      throw std::overflow_error("Particle count exceeds the Morton index representation");
  }
  void build(const double *x, const double *y, const double *z, std::size_t count, const Bbox &boundingBox) {
    keys_.allocate(count);
    indices_.allocate(count);
    nbb::throwStatus(nbb_morton_keys(x, y, z, count, boundingBox.device_data(), keys_.data(), indices_.data()));
  }
  DeviceBuffer<MortonKey> keys_;
  DeviceBuffer<ParticleIndex> indices_;
};

// src/morton_leaf_groups.hpp:8-41: runs of equal sorted keys.
struct MortonLeafGroupsView {
  int nParticles = 0;
  int nGroups = 0;
  int capacity = 0;
  const std::uint32_t *uniqueKeys = nullptr;
  const int *firstParticle = nullptr;
  const int *particleCount = nullptr;
};

struct MortonLeafGroups {
  int nParticles = 0;
  int nGroups = 0;
  int capacity = 0;
  DeviceBuffer<std::uint32_t> uniqueKeys;
  DeviceBuffer<int> firstParticle;
  DeviceBuffer<int> particleCount;
  [[nodiscard]] MortonLeafGroupsView view() const noexcept {
    return {nParticles, nGroups, capacity, uniqueKeys.data(), firstParticle.data(), particleCount.data()};
  }
};

inline void freeMortonLeafGroups(MortonLeafGroups &groups) noexcept { groups = MortonLeafGroups{}; }

inline void allocateMortonLeafGroups(MortonLeafGroups &groups, int capacity) {
  if (capacity <= 0) throw std::invalid_argument("MortonLeafGroups capacity must be positive");
  if (!groups.uniqueKeys.empty() || !groups.firstParticle.empty() || !groups.particleCount.empty())
    throw std::logic_error("MortonLeafGroups memory is already allocated");
  const auto size = static_cast<std::size_t>(capacity);
  try {
    groups.uniqueKeys.allocate(size);
    groups.firstParticle.allocate(size);
    groups.particleCount.allocate(size);
  } catch (...) {
    freeMortonLeafGroups(groups);
    throw;
  }
  groups.capacity = capacity;
  groups.nParticles = 0;
  groups.nGroups = 0;
}

inline void buildMortonLeafGroups(MortonLeafGroups &groups, const std::uint32_t *d_sortedKeys, int nParticles) {
  if (nParticles <= 0) throw std::invalid_argument("buildMortonLeafGroups requires nParticles >= 1");
  if (nParticles > groups.capacity) throw std::invalid_argument("nParticles exceeds MortonLeafGroups capacity");
  if (d_sortedKeys == nullptr) throw std::invalid_argument("d_sortedKeys must not be null");
  if (groups.uniqueKeys.data() == nullptr || groups.firstParticle.data() == nullptr ||
      groups.particleCount.data() == nullptr)
    throw std::logic_error("MortonLeafGroups memory has not been allocated");
  groups.nParticles = 0;
  groups.nGroups = 0;
  int g = 0;
  nbb::throwStatus(nbb_leaf_groups(d_sortedKeys, nParticles, groups.uniqueKeys.data(), groups.firstParticle.data(),
                                   groups.particleCount.data(), &g));
  groups.nParticles = nParticles;
  groups.nGroups = g;
}

// src/tree_types.hpp:48-109: the Karras radix tree over the unique keys
// (internal nodes first, leaves numbered nLeaves .. in parent indices).
struct Tree {
  int nLeaves = 0;
  int nInternalNodes = 0;
  DeviceBuffer<int> left;
  DeviceBuffer<int> right;
  DeviceBuffer<int> parent;
  DeviceBuffer<int> rangeFirst;
  DeviceBuffer<int> rangeLast;
  DeviceBuffer<int> prefixLength;
  DeviceBuffer<double> mass;
  DeviceBuffer<double> comX;
  DeviceBuffer<double> comY;
  DeviceBuffer<double> comZ;
  DeviceBuffer<int> visitCount;
};

inline void freeTree(Tree &tree) noexcept { tree = Tree{}; }

inline void allocateTreeTopology(Tree &tree, int N) {
  if (N <= 0) throw std::invalid_argument("N must be positive");
  if (!tree.left.empty() || !tree.right.empty() || !tree.parent.empty() || !tree.rangeFirst.empty() ||
      !tree.rangeLast.empty() || !tree.prefixLength.empty() || !tree.mass.empty() || !tree.comX.empty() ||
      !tree.comY.empty() || !tree.comZ.empty() || !tree.visitCount.empty())
    throw std::logic_error("Tree memory is already allocated");
  const auto internal = static_cast<std::size_t>(N - 1);
  const auto total = static_cast<std::size_t>(N) * 2 - 1;
  try {
    if (N > 1) {
      tree.left.allocate(internal);
      tree.right.allocate(internal);
      tree.rangeFirst.allocate(internal);
      tree.rangeLast.allocate(internal);
      tree.prefixLength.allocate(internal);
    }
    tree.parent.allocate(total);
  } catch (...) {
    freeTree(tree);
    throw;
  }
  tree.nLeaves = N;
  tree.nInternalNodes = N - 1;
}

inline void allocateTree(Tree &tree, int N) {
  allocateTreeTopology(tree, N);
  const auto internal = static_cast<std::size_t>(N - 1);
  const auto total = static_cast<std::size_t>(N) * 2 - 1;
  try {
    if (N > 1) tree.visitCount.allocate(internal);
    tree.mass.allocate(total);
    tree.comX.allocate(total);
    tree.comY.allocate(total);
    tree.comZ.allocate(total);
  } catch (...) {
    freeTree(tree);
    throw;
  }
}

inline void buildTree(Tree &tree, const std::uint32_t *d_sortedKeys, int N) {
  if (N <= 0) throw std::invalid_argument("buildTree requires N >= 1");
  if (N != tree.nLeaves) throw std::invalid_argument("buildTree N does not match allocated tree size");
  if (tree.parent.data() == nullptr ||
      (N > 1 && (tree.left.data() == nullptr || tree.right.data() == nullptr || tree.rangeFirst.data() == nullptr ||
                 tree.rangeLast.data() == nullptr || tree.prefixLength.data() == nullptr)))
    throw std::logic_error("Tree memory has not been allocated");
  if (d_sortedKeys == nullptr) throw std::invalid_argument("d_sortedKeys must not be null");
  nbb::throwStatus(nbb_radix_tree_device(d_sortedKeys, N, tree.left.data(), tree.right.data(),
                                         tree.rangeFirst.data(), tree.rangeLast.data(), tree.prefixLength.data(),
                                         tree.parent.data()));
}

inline void buildTreeFromMortonGroups(Tree &tree, const MortonLeafGroups &groups) {
  if (groups.nParticles <= 0) throw std::invalid_argument("MortonLeafGroups has no particles");
  if (groups.nGroups <= 0) throw std::invalid_argument("MortonLeafGroups has no groups");
  if (groups.nGroups > groups.nParticles || groups.nParticles > groups.capacity)
    throw std::logic_error("MortonLeafGroups metadata is inconsistent");
  if (groups.uniqueKeys.data() == nullptr) throw std::logic_error("MortonLeafGroups uniqueKeys is not allocated");
  if (tree.nLeaves != groups.nGroups)
    throw std::invalid_argument("Tree leaf count does not match Morton group count");
  buildTree(tree, groups.uniqueKeys.data(), groups.nGroups);
}

// src/radix_to_octree.hpp:10-65: per radix node, its octree level and the
// octree nodes its edge generates.
constexpr int kMortonDimensions = 3;
constexpr int kMortonBitsPerAxis = 10;
constexpr int kMortonSpatialBits = kMortonDimensions * kMortonBitsPerAxis;
constexpr int kMortonStorageBits = 32;
constexpr int kMortonPaddingBits = kMortonStorageBits - kMortonSpatialBits;
constexpr int kOctreeMaxLevel = kMortonBitsPerAxis;
constexpr std::uint32_t kMortonSpatialMask = 0x3FFFFFFFu;

struct RadixToOctreePlan {
  int nRadixNodes = 0;
  int nOctreeNodes = 0;
  DeviceBuffer<int> radixLevel;
  DeviceBuffer<int> edgeNodeCount;
  DeviceBuffer<int> edgeNodeOffset;
};

inline void freeRadixToOctreePlan(RadixToOctreePlan &plan) noexcept { plan = RadixToOctreePlan{}; }

inline void allocateRadixToOctreePlan(RadixToOctreePlan &plan, int nRadixNodes) {
  if (nRadixNodes <= 0) throw std::invalid_argument("nRadixNodes must be positive");
  if (!plan.radixLevel.empty() || !plan.edgeNodeCount.empty() || !plan.edgeNodeOffset.empty())
    throw std::logic_error("RadixToOctreePlan memory is already allocated");
  const auto count = static_cast<std::size_t>(nRadixNodes);
  try {
    plan.radixLevel.allocate(count);
    plan.edgeNodeCount.allocate(count);
    plan.edgeNodeOffset.allocate(count);
  } catch (...) {
    freeRadixToOctreePlan(plan);
    throw;
  }
  plan.nRadixNodes = nRadixNodes;
  plan.nOctreeNodes = 0;
}

inline void buildRadixToOctreePlan(RadixToOctreePlan &plan, const Tree &radixTree, const MortonLeafGroups &groups) {
  if (radixTree.nLeaves <= 0) throw std::invalid_argument("The radix tree has no leaves");
  if (groups.nGroups != radixTree.nLeaves)
    throw std::invalid_argument("Morton group count does not match radix-tree leaf count");
  if (groups.uniqueKeys.data() == nullptr) throw std::logic_error("Morton unique keys are not allocated");
  if (radixTree.parent.data() == nullptr) throw std::logic_error("Radix-tree parent array is not allocated");
  if (radixTree.nLeaves > 1 && radixTree.prefixLength.data() == nullptr)
    throw std::logic_error("Radix-tree prefix metadata is not allocated");
  if (plan.nRadixNodes != 2 * radixTree.nLeaves - 1)
    throw std::invalid_argument("RadixToOctreePlan size does not match the radix tree");
  if (plan.radixLevel.data() == nullptr || plan.edgeNodeCount.data() == nullptr || plan.edgeNodeOffset.data() == nullptr)
    throw std::logic_error("RadixToOctreePlan memory is not allocated");
  plan.nOctreeNodes = 0;
  int m = 0;
  nbb::throwStatus(nbb_octree_plan(groups.uniqueKeys.data(), radixTree.nLeaves, radixTree.prefixLength.data(),
                                   radixTree.parent.data(), plan.radixLevel.data(), plan.edgeNodeCount.data(),
                                   plan.edgeNodeOffset.data(), &m));
  plan.nOctreeNodes = m;
}

// src/octree_types.hpp:73-178: the sparse octree, node-major children
// (children[node * 8 + octant], -1 empty), root 0.
struct Octree {
  int nParticles = 0;
  int nLeaves = 0;
  int nNodes = 0;
  int root = -1;
  DeviceBuffer<int> children;
  DeviceBuffer<int> parent;
  DeviceBuffer<int> level;
  DeviceBuffer<std::uint32_t> prefix;
  DeviceBuffer<int> firstParticle;
  DeviceBuffer<int> particleCount;
  DeviceBuffer<double> mass;
  DeviceBuffer<double> comX;
  DeviceBuffer<double> comY;
  DeviceBuffer<double> comZ;
  DeviceBuffer<double> centerX;
  DeviceBuffer<double> centerY;
  DeviceBuffer<double> centerZ;
  DeviceBuffer<double> halfSize;
  DeviceBuffer<int> pendingChildren;
  DeviceBuffer<int> childCount;
};

inline void freeOctree(Octree &octree) noexcept { octree = Octree{}; }

inline void allocateOctreeTopology(Octree &octree, int nNodes) {
  if (nNodes <= 0) throw std::invalid_argument("Octree node count must be positive");
  if (!octree.children.empty() || !octree.parent.empty() || !octree.level.empty() || !octree.prefix.empty() ||
      !octree.firstParticle.empty() || !octree.particleCount.empty() || !octree.mass.empty() ||
      !octree.comX.empty() || !octree.comY.empty() || !octree.comZ.empty() || !octree.centerX.empty() ||
      !octree.centerY.empty() || !octree.centerZ.empty() || !octree.halfSize.empty() ||
      !octree.pendingChildren.empty() || !octree.childCount.empty())
    throw std::logic_error("Octree memory is already allocated");
  const auto count = static_cast<std::size_t>(nNodes);
  try {
    octree.children.allocate(count * 8);
    octree.parent.allocate(count);
    octree.level.allocate(count);
    octree.prefix.allocate(count);
    octree.firstParticle.allocate(count);
    octree.particleCount.allocate(count);
  } catch (...) {
    freeOctree(octree);
    throw;
  }
  octree.nNodes = nNodes;
}

inline void buildSparseOctreeTopology(Octree &octree, const Tree &radixTree, const MortonLeafGroups &groups,
                                      const RadixToOctreePlan &plan) {
  if (groups.nGroups <= 0) throw std::invalid_argument("Morton groups are empty");
  if (groups.nGroups != radixTree.nLeaves)
    throw std::invalid_argument("Morton groups and radix tree have different leaf counts");
  if (groups.uniqueKeys.data() == nullptr || groups.firstParticle.data() == nullptr ||
      groups.particleCount.data() == nullptr)
    throw std::logic_error("Morton group arrays are not allocated");
  if (plan.nRadixNodes != 2 * radixTree.nLeaves - 1)
    throw std::invalid_argument("Radix-to-octree plan does not match the radix tree");
  if (plan.nOctreeNodes <= 0) throw std::invalid_argument("Radix-to-octree plan has no octree nodes");
  if (octree.nNodes != plan.nOctreeNodes)
    throw std::invalid_argument("Allocated octree size does not match the construction plan");
  nbb::throwStatus(nbb_octree_topology(groups.uniqueKeys.data(), groups.firstParticle.data(),
                                       groups.particleCount.data(), groups.nGroups, radixTree.rangeFirst.data(),
                                       radixTree.parent.data(), plan.radixLevel.data(), plan.edgeNodeCount.data(),
                                       plan.edgeNodeOffset.data(), octree.nNodes, octree.children.data(),
                                       octree.parent.data(), octree.level.data(), octree.prefix.data(),
                                       octree.firstParticle.data(), octree.particleCount.data()));
  octree.nParticles = groups.nParticles;
  octree.nLeaves = groups.nGroups;
  octree.root = 0;
}

// src/octree_geometry.hpp
inline void allocateOctreeGeometry(Octree &octree) {
  if (octree.nNodes <= 0) throw std::invalid_argument("Octree topology must be allocated before geometry");
  if (octree.level.data() == nullptr || octree.prefix.data() == nullptr)
    throw std::logic_error("Octree topology arrays required for geometry are not allocated");
  if (!octree.centerX.empty() || !octree.centerY.empty() || !octree.centerZ.empty() || !octree.halfSize.empty())
    throw std::logic_error("Octree geometry is already allocated");
  const auto count = static_cast<std::size_t>(octree.nNodes);
  try {
    octree.centerX.allocate(count);
    octree.centerY.allocate(count);
    octree.centerZ.allocate(count);
    octree.halfSize.allocate(count);
  } catch (...) {
    octree.centerX.reset();
    octree.centerY.reset();
    octree.centerZ.reset();
    octree.halfSize.reset();
    throw;
  }
}

inline void computeOctreeGeometry(Octree &octree, const Bbox &boundingBox) {
  if (octree.nNodes <= 0 || octree.root != 0) throw std::logic_error("Octree topology is not valid");
  if (octree.level.data() == nullptr || octree.prefix.data() == nullptr)
    throw std::logic_error("Octree topology arrays required for geometry are not allocated");
  if (octree.centerX.data() == nullptr || octree.centerY.data() == nullptr || octree.centerZ.data() == nullptr ||
      octree.halfSize.data() == nullptr)
    throw std::logic_error("Octree geometry arrays are not allocated");
  nbb::throwStatus(nbb_octree_geometry(octree.nNodes, octree.level.data(), octree.prefix.data(),
                                       boundingBox.device_data(), octree.centerX.data(), octree.centerY.data(),
                                       octree.centerZ.data(), octree.halfSize.data()));
}

// src/octree_physics.hpp
inline void allocateOctreePhysicalData(Octree &octree) {
  if (octree.nNodes <= 0) throw std::invalid_argument("Octree topology must be allocated first");
  if (!octree.mass.empty() || !octree.comX.empty() || !octree.comY.empty() || !octree.comZ.empty() ||
      !octree.pendingChildren.empty() || !octree.childCount.empty())
    throw std::logic_error("Octree physical data is already allocated");
  const auto count = static_cast<std::size_t>(octree.nNodes);
  try {
    octree.mass.allocate(count);
    octree.comX.allocate(count);
    octree.comY.allocate(count);
    octree.comZ.allocate(count);
    octree.pendingChildren.allocate(count);
    octree.childCount.allocate(count);
  } catch (...) {
    octree.mass.reset();
    octree.comX.reset();
    octree.comY.reset();
    octree.comZ.reset();
    octree.pendingChildren.reset();
    octree.childCount.reset();
    throw;
  }
}

inline void computeOctreeMassAndCenterOfMass(Octree &octree, const std::uint32_t *d_sortedIndices, const double *d_mass,
                                             const double *d_positionX, const double *d_positionY,
                                             const double *d_positionZ) {
  if (octree.nParticles <= 0 || octree.nLeaves <= 0 || octree.nNodes <= 0 || octree.root != 0)
    throw std::logic_error("Octree topology is not valid");
  if (octree.children.data() == nullptr || octree.parent.data() == nullptr || octree.firstParticle.data() == nullptr ||
      octree.particleCount.data() == nullptr)
    throw std::logic_error("Octree topology arrays are not allocated");
  if (octree.mass.data() == nullptr || octree.comX.data() == nullptr || octree.comY.data() == nullptr ||
      octree.comZ.data() == nullptr || octree.pendingChildren.data() == nullptr || octree.childCount.data() == nullptr)
    throw std::logic_error("Octree physical arrays are not allocated");
  nbb::throwStatus(nbb_octree_mass(octree.nNodes, octree.nParticles, octree.children.data(), octree.level.data(),
                                   octree.firstParticle.data(), octree.particleCount.data(), d_sortedIndices, d_mass,
                                   d_positionX, d_positionY, d_positionZ, octree.childCount.data(),
                                   octree.mass.data(), octree.comX.data(), octree.comY.data(), octree.comZ.data()));
}

// src/barnes_hut.hpp:21 on the Octree structure.
inline void computeBarnesHutAcceleration(const Octree &octree, const std::uint32_t *d_sortedIndices,
                                         const double *d_mass, const double *d_positionX,
                                         const double *d_positionY, const double *d_positionZ,
                                         double *d_accelerationX, double *d_accelerationY,
                                         double *d_accelerationZ, std::size_t particleCount,
                                         const BarnesHutParameters &parameters,
                                         BarnesHutParticleOrder particleOrder = BarnesHutParticleOrder::original) {
  // gpu/cuda_kernels/barnes_hut.cu:328-345
  if (octree.nParticles <= 0 || octree.nNodes <= 0 || octree.root != 0)
    throw std::logic_error("Octree is not valid for Barnes-Hut traversal");
  if (particleCount != static_cast<std::size_t>(octree.nParticles))
    throw std::invalid_argument("Particle count does not match the octree");
  if (octree.children.data() == nullptr || octree.parent.data() == nullptr || octree.firstParticle.data() == nullptr ||
      octree.particleCount.data() == nullptr)
    throw std::logic_error("Octree topology arrays required for traversal are not allocated");
  if (octree.mass.data() == nullptr || octree.comX.data() == nullptr || octree.comY.data() == nullptr ||
      octree.comZ.data() == nullptr)
    throw std::logic_error("Octree physical data is not allocated");
  if (octree.centerX.data() == nullptr || octree.centerY.data() == nullptr || octree.centerZ.data() == nullptr ||
      octree.halfSize.data() == nullptr)
    throw std::logic_error("Octree geometry is not allocated");
  const nbb_octree_view view{octree.nNodes,        octree.nParticles,     octree.children.data(),
                             octree.parent.data(), octree.firstParticle.data(), octree.particleCount.data(),
                             octree.mass.data(),   octree.comX.data(),    octree.comY.data(),
                             octree.comZ.data(),   octree.centerX.data(), octree.centerY.data(),
                             octree.centerZ.data(), octree.halfSize.data()};
  computeBarnesHutAcceleration(view, d_sortedIndices, d_mass, d_positionX, d_positionY, d_positionZ,
                               d_accelerationX, d_accelerationY, d_accelerationZ, particleCount, parameters,
                               particleOrder);
}
