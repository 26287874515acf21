// The reference accuracy harness's call sequence
// (tests/integration/cuda/barnes_hut_accuracy_test.cu:404-711) compiled
// against nbb_build.hpp: Bbox, MortonKeys, allocate/build of the leaf groups,
// radix tree, plan and octree, geometry, mass / centre of mass, then
// computeBarnesHutAcceleration on the Octree for theta 0, 0.3, 0.5, 0.7, 1
// (softening 0.02, G = 1, original particle order).  Device arrays are
// DeviceBuffers filled with nbb_memcpy where the harness uses
// thrust::device_vector.
//
//   build_api_test INPUT OUTPUT
// INPUT: uint64 n, then n doubles each of mass, x, y, z.  OUTPUT: every
// intermediate and the accelerations of each theta (layout in write_output).
// Also checks the reference's argument errors; prints "ok" on success.
#include <array>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nbb_build.hpp"

namespace {

int failures = 0;

template <typename E, typename F>
void expect_throw(F f, const std::string &what) {
  try {
    f();
  } catch (const E &) {
    return;
  } catch (const std::exception &e) {
    std::cerr << "FAILED: " << what << " threw another exception: " << e.what() << '\n';
    ++failures;
    return;
  }
  std::cerr << "FAILED: " << what << " did not throw\n";
  ++failures;
}

template <typename T>
std::vector<T> copyFromDevice(const T *d, std::size_t count) {
  std::vector<T> h(count);
  if (count) nbb::throwStatus(nbb_memcpy(h.data(), d, count * sizeof(T), 1));
  return h;
}

template <typename T>
void put(std::ofstream &out, const std::vector<T> &v) {
  const std::uint64_t count = v.size();
  out.write(reinterpret_cast<const char *>(&count), sizeof(count));
  out.write(reinterpret_cast<const char *>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

struct SpatialResources {
  MortonLeafGroups groups;
  Tree radixTree;
  RadixToOctreePlan plan;
  Octree octree;
  ~SpatialResources() {
    freeOctree(octree);
    freeRadixToOctreePlan(plan);
    freeTree(radixTree);
    freeMortonLeafGroups(groups);
  }
};

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::cerr << "usage: build_api_test INPUT OUTPUT\n";
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  std::uint64_t n64 = 0;
  in.read(reinterpret_cast<char *>(&n64), sizeof(n64));
  const std::size_t particleCount = n64;
  const int particleCountInt = static_cast<int>(particleCount);
  std::array<std::vector<double>, 4> host;
  for (auto &v : host) {
    v.resize(particleCount);
    in.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(particleCount * sizeof(double)));
  }
  if (!in) {
    std::cerr << "short input\n";
    return 2;
  }
  std::array<DeviceBuffer<double>, 4> dev;
  for (int k = 0; k < 4; ++k) {
    dev[k].allocate(particleCount);
    nbb::throwStatus(nbb_memcpy(dev[k].data(), host[k].data(), particleCount * sizeof(double), 0));
  }
  const double *dMass = dev[0].data(), *dX = dev[1].data(), *dY = dev[2].data(), *dZ = dev[3].data();

  // Build exactly the spatial pipeline used by the real simulation.
  Bbox boundingBox(dX, dY, dZ, particleCount);
  MortonKeys morton(dX, dY, dZ, particleCount, boundingBox);
  SpatialResources resources;
  allocateMortonLeafGroups(resources.groups, particleCountInt);
  buildMortonLeafGroups(resources.groups, morton.keys_device_data(), particleCountInt);
  allocateTree(resources.radixTree, resources.groups.nGroups);
  buildTreeFromMortonGroups(resources.radixTree, resources.groups);
  allocateRadixToOctreePlan(resources.plan, 2 * resources.groups.nGroups - 1);
  buildRadixToOctreePlan(resources.plan, resources.radixTree, resources.groups);
  allocateOctreeTopology(resources.octree, resources.plan.nOctreeNodes);
  buildSparseOctreeTopology(resources.octree, resources.radixTree, resources.groups, resources.plan);
  allocateOctreeGeometry(resources.octree);
  computeOctreeGeometry(resources.octree, boundingBox);
  allocateOctreePhysicalData(resources.octree);
  computeOctreeMassAndCenterOfMass(resources.octree, morton.indices_device_data(), dMass, dX, dY, dZ);

  constexpr double gravitationalConstant = 1.0;
  constexpr double softening = 0.02;
  DeviceBuffer<double> dAx(particleCount), dAy(particleCount), dAz(particleCount);
  constexpr std::array<double, 5> thetaValues{0.0, 0.3, 0.5, 0.7, 1.0};

  std::ofstream out(argv[2], std::ios::binary);
  const BboxValues box = boundingBox.values();
  put(out, std::vector<double>{box.center_x, box.center_y, box.center_z, box.side});
  const Octree &o = resources.octree;
  const std::size_t G = static_cast<std::size_t>(resources.groups.nGroups);
  const std::size_t I = G > 1 ? G - 1 : 0, R = 2 * G - 1, M = static_cast<std::size_t>(o.nNodes);
  put(out, copyFromDevice(morton.keys_device_data(), particleCount));
  put(out, copyFromDevice(morton.indices_device_data(), particleCount));
  put(out, copyFromDevice(resources.groups.uniqueKeys.data(), G));
  put(out, copyFromDevice(resources.groups.firstParticle.data(), G));
  put(out, copyFromDevice(resources.groups.particleCount.data(), G));
  put(out, copyFromDevice(resources.radixTree.left.data(), I));
  put(out, copyFromDevice(resources.radixTree.right.data(), I));
  put(out, copyFromDevice(resources.radixTree.rangeFirst.data(), I));
  put(out, copyFromDevice(resources.radixTree.rangeLast.data(), I));
  put(out, copyFromDevice(resources.radixTree.prefixLength.data(), I));
  put(out, copyFromDevice(resources.radixTree.parent.data(), R));
  put(out, copyFromDevice(resources.plan.radixLevel.data(), R));
  put(out, copyFromDevice(resources.plan.edgeNodeCount.data(), R));
  put(out, copyFromDevice(resources.plan.edgeNodeOffset.data(), R));
  put(out, copyFromDevice(o.children.data(), 8 * M));
  put(out, copyFromDevice(o.parent.data(), M));
  put(out, copyFromDevice(o.level.data(), M));
  put(out, copyFromDevice(o.prefix.data(), M));
  put(out, copyFromDevice(o.firstParticle.data(), M));
  put(out, copyFromDevice(o.particleCount.data(), M));
  put(out, copyFromDevice(o.childCount.data(), M));
  put(out, copyFromDevice(o.centerX.data(), M));
  put(out, copyFromDevice(o.centerY.data(), M));
  put(out, copyFromDevice(o.centerZ.data(), M));
  put(out, copyFromDevice(o.halfSize.data(), M));
  put(out, copyFromDevice(o.mass.data(), M));
  put(out, copyFromDevice(o.comX.data(), M));
  put(out, copyFromDevice(o.comY.data(), M));
  put(out, copyFromDevice(o.comZ.data(), M));
  for (const double theta : thetaValues) {
    BarnesHutParameters parameters;
    parameters.theta = theta;
    parameters.softening = softening;
    parameters.gravitationalConstant = gravitationalConstant;
    computeBarnesHutAcceleration(resources.octree, morton.indices_device_data(), dMass, dX, dY, dZ, dAx.data(),
                                 dAy.data(), dAz.data(), particleCount, parameters);
    put(out, copyFromDevice(dAx.data(), particleCount));
    put(out, copyFromDevice(dAy.data(), particleCount));
    put(out, copyFromDevice(dAz.data(), particleCount));
  }

  // the reference's argument errors
  expect_throw<std::invalid_argument>([&] { Bbox b(dX, dY, dZ, 0); }, "empty Bbox");
  expect_throw<std::invalid_argument>([&] { MortonKeys k(dX, dY, dZ, 0); }, "empty MortonKeys");
  expect_throw<std::invalid_argument>([&] { MortonKeys k(nullptr, dY, dZ, 4); }, "null MortonKeys");
  expect_throw<std::invalid_argument>([&] { MortonKeys k(dX, dY, dZ, 4, Bbox{}); }, "uncomputed box");
  expect_throw<std::invalid_argument>([&] { MortonLeafGroups g; allocateMortonLeafGroups(g, 0); },
                                      "zero group capacity");
  expect_throw<std::logic_error>([&] { allocateMortonLeafGroups(resources.groups, 4); }, "groups allocated twice");
  expect_throw<std::invalid_argument>([&] { Tree t; allocateTree(t, 0); }, "empty tree");
  expect_throw<std::invalid_argument>(
      [&] {
        Tree t;
        allocateTree(t, resources.groups.nGroups + 1);
        buildTreeFromMortonGroups(t, resources.groups);
      },
      "tree leaf count mismatch");
  expect_throw<std::invalid_argument>(
      [&] {
        Octree wrong;
        allocateOctreeTopology(wrong, resources.plan.nOctreeNodes + 1);
        buildSparseOctreeTopology(wrong, resources.radixTree, resources.groups, resources.plan);
      },
      "octree size mismatch");
  expect_throw<std::logic_error>(
      [&] {
        Octree empty;
        computeOctreeGeometry(empty, boundingBox);
      },
      "geometry of an empty octree");
  expect_throw<std::invalid_argument>(
      [&] {
        computeBarnesHutAcceleration(resources.octree, morton.indices_device_data(), dMass, dX, dY, dZ, dAx.data(),
                                     dAy.data(), dAz.data(), particleCount + 1, BarnesHutParameters{});
      },
      "particle count mismatch");
  {
    // non-finite positions: std::domain_error from the box
    std::vector<double> bad = host[1];
    bad[particleCount / 2] = std::numeric_limits<double>::quiet_NaN();
    DeviceBuffer<double> dBad(particleCount);
    nbb::throwStatus(nbb_memcpy(dBad.data(), bad.data(), particleCount * sizeof(double), 0));
    expect_throw<std::domain_error>([&] { Bbox b(dBad.data(), dY, dZ, particleCount); }, "non-finite Bbox");
  }
  if (failures) return 1;
  std::cout << "ok\n";
  return 0;
}
