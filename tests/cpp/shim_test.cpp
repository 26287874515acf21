// GPU checks of the C++ layer (nbb_simulation.hpp) with the reference's
// names: state machine and validation of Simulation
// (tests/integration/cuda/simulation_test.cu:115-160), a free particle at
// constant velocity (:162-190) and the leapfrog integrator's analytic
// constant-acceleration result (tests/unit/cuda/integrator_test.cu:181-305).
// Prints "ok" and exits 0 when every check passes.
#include <cuda_runtime.h>

#include <cmath>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "nbb_simulation.hpp"

namespace {

int failures = 0;

void check(bool cond, const std::string &what) {
  if (!cond) {
    std::cerr << "FAILED: " << what << '\n';
    ++failures;
  }
}

template <typename E, typename F>
void expect_throw(F f, const std::string &what) {
  try {
    f();
    check(false, what + " did not throw");
  } catch (const E &) {
  } catch (const std::exception &e) {
    check(false, what + " threw the wrong type: " + e.what());
  }
}

Particles one() { return Particles({1.0}, {0.5}, {-1.0}, {2.0}, {0.1}, {0.2}, {-0.3}); }

std::vector<double> host(const double *d, std::size_t n) {
  std::vector<double> h(n);
  cudaMemcpy(h.data(), d, n * 8, cudaMemcpyDeviceToHost);
  return h;
}

}  // namespace

int main() {
  const double nan = std::numeric_limits<double>::quiet_NaN();
  for (const SimulationConfig bad : {SimulationConfig{0.0, 0.5, 0.01}, SimulationConfig{-1.0, 0.5, 0.01},
                                     SimulationConfig{nan, 0.5, 0.01}, SimulationConfig{1.0, -0.1, 0.01},
                                     SimulationConfig{1.0, nan, 0.01}, SimulationConfig{1.0, 0.5, -0.01},
                                     SimulationConfig{1.0, 0.5, nan}})
    expect_throw<std::invalid_argument>([&] { Simulation s(one(), bad); }, "invalid configuration");
  {
    Simulation sim(one(), {0.25, 0.5, 0.01});
    expect_throw<std::logic_error>([&] { sim.step(); }, "step before initialize");
    expect_throw<std::logic_error>([&] { sim.run(1); }, "run before initialize");
    sim.initialize();
    check(sim.time() == 0.0 && sim.stepNumber() == 0, "initialize does not advance");
    expect_throw<std::logic_error>([&] { sim.initialize(); }, "second initialize");
  }
  {
    Simulation sim(one(), {0.25, 0.6, 0.03});
    sim.initialize();
    sim.run(4);
    const DeviceParticlesView v = sim.particles();
    const auto x = host(v.x, 1), y = host(v.y, 1), z = host(v.z, 1), vx = host(v.vx, 1);
    check(std::fabs(x[0] - 0.6) < 1e-12 && std::fabs(y[0] + 0.8) < 1e-12 && std::fabs(z[0] - 1.7) < 1e-12,
          "free particle position");
    check(vx[0] == 0.1, "free particle velocity");
    check(sim.time() == 1.0 && sim.stepNumber() == 4, "time and step number");
  }
  {
    double *d = nullptr;
    cudaMalloc(&d, 9 * sizeof(double));
    const double h[9] = {1.0, -2.0, 3.0, 4.0, 5.0, -6.0, 2.0, -4.0, 1.0};
    cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    const double dt = 0.25;
    leapfrogKickDrift(d, d + 1, d + 2, d + 3, d + 4, d + 5, d + 6, d + 7, d + 8, 1, dt);
    leapfrogKick(d + 3, d + 4, d + 5, d + 6, d + 7, d + 8, 1, dt);
    const auto r = host(d, 9);
    check(std::fabs(r[0] - (1.0 + 4.0 * dt + dt * dt)) < 1e-14, "leapfrog x");
    check(std::fabs(r[3] - (4.0 + 2.0 * dt)) < 1e-14, "leapfrog vx");
    expect_throw<std::invalid_argument>([&] { leapfrogKick(d + 3, d + 4, d + 5, d + 6, d + 7, d + 8, 1, 0.0); },
                                        "zero timestep");
    cudaFree(d);
  }
  if (failures) return 1;
  std::cout << "ok\n";
  return 0;
}
