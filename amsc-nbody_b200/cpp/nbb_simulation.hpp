// nbb_simulation.hpp -- header-only C++ layer with the reference's public
// names over the C ABI of libnbb.so (include/nbb.h).
//
// A program written against sytrams/AMSC-Nbody's hot-path headers
// (src/simulation.hpp, src/particle.hpp, src/barnes_hut.hpp,
// src/integrator.hpp) switches by including this header instead and linking
// libnbb.so.  Names, argument meaning and the exception types thrown follow
// the reference:
//   std::invalid_argument  bad arguments          (NBB_ERR_INVALID_ARGUMENT)
//   std::domain_error      non-finite positions   (NBB_ERR_DOMAIN)
//   std::logic_error       call order / state     (NBB_ERR_LOGIC)
//   std::overflow_error    size limits            (NBB_ERR_OVERFLOW)
//   std::runtime_error     CUDA / device errors   (other statuses)
// Differences: Particles keeps the loaded state on the host until a
// Simulation copies it to the device; SimulationOptions adds the traversal
// precision and the gravitational constant (default: the SI value the
// reference's Simulation uses).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "nbb.h"

// src/particle.hpp:16-17
inline constexpr double G = 6.67430e-11;
inline constexpr double K = 8.98755e9;

// src/particle_type.hpp:7-18
enum class ParticleType : std::uint8_t { Unknown = 0, Star = 1, Planet = 2, Moon = 3, Asteroid = 4 };
[[nodiscard]] inline constexpr bool isValidParticleType(std::uint8_t value) noexcept {
  return value <= static_cast<std::uint8_t>(ParticleType::Asteroid);
}

namespace nbb {

inline void throwStatus(int status) {
  if (status == NBB_OK) return;
  const std::string message = nbb_last_error_message();
  switch (status) {
    case NBB_ERR_INVALID_ARGUMENT: throw std::invalid_argument(message);
    case NBB_ERR_DOMAIN: throw std::domain_error(message);
    case NBB_ERR_LOGIC: throw std::logic_error(message);
    case NBB_ERR_OVERFLOW: throw std::overflow_error(message);
    default: throw std::runtime_error(message);
  }
}

}  // namespace nbb

// src/particle.hpp:85-109
struct DeviceParticlesView {
  std::size_t count;
  double *mass;
  double *x;
  double *y;
  double *z;
  double *vx;
  double *vy;
  double *vz;
  std::uint8_t *type;
};

struct ConstDeviceParticlesView {
  std::size_t count;
  const double *mass;
  const double *x;
  const double *y;
  const double *z;
  const double *vx;
  const double *vy;
  const double *vz;
  const std::uint8_t *type;
};

// Planar particle file (src/particle.hpp:26-81, 145-225): a 64-bit or
// 32-bit particle count, then the mass, x, y, z, vx, vy, vz blocks of
// doubles, then optionally one uint8 particle type per particle.  Layout
// detection, validation and messages follow the reference.
class Particles {
 public:
  explicit Particles(std::ifstream &inFile) {
    if (!inFile.is_open() || !inFile.good())
      throw std::runtime_error("Invalid or unreadable file stream provided.");
    const Header header = detect(inFile);
    count_ = header.count;
    if (count_ == 0) throw std::runtime_error("Particle count is zero.");
    inFile.clear();
    inFile.seekg(header.bytes, std::ios::beg);
    const auto bytes = static_cast<std::streamsize>(count_ * sizeof(double));
    const char *names[7] = {"mass", "x position", "y position", "z position",
                            "x velocity", "y velocity", "z velocity"};
    std::vector<double> *blocks[7] = {&mass_, &x_, &y_, &z_, &vx_, &vy_, &vz_};
    for (int b = 0; b < 7; ++b) {
      std::vector<double> &dst = *blocks[b];
      dst.resize(count_);
      inFile.read(reinterpret_cast<char *>(dst.data()), bytes);
      if (inFile.gcount() != bytes) throw std::runtime_error("Incomplete " + std::string(names[b]) + " block");
      for (std::size_t i = 0; i < count_; ++i) {
        if (!std::isfinite(dst[i]))
          throw std::runtime_error("Non-finite " + std::string(names[b]) + " value at particle " +
                                   std::to_string(i));
        if (b == 0 && dst[i] < 0.0)
          throw std::runtime_error("Negative mass value at particle " + std::to_string(i));
      }
    }
    type_.assign(count_, static_cast<std::uint8_t>(ParticleType::Unknown));
    if (header.typed) {
      const auto tbytes = static_cast<std::streamsize>(count_);
      inFile.read(reinterpret_cast<char *>(type_.data()), tbytes);
      if (inFile.gcount() != tbytes) throw std::runtime_error("Incomplete particle type block");
      for (const std::uint8_t t : type_)
        if (!isValidParticleType(t)) throw std::runtime_error("Unsupported particle type value");
    }
    if (!inFile) throw std::runtime_error("Failed to read all expected particle data. File may be truncated.");
  }

  // Host-side construction from planar arrays (mass, positions, velocities).
  Particles(std::vector<double> mass, std::vector<double> x, std::vector<double> y, std::vector<double> z,
            std::vector<double> vx, std::vector<double> vy, std::vector<double> vz)
      : count_(mass.size()), mass_(std::move(mass)), x_(std::move(x)), y_(std::move(y)), z_(std::move(z)),
        vx_(std::move(vx)), vy_(std::move(vy)), vz_(std::move(vz)), type_(count_, 0) {
    for (const auto *v : {&x_, &y_, &z_, &vx_, &vy_, &vz_})
      if (v->size() != count_) throw std::invalid_argument("Particle arrays must have equal sizes");
  }

  [[nodiscard]] std::size_t size() const noexcept { return count_; }
  [[nodiscard]] const std::vector<double> &mass() const noexcept { return mass_; }
  [[nodiscard]] const std::vector<double> &x() const noexcept { return x_; }
  [[nodiscard]] const std::vector<double> &y() const noexcept { return y_; }
  [[nodiscard]] const std::vector<double> &z() const noexcept { return z_; }
  [[nodiscard]] const std::vector<double> &vx() const noexcept { return vx_; }
  [[nodiscard]] const std::vector<double> &vy() const noexcept { return vy_; }
  [[nodiscard]] const std::vector<double> &vz() const noexcept { return vz_; }
  [[nodiscard]] const std::vector<std::uint8_t> &type() const noexcept { return type_; }

 private:
  struct Header {
    std::uint32_t count;
    std::streamoff bytes;
    bool typed;
  };

  static Header detect(std::ifstream &in) {
    in.clear();
    in.seekg(0, std::ios::end);
    const auto size = in.tellg();
    if (size < 0) throw std::runtime_error("Failed to determine particle file size.");
    const std::streamoff per = static_cast<std::streamoff>(7 * sizeof(double));
    auto fits = [&](std::uint64_t n, std::streamoff head, bool typed) {
      return size == head + static_cast<std::streamoff>(n) * per + (typed ? static_cast<std::streamoff>(n) : 0);
    };
    in.seekg(0, std::ios::beg);
    std::uint64_t n64 = 0;
    in.read(reinterpret_cast<char *>(&n64), sizeof(n64));
    if (in && n64 > 0 && n64 <= std::numeric_limits<std::uint32_t>::max()) {
      const auto head = static_cast<std::streamoff>(sizeof(std::uint64_t));
      if (fits(n64, head, true)) return {static_cast<std::uint32_t>(n64), head, true};
      if (fits(n64, head, false)) return {static_cast<std::uint32_t>(n64), head, false};
    }
    in.clear();
    in.seekg(0, std::ios::beg);
    std::uint32_t n32 = 0;
    in.read(reinterpret_cast<char *>(&n32), sizeof(n32));
    if (in && n32 > 0) {
      const auto head = static_cast<std::streamoff>(sizeof(std::uint32_t));
      if (fits(n32, head, true)) return {n32, head, true};
      if (fits(n32, head, false)) return {n32, head, false};
    }
    throw std::runtime_error(
        "Unsupported particle file layout. Expected planar doubles with a 32-bit or 64-bit particle count "
        "header, optionally followed by one uint8 particle type per particle.");
  }

  std::size_t count_ = 0;
  std::vector<double> mass_, x_, y_, z_, vx_, vy_, vz_;
  std::vector<std::uint8_t> type_;
};

// src/simulation.hpp:18-22
struct SimulationConfig {
  double timeStep;
  double theta;
  double softening;
};

// Additions of this library to the reference's configuration.
struct SimulationOptions {
  double gravitationalConstant = G;
  int precision = NBB_PRECISION_FP64;
  int device = 0;
  bool useGraph = true;
};

// src/simulation.hpp:24-66: initialize() once, then step()/run(n).
class Simulation {
 public:
  Simulation(Particles particles, SimulationConfig config, SimulationOptions options = {}) {
    nbb_config c;
    nbb_config_default(&c);
    c.time_step = config.timeStep;
    c.theta = config.theta;
    c.softening = config.softening;
    c.gravitational_constant = options.gravitationalConstant;
    c.precision = options.precision;
    c.device = options.device;
    c.use_graph = options.useGraph ? 1 : 0;
    nbb::throwStatus(nbb_sim_create(&c, particles.size(), particles.mass().data(), particles.x().data(),
                                    particles.y().data(), particles.z().data(), particles.vx().data(),
                                    particles.vy().data(), particles.vz().data(), particles.type().data(), 0,
                                    &sim_));
  }
  ~Simulation() noexcept {
    if (sim_) nbb_sim_destroy(sim_);
  }
  Simulation(const Simulation &) = delete;
  Simulation &operator=(const Simulation &) = delete;

  void initialize() { nbb::throwStatus(nbb_sim_initialize(sim_)); }
  void step() { nbb::throwStatus(nbb_sim_step(sim_)); }
  void run(std::size_t numberOfSteps) { nbb::throwStatus(nbb_sim_run(sim_, numberOfSteps)); }
  [[nodiscard]] double time() const noexcept { return nbb_sim_time(sim_); }
  [[nodiscard]] std::size_t stepNumber() const noexcept {
    return static_cast<std::size_t>(nbb_sim_step_number(sim_));
  }
  [[nodiscard]] DeviceParticlesView particles() noexcept {
    nbb_state_view v{};
    nbb_sim_state(sim_, &v);
    return {v.count, v.mass, v.x, v.y, v.z, v.vx, v.vy, v.vz, v.type};
  }
  [[nodiscard]] nbb_sim *handle() noexcept { return sim_; }

 private:
  nbb_sim *sim_ = nullptr;
};

// src/barnes_hut.hpp:8-19
struct BarnesHutParameters {
  double theta = 0.5;
  double softening = 1.0e-6;
  double gravitationalConstant = 6.67430e-11;
};

enum class BarnesHutParticleOrder { original, morton };

// computeBarnesHutAcceleration on an octree in the reference's node layout
// (src/octree_types.hpp:73-104), device pointers as in the reference.
inline void computeBarnesHutAcceleration(const nbb_octree_view &octree, const std::uint32_t *d_sortedIndices,
                                         const double *d_mass, const double *d_positionX,
                                         const double *d_positionY, const double *d_positionZ,
                                         double *d_accelerationX, double *d_accelerationY,
                                         double *d_accelerationZ, std::size_t particleCount,
                                         const BarnesHutParameters &parameters,
                                         BarnesHutParticleOrder particleOrder = BarnesHutParticleOrder::original) {
  if (particleCount != static_cast<std::size_t>(octree.n_particles))
    throw std::invalid_argument("Particle count does not match the octree");
  nbb::throwStatus(nbb_accel_octree(&octree, d_sortedIndices, d_mass, d_positionX, d_positionY, d_positionZ,
                                    d_accelerationX, d_accelerationY, d_accelerationZ, parameters.theta,
                                    parameters.softening, parameters.gravitationalConstant,
                                    particleOrder == BarnesHutParticleOrder::morton ? 1 : 0, 1));
}

// src/integrator.hpp:5-7
inline void leapfrogKickDrift(double *d_positionX, double *d_positionY, double *d_positionZ, double *d_velocityX,
                              double *d_velocityY, double *d_velocityZ, const double *d_accelerationX,
                              const double *d_accelerationY, const double *d_accelerationZ,
                              std::size_t particleCount, double dt) {
  nbb::throwStatus(nbb_kick_drift(d_positionX, d_positionY, d_positionZ, d_velocityX, d_velocityY, d_velocityZ,
                                  d_accelerationX, d_accelerationY, d_accelerationZ, particleCount, dt, nullptr));
}

inline void leapfrogKick(double *d_velocityX, double *d_velocityY, double *d_velocityZ,
                         const double *d_accelerationX, const double *d_accelerationY,
                         const double *d_accelerationZ, std::size_t particleCount, double dt) {
  nbb::throwStatus(nbb_kick(d_velocityX, d_velocityY, d_velocityZ, d_accelerationX, d_accelerationY,
                            d_accelerationZ, particleCount, dt, nullptr));
}
