// nbb_streaming.hpp -- headless frame output with the reference's names
// (src/streaming/frame.hpp:12-129 and src/streaming/device_capture.hpp:12-35
// of sytrams/AMSC-Nbody) over nbb_sim_capture_frame.
//
// FrameSampler and FrameSpool behave as the reference's (wall-clock sampling
// that skips missed intervals; run-<session>-frame-<20-digit sequence>.nbsnap
// files written through a .part file and renamed; a run-<session>.complete
// marker).  DeviceFrameWriter captures from a Simulation handle rather than
// from a device particle view, and takes the step and time from that handle.
// No viewer, server or network is part of this library.
#pragma once

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#if defined(__unix__) || defined(__APPLE__)
#include <unistd.h>
#endif

#include "nbb.h"
#include "nbb_simulation.hpp"

namespace nbody::streaming {

inline constexpr std::uint32_t kFrameVersion = 3;
inline constexpr std::size_t kFrameHeaderBytes = 128;
inline constexpr std::size_t kPositionComponents = 3;
inline constexpr std::uint16_t kQuantizedPositionMaximum = 65535;

class FrameSampler {
 public:
  explicit FrameSampler(double samplesPerSecond = 60.0) : rate_(samplesPerSecond), interval_(1.0 / samplesPerSecond) {
    if (!std::isfinite(samplesPerSecond) || samplesPerSecond <= 0.0)
      throw std::invalid_argument("Frame sample rate must be finite and positive");
  }

  [[nodiscard]] bool isDue(double elapsedWallSeconds) {
    if (!std::isfinite(elapsedWallSeconds) || elapsedWallSeconds < 0.0)
      throw std::invalid_argument("Frame sampling time must be finite and non-negative");
    const double tolerance =
        std::numeric_limits<double>::epsilon() * std::max(1.0, std::abs(elapsedWallSeconds)) * 8.0;
    if (elapsedWallSeconds + tolerance < next_) return false;
    const double skipped = std::floor(std::max(0.0, elapsedWallSeconds - next_) / interval_);
    next_ += (skipped + 1.0) * interval_;
    return true;
  }
  [[nodiscard]] std::uint64_t takeSequence() noexcept { return sequence_++; }
  [[nodiscard]] double rate() const noexcept { return rate_; }

 private:
  double rate_;
  double interval_;
  double next_ = 0.0;
  std::uint64_t sequence_ = 0;
};

class FrameSpool {
 public:
  explicit FrameSpool(std::filesystem::path directory, std::string sessionId = {})
      : directory_(std::move(directory)), sessionId_(sessionId.empty() ? defaultSession() : std::move(sessionId)) {
    if (directory_.empty()) throw std::invalid_argument("Frame spool directory cannot be empty");
    if (sessionId_.find_first_not_of("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789-_") !=
        std::string::npos)
      throw std::invalid_argument("Frame session id may contain only letters, numbers, '-' and '_'");
    std::error_code error;
    std::filesystem::create_directories(directory_, error);
    if (error)
      throw std::runtime_error("Could not create frame spool directory '" + directory_.string() +
                               "': " + error.message());
  }

  [[nodiscard]] const std::filesystem::path &directory() const noexcept { return directory_; }
  [[nodiscard]] const std::string &sessionId() const noexcept { return sessionId_; }

  // Publishes one frame (as produced by nbb_sim_capture_frame) under its
  // sequence number.
  std::filesystem::path writeFrame(std::uint64_t sequence, const std::vector<unsigned char> &frame) const {
    char digits[32];
    std::snprintf(digits, sizeof(digits), "%020llu", static_cast<unsigned long long>(sequence));
    const std::filesystem::path finalPath = directory_ / ("run-" + sessionId_ + "-frame-" + digits + ".nbsnap");
    std::error_code error;
    if (std::filesystem::exists(finalPath, error) && !error)
      throw std::runtime_error("Refusing to overwrite queued frame: " + finalPath.string());
    std::filesystem::path part = finalPath;
    part += ".part";
    {
      std::ofstream out(part, std::ios::binary | std::ios::trunc);
      if (!out.is_open()) throw std::runtime_error("Could not create temporary frame: " + part.string());
      out.write(reinterpret_cast<const char *>(frame.data()), static_cast<std::streamsize>(frame.size()));
      out.flush();
      if (!out) {
        std::filesystem::remove(part, error);
        throw std::runtime_error("Failed while writing frame payload: " + part.string());
      }
    }
    std::filesystem::rename(part, finalPath, error);
    if (error) {
      std::filesystem::remove(part, error);
      throw std::runtime_error("Could not publish frame: " + finalPath.string());
    }
    return finalPath;
  }

  [[nodiscard]] std::filesystem::path markComplete() const {
    const std::filesystem::path finalPath = directory_ / ("run-" + sessionId_ + ".complete");
    std::error_code error;
    if (std::filesystem::exists(finalPath, error) && !error) return finalPath;
    std::filesystem::path part = finalPath;
    part += ".part";
    {
      std::ofstream out(part, std::ios::out | std::ios::trunc | std::ios::binary);
      if (!out.is_open()) throw std::runtime_error("Could not create completion marker: " + part.string());
      out << sessionId_ << '\n';
    }
    std::filesystem::rename(part, finalPath, error);
    if (error) throw std::runtime_error("Could not publish completion marker '" + finalPath.string() + "'");
    return finalPath;
  }

 private:
  static std::string defaultSession() {
    const auto us = std::chrono::duration_cast<std::chrono::microseconds>(
                        std::chrono::system_clock::now().time_since_epoch())
                        .count();
#if defined(__unix__) || defined(__APPLE__)
    const auto process = static_cast<unsigned long long>(::getpid());
#else
    const auto process = 0ULL;
#endif
    return std::to_string(us) + "-" + std::to_string(process);
  }

  std::filesystem::path directory_;
  std::string sessionId_;
};

// src/streaming/device_capture.hpp:12-35: quantized frames of a simulation's
// current positions, built on the device.
class DeviceFrameWriter {
 public:
  DeviceFrameWriter(Simulation &simulation, std::size_t maximumParticles)
      : sim_(simulation.handle()), maximumParticles_(maximumParticles) {
    nbb_state_view v{};
    nbb::throwStatus(nbb_sim_state(sim_, &v));
    if (v.count == 0) throw std::invalid_argument("Cannot capture an empty or incomplete device particle view");
    source_ = v.count;
    sample_ = (maximumParticles == 0) ? v.count : std::min(v.count, maximumParticles);
    buffer_.resize(nbb_frame_bytes(sim_, maximumParticles));
  }

  [[nodiscard]] std::size_t sourceParticleCount() const noexcept { return source_; }
  [[nodiscard]] std::size_t sampleParticleCount() const noexcept { return sample_; }

  // Captures and publishes one frame; the step and time in its header are
  // the simulation's own.
  std::filesystem::path write(const FrameSpool &spool, std::uint64_t sequence) {
    std::size_t written = 0;
    nbb::throwStatus(
        nbb_sim_capture_frame(sim_, maximumParticles_, sequence, buffer_.data(), buffer_.size(), &written, 0));
    buffer_.resize(written);
    return spool.writeFrame(sequence, buffer_);
  }

 private:
  nbb_sim *sim_;
  std::size_t maximumParticles_;
  std::size_t source_ = 0, sample_ = 0;
  std::vector<unsigned char> buffer_;
};

}  // namespace nbody::streaming
