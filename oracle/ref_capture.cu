// ref_capture.cu -- TEST INFRASTRUCTURE ONLY: drives the reference's own
// frame capture (src/streaming/device_capture.cu, src/streaming/frame.cpp of
// sytrams/AMSC-Nbody, compiled unmodified by oracle/Makefile) so that the
// library's frames can be compared byte for byte with the reference's.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "particle.hpp"
#include "streaming/device_capture.hpp"
#include "streaming/frame.hpp"

namespace {
std::string g_capture_message;

template <typename T>
T *to_device(const T *host, std::size_t n) {
  T *d = nullptr;
  if (cudaMalloc(reinterpret_cast<void **>(&d), n * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
  if (cudaMemcpy(d, host, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) throw std::runtime_error("cudaMemcpy");
  return d;
}
}  // namespace

extern "C" {

const char *ref_capture_last_error(void) { return g_capture_message.c_str(); }

// Writes one frame of (x, y, z, type) with DeviceFrameWriter into `dir`
// (session id "ref"); its path goes to path_out.  Returns 0, or 1 with the
// reference's exception message in ref_capture_last_error().
int ref_capture_frame(std::size_t n, const double *x, const double *y, const double *z, const uint8_t *type,
                      std::size_t max_particles, uint64_t sequence, uint64_t step, double time, const char *dir,
                      char *path_out, std::size_t path_cap) {
  double *dx = nullptr, *dy = nullptr, *dz = nullptr;
  uint8_t *dt = nullptr;
  int status = 0;
  try {
    dx = to_device(x, n);
    dy = to_device(y, n);
    dz = to_device(z, n);
    dt = to_device(type, n);
    const ConstDeviceParticlesView view{n, nullptr, dx, dy, dz, nullptr, nullptr, nullptr, dt};
    nbody::streaming::DeviceFrameWriter writer(view, max_particles);
    nbody::streaming::FrameSpool spool(dir, "ref");
    const std::string path = writer.write(spool, sequence, step, time).string();
    std::strncpy(path_out, path.c_str(), path_cap - 1);
    path_out[path_cap - 1] = '\0';
  } catch (const std::exception &e) {
    g_capture_message = e.what();
    status = 1;
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dz);
  cudaFree(dt);
  return status;
}

}  // extern "C"
