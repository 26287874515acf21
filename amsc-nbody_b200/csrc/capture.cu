// capture.cu -- quantized position frames of the particle state, assembled
// on the device: the reference's graphical capture (src/streaming/
// device_capture.cu:27-330 of sytrams/AMSC-Nbody: strided sample, bounds,
// 16-bit quantization, particle types) and its version-3 frame layout
// (src/streaming/frame.cpp:68-95 and 341-470), with no viewer or network
// behind it: the frame is a byte buffer the caller stores or sends.
//
//   frame_bounds_kernel    sampled positions' extrema (order-preserving u64
//                          atomics, one per warp and axis) + non-finite flag
//   frame_payload_kernel   quantized xyz (3 x u16 per sample) and types
//   frame_header_kernel    the 128-byte little-endian header
//
// Sample i of s reads particle (i * n) / s.  Quantization is the
// reference's: 0 when an axis collapses, else
// u16(clamp((p - min) / (max - min), 0, 1) * 65535 + 0.5) with the product
// and the addition fused, as nvcc compiles the reference's expression.
#include "nbb_internal.cuh"

#include <cmath>

namespace nbb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ unsigned long long sample_source(unsigned long long i, unsigned long long n,
                                                            unsigned long long s) {
  return (i * n) / s;
}

__global__ void frame_reset_kernel(FrameScalars *f) {
  if (threadIdx.x < 3) {
    f->lo[threadIdx.x] = ~0ull;
    f->hi[threadIdx.x] = 0ull;
  }
  if (threadIdx.x == 0) {
    f->nonfinite = 0;
    f->bad_type = 0;
  }
}

__global__ void __launch_bounds__(kThreads) frame_bounds_kernel(const double *x, const double *y, const double *z,
                                                                unsigned long long n, unsigned long long s,
                                                                FrameScalars *f) {
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
  bool bad = false;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < s;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long src = sample_source(i, n, s);
    const double v[3] = {x[src], y[src], z[src]};
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) {
      bad = true;
      continue;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const unsigned long long b = order_bits(v[a]);
      lo[a] = b < lo[a] ? b : lo[a];
      hi[a] = b > hi[a] ? b : hi[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long l = __shfl_xor_sync(0xffffffffu, lo[a], o);
      const unsigned long long h = __shfl_xor_sync(0xffffffffu, hi[a], o);
      lo[a] = l < lo[a] ? l : lo[a];
      hi[a] = h > hi[a] ? h : hi[a];
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (lo[a] != ~0ull) atomicMin(&f->lo[a], lo[a]);
      if (hi[a] != 0ull) atomicMax(&f->hi[a], hi[a]);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(&f->nonfinite, 1);
}

__device__ __forceinline__ uint16_t quantize16(double p, double lo, double hi) {
  if (hi == lo) return 0;
  double u = __ddiv_rn(__dsub_rn(p, lo), __dsub_rn(hi, lo));
  u = fmin(1.0, fmax(0.0, u));
  return (uint16_t)__fma_rn(u, 65535.0, 0.5);
}

// Positions are quantized against the bounds the previous kernel left in f.
__global__ void __launch_bounds__(kThreads) frame_payload_kernel(const double *x, const double *y, const double *z,
                                                                 const uint8_t *type, unsigned long long n,
                                                                 unsigned long long s, FrameScalars *f,
                                                                 unsigned char *frame, unsigned long long header) {
  if (f->nonfinite) return;
  const double lo[3] = {order_value(f->lo[0]), order_value(f->lo[1]), order_value(f->lo[2])};
  const double hi[3] = {order_value(f->hi[0]), order_value(f->hi[1]), order_value(f->hi[2])};
  uint16_t *xyz = reinterpret_cast<uint16_t *>(frame + header);
  uint8_t *types = frame + header + 6 * s;
  bool bad = false;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < s;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long src = sample_source(i, n, s);
    xyz[3 * i + 0] = quantize16(x[src], lo[0], hi[0]);
    xyz[3 * i + 1] = quantize16(y[src], lo[1], hi[1]);
    xyz[3 * i + 2] = quantize16(z[src], lo[2], hi[2]);
    const uint8_t t = type ? type[src] : 0;  // particle_type.hpp: 0..4 (Unknown..Asteroid)
    bad |= t > 4;
    types[i] = t;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(&f->bad_type, 1);
}

__device__ __forceinline__ unsigned char *put_le(unsigned char *p, unsigned long long v, int bytes) {
  for (int b = 0; b < bytes; ++b) p[b] = (unsigned char)((v >> (8 * b)) & 0xffu);
  return p + bytes;
}

// frame.cpp:68-95, version 3 (positions + types).
__global__ void frame_header_kernel(const FrameScalars *f, FrameHeaderFields h, unsigned char *frame) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned char *p = frame;
  const char magic[8] = {'N', 'B', 'S', 'N', 'A', 'P', '0', '1'};
  for (int k = 0; k < 8; ++k) p[k] = (unsigned char)magic[k];
  p += 8;
  p = put_le(p, 3, 4);
  p = put_le(p, kFrameHeaderBytes, 4);
  p = put_le(p, h.sequence, 8);
  p = put_le(p, h.step, 8);
  p = put_le(p, (unsigned long long)__double_as_longlong(h.time), 8);
  p = put_le(p, h.source_count, 8);
  p = put_le(p, h.sample_count, 8);
  p = put_le(p, 2, 4);
  p = put_le(p, 3, 4);
  p = put_le(p, 7 * h.sample_count, 8);
  for (int a = 0; a < 3; ++a) p = put_le(p, (unsigned long long)__double_as_longlong(order_value(f->lo[a])), 8);
  for (int a = 0; a < 3; ++a) p = put_le(p, (unsigned long long)__double_as_longlong(order_value(f->hi[a])), 8);
  put_le(p, h.sample_count, 8);
}

inline int blocks_for(unsigned long long s) {
  unsigned long long b = (s + kThreads - 1) / kThreads;
  if (b > 148ull * 8) b = 148ull * 8;
  return b < 1 ? 1 : (int)b;
}

}  // namespace

cudaError_t launch_frame_capture(const double *x, const double *y, const double *z, const uint8_t *type, size_t n,
                                 size_t s, FrameScalars *f, const FrameHeaderFields &h, unsigned char *frame,
                                 cudaStream_t st) {
  frame_reset_kernel<<<1, 32, 0, st>>>(f);
  frame_bounds_kernel<<<blocks_for(s), kThreads, 0, st>>>(x, y, z, n, s, f);
  frame_payload_kernel<<<blocks_for(s), kThreads, 0, st>>>(x, y, z, type, n, s, f, frame, kFrameHeaderBytes);
  frame_header_kernel<<<1, 32, 0, st>>>(f, h, frame);
  count_launches(4);
  return cudaGetLastError();
}

}  // namespace nbb
