// noalloc.cu -- Morton keys and their stable sorted permutation without any
// device allocation, for callers that must not allocate.
//
// Some hosts own all device memory through their own pool or budget and do
// not let a library call cudaMalloc/cudaFree (those calls can synchronise the
// device and fragment the host's pool); a real-time visualisation loop or a
// plugin host with a fixed memory budget are typical.  This entry point keeps
// its scratch memory -- device scalars, radix-sort digit histograms and
// look-back status, and two packed-pair buffers -- in one file-scope device
// array of fixed size.  Every GPU that loads the library holds that array
// until the process exits.
#include "nbb.h"
#include "nbb_internal.cuh"

#include <cmath>
#include <string>

namespace {

using nbb::DevScalars;
using nbb::kSortPasses;
using nbb::kSortTile;
using nbb::Workspace;

constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

constexpr size_t kMaxN = NBB_NOALLOC_MAX_PARTICLES;
constexpr size_t kMaxTiles = (kMaxN + kSortTile - 1) / kSortTile;
constexpr size_t kOffScalars = 0;
constexpr size_t kOffSysBB = round_up(kOffScalars + sizeof(DevScalars));
constexpr size_t kOffSysBox = round_up(kOffSysBB + 6 * sizeof(unsigned long long));
constexpr size_t kOffHist = round_up(kOffSysBox + 4 * sizeof(double));
constexpr size_t kOffStatus = round_up(kOffHist + sizeof(uint32_t) * nbb::kMaxSortPasses * 256);
constexpr size_t kOffPairsA = round_up(kOffStatus + sizeof(uint32_t) * kSortPasses * kMaxTiles * 256);
constexpr size_t kOffPairsB = round_up(kOffPairsA + sizeof(unsigned long long) * kMaxN);
constexpr size_t kScratchBytes = round_up(kOffPairsB + sizeof(unsigned long long) * kMaxN);

// The scratch array.  In host code this name is only a host-side stand-in:
// its device address comes from cudaGetSymbolAddress in the current context,
// asked on every call (no address is cached: a reset device or another
// context on the same device has its own instance of the module).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

thread_local std::string t_msg;

int fail(int status, const std::string &msg) {
  t_msg = msg;
  return status;
}

}  // namespace

extern "C" {

int nbb_morton_sort_noalloc(const double *x, const double *y, const double *z, size_t n, uint32_t *keys,
                            uint32_t *idx, void *stream) {
  if (n == 0) return fail(NBB_ERR_INVALID_ARGUMENT, "Cannot compute Morton keys for an empty particle set");
  if (n > kMaxN)
    return fail(NBB_ERR_INVALID_ARGUMENT,
                "nbb_morton_sort_noalloc: n = " + std::to_string(n) + " exceeds NBB_NOALLOC_MAX_PARTICLES (" +
                    std::to_string(kMaxN) + ")");
  if (!x || !y || !z || !keys || !idx)
    return fail(NBB_ERR_INVALID_ARGUMENT, "Morton coordinate and output device pointers must not be null");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(NBB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    // the call ends with a device-to-host read and a stream synchronisation,
    // neither of which a stream capture allows
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess)
      return fail(NBB_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
      return fail(NBB_ERR_INVALID_ARGUMENT, "nbb_morton_sort_noalloc cannot be captured in a CUDA graph");
  }
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return fail(NBB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned char *base = static_cast<unsigned char *>(p);
  Workspace ws{};
  ws.n = (int)n;
  cudaDeviceGetAttribute(&ws.num_sms, cudaDevAttrMultiProcessorCount, dev);
  ws.x = const_cast<double *>(x);
  ws.y = const_cast<double *>(y);
  ws.z = const_cast<double *>(z);
  ws.sc = reinterpret_cast<DevScalars *>(base + kOffScalars);
  ws.sys_bb = reinterpret_cast<unsigned long long *>(base + kOffSysBB);
  ws.sys_box = reinterpret_cast<double *>(base + kOffSysBox);
  ws.digit_hist = reinterpret_cast<uint32_t *>(base + kOffHist);
  ws.sort_tiles = (int)((n + kSortTile - 1) / kSortTile);
  ws.sort_status = reinterpret_cast<uint32_t *>(base + kOffStatus);
  ws.pairs_a = reinterpret_cast<unsigned long long *>(base + kOffPairsA);
  ws.pairs_b = reinterpret_cast<unsigned long long *>(base + kOffPairsB);
  // the sticky error word must start at zero for this call
  e = cudaMemsetAsync(&ws.sc->error, 0, sizeof(int), s);
  if (e == cudaSuccess) e = nbb::launch_morton_sort_only(ws, keys, idx, s);
  int word = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&word, &ws.sc->error, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(NBB_ERR_CUDA, std::string("nbb_morton_sort_noalloc: ") + cudaGetErrorString(e));
  if (word == nbb::kStageBbox * 100 + 1)
    return fail(NBB_ERR_DOMAIN, "Particle positions must be finite to compute a bounding box.");
  if (word != 0) return fail(NBB_ERR_DEVICE, "nbb_morton_sort_noalloc: device error " + std::to_string(word));
  t_msg.clear();
  return NBB_OK;
}

const char *nbb_noalloc_last_error_message(void) { return t_msg.c_str(); }

}  // extern "C"
