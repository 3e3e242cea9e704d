// tba_scene_cost_noalloc: the robust cost of a packed scene that already lives in device memory,
// computed without allocating anything.
//
// Who needs it.  Some callers cannot call cudaMalloc.  A host application that embeds the
// operator next to its own CUDA work often owns all device memory through its own allocator
// (a caching pool or an arena reserved at start-up), so a cudaMalloc from a library either fails
// at the memory limit or fragments memory the application manages.  Code on a latency-critical
// thread cannot afford cudaMalloc or cudaFree either, because both can synchronise the device.
// Such callers keep the packed scene in their own device buffers and need its cost (to decide
// whether to run a bundle adjustment, or to filter observations after one) without the library
// allocating a workspace, as tba_bundle_adjust does.
//
// How.  This is a variant of the grid engine's scene-cost kernel (k_cost, tba_kernels.cu), whose
// per-block partial sums are scratch memory.  Here the partials live in one file-scope
// `static __device__` array of a fixed size: every GPU that loads the library holds it (128 KiB)
// until the process exits.  Work is cut into tiles of kTileObs observations, one block per tile,
// so the scratch bounds the problem: at most kMaxTiles tiles.  A second one-block kernel sums the
// tile partials in a fixed order into the caller's result.  Nothing is allocated: no cudaMalloc,
// no cudaFree, no library routine that allocates.
//
// Caller buffers are checked before any launch: each of scene, index and result must be device
// memory of the current device (cudaPointerGetAttributes), and the allocation it lies in must hold
// the length the caller states (the driver's cuMemGetAddressRange), so that a host pointer or a
// buffer shorter than the control implies is refused instead of faulting the caller's context.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/tba.h"
#include "tba_math.cuh"

namespace {

constexpr uint32_t kTileObs = 4096;    // observations per tile (one block)
constexpr uint32_t kMaxTiles = 4096;   // tiles the scratch holds: at most 16,777,216 observations
constexpr uint32_t kThreads = 256;
constexpr int kMaxDevices = 64;

// Per tile: robust cost, squared error, failed projections, out-of-range indices.
static __device__ __align__(256) double g_tile_partials[kMaxTiles * 4];

__global__ void __launch_bounds__(kThreads)
k_tile_cost(const double* scene, const uint32_t* index, uint32_t C, uint32_t P, uint32_t M, uint32_t D,
            double huber, double* partials) {
  __shared__ double red[4 * (kThreads / 32)];
  const uint32_t begin = blockIdx.x * kTileObs;
  const uint32_t end = begin + kTileObs < M ? begin + kTileObs : M;
  const double* poses = scene;
  const double* points = scene + 12 * size_t(C);
  const double* cams = points + 3 * size_t(P);
  const double* pixels = cams + 6 * size_t(C);
  double v[4] = {0, 0, 0, 0};
  for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const uint32_t c = index[i], pt = index[M + i];
    if (c >= C || pt >= P) {  // caller-owned indices are not trusted: skip and count
      v[3] += 1;
      continue;
    }
    const double* pose = poses + 12 * size_t(c);
    const double* X = points + 3 * size_t(pt);
    const double* k = cams + 6 * size_t(c);
    const tba::Camera cam{k[0], k[1], k[2], k[3], k[4], k[5]};
    const bool directional = pt >= P - D;
    double q[3];
    for (int j = 0; j < 3; j++) {
      q[j] = pose[j * 3] * X[0] + pose[j * 3 + 1] * X[1] + pose[j * 3 + 2] * X[2];
      if (!directional) q[j] += pose[9 + j];
    }
    double pixel[2], du[3], dv[3];
    if (!tba::project(cam, q, pixel, du, dv)) {
      v[2] += 1;
      continue;
    }
    const double ru = pixel[0] - pixels[2 * size_t(i)], rv = pixel[1] - pixels[2 * size_t(i) + 1];
    const double sq = ru * ru + rv * rv;
    v[0] += tba::robust_cost(sqrt(sq), huber);
    v[1] += sq;
  }
  // Fixed-order block sum: warp butterflies, then the warps in order.
  for (int n = 0; n < 4; n++)
    for (int d = 16; d > 0; d >>= 1) v[n] += __shfl_xor_sync(0xffffffffu, v[n], d);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int n = 0; n < 4; n++) red[warp * 4 + n] = v[n];
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int w = 0; w < int(kThreads / 32); w++) s += red[w * 4 + threadIdx.x];
    partials[4 * blockIdx.x + threadIdx.x] = s;  // every tile row is written on every call
  }
}

__global__ void __launch_bounds__(kThreads) k_tile_finish(const double* partials, uint32_t tiles, double* result) {
  __shared__ double red[4 * (kThreads / 32)];
  double v[4] = {0, 0, 0, 0};
  for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x)
    for (int n = 0; n < 4; n++) v[n] += partials[4 * t + n];
  for (int n = 0; n < 4; n++)
    for (int d = 16; d > 0; d >>= 1) v[n] += __shfl_xor_sync(0xffffffffu, v[n], d);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int n = 0; n < 4; n++) red[warp * 4 + n] = v[n];
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int w = 0; w < int(kThreads / 32); w++) s += red[w * 4 + threadIdx.x];
    result[threadIdx.x] = s;
  }
}

// The scratch's device address, per device ordinal, with the context it was looked up in: a caller
// that resets the device (cudaDeviceReset) or binds another context gets a fresh look-up.
struct Scratch {
  CUcontext context = nullptr;
  double* address = nullptr;
};
std::mutex g_setup;
Scratch g_scratch[kMaxDevices];

// Driver calls reached through the runtime's entry-point table (no link against libcuda).
using GetAddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
using GetCurrentContext = CUresult (*)(CUcontext*);
GetAddressRange g_range = nullptr;
GetCurrentContext g_context = nullptr;

void say(char* message, size_t len, const char* text) {
  if (message && len) {
    std::strncpy(message, text, len - 1);
    message[len - 1] = 0;
  }
}

bool driver_calls(char* message, size_t len) {
  if (g_range && g_context) return true;
  void* range = nullptr;
  void* context = nullptr;
  cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &range, cudaEnableDefault, &q1) != cudaSuccess ||
      cudaGetDriverEntryPoint("cuCtxGetCurrent", &context, cudaEnableDefault, &q2) != cudaSuccess ||
      q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !range || !context) {
    cudaGetLastError();
    say(message, len, "tba_scene_cost_noalloc: the CUDA driver does not provide cuMemGetAddressRange/cuCtxGetCurrent");
    return false;
  }
  g_range = reinterpret_cast<GetAddressRange>(range);
  g_context = reinterpret_cast<GetCurrentContext>(context);
  return true;
}

// True when `p` is device (or managed) memory of device `dev` whose allocation holds `bytes` from
// `p` on; otherwise the message says why.  Nothing here touches the memory.
bool device_buffer(const void* p, size_t bytes, int dev, const char* name, char* message, size_t len) {
  char text[256];
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    std::snprintf(text, sizeof text, "tba_scene_cost_noalloc: %s is not a pointer CUDA knows", name);
    say(message, len, text);
    return false;
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) {
    std::snprintf(text, sizeof text, "tba_scene_cost_noalloc: %s is %s memory, not device memory", name,
                  attr.type == cudaMemoryTypeHost ? "page-locked host" : "host");
    say(message, len, text);
    return false;
  }
  if (attr.type == cudaMemoryTypeDevice && attr.device != dev) {
    std::snprintf(text, sizeof text, "tba_scene_cost_noalloc: %s is memory of device %d, not of the current device %d",
                  name, attr.device, dev);
    say(message, len, text);
    return false;
  }
  CUdeviceptr base = 0;
  size_t size = 0;
  const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p);
  if (g_range(&base, &size, at) != CUDA_SUCCESS) {
    std::snprintf(text, sizeof text, "tba_scene_cost_noalloc: %s lies in no device allocation the driver can size", name);
    say(message, len, text);
    return false;
  }
  if (at < base || at - base > size || size - (at - base) < bytes) {
    std::snprintf(text, sizeof text,
                  "tba_scene_cost_noalloc: %s length claims %zu bytes but its allocation holds %zu from that pointer",
                  name, bytes, at >= base && at - base <= size ? size_t(size - (at - base)) : size_t(0));
    say(message, len, text);
    return false;
  }
  return true;
}

}  // namespace

extern "C" tba_status tba_scene_cost_noalloc(const tba_control* control, const double* scene, size_t scene_len,
                                             const uint32_t* index, size_t index_len, double* result,
                                             size_t result_len, void* stream, char* message, size_t message_len) {
  say(message, message_len, "");
  if (!control || !scene || !index || !result) {
    say(message, message_len, "tba_scene_cost_noalloc: null control or device pointer");
    return TBA_ERROR_ARGUMENT;
  }
  const uint32_t C = control->cameras, P = control->points, M = control->observations, D = control->directional_points;
  if (C < 1 || P < 1 || D >= P || M < 1 || !(control->huber >= 1e-12 && control->huber <= 1e6)) {
    say(message, message_len, "tba_scene_cost_noalloc: invalid control (cameras, points, observations or huber)");
    return TBA_ERROR_ARGUMENT;
  }
  const uint64_t tiles = (uint64_t(M) + kTileObs - 1) / kTileObs;
  if (tiles > kMaxTiles) {
    char text[256];
    std::snprintf(text, sizeof text,
                  "tba_scene_cost_noalloc: %u observations exceed the fixed scratch of %u tiles x %u observations "
                  "(%u); use tba_bundle_adjust with iterations = 0",
                  M, kMaxTiles, kTileObs, kMaxTiles * kTileObs);
    say(message, message_len, text);
    return TBA_ERROR_ARGUMENT;
  }
  // The lengths the control implies: the packed arrays of tba_bundle_adjust, and 4 result words.
  if (scene_len != tba_scene_size(control) || index_len != tba_index_size(control) || result_len < 4) {
    char text[256];
    std::snprintf(text, sizeof text,
                  "tba_scene_cost_noalloc: array lengths (scene %zu, index %zu, result %zu) differ from the control's "
                  "(scene %zu, index %zu, result 4)",
                  scene_len, index_len, result_len, tba_scene_size(control), tba_index_size(control));
    say(message, message_len, text);
    return TBA_ERROR_ARGUMENT;
  }
  if (reinterpret_cast<uintptr_t>(scene) % alignof(double) || reinterpret_cast<uintptr_t>(index) % alignof(uint32_t) ||
      reinterpret_cast<uintptr_t>(result) % alignof(double)) {
    say(message, message_len, "tba_scene_cost_noalloc: misaligned device pointer");
    return TBA_ERROR_ARGUMENT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    say(message, message_len, e != cudaSuccess ? cudaGetErrorString(e) : "tba_scene_cost_noalloc: device ordinal >= 64");
    return e != cudaSuccess ? TBA_ERROR_CUDA : TBA_ERROR_ARGUMENT;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup);
    if (!driver_calls(message, message_len)) return TBA_ERROR_CUDA;
    // Every buffer is checked before anything is launched.
    if (!device_buffer(scene, scene_len * sizeof(double), dev, "scene", message, message_len) ||
        !device_buffer(index, index_len * sizeof(uint32_t), dev, "index", message, message_len) ||
        !device_buffer(result, 4 * sizeof(double), dev, "result", message, message_len))
      return TBA_ERROR_ARGUMENT;
    // Set-up, once per device and context, with that device current: the scratch's device address.
    CUcontext ctx = nullptr;
    if (g_context(&ctx) != CUDA_SUCCESS || !ctx) {
      say(message, message_len, "tba_scene_cost_noalloc: no current CUDA context");
      return TBA_ERROR_CUDA;
    }
    Scratch& slot = g_scratch[dev];
    if (slot.context != ctx || !slot.address) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_tile_partials);
      if (e != cudaSuccess) {
        say(message, message_len, cudaGetErrorString(e));
        return TBA_ERROR_CUDA;
      }
      slot.context = ctx;
      slot.address = static_cast<double*>(ptr);
    }
    scratch = slot.address;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_tile_cost<<<uint32_t(tiles), kThreads, 0, s>>>(scene, index, C, P, M, D, control->huber, scratch);
  k_tile_finish<<<1, kThreads, 0, s>>>(scratch, uint32_t(tiles), result);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    say(message, message_len, cudaGetErrorString(e));
    return TBA_ERROR_CUDA;
  }
  return TBA_OK;
}
