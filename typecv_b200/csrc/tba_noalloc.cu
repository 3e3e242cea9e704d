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

std::mutex g_setup;
double* g_scratch[kMaxDevices] = {};  // device address of g_tile_partials, per device ordinal

void say(char* message, size_t len, const char* text) {
  if (message && len) {
    std::strncpy(message, text, len - 1);
    message[len - 1] = 0;
  }
}

}  // namespace

extern "C" tba_status tba_scene_cost_noalloc(const tba_control* control, const double* scene, const uint32_t* index,
                                             double* result, void* stream, char* message, size_t message_len) {
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
  if (reinterpret_cast<uintptr_t>(scene) % alignof(double) || reinterpret_cast<uintptr_t>(index) % alignof(uint32_t) ||
      reinterpret_cast<uintptr_t>(result) % alignof(double)) {
    say(message, message_len, "tba_scene_cost_noalloc: misaligned device pointer");
    return TBA_ERROR_ARGUMENT;
  }
  // Set-up, once per device, with that device current: the scratch's device address.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    say(message, message_len, e != cudaSuccess ? cudaGetErrorString(e) : "tba_scene_cost_noalloc: device ordinal >= 64");
    return e != cudaSuccess ? TBA_ERROR_CUDA : TBA_ERROR_ARGUMENT;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup);
    if (!g_scratch[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_tile_partials);
      if (e != cudaSuccess) {
        say(message, message_len, cudaGetErrorString(e));
        return TBA_ERROR_CUDA;
      }
      g_scratch[dev] = static_cast<double*>(ptr);
    }
    scratch = g_scratch[dev];
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
