// Observation evaluation of a fixed scene (evaluateObservationsGpu,
// src/geometry/gpu/observations.ts:34-125; kernels of src/geometry/gpu/observation-evaluation.shade.ts),
// sm_100a, FP64.
//
//   k_obs_project   per observation: project the point in its camera; an inlier when the
//                   projection is in the model's domain and its error is within the threshold
//                   (projectIndexedObservations)
//   k_obs_depth     per track (only with a depth bound): the linearised depth sensitivity of the
//                   track's point to independent pixel noise, from its inlier observations with the
//                   poses and intrinsics fixed; a track above the bound loses all its inliers
//                   (filterIndexedObservationDepth, stableDepth).  One thread per track: groups of
//                   8 lanes per track measured slower (fewer independent tracks in flight per warp);
//                   capped at 64 registers for 8 blocks of 128 per SM (a few spilled words), which
//                   hides more of its gathers' latency: 0.925 -> 0.873 ms over 1M tracks and
//                   6.18M observations
//   k_obs_partials  the inlier error sum and count of each run of 64 observations, each run summed
//                   in order (indexedObservationPartials), then k_obs_summary sums the runs in a
//                   fixed tree (observationSummary)
//
// Layout (observationLayout, src/geometry/gpu/observation-layout.ts): one 18-word record per
// referenced camera (pose R row-major, t, then fx, fy, cx, cy, k1, k2), 3 words per point, 2 per
// observation pixel, and per observation its camera and point index interleaved.
#include <cuda_runtime.h>

#include <algorithm>

#include "tba_math.cuh"
#include "tba_observations.cuh"

namespace tba {
namespace {

__device__ inline void obs_camera(const ObsParams& A, uint32_t i, double pose[12], Camera& k) {
  const double* r = A.cameras + 18 * size_t(A.indices[2 * size_t(i)]);
  for (int j = 0; j < 12; j++) pose[j] = r[j];
  k = Camera{r[12], r[13], r[14], r[15], r[16], r[17]};
}

__device__ inline void obs_transform(const double pose[12], const double* X, double q[3]) {
  for (int r = 0; r < 3; r++) q[r] = pose[3 * r] * X[0] + pose[3 * r + 1] * X[1] + pose[3 * r + 2] * X[2] + pose[9 + r];
}

__global__ void __launch_bounds__(256) k_obs_project(ObsParams A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.M) return;
  A.flags[i] = 0;
  A.errors[i] = 0;
  double pose[12], q[3], pixel[2], du[3], dv[3];
  Camera k;
  obs_camera(A, i, pose, k);
  obs_transform(pose, A.points + 3 * size_t(A.indices[2 * size_t(i) + 1]), q);
  if (!project(k, q, pixel, du, dv)) return;
  const double x = pixel[0] - A.pixels[2 * size_t(i)], y = pixel[1] - A.pixels[2 * size_t(i) + 1];
  const double e = sqrt(x * x + y * y);
  if (e <= A.max_error) {
    A.flags[i] = 1;
    A.errors[i] = e;
  }
}

// stableDepth: the information matrix of the point from the inlier observations (unweighted point
// Jacobians), then for each inlier the variance of its camera-frame depth, sigma_z^2 = a^T A^-1 a
// with a the camera's optical axis, against the relative bound noise * sigma_z / z.
__device__ bool obs_stable_depth(const ObsParams& A, uint32_t start, uint32_t end, const double* X) {
  double M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t count = 0;
  for (uint32_t i = start; i < end; i++) {
    if (A.flags[i] == 0) continue;
    count++;
    double pose[12], q[3], pixel[2], du[3], dv[3];
    Camera k;
    obs_camera(A, i, pose, k);
    obs_transform(pose, X, q);
    if (!project(k, q, pixel, du, dv)) return false;
    for (int row = 0; row < 2; row++) {
      const double* g = row == 0 ? du : dv;
      const double J[3] = {g[0] * pose[0] + g[1] * pose[3] + g[2] * pose[6],
                           g[0] * pose[1] + g[1] * pose[4] + g[2] * pose[7],
                           g[0] * pose[2] + g[1] * pose[5] + g[2] * pose[8]};
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) M[3 * r + c] += J[r] * J[c];
    }
  }
  if (count < 2) return false;
  for (uint32_t i = start; i < end; i++) {
    if (A.flags[i] == 0) continue;
    double pose[12], q[3], s[3];
    Camera k;
    obs_camera(A, i, pose, k);
    const double axis[3] = {pose[6], pose[7], pose[8]};
    obs_transform(pose, X, q);
    if (!solve3_spd(M, axis, s) || !(q[2] > 0)) return false;
    const double variance = axis[0] * s[0] + axis[1] * s[1] + axis[2] * s[2];
    if (!(variance >= 0)) return false;
    const double relative = A.noise * sqrt(variance) / q[2];
    if (!(relative <= A.max_relative_depth)) return false;
  }
  return true;
}

__global__ void __launch_bounds__(128, 8) k_obs_depth(ObsParams A) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= A.P) return;
  const uint32_t start = A.offsets[h], end = A.offsets[h + 1];
  A.flags[A.M + h] = 0;
  if (end <= start) return;
  uint32_t accepted = 0;
  for (uint32_t i = start; i < end; i++) accepted += A.flags[i] != 0;
  if (accepted < 2) return;
  if (!obs_stable_depth(A, start, end, A.points + 3 * size_t(A.indices[2 * size_t(start) + 1]))) {
    A.flags[A.M + h] = 1;
    for (uint32_t i = start; i < end; i++) {
      A.flags[i] = 0;
      A.errors[i] = 0;
    }
  }
}

// One thread per run of 64 observations: its inlier error sum (in order) and inlier count.
__global__ void __launch_bounds__(256) k_obs_partials(ObsParams A) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t runs = (A.M + 63) / 64;
  if (b >= runs) return;
  double e = 0, n = 0;
  const uint32_t end = min(A.M, 64 * b + 64);
  for (uint32_t i = 64 * b; i < end; i++)
    if (A.flags[i] != 0) {
      e += A.errors[i];
      n += 1;
    }
  A.partials[2 * size_t(b)] = e;
  A.partials[2 * size_t(b) + 1] = n;
}

__global__ void __launch_bounds__(1024) k_obs_summary(ObsParams A) {
  __shared__ double se[1024], sn[1024];
  const uint32_t runs = (A.M + 63) / 64;
  double e = 0, n = 0;
  for (uint32_t b = threadIdx.x; b < runs; b += blockDim.x) {
    e += A.partials[2 * size_t(b)];
    n += A.partials[2 * size_t(b) + 1];
  }
  se[threadIdx.x] = e;
  sn[threadIdx.x] = n;
  __syncthreads();
  for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sn[threadIdx.x] += sn[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    A.summary[0] = se[0];
    A.summary[1] = sn[0];
  }
}

}  // namespace

void launch_observations(const ObsParams& a, cudaStream_t s) {
  if (a.M) k_obs_project<<<(a.M + 255) / 256, 256, 0, s>>>(a);
  if (a.guarded && a.P) k_obs_depth<<<(a.P + 127) / 128, 128, 0, s>>>(a);
  const uint32_t runs = (a.M + 63) / 64;
  if (runs) k_obs_partials<<<(runs + 255) / 256, 256, 0, s>>>(a);
  k_obs_summary<<<1, 1024, 0, s>>>(a);
}

}  // namespace tba

// ---- inverse-depth linearisation (linearizeInverseDepth, src/sfm/depth/gpu/inverse-depth.shade.ts) ----
//
// One row per thread.  Input row (34 words): the anchored point's parameters a, b, rho
// (normalised image coordinates and inverse depth in its reference camera), the reference pose
// (R row-major, t), the observing pose, the observing camera (fx, fy, cx, cy, k1, k2) and its
// squared radial limit.  Output row (23 words): valid flag, the projected pixel, the pixel's
// derivatives with respect to (a, b, rho) and to the observing pose's rotation and translation,
// and with respect to the log of a shared focal scale.  The point in the observing camera is
// q = a A0 + b A1 + A2 + rho T with A_k the observing rotation applied to the reference rotation's
// k-th row and T the observing rotation applied to the reference centre plus the observing
// translation: the point scaled by rho, so its projection is unchanged.
//
// The rows are 272 and 184 bytes long, so one thread per row reading its own row from global
// memory would touch 32 sectors per warp load.  Instead the kernel is persistent (two blocks per
// SM) and streams tiles of 128 rows through shared memory with the bulk-copy engine: the block's
// producer thread keeps two input tiles in flight (cp.async.bulk global -> shared, completion on
// an mbarrier per stage), the 128 threads compute one row each from shared memory into an output
// tile, and the producer writes the output tile back with one bulk store (cp.async.bulk
// shared -> global).  Every DRAM byte moves once, in whole lines, with no register cost for the
// bytes in flight (two blocks x two 34.8 KB tiles per SM).  Waits on an mbarrier are bounded: a
// wait that runs out sets the error word and the block stops.
namespace tba {
namespace {

constexpr int kIdRows = 128;
constexpr int kIdIn = 34, kIdOut = 23;
constexpr int kIdStages = 2;
constexpr uint32_t kIdTileIn = kIdRows * kIdIn * 8, kIdTileOut = kIdRows * kIdOut * 8;
constexpr size_t kIdSmem = size_t(kIdStages) * kIdTileIn + kIdTileOut + 64;
constexpr uint32_t kIdWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void id_bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

// One arrival that also announces `bytes` of transactions, then the bulk load that completes them.
__device__ __forceinline__ void id_load_tile(uint32_t bar, uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool id_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t k = 0; k < kIdWaitLimit; k++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void inverse_depth_row(const double* m, double* o) {
  for (int k = 0; k < kIdOut; k++) o[k] = 0;
  const double a = m[0], b = m[1], rho = m[2];
  double cx = 0, cy = 0, cz = 0;
  for (int k = 0; k < 3; k++) {
    cx -= m[3 + 3 * k] * m[12 + k];
    cy -= m[4 + 3 * k] * m[12 + k];
    cz -= m[5 + 3 * k] * m[12 + k];
  }
  double A0[3], A1[3], A2[3], T[3];
  for (int row = 0; row < 3; row++) {
    const double r0 = m[15 + 3 * row], r1 = m[16 + 3 * row], r2 = m[17 + 3 * row];
    A0[row] = r0 * m[3] + r1 * m[4] + r2 * m[5];
    A1[row] = r0 * m[6] + r1 * m[7] + r2 * m[8];
    A2[row] = r0 * m[9] + r1 * m[10] + r2 * m[11];
    T[row] = (r0 * cx + r1 * cy + r2 * cz) + m[24 + row];
  }
  double q[3];
  for (int r = 0; r < 3; r++) q[r] = a * A0[r] + b * A1[r] + A2[r] + rho * T[r];
  if (!(q[2] > 0.000000000001)) return;
  const double x = q[0] / q[2], y = q[1] / q[2], r2 = x * x + y * y;
  const double fx = m[27], fy = m[28], k1 = m[31], k2 = m[32];
  if (!(r2 < m[33])) return;
  const double d = 1. + k1 * r2 + k2 * r2 * r2;
  if (!(d > 0. && 1. + 3. * k1 * r2 + 5. * k2 * r2 * r2 > 0.)) return;
  const double g = 2. * (k1 + 2. * k2 * r2);
  const double xx = d + g * x * x, xy = g * x * y, yy = d + g * y * y;
  const double J0[3] = {fx * xx / q[2], fx * xy / q[2], -fx * (xx * x + xy * y) / q[2]};
  const double J1[3] = {fy * xy / q[2], fy * yy / q[2], -fy * (xy * x + yy * y) / q[2]};
  o[0] = 1.;
  o[1] = fx * x * d + m[29];
  o[2] = fy * y * d + m[30];
  for (int row = 0; row < 2; row++) {
    const double* J = row == 0 ? J0 : J1;
    o[3 + row * 3] = J[0] * A0[0] + J[1] * A0[1] + J[2] * A0[2];
    o[4 + row * 3] = J[0] * A1[0] + J[1] * A1[1] + J[2] * A1[2];
    o[5 + row * 3] = J[0] * T[0] + J[1] * T[1] + J[2] * T[2];
    double* at = o + 9 + row * 6;
    at[0] = -J[1] * q[2] + J[2] * q[1];
    at[1] = J[0] * q[2] - J[2] * q[0];
    at[2] = -J[0] * q[1] + J[1] * q[0];
    at[3] = rho * J[0];
    at[4] = rho * J[1];
    at[5] = rho * J[2];
  }
  o[21] = fx * x * d;
  o[22] = fy * y * d;
}

// Tiles of kIdRows rows; tile k starts at row k * kIdRows, so both tiles' global addresses are
// 16-byte aligned when the arrays are, and an input tile (n * 272 bytes) is whole 16-byte words.
// An output tile (n * 184 bytes) is whole 16-byte words but for a last 8 bytes when n is odd; those
// are written with a plain store.
__global__ void __launch_bounds__(kIdRows) k_linearize_inverse_depth(uint32_t count, const double* __restrict__ in,
                                                                      double* __restrict__ out, uint32_t* error) {
  extern __shared__ __align__(128) unsigned char id_smem[];
  double* stage = reinterpret_cast<double*>(id_smem);
  double* tile_out = reinterpret_cast<double*>(id_smem + kIdStages * size_t(kIdTileIn));
  uint64_t* bars = reinterpret_cast<uint64_t*>(id_smem + kIdStages * size_t(kIdTileIn) + kIdTileOut);
  __shared__ uint32_t abort_flag;
  const uint32_t tiles = (count + kIdRows - 1) / kIdRows;
  const bool producer = threadIdx.x == 0;
  auto rows_of = [&](uint32_t tile) { return min(uint32_t(kIdRows), count - tile * kIdRows); };
  if (producer) {
    abort_flag = 0;
    for (int k = 0; k < kIdStages; k++) id_bar_init(smem_addr(bars + k));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int k = 0; k < kIdStages; k++) {
      const uint32_t tile = blockIdx.x + k * gridDim.x;
      if (tile < tiles)
        id_load_tile(smem_addr(bars + k), smem_addr(stage + size_t(k) * kIdRows * kIdIn),
                     in + size_t(tile) * kIdRows * kIdIn, rows_of(tile) * kIdIn * 8);
    }
  }
  __syncthreads();
  uint32_t k = 0, tile = blockIdx.x;
  for (; tile < tiles; tile += gridDim.x, k++) {
    const uint32_t s = k % kIdStages, parity = (k / kIdStages) & 1;
    const uint32_t n = rows_of(tile);
    if (!id_wait(smem_addr(bars + s), parity)) {
      atomicExch(error, 1u);
      abort_flag = 1;
    }
    // The previous tile's bulk store has to have read the output tile before it is rewritten.
    if (producer) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    __syncthreads();
    if (abort_flag) break;
    double* rows = stage + size_t(s) * kIdRows * kIdIn;
    if (threadIdx.x < n) inverse_depth_row(rows + threadIdx.x * kIdIn, tile_out + threadIdx.x * kIdOut);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (producer) {
      double* dst = out + size_t(tile) * kIdRows * kIdOut;
      const uint32_t bytes = n * kIdOut * 8, whole = bytes & ~15u;
      asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(tile_out)),
                   "r"(whole)
                   : "memory");
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      if (whole != bytes) dst[n * kIdOut - 1] = tile_out[n * kIdOut - 1];
      // Refill this stage with the tile kIdStages turns ahead: every thread has finished reading it.
      const uint32_t next = tile + kIdStages * gridDim.x;
      if (next < tiles)
        id_load_tile(smem_addr(bars + s), smem_addr(rows), in + size_t(next) * kIdRows * kIdIn,
                     rows_of(next) * kIdIn * 8);
    }
  }
  // After a load that did not complete in time, let this block's loads still in flight (the
  // aborted tile's and those issued ahead of it) land before its shared memory is released; each
  // wait is bounded.
  if (abort_flag && producer)
    for (uint32_t j = 0; j < uint32_t(kIdStages); j++)
      if (tile + j * gridDim.x < tiles) id_wait(smem_addr(bars + (k + j) % kIdStages), ((k + j) / kIdStages) & 1);
  if (producer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace

cudaError_t launch_linearize_inverse_depth(uint32_t count, const double* in, double* out, uint32_t* error,
                                           int sms, cudaStream_t s) {
  if (!count) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(k_linearize_inverse_depth, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kIdSmem));
  if (e != cudaSuccess) return e;
  const uint32_t tiles = (count + kIdRows - 1) / kIdRows;
  const uint32_t grid = std::min<uint32_t>(tiles, 2u * uint32_t(sms > 0 ? sms : 1));
  k_linearize_inverse_depth<<<grid, kIdRows, kIdSmem, s>>>(count, in, out, error);
  return cudaGetLastError();
}

}  // namespace tba
