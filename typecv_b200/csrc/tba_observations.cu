// Observation evaluation of a fixed scene (evaluateObservationsGpu,
// src/geometry/gpu/observations.ts:34-125; kernels of src/geometry/gpu/observation-evaluation.shade.ts),
// sm_100a, FP64.
//
//   k_obs_project   per observation: project the point in its camera; an inlier when the
//                   projection is in the model's domain and its error is within the threshold
//                   (projectIndexedObservations)
//   k_obs_tracks    with a depth bound: projectIndexedObservations fused with the depth filter
//                   (filterIndexedObservationDepth, stableDepth): the linearised depth sensitivity
//                   of each track's point to independent pixel noise, from its inlier
//                   observations with the poses and intrinsics fixed; a track above the bound
//                   loses all its inliers.  Observation-parallel: warp tasks of whole tracks (at
//                   most 32 observations, one per lane; a longer track is a task of its own, swept
//                   in rounds), the tracks' 3x3 information matrices summed by segmented warp
//                   scans, every inlier's depth variance checked in its own lane, and a track's
//                   verdict formed by a warp vote.  Each observation is read once and its flag and
//                   error written once.
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
#include "tba_warp.cuh"

namespace tba {
namespace {

constexpr unsigned kObsFull = 0xffffffffu;

__device__ inline void warp_sum7(double (&v)[7]) {
  for (int d = 16; d > 0; d >>= 1)
    for (int c = 0; c < 7; c++) v[c] += __shfl_xor_sync(kObsFull, v[c], d);
}

// The 18-word camera record of observation i, as nine 16-byte loads (records start 144-byte
// aligned in a 16-byte aligned array).
__device__ inline void obs_camera(const ObsParams& A, uint32_t i, double pose[12], Camera& k) {
  const double2* r = reinterpret_cast<const double2*>(A.cameras + 18 * size_t(A.indices[2 * size_t(i)]));
  double w[18];
  for (int j = 0; j < 9; j++) {
    const double2 d = __ldg(r + j);
    w[2 * j] = d.x;
    w[2 * j + 1] = d.y;
  }
  for (int j = 0; j < 12; j++) pose[j] = w[j];
  k = Camera{w[12], w[13], w[14], w[15], w[16], w[17]};
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

// The point Jacobian rows' information (J^T J, 6 unique) from the projection's derivative rows.
__device__ inline void information_rows(const double pose[12], const double du[3], const double dv[3], double (&v)[6]) {
  for (int n = 0; n < 6; n++) v[n] = 0;
  for (int row = 0; row < 2; row++) {
    const double* g = row == 0 ? du : dv;
    const double J[3] = {g[0] * pose[0] + g[1] * pose[3] + g[2] * pose[6], g[0] * pose[1] + g[1] * pose[4] + g[2] * pose[7],
                         g[0] * pose[2] + g[1] * pose[5] + g[2] * pose[8]};
    v[0] += J[0] * J[0];
    v[1] += J[0] * J[1];
    v[2] += J[0] * J[2];
    v[3] += J[1] * J[1];
    v[4] += J[1] * J[2];
    v[5] += J[2] * J[2];
  }
}

// The information and camera-frame depth of one observation of a track's point X; false when the
// projection leaves the model's domain.
__device__ inline bool obs_information(const double pose[12], const Camera& k, const double* X, double (&v)[6],
                                       double& depth) {
  double q[3], pixel[2], du[3], dv[3];
  obs_transform(pose, X, q);
  depth = q[2];
  if (!project(k, q, pixel, du, dv)) return false;
  information_rows(pose, du, dv, v);
  return true;
}

// One inlier's share of stableDepth's verdict: its depth's relative standard deviation within the
// bound, from the track's information v (6 unique) and the inlier's camera axis.
__device__ inline bool obs_depth_ok(const ObsParams& A, const double (&v)[6], const double pose[12], double depth) {
  const double M[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  const double axis[3] = {pose[6], pose[7], pose[8]};
  double s[3];
  if (!solve3_spd(M, axis, s) || !(depth > 0)) return false;
  const double variance = axis[0] * s[0] + axis[1] * s[1] + axis[2] * s[2];
  if (!(variance >= 0)) return false;
  return A.noise * sqrt(variance) / depth <= A.max_relative_depth;
}

// One observation's projection against its pixel: inlier flag and error (projectIndexedObservations).
__device__ inline bool obs_inlier(const ObsParams& A, uint32_t i, const double pose[12], const Camera& k, double& e) {
  double q[3], pixel[2], du[3], dv[3];
  obs_transform(pose, A.points + 3 * size_t(A.indices[2 * size_t(i) + 1]), q);
  e = 0;
  if (!project(k, q, pixel, du, dv)) return false;
  const double x = pixel[0] - A.pixels[2 * size_t(i)], y = pixel[1] - A.pixels[2 * size_t(i) + 1];
  e = sqrt(x * x + y * y);
  return e <= A.max_error;
}

__global__ void __launch_bounds__(256, 2) k_obs_tracks(ObsParams A) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < A.ntasks; t += warps) {
    const uint32_t h0 = A.tasks[t], h1 = A.tasks[t + 1];
    const uint32_t o0 = A.offsets[h0], n = A.offsets[h1] - o0;
    if (n <= 32) {
      // The task's tracks: a head bit at each non-empty track's first observation.
      unsigned heads = 0;
      for (uint32_t base = h0; base < h1; base += 32) {
        const uint32_t h = base + uint32_t(lane);
        unsigned bit = 0;
        if (h < h1 && A.offsets[h + 1] > A.offsets[h]) bit = 1u << (A.offsets[h] - o0);
        heads |= __reduce_or_sync(kObsFull, bit);
      }
      const bool valid = uint32_t(lane) < n;
      const uint32_t i = o0 + (valid ? uint32_t(lane) : 0u);
      const int head = valid ? 31 - __clz(heads & (kObsFull >> (31 - lane))) : lane;
      // One projection per observation: its inlier flag and error, and (for an inlier of the
      // track's own point, the usual case) its information and depth.
      double pose[12], q[3], pixel[2], du[3], dv[3], e = 0;
      Camera k;
      obs_camera(A, i, pose, k);
      const uint32_t pi = A.indices[2 * size_t(i) + 1];
      obs_transform(pose, A.points + 3 * size_t(pi), q);
      bool inlier = valid && project(k, q, pixel, du, dv);
      if (inlier) {
        const double x = pixel[0] - A.pixels[2 * size_t(i)], y = pixel[1] - A.pixels[2 * size_t(i) + 1];
        e = sqrt(x * x + y * y);
        inlier = e <= A.max_error;
      }
      // The track's point is its first observation's.
      const uint32_t xi = __shfl_sync(kObsFull, pi, head);
      double v[7] = {0, 0, 0, 0, 0, 0, 0}, depth = q[2];
      bool projected = true;
      if (inlier) {
        double w[6];
        if (xi == pi) information_rows(pose, du, dv, w);
        else projected = obs_information(pose, k, A.points + 3 * size_t(xi), w, depth);
        for (int c = 0; c < 6; c++) v[c] = projected ? w[c] : 0.0;
        v[6] = 1;
      }
      const int seg = valid ? head : -1 - lane;
      const Runs runs = lane_runs(seg, lane);
      run_scan(v, runs);
      const bool tail = valid && run_tail(runs, lane);
      const unsigned tails = __ballot_sync(kObsFull, tail);
      const int src = valid ? __ffs(tails & (kObsFull << lane)) - 1 : lane;
      for (int c = 0; c < 7; c++) v[c] = __shfl_sync(kObsFull, v[c], src);
      // Tracks with fewer than two inliers are not filtered.
      const bool checked = v[6] >= 2;
      bool ok = true;
      if (inlier && checked) {
        const double w[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
        ok = projected && obs_depth_ok(A, w, pose, depth);
      }
      const unsigned failed = __ballot_sync(kObsFull, inlier && checked && !ok);
      // This lane's track: lanes head .. src.
      const unsigned span = valid ? ((src == 31 ? kObsFull : ((1u << (src + 1)) - 1u)) & (kObsFull << head)) : 0u;
      const bool rejected = (failed & span) != 0;
      if (valid) {
        const bool keep = inlier && !rejected;
        A.flags[i] = keep ? 1u : 0u;
        A.errors[i] = keep ? e : 0.0;
      }
      // Track flags: the head lane's verdict; empty tracks keep 0.
      const unsigned verdicts = __ballot_sync(kObsFull, valid && uint32_t(lane) == uint32_t(head) && rejected);
      for (uint32_t base = h0; base < h1; base += 32) {
        const uint32_t h = base + uint32_t(lane);
        if (h < h1) {
          const uint32_t start = A.offsets[h];
          A.flags[A.M + h] = (A.offsets[h + 1] > start && ((verdicts >> (start - o0)) & 1u)) ? 1u : 0u;
        }
      }
      continue;
    }
    // One track longer than 32 observations: rounds of 32 lanes.
    const uint32_t xi = A.indices[2 * size_t(o0) + 1];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    bool projected = true;
    for (uint32_t base = 0; base < n; base += 32) {
      const uint32_t i = o0 + base + uint32_t(lane);
      if (i >= o0 + n) continue;
      double pose[12], e, depth;
      Camera k;
      obs_camera(A, i, pose, k);
      const bool inlier = obs_inlier(A, i, pose, k, e);
      A.flags[i] = inlier ? 1u : 0u;
      A.errors[i] = inlier ? e : 0.0;
      if (inlier) {
        double w[6];
        if (obs_information(pose, k, A.points + 3 * size_t(xi), w, depth))
          for (int c = 0; c < 6; c++) v[c] += w[c];
        else
          projected = false;
        v[6] += 1;
      }
    }
    warp_sum7(v);
    const bool all_projected = __all_sync(kObsFull, projected);
    bool ok = true;
    if (v[6] >= 2) {
      const double w[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
      for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t i = o0 + base + uint32_t(lane);
        if (i >= o0 + n || A.flags[i] == 0) continue;
        double pose[12], q[3];
        Camera k;
        obs_camera(A, i, pose, k);
        obs_transform(pose, A.points + 3 * size_t(xi), q);
        if (!obs_depth_ok(A, w, pose, q[2])) ok = false;
      }
      ok = __all_sync(kObsFull, ok) && all_projected;
    }
    if (lane == 0) A.flags[A.M + h0] = ok ? 0u : 1u;
    if (!ok)
      for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t i = o0 + base + uint32_t(lane);
        if (i < o0 + n) {
          A.flags[i] = 0;
          A.errors[i] = 0;
        }
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
  if (a.guarded && a.ntasks) k_obs_tracks<<<(a.ntasks + 7) / 8, 256, 0, s>>>(a);
  else if (a.M) k_obs_project<<<(a.M + 255) / 256, 256, 0, s>>>(a);
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
// wait that runs out sets the error word to 1 and the block stops, after waiting (with the full
// bound) for its own loads still in flight; a wait of that drain that runs out too sets it to 2.
// The main-loop waits poll at most `wait_limit` times (kIdWaitLimit unless a test shortens it to
// make them run out); the drain always uses kIdWaitLimit.
namespace tba {
namespace {

constexpr int kIdRows = 128;
constexpr int kIdIn = 34, kIdOut = 23;
constexpr int kIdStages = 2;
constexpr uint32_t kIdTileIn = kIdRows * kIdIn * 8, kIdTileOut = kIdRows * kIdOut * 8;
constexpr size_t kIdSmem = size_t(kIdStages) * kIdTileIn + kIdTileOut + 64;
constexpr uint32_t kIdWaitLimit = kIdWaitPolls;

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

__device__ __forceinline__ bool id_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t k = 0; k < limit; k++) {
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
                                                                      double* __restrict__ out, uint32_t* error,
                                                                      uint32_t wait_limit) {
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
    if (!id_wait(smem_addr(bars + s), parity, wait_limit)) {
      atomicMax(error, 1u);
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
  // wait is bounded, and one that runs out is recorded as a drain failure (2).
  if (abort_flag && producer)
    for (uint32_t j = 0; j < uint32_t(kIdStages); j++)
      if (tile + j * gridDim.x < tiles &&
          !id_wait(smem_addr(bars + (k + j) % kIdStages), ((k + j) / kIdStages) & 1, kIdWaitLimit))
        atomicMax(error, 2u);
  if (producer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace

cudaError_t launch_linearize_inverse_depth(uint32_t count, const double* in, double* out, uint32_t* error,
                                           int sms, cudaStream_t s, uint32_t wait_limit) {
  if (!count) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(k_linearize_inverse_depth, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kIdSmem));
  if (e != cudaSuccess) return e;
  const uint32_t tiles = (count + kIdRows - 1) / kIdRows;
  const uint32_t grid = std::min<uint32_t>(tiles, 2u * uint32_t(sms > 0 ? sms : 1));
  k_linearize_inverse_depth<<<grid, kIdRows, kIdSmem, s>>>(count, in, out, error, wait_limit);
  return cudaGetLastError();
}

}  // namespace tba
