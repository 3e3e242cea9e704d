// Kernels of the grid engine (one bundle adjustment over the whole GPU), sm_100a, FP64.
//
// Kernel                 reference kernel(s) it replaces (src/sfm/bundle/gpu/*.shade.ts)
// k_initialize           initializeBundle (K1)
// k_cost/k_finish_metrics bundleMetricPartials + finishBundleMetrics (K3/K4)
// k_point_pass           linearizeBundle + bundlePointBlocks + bundleFocalObservations +
//                        bundleFocalPoints (K2/K5/K21)
// k_camera_pass/_finish  bundleCameraRows + bundleFocalCameraRows + invertBundleCameraColumns +
//                        finalizeBundleCameraInverse (K6/K8/K21)
// k_pcg_init             dampBundleFocal + initializeBundleCg (K9/K21)
// k_product/_finish      bundleSchurPoint + bundleSchurCamera (+ focal row) + advanceBundleCg
//                        (K10/K11/K12): one pass over W with per-block shared-memory camera
//                        accumulators, then a reduction of the block partials whose last block
//                        runs the PCG step
// k_update_cameras       updateBundleCandidate (cameras, focal) + bundleCandidateGauge +
//                        normalizeBundleCandidate (cameras) (K14/K15/K16)
// k_update_points        updateBundleCandidate (points) + normalizeBundleCandidate (points) +
//                        bundleCandidatePartials (K14/K16/K17)
// k_accept/k_commit      acceptBundleCandidate + commitBundleCandidate (K18/K19)
// k_pack                 packBundleResult (K20)
//
// Every reduction runs in a fixed order (fixed grids, fixed trees), so a solve is reproducible
// run to run, except the shared-memory accumulation of the Schur product, whose FP64 atomic
// adds commute only up to rounding.
#include <cuda_runtime.h>

#include "tba_engine.cuh"

// Compile-time tuning of the heavy kernels (occupancy floors of __launch_bounds__, and whether
// the Schur product keeps a lane's W block in registers between its two uses or re-reads it
// from L1 for the scatter).
#ifndef TBA_PRODUCT_MIN_BLOCKS
#define TBA_PRODUCT_MIN_BLOCKS 2
#endif
#ifndef TBA_PRODUCT_RELOAD
#define TBA_PRODUCT_RELOAD 1
#endif
#ifndef TBA_POINT_MIN_BLOCKS
#define TBA_POINT_MIN_BLOCKS 2
#endif
#ifndef TBA_CAMERA_MIN_BLOCKS
#define TBA_CAMERA_MIN_BLOCKS 3
#endif

namespace tba {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ inline Camera camera_at(const Params& P, uint32_t c, double log_scale) {
  const double* k = P.cams + 6 * size_t(c);
  Camera cam{k[0], k[1], k[2], k[3], k[4], k[5]};
  if (P.shared) {
    const double s = exp(log_scale);
    cam.fx *= s;
    cam.fy *= s;
  }
  return cam;
}

__device__ inline void load_pose(const double* poses, uint32_t c, double out[12]) {
  const double2* src = reinterpret_cast<const double2*>(poses + 12 * size_t(c));
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const double2 v = src[k];
    out[2 * k] = v.x;
    out[2 * k + 1] = v.y;
  }
}

// Inclusive segmented sum over lanes: lanes with equal `seg` form contiguous runs.
template <int N>
__device__ inline void seg_scan(double (&v)[N], int seg, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int s = __shfl_up_sync(kFull, seg, d);
    double t[N];
#pragma unroll
    for (int n = 0; n < N; n++) t[n] = __shfl_up_sync(kFull, v[n], d);
    if (lane >= d && s == seg) {
#pragma unroll
      for (int n = 0; n < N; n++) v[n] += t[n];
    }
  }
}

template <int N>
__device__ inline void warp_allsum(double (&v)[N]) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
    for (int n = 0; n < N; n++) v[n] += __shfl_xor_sync(kFull, v[n], d);
  }
}

// Sum N values over the block in a fixed order; the result is valid in thread 0.
template <int N>
__device__ inline void block_sum(double (&v)[N], double* smem) {
  warp_allsum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int n = 0; n < N; n++) smem[warp * N + n] = v[n];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; n++) {
      double s = 0;
      for (int w = 0; w < nwarps; w++) s += smem[w * N + n];
      v[n] = s;
    }
  }
  __syncthreads();
}

// The tasks [begin, end) of this block: a contiguous share of the task list.
__device__ inline void block_tasks(const Params& P, uint32_t& begin, uint32_t& end) {
  begin = uint32_t(uint64_t(P.ntasks) * blockIdx.x / gridDim.x);
  end = uint32_t(uint64_t(P.ntasks) * (blockIdx.x + 1) / gridDim.x);
}

__device__ inline bool directional(const Params& P, uint32_t pt) { return pt >= P.P - P.D; }

// ---- K1: initializeBundle ----------------------------------------------------------------------

__global__ void k_initialize(Params P) {
  double* st = P.state;
  for (int j = 0; j < S_WORDS; j++) st[j] = 0;
  st[S_LAMBDA] = 1e-3;
  st[S_ACTIVE] = 1;
  double o[3], s[3];
  const double* a = P.poses + 12 * size_t(P.anchor);
  const double* b = P.poses + 12 * size_t(P.scale_view);
  for (int i = 0; i < 3; i++) {
    o[i] = -a[i] * a[9] - a[i + 3] * a[10] - a[i + 6] * a[11];
    s[i] = -b[i] * b[9] - b[i + 3] * b[10] - b[i + 6] * b[11];
  }
  const double baseline = sqrt((o[0] - s[0]) * (o[0] - s[0]) + (o[1] - s[1]) * (o[1] - s[1]) +
                               (o[2] - s[2]) * (o[2] - s[2]));
  st[S_BASELINE] = baseline;
  for (int i = 0; i < 3; i++) st[S_ORIGIN + i] = o[i];
  if (!(baseline > 1e-10)) {
    st[S_INPUT_ERROR] = 1;
    st[S_ACTIVE] = 0;
  }
  for (int k = 0; k < 8; k++) P.ticket[k] = 0;
}

// ---- K3/K4: the linearised cost of the scene ---------------------------------------------------

__global__ void __launch_bounds__(kPointThreads) k_cost(Params P) {
  __shared__ double red[3 * (kPointThreads / 32)];
  double v[3] = {0, 0, 0};  // cost, squared error, invalid projections
  const double logf = P.state[S_LOG_FOCAL];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.M; i += gridDim.x * blockDim.x) {
    const uint32_t c = P.obs_camera[i], pt = P.obs_point[i];
    double pose[12];
    load_pose(P.poses, c, pose);
    const Camera k = camera_at(P, c, logf);
    const double* X = P.points + 3 * size_t(pt);
    const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
    double cost, sq;
    double q[3];
    const bool dir = directional(P, pt);
    for (int j = 0; j < 3; j++) {
      q[j] = pose[j * 3] * X[0] + pose[j * 3 + 1] * X[1] + pose[j * 3 + 2] * X[2];
      if (!dir) q[j] += pose[9 + j];
    }
    double pixel[2], du[3], dv[3];
    if (!project(k, q, pixel, du, dv)) {
      v[2] += 1;
      continue;
    }
    const double ru = pixel[0] - uv.x, rv = pixel[1] - uv.y;
    sq = ru * ru + rv * rv;
    cost = robust_cost(sqrt(sq), P.huber);
    v[0] += cost;
    v[1] += sq;
  }
  block_sum(v, red);
  if (threadIdx.x == 0)
    for (int n = 0; n < 3; n++) P.cost_part[4 * blockIdx.x + n] = v[n];
}

__global__ void k_finish_metrics(Params P) {
  __shared__ double red[3 * 32];
  double* st = P.state;
  double v[3] = {0, 0, 0};
  for (uint32_t b = threadIdx.x; b < P.task_blocks; b += blockDim.x)
    for (int n = 0; n < 3; n++) v[n] += P.cost_part[4 * b + n];
  block_sum(v, red);
  if (threadIdx.x != 0 || st[S_INPUT_ERROR] != 0) return;
  if (v[2] > 0) {
    st[S_INPUT_ERROR] = 2;
    st[S_ACTIVE] = 0;
    return;
  }
  st[S_COST] = st[S_COST0] = v[0];
  st[S_SSE] = st[S_SSE0] = v[1];
  if (v[0] < 1e-20) st[S_ACTIVE] = 0;
}

// ---- K2/K5/K21: linearisation and point blocks -------------------------------------------------

// One observation of the point pass: its contributions to the point block (V 6 unique,
// b_p 3, focal cross sum 3, invalid 1) and its W_i, written to the component-major store.
template <bool SHARED>
__device__ inline void point_obs(const Params& P, uint32_t i, uint32_t pt, double logf,
                                 double (&v)[13], double& hff, double& bf) {
  const uint32_t c = P.obs_camera[i];
  double pose[12];
  load_pose(P.poses, c, pose);
  const Camera k = camera_at(P, c, logf);
  const double* X = P.points + 3 * size_t(pt);
  const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
  ObsLin o;
  const size_t M = P.M;
  if (!linearize(pose, k, X, P.active[c] != 0, directional(P, pt), uv.x, uv.y, P.huber, o)) {
    v[12] = 1;
    for (uint32_t n = 0; n < P.wdim; n++) P.W[n * M + i] = 0;
    return;
  }
  const double w = o.w;
  double wjp[2][3];
#pragma unroll
  for (int row = 0; row < 2; row++)
#pragma unroll
    for (int j = 0; j < 3; j++) wjp[row][j] = w * o.jp[row][j];
  v[0] = wjp[0][0] * o.jp[0][0] + wjp[1][0] * o.jp[1][0];
  v[1] = wjp[0][0] * o.jp[0][1] + wjp[1][0] * o.jp[1][1];
  v[2] = wjp[0][0] * o.jp[0][2] + wjp[1][0] * o.jp[1][2];
  v[3] = wjp[0][1] * o.jp[0][1] + wjp[1][1] * o.jp[1][1];
  v[4] = wjp[0][1] * o.jp[0][2] + wjp[1][1] * o.jp[1][2];
  v[5] = wjp[0][2] * o.jp[0][2] + wjp[1][2] * o.jp[1][2];
#pragma unroll
  for (int j = 0; j < 3; j++) v[6 + j] = -(wjp[0][j] * o.r[0] + wjp[1][j] * o.r[1]);
#pragma unroll
  for (int kk = 0; kk < 6; kk++)
#pragma unroll
    for (int j = 0; j < 3; j++) P.W[(kk * 3 + j) * M + i] = o.jc[0][kk] * wjp[0][j] + o.jc[1][kk] * wjp[1][j];
  if (SHARED) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      v[9 + j] = o.jf[0] * wjp[0][j] + o.jf[1] * wjp[1][j];
      P.W[(18 + j) * M + i] = v[9 + j];
    }
    hff += w * (o.jf[0] * o.jf[0] + o.jf[1] * o.jf[1]);
    bf += w * (o.jf[0] * o.r[0] + o.jf[1] * o.r[1]);
  }
}

// The point block of `pt` from its summed contributions: damping, equilibrated inverse,
// right-hand side, and the point's share of the focal diagonal and right-hand side.
template <bool SHARED>
__device__ inline void point_finish(const Params& P, uint32_t pt, const double (&v)[13], double lambda,
                                    double& diag_pt, double& rhs_pt) {
  double V[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  for (int j = 0; j < 3; j++) V[j * 4] += lambda * fmax(V[j * 4], 1e-10);
  double inv[6];
  const bool ok = v[12] == 0 && inverse3_spd(V, inv);
  const size_t Pn = P.P;
  if (!ok) {
    P.state[S_POINT_FAILED] = 1;
    for (int k = 0; k < 6; k++) P.vinv[k * Pn + pt] = 0;
    for (int k = 0; k < 3; k++) P.bp[k * Pn + pt] = 0;
    return;
  }
  for (int k = 0; k < 6; k++) P.vinv[k * Pn + pt] = inv[k];
  for (int k = 0; k < 3; k++) P.bp[k * Pn + pt] = v[6 + k];
  if (SHARED) {
    const double I[9] = {inv[0], inv[1], inv[2], inv[1], inv[3], inv[4], inv[2], inv[4], inv[5]};
    for (int j = 0; j < 3; j++) {
      const double t = v[9] * I[j] + v[10] * I[3 + j] + v[11] * I[6 + j];
      diag_pt += t * v[9 + j];
      rhs_pt += t * v[6 + j];
    }
  }
}

template <bool SHARED>
__global__ void __launch_bounds__(kPointThreads, TBA_POINT_MIN_BLOCKS) k_point_pass(Params P) {
  __shared__ double red[kScalarPartials * (kPointThreads / 32)];
  if (P.state[S_ACTIVE] == 0) return;
  const double lambda = P.state[S_LAMBDA], logf = P.state[S_LOG_FOCAL];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double sc[kScalarPartials] = {0, 0, 0, 0};  // hff, bf, diag_pt, rhs_pt (lane-local)
  uint32_t tb, te;
  block_tasks(P, tb, te);
  for (uint32_t t = tb + warp; t < te; t += nwarps) {
    const uint32_t p0 = P.tasks[t], p1 = P.tasks[t + 1];
    const uint32_t o0 = P.point_start[p0], n = P.point_start[p1] - o0;
    if (n <= uint32_t(kTaskObs)) {
      double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      int seg = -1 - lane;
      uint32_t pt = 0;
      if (uint32_t(lane) < n) {
        pt = P.obs_point[o0 + lane];
        seg = int(pt - p0);
        point_obs<SHARED>(P, o0 + lane, pt, logf, v, sc[0], sc[1]);
      }
      seg_scan(v, seg, lane);
      const int next = __shfl_down_sync(kFull, seg, 1);
      if (uint32_t(lane) < n && (uint32_t(lane) == n - 1 || next != seg))
        point_finish<SHARED>(P, pt, v, lambda, sc[2], sc[3]);
    } else {
      double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs) {
        if (base + lane < n) {
          double u[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
          point_obs<SHARED>(P, o0 + base + lane, p0, logf, u, sc[0], sc[1]);
          for (int k = 0; k < 13; k++) v[k] += u[k];
        }
      }
      warp_allsum(v);
      if (lane == 0) point_finish<SHARED>(P, p0, v, lambda, sc[2], sc[3]);
    }
  }
  block_sum(sc, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kScalarPartials; k++) P.scal_part[kScalarPartials * blockIdx.x + k] = sc[k];
}

// ---- K6/K8/K21: camera blocks ------------------------------------------------------------------

__global__ void __launch_bounds__(kCameraThreads, TBA_CAMERA_MIN_BLOCKS) k_camera_pass(Params P) {
  __shared__ double red[kCameraPartials * (kCameraThreads / 32)];
  if (P.state[S_ACTIVE] == 0) return;
  const uint32_t ch = blockIdx.x, c = P.chunk_cam[ch];
  if (P.active[c] == 0) return;
  const uint32_t k0 = P.chunk_beg[ch], k1 = P.chunk_beg[ch + 1];
  double pose[12];
  load_pose(P.poses, c, pose);
  const Camera cam = camera_at(P, c, P.state[S_LOG_FOCAL]);
  const size_t Pn = P.P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // Pass 1: U_c (lower triangle), b_c, H_cf.
  {
    double a[33];
    for (int j = 0; j < 33; j++) a[j] = 0;
    for (uint32_t kk = k0 + threadIdx.x; kk < k1; kk += blockDim.x) {
      const uint32_t i = P.camera_obs[kk], pt = P.obs_point[i];
      const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
      ObsLin o;
      if (!linearize(pose, cam, P.points + 3 * size_t(pt), true, directional(P, pt), uv.x, uv.y, P.huber, o))
        continue;
      double wjc[2][6];
      for (int row = 0; row < 2; row++)
        for (int j = 0; j < 6; j++) wjc[row][j] = o.w * o.jc[row][j];
      for (int j = 0; j < 6; j++) {
        for (int l = 0; l <= j; l++) a[sym6(j, l)] += wjc[0][j] * o.jc[0][l] + wjc[1][j] * o.jc[1][l];
        a[21 + j] -= wjc[0][j] * o.r[0] + wjc[1][j] * o.r[1];
        a[27 + j] += wjc[0][j] * o.jf[0] + wjc[1][j] * o.jf[1];
      }
    }
    for (int j = 0; j < 33; j++) {
      double s = a[j];
      for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(kFull, s, d);
      if (lane == 0) red[warp * kCameraPartials + j] = s;
    }
  }
  // Pass 2: W V^-1 W^T (lower triangle) and W V^-1 b_p.
  {
    double b[27];
    for (int j = 0; j < 27; j++) b[j] = 0;
    for (uint32_t kk = k0 + threadIdx.x; kk < k1; kk += blockDim.x) {
      const uint32_t i = P.camera_obs[kk], pt = P.obs_point[i];
      const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
      ObsLin o;
      if (!linearize(pose, cam, P.points + 3 * size_t(pt), true, directional(P, pt), uv.x, uv.y, P.huber, o))
        continue;
      double Wc[6][3];
      for (int j = 0; j < 6; j++)
        for (int l = 0; l < 3; l++)
          Wc[j][l] = o.jc[0][j] * (o.w * o.jp[0][l]) + o.jc[1][j] * (o.w * o.jp[1][l]);
      const double v0 = P.vinv[pt], v1 = P.vinv[Pn + pt], v2 = P.vinv[2 * Pn + pt], v3 = P.vinv[3 * Pn + pt],
                   v4 = P.vinv[4 * Pn + pt], v5 = P.vinv[5 * Pn + pt];
      const double b0 = P.bp[pt], b1 = P.bp[Pn + pt], b2 = P.bp[2 * Pn + pt];
      for (int j = 0; j < 6; j++) {
        const double t0 = Wc[j][0] * v0 + Wc[j][1] * v1 + Wc[j][2] * v2;
        const double t1 = Wc[j][0] * v1 + Wc[j][1] * v3 + Wc[j][2] * v4;
        const double t2 = Wc[j][0] * v2 + Wc[j][1] * v4 + Wc[j][2] * v5;
        for (int l = 0; l <= j; l++) b[sym6(j, l)] += t0 * Wc[l][0] + t1 * Wc[l][1] + t2 * Wc[l][2];
        b[21 + j] += t0 * b0 + t1 * b1 + t2 * b2;
      }
    }
    for (int j = 0; j < 27; j++) {
      double s = b[j];
      for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(kFull, s, d);
      if (lane == 0) red[warp * kCameraPartials + 33 + j] = s;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < kCameraPartials; j += blockDim.x) {
    double s = 0;
    for (int w = 0; w < nwarps; w++) s += red[w * kCameraPartials + j];
    P.chunk_part[size_t(kCameraPartials) * ch + j] = s;
  }
}

__global__ void k_camera_finish(Params P) {
  if (P.state[S_ACTIVE] == 0) return;
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.C) return;
  double* U = P.camU + 21 * size_t(c);
  double* Minv = P.camMinv + 36 * size_t(c);
  double* rhs = P.camRhs + 6 * size_t(c);
  double* hcf = P.camHcf + 6 * size_t(c);
  if (P.active[c] == 0) {
    for (int j = 0; j < 21; j++) U[j] = 0;
    for (int j = 0; j < 36; j++) Minv[j] = 0;
    for (int j = 0; j < 6; j++) {
      U[sym6(j, j)] = 1;
      Minv[j * 7] = 1;
      rhs[j] = 0;
      hcf[j] = 0;
    }
    return;
  }
  double a[kCameraPartials];
  for (int j = 0; j < kCameraPartials; j++) a[j] = 0;
  for (uint32_t ch = P.cam_chunk[c]; ch < P.cam_chunk[c + 1]; ch++)
    for (int j = 0; j < kCameraPartials; j++) a[j] += P.chunk_part[size_t(kCameraPartials) * ch + j];
  const double lambda = P.state[S_LAMBDA];
  for (int j = 0; j < 6; j++) a[sym6(j, j)] += lambda * fmax(a[sym6(j, j)], 1e-10);
  double S[21];
  for (int j = 0; j < 21; j++) {
    U[j] = a[j];
    S[j] = a[j] - a[33 + j];
  }
  for (int j = 0; j < 6; j++) {
    rhs[j] = a[21 + j] - a[54 + j];
    hcf[j] = a[27 + j];
  }
  double inv[36];
  if (inverse6_spd(S, inv)) {
    for (int j = 0; j < 36; j++) Minv[j] = inv[j];
  } else {
    for (int j = 0; j < 36; j++) Minv[j] = 0;
    Minv[0] = -1;
  }
}

// ---- K9/K21: damped focal scalars and the PCG start --------------------------------------------

__device__ inline double precondition(const Params& P, uint32_t i) {
  if (P.shared && i == P.m - 1) return P.state[S_FOCAL_INV] * P.r[i];
  const uint32_t c = i / 6, j = i % 6;
  const double* Mi = P.camMinv + 36 * size_t(c) + 6 * j;
  const double* rc = P.r + 6 * size_t(c);
  return Mi[0] * rc[0] + Mi[1] * rc[1] + Mi[2] * rc[2] + Mi[3] * rc[3] + Mi[4] * rc[4] + Mi[5] * rc[5];
}

__global__ void __launch_bounds__(1024) k_pcg_init(Params P) {
  __shared__ double red[4 * 32];
  __shared__ int fail;
  double* st = P.state;
  if (threadIdx.x == 0)
    for (int j = S_RHO; j <= 25; j++) st[j] = 0;
  __syncthreads();
  if (st[S_ACTIVE] == 0) return;
  if (P.shared) {
    double v[4] = {0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < P.task_blocks; b += blockDim.x)
      for (int k = 0; k < 4; k++) v[k] += P.scal_part[kScalarPartials * b + k];
    block_sum(v, red);
    if (threadIdx.x == 0) {
      double diag = v[0];
      diag += st[S_LAMBDA] * fmax(diag, 1e-10);
      st[S_FOCAL_DIAG] = diag;
      const double sff = diag - v[2];
      st[S_FOCAL_INV] = sff > 0 ? 1 / sff : -1;
      st[S_FOCAL_RHS] = -v[1] - v[3];
    }
  }
  if (threadIdx.x == 0) fail = st[S_POINT_FAILED] != 0 || (P.shared && !(st[S_FOCAL_INV] > 0));
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < P.C; c += blockDim.x)
    if (!(P.camMinv[36 * size_t(c)] > 0)) fail = 1;
  __syncthreads();
  if (fail) {
    if (threadIdx.x == 0) st[S_CG_FAILED] = 1;
    return;
  }
  for (uint32_t i = threadIdx.x; i < P.m; i += blockDim.x) P.r[i] = (P.shared && i == P.m - 1) ? st[S_FOCAL_RHS] : P.camRhs[i];
  __syncthreads();
  double v[2] = {0, 0};
  for (uint32_t i = threadIdx.x; i < P.m; i += blockDim.x) {
    const double rr = P.r[i], zz = precondition(P, i);
    P.x[i] = 0;
    P.p[i] = zz;
    P.z[i] = zz;
    v[0] += rr * zz;
    v[1] += rr * rr;
  }
  block_sum(v, red);
  if (threadIdx.x == 0) {
    st[S_RHO] = v[0];
    st[S_R0] = st[S_R2] = v[1];
    if (v[1] > 0 && v[0] > 0) st[S_CG_ACTIVE] = 1;
    else if (v[1] > 1e-24) st[S_CG_FAILED] = 1;
  }
}

// ---- K10/K11: the Schur product S p, one pass over W -------------------------------------------

template <bool SHARED>
__global__ void __launch_bounds__(kProductThreads, TBA_PRODUCT_MIN_BLOCKS) k_product(Params P) {
  extern __shared__ double acc[];
  if (P.state[S_CG_ACTIVE] == 0) return;
  const uint32_t m = P.m;
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) acc[j] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const size_t M = P.M, Pn = P.P;
  const double* __restrict__ pv = P.p;
  const double pf = SHARED ? pv[m - 1] : 0.0;
  constexpr int WD = SHARED ? 21 : 18;
  double ef = 0;  // focal row share of this lane
  uint32_t tb, te;
  block_tasks(P, tb, te);
  for (uint32_t t = tb + warp; t < te; t += nwarps) {
    const uint32_t p0 = P.tasks[t], p1 = P.tasks[t + 1];
    const uint32_t o0 = P.point_start[p0], n = P.point_start[p1] - o0;
    if (n <= uint32_t(kTaskObs)) {
      const bool valid = uint32_t(lane) < n;
      const uint32_t i = o0 + lane;
      double w[WD];
      double s[3] = {0, 0, 0};
      int seg = -1 - lane;
      uint32_t pt = 0, c = 0;
      if (valid) {
        pt = P.obs_point[i];
        c = P.obs_camera[i];
        seg = int(pt - p0);
#pragma unroll
        for (int k = 0; k < WD; k++) w[k] = __ldg(P.W + k * M + i);
        const double* xc = pv + 6 * size_t(c);
        double x6[6];
#pragma unroll
        for (int k = 0; k < 6; k++) x6[k] = __ldg(xc + k);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          double a = SHARED ? w[18 + j] * pf : 0.0;
#pragma unroll
          for (int k = 0; k < 6; k++) a += w[k * 3 + j] * x6[k];
          s[j] = a;
        }
      }
      seg_scan(s, seg, lane);
      // The last lane of each point forms y_p = V_p^-1 s_p; every lane of the point takes it.
      double y[3] = {0, 0, 0};
      if (valid && (uint32_t(lane) == n - 1 || __ldg(P.point_start + pt + 1) == i + 1)) {
        const double v0 = __ldg(P.vinv + pt), v1 = __ldg(P.vinv + Pn + pt), v2 = __ldg(P.vinv + 2 * Pn + pt),
                     v3 = __ldg(P.vinv + 3 * Pn + pt), v4 = __ldg(P.vinv + 4 * Pn + pt), v5 = __ldg(P.vinv + 5 * Pn + pt);
        y[0] = v0 * s[0] + v1 * s[1] + v2 * s[2];
        y[1] = v1 * s[0] + v3 * s[1] + v4 * s[2];
        y[2] = v2 * s[0] + v4 * s[1] + v5 * s[2];
      }
      const int tail = valid ? int(__ldg(P.point_start + pt + 1) - 1 - o0) : lane;
#pragma unroll
      for (int j = 0; j < 3; j++) y[j] = __shfl_sync(kFull, y[j], tail);
      if (valid) {
        double* ac = acc + 6 * size_t(c);
        if (TBA_PRODUCT_RELOAD) {
#pragma unroll
          for (int k = 0; k < WD; k++) w[k] = __ldg(P.W + k * M + i);
        }
#pragma unroll
        for (int k = 0; k < 6; k++) atomicAdd(ac + k, -(w[k * 3] * y[0] + w[k * 3 + 1] * y[1] + w[k * 3 + 2] * y[2]));
        if (SHARED) ef += w[18] * y[0] + w[19] * y[1] + w[20] * y[2];
      }
    } else {
      // A point with more than 32 observations: two sweeps over its observations.
      const uint32_t pt = p0;
      double s[3] = {0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs) {
        if (base + lane < n) {
          const uint32_t i = o0 + base + lane, c = P.obs_camera[i];
          const double* xc = pv + 6 * size_t(c);
#pragma unroll
          for (int j = 0; j < 3; j++) {
            double a = SHARED ? __ldg(P.W + (18 + j) * M + i) * pf : 0.0;
#pragma unroll
            for (int k = 0; k < 6; k++) a += __ldg(P.W + (k * 3 + j) * M + i) * __ldg(xc + k);
            s[j] += a;
          }
        }
      }
      warp_allsum(s);
      const double v0 = __ldg(P.vinv + pt), v1 = __ldg(P.vinv + Pn + pt), v2 = __ldg(P.vinv + 2 * Pn + pt),
                   v3 = __ldg(P.vinv + 3 * Pn + pt), v4 = __ldg(P.vinv + 4 * Pn + pt), v5 = __ldg(P.vinv + 5 * Pn + pt);
      const double y0 = v0 * s[0] + v1 * s[1] + v2 * s[2];
      const double y1 = v1 * s[0] + v3 * s[1] + v4 * s[2];
      const double y2 = v2 * s[0] + v4 * s[1] + v5 * s[2];
      for (uint32_t base = 0; base < n; base += kTaskObs) {
        if (base + lane < n) {
          const uint32_t i = o0 + base + lane, c = P.obs_camera[i];
          double* ac = acc + 6 * size_t(c);
#pragma unroll
          for (int k = 0; k < 6; k++)
            atomicAdd(ac + k, -(__ldg(P.W + (k * 3) * M + i) * y0 + __ldg(P.W + (k * 3 + 1) * M + i) * y1 +
                                __ldg(P.W + (k * 3 + 2) * M + i) * y2));
          if (SHARED)
            ef += __ldg(P.W + 18 * M + i) * y0 + __ldg(P.W + 19 * M + i) * y1 + __ldg(P.W + 20 * M + i) * y2;
        }
      }
    }
  }
  if (SHARED) {
    for (int d = 16; d > 0; d >>= 1) ef += __shfl_xor_sync(kFull, ef, d);
    if (lane == 0) atomicAdd(acc + (m - 1), -ef);
  }
  __syncthreads();
  double* out = P.acc_part + size_t(blockIdx.x) * m;
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) out[j] = acc[j];
}

// ---- K12: one PCG step, in three short kernels --------------------------------------------------
//
// k_product_reduce   column-parallel sum of the product blocks' partial rows (fixed order), the
//                    camera rows of S p = U_c p_c + H_cf p_f - sum, their p . Sp share; its last
//                    block adds the focal row and forms alpha = rho / p.Sp (with the reference's
//                    breakdown checks).
// k_pcg_update       x += alpha p, r -= alpha Sp, z = M^-1 r by camera blocks (252 rows per block,
//                    so no camera straddles two blocks); its last block forms the residual, rho,
//                    the convergence test and beta.
// k_pcg_direction    p = z + beta p.

constexpr int kReduceThreads = 256;  // 8 warps; 32 columns per block
constexpr int kUpdateRows = 252;     // 42 cameras per block
constexpr int kUpdateThreads = 256;

// True in the block that finishes last.  Every thread fences its own writes before the barrier,
// so the last block sees every block's results (read them with __ldcg).
__device__ inline bool last_block(uint32_t* ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) __threadfence();
  return last;
}

template <bool SHARED>
__global__ void __launch_bounds__(kReduceThreads) k_product_reduce(Params P) {
  __shared__ double part[8][33];
  __shared__ double red[2 * (kReduceThreads / 32)];
  if (P.state[S_CG_ACTIVE] == 0) return;
  const uint32_t n = 6 * P.C, m = P.m;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t j = blockIdx.x * 32 + lane;
  double s = 0;
  if (j < m)
    for (uint32_t g = warp; g < P.prod_blocks; g += 8) s += P.acc_part[size_t(g) * m + j];
  part[warp][lane] = s;
  __syncthreads();
  double v[2] = {0, 0};  // p . Sp over camera rows, H_cf . p (the focal row's camera share)
  if (warp == 0) {
    double sum = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) sum += part[w][lane];
    if (j < n) {
      const uint32_t c = j / 6, r = j % 6;
      const double* U = P.camU + 21 * size_t(c);
      const double* pc = P.p + 6 * size_t(c);
      double up = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) up += U[sym6(r, k)] * pc[k];
      double sp = up + sum;
      if (SHARED) {
        sp += P.camHcf[j] * P.p[m - 1];
        v[1] = P.camHcf[j] * P.p[j];
      }
      P.Sp[j] = sp;
      v[0] = P.p[j] * sp;
    } else if (SHARED && j == n) {
      P.Sp[n] = sum;  // the observation share of the focal row; completed by the last block
    }
  }
  block_sum(v, red);
  if (threadIdx.x == 0) {
    P.blk_part[2 * blockIdx.x] = v[0];
    P.blk_part[2 * blockIdx.x + 1] = v[1];
  }
  if (!last_block(P.ticket)) return;
  double t[2] = {0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    t[0] += __ldcg(P.blk_part + 2 * b);
    t[1] += __ldcg(P.blk_part + 2 * b + 1);
  }
  block_sum(t, red);
  if (threadIdx.x != 0) return;
  double* st = P.state;
  double den = t[0];
  if (SHARED) {
    const double pf = P.p[n];
    const double spf = st[S_FOCAL_DIAG] * pf + t[1] + __ldcg(P.Sp + n);
    P.Sp[n] = spf;
    den += pf * spf;
  }
  *P.ticket = 0;
  const double alpha = st[S_RHO] / den;
  if (!(den > 0) || !(fabs(alpha) < 1e20)) {
    st[S_CG_ACTIVE] = 0;
    st[S_CG_FAILED] = 1;
    return;
  }
  st[S_ALPHA] = alpha;
}

__global__ void __launch_bounds__(kUpdateThreads) k_pcg_update(Params P) {
  __shared__ double rs[kUpdateRows];
  __shared__ double red[2 * (kUpdateThreads / 32)];
  double* st = P.state;
  if (st[S_CG_ACTIVE] == 0) return;
  const double alpha = st[S_ALPHA];
  const uint32_t row = blockIdx.x * kUpdateRows + threadIdx.x;
  const bool mine = threadIdx.x < uint32_t(kUpdateRows) && row < P.m;
  double rr = 0;
  if (mine) {
    P.x[row] += alpha * P.p[row];
    rr = P.r[row] - alpha * __ldcg(P.Sp + row);
    P.r[row] = rr;
    rs[threadIdx.x] = rr;
  }
  __syncthreads();
  double v[2] = {0, 0};  // r . r, z . r
  if (mine) {
    double zz;
    if (P.shared && row == P.m - 1) {
      zz = st[S_FOCAL_INV] * rr;
    } else {
      const uint32_t jr = row % 6, base = threadIdx.x - jr;
      const double* Mi = P.camMinv + 36 * size_t(row / 6) + 6 * jr;
      zz = Mi[0] * rs[base] + Mi[1] * rs[base + 1] + Mi[2] * rs[base + 2] + Mi[3] * rs[base + 3] +
           Mi[4] * rs[base + 4] + Mi[5] * rs[base + 5];
    }
    P.z[row] = zz;
    v[0] = rr * rr;
    v[1] = zz * rr;
  }
  block_sum(v, red);
  if (threadIdx.x == 0) {
    P.blk_part[2 * blockIdx.x] = v[0];
    P.blk_part[2 * blockIdx.x + 1] = v[1];
  }
  if (!last_block(P.ticket + 1)) return;
  double t[2] = {0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    t[0] += __ldcg(P.blk_part + 2 * b);
    t[1] += __ldcg(P.blk_part + 2 * b + 1);
  }
  block_sum(t, red);
  if (threadIdx.x != 0) return;
  P.ticket[1] = 0;
  const double residual = t[0], rho = t[1];
  st[S_CG_STEPS] += 1;
  st[S_CG_SOLVE_STEPS] += 1;
  st[S_R2] = residual;
  if (residual <= P.tol * P.tol * st[S_R0]) {
    st[S_CG_ACTIVE] = 0;
    st[S_CG_CONVERGED] = 1;
  } else if (!(rho > 0)) {
    st[S_CG_ACTIVE] = 0;
    st[S_CG_FAILED] = 1;
  } else {
    st[S_BETA] = rho / st[S_RHO];
    st[S_RHO] = rho;
  }
}

__global__ void k_pcg_direction(Params P) {
  if (P.state[S_CG_ACTIVE] == 0) return;
  const double beta = P.state[S_BETA];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P.m) P.p[i] = P.z[i] + beta * P.p[i];
}

// ---- K14/K15/K16: the candidate cameras, the focal scale and the gauge --------------------------

__global__ void __launch_bounds__(256) k_update_cameras(Params P) {
  __shared__ int ok;
  double* st = P.state;
  if (threadIdx.x == 0) st[S_TRIAL_VALID] = 0;
  __syncthreads();
  if (st[S_ACTIVE] == 0 || st[S_CG_FAILED] != 0) return;
  const uint32_t C = P.C;
  if (threadIdx.x == 0) {
    ok = 1;
    if (P.shared) st[S_LOG_FOCAL_TRIAL] = st[S_LOG_FOCAL] + P.x[P.m - 1];
    // An unconverged PCG solve is rejected rather than treated as exact.
    if (st[S_R0] > 0 && st[S_R2] > P.tol * P.tol * st[S_R0]) {
      st[S_CG_FAILED] = 1;
      ok = 0;
    }
  }
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
    double pose[12], moved[12];
    for (int j = 0; j < 12; j++) pose[j] = P.poses[12 * size_t(c) + j];
    if (P.active[c]) move_pose(pose, P.x + 6 * size_t(c), moved);
    else
      for (int j = 0; j < 12; j++) moved[j] = pose[j];
    for (int j = 0; j < 12; j++) P.tposes[12 * size_t(c) + j] = moved[j];
  }
  __syncthreads();
  if (!ok) return;
  const double o[3] = {st[S_ORIGIN], st[S_ORIGIN + 1], st[S_ORIGIN + 2]};
  if (P.shared) {
    const double ls = st[S_LOG_FOCAL_TRIAL];
    if (!(fabs(ls) < 700)) return;
    const double fs = exp(ls);
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
      const double fx = P.cams[6 * size_t(c)] * fs, fy = P.cams[6 * size_t(c) + 1] * fs;
      if (!(fx >= 1e-6 && fy >= 1e-6 && fx <= 1e6 && fy <= 1e6)) ok = 0;
    }
  }
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
    const double* p = P.tposes + 12 * size_t(c);
    for (int j = 0; j < 12; j++)
      if (!(fabs(p[j]) <= 1e9)) ok = 0;
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        double d = p[j * 3] * p[k * 3] + p[j * 3 + 1] * p[k * 3 + 1] + p[j * 3 + 2] * p[k * 3 + 2];
        if (j == k) d -= 1;
        if (!(fabs(d) < 1e-6)) ok = 0;
      }
  }
  __shared__ double scale;
  if (threadIdx.x == 0) {
    const double* p = P.tposes + 12 * size_t(P.scale_view);
    double cc[3];
    for (int i = 0; i < 3; i++) cc[i] = -p[i] * p[9] - p[i + 3] * p[10] - p[i + 6] * p[11];
    const double baseline = sqrt((o[0] - cc[0]) * (o[0] - cc[0]) + (o[1] - cc[1]) * (o[1] - cc[1]) +
                                 (o[2] - cc[2]) * (o[2] - cc[2]));
    scale = 1;
    if (!(baseline > 1e-12)) ok = 0;
    else if (P.normalize_scale) scale = st[S_BASELINE] / baseline;
    if (!(scale > 1e-9 && scale < 1e9)) ok = 0;
  }
  __syncthreads();
  if (!ok) return;
  if (threadIdx.x == 0) {
    st[S_SCALE] = scale;
    st[S_TRIAL_VALID] = 1;
  }
  if (!P.normalize_scale) return;
  const double s = scale;
  for (uint32_t h = threadIdx.x; h < C; h += blockDim.x) {
    if (h == P.anchor) continue;
    double* p = P.tposes + 12 * size_t(h);
    double rot[3];
    for (int i = 0; i < 3; i++) rot[i] = (p[i * 3] * o[0] + p[i * 3 + 1] * o[1] + p[i * 3 + 2] * o[2] + p[9 + i]) - p[9 + i];
    for (int i = 0; i < 3; i++) p[9 + i] = s * p[9 + i] + (s - 1) * rot[i];
  }
}

// ---- K14/K16/K17: candidate points and the candidate cost ---------------------------------------

template <bool SHARED>
__device__ inline void candidate_point(const Params& P, uint32_t pt, const double s[3], double X[3]) {
  const size_t Pn = P.P;
  const double v0 = P.vinv[pt], v1 = P.vinv[Pn + pt], v2 = P.vinv[2 * Pn + pt], v3 = P.vinv[3 * Pn + pt],
               v4 = P.vinv[4 * Pn + pt], v5 = P.vinv[5 * Pn + pt];
  const double r0 = P.bp[pt] - s[0], r1 = P.bp[Pn + pt] - s[1], r2 = P.bp[2 * Pn + pt] - s[2];
  const double* X0 = P.points + 3 * size_t(pt);
  X[0] = X0[0] + (v0 * r0 + v1 * r1 + v2 * r2);
  X[1] = X0[1] + (v1 * r0 + v3 * r1 + v4 * r2);
  X[2] = X0[2] + (v2 * r0 + v4 * r1 + v5 * r2);
  const double* st = P.state;
  if (directional(P, pt)) {
    const double norm = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    if (norm > 1e-12)
      for (int j = 0; j < 3; j++) X[j] = X[j] / norm;
  } else if (P.normalize_scale) {
    const double sc = st[S_SCALE];
    for (int j = 0; j < 3; j++) X[j] = st[S_ORIGIN + j] + sc * (X[j] - st[S_ORIGIN + j]);
  }
  double* out = P.tpoints + 3 * size_t(pt);
  out[0] = X[0];
  out[1] = X[1];
  out[2] = X[2];
}

template <bool SHARED>
__device__ inline void candidate_obs(const Params& P, uint32_t i, uint32_t pt, const double X[3], double logf,
                                     double& cost, double& sq) {
  const uint32_t c = P.obs_camera[i];
  double pose[12];
  load_pose(P.tposes, c, pose);
  const Camera k = camera_at(P, c, logf);
  const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
  double oc, os;
  candidate_cost(pose, k, X, directional(P, pt), uv.x, uv.y, P.huber, oc, os);
  cost += oc;
  sq += os;
}

template <bool SHARED>
__global__ void __launch_bounds__(kPointThreads) k_update_points(Params P) {
  __shared__ double red[2 * (kPointThreads / 32)];
  const double* st = P.state;
  if (st[S_ACTIVE] == 0 || st[S_CG_FAILED] != 0 || st[S_TRIAL_VALID] == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const size_t M = P.M;
  const double* __restrict__ xv = P.x;
  const double xf = SHARED ? xv[P.m - 1] : 0.0;
  const double logf = SHARED ? st[S_LOG_FOCAL_TRIAL] : 0.0;
  double cs[2] = {0, 0};
  uint32_t tb, te;
  block_tasks(P, tb, te);
  for (uint32_t t = tb + warp; t < te; t += nwarps) {
    const uint32_t p0 = P.tasks[t], p1 = P.tasks[t + 1];
    const uint32_t o0 = P.point_start[p0], n = P.point_start[p1] - o0;
    if (n <= uint32_t(kTaskObs)) {
      const bool valid = uint32_t(lane) < n;
      const uint32_t i = o0 + lane;
      double s[3] = {0, 0, 0};
      int seg = -1 - lane;
      uint32_t pt = 0;
      if (valid) {
        pt = P.obs_point[i];
        seg = int(pt - p0);
        const uint32_t c = P.obs_camera[i];
        const double* xc = xv + 6 * size_t(c);
        for (int j = 0; j < 3; j++) {
          double a = SHARED ? P.W[(18 + j) * M + i] * xf : 0.0;
          for (int k = 0; k < 6; k++) a += P.W[(k * 3 + j) * M + i] * xc[k];
          s[j] = a;
        }
      }
      seg_scan(s, seg, lane);
      double X[3] = {0, 0, 0};
      const uint32_t end = valid ? P.point_start[pt + 1] : 0;
      if (valid && end == i + 1) candidate_point<SHARED>(P, pt, s, X);
      const int tail = valid ? int(end - 1 - o0) : lane;
      for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], tail);
      if (valid) candidate_obs<SHARED>(P, i, pt, X, logf, cs[0], cs[1]);
    } else {
      const uint32_t pt = p0;
      double s[3] = {0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs)
        if (base + lane < n) {
          const uint32_t i = o0 + base + lane, c = P.obs_camera[i];
          const double* xc = xv + 6 * size_t(c);
          for (int j = 0; j < 3; j++) {
            double a = SHARED ? P.W[(18 + j) * M + i] * xf : 0.0;
            for (int k = 0; k < 6; k++) a += P.W[(k * 3 + j) * M + i] * xc[k];
            s[j] += a;
          }
        }
      warp_allsum(s);
      double X[3] = {0, 0, 0};
      if (lane == 0) candidate_point<SHARED>(P, pt, s, X);
      for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], 0);
      for (uint32_t base = 0; base < n; base += kTaskObs)
        if (base + lane < n) candidate_obs<SHARED>(P, o0 + base + lane, pt, X, logf, cs[0], cs[1]);
    }
  }
  block_sum(cs, red);
  if (threadIdx.x == 0) {
    P.cost_part[4 * blockIdx.x] = cs[0];
    P.cost_part[4 * blockIdx.x + 1] = cs[1];
  }
}

// ---- K18/K19: acceptance and commit ------------------------------------------------------------

__global__ void __launch_bounds__(256) k_accept(Params P) {
  __shared__ double red[2 * 8];
  double* st = P.state;
  double v[2] = {0, 0};
  const bool valid = st[S_TRIAL_VALID] != 0;
  if (valid)
    for (uint32_t b = threadIdx.x; b < P.task_blocks; b += blockDim.x) {
      v[0] += P.cost_part[4 * b];
      v[1] += P.cost_part[4 * b + 1];
    }
  block_sum(v, red);
  if (threadIdx.x != 0) return;
  st[S_COMMIT] = 0;
  if (st[S_ACTIVE] == 0) return;
  const double cost = v[0], squares = v[1];
  if (valid && cost < st[S_COST]) {
    const double change = st[S_COST] - cost;
    st[S_COST] = cost;
    st[S_SSE] = squares;
    st[S_ACCEPTED] += 1;
    st[S_COMMIT] = 1;
    st[S_LAMBDA] = fmax(1e-10, st[S_LAMBDA] / 3);
    if (change < fmax(P.stall, 1e-9) * fmax(1.0, cost)) st[S_ACTIVE] = 0;
  } else {
    st[S_REJECTED] += 1;
    st[S_LAMBDA] *= 10;
    if (st[S_CG_FAILED] != 0) st[S_FAILED_SOLVES] += 1;
    if (st[S_LAMBDA] > 1e12) st[S_ACTIVE] = 0;
  }
  st[S_POINT_FAILED] = 0;
}

__global__ void k_commit(Params P) {
  const double* st = P.state;
  if (st[S_COMMIT] == 0) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 12 * P.C) P.poses[i] = P.tposes[i];
  if (i < 3 * P.P) P.points[i] = P.tpoints[i];
  if (i == 0 && P.shared) P.state[S_LOG_FOCAL] = st[S_LOG_FOCAL_TRIAL];
}

// ---- K20: packBundleResult ----------------------------------------------------------------------

__global__ void k_pack(Params P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t np = 12 * P.C, total = np + 3 * P.P;
  if (i < np) P.output[i] = P.poses[i];
  else if (i < total) P.output[i] = P.points[i - np];
  else if (i < total + 26) {
    const uint32_t w = i - total;
    double v = P.state[w];
    if (w == 24) v = sqrt(P.state[S_SSE0] / double(float(P.M)));
    if (w == 25) v = sqrt(P.state[S_SSE] / double(float(P.M)));
    P.output[i] = v;
  } else if (i == total + 26 && P.shared) {
    P.output[i] = P.state[S_LOG_FOCAL];
  }
}

}  // namespace

// ---- launches ----------------------------------------------------------------------------------

uint32_t product_finish_blocks(const Params& p) {
  const uint32_t a = (p.m + 31) / 32, b = (p.m + kUpdateRows - 1) / kUpdateRows;
  return a > b ? a : b;
}
size_t product_smem_bytes(const Params& p) { return size_t(p.m) * sizeof(double); }
uint32_t product_max_unknowns() { return (227 * 1024) / sizeof(double) - 64; }

cudaError_t configure_kernels() {
  const int bytes = 227 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_product<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_product<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

int product_blocks_per_sm(size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_product<true>, kProductThreads, smem) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

void launch_initialize(const Params& p, cudaStream_t s) { k_initialize<<<1, 1, 0, s>>>(p); }
void launch_cost(const Params& p, cudaStream_t s) { k_cost<<<p.task_blocks, kPointThreads, 0, s>>>(p); }
void launch_finish_metrics(const Params& p, cudaStream_t s) { k_finish_metrics<<<1, 1024, 0, s>>>(p); }
void launch_point_pass(const Params& p, cudaStream_t s) {
  if (p.shared) k_point_pass<true><<<p.task_blocks, kPointThreads, 0, s>>>(p);
  else k_point_pass<false><<<p.task_blocks, kPointThreads, 0, s>>>(p);
}
void launch_camera_pass(const Params& p, cudaStream_t s) { k_camera_pass<<<p.nchunks, kCameraThreads, 0, s>>>(p); }
void launch_camera_finish(const Params& p, cudaStream_t s) { k_camera_finish<<<(p.C + 127) / 128, 128, 0, s>>>(p); }
void launch_pcg_init(const Params& p, cudaStream_t s) { k_pcg_init<<<1, 1024, 0, s>>>(p); }
void launch_product(const Params& p, cudaStream_t s) {
  if (p.shared) k_product<true><<<p.prod_blocks, kProductThreads, product_smem_bytes(p), s>>>(p);
  else k_product<false><<<p.prod_blocks, kProductThreads, product_smem_bytes(p), s>>>(p);
}
void launch_product_finish(const Params& p, cudaStream_t s) {
  if (p.shared) k_product_reduce<true><<<(p.m + 31) / 32, kReduceThreads, 0, s>>>(p);
  else k_product_reduce<false><<<(p.m + 31) / 32, kReduceThreads, 0, s>>>(p);
  k_pcg_update<<<(p.m + kUpdateRows - 1) / kUpdateRows, kUpdateThreads, 0, s>>>(p);
  k_pcg_direction<<<(p.m + 255) / 256, 256, 0, s>>>(p);
}
void launch_update_cameras(const Params& p, cudaStream_t s) { k_update_cameras<<<1, 256, 0, s>>>(p); }
void launch_update_points(const Params& p, cudaStream_t s) {
  if (p.shared) k_update_points<true><<<p.task_blocks, kPointThreads, 0, s>>>(p);
  else k_update_points<false><<<p.task_blocks, kPointThreads, 0, s>>>(p);
}
void launch_accept(const Params& p, cudaStream_t s) { k_accept<<<1, 256, 0, s>>>(p); }
void launch_commit(const Params& p, cudaStream_t s) {
  const uint32_t n = (12 * p.C > 3 * p.P ? 12 * p.C : 3 * p.P);
  k_commit<<<(n + 255) / 256, 256, 0, s>>>(p);
}
void launch_pack(const Params& p, cudaStream_t s) {
  const uint32_t n = 12 * p.C + 3 * p.P + 27;
  k_pack<<<(n + 255) / 256, 256, 0, s>>>(p);
}

}  // namespace tba
