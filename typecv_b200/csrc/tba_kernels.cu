// Kernels of the grid engine (one bundle adjustment over the whole GPU), sm_100a, FP64.
//
// Kernel                  reference kernel(s) it replaces (src/sfm/bundle/gpu/*.shade.ts)
// k_initialize, k_setup   initializeBundle (K1); per-camera radial limits and the camera-major
//                         copies of the observations' point and pixel
// k_cost/k_finish_metrics bundleMetricPartials + finishBundleMetrics (K3/K4)
// k_point_pass            linearizeBundle + bundlePointBlocks + bundleFocalObservations +
//                         bundleFocalPoints (K2/K5/K21)
// k_camera_pass/_finish   bundleCameraRows + bundleFocalCameraRows + invertBundleCameraColumns +
//                         finalizeBundleCameraInverse (K6/K8/K21)
// k_pcg_init              dampBundleFocal + initializeBundleCg (K9/K21)
// k_product_f             bundleSchurPoint + bundleSchurCamera (K10/K11) in one pass over the
//                         stored world-axis Jacobian factors, camera sums in shared memory
// k_product_columns       the fixed-order sum of the product blocks' partial rows
// k_schur_points          (two-pass form, for camera systems too large for shared memory)
//                         bundleSchurPoint (K10): y_p = V_p^-1 sum_i W_i^T p, point-major
// k_schur_cameras         bundleSchurCamera (K11): sum_i W_i y_p per camera chunk, camera-major
// k_product_reduce,       advanceBundleCg (K12), split into a reduction with alpha, a
// k_pcg_update/_direction distributed update with beta, and the new direction
// k_update_cameras        updateBundleCandidate (cameras, focal) + bundleCandidateGauge +
//                         normalizeBundleCandidate (cameras) (K14/K15/K16)
// k_update_points         updateBundleCandidate (points) + normalizeBundleCandidate (points) +
//                         bundleCandidatePartials (K14/K16/K17)
// k_accept/k_commit       acceptBundleCandidate + commitBundleCandidate (K18/K19)
// k_pack                  packBundleResult (K20)
//
// No kernel stores the Schur cross blocks W_i = w J_c^T J_p (21 words per observation).  The
// point pass stores 12 world-axis Jacobian factors per observation instead (q~ = R^T q, R^T du,
// R^T dv, w, jf; FP64, and an FP32 copy in the mixed form), from which every product is a few dozen FMAs;
// the camera passes recompute the factors from the pose, the camera, the point and the pixel.
// Every reduction runs in a fixed order (fixed grids, fixed trees, fixed chunking), except the
// shared-memory camera sums of k_product_f, whose FP64 atomic adds commute only up to rounding.
#include <cuda_runtime.h>

#include <type_traits>

#include "tba_engine.cuh"
#include "tba_warp.cuh"

// Compile-time tuning: occupancy floors of __launch_bounds__ for the heavy kernels.
#ifndef TBA_POINT_MIN_BLOCKS
#define TBA_POINT_MIN_BLOCKS 2
#endif
#ifndef TBA_CAMERA_MIN_BLOCKS
#define TBA_CAMERA_MIN_BLOCKS 3
#endif
#ifndef TBA_SCHUR_MIN_BLOCKS
#define TBA_SCHUR_MIN_BLOCKS 2
#endif

namespace tba {
namespace {

// The camera record with the accepted (or candidate) focal scale applied.
__device__ inline Camera camera_at(const Params& P, uint32_t c, double fscale) {
  const double2* k = reinterpret_cast<const double2*>(P.cams + 6 * size_t(c));
  const double2 a = k[0], b = k[1], e = k[2];
  return Camera{a.x * fscale, a.y * fscale, b.x, b.y, e.x, e.y};
}

__device__ inline double focal_scale(const Params& P, double log_scale) { return P.shared ? exp(log_scale) : 1.0; }

// The tasks [begin, end) of this block: a contiguous share of the task list.
__device__ inline void block_tasks(const Params& P, uint32_t& begin, uint32_t& end) {
  begin = uint32_t(uint64_t(P.ntasks) * blockIdx.x / gridDim.x);
  end = uint32_t(uint64_t(P.ntasks) * (blockIdx.x + 1) / gridDim.x);
}

__device__ inline bool directional(const Params& P, uint32_t pt) { return pt >= P.P - P.D; }

// The point-major observation i of point pt: its Jacobian factors at the accepted scene.
__device__ inline bool observe(const Params& P, uint32_t i, uint32_t c, uint32_t pt, double fscale, double pose[12],
                               Geo& g) {
  load_pose(P.poses, c, pose);
  const Camera k = camera_at(P, c, fscale);
  const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
  return geometry(pose, k, P.rlim[c], P.points + 3 * size_t(pt), directional(P, pt), uv.x, uv.y, P.huber, g);
}

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

// ---- K1: initializeBundle, and the per-solve set-up -----------------------------------------------

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

// Per-camera radial limits; the camera-major copies of each observation's point and pixel.
__global__ void k_setup(Params P) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < P.C) P.rlim[k] = radial_limit(P.cams[6 * size_t(k) + 4], P.cams[6 * size_t(k) + 5]);
  if (k < P.M) {
    const uint32_t i = P.camera_obs[k];
    P.cm_point[k] = P.obs_point[i];
    reinterpret_cast<double2*>(P.cm_pixel)[k] = reinterpret_cast<const double2*>(P.pixels)[i];
  }
}

// ---- K3/K4: the linearised cost of the scene ---------------------------------------------------

__global__ void __launch_bounds__(kPointThreads) k_cost(Params P) {
  __shared__ double red[3 * (kPointThreads / 32)];
  double v[3] = {0, 0, 0};  // cost, squared error, invalid projections
  const double fscale = focal_scale(P, P.state[S_LOG_FOCAL]);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.M; i += gridDim.x * blockDim.x) {
    double pose[12];
    Geo g;
    if (!observe(P, i, P.obs_camera[i], P.obs_point[i], fscale, pose, g)) {
      v[2] += 1;
      continue;
    }
    v[0] += robust_cost(sqrt(g.sq), P.huber);
    v[1] += g.sq;
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

// One observation's contributions to its point block: V (6 unique), b_p (3), the focal cross sum
// w J_p^T jf (3) and an invalid flag; and its share of the focal diagonal and right-hand side.
template <bool SHARED>
__device__ inline void point_obs(const Params& P, uint32_t i, uint32_t pt, double fscale, double (&v)[13],
                                 double& hff, double& bf) {
  double pose[12];
  Geo g;
  if (!observe(P, i, P.obs_camera[i], pt, fscale, pose, g)) {
    v[12] = 1;
    return;
  }
  double jp[2][3];
  for (int c = 0; c < 3; c++) {
    jp[0][c] = g.du[0] * pose[c] + g.du[1] * pose[3 + c] + g.du[2] * pose[6 + c];
    jp[1][c] = g.dv[0] * pose[c] + g.dv[1] * pose[3 + c] + g.dv[2] * pose[6 + c];
  }
  if (P.factored) {
    // The world-axis factors of the products: q~ = R^T q, R^T du, R^T dv, w, jf.
    double f[kFactors];
    for (int c = 0; c < 3; c++) {
      f[c] = g.q[0] * pose[c] + g.q[1] * pose[3 + c] + g.q[2] * pose[6 + c];
      f[3 + c] = jp[0][c];
      f[6 + c] = jp[1][c];
    }
    f[9] = g.w;
    f[10] = g.jf[0];
    f[11] = g.jf[1];
    const size_t stride = P.Mpad;
    // FP64 factors always; the mixed form's PCG reads an FP32 copy.
    if (P.F)
      for (int k = 0; k < kFactors; k++) P.F[k * stride + i] = f[k];
    if (P.F32)
      for (int k = 0; k < kFactors; k++) P.F32[k * stride + i] = float(f[k]);
  }
  double wjp[2][3];
  for (int row = 0; row < 2; row++)
    for (int j = 0; j < 3; j++) wjp[row][j] = g.w * jp[row][j];
  v[0] = wjp[0][0] * jp[0][0] + wjp[1][0] * jp[1][0];
  v[1] = wjp[0][0] * jp[0][1] + wjp[1][0] * jp[1][1];
  v[2] = wjp[0][0] * jp[0][2] + wjp[1][0] * jp[1][2];
  v[3] = wjp[0][1] * jp[0][1] + wjp[1][1] * jp[1][1];
  v[4] = wjp[0][1] * jp[0][2] + wjp[1][1] * jp[1][2];
  v[5] = wjp[0][2] * jp[0][2] + wjp[1][2] * jp[1][2];
  for (int j = 0; j < 3; j++) v[6 + j] = -(wjp[0][j] * g.r[0] + wjp[1][j] * g.r[1]);
  if (SHARED) {
    for (int j = 0; j < 3; j++) v[9 + j] = g.jf[0] * wjp[0][j] + g.jf[1] * wjp[1][j];
    hff += g.w * (g.jf[0] * g.jf[0] + g.jf[1] * g.jf[1]);
    bf += g.w * (g.jf[0] * g.r[0] + g.jf[1] * g.r[1]);
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
  double2* blk = reinterpret_cast<double2*>(P.pblk + 12 * size_t(pt));
  float2* blk32 = P.pblk32 ? reinterpret_cast<float2*>(P.pblk32 + 6 * size_t(pt)) : nullptr;
  if (!ok) {
    P.state[S_POINT_FAILED] = 1;
    for (int k = 0; k < 6; k++) blk[k] = make_double2(0, 0);
    if (blk32)
      for (int k = 0; k < 3; k++) blk32[k] = make_float2(0, 0);
    return;
  }
  blk[0] = make_double2(inv[0], inv[1]);
  blk[1] = make_double2(inv[2], inv[3]);
  blk[2] = make_double2(inv[4], inv[5]);
  if (blk32)  // the FP32 product's copy of the FP64 inverse
    for (int k = 0; k < 3; k++) blk32[k] = make_float2(float(inv[2 * k]), float(inv[2 * k + 1]));
  blk[3] = make_double2(v[6], v[7]);
  blk[4] = make_double2(v[8], 0);
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
  const double lambda = P.state[S_LAMBDA], fscale = focal_scale(P, P.state[S_LOG_FOCAL]);
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
        seg = int(pt);
        point_obs<SHARED>(P, o0 + lane, pt, fscale, v, sc[0], sc[1]);
      }
      const Runs runs = lane_runs(seg, lane);
      run_scan(v, runs);
      if (uint32_t(lane) < n && run_tail(runs, lane))
        point_finish<SHARED>(P, pt, v, lambda, sc[2], sc[3]);
    } else {
      const uint32_t pt = P.obs_point[o0];
      double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs) {
        if (base + lane < n) {
          double u[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
          point_obs<SHARED>(P, o0 + base + lane, pt, fscale, u, sc[0], sc[1]);
          for (int k = 0; k < 13; k++) v[k] += u[k];
        }
      }
      warp_allsum(v);
      if (lane == 0) point_finish<SHARED>(P, pt, v, lambda, sc[2], sc[3]);
    }
  }
  block_sum(sc, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kScalarPartials; k++) P.scal_part[kScalarPartials * blockIdx.x + k] = sc[k];
}

// ---- K6/K8/K21: camera blocks ------------------------------------------------------------------

// The camera rows of one observation: J_c (zero translation for a bearing).
__device__ inline void camera_rows(const Geo& g, bool dir, double jc[2][6]) {
  pose_row(g.q, g.du, jc[0]);
  pose_row(g.q, g.dv, jc[1]);
  if (dir)
    for (int c = 3; c < 6; c++) jc[0][c] = jc[1][c] = 0;
}

__global__ void __launch_bounds__(kCameraThreads, TBA_CAMERA_MIN_BLOCKS) k_camera_pass(Params P) {
  __shared__ double red[kCameraPartials * (kCameraThreads / 32)];
  if (P.state[S_ACTIVE] == 0) return;
  const uint32_t ch = blockIdx.x, c = P.chunk_cam[ch];
  if (P.active[c] == 0) return;
  const uint32_t k0 = P.chunk_beg[ch], k1 = P.chunk_beg[ch + 1];
  double pose[12];
  load_pose(P.poses, c, pose);
  const Camera cam = camera_at(P, c, focal_scale(P, P.state[S_LOG_FOCAL]));
  const double limit = P.rlim[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // Pass 1: U_c (lower triangle), b_c, H_cf.
  {
    double a[33];
    for (int j = 0; j < 33; j++) a[j] = 0;
    for (uint32_t kk = k0 + threadIdx.x; kk < k1; kk += blockDim.x) {
      const uint32_t pt = P.cm_point[kk];
      const double2 uv = reinterpret_cast<const double2*>(P.cm_pixel)[kk];
      Geo g;
      if (!geometry(pose, cam, limit, P.points + 3 * size_t(pt), directional(P, pt), uv.x, uv.y, P.huber, g))
        continue;
      double jc[2][6];
      camera_rows(g, directional(P, pt), jc);
      for (int j = 0; j < 6; j++) {
        const double w0 = g.w * jc[0][j], w1 = g.w * jc[1][j];
        for (int l = 0; l <= j; l++) a[sym6(j, l)] += w0 * jc[0][l] + w1 * jc[1][l];
        a[21 + j] -= w0 * g.r[0] + w1 * g.r[1];
        a[27 + j] += w0 * g.jf[0] + w1 * g.jf[1];
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
      const uint32_t pt = P.cm_point[kk];
      const double2 uv = reinterpret_cast<const double2*>(P.cm_pixel)[kk];
      Geo g;
      if (!geometry(pose, cam, limit, P.points + 3 * size_t(pt), directional(P, pt), uv.x, uv.y, P.huber, g))
        continue;
      double jc[2][6];
      camera_rows(g, directional(P, pt), jc);
      double jp[2][3];
      for (int l = 0; l < 3; l++) {
        jp[0][l] = g.w * (g.du[0] * pose[l] + g.du[1] * pose[3 + l] + g.du[2] * pose[6 + l]);
        jp[1][l] = g.w * (g.dv[0] * pose[l] + g.dv[1] * pose[3 + l] + g.dv[2] * pose[6 + l]);
      }
      double Wc[6][3];
      for (int j = 0; j < 6; j++)
        for (int l = 0; l < 3; l++) Wc[j][l] = jc[0][j] * jp[0][l] + jc[1][j] * jp[1][l];
      double vb[6], bb[3];
      load6(P.pblk + 12 * size_t(pt), vb);
      bb[0] = P.pblk[12 * size_t(pt) + 6];
      bb[1] = P.pblk[12 * size_t(pt) + 7];
      bb[2] = P.pblk[12 * size_t(pt) + 8];
      for (int j = 0; j < 6; j++) {
        const double t0 = Wc[j][0] * vb[0] + Wc[j][1] * vb[1] + Wc[j][2] * vb[2];
        const double t1 = Wc[j][0] * vb[1] + Wc[j][1] * vb[3] + Wc[j][2] * vb[4];
        const double t2 = Wc[j][0] * vb[2] + Wc[j][1] * vb[4] + Wc[j][2] * vb[5];
        for (int l = 0; l <= j; l++) b[sym6(j, l)] += t0 * Wc[l][0] + t1 * Wc[l][1] + t2 * Wc[l][2];
        b[21 + j] += t0 * bb[0] + t1 * bb[1] + t2 * bb[2];
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
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < P.C; c += blockDim.x) {
    double pc[6];
    for (int k = 0; k < 6; k++) pc[k] = P.p[6 * c + k];
    to_world(P.poses + 12 * size_t(c), pc, P.pw + 6 * size_t(c));
  }
  block_sum(v, red);
  if (threadIdx.x == 0) {
    st[S_RHO] = v[0];
    st[S_R0] = st[S_R2] = st[S_INNER_R0] = v[1];
    if (v[1] > 0 && v[0] > 0) st[S_CG_ACTIVE] = 1;
    else if (v[1] > 1e-24) st[S_CG_FAILED] = 1;
  }
}

// ---- K10/K11: the Schur product S p ------------------------------------------------------------
//
// Pass 1, point-major (warp tasks): y_p = V_p^-1 sum_i W_i^T p_c(i) (+ W_f p_f), written per point.
// Pass 2, camera-major (the camera chunks): sum_i W_i y_p(i) and the focal shares, per chunk.
// W_i is recomputed in both passes; neither pass has atomics.

template <bool SHARED>
__device__ inline void schur_point_obs(const Params& P, uint32_t i, uint32_t pt, double fscale, double pf,
                                       double t[3]) {
  const uint32_t c = P.obs_camera[i];
  double pose[12];
  Geo g;
  if (!observe(P, i, c, pt, fscale, pose, g)) {
    t[0] = t[1] = t[2] = 0;
    return;
  }
  double xc[6];
  load6(P.p + 6 * size_t(c), xc);
  wt_product(g, pose, xc, pf, P.active[c] != 0, directional(P, pt), SHARED, t);
}

__device__ inline void schur_point_finish(const Params& P, uint32_t pt, const double s[3]) {
  double vb[6];
  load6(P.pblk + 12 * size_t(pt), vb);
  double2* y = reinterpret_cast<double2*>(P.y + 4 * size_t(pt));
  y[0] = make_double2(vb[0] * s[0] + vb[1] * s[1] + vb[2] * s[2], vb[1] * s[0] + vb[3] * s[1] + vb[4] * s[2]);
  y[1] = make_double2(vb[2] * s[0] + vb[4] * s[1] + vb[5] * s[2], 0);
}

// The two-pass product runs while the PCG is active, or, with P.refine, on the refinement's x.
__device__ inline bool product_idle(const Params& P) {
  return P.refine ? P.state[S_REFINE] == 0 : P.state[S_CG_ACTIVE] == 0;
}

template <bool SHARED>
__global__ void __launch_bounds__(kPointThreads, TBA_SCHUR_MIN_BLOCKS) k_schur_points(Params P) {
  if (product_idle(P)) return;
  const double fscale = focal_scale(P, P.state[S_LOG_FOCAL]);
  const double pf = SHARED ? P.p[P.m - 1] : 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint32_t tb, te;
  block_tasks(P, tb, te);
  for (uint32_t t = tb + warp; t < te; t += nwarps) {
    const uint32_t p0 = P.tasks[t], p1 = P.tasks[t + 1];
    const uint32_t o0 = P.point_start[p0], n = P.point_start[p1] - o0;
    if (n <= uint32_t(kTaskObs)) {
      double s[3] = {0, 0, 0};
      int seg = -1 - lane;
      uint32_t pt = 0;
      if (uint32_t(lane) < n) {
        pt = P.obs_point[o0 + lane];
        seg = int(pt);
        schur_point_obs<SHARED>(P, o0 + lane, pt, fscale, pf, s);
      }
      const Runs runs = lane_runs(seg, lane);
      run_scan(s, runs);
      if (uint32_t(lane) < n && run_tail(runs, lane)) schur_point_finish(P, pt, s);
    } else {
      const uint32_t pt = P.obs_point[o0];
      double s[3] = {0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs)
        if (base + lane < n) {
          double u[3];
          schur_point_obs<SHARED>(P, o0 + base + lane, pt, fscale, pf, u);
          s[0] += u[0];
          s[1] += u[1];
          s[2] += u[2];
        }
      warp_allsum(s);
      if (lane == 0) schur_point_finish(P, pt, s);
    }
  }
}

template <bool SHARED>
__global__ void __launch_bounds__(kCameraThreads, TBA_CAMERA_MIN_BLOCKS) k_schur_cameras(Params P) {
  __shared__ double red[7 * (kCameraThreads / 32)];
  if (product_idle(P)) return;
  const uint32_t ch = blockIdx.x, c = P.chunk_cam[ch];
  const bool variable = P.active[c] != 0;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};  // sum_i W_i y (6), focal share (1)
  if (variable || SHARED) {
    const uint32_t k0 = P.chunk_beg[ch], k1 = P.chunk_beg[ch + 1];
    double pose[12];
    load_pose(P.poses, c, pose);
    const Camera cam = camera_at(P, c, focal_scale(P, P.state[S_LOG_FOCAL]));
    const double limit = P.rlim[c];
    for (uint32_t kk = k0 + threadIdx.x; kk < k1; kk += blockDim.x) {
      const uint32_t pt = P.cm_point[kk];
      const double2 uv = reinterpret_cast<const double2*>(P.cm_pixel)[kk];
      Geo g;
      const bool dir = directional(P, pt);
      if (!geometry(pose, cam, limit, P.points + 3 * size_t(pt), dir, uv.x, uv.y, P.huber, g)) continue;
      const double2* yp = reinterpret_cast<const double2*>(P.y + 4 * size_t(pt));
      const double2 y01 = yp[0], y2 = yp[1];
      const double y[3] = {y01.x, y01.y, y2.x};
      double d[6], e;
      w_product(g, pose, y, variable, dir, d, e);
      for (int j = 0; j < 6; j++) v[j] += d[j];
      v[6] += e;
    }
  }
  block_sum(v, red);
  if (threadIdx.x == 0)
    for (int j = 0; j < 7; j++) P.chunk_prod[8 * size_t(ch) + j] = v[j];
}

// ---- K10/K11, factored: the Schur product S p in one pass over the stored factors -------------
//
// Each warp task forms y_p = V_p^-1 sum_i W_i^T p for its points from the observations' factors
// (one observation per lane, a segmented warp scan per point), then scatters -W_i y_p into this
// block's copy of the camera sums in shared memory (world axes; FP64).  At the end the block
// rotates each camera's sums into the camera's axes (R [q~ x h~; h~] = J_c^T g) and writes them
// as one partial row; k_product_columns adds the rows in a fixed order.  T is the factors'
// storage type: double for the FP64 form, float for the mixed form (the per-observation
// arithmetic then runs in FP32 and every sum in FP64).

// STAGED: the direction of every camera (world axes, 6C values of T) is staged in shared memory
// after the camera sums, so the per-observation read of it is an on-chip gather; one block of
// kStagedThreads per SM.  With FP32 factors the kernel fits 64 registers and takes 1,024 threads
// (32 warps to cover the latency of the loads each lane issues before its arithmetic): 0.157 ->
// 0.137 ms for 1,500 cameras / 6.18M observations.  The FP64 kernel runs 768 threads at 80
// registers; from kWideObservations observations (WIDE) it is compiled for 1,024 threads at 64
// registers (4-8 bytes spilled): 0.197 -> 0.188 ms at 6.18M observations, while at 0.75M (under
// six tasks a warp) the extra warps cost more in the block's tail than they hide (1-5% slower).
// Otherwise it is read from global memory, two blocks of kProductThreads.
// Both shared arrays are component-major (the sums: value j of camera c at j * C + c; the direction:
// pair k of camera c at k * C + c, read as one 16- or 8-byte word): the lanes of a warp touch random
// cameras, and with camera-major records of 6 words the 8-byte accesses of a warp would fall on only
// 8 of the 16 bank pairs (6c mod 16 is even); component-major they spread over all of them.
// The PCG direction of every camera in world axes, staged in shared memory for the one-pass
// product, read at random cameras by the lanes of a warp.  FP32: one array of C float4 (the
// rotation part and the first translation value) and one of C float2 (the rest), two loads a
// lane; FP64: three arrays of C double2, three loads.  Component-major arrays spread random
// cameras over all bank groups (a camera-major 6-word record would put a warp's accesses on only
// half of them).
template <typename T>
struct StagedDirection;

template <>
struct StagedDirection<float> {
  float4* a;
  float2* b;
  __device__ StagedDirection(unsigned char* base, uint32_t C)
      : a(reinterpret_cast<float4*>(base)), b(reinterpret_cast<float2*>(base + 16 * size_t(C))) {}
  __device__ void store(uint32_t c, const double* v) const {
    a[c] = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
    b[c] = make_float2(float(v[4]), float(v[5]));
  }
  __device__ void load(uint32_t c, float (&x)[6]) const {
    const float4 u = a[c];
    const float2 w = b[c];
    x[0] = u.x;
    x[1] = u.y;
    x[2] = u.z;
    x[3] = u.w;
    x[4] = w.x;
    x[5] = w.y;
  }
};

template <>
struct StagedDirection<double> {
  double2* a;
  uint32_t C;
  __device__ StagedDirection(unsigned char* base, uint32_t C) : a(reinterpret_cast<double2*>(base)), C(C) {}
  __device__ void store(uint32_t c, const double* v) const {
    for (int k = 0; k < 3; k++) a[k * C + c] = make_double2(v[2 * k], v[2 * k + 1]);
  }
  __device__ void load(uint32_t c, double (&x)[6]) const {
    for (int k = 0; k < 3; k++) {
      const double2 u = a[k * C + c];
      x[2 * k] = u.x;
      x[2 * k + 1] = u.y;
    }
  }
};

// V_p^-1 (6 unique values) in the product's arithmetic type: the FP32 copy when the FP32 product
// has one, else the FP64 block.
template <typename T>
__device__ inline void load_point_inverse(const Params& P, uint32_t pt, T (&vb)[6]) {
  if constexpr (sizeof(T) == 4) {
    if (P.pblk32) {
      const float2* b = reinterpret_cast<const float2*>(P.pblk32 + 6 * size_t(pt));
      for (int k = 0; k < 3; k++) {
        const float2 d = b[k];
        vb[2 * k] = d.x;
        vb[2 * k + 1] = d.y;
      }
      return;
    }
  }
  double d[6];
  load6(P.pblk + 12 * size_t(pt), d);
  for (int k = 0; k < 6; k++) vb[k] = T(d[k]);
}

// W_i^T x in the factors' arithmetic type, from the camera's step in world axes xw and the focal
// step xf (a bearing has no translation rows).
template <typename T>
__device__ inline void factor_wt_t(const Factors<T>& f, const T (&xw)[6], T xf, bool dir, bool shared, T t[3]) {
  T m0 = xw[1] * f.q[2] - xw[2] * f.q[1], m1 = xw[2] * f.q[0] - xw[0] * f.q[2], m2 = xw[0] * f.q[1] - xw[1] * f.q[0];
  if (!dir) {
    m0 += xw[3];
    m1 += xw[4];
    m2 += xw[5];
  }
  T au = f.ju[0] * m0 + f.ju[1] * m1 + f.ju[2] * m2;
  T av = f.jv[0] * m0 + f.jv[1] * m1 + f.jv[2] * m2;
  if (shared) {
    au += f.jf[0] * xf;
    av += f.jf[1] * xf;
  }
  au *= f.w;
  av *= f.w;
  for (int k = 0; k < 3; k++) t[k] = au * f.ju[k] + av * f.jv[k];
}

template <bool SHARED, typename T, typename A, bool STAGED, bool WIDE = false>
__global__ void __launch_bounds__(STAGED ? (sizeof(T) == 4 ? kStagedThreadsF32 : (WIDE ? kStagedThreadsWide : kStagedThreads))
                                         : kProductThreads,
                                  STAGED ? 1 : 2) k_product_f(Params P) {
  extern __shared__ double4 product_smem[];
  __shared__ double focal_acc;
  // It runs while the PCG is active, or, with P.refine, on the mixed form's refinement of x.
  if (P.state[S_CG_ACTIVE] == 0 && !(P.refine && P.state[S_REFINE] != 0)) return;
  const uint32_t m = P.m, C = P.C;
  // The camera sums (6C values of A: a block's share of each camera), then the staged direction
  // (StagedDirection: 6 values of T per camera).
  A* acc = reinterpret_cast<A*>(product_smem);
  const StagedDirection<T> pws{reinterpret_cast<unsigned char*>(product_smem) + product_sums_bytes(C, sizeof(A)), C};
  for (uint32_t j = threadIdx.x; j < 6 * C; j += blockDim.x) acc[j] = A(0);
  if (threadIdx.x == 0) focal_acc = 0;
  if (STAGED)
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) pws.store(c, P.pw + 6 * size_t(c));
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const T* FT = sizeof(T) == 4 ? reinterpret_cast<const T*>(P.F32) : reinterpret_cast<const T*>(P.F);
  const size_t stride = P.Mpad;
  const double pf = SHARED ? P.p[m - 1] : 0.0;
  double ef = 0;
  uint32_t tb, te;
  block_tasks(P, tb, te);
  uint32_t t = tb + warp;
  uint32_t o_next = t < te ? P.task_obs[t] : 0, e_next = t < te ? P.task_obs[t + 1] : 0;
  for (; t < te; t += nwarps) {
    const uint32_t o0 = o_next, n = e_next - o0;
    if (t + nwarps < te) {  // the next task's bounds, early
      o_next = P.task_obs[t + nwarps];
      e_next = P.task_obs[t + nwarps + 1];
    }
    if (n <= uint32_t(kTaskObs)) {
      // One observation per lane (point-major), reduced per point with a segmented warp scan; each
      // observation's camera share -W_i y_p goes to the block's camera sums with its own atomic
      // adds.  (Grouping a task's observations by camera to add one share per camera was measured
      // slower: points ordered so that a task's observations share cameras make their atomics
      // collide, and the grouping's shuffles cost what it saves.)  Every load a lane needs is
      // issued before any arithmetic; only the last lane of each point loads its V_p^-1.
      const bool valid = uint32_t(lane) < n;
      const uint32_t i = o0 + (valid ? uint32_t(lane) : 0u);
      const uint32_t c = __ldg(P.obs_camera + i), pq = __ldg(P.obs_point + i);
      Factors<T> f;
      load_factors(FT, stride, i, f);
      const uint32_t pn = __shfl_down_sync(kFull, pq, 1);
      const bool ptail = valid && (uint32_t(lane) + 1 == n || pn != pq);
      T vb[6] = {0, 0, 0, 0, 0, 0};
      if (ptail) load_point_inverse(P, pq, vb);
      T xw[6];
      if (STAGED) {
        pws.load(c, xw);
      } else {
        double d[6];
        load6(P.pw + 6 * size_t(c), d);
        for (int k = 0; k < 6; k++) xw[k] = T(d[k]);
      }
      // A fixed camera's direction is zero, so its observations add nothing on the point side; their
      // camera shares land in the fixed camera's rows, which k_product_columns discards.
      const bool dir = directional(P, pq);
      T sc[3] = {0, 0, 0};
      if (valid) factor_wt_t(f, xw, T(pf), dir, SHARED, sc);
      const Runs pr = lane_runs(valid ? int(pq) : -1 - lane, lane);
      run_scan(sc, pr);
      T y[3] = {0, 0, 0};
      if (ptail) {
        y[0] = vb[0] * sc[0] + vb[1] * sc[1] + vb[2] * sc[2];
        y[1] = vb[1] * sc[0] + vb[3] * sc[1] + vb[4] * sc[2];
        y[2] = vb[2] * sc[0] + vb[4] * sc[1] + vb[5] * sc[2];
      }
      const unsigned tails = __ballot_sync(kFull, ptail);
      const int src = valid ? __ffs(tails & (kFull << lane)) - 1 : lane;
      for (int k = 0; k < 3; k++) y[k] = __shfl_sync(kFull, y[k], src);
      if (!valid) continue;
      // -W_i y_p in world axes (rotation rows q~ x h, translation rows h).
      const T gu = f.w * (f.ju[0] * y[0] + f.ju[1] * y[1] + f.ju[2] * y[2]);
      const T gv = f.w * (f.jv[0] * y[0] + f.jv[1] * y[1] + f.jv[2] * y[2]);
      if (SHARED) ef += double(gu * f.jf[0] + gv * f.jf[1]);
      const T h0 = gu * f.ju[0] + gv * f.jv[0], h1 = gu * f.ju[1] + gv * f.jv[1], h2 = gu * f.ju[2] + gv * f.jv[2];
      A* ac = acc + c;
      atomicAdd(ac, A(-(f.q[1] * h2 - f.q[2] * h1)));
      atomicAdd(ac + C, A(-(f.q[2] * h0 - f.q[0] * h2)));
      atomicAdd(ac + 2 * C, A(-(f.q[0] * h1 - f.q[1] * h0)));
      if (!dir) {
        atomicAdd(ac + 3 * C, A(-h0));
        atomicAdd(ac + 4 * C, A(-h1));
        atomicAdd(ac + 5 * C, A(-h2));
      }
      continue;
    }
    // A point with more than 32 observations: rounds of 32, one warp-wide sum.
    const uint32_t p0 = P.obs_point[o0];
    const uint32_t rounds = (n + kTaskObs - 1) / kTaskObs;
    double s[3] = {0, 0, 0};
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k < n) {
        const uint32_t i = o0 + k;
        const uint32_t c = P.obs_camera[i];
        Factors<T> f;
        load_factors(FT, stride, i, f);
        double xw[6], u[3];
        if (STAGED) {
          T d[6];
          pws.load(c, d);
          for (int k = 0; k < 6; k++) xw[k] = double(d[k]);
        } else
          load6(P.pw + 6 * size_t(c), xw);
        factor_wt(f, xw, pf, true, directional(P, p0), SHARED, u);
        s[0] += u[0];
        s[1] += u[1];
        s[2] += u[2];
      }
    }
    warp_allsum(s);
    double vb[6];
    load6(P.pblk + 12 * size_t(p0), vb);
    const T y0 = T(vb[0] * s[0] + vb[1] * s[1] + vb[2] * s[2]);
    const T y1 = T(vb[1] * s[0] + vb[3] * s[1] + vb[4] * s[2]);
    const T y2 = T(vb[2] * s[0] + vb[4] * s[1] + vb[5] * s[2]);
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k >= n) continue;
      const uint32_t i = o0 + k;
      const uint32_t c = P.obs_camera[i];
      Factors<T> f;
      load_factors(FT, stride, i, f);
      const T gu = f.w * (f.ju[0] * y0 + f.ju[1] * y1 + f.ju[2] * y2);
      const T gv = f.w * (f.jv[0] * y0 + f.jv[1] * y1 + f.jv[2] * y2);
      if (SHARED) ef += double(gu * f.jf[0] + gv * f.jf[1]);
      const T h0 = gu * f.ju[0] + gv * f.jv[0], h1 = gu * f.ju[1] + gv * f.jv[1], h2 = gu * f.ju[2] + gv * f.jv[2];
      A* ac = acc + c;
      atomicAdd(ac, A(-(f.q[1] * h2 - f.q[2] * h1)));
      atomicAdd(ac + C, A(-(f.q[2] * h0 - f.q[0] * h2)));
      atomicAdd(ac + 2 * C, A(-(f.q[0] * h1 - f.q[1] * h0)));
      if (!directional(P, p0)) {
        atomicAdd(ac + 3 * C, A(-h0));
        atomicAdd(ac + 4 * C, A(-h1));
        atomicAdd(ac + 5 * C, A(-h2));
      }
    }
  }
  if (SHARED) {
    for (int d = 16; d > 0; d >>= 1) ef += __shfl_xor_sync(kFull, ef, d);
    if (lane == 0) atomicAdd(&focal_acc, -ef);
  }
  __syncthreads();
  // This block's partial row: each camera's sums in world axes and in A (the column sums add the
  // blocks' rows in FP64 and rotate each camera's total into its axes once).
  A* out = reinterpret_cast<A*>(P.acc_part) + size_t(blockIdx.x) * m;
  for (uint32_t j = threadIdx.x; j < 6 * C; j += blockDim.x) out[j] = acc[(j % 6) * C + j / 6];
  if (SHARED && threadIdx.x == 0) out[m - 1] = A(focal_acc);
}

// Column j of the one-pass product's partial rows summed over the blocks in a fixed order (world
// axes for a camera row), from FP32 rows when the product ran on FP32 factors.
__device__ inline double partial_column(const Params& P, bool f32, uint32_t j, uint32_t first, uint32_t step) {
  double s = 0;
  if (f32) {
    const float* rows = reinterpret_cast<const float*>(P.acc_part);
    for (uint32_t g = first; g < P.prod_blocks; g += step) s += double(__ldcg(rows + size_t(g) * P.m + j));
  } else {
    for (uint32_t g = first; g < P.prod_blocks; g += step) s += __ldcg(P.acc_part + size_t(g) * P.m + j);
  }
  return s;
}

// Row r (0..5) of camera c's world-axis sums w6 turned into the camera's axes: R w for the rotation
// rows (0..2), R w for the translation rows (3..5).
__device__ inline double camera_axis_row(const double* R, const double* w6, uint32_t r) {
  const uint32_t i = r % 3, b = r < 3 ? 0 : 3;
  return R[3 * i] * w6[b] + R[3 * i + 1] * w6[b + 1] + R[3 * i + 2] * w6[b + 2];
}

// The column sums of the one-pass product's partial rows (fixed order), then the camera rows of
// S p = U_c p_c + H_cf p_f + sum, their p . Sp share; the last block adds the focal row and forms
// alpha (the reference's breakdown checks).
constexpr uint32_t kColumnRows = 30;  // rows of a column block: five whole cameras

template <bool SHARED>
__global__ void __launch_bounds__(256) k_product_columns(Params P) {
  __shared__ double part[8][33];
  __shared__ double world[32];
  __shared__ double red[2 * 8];
  if (P.state[S_CG_ACTIVE] == 0) return;
  const uint32_t n = 6 * P.C, m = P.m;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t j = blockIdx.x * kColumnRows + lane;
  const bool row = uint32_t(lane) < kColumnRows && j < m;
  part[warp][lane] = row ? partial_column(P, P.F32 != nullptr, j, warp, 8) : 0.0;
  __syncthreads();
  double v[2] = {0, 0};
  if (warp == 0) {
    double sum = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) sum += part[w][lane];
    world[lane] = sum;
    __syncwarp();
    if (row && j < n) {
      const uint32_t c = j / 6, r = j % 6;
      sum = camera_axis_row(P.poses + 12 * size_t(c), world + 6 * (uint32_t(lane) / 6), r);
      const double* U = P.camU + 21 * size_t(c);
      const double* pc = P.p + 6 * size_t(c);
      double up = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) up += U[sym6(r, k)] * pc[k];
      double sp = up + (P.active[c] != 0 ? sum : 0.0);  // a fixed camera's rows: U = I, p = 0
      if (SHARED) {
        sp += P.camHcf[j] * P.p[m - 1];
        v[1] = P.camHcf[j] * P.p[j];
      }
      P.Sp[j] = sp;
      v[0] = P.p[j] * sp;
    } else if (SHARED && row && j == n) {
      P.Sp[n] = sum;
    }
  }
  block_sum(v, red);
  if (threadIdx.x == 0) {
    P.blk_part[4 * blockIdx.x] = v[0];
    P.blk_part[4 * blockIdx.x + 1] = v[1];
  }
  if (!last_block(P.ticket)) return;
  double t[2] = {0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    t[0] += __ldcg(P.blk_part + 4 * b);
    t[1] += __ldcg(P.blk_part + 4 * b + 1);
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

// ---- K12: one PCG step, in three short kernels --------------------------------------------------
//
// k_product_reduce   per camera row: S p = U_c p_c + H_cf p_f - sum over the camera's chunks; the
//                    p . Sp share; the focal row's shares; its last block completes the focal row
//                    and forms alpha = rho / p.Sp (with the reference's breakdown checks).
// k_pcg_update       x += alpha p, r -= alpha Sp, z = M^-1 r by camera blocks (252 rows per block,
//                    so no camera straddles two blocks); its last block forms the residual, rho,
//                    the convergence test and beta.
// k_pcg_direction    p = z + beta p.

constexpr int kReduceThreads = 256;
constexpr int kUpdateRows = 252;  // 42 cameras per block
constexpr int kUpdateThreads = 256;

template <bool SHARED>
__global__ void __launch_bounds__(kReduceThreads) k_product_reduce(Params P) {
  __shared__ double red[3 * (kReduceThreads / 32)];
  if (P.state[S_CG_ACTIVE] == 0) return;
  const uint32_t n = 6 * P.C, m = P.m;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  double v[3] = {0, 0, 0};  // p . Sp over camera rows, H_cf . p, observation share of the focal row
  if (j < n) {
    const uint32_t c = j / 6, r = j % 6;
    double sum = 0;
    for (uint32_t ch = P.cam_chunk[c]; ch < P.cam_chunk[c + 1]; ch++) sum += P.chunk_prod[8 * size_t(ch) + r];
    const double* U = P.camU + 21 * size_t(c);
    double pc[6];
    load6(P.p + 6 * size_t(c), pc);
    double up = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) up += U[sym6(r, k)] * pc[k];
    double sp = up - sum;
    if (SHARED) {
      sp += P.camHcf[j] * P.p[m - 1];
      v[1] = P.camHcf[j] * pc[r];
    }
    P.Sp[j] = sp;
    v[0] = pc[r] * sp;
  }
  if (SHARED)
    for (uint32_t ch = j; ch < P.nchunks; ch += gridDim.x * blockDim.x) v[2] += P.chunk_prod[8 * size_t(ch) + 6];
  block_sum(v, red);
  if (threadIdx.x == 0) {
    P.blk_part[4 * blockIdx.x] = v[0];
    P.blk_part[4 * blockIdx.x + 1] = v[1];
    P.blk_part[4 * blockIdx.x + 2] = v[2];
  }
  if (!last_block(P.ticket)) return;
  double t[3] = {0, 0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    for (int k = 0; k < 3; k++) t[k] += __ldcg(P.blk_part + 4 * b + k);
  block_sum(t, red);
  if (threadIdx.x != 0) return;
  double* st = P.state;
  double den = t[0];
  if (SHARED) {
    const double pf = P.p[n];
    const double spf = st[S_FOCAL_DIAG] * pf + t[1] - t[2];
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
  // An inner run ends at the solve's tolerance, or (mixed form) once it has reduced its own starting
  // residual as far as its FP32 product resolves; the FP64 refinement then takes over.
  if (residual <= fmax(P.tol * P.tol * st[S_R0], P.tol_inner * P.tol_inner * st[S_INNER_R0])) {
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
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < P.C) {
    double v[6];
    for (int k = 0; k < 6; k++) {
      v[k] = P.z[6 * c + k] + beta * P.p[6 * c + k];
      P.p[6 * c + k] = v[k];
    }
    to_world(P.poses + 12 * size_t(c), v, P.pw + 6 * size_t(c));
  } else if (c == P.C && P.shared) {
    P.p[P.m - 1] = P.z[P.m - 1] + beta * P.p[P.m - 1];
  }
}

// ---- Diagnostics: S p of one product, every row, into `out` --------------------------------------
//
// `onepass`: from the one-pass product's partial rows (which hold -sum_i W_i y_p in world axes),
// else from the two-pass product's chunk sums (+sum_i W_i y_p); then U_c p_c, the focal couplings
// and the focal row, as k_product_columns and k_product_reduce form them.  Writes no state.
__global__ void __launch_bounds__(256) k_product_rows(Params P, int onepass, double* out) {
  const uint32_t n = 6 * P.C, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    const uint32_t c = j / 6, r = j % 6;
    double sum = 0;
    if (onepass) {
      if (P.active[c] != 0) {
        // The world-axis sums of this row's triple, rotated into the camera's axes.
        double w6[6] = {0, 0, 0, 0, 0, 0};
        const uint32_t base = r < 3 ? 0 : 3;
        for (uint32_t k = 0; k < 3; k++) w6[base + k] = partial_column(P, P.F32 != nullptr, 6 * c + base + k, 0, 1);
        sum = camera_axis_row(P.poses + 12 * size_t(c), w6, r);
      }
    } else {
      for (uint32_t ch = P.cam_chunk[c]; ch < P.cam_chunk[c + 1]; ch++) sum -= P.chunk_prod[8 * size_t(ch) + r];
    }
    const double* U = P.camU + 21 * size_t(c);
    const double* pc = P.p + 6 * size_t(c);
    double sp = sum;
    for (int k = 0; k < 6; k++) sp += U[sym6(r, k)] * pc[k];
    if (P.shared) sp += P.camHcf[j] * P.p[P.m - 1];
    out[j] = sp;
  } else if (j == n && P.shared) {
    double sp = P.state[S_FOCAL_DIAG] * P.p[n];
    for (uint32_t k = 0; k < n; k++) sp += P.camHcf[k] * P.p[k];
    if (onepass)
      sp += partial_column(P, P.F32 != nullptr, n, 0, 1);
    else
      for (uint32_t ch = 0; ch < P.nchunks; ch++) sp -= P.chunk_prod[8 * size_t(ch) + 6];
    out[n] = sp;
  }
}

// ---- The device-side PCG loop --------------------------------------------------------------------
//
// A solve runs its PCG steps as one CUDA graph: a while node whose body is one step (the product,
// the column sums with alpha, the x/r/z update with beta, the new direction) followed by
// k_pcg_loop_next.  The loop ends on the device when the PCG stops (converged, broken down) or its
// budget of steps is spent, with no host round trip per step and no launches past convergence.
// k_pcg_loop_next runs at the end of every body iteration, so the loop always ends within its budget.

__global__ void k_pcg_loop_begin(Params P, uint32_t limit) {
  P.state[S_LOOP_ITERS] = 0;
  P.state[S_LOOP_LIMIT] = limit;
}

__global__ void k_pcg_loop_next(Params P) {
  double* st = P.state;
  const double iters = st[S_LOOP_ITERS] + 1;
  st[S_LOOP_ITERS] = iters;
  cudaGraphSetConditional(P.pcg_loop, st[S_CG_ACTIVE] != 0 && iters < st[S_LOOP_LIMIT] ? 1u : 0u);
}

// ---- Mixed form: FP64 iterative refinement of the PCG solution ----------------------------------
//
// After the PCG ran on the FP32-factor product, k_refine_begin marks the refinement, an FP64 product
// evaluates S x (launched with p := x: one pass over the FP64 factors, which the mixed form keeps
// beside the FP32 ones because that costs less than recomputing the FP64 Jacobians in the two-pass
// product, or that two-pass product when the engine keeps no factors), and k_refine forms the true residual
// r = b - S x, z = M^-1 r, p = z, rho and r.r.  Its last block adds the focal row and either accepts
// x (r.r within the tolerance: the PCG stays finished) or restarts the PCG from x with this r.

__global__ void k_refine_begin(Params P) {
  double* st = P.state;
  st[S_REFINE] = (st[S_ACTIVE] != 0 && st[S_CG_FAILED] == 0 && st[S_R0] > 0) ? 1 : 0;
}

// The refinement's vector x in world axes, for the one-pass product over the FP64 factors.
__global__ void k_refine_direction(Params P) {
  if (P.state[S_REFINE] == 0) return;
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < P.C) to_world(P.poses + 12 * size_t(c), P.x + 6 * size_t(c), P.pw + 6 * size_t(c));
}

__global__ void __launch_bounds__(kUpdateThreads) k_refine(Params P) {
  __shared__ double rs[kUpdateRows];
  __shared__ double ws[kUpdateRows];
  __shared__ double red[4 * (kUpdateThreads / 32)];
  double* st = P.state;
  if (st[S_REFINE] == 0) return;
  const uint32_t n = 6 * P.C;
  const uint32_t row = blockIdx.x * kUpdateRows + threadIdx.x;
  const bool mine = threadIdx.x < uint32_t(kUpdateRows) && row < n;
  const bool onepass = P.factored && P.F;
  // The one-pass product (over the FP64 factors) left world-axis FP64 partial rows; a block's rows
  // are whole cameras, so each camera's column sums meet in shared memory to be rotated.
  if (onepass && threadIdx.x < uint32_t(kUpdateRows)) ws[threadIdx.x] = mine ? partial_column(P, false, row, 0, 1) : 0.0;
  __syncthreads();
  double rr = 0;
  double v[4] = {0, 0, 0, 0};  // r.r, r.z (camera rows), H_cf . x, observation share of the focal row
  if (mine) {
    const uint32_t c = row / 6, j = row % 6;
    // sum_i W_i y_p of the camera: the column sum of the one-pass product's partial rows (which hold
    // its negative; a fixed camera's rows are discarded), or the two-pass product's chunk sums.
    double sum = 0;
    if (onepass) {
      if (P.active[c] != 0)
        sum = -camera_axis_row(P.poses + 12 * size_t(c), ws + (threadIdx.x - j), j);
    } else {
      for (uint32_t ch = P.cam_chunk[c]; ch < P.cam_chunk[c + 1]; ch++) sum += P.chunk_prod[8 * size_t(ch) + j];
    }
    const double* U = P.camU + 21 * size_t(c);
    const double* xc = P.x + 6 * size_t(c);
    double ux = 0;
    for (int k = 0; k < 6; k++) ux += U[sym6(j, k)] * xc[k];
    double sx = ux - sum;
    if (P.shared) {
      sx += P.camHcf[row] * P.x[P.m - 1];
      v[2] = P.camHcf[row] * xc[j];
    }
    rr = P.camRhs[row] - sx;
    P.r[row] = rr;
    rs[threadIdx.x] = rr;
  }
  if (P.shared) {
    if (onepass)
      for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < P.prod_blocks; b += gridDim.x * blockDim.x)
        v[3] -= P.acc_part[size_t(b) * P.m + (P.m - 1)];
    else
      for (uint32_t ch = blockIdx.x * blockDim.x + threadIdx.x; ch < P.nchunks; ch += gridDim.x * blockDim.x)
        v[3] += P.chunk_prod[8 * size_t(ch) + 6];
  }
  __syncthreads();
  if (mine) {
    const uint32_t jr = row % 6, base = threadIdx.x - jr;
    const double* Mi = P.camMinv + 36 * size_t(row / 6) + 6 * jr;
    const double zz = Mi[0] * rs[base] + Mi[1] * rs[base + 1] + Mi[2] * rs[base + 2] + Mi[3] * rs[base + 3] +
                      Mi[4] * rs[base + 4] + Mi[5] * rs[base + 5];
    P.z[row] = zz;
    P.p[row] = zz;
    v[0] = rr * rr;
    v[1] = rr * zz;
  }
  __syncthreads();
  if (threadIdx.x < uint32_t(kUpdateRows / 6)) {
    const uint32_t c = blockIdx.x * (kUpdateRows / 6) + threadIdx.x;
    if (c < P.C) {
      double pc[6];
      for (int k = 0; k < 6; k++) pc[k] = P.p[6 * c + k];
      to_world(P.poses + 12 * size_t(c), pc, P.pw + 6 * size_t(c));
    }
  }
  block_sum(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) P.blk_part[4 * blockIdx.x + k] = v[k];
  if (!last_block(P.ticket + 2)) return;
  double t[4] = {0, 0, 0, 0};
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    for (int k = 0; k < 4; k++) t[k] += __ldcg(P.blk_part + 4 * b + k);
  block_sum(t, red);
  if (threadIdx.x != 0) return;
  P.ticket[2] = 0;
  double residual = t[0], rho = t[1];
  if (P.shared) {
    const double xf = P.x[n];
    const double sxf = st[S_FOCAL_DIAG] * xf + t[2] - t[3];
    const double rf = st[S_FOCAL_RHS] - sxf, zf = st[S_FOCAL_INV] * rf;
    P.r[n] = rf;
    P.z[n] = zf;
    P.p[n] = zf;
    residual += rf * rf;
    rho += rf * zf;
  }
  st[S_REFINE] = 0;
  st[S_R2] = residual;
  if (residual <= P.tol * P.tol * st[S_R0]) {
    st[S_CG_ACTIVE] = 0;
    st[S_CG_CONVERGED] = 1;
  } else if (rho > 0) {
    st[S_RHO] = rho;
    st[S_INNER_R0] = residual;
    st[S_CG_ACTIVE] = 1;
    st[S_REFINED] += 1;
  } else {
    st[S_CG_FAILED] = 1;  // no descent direction, or a residual that is not finite
  }
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
    to_world(pose, P.x + 6 * size_t(c), P.xw + 6 * size_t(c));
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

// W_i^T x of one observation for the candidate update: from the stored FP64 factors when the
// engine keeps them (both forms), else recomputed in FP64.
__device__ inline void update_wt(const Params& P, uint32_t i, uint32_t c, uint32_t pt, double fscale, double xf,
                                 bool shared, double t[3]) {
  t[0] = t[1] = t[2] = 0;
  if (P.factored && P.F) {
    Factors<double> f;
    load_factors(static_cast<const double*>(P.F), P.Mpad, i, f);
    double xw[6];
    load6(P.xw + 6 * size_t(c), xw);
    factor_wt(f, xw, xf, P.active[c] != 0, directional(P, pt), shared, t);
    return;
  }
  if (P.factored && P.F32) {  // mixed form: the back-substitution's W_i^T x in FP32
    Factors<float> f;
    load_factors(static_cast<const float*>(P.F32), P.Mpad, i, f);
    double xw[6];
    load6(P.xw + 6 * size_t(c), xw);
    factor_wt(f, xw, xf, P.active[c] != 0, directional(P, pt), shared, t);
    return;
  }
  double pose[12], xc[6];
  Geo g;
  if (observe(P, i, c, pt, fscale, pose, g)) {
    load6(P.x + 6 * size_t(c), xc);
    wt_product(g, pose, xc, xf, P.active[c] != 0, directional(P, pt), shared, t);
  }
}

// ---- K14/K16/K17: candidate points and the candidate cost ---------------------------------------

// The candidate point: X + V^-1 (b_p - sum_i W_i^T x), then the bearing or similarity
// normalisation of the gauge.
__device__ inline void candidate_point(const Params& P, uint32_t pt, const double s[3], double X[3]) {
  double vb[6];
  load6(P.pblk + 12 * size_t(pt), vb);
  const double* bb = P.pblk + 12 * size_t(pt) + 6;
  const double r0 = bb[0] - s[0], r1 = bb[1] - s[1], r2 = bb[2] - s[2];
  const double* X0 = P.points + 3 * size_t(pt);
  X[0] = X0[0] + (vb[0] * r0 + vb[1] * r1 + vb[2] * r2);
  X[1] = X0[1] + (vb[1] * r0 + vb[3] * r1 + vb[4] * r2);
  X[2] = X0[2] + (vb[2] * r0 + vb[4] * r1 + vb[5] * r2);
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

__device__ inline void candidate_obs(const Params& P, uint32_t i, uint32_t pt, const double X[3], double fscale_trial,
                                     double& cost, double& sq) {
  const uint32_t c = P.obs_camera[i];
  double pose[12];
  load_pose(P.tposes, c, pose);
  const Camera k = camera_at(P, c, fscale_trial);
  const double2 uv = reinterpret_cast<const double2*>(P.pixels)[i];
  double oc, os;
  candidate_cost(pose, k, X, directional(P, pt), uv.x, uv.y, P.huber, oc, os);
  cost += oc;
  sq += os;
}

template <bool SHARED>
__global__ void __launch_bounds__(kPointThreads, TBA_SCHUR_MIN_BLOCKS) k_update_points(Params P) {
  __shared__ double red[2 * (kPointThreads / 32)];
  const double* st = P.state;
  if (st[S_ACTIVE] == 0 || st[S_CG_FAILED] != 0 || st[S_TRIAL_VALID] == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const double fscale = focal_scale(P, st[S_LOG_FOCAL]), fscale_trial = focal_scale(P, st[S_LOG_FOCAL_TRIAL]);
  const double xf = SHARED ? P.x[P.m - 1] : 0.0;
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
        seg = int(pt);
        update_wt(P, i, P.obs_camera[i], pt, fscale, xf, SHARED, s);
      }
      const Runs runs = lane_runs(seg, lane);
      run_scan(s, runs);
      const bool tail = valid && run_tail(runs, lane);
      double X[3] = {0, 0, 0};
      if (tail) candidate_point(P, pt, s, X);
      const unsigned tails = __ballot_sync(kFull, tail);
      const int src = valid ? __ffs(tails & (kFull << lane)) - 1 : lane;
      for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], src);
      if (valid) candidate_obs(P, i, pt, X, fscale_trial, cs[0], cs[1]);
    } else {
      const uint32_t pt = P.obs_point[o0];
      double s[3] = {0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs)
        if (base + lane < n) {
          const uint32_t i = o0 + base + lane;
          double u[3];
          update_wt(P, i, P.obs_camera[i], pt, fscale, xf, SHARED, u);
          s[0] += u[0];
          s[1] += u[1];
          s[2] += u[2];
        }
      warp_allsum(s);
      double X[3] = {0, 0, 0};
      if (lane == 0) candidate_point(P, pt, s, X);
      for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], 0);
      for (uint32_t base = 0; base < n; base += kTaskObs)
        if (base + lane < n) candidate_obs(P, o0 + base + lane, pt, X, fscale_trial, cs[0], cs[1]);
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
  const uint32_t a = (6 * p.C + kReduceThreads - 1) / kReduceThreads, b = (p.m + kUpdateRows - 1) / kUpdateRows;
  const uint32_t c = (p.m + kColumnRows - 1) / kColumnRows;
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

uint32_t product_max_unknowns() { return uint32_t(kStagedSmemLimit / sizeof(double)) - 64; }

// Bytes of a block's camera sum: the factors' type.  With FP32 factors a block sums its share of
// each camera in FP32 (about 28 terms a camera and block at 1,500 cameras / 6.18M observations) and
// the blocks' shares are summed in FP64; FP64 block sums (8-byte shared atomics) measured 14% slower
// per product (0.138 against 0.121 ms there).
size_t product_sum_word(const Params& p) { return p.F32 ? sizeof(float) : sizeof(double); }

// The direction is staged in shared memory when the camera sums and it fit one block.
bool product_staged(const Params& p) {
  const size_t word = p.F32 ? sizeof(float) : sizeof(double);
  return product_sums_bytes(p.C, product_sum_word(p)) + 6 * size_t(p.C) * word <= size_t(kStagedSmemLimit);
}

size_t product_smem_bytes(const Params& p) {
  const size_t word = p.F32 ? sizeof(float) : sizeof(double);
  return product_sums_bytes(p.C, product_sum_word(p)) + (product_staged(p) ? 6 * size_t(p.C) * word : 0);
}

// The FP64 staged product takes 1,024 threads on large problems (enough tasks a warp).
bool product_wide(const Params& p) { return !p.F32 && product_staged(p) && p.M >= kWideObservations; }

int product_threads(const Params& p) {
  if (!product_staged(p)) return kProductThreads;
  return p.F32 ? kStagedThreadsF32 : (product_wide(p) ? kStagedThreadsWide : kStagedThreads);
}

namespace {

// The product kernel of a solve: focal route, factor type, sum type and staging.
template <bool SHARED>
const void* product_kernel_of(const Params& p) {
  const bool st = product_staged(p);
  if (!p.F32) {
    if (product_wide(p)) return reinterpret_cast<const void*>(k_product_f<SHARED, double, double, true, true>);
    return st ? reinterpret_cast<const void*>(k_product_f<SHARED, double, double, true>)
              : reinterpret_cast<const void*>(k_product_f<SHARED, double, double, false>);
  }
  return st ? reinterpret_cast<const void*>(k_product_f<SHARED, float, float, true>)
            : reinterpret_cast<const void*>(k_product_f<SHARED, float, float, false>);
}

const void* product_kernel(const Params& p) { return p.shared ? product_kernel_of<true>(p) : product_kernel_of<false>(p); }

}  // namespace

cudaError_t configure_kernels() {
  const int bytes = kStagedSmemLimit;  // the products also hold a few static bytes
  const void* kernels[] = {
      reinterpret_cast<const void*>(k_product_f<false, double, double, false>),
      reinterpret_cast<const void*>(k_product_f<true, double, double, false>),
      reinterpret_cast<const void*>(k_product_f<false, double, double, true>),
      reinterpret_cast<const void*>(k_product_f<true, double, double, true>),
      reinterpret_cast<const void*>(k_product_f<false, double, double, true, true>),
      reinterpret_cast<const void*>(k_product_f<true, double, double, true, true>),
      reinterpret_cast<const void*>(k_product_f<false, float, float, false>),
      reinterpret_cast<const void*>(k_product_f<true, float, float, false>),
      reinterpret_cast<const void*>(k_product_f<false, float, float, true>),
      reinterpret_cast<const void*>(k_product_f<true, float, float, true>),
  };
  for (const void* f : kernels) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int product_blocks_per_sm(const Params& p) {
  int n = 0;
  Params q = p;
  q.shared = 1;  // both focal routes have the same resources
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, product_kernel(q), product_threads(p), product_smem_bytes(p)) !=
      cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

void launch_initialize(const Params& p, cudaStream_t s) {
  k_initialize<<<1, 1, 0, s>>>(p);
  const uint32_t n = p.M > p.C ? p.M : p.C;
  k_setup<<<(n + 255) / 256, 256, 0, s>>>(p);
}
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
  if (p.factored) {
    Params q = p;
    void* args[] = {&q};
    cudaLaunchKernel(product_kernel(p), dim3(p.prod_blocks), dim3(product_threads(p)), args, product_smem_bytes(p), s);
    return;
  }
  if (p.shared) {
    k_schur_points<true><<<p.task_blocks, kPointThreads, 0, s>>>(p);
    k_schur_cameras<true><<<p.nchunks, kCameraThreads, 0, s>>>(p);
  } else {
    k_schur_points<false><<<p.task_blocks, kPointThreads, 0, s>>>(p);
    k_schur_cameras<false><<<p.nchunks, kCameraThreads, 0, s>>>(p);
  }
}
void launch_product_finish(const Params& p, cudaStream_t s) {
  if (p.factored) {
    if (p.shared) k_product_columns<true><<<(p.m + kColumnRows - 1) / kColumnRows, 256, 0, s>>>(p);
    else k_product_columns<false><<<(p.m + kColumnRows - 1) / kColumnRows, 256, 0, s>>>(p);
  } else {
    const uint32_t rb = (6 * p.C + kReduceThreads - 1) / kReduceThreads;
    if (p.shared) k_product_reduce<true><<<rb, kReduceThreads, 0, s>>>(p);
    else k_product_reduce<false><<<rb, kReduceThreads, 0, s>>>(p);
  }
  k_pcg_update<<<(p.m + kUpdateRows - 1) / kUpdateRows, kUpdateThreads, 0, s>>>(p);
  k_pcg_direction<<<(p.C + 1 + 255) / 256, 256, 0, s>>>(p);
}
void launch_pcg_loop_begin(const Params& p, uint32_t limit, cudaStream_t s) { k_pcg_loop_begin<<<1, 1, 0, s>>>(p, limit); }
void launch_pcg_loop_next(const Params& p, cudaStream_t s) { k_pcg_loop_next<<<1, 1, 0, s>>>(p); }
void launch_refine(const Params& p, cudaStream_t s) {
  k_refine_begin<<<1, 1, 0, s>>>(p);
  Params q = p;
  q.refine = 1;
  q.p = p.x;
  if (p.factored && p.F) {
    // S x in one pass over stored FP64 factors.
    q.F32 = nullptr;
    k_refine_direction<<<(p.C + 255) / 256, 256, 0, s>>>(q);
    launch_product(q, s);
  } else if (p.shared) {  // S x by the two-pass product, recomputing the FP64 Jacobians
    k_schur_points<true><<<p.task_blocks, kPointThreads, 0, s>>>(q);
    k_schur_cameras<true><<<p.nchunks, kCameraThreads, 0, s>>>(q);
  } else {
    k_schur_points<false><<<p.task_blocks, kPointThreads, 0, s>>>(q);
    k_schur_cameras<false><<<p.nchunks, kCameraThreads, 0, s>>>(q);
  }
  k_refine<<<(6 * p.C + kUpdateRows - 1) / kUpdateRows, kUpdateThreads, 0, s>>>(p);
}
void launch_product_rows(const Params& p, double* out, cudaStream_t s) {
  k_product_rows<<<(p.m + 255) / 256, 256, 0, s>>>(p, p.factored ? 1 : 0, out);
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
