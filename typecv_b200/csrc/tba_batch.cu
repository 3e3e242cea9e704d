// The batched block solver (tba_batch.cuh), sm_100a.
//
// One persistent launch solves a whole batch.  Each block repeatedly takes the next problem from
// a queue ordered largest first and runs that problem's LM loop to the end:
//
//   b_init / b_cost          initializeBundle + bundleMetricPartials/finishBundleMetrics (K1/K3/K4)
//   b_point_pass             linearizeBundle + bundlePointBlocks + the focal sums (K2/K5/K21);
//                            stores the 12 world-axis Jacobian factors of every observation
//   b_camera_pass            bundleCameraRows + invertBundleCameraColumns (K6/K8/K21), camera-major,
//                            sums flushed into shared memory when a lane's camera changes
//   b_pcg_init, b_product_f, initializeBundleCg + bundleSchurPoint/bundleSchurCamera +
//   b_columns, b_pcg_update  advanceBundleCg (K9-K12): the whole PCG state (6C + 1 unknowns),
//                            the camera blocks and the preconditioner live in shared memory
//   b_refine, b_product_r    mixed form: the FP64 residual of the FP32-factor PCG solution (FP64
//                            recompute product); the restarted run reads an FP64 copy of the factors
//   b_update_cameras,        updateBundleCandidate + bundleCandidateGauge +
//   b_update_points          normalizeBundleCandidate + bundleCandidatePartials +
//                            acceptBundleCandidate + commitBundleCandidate (K14-K19)
//   b_pack                   packBundleResult (K20)
//
// (kernel names of src/sfm/bundle/gpu/bundle.shade.ts and joint-focal.shade.ts).  Barriers
// replace the grid engine's kernel boundaries; the LM and PCG loops run on the device with no
// host round trip.  Point blocks, candidate points and factors stay in HBM.
#include <cuda_runtime.h>

#include <type_traits>

#include "tba_batch.cuh"
#include "tba_engine.cuh"
#include "tba_math.cuh"
#include "tba_warp.cuh"

namespace tba {
namespace {

// Pointers into the block's dynamic shared memory and the problem-independent arguments.
struct Sh {
  double *st, *scal, *red, *pose, *tpose, *cam, *rlim, *U, *Minv, *rhs, *hcf, *aux;
  double *x, *r, *p, *z, *Sp, *acc, *pw, *xw;
  double huber, tol, tol_inner, stall;
  uint32_t iterations, max_cg;
  int ok, ok2;
  uint32_t job;
};

// The layout of the dynamic shared memory for Cm cameras (every section 16-byte aligned).
__host__ __device__ inline uint32_t layout_words(uint32_t Cm, double* base, Sh* S) {
  const uint32_t mm = (6 * Cm + 2);
  uint32_t at = 0;
  auto take = [&](uint32_t n) {
    const uint32_t o = at;
    at += (n + 1) & ~1u;
    return base ? base + o : nullptr;
  };
  double* st = take(S_WORDS);
  double* scal = take(8);
  double* red = take(8 * 32);
  double* pose = take(12 * Cm);
  double* tpose = take(12 * Cm);
  double* cam = take(6 * Cm);
  double* rlim = take(Cm);
  double* U = take(21 * Cm);
  double* Minv = take(36 * Cm);
  double* rhs = take(6 * Cm);
  double* hcf = take(6 * Cm);
  double* aux = take(27 * Cm);
  double* x = take(mm);
  double* r = take(mm);
  double* p = take(mm);
  double* z = take(mm);
  double* Sp = take(mm);
  double* acc = take(mm);
  double* pw = take(6 * Cm);
  double* xw = take(6 * Cm);
  if (S) {
    S->st = st; S->scal = scal; S->red = red; S->pose = pose; S->tpose = tpose; S->cam = cam;
    S->rlim = rlim; S->U = U; S->Minv = Minv; S->rhs = rhs; S->hcf = hcf; S->aux = aux;
    S->x = x; S->r = r; S->p = p; S->z = z; S->Sp = Sp; S->acc = acc; S->pw = pw; S->xw = xw;
  }
  return at;
}

// Block sum of N values, the result in every thread.
template <int N>
__device__ __forceinline__ void bsum_all(double (&v)[N], double* red) {
  warp_allsum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0)
    for (int n = 0; n < N; n++) red[warp * N + n] = v[n];
  __syncthreads();
  for (int n = 0; n < N; n++) {
    double s = 0;
    for (int w = 0; w < nw; w++) s += red[w * N + n];
    v[n] = s;
  }
  __syncthreads();
}

__device__ __forceinline__ Camera cam_at(const Sh& S, uint32_t c, double fscale) {
  const double* k = S.cam + 6 * c;
  return Camera{k[0] * fscale, k[1] * fscale, k[2], k[3], k[4], k[5]};
}

template <bool SHARED>
__device__ __forceinline__ double fscale_of(double log_scale) {
  return SHARED ? exp(log_scale) : 1.0;
}

__device__ __forceinline__ void pose_of(const double* poses, uint32_t c, double pose[12]) {
  for (int j = 0; j < 12; j++) pose[j] = poses[12 * c + j];
}

// Observation i (point-major) of point pt in camera c at the accepted scene.
__device__ __forceinline__ bool b_observe(const BatchProblem& Q, const Sh& S, uint32_t i, uint32_t c, uint32_t pt,
                                          double fscale, double pose[12], Geo& g) {
  pose_of(S.pose, c, pose);
  const Camera k = cam_at(S, c, fscale);
  return geometry(pose, k, S.rlim[c], Q.points + 3 * size_t(pt), false, Q.pixels[2 * size_t(i)],
                  Q.pixels[2 * size_t(i) + 1], S.huber, g);
}

// ---- K1, K3/K4 ----------------------------------------------------------------------------------

__device__ __noinline__ void b_init(const BatchProblem& Q, Sh& S) {
  const uint32_t C = Q.C, P = Q.P;
  for (uint32_t j = threadIdx.x; j < S_WORDS; j += blockDim.x) S.st[j] = 0;
  for (uint32_t j = threadIdx.x; j < 12 * C; j += blockDim.x) S.pose[j] = Q.poses0[j];
  for (uint32_t j = threadIdx.x; j < 6 * C; j += blockDim.x) S.cam[j] = Q.cams[j];
  for (uint32_t j = threadIdx.x; j < 3 * P; j += blockDim.x) Q.points[j] = Q.points0[j];
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) S.rlim[c] = radial_limit(S.cam[6 * c + 4], S.cam[6 * c + 5]);
  if (threadIdx.x == 0) {
    double* st = S.st;
    st[S_LAMBDA] = 1e-3;
    st[S_ACTIVE] = 1;
    const double* a = S.pose + 12 * Q.anchor;
    const double* b = S.pose + 12 * Q.scale_view;
    double o[3], s[3];
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
  }
  __syncthreads();
}

__device__ __noinline__ void b_cost(const BatchProblem& Q, Sh& S, bool shared) {
  double v[3] = {0, 0, 0};  // cost, squared error, invalid projections
  const double fscale = shared ? exp(S.st[S_LOG_FOCAL]) : 1.0;
  for (uint32_t i = threadIdx.x; i < Q.M; i += blockDim.x) {
    double pose[12];
    Geo g;
    if (!b_observe(Q, S, i, Q.obs_camera[i], Q.obs_point[i], fscale, pose, g)) {
      v[2] += 1;
      continue;
    }
    v[0] += robust_cost(sqrt(g.sq), S.huber);
    v[1] += g.sq;
  }
  bsum_all(v, S.red);
  if (threadIdx.x == 0 && S.st[S_INPUT_ERROR] == 0) {
    double* st = S.st;
    if (v[2] > 0) {
      st[S_INPUT_ERROR] = 2;
      st[S_ACTIVE] = 0;
    } else {
      st[S_COST] = st[S_COST0] = v[0];
      st[S_SSE] = st[S_SSE0] = v[1];
      if (v[0] < 1e-20) st[S_ACTIVE] = 0;
    }
  }
  __syncthreads();
}

// ---- K2/K5/K21: point blocks and the factors ----------------------------------------------------

template <bool SHARED, typename T>
__device__ __forceinline__ void b_point_obs(const BatchProblem& Q, const Sh& S, uint32_t i, uint32_t pt, double fscale,
                                            double (&v)[13], double& hff, double& bf) {
  double pose[12];
  Geo g;
  if (!b_observe(Q, S, i, Q.obs_camera[i], pt, fscale, pose, g)) {
    v[12] = 1;
    return;
  }
  double jp[2][3];
  for (int c = 0; c < 3; c++) {
    jp[0][c] = g.du[0] * pose[c] + g.du[1] * pose[3 + c] + g.du[2] * pose[6 + c];
    jp[1][c] = g.dv[0] * pose[c] + g.dv[1] * pose[3 + c] + g.dv[2] * pose[6 + c];
  }
  T* F = static_cast<T*>(Q.F);
  const size_t stride = Q.Mpad;
  for (int c = 0; c < 3; c++) {
    F[c * stride + i] = T(g.q[0] * pose[c] + g.q[1] * pose[3 + c] + g.q[2] * pose[6 + c]);
    F[(3 + c) * stride + i] = T(jp[0][c]);
    F[(6 + c) * stride + i] = T(jp[1][c]);
  }
  F[9 * stride + i] = T(g.w);
  F[10 * stride + i] = T(g.jf[0]);
  F[11 * stride + i] = T(g.jf[1]);
  if (sizeof(T) == 4) {  // the mixed form's FP64 copy
    double* D = Q.F64;
    for (int c = 0; c < 3; c++) {
      D[c * stride + i] = g.q[0] * pose[c] + g.q[1] * pose[3 + c] + g.q[2] * pose[6 + c];
      D[(3 + c) * stride + i] = jp[0][c];
      D[(6 + c) * stride + i] = jp[1][c];
    }
    D[9 * stride + i] = g.w;
    D[10 * stride + i] = g.jf[0];
    D[11 * stride + i] = g.jf[1];
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

template <bool SHARED>
__device__ __forceinline__ void b_point_finish(const BatchProblem& Q, const Sh& S, uint32_t pt, const double (&v)[13],
                                               double lambda, double& diag_pt, double& rhs_pt) {
  double V[9] = {v[0], v[1], v[2], v[1], v[3], v[4], v[2], v[4], v[5]};
  for (int j = 0; j < 3; j++) V[j * 4] += lambda * fmax(V[j * 4], 1e-10);
  double inv[6];
  const bool ok = v[12] == 0 && inverse3_spd(V, inv);
  double* blk = Q.pblk + 12 * size_t(pt);
  if (!ok) {
    S.st[S_POINT_FAILED] = 1;
    for (int k = 0; k < 12; k++) blk[k] = 0;
    return;
  }
  for (int k = 0; k < 6; k++) blk[k] = inv[k];
  blk[6] = v[6];
  blk[7] = v[7];
  blk[8] = v[8];
  if (SHARED) {
    const double I[9] = {inv[0], inv[1], inv[2], inv[1], inv[3], inv[4], inv[2], inv[4], inv[5]};
    for (int j = 0; j < 3; j++) {
      const double t = v[9] * I[j] + v[10] * I[3 + j] + v[11] * I[6 + j];
      diag_pt += t * v[9 + j];
      rhs_pt += t * v[6 + j];
    }
  }
}

template <bool SHARED, typename T>
__device__ __noinline__ void b_point_pass(const BatchProblem& Q, Sh& S) {
  const double lambda = S.st[S_LAMBDA], fscale = fscale_of<SHARED>(S.st[S_LOG_FOCAL]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double sc[4] = {0, 0, 0, 0};  // hff, bf, diag_pt, rhs_pt
  for (uint32_t t = warp; t < Q.ntasks; t += nw) {
    const uint32_t p0 = Q.tasks[t], p1 = Q.tasks[t + 1];
    const uint32_t o0 = Q.point_start[p0], n = Q.point_start[p1] - o0;
    if (n <= uint32_t(kTaskObs)) {
      double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      int seg = -1 - lane;
      uint32_t pt = 0;
      if (uint32_t(lane) < n) {
        pt = Q.obs_point[o0 + lane];
        seg = int(pt - p0);
        b_point_obs<SHARED, T>(Q, S, o0 + lane, pt, fscale, v, sc[0], sc[1]);
      }
      const Runs runs = lane_runs(seg, lane);
      run_scan(v, runs);
      if (uint32_t(lane) < n && run_tail(runs, lane))
        b_point_finish<SHARED>(Q, S, pt, v, lambda, sc[2], sc[3]);
    } else {
      double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (uint32_t base = 0; base < n; base += kTaskObs) {
        if (base + lane < n) {
          double u[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
          b_point_obs<SHARED, T>(Q, S, o0 + base + lane, p0, fscale, u, sc[0], sc[1]);
          for (int k = 0; k < 13; k++) v[k] += u[k];
        }
      }
      warp_allsum(v);
      if (lane == 0) b_point_finish<SHARED>(Q, S, p0, v, lambda, sc[2], sc[3]);
    }
  }
  bsum_all(sc, S.red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) S.scal[k] = sc[k];
  __syncthreads();
}

// ---- K6/K8/K21: camera blocks --------------------------------------------------------------------
//
// Each warp walks a contiguous range of the camera-major observation list, one observation per
// lane; a lane keeps its camera's sums in registers and adds them to the camera's shared-memory
// block (atomics) when its camera changes.

__device__ __forceinline__ void b_camera_rows(const Geo& g, double jc[2][6]) {
  pose_row(g.q, g.du, jc[0]);
  pose_row(g.q, g.dv, jc[1]);
}

template <int N>
__device__ __forceinline__ void b_flush(double (&a)[N], uint32_t c, double* dst_a, int na, double* dst_b, int nb,
                                        double* dst_c, int nc) {
  for (int j = 0; j < na; j++) atomicAdd(dst_a + na * c + j, a[j]);
  for (int j = 0; j < nb; j++) atomicAdd(dst_b + nb * c + j, a[na + j]);
  for (int j = 0; j < nc; j++) atomicAdd(dst_c + nc * c + j, a[na + nb + j]);
  for (int j = 0; j < N; j++) a[j] = 0;
}

template <bool SHARED>
__device__ __noinline__ void b_camera_pass(const BatchProblem& Q, Sh& S) {
  const uint32_t C = Q.C, M = Q.M;
  for (uint32_t j = threadIdx.x; j < 21 * C; j += blockDim.x) S.U[j] = 0;
  for (uint32_t j = threadIdx.x; j < 27 * C; j += blockDim.x) S.aux[j] = 0;
  for (uint32_t j = threadIdx.x; j < 6 * C; j += blockDim.x) {
    S.rhs[j] = 0;
    S.hcf[j] = 0;
  }
  __syncthreads();
  const double fscale = fscale_of<SHARED>(S.st[S_LOG_FOCAL]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t span = ((M + nw - 1) / nw + 31) / 32 * 32;
  const uint32_t k0 = warp * span, k1 = min(M, k0 + span);
  // Pass 1: U_c (lower triangle), b_c, H_cf.
  {
    double a[33];
    for (int j = 0; j < 33; j++) a[j] = 0;
    uint32_t cur = 0xffffffffu;
    for (uint32_t k = k0 + lane; k < k1; k += 32) {
      const uint32_t i = Q.camera_obs[k], c = Q.obs_camera[i];
      if (c != cur) {
        if (cur != 0xffffffffu) b_flush(a, cur, S.U, 21, S.rhs, 6, S.hcf, 6);
        cur = c;
      }
      if (Q.active[c] == 0) continue;
      double pose[12];
      Geo g;
      if (!b_observe(Q, S, i, c, Q.obs_point[i], fscale, pose, g)) continue;
      double jc[2][6];
      b_camera_rows(g, jc);
      for (int j = 0; j < 6; j++) {
        const double w0 = g.w * jc[0][j], w1 = g.w * jc[1][j];
        for (int l = 0; l <= j; l++) a[sym6(j, l)] += w0 * jc[0][l] + w1 * jc[1][l];
        a[21 + j] -= w0 * g.r[0] + w1 * g.r[1];
        a[27 + j] += w0 * g.jf[0] + w1 * g.jf[1];
      }
    }
    if (cur != 0xffffffffu) b_flush(a, cur, S.U, 21, S.rhs, 6, S.hcf, 6);
  }
  // Pass 2: W V^-1 W^T (lower triangle) and W V^-1 b_p, into aux.
  {
    double b[27];
    for (int j = 0; j < 27; j++) b[j] = 0;
    uint32_t cur = 0xffffffffu;
    for (uint32_t k = k0 + lane; k < k1; k += 32) {
      const uint32_t i = Q.camera_obs[k], c = Q.obs_camera[i];
      if (c != cur) {
        if (cur != 0xffffffffu) b_flush(b, cur, S.aux, 27, nullptr, 0, nullptr, 0);
        cur = c;
      }
      if (Q.active[c] == 0) continue;
      const uint32_t pt = Q.obs_point[i];
      double pose[12];
      Geo g;
      if (!b_observe(Q, S, i, c, pt, fscale, pose, g)) continue;
      double jc[2][6];
      b_camera_rows(g, jc);
      double jp[2][3];
      for (int l = 0; l < 3; l++) {
        jp[0][l] = g.w * (g.du[0] * pose[l] + g.du[1] * pose[3 + l] + g.du[2] * pose[6 + l]);
        jp[1][l] = g.w * (g.dv[0] * pose[l] + g.dv[1] * pose[3 + l] + g.dv[2] * pose[6 + l]);
      }
      double Wc[6][3];
      for (int j = 0; j < 6; j++)
        for (int l = 0; l < 3; l++) Wc[j][l] = jc[0][j] * jp[0][l] + jc[1][j] * jp[1][l];
      const double* blk = Q.pblk + 12 * size_t(pt);
      double vb[6];
      for (int k = 0; k < 6; k++) vb[k] = blk[k];
      const double bb[3] = {blk[6], blk[7], blk[8]};
      for (int j = 0; j < 6; j++) {
        const double t0 = Wc[j][0] * vb[0] + Wc[j][1] * vb[1] + Wc[j][2] * vb[2];
        const double t1 = Wc[j][0] * vb[1] + Wc[j][1] * vb[3] + Wc[j][2] * vb[4];
        const double t2 = Wc[j][0] * vb[2] + Wc[j][1] * vb[4] + Wc[j][2] * vb[5];
        for (int l = 0; l <= j; l++) b[sym6(j, l)] += t0 * Wc[l][0] + t1 * Wc[l][1] + t2 * Wc[l][2];
        b[21 + j] += t0 * bb[0] + t1 * bb[1] + t2 * bb[2];
      }
    }
    if (cur != 0xffffffffu) b_flush(b, cur, S.aux, 27, nullptr, 0, nullptr, 0);
  }
  __syncthreads();
  // The damped camera blocks, the reduced right-hand side and the block-Jacobi preconditioner.
  const double lambda = S.st[S_LAMBDA];
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
    double* U = S.U + 21 * c;
    double* Minv = S.Minv + 36 * c;
    double* rhs = S.rhs + 6 * c;
    double* hcf = S.hcf + 6 * c;
    if (Q.active[c] == 0) {
      for (int j = 0; j < 21; j++) U[j] = 0;
      for (int j = 0; j < 36; j++) Minv[j] = 0;
      for (int j = 0; j < 6; j++) {
        U[sym6(j, j)] = 1;
        Minv[j * 7] = 1;
        rhs[j] = 0;
        hcf[j] = 0;
      }
      continue;
    }
    const double* aux = S.aux + 27 * c;
    for (int j = 0; j < 6; j++) U[sym6(j, j)] += lambda * fmax(U[sym6(j, j)], 1e-10);
    double Sb[21];
    for (int j = 0; j < 21; j++) Sb[j] = U[j] - aux[j];
    for (int j = 0; j < 6; j++) rhs[j] -= aux[21 + j];
    double inv[36];
    if (inverse6_spd(Sb, inv)) {
      for (int j = 0; j < 36; j++) Minv[j] = inv[j];
    } else {
      for (int j = 0; j < 36; j++) Minv[j] = 0;
      Minv[0] = -1;
    }
  }
  __syncthreads();
}

// ---- K9-K12: the PCG ------------------------------------------------------------------------------

template <bool SHARED>
__device__ __forceinline__ double b_precondition(const Sh& S, uint32_t i, uint32_t m) {
  if (SHARED && i == m - 1) return S.st[S_FOCAL_INV] * S.r[i];
  const uint32_t c = i / 6, j = i % 6;
  const double* Mi = S.Minv + 36 * c + 6 * j;
  const double* rc = S.r + 6 * c;
  return Mi[0] * rc[0] + Mi[1] * rc[1] + Mi[2] * rc[2] + Mi[3] * rc[3] + Mi[4] * rc[4] + Mi[5] * rc[5];
}

__device__ __forceinline__ void b_world(const Sh& S, uint32_t C, const double* v, double* out) {
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) to_world(S.pose + 12 * c, v + 6 * c, out + 6 * c);
}

template <bool SHARED>
__device__ __noinline__ void b_pcg_init(const BatchProblem& Q, Sh& S) {
  const uint32_t C = Q.C, m = 6 * C + (SHARED ? 1 : 0);
  double* st = S.st;
  if (threadIdx.x == 0) {
    for (int j = S_RHO; j <= 25; j++) st[j] = 0;
    if (SHARED) {
      double diag = S.scal[0];
      diag += st[S_LAMBDA] * fmax(diag, 1e-10);
      st[S_FOCAL_DIAG] = diag;
      const double sff = diag - S.scal[2];
      st[S_FOCAL_INV] = sff > 0 ? 1 / sff : -1;
      st[S_FOCAL_RHS] = -S.scal[1] - S.scal[3];
    }
    S.ok = !(st[S_POINT_FAILED] != 0 || (SHARED && !(st[S_FOCAL_INV] > 0)));
  }
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x)
    if (!(S.Minv[36 * c] > 0)) S.ok = 0;
  __syncthreads();
  if (!S.ok) {
    if (threadIdx.x == 0) st[S_CG_FAILED] = 1;
    __syncthreads();
    return;
  }
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) S.r[i] = (SHARED && i == m - 1) ? st[S_FOCAL_RHS] : S.rhs[i];
  __syncthreads();
  double v[2] = {0, 0};
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const double rr = S.r[i], zz = b_precondition<SHARED>(S, i, m);
    S.x[i] = 0;
    S.p[i] = zz;
    S.z[i] = zz;
    v[0] += rr * zz;
    v[1] += rr * rr;
  }
  __syncthreads();
  b_world(S, C, S.p, S.pw);
  bsum_all(v, S.red);
  if (threadIdx.x == 0) {
    st[S_RHO] = v[0];
    st[S_R0] = st[S_R2] = st[S_INNER_R0] = v[1];
    if (v[1] > 0 && v[0] > 0) st[S_CG_ACTIVE] = 1;
    else if (v[1] > 1e-24) st[S_CG_FAILED] = 1;
  }
  __syncthreads();
}

// The one-pass product over the stored factors FT: -sum_i W_i y_p in world axes into acc (plus the
// focal share), exactly the grid engine's k_product_f restricted to one problem.
template <bool SHARED, typename T>
__device__ __noinline__ void b_product_f(const BatchProblem& Q, Sh& S, const T* FT, const double* vec) {
  const uint32_t m = 6 * Q.C + (SHARED ? 1 : 0);
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) S.acc[j] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const size_t stride = Q.Mpad;
  const double pf = SHARED ? vec[m - 1] : 0.0;  // the focal element of the vector (its cameras: S.pw)
  double ef = 0;
  for (uint32_t t = warp; t < Q.ntasks; t += nw) {
    const uint32_t p0 = Q.tasks[t], p1 = Q.tasks[t + 1];
    const uint32_t o0 = Q.point_start[p0], n = Q.point_start[p1] - o0;
    const uint32_t rounds = n <= uint32_t(kTaskObs) ? 1 : (n + kTaskObs - 1) / kTaskObs;
    double s[3] = {0, 0, 0};
    int seg = -1 - lane;
    uint32_t pt = 0;
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k < n) {
        const uint32_t i = o0 + k;
        const uint32_t c = Q.obs_camera[i];
        pt = Q.obs_point[i];
        seg = int(pt - p0);
        Factors<T> f;
        load_factors(FT, stride, i, f);
        double u[3];
        factor_wt(f, S.pw + 6 * c, pf, Q.active[c] != 0, false, SHARED, u);
        s[0] += u[0];
        s[1] += u[1];
        s[2] += u[2];
      }
    }
    Runs runs{0u, 0, 0};
    if (rounds == 1) {
      runs = lane_runs(seg, lane);
      run_scan(s, runs);
    } else {
      warp_allsum(s);
    }
    const bool valid = uint32_t(lane) < n;
    const bool tail = rounds == 1 ? (valid && run_tail(runs, lane)) : lane == 0;
    double y[3] = {0, 0, 0};
    if (tail) {
      const double* vb = Q.pblk + 12 * size_t(rounds == 1 ? pt : p0);
      y[0] = vb[0] * s[0] + vb[1] * s[1] + vb[2] * s[2];
      y[1] = vb[1] * s[0] + vb[3] * s[1] + vb[4] * s[2];
      y[2] = vb[2] * s[0] + vb[4] * s[1] + vb[5] * s[2];
    }
    const unsigned tails = __ballot_sync(kFull, tail);
    const int src = rounds == 1 ? (valid ? __ffs(tails & (kFull << lane)) - 1 : lane) : 0;
    for (int j = 0; j < 3; j++) y[j] = __shfl_sync(kFull, y[j], src);
    const T y0 = T(y[0]), y1 = T(y[1]), y2 = T(y[2]);
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k >= n) continue;
      const uint32_t i = o0 + k;
      const uint32_t c = Q.obs_camera[i];
      Factors<T> f;
      load_factors(FT, stride, i, f);
      const T gu = f.w * (f.ju[0] * y0 + f.ju[1] * y1 + f.ju[2] * y2);
      const T gv = f.w * (f.jv[0] * y0 + f.jv[1] * y1 + f.jv[2] * y2);
      if (SHARED) ef += double(gu * f.jf[0] + gv * f.jf[1]);
      if (Q.active[c] == 0) continue;
      const T h0 = gu * f.ju[0] + gv * f.jv[0], h1 = gu * f.ju[1] + gv * f.jv[1], h2 = gu * f.ju[2] + gv * f.jv[2];
      double* ac = S.acc + 6 * c;
      atomicAdd(ac + 0, -double(f.q[1] * h2 - f.q[2] * h1));
      atomicAdd(ac + 1, -double(f.q[2] * h0 - f.q[0] * h2));
      atomicAdd(ac + 2, -double(f.q[0] * h1 - f.q[1] * h0));
      atomicAdd(ac + 3, -double(h0));
      atomicAdd(ac + 4, -double(h1));
      atomicAdd(ac + 5, -double(h2));
    }
  }
  if (SHARED) {
    for (int d = 16; d > 0; d >>= 1) ef += __shfl_xor_sync(kFull, ef, d);
    if (lane == 0) atomicAdd(S.acc + (m - 1), -ef);
  }
  __syncthreads();
}

// The FP64 recompute product of the vector v (camera axes): +sum_i W_i y_p per camera into acc,
// the focal share into acc[m-1]; the geometry is recomputed from the accepted scene.
template <bool SHARED>
__device__ __noinline__ void b_product_r(const BatchProblem& Q, Sh& S, const double* vec) {
  const uint32_t m = 6 * Q.C + (SHARED ? 1 : 0);
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) S.acc[j] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double fscale = fscale_of<SHARED>(S.st[S_LOG_FOCAL]);
  const double vf = SHARED ? vec[m - 1] : 0.0;
  double ef = 0;
  for (uint32_t t = warp; t < Q.ntasks; t += nw) {
    const uint32_t p0 = Q.tasks[t], p1 = Q.tasks[t + 1];
    const uint32_t o0 = Q.point_start[p0], n = Q.point_start[p1] - o0;
    const uint32_t rounds = n <= uint32_t(kTaskObs) ? 1 : (n + kTaskObs - 1) / kTaskObs;
    double s[3] = {0, 0, 0};
    int seg = -1 - lane;
    uint32_t pt = 0;
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k < n) {
        const uint32_t i = o0 + k;
        const uint32_t c = Q.obs_camera[i];
        pt = Q.obs_point[i];
        seg = int(pt - p0);
        double pose[12];
        Geo g;
        if (b_observe(Q, S, i, c, pt, fscale, pose, g)) {
          double u[3];
          wt_product(g, pose, vec + 6 * c, vf, Q.active[c] != 0, false, SHARED, u);
          s[0] += u[0];
          s[1] += u[1];
          s[2] += u[2];
        }
      }
    }
    Runs runs{0u, 0, 0};
    if (rounds == 1) {
      runs = lane_runs(seg, lane);
      run_scan(s, runs);
    } else {
      warp_allsum(s);
    }
    const bool valid = uint32_t(lane) < n;
    const bool tail = rounds == 1 ? (valid && run_tail(runs, lane)) : lane == 0;
    double y[3] = {0, 0, 0};
    if (tail) {
      const double* vb = Q.pblk + 12 * size_t(rounds == 1 ? pt : p0);
      y[0] = vb[0] * s[0] + vb[1] * s[1] + vb[2] * s[2];
      y[1] = vb[1] * s[0] + vb[3] * s[1] + vb[4] * s[2];
      y[2] = vb[2] * s[0] + vb[4] * s[1] + vb[5] * s[2];
    }
    const unsigned tails = __ballot_sync(kFull, tail);
    const int src = rounds == 1 ? (valid ? __ffs(tails & (kFull << lane)) - 1 : lane) : 0;
    for (int j = 0; j < 3; j++) y[j] = __shfl_sync(kFull, y[j], src);
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kTaskObs + lane;
      if (k >= n) continue;
      const uint32_t i = o0 + k;
      const uint32_t c = Q.obs_camera[i];
      double pose[12];
      Geo g;
      if (!b_observe(Q, S, i, c, Q.obs_point[i], fscale, pose, g)) continue;
      double d[6], e;
      w_product(g, pose, y, Q.active[c] != 0, false, d, e);
      if (SHARED) ef += e;
      if (Q.active[c] == 0) continue;
      for (int j = 0; j < 6; j++) atomicAdd(S.acc + 6 * c + j, d[j]);
    }
  }
  if (SHARED) {
    for (int d = 16; d > 0; d >>= 1) ef += __shfl_xor_sync(kFull, ef, d);
    if (lane == 0) atomicAdd(S.acc + (m - 1), ef);
  }
  __syncthreads();
}

// S p from the product sums (world: acc holds -sum W y in world axes; else +sum W y in camera
// axes), p . Sp and alpha (the reference's breakdown checks).
template <bool SHARED>
__device__ __noinline__ void b_columns(const BatchProblem& Q, Sh& S, bool world) {
  const uint32_t C = Q.C, n = 6 * C, m = n + (SHARED ? 1 : 0);
  double v[2] = {0, 0};  // p . Sp over camera rows, H_cf . p
  const double pf = SHARED ? S.p[m - 1] : 0.0;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t c = j / 6, r = j % 6;
    const double* a = S.acc + 6 * c;
    double prod;
    if (world) {
      const double* R = S.pose + 12 * c;
      const uint32_t rr = r % 3, h = r < 3 ? 0 : 3;
      prod = R[3 * rr] * a[h] + R[3 * rr + 1] * a[h + 1] + R[3 * rr + 2] * a[h + 2];
    } else {
      prod = -a[r];
    }
    const double* U = S.U + 21 * c;
    const double* pc = S.p + 6 * c;
    double up = 0;
    for (int k = 0; k < 6; k++) up += U[sym6(r, k)] * pc[k];
    double sp = up + prod;
    if (SHARED) {
      sp += S.hcf[j] * pf;
      v[1] += S.hcf[j] * pc[r];
    }
    S.Sp[j] = sp;
    v[0] += pc[r] * sp;
  }
  bsum_all(v, S.red);
  if (threadIdx.x == 0) {
    double* st = S.st;
    double den = v[0];
    if (SHARED) {
      const double focal = world ? S.acc[n] : -S.acc[n];
      const double spf = st[S_FOCAL_DIAG] * pf + v[1] + focal;
      S.Sp[n] = spf;
      den += pf * spf;
    }
    const double alpha = st[S_RHO] / den;
    if (!(den > 0) || !(fabs(alpha) < 1e20)) {
      st[S_CG_ACTIVE] = 0;
      st[S_CG_FAILED] = 1;
    } else {
      st[S_ALPHA] = alpha;
    }
  }
  __syncthreads();
}

template <bool SHARED>
__device__ __noinline__ void b_pcg_update(const BatchProblem& Q, Sh& S, double tol_inner) {
  double* st = S.st;
  if (st[S_CG_ACTIVE] == 0) return;
  const uint32_t C = Q.C, m = 6 * C + (SHARED ? 1 : 0);
  const double alpha = st[S_ALPHA];
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    S.x[i] += alpha * S.p[i];
    S.r[i] -= alpha * S.Sp[i];
  }
  __syncthreads();
  double v[2] = {0, 0};
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const double rr = S.r[i], zz = b_precondition<SHARED>(S, i, m);
    S.z[i] = zz;
    v[0] += rr * rr;
    v[1] += zz * rr;
  }
  bsum_all(v, S.red);
  if (threadIdx.x == 0) {
    const double residual = v[0], rho = v[1];
    st[S_CG_STEPS] += 1;
    st[S_CG_SOLVE_STEPS] += 1;
    st[S_R2] = residual;
    if (residual <= fmax(S.tol * S.tol * st[S_R0], tol_inner * tol_inner * st[S_INNER_R0])) {
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
  __syncthreads();
  if (st[S_CG_ACTIVE] == 0) return;
  const double beta = st[S_BETA];
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) S.p[i] = S.z[i] + beta * S.p[i];
  __syncthreads();
  b_world(S, C, S.p, S.pw);
  __syncthreads();
}

// Mixed form: r = b - S x in FP64 (recompute product), z = M^-1 r, p = z; x is accepted when the
// true residual meets the tolerance, else the PCG restarts from it.
template <bool SHARED>
__device__ __noinline__ void b_refine(const BatchProblem& Q, Sh& S) {
  double* st = S.st;
  if (!(st[S_ACTIVE] != 0 && st[S_CG_FAILED] == 0 && st[S_R0] > 0)) return;
  const uint32_t C = Q.C, n = 6 * C, m = n + (SHARED ? 1 : 0);
  // S x over the FP64 copy of the factors when it is kept (world-axis sums of -W_i y_p), else by
  // the recompute product (camera-axis sums of +W_i y_p).
  const bool one_pass = Q.F64 != nullptr;
  if (one_pass) {
    b_world(S, C, S.x, S.pw);
    b_product_f<SHARED, double>(Q, S, Q.F64, S.x);
  } else {
    b_product_r<SHARED>(Q, S, S.x);
  }
  const double xf = SHARED ? S.x[n] : 0.0;
  double hx = 0;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint32_t c = j / 6, r = j % 6;
    const double* U = S.U + 21 * c;
    const double* xc = S.x + 6 * c;
    double sx = 0;
    for (int k = 0; k < 6; k++) sx += U[sym6(r, k)] * xc[k];
    if (one_pass) {
      const double* R = S.pose + 12 * c;
      const double* a = S.acc + 6 * c;
      const uint32_t rr = r % 3, h = r < 3 ? 0 : 3;
      sx += R[3 * rr] * a[h] + R[3 * rr + 1] * a[h + 1] + R[3 * rr + 2] * a[h + 2];
    } else {
      sx -= S.acc[j];
    }
    if (SHARED) {
      sx += S.hcf[j] * xf;
      hx += S.hcf[j] * xc[r];
    }
    S.r[j] = S.rhs[j] - sx;
  }
  __syncthreads();
  double v[3] = {0, 0, hx};  // r . r, r . z, H_cf . x
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const double rr = S.r[j], zz = b_precondition<SHARED>(S, j, m);
    S.z[j] = zz;
    S.p[j] = zz;
    v[0] += rr * rr;
    v[1] += rr * zz;
  }
  bsum_all(v, S.red);
  b_world(S, C, S.p, S.pw);  // the restarted direction in world axes, for the one-pass product
  if (threadIdx.x == 0) {
    double residual = v[0], rho = v[1];
    if (SHARED) {
      const double sxf = st[S_FOCAL_DIAG] * xf + v[2] + (one_pass ? S.acc[n] : -S.acc[n]);
      const double rf = st[S_FOCAL_RHS] - sxf, zf = st[S_FOCAL_INV] * rf;
      S.r[n] = rf;
      S.z[n] = zf;
      S.p[n] = zf;
      residual += rf * rf;
      rho += rf * zf;
    }
    st[S_R2] = residual;
    if (residual <= S.tol * S.tol * st[S_R0]) {
      st[S_CG_ACTIVE] = 0;
      st[S_CG_CONVERGED] = 1;
    } else if (rho > 0) {
      st[S_RHO] = rho;
      st[S_INNER_R0] = residual;
      st[S_CG_ACTIVE] = 1;
      st[S_REFINED] += 1;
    } else {
      st[S_CG_FAILED] = 1;
    }
  }
  __syncthreads();
}

// ---- K14-K19: candidate, gauge, cost, acceptance, commit ------------------------------------------

template <bool SHARED>
__device__ __noinline__ void b_update_cameras(const BatchProblem& Q, Sh& S) {
  double* st = S.st;
  const uint32_t C = Q.C, m = 6 * C + (SHARED ? 1 : 0);
  __syncthreads();
  if (threadIdx.x == 0) {
    st[S_TRIAL_VALID] = 0;
    S.ok = st[S_ACTIVE] != 0 && st[S_CG_FAILED] == 0;
    S.ok2 = 1;
    if (S.ok) {
      if (SHARED) st[S_LOG_FOCAL_TRIAL] = st[S_LOG_FOCAL] + S.x[m - 1];
      if (st[S_R0] > 0 && st[S_R2] > S.tol * S.tol * st[S_R0]) {
        st[S_CG_FAILED] = 1;
        S.ok2 = 0;
      } else if (SHARED && !(fabs(st[S_LOG_FOCAL_TRIAL]) < 700)) {
        S.ok2 = 0;
      }
    }
  }
  __syncthreads();
  if (!S.ok) return;
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
    const double* pose = S.pose + 12 * c;
    to_world(pose, S.x + 6 * c, S.xw + 6 * c);
    double moved[12];
    if (Q.active[c]) move_pose(pose, S.x + 6 * c, moved);
    else
      for (int j = 0; j < 12; j++) moved[j] = pose[j];
    for (int j = 0; j < 12; j++) S.tpose[12 * c + j] = moved[j];
  }
  __syncthreads();
  if (!S.ok2) return;
  if (SHARED) {
    const double fs = exp(st[S_LOG_FOCAL_TRIAL]);
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
      const double fx = S.cam[6 * c] * fs, fy = S.cam[6 * c + 1] * fs;
      if (!(fx >= 1e-6 && fy >= 1e-6 && fx <= 1e6 && fy <= 1e6)) S.ok2 = 0;
    }
  }
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) {
    const double* p = S.tpose + 12 * c;
    for (int j = 0; j < 12; j++)
      if (!(fabs(p[j]) <= 1e9)) S.ok2 = 0;
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) {
        double d = p[j * 3] * p[k * 3] + p[j * 3 + 1] * p[k * 3 + 1] + p[j * 3 + 2] * p[k * 3 + 2];
        if (j == k) d -= 1;
        if (!(fabs(d) < 1e-6)) S.ok2 = 0;
      }
  }
  __syncthreads();
  const double o[3] = {st[S_ORIGIN], st[S_ORIGIN + 1], st[S_ORIGIN + 2]};
  if (threadIdx.x == 0 && S.ok2) {
    const double* p = S.tpose + 12 * Q.scale_view;
    double cc[3];
    for (int i = 0; i < 3; i++) cc[i] = -p[i] * p[9] - p[i + 3] * p[10] - p[i + 6] * p[11];
    const double baseline = sqrt((o[0] - cc[0]) * (o[0] - cc[0]) + (o[1] - cc[1]) * (o[1] - cc[1]) +
                                 (o[2] - cc[2]) * (o[2] - cc[2]));
    double scale = 1;
    if (!(baseline > 1e-12)) S.ok2 = 0;
    else if (Q.normalize_scale) scale = st[S_BASELINE] / baseline;
    if (!(scale > 1e-9 && scale < 1e9)) S.ok2 = 0;
    if (S.ok2) {
      st[S_SCALE] = scale;
      st[S_TRIAL_VALID] = 1;
    }
  }
  __syncthreads();
  if (!S.ok2 || !Q.normalize_scale) return;
  const double s = st[S_SCALE];
  for (uint32_t h = threadIdx.x; h < C; h += blockDim.x) {
    if (h == Q.anchor) continue;
    double* p = S.tpose + 12 * h;
    double rot[3];
    for (int i = 0; i < 3; i++) rot[i] = (p[i * 3] * o[0] + p[i * 3 + 1] * o[1] + p[i * 3 + 2] * o[2] + p[9 + i]) - p[9 + i];
    for (int i = 0; i < 3; i++) p[9 + i] = s * p[9 + i] + (s - 1) * rot[i];
  }
  __syncthreads();
}

// W_i^T x of one observation for the back-substitution: from the FP64 factors, or recomputed in
// FP64 when the factors are FP32 and no FP64 copy is kept.
template <bool SHARED, typename T>
__device__ __forceinline__ void b_update_wt(const BatchProblem& Q, const Sh& S, uint32_t i, uint32_t c, uint32_t pt,
                                            double fscale, double xf, double t[3]) {
  t[0] = t[1] = t[2] = 0;
  if (sizeof(T) == 8 || Q.F64) {
    Factors<double> f;
    load_factors(sizeof(T) == 8 ? static_cast<const double*>(Q.F) : static_cast<const double*>(Q.F64), Q.Mpad, i, f);
    factor_wt(f, S.xw + 6 * c, xf, Q.active[c] != 0, false, SHARED, t);
    return;
  }
  double pose[12];
  Geo g;
  if (b_observe(Q, S, i, c, pt, fscale, pose, g)) wt_product(g, pose, S.x + 6 * c, xf, Q.active[c] != 0, false, SHARED, t);
}

__device__ __forceinline__ void b_candidate_point(const BatchProblem& Q, const Sh& S, uint32_t pt, const double s[3],
                                                  double X[3]) {
  const double* blk = Q.pblk + 12 * size_t(pt);
  const double r0 = blk[6] - s[0], r1 = blk[7] - s[1], r2 = blk[8] - s[2];
  const double* X0 = Q.points + 3 * size_t(pt);
  X[0] = X0[0] + (blk[0] * r0 + blk[1] * r1 + blk[2] * r2);
  X[1] = X0[1] + (blk[1] * r0 + blk[3] * r1 + blk[4] * r2);
  X[2] = X0[2] + (blk[2] * r0 + blk[4] * r1 + blk[5] * r2);
  if (Q.normalize_scale) {
    const double sc = S.st[S_SCALE];
    for (int j = 0; j < 3; j++) X[j] = S.st[S_ORIGIN + j] + sc * (X[j] - S.st[S_ORIGIN + j]);
  }
  double* out = Q.tpoints + 3 * size_t(pt);
  out[0] = X[0];
  out[1] = X[1];
  out[2] = X[2];
}

__device__ __forceinline__ void b_candidate_obs(const BatchProblem& Q, const Sh& S, uint32_t i, const double X[3],
                                                double fscale_trial, double& cost, double& sq) {
  const uint32_t c = Q.obs_camera[i];
  double pose[12];
  pose_of(S.tpose, c, pose);
  const Camera k = cam_at(S, c, fscale_trial);
  double oc, os;
  candidate_cost(pose, k, X, false, Q.pixels[2 * size_t(i)], Q.pixels[2 * size_t(i) + 1], S.huber, oc, os);
  cost += oc;
  sq += os;
}

template <bool SHARED, typename T>
__device__ __noinline__ void b_update_points(const BatchProblem& Q, Sh& S) {
  double* st = S.st;
  double cs[2] = {0, 0};
  const bool valid = st[S_TRIAL_VALID] != 0;
  if (st[S_ACTIVE] != 0 && st[S_CG_FAILED] == 0 && valid) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double fscale = fscale_of<SHARED>(st[S_LOG_FOCAL]), fscale_trial = fscale_of<SHARED>(st[S_LOG_FOCAL_TRIAL]);
    const double xf = SHARED ? S.x[6 * Q.C] : 0.0;
    for (uint32_t t = warp; t < Q.ntasks; t += nw) {
      const uint32_t p0 = Q.tasks[t], p1 = Q.tasks[t + 1];
      const uint32_t o0 = Q.point_start[p0], n = Q.point_start[p1] - o0;
      if (n <= uint32_t(kTaskObs)) {
        const bool ok = uint32_t(lane) < n;
        const uint32_t i = o0 + lane;
        double s[3] = {0, 0, 0};
        int seg = -1 - lane;
        uint32_t pt = 0;
        if (ok) {
          pt = Q.obs_point[i];
          seg = int(pt - p0);
          b_update_wt<SHARED, T>(Q, S, i, Q.obs_camera[i], pt, fscale, xf, s);
        }
        const Runs runs = lane_runs(seg, lane);
        run_scan(s, runs);
        const bool tail = ok && run_tail(runs, lane);
        double X[3] = {0, 0, 0};
        if (tail) b_candidate_point(Q, S, pt, s, X);
        const unsigned tails = __ballot_sync(kFull, tail);
        const int src = ok ? __ffs(tails & (kFull << lane)) - 1 : lane;
        for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], src);
        if (ok) b_candidate_obs(Q, S, i, X, fscale_trial, cs[0], cs[1]);
      } else {
        double s[3] = {0, 0, 0};
        for (uint32_t base = 0; base < n; base += kTaskObs)
          if (base + lane < n) {
            const uint32_t i = o0 + base + lane;
            double u[3];
            b_update_wt<SHARED, T>(Q, S, i, Q.obs_camera[i], p0, fscale, xf, u);
            s[0] += u[0];
            s[1] += u[1];
            s[2] += u[2];
          }
        warp_allsum(s);
        double X[3] = {0, 0, 0};
        if (lane == 0) b_candidate_point(Q, S, p0, s, X);
        for (int j = 0; j < 3; j++) X[j] = __shfl_sync(kFull, X[j], 0);
        for (uint32_t base = 0; base < n; base += kTaskObs)
          if (base + lane < n) b_candidate_obs(Q, S, o0 + base + lane, X, fscale_trial, cs[0], cs[1]);
      }
    }
  }
  bsum_all(cs, S.red);
  // acceptBundleCandidate (K18).
  if (threadIdx.x == 0) {
    st[S_COMMIT] = 0;
    if (st[S_ACTIVE] != 0) {
      const double cost = cs[0], squares = cs[1];
      if (valid && cost < st[S_COST]) {
        const double change = st[S_COST] - cost;
        st[S_COST] = cost;
        st[S_SSE] = squares;
        st[S_ACCEPTED] += 1;
        st[S_COMMIT] = 1;
        st[S_LAMBDA] = fmax(1e-10, st[S_LAMBDA] / 3);
        if (change < fmax(S.stall, 1e-9) * fmax(1.0, cost)) st[S_ACTIVE] = 0;
      } else {
        st[S_REJECTED] += 1;
        st[S_LAMBDA] *= 10;
        if (st[S_CG_FAILED] != 0) st[S_FAILED_SOLVES] += 1;
        if (st[S_LAMBDA] > 1e12) st[S_ACTIVE] = 0;
      }
    }
    st[S_POINT_FAILED] = 0;
  }
  __syncthreads();
  // commitBundleCandidate (K19).
  if (st[S_COMMIT] != 0) {
    for (uint32_t j = threadIdx.x; j < 12 * Q.C; j += blockDim.x) S.pose[j] = S.tpose[j];
    for (uint32_t j = threadIdx.x; j < 3 * Q.P; j += blockDim.x) Q.points[j] = Q.tpoints[j];
    if (SHARED && threadIdx.x == 0) st[S_LOG_FOCAL] = st[S_LOG_FOCAL_TRIAL];
  }
  __syncthreads();
}

// ---- K20 -------------------------------------------------------------------------------------------

__device__ __noinline__ void b_pack(const BatchProblem& Q, Sh& S, bool shared) {
  const uint32_t np = 12 * Q.C, total = np + 3 * Q.P;
  for (uint32_t j = threadIdx.x; j < np; j += blockDim.x) Q.output[j] = S.pose[j];
  for (uint32_t w = threadIdx.x; w < 26; w += blockDim.x) {
    double v = S.st[w];
    if (w == 24) v = sqrt(S.st[S_SSE0] / double(float(Q.M)));
    if (w == 25) v = sqrt(S.st[S_SSE] / double(float(Q.M)));
    Q.output[total + w] = v;
  }
  if (shared && threadIdx.x == 0) Q.output[total + 26] = S.st[S_LOG_FOCAL];
  __syncthreads();
}

// ---- the persistent kernel ---------------------------------------------------------------------

template <bool SHARED, bool MIXED>
__device__ __forceinline__ void b_solve(const BatchProblem& Q, Sh& S) {
  using T = typename std::conditional<MIXED, float, double>::type;
  b_init(Q, S);
  b_cost(Q, S, SHARED);
  for (uint32_t it = 0; it < S.iterations && S.st[S_ACTIVE] != 0; it++) {
    b_point_pass<SHARED, T>(Q, S);
    b_camera_pass<SHARED>(Q, S);
    b_pcg_init<SHARED>(Q, S);
    for (uint32_t k = 0; k < S.max_cg && S.st[S_CG_ACTIVE] != 0; k++) {
      b_product_f<SHARED, T>(Q, S, static_cast<const T*>(Q.F), S.p);
      b_columns<SHARED>(Q, S, true);
      b_pcg_update<SHARED>(Q, S, S.tol_inner);
    }
    if (MIXED) {
      // The true FP64 residual, then (when it is above the tolerance) the restarted PCG on the
      // one-pass product over the FP64 copy of the factors.
      b_refine<SHARED>(Q, S);
      for (uint32_t k = 0; k < S.max_cg && S.st[S_CG_ACTIVE] != 0; k++) {
        b_product_f<SHARED, double>(Q, S, Q.F64, S.p);
        b_columns<SHARED>(Q, S, true);
        b_pcg_update<SHARED>(Q, S, 0.0);
      }
    }
    b_update_cameras<SHARED>(Q, S);
    b_update_points<SHARED, T>(Q, S);
  }
  b_pack(Q, S, SHARED);
}

template <int NT, int MINB, bool SHARED, bool MIXED>
__global__ void __launch_bounds__(NT, MINB) k_batch(BatchArgs A) {
  extern __shared__ __align__(16) double smem[];
  __shared__ Sh S;
  __shared__ BatchProblem Q;
  if (threadIdx.x == 0) {
    layout_words(A.Cmax, smem, &S);
    S.huber = A.huber;
    S.tol = A.tol;
    S.tol_inner = A.tol_inner;
    S.stall = A.stall;
    S.iterations = A.iterations;
    S.max_cg = A.max_cg;
  }
  for (;;) {
    if (threadIdx.x == 0) S.job = atomicAdd(A.queue, 1u);
    __syncthreads();
    const uint32_t job = S.job;
    if (job >= A.count) break;
    if (threadIdx.x == 0) Q = A.problems[A.order[job]];
    __syncthreads();
    b_solve<SHARED, MIXED>(Q, S);
    __syncthreads();
  }
}

template <int NT, int MINB>
struct Variants {
  static const void* get(bool shared, bool mixed) {
    if (shared) return mixed ? reinterpret_cast<const void*>(k_batch<NT, MINB, true, true>)
                             : reinterpret_cast<const void*>(k_batch<NT, MINB, true, false>);
    return mixed ? reinterpret_cast<const void*>(k_batch<NT, MINB, false, true>)
                 : reinterpret_cast<const void*>(k_batch<NT, MINB, false, false>);
  }
};

constexpr BatchShape kShapes[kBatchShapes] = {{256, 2}, {256, 3}, {384, 2}, {512, 1}};

const void* batch_kernel(int k, bool shared, bool mixed) {
  switch (k) {
    case 0: return Variants<256, 2>::get(shared, mixed);
    case 1: return Variants<256, 3>::get(shared, mixed);
    case 2: return Variants<384, 2>::get(shared, mixed);
    default: return Variants<512, 1>::get(shared, mixed);
  }
}

}  // namespace

BatchShape batch_shape(int k) { return kShapes[k < 0 ? 0 : (k >= kBatchShapes ? kBatchShapes - 1 : k)]; }

size_t batch_smem_bytes(uint32_t Cmax) { return size_t(layout_words(Cmax, nullptr, nullptr)) * sizeof(double); }

uint32_t batch_max_cameras() {
  uint32_t c = 1;
  while (batch_smem_bytes(c + 1) <= 200 * 1024) c++;
  return c;
}

cudaError_t batch_configure() {
  const int bytes = 227 * 1024 - int(sizeof(Sh) + sizeof(BatchProblem)) - 1024;
  for (int k = 0; k < kBatchShapes; k++)
    for (int s = 0; s < 2; s++)
      for (int x = 0; x < 2; x++) {
        const cudaError_t e = cudaFuncSetAttribute(batch_kernel(k, s != 0, x != 0),
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

int batch_blocks_per_sm(int k, bool shared, bool mixed, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel(k, shared, mixed), batch_shape(k).threads,
                                                    smem) != cudaSuccess)
    return 0;
  return n;
}

cudaError_t launch_batch(int k, bool shared, bool mixed, const BatchArgs& a, int blocks, size_t smem, cudaStream_t s) {
  void* args[] = {const_cast<BatchArgs*>(&a)};
  return cudaLaunchKernel(batch_kernel(k, shared, mixed), dim3(blocks), dim3(batch_shape(k).threads), args, smem, s);
}

}  // namespace tba
