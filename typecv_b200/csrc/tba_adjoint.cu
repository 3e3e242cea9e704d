// Kernels of the adjoint (tba_adjoint.cuh), sm_100a, FP64.
//
//   k_adj_obs        per observation: residual, robust weight, the exact 9x9 Hessian block of the
//                    robust cost in the local coordinates (omega, v, dX) and the gradient share
//   k_adj_points     per point: V_p = sum of its blocks, V_p^-1, the point right-hand side
//   k_adj_cameras    per camera: U_c, the Schur diagonal U_c - sum W V^-1 W^T, the block-Jacobi
//                    preconditioner and the reduced right-hand side (plus the gauge term)
//   k_adj_prod_*     the Schur product S p = U p - sum_i W_i V^-1 sum_j W_j^T p, two passes over
//                    the stored cross blocks
//   k_adj_vec        one PCG step on the camera vectors (one block)
//   k_adj_back       point back-substitution
//   k_adj_vjp        per observation: ybar_i = W~_i J_i lambda_i, and the intrinsics' shares
//   k_adj_newton_*   the candidate theta (+) delta with the solver's own pose update and gauge
//                    normalisation, k_adj_cost its robust cost, k_adj_commit its acceptance
//
// Per observation i (camera c, point p): q = R X + t, pixel pi(q) (pinhole + two-term radial),
// residual r = pi - y, Huber rho(|r|) with threshold h.  The robust cost's gradient in local
// coordinates is w J^T r (w = 1 or h/|r|) and its Hessian is
//   J^T W~ J + w sum_k r_k (Q^T (d2 pi_k / dq2) Q + (d pi_k / dq) . d2q),
// W~ = I for an inlier and w (I - r^ r^T) beyond the threshold; Q = dq/d(omega, v, dX) =
// [-[q]x, I, R]; d2q/(d omega_a d omega_b) = (e_b q_a + e_a q_b)/2 - q delta_ab and
// d2q/(d omega_a dX_m) = e_a x R e_m are the second-order terms of q = exp(omega)(R X + t) + v.
#include <cuda_runtime.h>

#include <algorithm>

#include "tba_adjoint.cuh"
#include "tba_engine.cuh"
#include "tba_math.cuh"
#include "tba_warp.cuh"

namespace tba {
namespace {

constexpr unsigned kAll = 0xffffffffu;

struct ObsSecond {
  double J[2][9];   // d r / d (omega, v, dX); camera columns zero for a fixed camera
  double Wt[3];     // W~ (00, 01, 11)
  double r[2];
  double w;
  double jf[2];     // d r / d log focal scale
  double jk[2];     // d r / d k1
  double Jk[2][9];  // d J / d k1
};

// The observation's second-order quantities; H receives the exact 9x9 Hessian (full).  False
// outside the projection's domain (the same domain as geometry()).
__device__ bool obs_second(const double pose[12], const Camera& k, double limit, const double X[3], double u,
                           double v, double huber, bool variable, ObsSecond& o, double H[9][9]) {
  double q[3];
  for (int i = 0; i < 3; i++) q[i] = pose[3 * i] * X[0] + pose[3 * i + 1] * X[1] + pose[3 * i + 2] * X[2] + pose[9 + i];
  if (!(q[2] > 1e-12)) return false;
  const double iz = 1.0 / q[2], x = q[0] * iz, y = q[1] * iz, r2 = x * x + y * y;
  if (!(r2 < limit && r2 < 1e8)) return false;
  const double d = 1 + k.k1 * r2 + k.k2 * r2 * r2, d1 = k.k1 + 2 * k.k2 * r2, d2 = 2 * k.k2;
  if (!(d > 0 && 1 + 3 * k.k1 * r2 + 5 * k.k2 * r2 * r2 > 0)) return false;
  const double px = k.fx * x * d, py = k.fy * y * d;
  // first and second derivatives of the pixel with respect to (x, y)
  const double Pux = k.fx * (d + 2 * x * x * d1), Puy = 2 * k.fx * x * y * d1;
  const double Pvx = 2 * k.fy * x * y * d1, Pvy = k.fy * (d + 2 * y * y * d1);
  const double Uxx = k.fx * (6 * x * d1 + 4 * x * x * x * d2), Uxy = k.fx * (2 * y * d1 + 4 * x * x * y * d2),
               Uyy = 2 * k.fx * x * (d1 + 2 * y * y * d2);
  const double Vxx = 2 * k.fy * y * (d1 + 2 * x * x * d2), Vxy = k.fy * (2 * x * d1 + 4 * x * y * y * d2),
               Vyy = k.fy * (6 * y * d1 + 4 * y * y * y * d2);
  const double Dx[3] = {iz, 0, -x * iz}, Dy[3] = {0, iz, -y * iz};
  double G[2][3];
  for (int j = 0; j < 3; j++) {
    G[0][j] = Pux * Dx[j] + Puy * Dy[j];
    G[1][j] = Pvx * Dx[j] + Pvy * Dy[j];
  }
  const double mp = fmax(fabs(px + k.cx), fabs(py + k.cy));
  const double mu = fmax(fmax(fabs(G[0][0]), fabs(G[0][1])), fabs(G[0][2]));
  const double mv = fmax(fmax(fabs(G[1][0]), fabs(G[1][1])), fabs(G[1][2]));
  if (!(mp < 1e12 && mu < 1e12 && mv < 1e12)) return false;
  // d2 pi_k / dq2
  const double iz2 = iz * iz;
  double Hq[2][3][3];
  {
    const double Pa[2] = {Pux, Pvx}, Pb[2] = {Puy, Pvy};
    const double Aaa[2] = {Uxx, Vxx}, Aab[2] = {Uxy, Vxy}, Abb[2] = {Uyy, Vyy};
    for (int kk = 0; kk < 2; kk++) {
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          Hq[kk][i][j] = Aaa[kk] * Dx[i] * Dx[j] + Aab[kk] * (Dx[i] * Dy[j] + Dy[i] * Dx[j]) + Abb[kk] * Dy[i] * Dy[j];
      Hq[kk][0][2] -= Pa[kk] * iz2;
      Hq[kk][2][0] -= Pa[kk] * iz2;
      Hq[kk][2][2] += 2 * x * iz2 * Pa[kk];
      Hq[kk][1][2] -= Pb[kk] * iz2;
      Hq[kk][2][1] -= Pb[kk] * iz2;
      Hq[kk][2][2] += 2 * y * iz2 * Pb[kk];
    }
  }
  // Q = dq / d(omega, v, dX)
  double Q[3][9];
  for (int i = 0; i < 3; i++)
    for (int c = 0; c < 9; c++) Q[i][c] = 0;
  if (variable) {
    Q[0][1] = q[2];
    Q[0][2] = -q[1];
    Q[1][0] = -q[2];
    Q[1][2] = q[0];
    Q[2][0] = q[1];
    Q[2][1] = -q[0];
    Q[0][3] = Q[1][4] = Q[2][5] = 1;
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) Q[i][6 + j] = pose[3 * i + j];
  for (int kk = 0; kk < 2; kk++)
    for (int c = 0; c < 9; c++) o.J[kk][c] = G[kk][0] * Q[0][c] + G[kk][1] * Q[1][c] + G[kk][2] * Q[2][c];
  // residual and robust weights
  o.r[0] = (px + k.cx) - u;
  o.r[1] = (py + k.cy) - v;
  const double sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
  if (sq > huber * huber) {
    const double e = sqrt(sq);
    o.w = huber / e;
    const double a = o.r[0] / e, b = o.r[1] / e;
    o.Wt[0] = o.w * (1 - a * a);
    o.Wt[1] = -o.w * a * b;
    o.Wt[2] = o.w * (1 - b * b);
  } else {
    o.w = 1;
    o.Wt[0] = 1;
    o.Wt[1] = 0;
    o.Wt[2] = 1;
  }
  o.jf[0] = px;
  o.jf[1] = py;
  o.jk[0] = k.fx * x * r2;
  o.jk[1] = k.fy * y * r2;
  {
    double gk[2][3];
    for (int j = 0; j < 3; j++) {
      gk[0][j] = k.fx * ((3 * x * x + y * y) * Dx[j] + 2 * x * y * Dy[j]);
      gk[1][j] = k.fy * (2 * x * y * Dx[j] + (x * x + 3 * y * y) * Dy[j]);
    }
    for (int kk = 0; kk < 2; kk++)
      for (int c = 0; c < 9; c++) o.Jk[kk][c] = gk[kk][0] * Q[0][c] + gk[kk][1] * Q[1][c] + gk[kk][2] * Q[2][c];
  }
  // Hessian: J^T W~ J + w sum_k r_k (Q^T Hq_k Q + dpi_k/dq . d2q)
  for (int a = 0; a < 9; a++) {
    const double ta = o.Wt[0] * o.J[0][a] + o.Wt[1] * o.J[1][a];
    const double tb = o.Wt[1] * o.J[0][a] + o.Wt[2] * o.J[1][a];
    for (int b = 0; b < 9; b++) H[a][b] = ta * o.J[0][b] + tb * o.J[1][b];
  }
  for (int kk = 0; kk < 2; kk++) {
    const double coef = o.w * o.r[kk];
    double T[3][9];
    for (int i = 0; i < 3; i++)
      for (int c = 0; c < 9; c++) T[i][c] = Hq[kk][i][0] * Q[0][c] + Hq[kk][i][1] * Q[1][c] + Hq[kk][i][2] * Q[2][c];
    for (int a = 0; a < 9; a++)
      for (int b = 0; b < 9; b++) H[a][b] += coef * (Q[0][a] * T[0][b] + Q[1][a] * T[1][b] + Q[2][a] * T[2][b]);
    if (variable) {
      const double* g = G[kk];
      const double gq = g[0] * q[0] + g[1] * q[1] + g[2] * q[2];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) H[a][b] += coef * (0.5 * (g[b] * q[a] + g[a] * q[b]) - (a == b ? gq : 0.0));
      for (int m = 0; m < 3; m++) {
        const double cm[3] = {pose[m], pose[3 + m], pose[6 + m]};
        const double cross[3] = {cm[1] * g[2] - cm[2] * g[1], cm[2] * g[0] - cm[0] * g[2], cm[0] * g[1] - cm[1] * g[0]};
        for (int a = 0; a < 3; a++) {
          H[a][6 + m] += coef * cross[a];
          H[6 + m][a] += coef * cross[a];
        }
      }
    }
  }
  return true;
}

__device__ inline Camera adj_camera(const AdjParams& A, uint32_t c) {
  const double* k = A.cams + 6 * size_t(c);
  return Camera{k[0], k[1], k[2], k[3], k[4], k[5]};
}

__device__ inline void adj_pose(const AdjParams& A, uint32_t c, double pose[12]) {
  for (int j = 0; j < 12; j++) pose[j] = A.poses[12 * size_t(c) + j];
}

template <int N>
__device__ inline void adj_block_sum(double (&v)[N], double* smem) {
  for (int n = 0; n < N; n++)
    for (int d = 16; d > 0; d >>= 1) v[n] += __shfl_xor_sync(kAll, v[n], d);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0)
    for (int n = 0; n < N; n++) smem[warp * N + n] = v[n];
  __syncthreads();
  for (int n = 0; n < N; n++) {
    double s = 0;
    for (int w = 0; w < nw; w++) s += smem[w * N + n];
    v[n] = s;
  }
  __syncthreads();
}

// ---- assembly ----------------------------------------------------------------------------------

__global__ void __launch_bounds__(128) k_adj_obs(AdjParams A) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.M; i += gridDim.x * blockDim.x) {
    const uint32_t c = A.obs_camera[i], pt = A.obs_point[i];
    double pose[12];
    adj_pose(A, c, pose);
    const Camera k = adj_camera(A, c);
    const double* X = A.points + 3 * size_t(pt);
    ObsSecond o;
    double H[9][9];
    double* hcp = A.Hcp + 18 * size_t(i);
    double* hcc = A.Hcc + 21 * size_t(i);
    double* hpp = A.Hpp + 6 * size_t(i);
    double* gc = A.gc + 6 * size_t(i);
    double* gp = A.gp + 3 * size_t(i);
    if (!obs_second(pose, k, radial_limit(k.k1, k.k2), X, A.pixels[2 * size_t(i)], A.pixels[2 * size_t(i) + 1],
                    A.huber, A.active[c] != 0, o, H)) {
      for (int j = 0; j < 18; j++) hcp[j] = 0;
      for (int j = 0; j < 21; j++) hcc[j] = 0;
      for (int j = 0; j < 6; j++) hpp[j] = gc[j] = 0;
      for (int j = 0; j < 3; j++) gp[j] = 0;
      atomicAdd(A.state + A_INVALID, 1.0);
      continue;
    }
    if (A.mu > 0)  // damping: + mu w J^T J, the observation's Gauss-Newton block with the IRLS weight
      for (int a = 0; a < 9; a++)
        for (int b = 0; b < 9; b++) H[a][b] += A.mu * o.w * (o.J[0][a] * o.J[0][b] + o.J[1][a] * o.J[1][b]);
    for (int a = 0; a < 6; a++)
      for (int m = 0; m < 3; m++) hcp[3 * a + m] = H[a][6 + m];
    for (int a = 0; a < 6; a++)
      for (int b = 0; b <= a; b++) hcc[sym6(a, b)] = H[a][b];
    hpp[0] = H[6][6];
    hpp[1] = H[6][7];
    hpp[2] = H[6][8];
    hpp[3] = H[7][7];
    hpp[4] = H[7][8];
    hpp[5] = H[8][8];
    for (int a = 0; a < 9; a++) {
      const double g = o.w * (o.J[0][a] * o.r[0] + o.J[1][a] * o.r[1]);
      if (a < 6) gc[a] = g;
      else gp[a - 6] = g;
    }
  }
}

__global__ void __launch_bounds__(256) k_adj_points(AdjParams A) {
  __shared__ double red[32];
  double gsq[1] = {0};
  for (uint32_t pt = blockIdx.x * blockDim.x + threadIdx.x; pt < A.P; pt += gridDim.x * blockDim.x) {
    double V[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0};
    for (uint32_t i = A.point_start[pt]; i < A.point_start[pt + 1]; i++) {
      for (int j = 0; j < 6; j++) V[j] += A.Hpp[6 * size_t(i) + j];
      for (int j = 0; j < 3; j++) g[j] += A.gp[3 * size_t(i) + j];
    }
    gsq[0] += g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    double M9[9] = {V[0], V[1], V[2], V[1], V[3], V[4], V[2], V[4], V[5]};
    double inv[6];
    double* vi = A.Vinv + 6 * size_t(pt);
    bool ok = inverse3_spd(M9, inv);
    if (!ok) {
      // Not positive definite (a point whose track is mostly beyond the Huber threshold has a nearly
      // flat cost along some direction): shift by the smallest power-of-ten multiple of the mean
      // diagonal that makes it definite, and count it.
      atomicAdd(A.state + A_POINT_FAILED, 1.0);
      const double scale = fmax(fabs(V[0] + V[3] + V[5]) / 3, 1e-12);
      for (double tau = 1e-8; tau <= 1e2 && !ok; tau *= 10) {
        M9[0] = V[0] + tau * scale;
        M9[4] = V[3] + tau * scale;
        M9[8] = V[5] + tau * scale;
        ok = inverse3_spd(M9, inv);
      }
    }
    if (!ok) {
      A.state[A_POINT_SINGULAR] = 1;
      for (int j = 0; j < 6; j++) vi[j] = 0;
    } else {
      for (int j = 0; j < 6; j++) vi[j] = inv[j];
    }
    for (int j = 0; j < 3; j++) A.bp[3 * size_t(pt) + j] = A.rhs_mode ? A.cot[6 * size_t(A.C) + 3 * size_t(pt) + j] : -g[j];
  }
  adj_block_sum(gsq, red);
  if (threadIdx.x == 0) atomicAdd(A.state + A_GNORM, gsq[0]);
}

// The unit gradient of the anchor-to-scale-camera baseline with respect to the scale camera's
// translation step (its only non-zero part): -R_s (centre_s - o) / |centre_s - o|.
__device__ inline void baseline_gradient(const AdjParams& A, double n[3], double& b) {
  const double* p = A.poses + 12 * size_t(A.scale_view);
  const double* st = A.state;
  double cc[3];
  for (int i = 0; i < 3; i++) cc[i] = -p[i] * p[9] - p[i + 3] * p[10] - p[i + 6] * p[11];
  const double e[3] = {cc[0] - st[A_ORIGIN], cc[1] - st[A_ORIGIN + 1], cc[2] - st[A_ORIGIN + 2]};
  b = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  for (int i = 0; i < 3; i++) n[i] = -(p[3 * i] * e[0] + p[3 * i + 1] * e[1] + p[3 * i + 2] * e[2]) / b;
}

__global__ void __launch_bounds__(128) k_adj_cameras(AdjParams A) {
  __shared__ double red[54 * 4];
  const uint32_t c = blockIdx.x;
  double* U = A.U + 21 * size_t(c);
  double* Minv = A.Minv + 36 * size_t(c);
  double* bc = A.bc + 6 * size_t(c);
  if (A.active[c] == 0) {
    if (threadIdx.x == 0) {
      for (int j = 0; j < 21; j++) U[j] = 0;
      for (int j = 0; j < 36; j++) Minv[j] = 0;
      for (int j = 0; j < 6; j++) {
        U[sym6(j, j)] = 1;
        Minv[7 * j] = 1;
        bc[j] = 0;
      }
    }
    return;
  }
  double s[54];  // Hcc 21 | gc 6 | W V^-1 W^T 21 | W V^-1 b_p 6
  for (int j = 0; j < 54; j++) s[j] = 0;
  for (uint32_t k = A.camera_start[c] + threadIdx.x; k < A.camera_start[c + 1]; k += blockDim.x) {
    const uint32_t i = A.camera_obs[k], pt = A.obs_point[i];
    for (int j = 0; j < 21; j++) s[j] += A.Hcc[21 * size_t(i) + j];
    for (int j = 0; j < 6; j++) s[21 + j] += A.gc[6 * size_t(i) + j];
    const double* W = A.Hcp + 18 * size_t(i);
    const double* vi = A.Vinv + 6 * size_t(pt);
    const double* b = A.bp + 3 * size_t(pt);
    for (int a = 0; a < 6; a++) {
      const double t0 = W[3 * a] * vi[0] + W[3 * a + 1] * vi[1] + W[3 * a + 2] * vi[2];
      const double t1 = W[3 * a] * vi[1] + W[3 * a + 1] * vi[3] + W[3 * a + 2] * vi[4];
      const double t2 = W[3 * a] * vi[2] + W[3 * a + 1] * vi[4] + W[3 * a + 2] * vi[5];
      for (int bb = 0; bb <= a; bb++) s[27 + sym6(a, bb)] += t0 * W[3 * bb] + t1 * W[3 * bb + 1] + t2 * W[3 * bb + 2];
      s[48 + a] += t0 * b[0] + t1 * b[1] + t2 * b[2];
    }
  }
  adj_block_sum(s, red);
  if (threadIdx.x != 0) return;
  for (int j = 0; j < 21; j++) U[j] = s[j];
  if (A.normalize_scale && c == A.scale_view) {
    double n[3], b;
    baseline_gradient(A, n, b);
    const double mu = fmax(1e-12, (s[sym6(3, 3)] + s[sym6(4, 4)] + s[sym6(5, 5)]) / 3);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j <= i; j++) U[sym6(3 + i, 3 + j)] += mu * n[i] * n[j];
  }
  double S[21];
  for (int j = 0; j < 21; j++) S[j] = U[j] - s[27 + j];
  double inv[36];
  if (inverse6_spd(S, inv)) {
    for (int j = 0; j < 36; j++) Minv[j] = inv[j];
  } else {
    for (int j = 0; j < 36; j++) Minv[j] = 0;
    Minv[0] = -1;
    A.state[A_CAMERA_FAILED] = 1;
  }
  double gsq = 0;
  for (int j = 0; j < 6; j++) {
    const double rhs = A.rhs_mode ? A.cot[6 * size_t(c) + j] : -s[21 + j];
    bc[j] = rhs - s[48 + j];
    gsq += s[21 + j] * s[21 + j];
  }
  atomicAdd(A.state + A_GNORM, gsq);
}

// ---- PCG on the camera system ------------------------------------------------------------------

__device__ inline double adj_precondition(const AdjParams& A, uint32_t row) {
  const uint32_t c = row / 6, j = row % 6;
  const double* Mi = A.Minv + 36 * size_t(c) + 6 * j;
  const double* rc = A.r + 6 * size_t(c);
  return Mi[0] * rc[0] + Mi[1] * rc[1] + Mi[2] * rc[2] + Mi[3] * rc[3] + Mi[4] * rc[4] + Mi[5] * rc[5];
}

__global__ void __launch_bounds__(1024) k_adj_pcg_init(AdjParams A) {
  __shared__ double red[64];
  double* st = A.state;
  const uint32_t m = 6 * A.C;
  const bool fail = st[A_POINT_SINGULAR] != 0 || st[A_CAMERA_FAILED] != 0;
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
    A.r[j] = A.bc[j];
    A.x[j] = 0;
  }
  __syncthreads();
  double v[2] = {0, 0};
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
    const double zz = adj_precondition(A, j);
    A.z[j] = zz;
    A.p[j] = zz;
    v[0] += A.r[j] * zz;
    v[1] += A.r[j] * A.r[j];
  }
  adj_block_sum(v, red);
  if (threadIdx.x == 0) {
    st[A_RHO] = v[0];
    st[A_R0] = st[A_R2] = v[1];
    st[A_STEPS] = 0;
    st[A_FAILED] = fail ? 1 : 0;
    st[A_ACTIVE] = (!fail && v[1] > 0 && v[0] > 0) ? 1 : 0;
    if (!fail && v[1] > 0 && !(v[0] > 0)) st[A_FAILED] = 1;
  }
}

__global__ void __launch_bounds__(256) k_adj_prod_points(AdjParams A) {
  if (A.state[A_ACTIVE] == 0) return;
  for (uint32_t pt = blockIdx.x * blockDim.x + threadIdx.x; pt < A.P; pt += gridDim.x * blockDim.x) {
    double t[3] = {0, 0, 0};
    for (uint32_t i = A.point_start[pt]; i < A.point_start[pt + 1]; i++) {
      const uint32_t c = A.obs_camera[i];
      if (A.active[c] == 0) continue;
      const double* W = A.Hcp + 18 * size_t(i);
      const double* pc = A.p + 6 * size_t(c);
      for (int a = 0; a < 6; a++) {
        t[0] += W[3 * a] * pc[a];
        t[1] += W[3 * a + 1] * pc[a];
        t[2] += W[3 * a + 2] * pc[a];
      }
    }
    const double* vi = A.Vinv + 6 * size_t(pt);
    double* y = A.yp + 3 * size_t(pt);
    y[0] = vi[0] * t[0] + vi[1] * t[1] + vi[2] * t[2];
    y[1] = vi[1] * t[0] + vi[3] * t[1] + vi[4] * t[2];
    y[2] = vi[2] * t[0] + vi[4] * t[1] + vi[5] * t[2];
  }
}

__global__ void __launch_bounds__(128) k_adj_prod_cameras(AdjParams A) {
  __shared__ double red[6 * 4];
  if (A.state[A_ACTIVE] == 0) return;
  const uint32_t c = blockIdx.x;
  double s[6] = {0, 0, 0, 0, 0, 0};
  if (A.active[c] != 0)
    for (uint32_t k = A.camera_start[c] + threadIdx.x; k < A.camera_start[c + 1]; k += blockDim.x) {
      const uint32_t i = A.camera_obs[k], pt = A.obs_point[i];
      const double* W = A.Hcp + 18 * size_t(i);
      const double* y = A.yp + 3 * size_t(pt);
      for (int a = 0; a < 6; a++) s[a] += W[3 * a] * y[0] + W[3 * a + 1] * y[1] + W[3 * a + 2] * y[2];
    }
  adj_block_sum(s, red);
  if (threadIdx.x != 0) return;
  const double* U = A.U + 21 * size_t(c);
  const double* pc = A.p + 6 * size_t(c);
  for (int a = 0; a < 6; a++) {
    double up = 0;
    for (int b = 0; b < 6; b++) up += U[sym6(a, b)] * pc[b];
    A.Sp[6 * size_t(c) + a] = up - s[a];
  }
}

// The Schur product in one pass over the cross blocks W_i (18 words, read once instead of twice):
// each warp task forms y_p = V_p^-1 sum_i W_i^T p_c for its points (one observation per lane, a
// segmented scan per point) and scatters -W_i y_p into the block's camera sums in shared memory;
// k_adj_columns adds the blocks' partial rows in a fixed order and U_c p_c.
constexpr int kAdjProductThreads = 352;  // 11 warps: two blocks fill 22 of the 25 warps 80 registers allow
constexpr int kAdjTaskObs = 32;

__device__ inline void adj_wt(const double* W, const double* pc, double u[3]) {
  u[0] = u[1] = u[2] = 0;
  for (int a = 0; a < 6; a++) {
    u[0] += W[3 * a] * pc[a];
    u[1] += W[3 * a + 1] * pc[a];
    u[2] += W[3 * a + 2] * pc[a];
  }
}

__device__ inline void adj_scatter(double* acc, uint32_t C, uint32_t c, const double* W, const double y[3]) {
  for (int a = 0; a < 6; a++)
    atomicAdd(acc + size_t(a) * C + c, -(W[3 * a] * y[0] + W[3 * a + 1] * y[1] + W[3 * a + 2] * y[2]));
}

// With few cameras every warp keeps its own copy of the camera sums (A.prod_copies = warps), so that
// the warps' atomic adds do not contend for the same few addresses; with more cameras fewer copies
// fit and warps share them (warp w adds to copy w % copies).  The copies are summed at the end.
__global__ void __launch_bounds__(kAdjProductThreads) k_adj_product(AdjParams A) {
  extern __shared__ double adj_smem[];  // prod_copies copies of 6C values, component-major
  if (A.state[A_ACTIVE] == 0) return;
  const uint32_t C = A.C;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t copies = A.prod_copies;
  for (uint32_t j = threadIdx.x; j < copies * 6 * C; j += blockDim.x) adj_smem[j] = 0;
  __syncthreads();
  double* adj_acc = adj_smem + size_t(uint32_t(warp) % copies) * 6 * C;
  const uint32_t tb = uint32_t(uint64_t(A.ntasks) * blockIdx.x / gridDim.x);
  const uint32_t te = uint32_t(uint64_t(A.ntasks) * (blockIdx.x + 1) / gridDim.x);
  for (uint32_t t = tb + warp; t < te; t += nwarps) {
    const uint32_t o0 = A.task_obs[t], n = A.task_obs[t + 1] - o0;
    if (n <= uint32_t(kAdjTaskObs)) {
      const bool valid = uint32_t(lane) < n;
      const uint32_t i = o0 + (valid ? lane : 0);
      const uint32_t c = A.obs_camera[i], pt = A.obs_point[i];
      const bool act = valid && A.active[c] != 0;
      double W[18], pc[6], vb[6];
      const double2* w2 = reinterpret_cast<const double2*>(A.Hcp + 18 * size_t(i));
      for (int k = 0; k < 9; k++) {
        const double2 v = w2[k];
        W[2 * k] = v.x;
        W[2 * k + 1] = v.y;
      }
      load6(A.p + 6 * size_t(c), pc);
      load6(A.Vinv + 6 * size_t(pt), vb);
      const uint32_t p0 = __shfl_sync(kFull, pt, 0);
      const int seg = valid ? int(pt - p0) : -1 - lane;
      double u[3] = {0, 0, 0};
      if (act) adj_wt(W, pc, u);
      const Runs runs = lane_runs(seg, lane);
      run_scan(u, runs);
      const bool tail = valid && run_tail(runs, lane);
      double y[3] = {0, 0, 0};
      if (tail) {
        y[0] = vb[0] * u[0] + vb[1] * u[1] + vb[2] * u[2];
        y[1] = vb[1] * u[0] + vb[3] * u[1] + vb[4] * u[2];
        y[2] = vb[2] * u[0] + vb[4] * u[1] + vb[5] * u[2];
      }
      const unsigned tails = __ballot_sync(kFull, tail);
      const int src = valid ? __ffs(tails & (kFull << lane)) - 1 : lane;
      for (int k = 0; k < 3; k++) y[k] = __shfl_sync(kFull, y[k], src);
      if (act) adj_scatter(adj_acc, C, c, W, y);
      continue;
    }
    // A point with more than 32 observations: rounds of 32, one warp-wide sum.
    const uint32_t p0 = A.obs_point[o0];
    const uint32_t rounds = (n + kAdjTaskObs - 1) / kAdjTaskObs;
    double u[3] = {0, 0, 0};
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kAdjTaskObs + lane;
      if (k >= n) continue;
      const uint32_t i = o0 + k, c = A.obs_camera[i];
      if (A.active[c] == 0) continue;
      double v[3];
      adj_wt(A.Hcp + 18 * size_t(i), A.p + 6 * size_t(c), v);
      u[0] += v[0];
      u[1] += v[1];
      u[2] += v[2];
    }
    warp_allsum(u);
    double vb[6];
    load6(A.Vinv + 6 * size_t(p0), vb);
    const double y[3] = {vb[0] * u[0] + vb[1] * u[1] + vb[2] * u[2], vb[1] * u[0] + vb[3] * u[1] + vb[4] * u[2],
                         vb[2] * u[0] + vb[4] * u[1] + vb[5] * u[2]};
    for (uint32_t r = 0; r < rounds; r++) {
      const uint32_t k = r * kAdjTaskObs + lane;
      if (k >= n) continue;
      const uint32_t i = o0 + k, c = A.obs_camera[i];
      if (A.active[c] != 0) adj_scatter(adj_acc, C, c, A.Hcp + 18 * size_t(i), y);
    }
  }
  __syncthreads();
  double* out = A.part + size_t(blockIdx.x) * 6 * C;
  for (uint32_t j = threadIdx.x; j < 6 * C; j += blockDim.x) {
    const size_t at = size_t(j % 6) * C + j / 6;
    double v = 0;
    for (uint32_t w = 0; w < copies; w++) v += adj_smem[size_t(w) * 6 * C + at];
    out[j] = v;
  }
}

// S p = U_c p_c + the blocks' partial rows: 32 rows per block, each of its kAdjColumnWarps warps
// summing every kAdjColumnWarps-th block's partial rows (coalesced; short dependent chains, about
// nine loads a lane at 296 product blocks), then the warps' sums in a fixed order.
constexpr int kAdjColumnWarps = 32;

__global__ void __launch_bounds__(32 * kAdjColumnWarps) k_adj_columns(AdjParams A) {
  __shared__ double part[kAdjColumnWarps][33];
  if (A.state[A_ACTIVE] == 0) return;
  const uint32_t n = 6 * A.C;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t j = blockIdx.x * 32 + lane;
  double s = 0;
  if (j < n)
    for (uint32_t b = warp; b < A.prod_blocks; b += kAdjColumnWarps) s += A.part[size_t(b) * n + j];
  part[warp][lane] = s;
  __syncthreads();
  if (warp != 0 || j >= n) return;
  double sum = 0;
  for (int w = 0; w < kAdjColumnWarps; w++) sum += part[w][lane];
  const uint32_t c = j / 6, a = j % 6;
  const double* U = A.U + 21 * size_t(c);
  const double* pc = A.p + 6 * size_t(c);
  double up = 0;
  for (int k = 0; k < 6; k++) up += U[sym6(a, k)] * pc[k];
  A.Sp[j] = up + (A.active[c] != 0 ? sum : 0.0);
}

__global__ void __launch_bounds__(1024) k_adj_vec(AdjParams A) {
  __shared__ double red[64];
  double* st = A.state;
  if (st[A_ACTIVE] == 0) return;
  const uint32_t m = 6 * A.C;
  double v[1] = {0};
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) v[0] += A.p[j] * A.Sp[j];
  adj_block_sum(v, red);
  const double den = v[0], alpha = st[A_RHO] / den;
  if (!(den > 0) || !(fabs(alpha) < 1e30)) {
    if (threadIdx.x == 0) {
      st[A_ACTIVE] = 0;
      st[A_FAILED] = 1;
    }
    return;
  }
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
    A.x[j] += alpha * A.p[j];
    A.r[j] -= alpha * A.Sp[j];
  }
  __syncthreads();
  double w[2] = {0, 0};
  for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
    const double zz = adj_precondition(A, j);
    A.z[j] = zz;
    w[0] += A.r[j] * zz;
    w[1] += A.r[j] * A.r[j];
  }
  adj_block_sum(w, red);
  const double rho = w[0], rr = w[1];
  const bool done = rr <= A.tol * A.tol * st[A_R0];
  const bool broke = !done && !(rho > 0);
  const double beta = rho / st[A_RHO];
  __syncthreads();
  if (!done && !broke)
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) A.p[j] = A.z[j] + beta * A.p[j];
  if (threadIdx.x == 0) {
    st[A_STEPS] += 1;
    st[A_R2] = rr;
    if (done) st[A_ACTIVE] = 0;
    else if (broke) {
      st[A_ACTIVE] = 0;
      st[A_FAILED] = 1;
    } else {
      st[A_RHO] = rho;
    }
  }
}

// The device-side PCG loop: k_adj_loop_next runs at the end of every body iteration, so the loop
// ends within its budget; it ends earlier when the PCG stops.
__global__ void k_adj_loop_begin(AdjParams A, uint32_t limit) {
  A.state[A_LOOP_ITERS] = 0;
  A.state[A_LOOP_LIMIT] = limit;
}

__global__ void k_adj_loop_next(AdjParams A) {
  double* st = A.state;
  const double iters = st[A_LOOP_ITERS] + 1;
  st[A_LOOP_ITERS] = iters;
  cudaGraphSetConditional(A.loop, st[A_ACTIVE] != 0 && iters < st[A_LOOP_LIMIT] ? 1u : 0u);
}

__global__ void __launch_bounds__(256) k_adj_back(AdjParams A) {
  for (uint32_t pt = blockIdx.x * blockDim.x + threadIdx.x; pt < A.P; pt += gridDim.x * blockDim.x) {
    double t[3] = {A.bp[3 * size_t(pt)], A.bp[3 * size_t(pt) + 1], A.bp[3 * size_t(pt) + 2]};
    for (uint32_t i = A.point_start[pt]; i < A.point_start[pt + 1]; i++) {
      const uint32_t c = A.obs_camera[i];
      if (A.active[c] == 0) continue;
      const double* W = A.Hcp + 18 * size_t(i);
      const double* xc = A.x + 6 * size_t(c);
      for (int a = 0; a < 6; a++) {
        t[0] -= W[3 * a] * xc[a];
        t[1] -= W[3 * a + 1] * xc[a];
        t[2] -= W[3 * a + 2] * xc[a];
      }
    }
    const double* vi = A.Vinv + 6 * size_t(pt);
    double* l = A.lp + 3 * size_t(pt);
    l[0] = vi[0] * t[0] + vi[1] * t[1] + vi[2] * t[2];
    l[1] = vi[1] * t[0] + vi[3] * t[1] + vi[4] * t[2];
    l[2] = vi[2] * t[0] + vi[4] * t[1] + vi[5] * t[2];
  }
}

// ---- the vector-Jacobian product --------------------------------------------------------------

__global__ void __launch_bounds__(128) k_adj_vjp(AdjParams A) {
  __shared__ double red[2 * 4];
  double acc[2] = {0, 0};  // -lambda . dF/ds, -lambda . dF/dk1
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.M; i += gridDim.x * blockDim.x) {
    const uint32_t c = A.obs_camera[i], pt = A.obs_point[i];
    double pose[12];
    adj_pose(A, c, pose);
    const Camera k = adj_camera(A, c);
    ObsSecond o;
    double H[9][9];
    double* yb = A.ybar + 2 * size_t(i);
    if (!obs_second(pose, k, radial_limit(k.k1, k.k2), A.points + 3 * size_t(pt), A.pixels[2 * size_t(i)],
                    A.pixels[2 * size_t(i) + 1], A.huber, A.active[c] != 0, o, H)) {
      yb[0] = yb[1] = 0;
      continue;
    }
    double lam[9];
    for (int a = 0; a < 6; a++) lam[a] = A.active[c] ? A.x[6 * size_t(c) + a] : 0.0;
    for (int m = 0; m < 3; m++) lam[6 + m] = A.lp[3 * size_t(pt) + m];
    double jl[2] = {0, 0}, kl[2] = {0, 0};
    for (int a = 0; a < 9; a++) {
      jl[0] += o.J[0][a] * lam[a];
      jl[1] += o.J[1][a] * lam[a];
      kl[0] += o.Jk[0][a] * lam[a];
      kl[1] += o.Jk[1][a] * lam[a];
    }
    // dF_i/dy_i = -J^T W~: ybar_i = W~ J lambda
    const double wj0 = o.Wt[0] * jl[0] + o.Wt[1] * jl[1], wj1 = o.Wt[1] * jl[0] + o.Wt[2] * jl[1];
    yb[0] = wj0;
    yb[1] = wj1;
    // dF_i/ds = w J^T r + J^T W~ jf;  dF_i/dk1 = w Jk^T r + J^T W~ jk
    const double Fs = o.w * (jl[0] * o.r[0] + jl[1] * o.r[1]) + (wj0 * o.jf[0] + wj1 * o.jf[1]);
    const double Fk = o.w * (kl[0] * o.r[0] + kl[1] * o.r[1]) + (wj0 * o.jk[0] + wj1 * o.jk[1]);
    acc[0] -= Fs;
    acc[1] -= Fk;
  }
  adj_block_sum(acc, red);
  if (threadIdx.x == 0) {
    atomicAdd(A.state + A_SBAR, acc[0]);
    atomicAdd(A.state + A_KBAR, acc[1]);
  }
}

// The cotangent of the output poses (R row-major, t) and points in local coordinates, and the
// v_s . g sum of its oblique gauge projection.
__global__ void __launch_bounds__(256) k_adj_cotangent(AdjParams A, const double* g) {
  __shared__ double red[8];
  const double* st = A.state;
  const double o[3] = {st[A_ORIGIN], st[A_ORIGIN + 1], st[A_ORIGIN + 2]};
  double dot[1] = {0};
  const uint32_t n = A.C + A.P;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j < A.C) {
      const uint32_t c = j;
      double* out = A.cot + 6 * size_t(c);
      if (A.active[c] == 0) {
        for (int k = 0; k < 6; k++) out[k] = 0;
        continue;
      }
      const double* R = A.poses + 12 * size_t(c);
      const double* t = R + 9;
      const double* gR = g + 12 * size_t(c);
      const double* gt = gR + 9;
      double Am[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Am[a][b] = gR[3 * a] * R[3 * b] + gR[3 * a + 1] * R[3 * b + 1] + gR[3 * a + 2] * R[3 * b + 2];
      out[0] = Am[2][1] - Am[1][2] + (t[1] * gt[2] - t[2] * gt[1]);
      out[1] = Am[0][2] - Am[2][0] + (t[2] * gt[0] - t[0] * gt[2]);
      out[2] = Am[1][0] - Am[0][1] + (t[0] * gt[1] - t[1] * gt[0]);
      out[3] = gt[0];
      out[4] = gt[1];
      out[5] = gt[2];
      // v_s on this camera: (0, t + R o)
      for (int i = 0; i < 3; i++) dot[0] += (t[i] + R[3 * i] * o[0] + R[3 * i + 1] * o[1] + R[3 * i + 2] * o[2]) * gt[i];
    } else {
      const uint32_t pt = j - A.C;
      const double* gX = g + 12 * size_t(A.C) + 3 * size_t(pt);
      const double* X = A.points + 3 * size_t(pt);
      double* out = A.cot + 6 * size_t(A.C) + 3 * size_t(pt);
      for (int i = 0; i < 3; i++) {
        out[i] = gX[i];
        dot[0] += (X[i] - o[i]) * gX[i];
      }
    }
  }
  adj_block_sum(dot, red);
  if (threadIdx.x == 0) atomicAdd(A.state + A_DOT, dot[0]);
}

__global__ void k_adj_cotangent_project(AdjParams A) {
  if (!A.normalize_scale) return;
  double n[3], b;
  baseline_gradient(A, n, b);
  const double s = A.state[A_DOT] / b;  // grad_c . v_s = b
  double* out = A.cot + 6 * size_t(A.scale_view) + 3;
  for (int i = 0; i < 3; i++) out[i] -= n[i] * s;
}

// ---- Newton steps ------------------------------------------------------------------------------

__global__ void k_adj_init(AdjParams A) {
  double* st = A.state;
  for (int j = 0; j < A_WORDS; j++) st[j] = 0;
  const double* a = A.poses + 12 * size_t(A.anchor);
  const double* b = A.poses + 12 * size_t(A.scale_view);
  double o[3], s[3];
  for (int i = 0; i < 3; i++) {
    o[i] = -a[i] * a[9] - a[i + 3] * a[10] - a[i + 6] * a[11];
    s[i] = -b[i] * b[9] - b[i + 3] * b[10] - b[i + 6] * b[11];
  }
  for (int i = 0; i < 3; i++) st[A_ORIGIN + i] = o[i];
  st[A_BASELINE] = sqrt((o[0] - s[0]) * (o[0] - s[0]) + (o[1] - s[1]) * (o[1] - s[1]) + (o[2] - s[2]) * (o[2] - s[2]));
}

__global__ void k_adj_reset(AdjParams A) {
  const int w = threadIdx.x;
  if (w == A_GNORM || w == A_INVALID || w == A_POINT_FAILED || w == A_POINT_SINGULAR || w == A_CAMERA_FAILED ||
      w == A_DOT || w == A_SBAR ||
      w == A_KBAR)
    A.state[w] = 0;
}

__global__ void __launch_bounds__(256) k_adj_newton_cameras(AdjParams A) {
  __shared__ double scale;
  double* st = A.state;
  for (uint32_t c = threadIdx.x; c < A.C; c += blockDim.x) {
    double pose[12], moved[12];
    for (int j = 0; j < 12; j++) pose[j] = A.poses[12 * size_t(c) + j];
    if (A.active[c] != 0) move_pose(pose, A.x + 6 * size_t(c), moved);
    else
      for (int j = 0; j < 12; j++) moved[j] = pose[j];
    for (int j = 0; j < 12; j++) A.tposes[12 * size_t(c) + j] = moved[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    scale = 1;
    if (A.normalize_scale) {
      const double* p = A.tposes + 12 * size_t(A.scale_view);
      double cc[3];
      for (int i = 0; i < 3; i++) cc[i] = -p[i] * p[9] - p[i + 3] * p[10] - p[i + 6] * p[11];
      const double e0 = cc[0] - st[A_ORIGIN], e1 = cc[1] - st[A_ORIGIN + 1], e2 = cc[2] - st[A_ORIGIN + 2];
      const double b = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
      if (b > 1e-12) scale = st[A_BASELINE] / b;
    }
    st[A_SCALE] = scale;
    st[A_COST] = 0;
  }
  __syncthreads();
  if (!A.normalize_scale) return;
  const double s = scale;
  const double o[3] = {st[A_ORIGIN], st[A_ORIGIN + 1], st[A_ORIGIN + 2]};
  for (uint32_t h = threadIdx.x; h < A.C; h += blockDim.x) {
    if (h == A.anchor) continue;
    double* p = A.tposes + 12 * size_t(h);
    double rot[3];
    for (int i = 0; i < 3; i++) rot[i] = (p[i * 3] * o[0] + p[i * 3 + 1] * o[1] + p[i * 3 + 2] * o[2] + p[9 + i]) - p[9 + i];
    for (int i = 0; i < 3; i++) p[9 + i] = s * p[9 + i] + (s - 1) * rot[i];
  }
}

__global__ void __launch_bounds__(256) k_adj_newton_points(AdjParams A) {
  const double* st = A.state;
  for (uint32_t pt = blockIdx.x * blockDim.x + threadIdx.x; pt < A.P; pt += gridDim.x * blockDim.x) {
    const double* X = A.points + 3 * size_t(pt);
    for (int i = 0; i < 3; i++) {
      double v = X[i] + A.lp[3 * size_t(pt) + i];
      if (A.normalize_scale) v = st[A_ORIGIN + i] + st[A_SCALE] * (v - st[A_ORIGIN + i]);
      A.tpoints[3 * size_t(pt) + i] = v;
    }
  }
}

// The robust cost of (poses, points) into A_COST (1e30 per observation outside the domain).
__global__ void __launch_bounds__(256) k_adj_cost(AdjParams A, const double* poses, const double* points) {
  __shared__ double red[8];
  double v[1] = {0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.M; i += gridDim.x * blockDim.x) {
    const uint32_t c = A.obs_camera[i], pt = A.obs_point[i];
    double pose[12];
    for (int j = 0; j < 12; j++) pose[j] = poses[12 * size_t(c) + j];
    const Camera k = adj_camera(A, c);
    double oc, os;
    candidate_cost(pose, k, points + 3 * size_t(pt), false, A.pixels[2 * size_t(i)], A.pixels[2 * size_t(i) + 1],
                   A.huber, oc, os);
    v[0] += oc;
  }
  adj_block_sum(v, red);
  if (threadIdx.x == 0) atomicAdd(A.state + A_COST, v[0]);
}

__global__ void __launch_bounds__(256) k_adj_commit(AdjParams A) {
  const uint32_t n = 12 * A.C + 3 * A.P;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (j < 12 * A.C) A.poses[j] = A.tposes[j];
    else A.points[j - 12 * A.C] = A.tpoints[j - 12 * A.C];
  }
}

__global__ void k_adj_zero_cost(AdjParams A) { A.state[A_COST] = 0; }

uint32_t grid_for(uint32_t n, uint32_t threads) {
  const uint32_t b = (n + threads - 1) / threads;
  return b < 1 ? 1 : (b > 65535 ? 65535 : b);
}

}  // namespace

// Each launcher returns the number of kernels it launched.
uint32_t adj_launch_init(const AdjParams& a, cudaStream_t s) {
  k_adj_init<<<1, 1, 0, s>>>(a);
  return 1;
}
uint32_t adj_launch_reset(const AdjParams& a, cudaStream_t s) {
  k_adj_reset<<<1, 32, 0, s>>>(a);
  return 1;
}

uint32_t adj_launch_assemble(const AdjParams& a, cudaStream_t s) {
  k_adj_obs<<<grid_for(a.M, 128), 128, 0, s>>>(a);
  k_adj_points<<<grid_for(a.P, 256), 256, 0, s>>>(a);
  k_adj_cameras<<<a.C, 128, 0, s>>>(a);
  return 3;
}

uint32_t adj_launch_pcg_init(const AdjParams& a, cudaStream_t s) {
  k_adj_pcg_init<<<1, 1024, 0, s>>>(a);
  return 1;
}

constexpr size_t kAdjSmemLimit = 227 * 1024 - 1024;

uint32_t adj_one_pass_max_cameras() { return uint32_t(kAdjSmemLimit / (6 * sizeof(double))); }

// As many copies of the camera sums (one per warp at most) as let two blocks share an SM; one copy
// when not even two fit.
uint32_t adj_product_copies(uint32_t C) {
  const size_t one = 6 * sizeof(double) * size_t(C ? C : 1), fit = (kAdjSmemLimit / 2) / one;
  return fit >= 2 ? uint32_t(std::min<size_t>(kAdjProductThreads / 32, fit)) : 1u;
}

size_t adj_product_smem(uint32_t C) { return size_t(adj_product_copies(C)) * 6 * sizeof(double) * C; }

// Resident blocks per SM of the one-pass product (registers and shared memory), from the runtime.
uint32_t adj_product_blocks_per_sm(uint32_t C) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_product, kAdjProductThreads, adj_product_smem(C)) !=
          cudaSuccess ||
      n < 1)
    return 1;
  return uint32_t(n);
}

cudaError_t adj_configure() {
  return cudaFuncSetAttribute(k_adj_product, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kAdjSmemLimit));
}

uint32_t adj_launch_pcg_step(const AdjParams& a, cudaStream_t s, cudaEvent_t before, cudaEvent_t after) {
  if (a.prod_blocks) {
    if (before) cudaEventRecord(before, s);
    k_adj_product<<<a.prod_blocks, kAdjProductThreads, adj_product_smem(a.C), s>>>(a);
    if (after) cudaEventRecord(after, s);
    k_adj_columns<<<(6 * a.C + 31) / 32, 32 * kAdjColumnWarps, 0, s>>>(a);
  } else {
    k_adj_prod_points<<<grid_for(a.P, 256), 256, 0, s>>>(a);
    k_adj_prod_cameras<<<a.C, 128, 0, s>>>(a);
  }
  k_adj_vec<<<1, 1024, 0, s>>>(a);
  return 3;
}

uint32_t adj_launch_loop_begin(const AdjParams& a, uint32_t limit, cudaStream_t s) {
  k_adj_loop_begin<<<1, 1, 0, s>>>(a, limit);
  return 1;
}

uint32_t adj_launch_loop_next(const AdjParams& a, cudaStream_t s) {
  k_adj_loop_next<<<1, 1, 0, s>>>(a);
  return 1;
}

uint32_t adj_launch_back_substitute(const AdjParams& a, cudaStream_t s) {
  k_adj_back<<<grid_for(a.P, 256), 256, 0, s>>>(a);
  return 1;
}

uint32_t adj_launch_newton_candidate(const AdjParams& a, cudaStream_t s) {
  k_adj_newton_cameras<<<1, 256, 0, s>>>(a);
  k_adj_newton_points<<<grid_for(a.P, 256), 256, 0, s>>>(a);
  k_adj_cost<<<grid_for(a.M, 256), 256, 0, s>>>(a, a.tposes, a.tpoints);
  return 3;
}

uint32_t adj_launch_newton_commit(const AdjParams& a, cudaStream_t s) {
  k_adj_commit<<<grid_for(12 * a.C + 3 * a.P, 256), 256, 0, s>>>(a);
  return 1;
}

uint32_t adj_launch_cost(const AdjParams& a, cudaStream_t s) {
  k_adj_zero_cost<<<1, 1, 0, s>>>(a);
  k_adj_cost<<<grid_for(a.M, 256), 256, 0, s>>>(a, a.poses, a.points);
  return 2;
}

uint32_t adj_launch_cotangent(const AdjParams& a, const double* cotangent, cudaStream_t s) {
  k_adj_cotangent<<<grid_for(a.C + a.P, 256), 256, 0, s>>>(a, cotangent);
  k_adj_cotangent_project<<<1, 1, 0, s>>>(a);
  return 2;
}

uint32_t adj_launch_vjp(const AdjParams& a, cudaStream_t s) {
  k_adj_vjp<<<grid_for(a.M, 128), 128, 0, s>>>(a);
  return 1;
}

}  // namespace tba
