// Per-observation and per-block math of the bundle adjustment, device side.
//
// Restates the reference's shared kernel math (src/device/gpu/numerics.shade.ts): the pinhole +
// two-term radial projection with its analytic 2x3 derivative (project, :79-99 and :141-173),
// the pose Jacobian row of a left-multiplied rotation (poseRow, :181-183), the Huber cost
// (robustCost, :184-187), the equilibrated 3x3 and 6x6 Cholesky solves (solve3, :25-45;
// solve6, :221-253) and the left SO(3) update (movePose, :254-281), in IEEE binary64.
#pragma once

#include <cstdint>

namespace tba {

struct Camera {
  double fx, fy, cx, cy, k1, k2;
};

// radialLimit: the first zero of the radial derivative bounds the injective branch.
__host__ __device__ inline double radial_limit(double k1, double k2) {
  if (k2 == 0) return k1 < 0 ? -1 / (3 * k1) : 1e30;
  const double a = 5 * k2, b = 3 * k1, d = b * b - 4 * a;
  if (d < 0) return 1e30;
  const double q = -0.5 * (b + (b < 0 ? -1.0 : 1.0) * sqrt(d));
  double limit = 1e30;
  const double first = q / a;
  if (first > 0) limit = fmin(limit, first);
  if (q != 0) {
    const double second = 1 / q;
    if (second > 0) limit = fmin(limit, second);
  }
  return limit;
}

// project: pixel and the derivative rows du, dv with respect to the camera-frame point q.
// Returns false outside the model's domain (behind the camera, beyond the radial fold or
// numerically unbounded), as the reference's `ok = 0`.
__host__ __device__ inline bool project(const Camera& k, const double q[3], double pixel[2],
                                        double du[3], double dv[3]) {
  if (!(q[2] > 1e-12)) return false;
  const double iz = 1.0 / q[2];
  const double x = q[0] / q[2], y = q[1] / q[2], r2 = x * x + y * y;
  if (!(r2 < radial_limit(k.k1, k.k2) && r2 < 1e8)) return false;
  const double d = 1 + k.k1 * r2 + k.k2 * r2 * r2, g = 2 * (k.k1 + 2 * k.k2 * r2);
  if (!(d > 0 && 1 + 3 * k.k1 * r2 + 5 * k.k2 * r2 * r2 > 0)) return false;
  const double xx = d + g * x * x, xy = g * x * y, yy = d + g * y * y;
  pixel[0] = k.fx * x * d + k.cx;
  pixel[1] = k.fy * y * d + k.cy;
  du[0] = k.fx * xx * iz;
  du[1] = k.fx * xy * iz;
  du[2] = -k.fx * (xx * x + xy * y) * iz;
  dv[0] = k.fy * xy * iz;
  dv[1] = k.fy * yy * iz;
  dv[2] = -k.fy * (xy * x + yy * y) * iz;
  const double mp = fmax(fabs(pixel[0]), fabs(pixel[1]));
  const double mu = fmax(fmax(fabs(du[0]), fabs(du[1])), fabs(du[2]));
  const double mv = fmax(fmax(fabs(dv[0]), fabs(dv[1])), fabs(dv[2]));
  return mp < 1e12 && mu < 1e12 && mv < 1e12;
}

// poseRow: d(pixel row)/d(rotation, translation) for q' = exp(w) q + v.
__host__ __device__ inline void pose_row(const double q[3], const double j[3], double out[6]) {
  out[0] = j[2] * q[1] - j[1] * q[2];
  out[1] = j[0] * q[2] - j[2] * q[0];
  out[2] = j[1] * q[0] - j[0] * q[1];
  out[3] = j[0];
  out[4] = j[1];
  out[5] = j[2];
}

__host__ __device__ inline double robust_cost(double e, double h) {
  return e <= h ? e * e : 2 * h * e - h * h;
}

// solve3 on the three unit vectors: the equilibrated Cholesky inverse of a 3x3 SPD block,
// symmetrised; `a` row-major.  Output: the 6 unique entries (00, 01, 02, 11, 12, 22).
__host__ __device__ inline bool inverse3_spd(const double a[9], double out[6]) {
  if (!(fmin(a[0], fmin(a[4], a[8])) > 0)) return false;
  const double d0 = 1 / sqrt(a[0]), d1 = 1 / sqrt(a[4]), d2 = 1 / sqrt(a[8]);
  const double l10 = a[3] * d0 * d1, l20 = a[6] * d0 * d2;
  const double pivot1 = 1 - l10 * l10;
  if (!(pivot1 > 1e-14)) return false;
  const double l11 = sqrt(pivot1), l21 = (a[7] * d1 * d2 - l20 * l10) / l11;
  const double pivot2 = 1 - l20 * l20 - l21 * l21;
  if (!(pivot2 > 1e-14)) return false;
  const double l22 = sqrt(pivot2);
  double inv[9];
  for (int column = 0; column < 3; column++) {
    const double b0 = column == 0, b1 = column == 1, b2 = column == 2;
    const double y0 = b0 * d0, y1 = (b1 * d1 - l10 * y0) / l11, y2 = (b2 * d2 - l20 * y0 - l21 * y1) / l22;
    const double x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = y0 - l10 * x1 - l20 * x2;
    inv[column] = x0 * d0;
    inv[3 + column] = x1 * d1;
    inv[6 + column] = x2 * d2;
  }
  out[0] = inv[0];
  out[1] = (inv[1] + inv[3]) * 0.5;
  out[2] = (inv[2] + inv[6]) * 0.5;
  out[3] = inv[4];
  out[4] = (inv[5] + inv[7]) * 0.5;
  out[5] = inv[8];
  return true;
}

// solve3: x = a^-1 b by the equilibrated Cholesky factorisation of the SPD block `a` (row-major),
// with the same pivot floors as inverse3_spd; false when `a` is not safely positive definite.
__host__ __device__ inline bool solve3_spd(const double a[9], const double b[3], double x[3]) {
  if (!(fmin(a[0], fmin(a[4], a[8])) > 0)) return false;
  const double d0 = 1 / sqrt(a[0]), d1 = 1 / sqrt(a[4]), d2 = 1 / sqrt(a[8]);
  const double l10 = a[3] * d0 * d1, l20 = a[6] * d0 * d2;
  const double pivot1 = 1 - l10 * l10;
  if (!(pivot1 > 1e-14)) return false;
  const double l11 = sqrt(pivot1), l21 = (a[7] * d1 * d2 - l20 * l10) / l11;
  const double pivot2 = 1 - l20 * l20 - l21 * l21;
  if (!(pivot2 > 1e-14)) return false;
  const double l22 = sqrt(pivot2), y0 = b[0] * d0;
  const double y1 = (b[1] * d1 - l10 * y0) / l11, y2 = (b[2] * d2 - l20 * y0 - l21 * y1) / l22;
  const double x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = y0 - l10 * x1 - l20 * x2;
  x[0] = x0 * d0;
  x[1] = x1 * d1;
  x[2] = x2 * d2;
  return true;
}

// Index of entry (i, j) of a symmetric 6x6 block stored as its lower triangle, row by row.
__host__ __device__ constexpr int sym6(int i, int j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// solve6 on the six unit vectors: the equilibrated Cholesky inverse of a 6x6 SPD block given by
// its lower triangle (21 entries, sym6 order), symmetrised, written full row-major (36).
__host__ __device__ inline bool inverse6_spd(const double s[21], double out[36]) {
  double L[21], scale[6];
  for (int i = 0; i < 6; i++) {
    const double dii = s[sym6(i, i)];
    if (!(dii > 0)) return false;
    scale[i] = 1 / sqrt(dii);
  }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j <= i; j++) {
      double value = s[sym6(i, j)] * scale[i] * scale[j];
      for (int k = 0; k < j; k++) value -= L[sym6(i, k)] * L[sym6(j, k)];
      if (i == j) {
        if (!(value > 1e-14)) return false;
        L[sym6(i, i)] = sqrt(value);
      } else {
        L[sym6(i, j)] = value / L[sym6(j, j)];
      }
    }
  for (int column = 0; column < 6; column++) {
    double v[6];
    for (int i = 0; i < 6; i++) {
      double t = (i == column ? 1.0 : 0.0) * scale[i];
      for (int j = 0; j < i; j++) t -= L[sym6(i, j)] * v[j];
      v[i] = t / L[sym6(i, i)];
    }
    for (int i = 5; i >= 0; i--) {
      double t = v[i];
      for (int j = i + 1; j < 6; j++) t -= L[sym6(j, i)] * v[j];
      v[i] = t / L[sym6(i, i)];
    }
    for (int i = 0; i < 6; i++) out[i * 6 + column] = v[i] * scale[i];
  }
  for (int j = 0; j < 6; j++)
    for (int k = j + 1; k < 6; k++) {
      const double v = (out[j * 6 + k] + out[k * 6 + j]) * 0.5;
      out[j * 6 + k] = v;
      out[k * 6 + j] = v;
    }
  return true;
}

// movePose: R' = exp(w) R, t' = exp(w) t + v, with the small-angle series below 1e-7 rad.
__host__ __device__ inline void move_pose(const double p[12], const double delta[6], double out[12]) {
  const double x = delta[0], y = delta[1], z = delta[2];
  const double theta = sqrt(x * x + y * y + z * z);
  double a = 1 - (theta * theta) / 6, b = 0.5 - (theta * theta) / 24;
  if (theta >= 1e-7) {
    a = sin(theta) / theta;
    b = (1 - cos(theta)) / (theta * theta);
  }
  const double W[9] = {0, -z, y, z, 0, -x, -y, x, 0};
  double dR[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dR[i * 3 + j] += a * W[i * 3 + j];
      for (int k = 0; k < 3; k++) dR[i * 3 + j] += b * W[i * 3 + k] * W[k * 3 + j];
    }
  for (int i = 0; i < 3; i++) {
    out[9 + i] = delta[3 + i];
    for (int j = 0; j < 3; j++) out[i * 3 + j] = 0;
    for (int k = 0; k < 3; k++) {
      out[9 + i] += dR[i * 3 + k] * p[9 + k];
      for (int j = 0; j < 3; j++) out[i * 3 + j] += dR[i * 3 + k] * p[k * 3 + j];
    }
  }
}

// The factors of one observation's Jacobian.  With the camera-frame point q, the projection's
// derivative rows du, dv (d pixel / d q), the focal column jf = pixel - principal point, the
// residual r and the Huber weight w, every product the solver needs is a few dozen FMAs (R the
// camera rotation, delta = (omega, v) a camera step, g a 2-vector):
//   J_c delta = [du . (omega x q + v), dv . (omega x q + v)]
//   J_c^T g   = [q x h ; h]            with h = g_u du + g_v dv
//   J_p y     = [du . (R y), dv . (R y)]
//   J_p^T g   = R^T (g_u du + g_v dv)
// so the Schur blocks W_i = w J_c^T J_p never need to be stored: they are recomputed from the
// pose, the camera, the point and the pixel.  A bearing has no translation columns; a fixed
// camera has no J_c.
struct Geo {
  double q[3], du[3], dv[3], jf[2], r[2], w, sq;
};

// radial_limit(k1, k2) is a per-camera constant; `limit` passes it in.
__host__ __device__ inline bool geometry(const double pose[12], const Camera& k, double limit, const double X[3],
                                         bool directional, double u, double v, double huber, Geo& g) {
  for (int i = 0; i < 3; i++) {
    g.q[i] = pose[i * 3] * X[0] + pose[i * 3 + 1] * X[1] + pose[i * 3 + 2] * X[2];
    if (!directional) g.q[i] += pose[9 + i];
  }
  if (!(g.q[2] > 1e-12)) return false;
  const double iz = 1.0 / g.q[2];
  const double x = g.q[0] * iz, y = g.q[1] * iz, r2 = x * x + y * y;
  if (!(r2 < limit && r2 < 1e8)) return false;
  const double d = 1 + k.k1 * r2 + k.k2 * r2 * r2, gg = 2 * (k.k1 + 2 * k.k2 * r2);
  if (!(d > 0 && 1 + 3 * k.k1 * r2 + 5 * k.k2 * r2 * r2 > 0)) return false;
  const double xx = d + gg * x * x, xy = gg * x * y, yy = d + gg * y * y;
  const double px = k.fx * x * d, py = k.fy * y * d;
  g.du[0] = k.fx * xx * iz;
  g.du[1] = k.fx * xy * iz;
  g.du[2] = -k.fx * (xx * x + xy * y) * iz;
  g.dv[0] = k.fy * xy * iz;
  g.dv[1] = k.fy * yy * iz;
  g.dv[2] = -k.fy * (xy * x + yy * y) * iz;
  const double mp = fmax(fabs(px + k.cx), fabs(py + k.cy));
  const double mu = fmax(fmax(fabs(g.du[0]), fabs(g.du[1])), fabs(g.du[2]));
  const double mv = fmax(fmax(fabs(g.dv[0]), fabs(g.dv[1])), fabs(g.dv[2]));
  if (!(mp < 1e12 && mu < 1e12 && mv < 1e12)) return false;
  g.jf[0] = px;
  g.jf[1] = py;
  g.r[0] = (px + k.cx) - u;
  g.r[1] = (py + k.cy) - v;
  g.sq = g.r[0] * g.r[0] + g.r[1] * g.r[1];
  g.w = g.sq > huber * huber ? huber / sqrt(g.sq) : 1.0;
  return true;
}

// W_i^T x = w J_p^T (J_c x_c + jf x_f): the point-side product of one observation.
__host__ __device__ inline void wt_product(const Geo& g, const double pose[12], const double* xc, double xf,
                                           bool variable, bool directional, bool shared, double t[3]) {
  double au = 0, av = 0;
  if (variable) {
    double m0 = xc[1] * g.q[2] - xc[2] * g.q[1];
    double m1 = xc[2] * g.q[0] - xc[0] * g.q[2];
    double m2 = xc[0] * g.q[1] - xc[1] * g.q[0];
    if (!directional) {
      m0 += xc[3];
      m1 += xc[4];
      m2 += xc[5];
    }
    au = g.du[0] * m0 + g.du[1] * m1 + g.du[2] * m2;
    av = g.dv[0] * m0 + g.dv[1] * m1 + g.dv[2] * m2;
  }
  if (shared) {
    au += g.jf[0] * xf;
    av += g.jf[1] * xf;
  }
  au *= g.w;
  av *= g.w;
  const double h0 = au * g.du[0] + av * g.dv[0], h1 = au * g.du[1] + av * g.dv[1], h2 = au * g.du[2] + av * g.dv[2];
  for (int c = 0; c < 3; c++) t[c] = pose[c] * h0 + pose[3 + c] * h1 + pose[6 + c] * h2;
}

// W_i y = w J_c^T (J_p y) (6, zero for a fixed camera) and the focal share w jf . (J_p y).
__host__ __device__ inline void w_product(const Geo& g, const double pose[12], const double y[3], bool variable,
                                          bool directional, double d[6], double& e) {
  const double R0 = pose[0] * y[0] + pose[1] * y[1] + pose[2] * y[2];
  const double R1 = pose[3] * y[0] + pose[4] * y[1] + pose[5] * y[2];
  const double R2 = pose[6] * y[0] + pose[7] * y[1] + pose[8] * y[2];
  const double bu = g.w * (g.du[0] * R0 + g.du[1] * R1 + g.du[2] * R2);
  const double bv = g.w * (g.dv[0] * R0 + g.dv[1] * R1 + g.dv[2] * R2);
  e = bu * g.jf[0] + bv * g.jf[1];
  if (!variable) {
    for (int c = 0; c < 6; c++) d[c] = 0;
    return;
  }
  const double h0 = bu * g.du[0] + bv * g.dv[0], h1 = bu * g.du[1] + bv * g.dv[1], h2 = bu * g.du[2] + bv * g.dv[2];
  d[0] = g.q[1] * h2 - g.q[2] * h1;
  d[1] = g.q[2] * h0 - g.q[0] * h2;
  d[2] = g.q[0] * h1 - g.q[1] * h0;
  d[3] = directional ? 0.0 : h0;
  d[4] = directional ? 0.0 : h1;
  d[5] = directional ? 0.0 : h2;
}

// The linearisation of one observation: everything the point block, the camera block and the
// Schur product need, from the pose, the camera, the point and the observed pixel.
struct ObsLin {
  double jc[2][6];  // pose Jacobian rows (zero for a fixed camera; no translation for a bearing)
  double jp[2][3];  // point Jacobian rows
  double jf[2];     // d pixel / d log focal scale = pixel - principal point
  double r[2];      // residual: projection - observation
  double w;         // IRLS Huber weight
  double cost;      // robust cost
  double sq;        // squared error
};

// linearizeBundle's per-observation body (bundle.shade.ts:251-297, joint-focal.shade.ts:266-316).
__host__ __device__ inline bool linearize(const double pose[12], const Camera& k, const double X[3],
                                          bool variable, bool directional, double u, double v,
                                          double huber, ObsLin& o) {
  double q[3];
  for (int i = 0; i < 3; i++) {
    q[i] = pose[i * 3] * X[0] + pose[i * 3 + 1] * X[1] + pose[i * 3 + 2] * X[2];
    if (!directional) q[i] += pose[9 + i];
  }
  double pixel[2], du[3], dv[3];
  if (!project(k, q, pixel, du, dv)) return false;
  o.r[0] = pixel[0] - u;
  o.r[1] = pixel[1] - v;
  o.sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
  const double e = sqrt(o.sq);
  o.w = e > huber ? huber / e : 1.0;
  o.cost = robust_cost(e, huber);
  if (variable) {
    pose_row(q, du, o.jc[0]);
    pose_row(q, dv, o.jc[1]);
    if (directional)
      for (int c = 3; c < 6; c++) o.jc[0][c] = o.jc[1][c] = 0;
  } else {
    for (int c = 0; c < 6; c++) o.jc[0][c] = o.jc[1][c] = 0;
  }
  for (int c = 0; c < 3; c++) {
    o.jp[0][c] = du[0] * pose[c] + du[1] * pose[3 + c] + du[2] * pose[6 + c];
    o.jp[1][c] = dv[0] * pose[c] + dv[1] * pose[3 + c] + dv[2] * pose[6 + c];
  }
  o.jf[0] = pixel[0] - k.cx;
  o.jf[1] = pixel[1] - k.cy;
  return true;
}

// The candidate cost of one observation (candidateLane, bundle.shade.ts:1024-1039): 1e30 for
// points beyond 1e9 or projections outside the model's domain.
__host__ __device__ inline void candidate_cost(const double pose[12], const Camera& k, const double X[3],
                                               bool directional, double u, double v, double huber,
                                               double& cost, double& sq) {
  if (!(fmax(fabs(X[0]), fmax(fabs(X[1]), fabs(X[2]))) <= 1e9)) {
    cost = sq = 1e30;
    return;
  }
  double q[3];
  for (int i = 0; i < 3; i++) {
    q[i] = pose[i * 3] * X[0] + pose[i * 3 + 1] * X[1] + pose[i * 3 + 2] * X[2];
    if (!directional) q[i] += pose[9 + i];
  }
  double pixel[2], du[3], dv[3];
  if (!project(k, q, pixel, du, dv)) {
    cost = sq = 1e30;
    return;
  }
  const double x = pixel[0] - u, y = pixel[1] - v;
  sq = x * x + y * y;
  cost = robust_cost(sqrt(sq), huber);
}

}  // namespace tba
