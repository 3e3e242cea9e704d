// TEST INFRASTRUCTURE ONLY — the oracle.  Nothing in the product (typecv_b200/) links, loads or
// calls this file.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
// it, and only as the checker.
//
// A plain C++17 restatement of TypeCV's bundle adjustment, in two parts:
//
//  (1) `oracle_cpu_bundle_adjust`: the reference's CPU bundle adjustment `bundleAdjust`
//      (src/sfm/bundle/bundle-adjustment.ts:80-301, src/sfm/bundle/joint-focal.ts:45-287): point
//      Schur elimination into a dense reduced camera system solved by partial-pivot elimination,
//      with the same loop order, damping, gauge normalisation and LM rule.
//
//  (2) `oracle_gpu_operator`: the semantics of the reference's GPU operator `bundleAdjustGpu`
//      (src/sfm/bundle/gpu/bundle.ts:89-800, joint-focal.ts:78-929) restated serially: the
//      matrix-free Schur product and block-Jacobi PCG of bundle.shade.ts (K1-K20) and
//      joint-focal.shade.ts (K21), resident (one window), with the host's stall monitor.
//      Its output array has the layout of the reference's `packBundleResult`.
//
//  (3) `oracle_linearize_inverse_depth`: the reference's CPU `inverseDepthJacobian`
//      (src/geometry/inverse-depth.ts:38-74, with cameraProjection and radialLimitSquared of
//      src/geometry/camera.ts:15-61) over rows in the device's 34-word layout, written in the
//      device's 23-word layout: the checker and CPU baseline of the inverse-depth linearisation.
//
//  (4) `oracle_evaluate_observations`: the observation-evaluation kernels
//      (src/geometry/gpu/observation-evaluation.shade.ts: projection and threshold, the per-track
//      depth-sensitivity filter, per-64 partials and their sum) over the packed request, as
//      oracle/observations.py restates them in Python: the CPU baseline of that evaluation.
//
// All are compiled with -ffp-contract=off and no FMA so that every product and sum rounds the
// way the reference's JavaScript does.  Parity is pinned by tests/golden (see tests/).  The
// operator's per-point, per-observation and per-camera-row loops run under OpenMP: their
// iterations are independent, so every value is the same as in a serial run.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

const double kInf = std::numeric_limits<double>::infinity();

struct Camera {
  double fx, fy, cx, cy, k1, k2;
};
struct Pose {
  double R[9];
  double t[3];
};

// ---- src/geometry/camera.ts ------------------------------------------------------------------

// radialLimitSquared, src/geometry/camera.ts:15-24.
double radial_limit_squared(double k1, double k2) {
  if (k2 == 0) return k1 < 0 ? -1 / (3 * k1) : kInf;
  const double A = 5 * k2, B = 3 * k1, D = B * B - 4 * A;
  if (D < 0) return kInf;
  const double q = -0.5 * (B + (B >= 0 ? 1 : -1) * std::sqrt(D));
  double best = kInf;
  const double roots[2] = {q / A, 1 / q};
  for (double x : roots)
    if (x > 0 && std::isfinite(x)) best = std::min(best, x);
  return best;
}

// cameraProjection, src/geometry/camera.ts:27-61: pixel and the 2x3 derivative with respect to
// the camera-frame point.  Returns false where the reference returns undefined.
bool camera_projection(const Camera& k, const double q[3], double pixel[2], double jac[6]) {
  const double X = q[0], Y = q[1], Z = q[2];
  if (!(Z > 1e-12) || !std::isfinite(X) || !std::isfinite(Y) || !std::isfinite(Z)) return false;
  const double x = X / Z, y = Y / Z, r2 = x * x + y * y, k1 = k.k1, k2 = k.k2;
  if (r2 >= radial_limit_squared(k1, k2)) return false;
  const double d = 1 + k1 * r2 + k2 * r2 * r2, g = 2 * (k1 + 2 * k2 * r2);
  const double xx = d + g * x * x, xy = g * x * y, yy = d + g * y * y;
  if (!(d > 0 && 1 + 3 * k1 * r2 + 5 * k2 * r2 * r2 > 0)) return false;
  pixel[0] = k.fx * x * d + k.cx;
  pixel[1] = k.fy * y * d + k.cy;
  jac[0] = (k.fx * xx) / Z;
  jac[1] = (k.fx * xy) / Z;
  jac[2] = (-k.fx * (xx * x + xy * y)) / Z;
  jac[3] = (k.fy * xy) / Z;
  jac[4] = (k.fy * yy) / Z;
  jac[5] = (-k.fy * (xy * x + yy * y)) / Z;
  for (int i = 0; i < 2; i++)
    if (!std::isfinite(pixel[i])) return false;
  for (int i = 0; i < 6; i++)
    if (!std::isfinite(jac[i])) return false;
  return true;
}

// ---- src/geometry/pose.ts --------------------------------------------------------------------

// transformPoint, src/geometry/pose.ts:34-39.
void transform_point(const Pose& p, const double X[3], double out[3]) {
  for (int i = 0; i < 3; i++)
    out[i] = p.R[i * 3] * X[0] + p.R[i * 3 + 1] * X[1] + p.R[i * 3 + 2] * X[2] + p.t[i];
}
// cameraCenter, src/geometry/pose.ts:40-45.
void camera_center(const Pose& p, double out[3]) {
  for (int i = 0; i < 3; i++)
    out[i] = -p.R[i] * p.t[0] - p.R[i + 3] * p.t[1] - p.R[i + 6] * p.t[2];
}
// multiply, src/geometry/linear.ts:8-16 (n = 3).
void multiply3(const double* a, const double* b, double* m) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += a[r * 3 + k] * b[k * 3 + c];
      m[r * 3 + c] = s;
    }
}
// rotationExp, src/geometry/pose.ts:46-56.
void rotation_exp(const double* w, double out[9]) {
  const double x = w[0], y = w[1], z = w[2];
  const double theta = std::hypot(x, y, z);
  const double a = theta < 1e-7 ? 1 - (theta * theta) / 6 : std::sin(theta) / theta;
  const double b = theta < 1e-7 ? 0.5 - (theta * theta) / 24 : (1 - std::cos(theta)) / (theta * theta);
  const double W[9] = {0, -z, y, z, 0, -x, -y, x, 0};
  double W2[9];
  multiply3(W, W, W2);
  for (int i = 0; i < 9; i++) out[i] = (i % 4 == 0 ? 1 : 0) + a * W[i] + b * W2[i];
}
// updatePose, src/geometry/pose.ts:58-62: left rotation, additive translation.
Pose update_pose(const Pose& p, const double* delta) {
  double dR[9];
  rotation_exp(delta, dR);
  Pose rot;
  std::memcpy(rot.R, dR, sizeof dR);
  rot.t[0] = rot.t[1] = rot.t[2] = 0;
  double rotated[3];
  transform_point(rot, p.t, rotated);
  Pose out;
  multiply3(dR, p.R, out.R);
  for (int i = 0; i < 3; i++) out.t[i] = rotated[i] + delta[i + 3];
  return out;
}

struct Jacobian {
  double pixel[2];
  double point[6];  // 2x3, row-major
  double pose[12];  // 2x6, row-major: rotation columns then translation columns
};

// observationJacobian, src/geometry/pose.ts:66-88, with the bearing rule of
// bundleObservationJacobian, src/sfm/bundle/bundle-directions.ts:105-114.
bool observation_jacobian(const Camera& camera, const Pose& pose_in, const double X[3],
                          bool directional, Jacobian& out) {
  Pose pose = pose_in;
  if (directional) pose.t[0] = pose.t[1] = pose.t[2] = 0;
  double q[3], J[6];
  transform_point(pose, X, q);
  if (!camera_projection(camera, q, out.pixel, J)) return false;
  const double B[9] = {0, q[2], -q[1], -q[2], 0, q[0], q[1], -q[0], 0};
  std::memset(out.point, 0, sizeof out.point);
  std::memset(out.pose, 0, sizeof out.pose);
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 3; j++) {
      for (int k = 0; k < 3; k++) {
        out.point[i * 3 + j] += J[i * 3 + k] * pose.R[k * 3 + j];
        out.pose[i * 6 + j] += J[i * 3 + k] * B[k * 3 + j];
      }
      out.pose[i * 6 + j + 3] = J[i * 3 + j];
    }
  if (directional)
    for (int at : {3, 4, 5, 9, 10, 11}) out.pose[at] = 0;
  return true;
}

// projectBundlePoint, src/sfm/bundle/bundle-directions.ts:117-124.
bool project_bundle_point(const Camera& camera, const Pose& pose_in, const double X[3],
                          bool directional, double pixel[2]) {
  Pose pose = pose_in;
  if (directional) pose.t[0] = pose.t[1] = pose.t[2] = 0;
  double q[3], J[6];
  transform_point(pose, X, q);
  return camera_projection(camera, q, pixel, J);
}

// ---- src/geometry/numerics.ts ----------------------------------------------------------------

// solveSystem, src/geometry/numerics.ts:71-100: pivoted elimination; false where the reference
// returns undefined.
bool solve_system(const std::vector<double>& matrix, const std::vector<double>& rhs,
                  std::vector<double>& out) {
  const size_t n = rhs.size();
  std::vector<std::vector<double>> a(n, std::vector<double>(n + 1));
  for (size_t i = 0; i < n; i++) {
    for (size_t j = 0; j < n; j++) a[i][j] = matrix[i * n + j];
    a[i][n] = rhs[i];
  }
  for (auto& row : a)
    for (double v : row)
      if (!std::isfinite(v)) return false;
  double scale = 0;
  for (auto& row : a)
    for (size_t j = 0; j < n; j++) scale = std::max(scale, std::fabs(row[j]));
  if (!(scale > 0)) {
    out.assign(n, 0);
    return n == 0;
  }
  for (size_t j = 0; j < n; j++) {
    size_t p = j;
    for (size_t i = j + 1; i < n; i++)
      if (std::fabs(a[i][j]) > std::fabs(a[p][j])) p = i;
    if (std::fabs(a[p][j]) < 1e-14 * scale) return false;
    std::swap(a[p], a[j]);
    for (size_t i = j + 1; i < n; i++) {
      const double f = a[i][j] / a[j][j];
      for (size_t k = j; k <= n; k++) a[i][k] -= f * a[j][k];
    }
  }
  out.assign(n, 0);
  for (size_t ii = n; ii-- > 0;) {
    double b = a[ii][n];
    for (size_t j = ii + 1; j < n; j++) b -= a[ii][j] * out[j];
    out[ii] = b / a[ii][ii];
  }
  for (double v : out)
    if (!std::isfinite(v)) return false;
  return true;
}

// inverse3, src/geometry/numerics.ts:103-131: adjugate inverse.
bool inverse3(const double* a, double out[9]) {
  const double a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[3], a11 = a[4], a12 = a[5], a20 = a[6],
               a21 = a[7], a22 = a[8];
  const double c00 = a11 * a22 - a12 * a21, c01 = a02 * a21 - a01 * a22,
               c02 = a01 * a12 - a02 * a11;
  const double det = a00 * c00 + a10 * c01 + a20 * c02;
  if (!std::isfinite(det) || det == 0) return false;
  out[0] = c00 / det;
  out[1] = c01 / det;
  out[2] = c02 / det;
  out[3] = (a12 * a20 - a10 * a22) / det;
  out[4] = (a00 * a22 - a02 * a20) / det;
  out[5] = (a02 * a10 - a00 * a12) / det;
  out[6] = (a10 * a21 - a11 * a20) / det;
  out[7] = (a01 * a20 - a00 * a21) / det;
  out[8] = (a00 * a11 - a01 * a10) / det;
  for (int i = 0; i < 9; i++)
    if (!std::isfinite(out[i])) return false;
  return true;
}

}  // namespace

extern "C" {

// The problem and options, in the order of the reference's packed arrays
// (src/sfm/bundle/gpu/bundle-host.ts:121-218) and its option names.
typedef struct {
  uint32_t cameras, points, observations, directional_points;
  uint32_t anchor, scale_view;  // camera indices (views order)
  uint32_t iterations, max_cg;
  uint32_t shared_focal;
  uint32_t focal_groups;  // CPU route only: number of focal groups (0 or 1 = one group)
  double huber, cg_tolerance, stall_tolerance;
} oracle_control;

}  // extern "C"

namespace {

// The packed views of the scene array: [poses 12C | points 3P | cameras 6C | pixels 2M] and
// the index array [obsCamera M | obsPoint M | pointStart P+1 | cameraStart C+1 |
// cameraObservations M | cameraActive C] (bundle-host.ts:121-143).
struct Problem {
  uint32_t C, P, M, D;
  std::vector<Pose> poses;
  std::vector<double> points;  // 3P
  std::vector<Camera> cams;
  const double* pixels;
  const uint32_t* obs_camera;
  const uint32_t* obs_point;
  const uint32_t* point_start;
  const uint32_t* camera_start;
  const uint32_t* camera_obs;
  const uint32_t* active;
  Problem(const oracle_control* c, const double* scene, const uint32_t* index)
      : C(c->cameras), P(c->points), M(c->observations), D(c->directional_points) {
    poses.resize(C);
    for (uint32_t i = 0; i < C; i++) {
      std::memcpy(poses[i].R, scene + 12 * i, 9 * sizeof(double));
      std::memcpy(poses[i].t, scene + 12 * i + 9, 3 * sizeof(double));
    }
    points.assign(scene + 12 * C, scene + 12 * C + 3 * P);
    cams.resize(C);
    const double* k = scene + 12 * C + 3 * P;
    for (uint32_t i = 0; i < C; i++)
      cams[i] = Camera{k[6 * i], k[6 * i + 1], k[6 * i + 2], k[6 * i + 3], k[6 * i + 4], k[6 * i + 5]};
    pixels = scene + 18 * size_t(C) + 3 * size_t(P);
    obs_camera = index;
    obs_point = index + M;
    point_start = index + 2 * size_t(M);
    camera_start = point_start + P + 1;
    camera_obs = camera_start + C + 1;
    active = camera_obs + M;
  }
  bool directional(uint32_t p) const { return p >= P - D; }
};

struct Metrics {
  double cost, rmse, squares;
  uint32_t observations;
};

// bundleMetrics, src/sfm/bundle/bundle-shared.ts:32-54.
Metrics bundle_metrics(const Problem& pb, const std::vector<Pose>& poses,
                       const std::vector<Camera>& cams, const std::vector<double>& pts,
                       double huber) {
  double cost = 0, squares = 0;
  uint32_t observations = 0;
  for (uint32_t p = 0; p < pb.P; p++)
    for (uint32_t i = pb.point_start[p]; i < pb.point_start[p + 1]; i++) {
      const uint32_t c = pb.obs_camera[i];
      double pixel[2];
      if (!project_bundle_point(cams[c], poses[c], &pts[3 * p], pb.directional(p), pixel))
        return Metrics{kInf, kInf, kInf, observations};
      const double e = std::hypot(pixel[0] - pb.pixels[2 * i], pixel[1] - pb.pixels[2 * i + 1]);
      cost += e <= huber ? e * e : 2 * huber * e - huber * huber;
      squares += e * e;
      observations++;
    }
  return Metrics{cost, std::sqrt(squares / observations), squares, observations};
}

// normalizeBundlePoint, src/sfm/bundle/bundle-directions.ts:127-138.
void normalize_point(double xyz[3], bool directional, const double origin[3], double s) {
  if (directional) {
    const double norm = std::hypot(xyz[0], xyz[1], xyz[2]);
    for (int j = 0; j < 3; j++) xyz[j] = xyz[j] / norm;
    return;
  }
  for (int j = 0; j < 3; j++) xyz[j] = origin[j] + s * (xyz[j] - origin[j]);
}

}  // namespace

extern "C" {

// Output of both entry points: [poses 12C | points 3P | state 26 | log focal scale |
// fx C | fy C], with the state words of BUNDLE_STATE (gpu/bundle-shared.ts:370-386):
// 2 baseline, 6 final cost, 7 final SSE, 8 initial cost, 9 initial SSE, 10 accepted,
// 11 rejected, 14 input error, 16 CG steps, 17 failed solves, 24/25 initial/final RMSE.
size_t oracle_output_size(uint32_t C, uint32_t P) { return 12 * size_t(C) + 3 * size_t(P) + 27 + 2 * size_t(C); }

// The reference's CPU bundle adjustment (both routes), on a problem whose inputs have already
// passed the host checks of the wrapper (validateReconstruction, gauge, window, connectivity).
// `group_of` gives each camera's dense focal group (shared-focal route; NULL = one group).
// Returns 0, or 2 when an observation does not initially project in front of its camera.
int oracle_cpu_bundle_adjust(const oracle_control* ctl, const double* scene,
                             const uint32_t* index, const uint32_t* group_of, double* output) {
  Problem pb(ctl, scene, index);
  const uint32_t C = pb.C, P = pb.P;
  const double huber = ctl->huber, stall = ctl->stall_tolerance;
  const bool shared = ctl->shared_focal != 0;
  const uint32_t anchor = ctl->anchor, scale_view = ctl->scale_view;
  double* state = output + 12 * size_t(C) + 3 * size_t(P);
  std::memset(output, 0, oracle_output_size(C, P) * sizeof(double));

  double origin[3], scale_center[3];
  camera_center(pb.poses[anchor], origin);
  camera_center(pb.poses[scale_view], scale_center);
  const double baseline = std::hypot(origin[0] - scale_center[0], origin[1] - scale_center[1],
                                     origin[2] - scale_center[2]);
  // The window: the anchor and the cameras outside `variableViewIds` are fixed
  // (bundle-adjustment.ts:137-142; joint-focal.ts:97-106).
  std::vector<int> row_of(C, -1);
  uint32_t active_count = 0, fixed_count = 0;
  for (uint32_t c = 0; c < C; c++) {
    if (pb.active[c]) row_of[c] = int(active_count++);
    else fixed_count++;
  }
  uint32_t groups = 1;
  if (shared && group_of)
    for (uint32_t c = 0; c < C; c++) groups = std::max(groups, group_of[c] + 1);
  const uint32_t focal = active_count * 6;
  const uint32_t n = shared ? focal + groups : active_count * 6;

  std::vector<Pose> poses = pb.poses;
  std::vector<Camera> cams = pb.cams;
  std::vector<double> pts = pb.points;
  const Metrics initial = bundle_metrics(pb, poses, cams, pts, huber);
  Metrics current = initial;
  double lambda = 1e-3;
  uint32_t accepted = 0, rejected = 0;
  int status = 0;
  if (!std::isfinite(initial.cost)) status = 2;

  for (uint32_t iteration = 0; status == 0 && iteration < ctl->iterations; iteration++) {
    std::vector<double> A(size_t(n) * n, 0.0), b(n, 0.0);
    struct Block {
      double V[9], bp[3], inverse[9];
      bool ok;
      std::vector<std::pair<uint32_t, std::vector<double>>> W;  // (row or camera row, cross)
    };
    std::vector<Block> blocks(P);
    for (uint32_t p = 0; p < P; p++) {
      Block& blk = blocks[p];
      std::memset(blk.V, 0, sizeof blk.V);
      std::memset(blk.bp, 0, sizeof blk.bp);
      auto cross_of = [&](uint32_t key, size_t len) -> std::vector<double>& {
        for (auto& kv : blk.W)
          if (kv.first == key) return kv.second;
        blk.W.emplace_back(key, std::vector<double>(len, 0.0));
        return blk.W.back().second;
      };
      for (uint32_t i = pb.point_start[p]; i < pb.point_start[p + 1]; i++) {
        const uint32_t c = pb.obs_camera[i];
        Jacobian jac;
        observation_jacobian(cams[c], poses[c], &pts[3 * p], pb.directional(p), jac);
        const double r[2] = {jac.pixel[0] - pb.pixels[2 * i], jac.pixel[1] - pb.pixels[2 * i + 1]};
        const double norm = std::hypot(r[0], r[1]);
        const double w = norm <= huber ? 1 : huber / norm;
        if (!shared) {
          // bundle-adjustment.ts:153-186.
          const int ci = row_of[c];
          std::vector<double>* cross = nullptr;
          if (ci >= 0) cross = &cross_of(uint32_t(ci), 18);
          for (int row = 0; row < 2; row++) {
            for (int k = 0; k < 3; k++) {
              blk.bp[k] -= w * jac.point[row * 3 + k] * r[row];
              for (int l = 0; l < 3; l++)
                blk.V[k * 3 + l] += w * jac.point[row * 3 + k] * jac.point[row * 3 + l];
            }
            if (ci >= 0)
              for (int k = 0; k < 6; k++) {
                const size_t ii = size_t(ci) * 6 + k;
                b[ii] -= w * jac.pose[row * 6 + k] * r[row];
                for (int l = 0; l < 6; l++)
                  A[ii * n + size_t(ci) * 6 + l] += w * jac.pose[row * 6 + k] * jac.pose[row * 6 + l];
                for (int l = 0; l < 3; l++)
                  (*cross)[k * 3 + l] += w * jac.pose[row * 6 + k] * jac.point[row * 3 + l];
              }
          }
        } else {
          // joint-focal.ts:131-168.
          const int base = row_of[c];
          const uint32_t focal_row = focal + (group_of ? group_of[c] : 0);
          uint32_t rows[7];
          int nrows = 0;
          if (base >= 0)
            for (int k = 0; k < 6; k++) rows[nrows++] = uint32_t(base) * 6 + k;
          rows[nrows++] = focal_row;
          for (int k = 0; k < nrows; k++) cross_of(rows[k], 3);
          for (int axis = 0; axis < 2; axis++) {
            double J[7];
            for (int k = 0; k < nrows; k++)
              J[k] = rows[k] == focal_row
                         ? jac.pixel[axis] - (axis == 0 ? cams[c].cx : cams[c].cy)
                         : jac.pose[axis * 6 + (rows[k] - uint32_t(base) * 6)];
            for (int k = 0; k < 3; k++) {
              blk.bp[k] -= w * jac.point[axis * 3 + k] * r[axis];
              for (int l = 0; l < 3; l++)
                blk.V[k * 3 + l] += w * jac.point[axis * 3 + k] * jac.point[axis * 3 + l];
            }
            for (int k = 0; k < nrows; k++) {
              const uint32_t row = rows[k];
              std::vector<double>& Wi = cross_of(row, 3);
              b[row] -= w * J[k] * r[axis];
              for (int l = 0; l < nrows; l++) A[size_t(row) * n + rows[l]] += w * J[k] * J[l];
              for (int l = 0; l < 3; l++) Wi[l] += w * J[k] * jac.point[axis * 3 + l];
            }
          }
        }
      }
      for (int k = 0; k < 3; k++) blk.V[k * 3 + k] += lambda * std::max(blk.V[k * 3 + k], 1e-10);
      blk.ok = inverse3(blk.V, blk.inverse);
    }
    bool all_ok = true;
    for (auto& blk : blocks) all_ok = all_ok && blk.ok;
    if (!all_ok) {
      lambda *= 10;
      rejected++;
      continue;
    }
    for (uint32_t k = 0; k < n; k++) A[size_t(k) * n + k] += lambda * std::max(A[size_t(k) * n + k], 1e-10);
    for (auto& blk : blocks) {
      if (!shared) {
        // bundle-adjustment.ts:196-217: S = A - W V^-1 W^T, b -= W V^-1 b_p.
        std::vector<std::vector<double>> temp;
        for (auto& kv : blk.W) {
          const uint32_t ci = kv.first;
          const std::vector<double>& W = kv.second;
          std::vector<double> T(18, 0.0);
          for (int i = 0; i < 6; i++)
            for (int j = 0; j < 3; j++)
              for (int k = 0; k < 3; k++) T[i * 3 + j] += W[i * 3 + k] * blk.inverse[k * 3 + j];
          for (int i = 0; i < 6; i++)
            for (int k = 0; k < 3; k++) b[ci * 6 + i] -= T[i * 3 + k] * blk.bp[k];
          temp.push_back(T);
        }
        for (size_t a = 0; a < blk.W.size(); a++) {
          const uint32_t ci = blk.W[a].first;
          const std::vector<double>& T = temp[a];
          for (auto& kv : blk.W) {
            const uint32_t cj = kv.first;
            const std::vector<double>& W = kv.second;
            for (int i = 0; i < 6; i++)
              for (int j = 0; j < 6; j++) {
                double value = 0;
                for (int k = 0; k < 3; k++) value += T[i * 3 + k] * W[j * 3 + k];
                A[(size_t(ci) * 6 + i) * n + cj * 6 + j] -= value;
              }
          }
        }
      } else {
        // joint-focal.ts:179-191.
        std::vector<std::vector<double>> temp;
        for (auto& kv : blk.W) {
          const uint32_t row = kv.first;
          const std::vector<double>& W = kv.second;
          std::vector<double> t(3, 0.0);
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) t[i] += W[j] * blk.inverse[j * 3 + i];
          for (int i = 0; i < 3; i++) b[row] -= t[i] * blk.bp[i];
          temp.push_back(t);
        }
        for (size_t a = 0; a < blk.W.size(); a++) {
          const uint32_t row = blk.W[a].first;
          for (auto& kv : blk.W)
            for (int i = 0; i < 3; i++) A[size_t(row) * n + kv.first] -= temp[a][i] * kv.second[i];
        }
      }
    }
    std::vector<double> delta;
    if (!solve_system(A, b, delta)) {
      lambda *= 10;
      rejected++;
      continue;
    }
    std::vector<Pose> new_poses = poses;
    std::vector<Camera> new_cams = cams;
    if (shared) {
      // joint-focal.ts:198-216.
      std::vector<double> scales(groups);
      bool ok = true;
      for (uint32_t g = 0; g < groups; g++) {
        scales[g] = std::exp(delta[focal + g]);
        if (!std::isfinite(scales[g]) || scales[g] <= 0) ok = false;
      }
      if (!ok) {
        lambda *= 10;
        rejected++;
        continue;
      }
      for (uint32_t c = 0; c < C; c++) {
        const double s = scales[group_of ? group_of[c] : 0];
        new_cams[c].fx = cams[c].fx * s;
        new_cams[c].fy = cams[c].fy * s;
      }
    }
    for (uint32_t c = 0; c < C; c++)
      if (row_of[c] >= 0) new_poses[c] = update_pose(poses[c], &delta[size_t(row_of[c]) * 6]);
    std::vector<double> new_pts = pts;
    for (uint32_t p = 0; p < P; p++) {
      const Block& blk = blocks[p];
      double rhs[3] = {blk.bp[0], blk.bp[1], blk.bp[2]};
      if (!shared) {
        // bundle-adjustment.ts:230-240.
        for (auto& kv : blk.W)
          for (int j = 0; j < 3; j++)
            for (int k = 0; k < 6; k++) rhs[j] -= kv.second[k * 3 + j] * delta[kv.first * 6 + k];
      } else {
        for (auto& kv : blk.W)
          for (int j = 0; j < 3; j++) rhs[j] -= kv.second[j] * delta[kv.first];
      }
      for (int j = 0; j < 3; j++) {
        double dp = 0;
        for (int k = 0; k < 3; k++) dp = dp + blk.inverse[j * 3 + k] * rhs[k];
        new_pts[3 * p + j] = pts[3 * p + j] + dp;
      }
    }
    double center[3];
    camera_center(new_poses[scale_view], center);
    const double new_baseline =
        std::hypot(origin[0] - center[0], origin[1] - center[1], origin[2] - center[2]);
    bool bad = !(new_baseline > 1e-12);
    if (shared)
      for (uint32_t c = 0; c < C; c++)
        if (!std::isfinite(new_cams[c].fx) || !std::isfinite(new_cams[c].fy) ||
            new_cams[c].fx <= 0 || new_cams[c].fy <= 0)
          bad = true;
    if (bad) {
      lambda *= 10;
      rejected++;
      continue;
    }
    const double s = fixed_count == 1 ? baseline / new_baseline : 1;
    // Similarity normalisation about the anchor centre (bundle-adjustment.ts:248-260).
    for (uint32_t c = 0; c < C; c++) {
      if (c == anchor) continue;
      Pose rot = new_poses[c];
      rot.t[0] = rot.t[1] = rot.t[2] = 0;
      double ro[3];
      transform_point(rot, origin, ro);
      for (int i = 0; i < 3; i++) new_poses[c].t[i] = s * new_poses[c].t[i] + (s - 1) * ro[i];
    }
    for (uint32_t p = 0; p < P; p++) normalize_point(&new_pts[3 * p], pb.directional(p), origin, s);
    const Metrics next = bundle_metrics(pb, new_poses, new_cams, new_pts, huber);
    if (next.cost < current.cost) {
      const double improvement = current.cost - next.cost;
      poses = new_poses;
      cams = new_cams;
      pts = new_pts;
      current = next;
      lambda = std::max(1e-10, lambda / 3);
      accepted++;
      // bundleStalled, bundle-shared.ts:19-21.
      if (improvement < stall * std::max(1.0, current.cost)) break;
    } else {
      lambda *= 10;
      rejected++;
      if (lambda > 1e12) break;
    }
  }
  for (uint32_t c = 0; c < C; c++) {
    std::memcpy(output + 12 * c, poses[c].R, 9 * sizeof(double));
    std::memcpy(output + 12 * c + 9, poses[c].t, 3 * sizeof(double));
    output[12 * size_t(C) + 3 * size_t(P) + 27 + c] = cams[c].fx;
    output[12 * size_t(C) + 3 * size_t(P) + 27 + C + c] = cams[c].fy;
  }
  std::memcpy(output + 12 * size_t(C), pts.data(), 3 * size_t(P) * sizeof(double));
  state[2] = baseline;
  state[6] = current.cost;
  state[7] = current.squares;
  state[8] = initial.cost;
  state[9] = initial.squares;
  state[10] = accepted;
  state[11] = rejected;
  state[14] = status;
  state[24] = initial.rmse;
  state[25] = current.rmse;
  return status;
}

}  // extern "C"

// =================================================================================================
// (2) The GPU operator's semantics, serial.  Arrays and state words as in bundle.shade.ts and
// joint-focal.shade.ts; resident (one window, no streaming); the 'rows' camera assembly and the
// serial camera product.
// =================================================================================================

namespace {

// project + radialLimit, src/device/gpu/numerics.shade.ts:79-99, 141-173.
double op_radial_limit(const Camera& k) {
  if (k.k2 == 0) return k.k1 < 0 ? -1 / (3 * k.k1) : 1e30;
  const double a = 5 * k.k2, b = 3 * k.k1, d = b * b - 4 * a;
  if (d < 0) return 1e30;
  const double sign = b < 0 ? -1 : 1;
  const double q = -0.5 * (b + sign * std::sqrt(d));
  double limit = 1e30;
  const double first = q / a;
  if (first > 0) limit = std::min(limit, first);
  if (q != 0) {
    const double second = 1 / q;
    if (second > 0) limit = std::min(limit, second);
  }
  return limit;
}
struct Projection {
  double pixel[2], du[3], dv[3];
  bool ok;
};
Projection op_project(const Camera& k, const double q[3]) {
  Projection out{};
  out.ok = false;
  if (!(q[2] > 1e-12)) return out;
  const double x = q[0] / q[2], y = q[1] / q[2], r2 = x * x + y * y;
  if (!(r2 < op_radial_limit(k) && r2 < 1e8)) return out;
  const double d = 1 + k.k1 * r2 + k.k2 * r2 * r2, g = 2 * (k.k1 + 2 * k.k2 * r2);
  if (!(d > 0 && 1 + 3 * k.k1 * r2 + 5 * k.k2 * r2 * r2 > 0)) return out;
  const double xx = d + g * x * x, xy = g * x * y, yy = d + g * y * y;
  out.pixel[0] = k.fx * x * d + k.cx;
  out.pixel[1] = k.fy * y * d + k.cy;
  out.du[0] = (k.fx * xx) / q[2];
  out.du[1] = (k.fx * xy) / q[2];
  out.du[2] = (-k.fx * (xx * x + xy * y)) / q[2];
  out.dv[0] = (k.fy * xy) / q[2];
  out.dv[1] = (k.fy * yy) / q[2];
  out.dv[2] = (-k.fy * (xy * x + yy * y)) / q[2];
  const double mp = std::max(std::fabs(out.pixel[0]), std::fabs(out.pixel[1]));
  const double mu = std::max(std::max(std::fabs(out.du[0]), std::fabs(out.du[1])), std::fabs(out.du[2]));
  const double mv = std::max(std::max(std::fabs(out.dv[0]), std::fabs(out.dv[1])), std::fabs(out.dv[2]));
  if (!(mp < 1e12 && mu < 1e12 && mv < 1e12)) return out;
  out.ok = true;
  return out;
}
// poseRow, numerics.shade.ts:181-183.
void op_pose_row(const double q[3], const double j[3], double out[6]) {
  out[0] = j[2] * q[1] - j[1] * q[2];
  out[1] = j[0] * q[2] - j[2] * q[0];
  out[2] = j[1] * q[0] - j[0] * q[1];
  out[3] = j[0];
  out[4] = j[1];
  out[5] = j[2];
}
// robustCost, numerics.shade.ts:184-187.
double op_robust(double e, double h) { return e <= h ? e * e : 2 * h * e - h * h; }
// solve3, numerics.shade.ts:25-45: equilibrated 3x3 Cholesky.
bool op_solve3(const double a[9], const double b[3], double x[3]) {
  if (!(std::min(a[0], std::min(a[4], a[8])) > 0)) return false;
  const double d0 = 1 / std::sqrt(a[0]), d1 = 1 / std::sqrt(a[4]), d2 = 1 / std::sqrt(a[8]);
  const double l10 = a[3] * d0 * d1, l20 = a[6] * d0 * d2;
  const double pivot1 = 1 - l10 * l10;
  if (!(pivot1 > 1e-14)) return false;
  const double l11 = std::sqrt(pivot1), l21 = (a[7] * d1 * d2 - l20 * l10) / l11;
  const double pivot2 = 1 - l20 * l20 - l21 * l21;
  if (!(pivot2 > 1e-14)) return false;
  const double l22 = std::sqrt(pivot2), y0 = b[0] * d0;
  const double y1 = (b[1] * d1 - l10 * y0) / l11, y2 = (b[2] * d2 - l20 * y0 - l21 * y1) / l22;
  const double x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = y0 - l10 * x1 - l20 * x2;
  x[0] = x0 * d0;
  x[1] = x1 * d1;
  x[2] = x2 * d2;
  return true;
}
// solve6, numerics.shade.ts:221-253: equilibrated 6x6 Cholesky.
bool op_solve6(const double m[36], const double rhs[6], double values[6]) {
  double L[36] = {0}, scale[6];
  for (int i = 0; i < 6; i++) values[i] = 0;
  for (int i = 0; i < 6; i++) {
    if (!(m[i * 6 + i] > 0)) return false;
    scale[i] = 1 / std::sqrt(m[i * 6 + i]);
  }
  for (int i = 0; i < 6; i++) {
    for (int j = 0; j <= i; j++) {
      double value = m[i * 6 + j] * scale[i] * scale[j];
      for (int k = 0; k < j; k++) value -= L[i * 6 + k] * L[j * 6 + k];
      if (i == j) {
        if (!(value > 1e-14)) return false;
        L[i * 6 + j] = std::sqrt(value);
      } else {
        L[i * 6 + j] = value / L[j * 6 + j];
      }
    }
    double v = rhs[i] * scale[i];
    for (int j = 0; j < i; j++) v -= L[i * 6 + j] * values[j];
    values[i] = v / L[i * 6 + i];
  }
  for (int i = 5; i >= 0; i--) {
    double v = values[i];
    for (int j = i + 1; j < 6; j++) v -= L[j * 6 + i] * values[j];
    values[i] = v / L[i * 6 + i];
  }
  for (int i = 0; i < 6; i++) values[i] *= scale[i];
  return true;
}
// movePose, numerics.shade.ts:254-281.
void op_move_pose(const double p[12], const double delta[6], double out[12]) {
  const double x = delta[0], y = delta[1], z = delta[2];
  const double theta = std::sqrt(x * x + y * y + z * z);
  double a = 1 - (theta * theta) / 6, b = 0.5 - (theta * theta) / 24;
  if (theta >= 1e-7) {
    a = std::sin(theta) / theta;
    b = (1 - std::cos(theta)) / (theta * theta);
  }
  const double W[9] = {0, -z, y, z, 0, -x, -y, x, 0};
  double dR[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 12; i++) out[i] = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dR[i * 3 + j] += a * W[i * 3 + j];
      for (int k = 0; k < 3; k++) dR[i * 3 + j] += b * W[i * 3 + k] * W[k * 3 + j];
    }
  for (int i = 0; i < 3; i++) {
    out[9 + i] = delta[3 + i];
    for (int k = 0; k < 3; k++) {
      out[9 + i] += dR[i * 3 + k] * p[9 + k];
      for (int j = 0; j < 3; j++) out[i * 3 + j] += dR[i * 3 + k] * p[k * 3 + j];
    }
  }
}
// focalScale, joint-focal.shade.ts:110-120: exp by range reduction and a Taylor series.
double op_focal_scale(double log_scale) {
  double x = log_scale;
  unsigned squarings = 0;
  for (int j = 0; j < 12; j++)
    if (std::fabs(x) > 0.25) {
      x *= 0.5;
      squarings++;
    }
  double value = 1, term = 1;
  for (int j = 1; j <= 20; j++) {
    term *= x / double(float(j));
    value += term;
  }
  for (unsigned j = 0; j < squarings; j++) value *= value;
  return value;
}

struct Operator {
  const Problem& pb;
  const oracle_control& ctl;
  const bool shared;
  const uint32_t C, P, M, m;  // m: unknowns of the reduced system (6C, +1 with the focal)
  double state[26];
  std::vector<double> scene_pose, scene_point, trial_pose, trial_point;
  std::vector<double> obs;     // 24 per observation (bundle.shade.ts blocks layout)
  std::vector<double> cross;   // 18 or 21 per observation
  std::vector<double> pointb;  // 13 per point
  std::vector<double> camA, camInv, camRhs, camS;  // 36, 36, 6, 36 per camera
  std::vector<double> focal;   // 6C direct H_cf, then 6 scalars, then Jf 2 per observation
  std::vector<double> vec;     // x r p Sp z (m each), y 3P
  Operator(const Problem& p, const oracle_control& c)
      : pb(p), ctl(c), shared(c.shared_focal != 0), C(p.C), P(p.P), M(p.M),
        m(6 * p.C + (c.shared_focal ? 1 : 0)) {
    std::memset(state, 0, sizeof state);
    scene_pose.resize(12 * size_t(C));
    for (uint32_t i = 0; i < C; i++) {
      std::memcpy(&scene_pose[12 * i], p.poses[i].R, 9 * sizeof(double));
      std::memcpy(&scene_pose[12 * i + 9], p.poses[i].t, 3 * sizeof(double));
    }
    scene_point = p.points;
    trial_pose.assign(12 * size_t(C), 0);
    trial_point.assign(3 * size_t(P), 0);
    obs.assign(24 * size_t(M), 0);
    cross.assign((shared ? 21 : 18) * size_t(M), 0);
    pointb.assign(13 * size_t(P), 0);
    camA.assign(36 * size_t(C), 0);
    camInv.assign(36 * size_t(C), 0);
    camRhs.assign(6 * size_t(C), 0);
    camS.assign(36 * size_t(C), 0);
    focal.assign(6 * size_t(C) + 6 + 2 * size_t(M), 0);
    vec.assign(5 * size_t(m) + 3 * size_t(P), 0);
  }
  size_t W() const { return shared ? 21 : 18; }
  double* x() { return &vec[0]; }
  double* r() { return &vec[m]; }
  double* p() { return &vec[2 * size_t(m)]; }
  double* Sp() { return &vec[3 * size_t(m)]; }
  double* z() { return &vec[4 * size_t(m)]; }
  double* y() { return &vec[5 * size_t(m)]; }
  bool variable(uint32_t c) const { return pb.active[c] != 0; }
  Camera camera_at(uint32_t c, bool candidate) const {
    Camera k = pb.cams[c];
    if (shared) {
      const double s = op_focal_scale(focal[6 * size_t(C) + (candidate ? 4 : 3)]);
      k.fx = k.fx * s;
      k.fy = k.fy * s;
    }
    return k;
  }
  const double* pose_at(uint32_t c, bool candidate) const {
    return candidate ? &trial_pose[12 * c] : &scene_pose[12 * c];
  }
  const double* point_at(uint32_t p_, bool candidate) const {
    return candidate ? &trial_point[3 * p_] : &scene_point[3 * p_];
  }
  void observed_point(const double* pose, const double* X, uint32_t point, double q[3]) const {
    // observedPoint, bundle.shade.ts:99-107: a bearing ignores the translation.
    const bool dir = pb.directional(point);
    for (int i = 0; i < 3; i++) {
      const double rx = pose[i * 3] * X[0] + pose[i * 3 + 1] * X[1] + pose[i * 3 + 2] * X[2];
      q[i] = dir ? rx : rx + pose[9 + i];
    }
  }
  void center(uint32_t c, bool candidate, double out[3]) const {
    const double* p_ = pose_at(c, candidate);
    out[0] = -p_[0] * p_[9] - p_[3] * p_[10] - p_[6] * p_[11];
    out[1] = -p_[1] * p_[9] - p_[4] * p_[10] - p_[7] * p_[11];
    out[2] = -p_[2] * p_[9] - p_[5] * p_[10] - p_[8] * p_[11];
  }

  // initializeBundle, bundle.shade.ts:235-250 (joint-focal.shade.ts:248-265).
  void initialize() {
    for (double& s : state) s = 0;
    state[0] = 1e-3;
    if (shared) focal[6 * size_t(C) + 3] = focal[6 * size_t(C) + 4] = 0;
    state[1] = 1;
    double o[3], s[3];
    center(ctl.anchor, false, o);
    center(ctl.scale_view, false, s);
    const double baseline = std::sqrt((o[0] - s[0]) * (o[0] - s[0]) + (o[1] - s[1]) * (o[1] - s[1]) +
                                      (o[2] - s[2]) * (o[2] - s[2]));
    state[2] = baseline;
    state[3] = o[0];
    state[4] = o[1];
    state[5] = o[2];
    if (!(baseline > 1e-10)) {
      state[14] = 1;
      state[1] = 0;
    }
  }
  // metricLane + bundleMetricPartials/finishBundleMetrics, bundle.shade.ts:300-377.
  void metrics() {
    if (state[14] != 0) return;
    double cost = 0, squares = 0, invalid = 0;
    for (uint32_t b = 0; b < (M + 63) / 64; b++) {
      double bc = 0, bs = 0, bi = 0;
      for (uint32_t i = b * 64; i < std::min(M, b * 64 + 64); i++) {
        const uint32_t c = pb.obs_camera[i], pt = pb.obs_point[i];
        double q[3];
        observed_point(pose_at(c, false), point_at(pt, false), pt, q);
        const Projection pr = op_project(camera_at(c, false), q);
        if (!pr.ok) {
          bi += 1;
          continue;
        }
        const double ru = pr.pixel[0] - pb.pixels[2 * i], rv = pr.pixel[1] - pb.pixels[2 * i + 1];
        const double sq = ru * ru + rv * rv;
        bc += op_robust(std::sqrt(sq), ctl.huber);
        bs += sq;
      }
      cost += bc;
      squares += bs;
      invalid += bi;
    }
    if (invalid > 0) {
      state[14] = 2;
      state[1] = 0;
      return;
    }
    state[6] = state[8] = cost;
    state[7] = state[9] = squares;
    if (cost < 1e-20) state[1] = 0;
  }
  // linearizeBundle, bundle.shade.ts:251-297 (joint-focal.shade.ts:266-316).
  void linearize() {
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < M; i++) {
      const uint32_t c = pb.obs_camera[i], pt = pb.obs_point[i];
      const double* pose = pose_at(c, false);
      double q[3];
      observed_point(pose, point_at(pt, false), pt, q);
      const Camera k = camera_at(c, false);
      const Projection pr = op_project(k, q);
      double* b = &obs[24 * size_t(i)];
      for (int j = 0; j < 24; j++) b[j] = 0;
      if (!pr.ok) {
        b[23] = 1;
        continue;
      }
      const double ru = pr.pixel[0] - pb.pixels[2 * i], rv = pr.pixel[1] - pb.pixels[2 * i + 1];
      const double squared = ru * ru + rv * rv, error = std::sqrt(squared);
      double weight = 1;
      if (error > ctl.huber) weight = ctl.huber / error;
      if (variable(c)) {
        double ju[6], jv[6];
        op_pose_row(q, pr.du, ju);
        op_pose_row(q, pr.dv, jv);
        for (int kk = 0; kk < 6; kk++)
          if (kk < 3 || !pb.directional(pt)) {
            b[kk] = ju[kk];
            b[6 + kk] = jv[kk];
          }
      }
      for (int kk = 0; kk < 3; kk++) {
        b[12 + kk] = pr.du[0] * pose[kk] + pr.du[1] * pose[3 + kk] + pr.du[2] * pose[6 + kk];
        b[15 + kk] = pr.dv[0] * pose[kk] + pr.dv[1] * pose[3 + kk] + pr.dv[2] * pose[6 + kk];
      }
      if (shared) {
        focal[6 * size_t(C) + 6 + 2 * size_t(i)] = pr.pixel[0] - k.cx;
        focal[6 * size_t(C) + 6 + 2 * size_t(i) + 1] = pr.pixel[1] - k.cy;
      }
      b[18] = ru;
      b[19] = rv;
      b[20] = weight;
      b[21] = op_robust(error, ctl.huber);
      b[22] = squared;
    }
  }
  const double* jf(uint32_t i) const { return &focal[6 * size_t(C) + 6 + 2 * size_t(i)]; }
  // bundlePointBlocks, bundle.shade.ts:378-422 (joint-focal.shade.ts:403-461).
  void point_blocks() {
#pragma omp parallel for schedule(static)
    for (uint32_t pt = 0; pt < P; pt++) {
      double V[9] = {0}, rhs[3] = {0};
      double* at = &pointb[13 * size_t(pt)];
      for (int j = 0; j < 13; j++) at[j] = 0;
      bool bad = false;
      for (uint32_t i = pb.point_start[pt]; i < pb.point_start[pt + 1]; i++) {
        const double* b = &obs[24 * size_t(i)];
        const double w = b[20];
        double* cr = &cross[W() * i];
        const bool act = variable(pb.obs_camera[i]);
        if (b[23] != 0) {
          bad = true;
          break;
        }
        for (size_t j = 0; j < W(); j++) cr[j] = 0;
        for (int row = 0; row < 2; row++)
          for (int j = 0; j < 3; j++) {
            const double g = b[12 + row * 3 + j];
            rhs[j] -= w * g * b[18 + row];
            for (int k = 0; k < 3; k++) V[j * 3 + k] += w * g * b[12 + row * 3 + k];
            if (shared) cr[18 + j] += w * jf(i)[row] * g;
            if (act)
              for (int k = 0; k < 6; k++) cr[k * 3 + j] += w * b[row * 6 + k] * g;
          }
      }
      if (bad) continue;
      for (int j = 0; j < 3; j++) V[j * 3 + j] += state[0] * std::max(V[j * 3 + j], 1e-10);
      bool ok = true;
      for (int column = 0; column < 3 && ok; column++) {
        double e[3] = {0, 0, 0}, s[3];
        e[column] = 1;
        if (!op_solve3(V, e, s)) {
          ok = false;
          break;
        }
        at[column] = s[0];
        at[3 + column] = s[1];
        at[6 + column] = s[2];
        at[9 + column] = rhs[column];
      }
      if (!ok) continue;
      for (int j = 0; j < 3; j++)
        for (int k = j + 1; k < 3; k++) {
          const double v = (at[j * 3 + k] + at[k * 3 + j]) * 0.5;
          at[j * 3 + k] = v;
          at[k * 3 + j] = v;
        }
      at[12] = 1;
    }
  }
  // bundleCameraRows, bundle.shade.ts:497-555, with invertBundleCameraColumns and
  // finalizeBundleCameraInverse, bundle.shade.ts:655-694.
  void camera_rows() {
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t c = 0; c < C; c++)
      for (int j = 0; j < 6; j++) {
        double aRow[6] = {0}, sRow[6] = {0}, rhs = 0;
        if (!variable(c)) {
          aRow[j] = 1;
          sRow[j] = 1;
        } else {
          for (uint32_t kk = pb.camera_start[c]; kk < pb.camera_start[c + 1]; kk++) {
            const uint32_t i = pb.camera_obs[kk], pt = pb.obs_point[i];
            const double* point = &pointb[13 * size_t(pt)];
            const double* b = &obs[24 * size_t(i)];
            const double* cr = &cross[W() * i];
            const double w = b[20];
            double T[3] = {0, 0, 0};
            for (int orow = 0; orow < 2; orow++) {
              const double value = b[orow * 6 + j];
              rhs -= w * value * b[18 + orow];
              for (int l = 0; l < 6; l++) aRow[l] += w * value * b[orow * 6 + l];
            }
            for (int l = 0; l < 3; l++)
              for (int rr = 0; rr < 3; rr++) T[l] += cr[j * 3 + rr] * point[rr * 3 + l];
            for (int l = 0; l < 3; l++) rhs -= T[l] * point[9 + l];
            for (int l = 0; l < 6; l++)
              for (int rr = 0; rr < 3; rr++) sRow[l] -= T[rr] * cr[l * 3 + rr];
          }
          aRow[j] += state[0] * std::max(aRow[j], 1e-10);
          for (int l = 0; l < 6; l++) sRow[l] += aRow[l];
        }
        for (int l = 0; l < 6; l++) {
          camA[36 * size_t(c) + j * 6 + l] = aRow[l];
          camS[36 * size_t(c) + j * 6 + l] = sRow[l];
        }
        camRhs[6 * size_t(c) + j] = rhs;
      }
#pragma omp parallel for schedule(static)
    for (uint32_t c = 0; c < C; c++) {
      double* inv = &camInv[36 * size_t(c)];
      for (int column = 0; column < 6; column++) {
        double e[6] = {0, 0, 0, 0, 0, 0}, s[6];
        e[column] = 1;
        if (!op_solve6(&camS[36 * size_t(c)], e, s)) {
          inv[column * 6 + column] = -1;
          continue;
        }
        for (int row = 0; row < 6; row++) inv[row * 6 + column] = s[row];
      }
      bool failed = false;
      for (int j = 0; j < 6; j++)
        if (inv[j * 6 + j] < 0) failed = true;
      if (failed) {
        inv[0] = -1;
        continue;
      }
      for (int j = 0; j < 6; j++)
        for (int k = j + 1; k < 6; k++) {
          const double v = (inv[j * 6 + k] + inv[k * 6 + j]) * 0.5;
          inv[j * 6 + k] = v;
          inv[k * 6 + j] = v;
        }
    }
  }
  // bundleFocalCameraRows, bundleFocalObservations, dampBundleFocal, bundleFocalPoints,
  // joint-focal.shade.ts:1138-1205.
  void focal_terms() {
    const size_t n = 6 * size_t(C);
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t c = 0; c < C; c++)
      for (int j = 0; j < 6; j++) {
        double value = 0;
        if (variable(c))
          for (uint32_t kk = pb.camera_start[c]; kk < pb.camera_start[c + 1]; kk++) {
            const uint32_t i = pb.camera_obs[kk];
            const double* b = &obs[24 * size_t(i)];
            value += b[20] * (b[j] * jf(i)[0] + b[6 + j] * jf(i)[1]);
          }
        focal[6 * c + j] = value;
      }
    double diagonal = 0, rhs = 0;
    for (uint32_t i = 0; i < M; i++) {
      const double* b = &obs[24 * size_t(i)];
      const double u = jf(i)[0], v = jf(i)[1], w = b[20];
      diagonal += w * (u * u + v * v);
      rhs -= w * (u * b[18] + v * b[19]);
    }
    diagonal += state[0] * std::max(diagonal, 1e-10);
    focal[n] = diagonal;
    for (uint32_t pt = 0; pt < P; pt++) {
      const double* at = &pointb[13 * size_t(pt)];
      double cr[3] = {0, 0, 0};
      for (uint32_t i = pb.point_start[pt]; i < pb.point_start[pt + 1]; i++)
        for (int j = 0; j < 3; j++) cr[j] += cross[W() * i + 18 + j];
      for (int j = 0; j < 3; j++) {
        double t = 0;
        for (int k = 0; k < 3; k++) t += cr[k] * at[k * 3 + j];
        diagonal -= t * cr[j];
        rhs -= t * at[9 + j];
      }
    }
    focal[n + 5] = diagonal;
    focal[n + 2] = rhs;
    focal[n + 1] = -1;
    if (diagonal > 0) focal[n + 1] = 1 / diagonal;
  }
  double precondition(uint32_t i) {
    if (shared && i == m - 1) return focal[6 * size_t(C) + 1] * r()[i];
    const uint32_t c = i / 6, j = i % 6;
    double zz = 0;
    for (int k = 0; k < 6; k++) zz += camInv[36 * size_t(c) + j * 6 + k] * r()[c * 6 + k];
    return zz;
  }
  // initializeBundleCg, bundle.shade.ts:695-741 (joint-focal.shade.ts:632-682).
  void init_cg() {
    for (int j = 18; j < 26; j++) state[j] = 0;
    if (state[1] == 0) return;
    for (uint32_t pt = 0; pt < P; pt++)
      if (pointb[13 * size_t(pt) + 12] == 0) {
        state[20] = 1;
        return;
      }
    double rho = 0, residual = 0;
    for (uint32_t c = 0; c < C; c++) {
      const double* inv = &camInv[36 * size_t(c)];
      const double* rhs = &camRhs[6 * size_t(c)];
      if (!(inv[0] > 0)) {
        state[20] = 1;
        return;
      }
      for (int j = 0; j < 6; j++) {
        const uint32_t i = c * 6 + j;
        const double rr = rhs[j];
        double zz = 0;
        for (int k = 0; k < 6; k++) zz += inv[j * 6 + k] * rhs[k];
        x()[i] = 0;
        r()[i] = rr;
        p()[i] = zz;
        z()[i] = zz;
        rho += rr * zz;
        residual += rr * rr;
      }
    }
    if (shared) {
      const size_t f = m - 1;
      const double rr = focal[f + 2], zz = focal[f + 1] * rr;
      if (!(focal[f + 1] > 0)) {
        state[20] = 1;
        return;
      }
      x()[f] = 0;
      r()[f] = rr;
      p()[f] = zz;
      z()[f] = zz;
      rho += rr * zz;
      residual += rr * rr;
    }
    state[18] = rho;
    state[21] = residual;
    state[22] = residual;
    if (residual > 0 && rho > 0) state[19] = 1;
    else if (residual > 1e-24) state[20] = 1;
  }
  // bundleSchurPoint + bundleSchurCamera (rows), bundle.shade.ts:185-225,
  // joint-focal.shade.ts:197-253.
  void schur_product() {
#pragma omp parallel for schedule(static)
    for (uint32_t pt = 0; pt < P; pt++) {
      const double* at = &pointb[13 * size_t(pt)];
      double rhs[3] = {0, 0, 0};
      for (uint32_t i = pb.point_start[pt]; i < pb.point_start[pt + 1]; i++) {
        const uint32_t c = pb.obs_camera[i];
        const double* cr = &cross[W() * i];
        for (int j = 0; j < 3; j++) {
          if (shared) rhs[j] += cr[18 + j] * p()[m - 1];
          for (int k = 0; k < 6; k++) rhs[j] += cr[k * 3 + j] * p()[c * 6 + k];
        }
      }
      for (int j = 0; j < 3; j++) {
        double v = 0;
        for (int k = 0; k < 3; k++) v += at[j * 3 + k] * rhs[k];
        y()[3 * size_t(pt) + j] = v;
      }
    }
#pragma omp parallel for schedule(dynamic, 6)
    for (uint32_t row = 0; row < 6 * C; row++) {
      const uint32_t c = row / 6, j = row % 6;
      const double* A = &camA[36 * size_t(c)];
      double v = 0;
      if (shared) v = focal[row] * p()[m - 1];
      for (int k = 0; k < 6; k++) v += A[j * 6 + k] * p()[c * 6 + k];
      for (uint32_t kk = pb.camera_start[c]; kk < pb.camera_start[c + 1]; kk++) {
        const uint32_t i = pb.camera_obs[kk], pt = pb.obs_point[i];
        const double* cr = &cross[W() * i];
        for (int k = 0; k < 3; k++) v -= cr[j * 3 + k] * y()[3 * size_t(pt) + k];
      }
      Sp()[row] = v;
    }
    if (shared) {
      const size_t n = 6 * size_t(C);
      double v = focal[n] * p()[n];
      for (size_t k = 0; k < n; k++) v += focal[k] * p()[k];
      for (uint32_t i = 0; i < M; i++) {
        const uint32_t pt = pb.obs_point[i];
        const double* cr = &cross[W() * i];
        for (int k = 0; k < 3; k++) v -= cr[18 + k] * y()[3 * size_t(pt) + k];
      }
      Sp()[n] = v;
    }
  }
  // advanceBundleCg, bundle.shade.ts:883-929.
  void advance() {
    if (state[19] == 0) return;
    double denominator = 0;
    for (uint32_t i = 0; i < m; i++) denominator += p()[i] * Sp()[i];
    if (!(denominator > 0)) {
      state[19] = 0;
      state[20] = 1;
      return;
    }
    const double alpha = state[18] / denominator;
    if (!(std::fabs(alpha) < 1e20)) {
      state[19] = 0;
      state[20] = 1;
      return;
    }
    double residual = 0, rho = 0;
    for (uint32_t i = 0; i < m; i++) {
      x()[i] += alpha * p()[i];
      r()[i] -= alpha * Sp()[i];
      residual += r()[i] * r()[i];
    }
    for (uint32_t i = 0; i < m; i++) {
      const double zz = precondition(i);
      z()[i] = zz;
      rho += zz * r()[i];
    }
    state[16]++;
    state[23]++;
    state[22] = residual;
    if (residual <= ctl.cg_tolerance * ctl.cg_tolerance * state[21]) {
      state[19] = 0;
      state[24] = 1;
      return;
    }
    if (!(rho > 0)) {
      state[19] = 0;
      state[20] = 1;
      return;
    }
    const double beta = rho / state[18];
    state[18] = rho;
    for (uint32_t i = 0; i < m; i++) p()[i] = z()[i] + beta * p()[i];
  }
  // updateBundleCandidate, bundle.shade.ts:930-961 (joint-focal.shade.ts:890-925).
  void update() {
    if (state[1] == 0 || state[20] != 0) return;
    if (shared) focal[6 * size_t(C) + 4] = focal[6 * size_t(C) + 3] + x()[m - 1];
    for (uint32_t c = 0; c < C; c++) {
      const double* p_ = pose_at(c, false);
      double moved[12];
      if (variable(c)) op_move_pose(p_, &x()[6 * size_t(c)], moved);
      else std::memcpy(moved, p_, sizeof moved);
      std::memcpy(&trial_pose[12 * size_t(c)], moved, sizeof moved);
    }
#pragma omp parallel for schedule(static)
    for (uint32_t pt = 0; pt < P; pt++) {
      const double* at = &pointb[13 * size_t(pt)];
      double rhs[3] = {at[9], at[10], at[11]};
      for (uint32_t i = pb.point_start[pt]; i < pb.point_start[pt + 1]; i++) {
        const uint32_t c = pb.obs_camera[i];
        const double* cr = &cross[W() * i];
        for (int j = 0; j < 3; j++) {
          if (shared) rhs[j] -= cr[18 + j] * x()[m - 1];
          for (int k = 0; k < 6; k++) rhs[j] -= cr[k * 3 + j] * x()[6 * size_t(c) + k];
        }
      }
      for (int j = 0; j < 3; j++) {
        double v = scene_point[3 * size_t(pt) + j];
        for (int k = 0; k < 3; k++) v += at[j * 3 + k] * rhs[k];
        trial_point[3 * size_t(pt) + j] = v;
      }
    }
  }
  // bundleCandidateGauge, bundle.shade.ts:962-993 (joint-focal.shade.ts:926-970).
  void gauge() {
    state[15] = 0;
    if (state[1] == 0 || state[20] != 0) return;
    const double tol2 = ctl.cg_tolerance * ctl.cg_tolerance;
    if (state[21] > 0 && state[22] > tol2 * state[21]) {
      state[20] = 1;
      return;
    }
    if (shared) {
      const double log_scale = focal[6 * size_t(C) + 4];
      if (!(std::fabs(log_scale) < 700)) return;
      const double fs = op_focal_scale(log_scale);
      for (uint32_t c = 0; c < C; c++) {
        const double fx = pb.cams[c].fx * fs, fy = pb.cams[c].fy * fs;
        if (!(fx >= 1e-6 && fy >= 1e-6 && fx <= 1e6 && fy <= 1e6)) return;
      }
    }
    double cc[3];
    center(ctl.scale_view, true, cc);
    const double baseline =
        std::sqrt((state[3] - cc[0]) * (state[3] - cc[0]) + (state[4] - cc[1]) * (state[4] - cc[1]) +
                  (state[5] - cc[2]) * (state[5] - cc[2]));
    if (!(baseline > 1e-12)) return;
    uint32_t fixed = 0;
    for (uint32_t c = 0; c < C; c++) fixed += variable(c) ? 0 : 1;
    double scale = 1;
    if (fixed == 1) scale = state[2] / baseline;
    if (!(scale > 1e-9 && scale < 1e9)) return;
    for (uint32_t c = 0; c < C; c++) {
      const double* p_ = pose_at(c, true);
      for (int j = 0; j < 12; j++)
        if (!(std::fabs(p_[j]) <= 1e9)) return;
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) {
          double d = 0;
          for (int rr = 0; rr < 3; rr++) d += p_[j * 3 + rr] * p_[k * 3 + rr];
          if (j == k) d -= 1;
          if (!(std::fabs(d) < 1e-6)) return;
        }
    }
    state[13] = scale;
    state[15] = 1;
  }
  // normalizeBundleCandidate, bundle.shade.ts:994-1023.
  void normalize() {
    if (state[1] == 0 || state[15] == 0) return;
    uint32_t fixed = 0;
    for (uint32_t c = 0; c < C; c++) fixed += variable(c) ? 0 : 1;
    for (uint32_t h = 0; h < P; h++)
      if (pb.directional(h)) {
        double* d = &trial_point[3 * size_t(h)];
        const double norm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (norm > 1e-12)
          for (int j = 0; j < 3; j++) d[j] = d[j] / norm;
      }
    if (fixed != 1) return;
    const double s = state[13];
    for (uint32_t h = 0; h < P; h++)
      if (!pb.directional(h))
        for (int j = 0; j < 3; j++)
          trial_point[3 * size_t(h) + j] = state[3 + j] + s * (trial_point[3 * size_t(h) + j] - state[3 + j]);
    for (uint32_t h = 0; h < C; h++) {
      if (h == ctl.anchor) continue;
      double* p_ = &trial_pose[12 * size_t(h)];
      const double o[3] = {state[3], state[4], state[5]};
      double rotated[3];
      for (int i = 0; i < 3; i++)
        rotated[i] = (p_[i * 3] * o[0] + p_[i * 3 + 1] * o[1] + p_[i * 3 + 2] * o[2] + p_[9 + i]) - p_[9 + i];
      for (int i = 0; i < 3; i++) p_[9 + i] = s * p_[9 + i] + (s - 1) * rotated[i];
    }
  }
  // candidateLane + bundleCandidatePartials + acceptBundleCandidate, bundle.shade.ts:1024-1096.
  void accept() {
    state[12] = 0;
    if (state[1] == 0) return;
    double cost = 0, squares = 0;
    if (state[15] != 0)
      for (uint32_t b = 0; b < (M + 63) / 64; b++) {
        double bc = 0, bs = 0;
        for (uint32_t i = b * 64; i < std::min(M, b * 64 + 64); i++) {
          const uint32_t c = pb.obs_camera[i], pt = pb.obs_point[i];
          const double* X = point_at(pt, true);
          if (!(std::max(std::fabs(X[0]), std::max(std::fabs(X[1]), std::fabs(X[2]))) <= 1e9)) {
            bc += 1e30;
            bs += 1e30;
            continue;
          }
          double q[3];
          observed_point(pose_at(c, true), X, pt, q);
          const Projection pr = op_project(camera_at(c, true), q);
          if (!pr.ok) {
            bc += 1e30;
            bs += 1e30;
            continue;
          }
          const double xx = pr.pixel[0] - pb.pixels[2 * i], yy = pr.pixel[1] - pb.pixels[2 * i + 1];
          const double sq = xx * xx + yy * yy;
          bc += op_robust(std::sqrt(sq), ctl.huber);
          bs += sq;
        }
        cost += bc;
        squares += bs;
      }
    if (state[15] != 0 && cost < state[6]) {
      const double change = state[6] - cost;
      state[6] = cost;
      state[7] = squares;
      state[10]++;
      state[12] = 1;
      state[0] = std::max(1e-10, state[0] / 3);
      if (change < 1e-9 * std::max(1.0, cost)) state[1] = 0;
    } else {
      state[11]++;
      state[0] *= 10;
      if (state[20] != 0) state[17]++;
      if (state[0] > 1e12) state[1] = 0;
    }
  }
  // commitBundleCandidate, bundle.shade.ts:1109-1114 (joint-focal.shade.ts:1112-1118).
  void commit() {
    if (state[12] == 0) return;
    scene_pose = trial_pose;
    scene_point = trial_point;
    if (shared) focal[6 * size_t(C) + 3] = focal[6 * size_t(C) + 4];
  }

  void run(double* output) {
    initialize();
    metrics();
    // The host stall monitor, gpu/bundle-shared.ts:83-123.
    const bool monitor = ctl.stall_tolerance > 1e-9;
    double monitor_cost = state[6];
    for (uint32_t iteration = 0; iteration < ctl.iterations && state[1] != 0; iteration++) {
      linearize();
      point_blocks();
      camera_rows();
      if (shared) focal_terms();
      init_cg();
      for (uint32_t k = 0; k < ctl.max_cg && state[19] != 0; k++) {
        schur_product();
        advance();
      }
      update();
      gauge();
      normalize();
      accept();
      commit();
      if (monitor) {
        const double next = state[6], change = monitor_cost - next;
        const bool accepted = state[12] == 1;
        monitor_cost = next;
        if (accepted && change < ctl.stall_tolerance * std::max(1.0, next)) break;
      }
    }
    // packBundleResult, bundle.shade.ts:1115-1125.
    std::memcpy(output, scene_pose.data(), 12 * size_t(C) * sizeof(double));
    std::memcpy(output + 12 * size_t(C), scene_point.data(), 3 * size_t(P) * sizeof(double));
    double* out_state = output + 12 * size_t(C) + 3 * size_t(P);
    for (int i = 0; i < 26; i++) out_state[i] = state[i];
    out_state[24] = std::sqrt(state[9] / double(float(M)));
    out_state[25] = std::sqrt(state[7] / double(float(M)));
    out_state[26] = shared ? focal[6 * size_t(C) + 3] : 0;
  }
};

}  // namespace

extern "C" {

// The GPU operator's algorithm on the CPU.  `output` holds oracle_output_size(C, P) doubles; the
// first 12C + 3P + 27 are the reference operator's output array (packBundleResult).
int oracle_gpu_operator(const oracle_control* ctl, const double* scene, const uint32_t* index,
                        double* output) {
  Problem pb(ctl, scene, index);
  std::memset(output, 0, oracle_output_size(pb.C, pb.P) * sizeof(double));
  Operator op(pb, *ctl);
  op.run(output);
  return int(output[12 * size_t(pb.C) + 3 * size_t(pb.P) + 14]);
}

// bundleMetrics of a packed scene (the cost and RMSE that the reference's tests recompute).
void oracle_metrics(const oracle_control* ctl, const double* scene, const uint32_t* index,
                    double* out3) {
  Problem pb(ctl, scene, index);
  const Metrics m = bundle_metrics(pb, pb.poses, pb.cams, pb.points, ctl->huber);
  out3[0] = m.cost;
  out3[1] = m.rmse;
  out3[2] = m.observations;
}

}  // extern "C"

// =================================================================================================
// (3) Inverse-depth linearisation on the CPU (inverseDepthJacobian), one row per measurement.
namespace {

void inverse_depth_row(const double* m, double* o) {
  for (int k = 0; k < 23; k++) o[k] = 0;
  const double* Rr = m + 3;
  const double* tr = m + 12;
  const double* Rv = m + 15;
  const double* tv = m + 24;
  double C[3], T[3], A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, q[3];
  for (int i = 0; i < 3; i++) C[i] = -Rr[i] * tr[0] - Rr[i + 3] * tr[1] - Rr[i + 6] * tr[2];
  for (int i = 0; i < 3; i++) T[i] = Rv[i * 3] * C[0] + Rv[i * 3 + 1] * C[1] + Rv[i * 3 + 2] * C[2] + tv[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) A[3 * i + j] += Rv[3 * i + k] * Rr[3 * j + k];
  for (int i = 0; i < 3; i++) q[i] = A[3 * i] * m[0] + A[3 * i + 1] * m[1] + A[3 * i + 2] + m[2] * T[i];
  const Camera cam_k{m[27], m[28], m[29], m[30], m[31], m[32]};
  double pixel[2], J[6];
  if (!camera_projection(cam_k, q, pixel, J)) return;
  const double B[9] = {0, q[2], -q[1], -q[2], 0, q[0], q[1], -q[0], 0};
  double point[6] = {0, 0, 0, 0, 0, 0}, cam[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int row = 0; row < 2; row++)
    for (int col = 0; col < 3; col++) {
      for (int k = 0; k < 3; k++) {
        point[3 * row + col] += J[3 * row + k] * (col < 2 ? A[3 * k + col] : T[k]);
        cam[6 * row + col] += J[3 * row + k] * B[3 * k + col];
      }
      cam[6 * row + col + 3] = m[2] * J[3 * row + col];
    }
  o[0] = 1;
  o[1] = pixel[0];
  o[2] = pixel[1];
  for (int k = 0; k < 6; k++) o[3 + k] = point[k];
  for (int k = 0; k < 12; k++) o[9 + k] = cam[k];
  o[21] = pixel[0] - cam_k.cx;
  o[22] = pixel[1] - cam_k.cy;
}

}  // namespace

extern "C" {

// in: n rows of 34 doubles (a, b, rho; reference pose R, t; observing pose R, t; fx, fy, cx, cy,
// k1, k2; the squared radial limit, unused here: the CPU projection derives it), out: n rows of 23.
void oracle_linearize_inverse_depth(uint32_t n, const double* in, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(n); i++) inverse_depth_row(in + 34 * i, out + 23 * i);
}

}  // extern "C"

// =================================================================================================
// (4) Observation evaluation (projectIndexedObservations, filterIndexedObservationDepth,
//     indexedObservationPartials, observationSummary), independent loops under OpenMP.
namespace {

struct ObsRecord {
  Pose pose;
  Camera k;
};

ObsRecord obs_record(const double* cameras, const uint32_t* indices, int64_t i) {
  const double* r = cameras + 18 * size_t(indices[2 * i]);
  ObsRecord out;
  for (int j = 0; j < 9; j++) out.pose.R[j] = r[j];
  for (int j = 0; j < 3; j++) out.pose.t[j] = r[9 + j];
  out.k = Camera{r[12], r[13], r[14], r[15], r[16], r[17]};
  return out;
}

void obs_transform(const Pose& p, const double* X, double q[3]) {
  for (int r = 0; r < 3; r++) q[r] = p.R[3 * r] * X[0] + p.R[3 * r + 1] * X[1] + p.R[3 * r + 2] * X[2] + p.t[r];
}

bool obs_stable_depth(const double* cameras, const uint32_t* indices, const uint32_t* flags, uint32_t start,
                      uint32_t end, const double* X, double noise, double limit) {
  double A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t count = 0;
  for (uint32_t i = start; i < end; i++) {
    if (flags[i] == 0) continue;
    count++;
    const ObsRecord rec = obs_record(cameras, indices, i);
    double q[3];
    obs_transform(rec.pose, X, q);
    const Projection pr = op_project(rec.k, q);
    if (!pr.ok) return false;
    for (int row = 0; row < 2; row++) {
      const double* g = row == 0 ? pr.du : pr.dv;
      const double* R = rec.pose.R;
      const double J[3] = {g[0] * R[0] + g[1] * R[3] + g[2] * R[6], g[0] * R[1] + g[1] * R[4] + g[2] * R[7],
                           g[0] * R[2] + g[1] * R[5] + g[2] * R[8]};
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[3 * r + c] += J[r] * J[c];
    }
  }
  if (count < 2) return false;
  for (uint32_t i = start; i < end; i++) {
    if (flags[i] == 0) continue;
    const ObsRecord rec = obs_record(cameras, indices, i);
    const double axis[3] = {rec.pose.R[6], rec.pose.R[7], rec.pose.R[8]};
    double q[3], s[3];
    obs_transform(rec.pose, X, q);
    if (!op_solve3(A, axis, s) || !(q[2] > 0)) return false;
    const double variance = axis[0] * s[0] + axis[1] * s[1] + axis[2] * s[2];
    if (!(variance >= 0)) return false;
    if (!(noise * std::sqrt(variance) / q[2] <= limit)) return false;
  }
  return true;
}

}  // namespace

extern "C" {

// The packed request of tba_evaluate_observations: 18-word camera records, 3 words per point, 2 per
// pixel, (camera, point) per observation, P + 1 track offsets.  flags: M observation flags, then P
// track flags when guarded; errors: M; summary: inlier error sum, inlier count.
void oracle_evaluate_observations(uint32_t P, uint32_t M, uint32_t guarded, double max_error, double noise,
                                  double limit, const double* cameras, const double* points, const double* pixels,
                                  const uint32_t* indices, const uint32_t* offsets, uint32_t* flags, double* errors,
                                  double* summary) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(M); i++) {
    flags[i] = 0;
    errors[i] = 0;
    const ObsRecord rec = obs_record(cameras, indices, i);
    double q[3];
    obs_transform(rec.pose, points + 3 * size_t(indices[2 * i + 1]), q);
    const Projection pr = op_project(rec.k, q);
    if (!pr.ok) continue;
    const double x = pr.pixel[0] - pixels[2 * i], y = pr.pixel[1] - pixels[2 * i + 1];
    const double e = std::sqrt(x * x + y * y);
    if (e <= max_error) {
      flags[i] = 1;
      errors[i] = e;
    }
  }
  if (guarded) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t h = 0; h < int64_t(P); h++) {
      const uint32_t start = offsets[h], end = offsets[h + 1];
      flags[M + h] = 0;
      if (end <= start) continue;
      uint32_t accepted = 0;
      for (uint32_t i = start; i < end; i++) accepted += flags[i] != 0;
      if (accepted < 2) continue;
      const double* X = points + 3 * size_t(indices[2 * size_t(start) + 1]);
      if (!obs_stable_depth(cameras, indices, flags, start, end, X, noise, limit)) {
        flags[M + h] = 1;
        for (uint32_t i = start; i < end; i++) {
          flags[i] = 0;
          errors[i] = 0;
        }
      }
    }
  }
  const int64_t runs = (int64_t(M) + 63) / 64;
  std::vector<double> pe(runs), pn(runs);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < runs; b++) {
    double e = 0, n = 0;
    for (int64_t i = 64 * b; i < std::min<int64_t>(M, 64 * b + 64); i++)
      if (flags[i]) {
        e += errors[i];
        n += 1;
      }
    pe[b] = e;
    pn[b] = n;
  }
  double te = 0, tn = 0;
  for (int64_t b = 0; b < runs; b++) {
    te += pe[b];
    tn += pn[b];
  }
  summary[0] = te;
  summary[1] = tn;
}

}  // extern "C"

