// The adjoint of the converged bundle adjustment (vector-Jacobian product by implicit
// differentiation) and the exact-Newton steps that share its linear algebra.
//
// At a converged solution theta* the robust cost's gradient F(theta, y, kappa) vanishes in every
// free direction, so d theta* = -H^-1 (F_y dy + F_kappa d kappa) with H the exact Hessian of the
// cost (second derivatives of the projection and of the Huber loss included; not the
// Gauss-Newton matrix).  The gauge: the anchor camera is fixed; with exactly one fixed camera the
// cost is also invariant to scaling the world about the anchor's centre, which the solver fixes
// by keeping the anchor-to-scale-camera baseline.  H is then singular along that scale direction
// v_s, and the derivative of the baseline-constrained solution uses the cotangent projected
// obliquely along v_s onto the constraint (g' = g - grad_c (v_s . g) / (grad_c . v_s)), and the
// system made definite by the rank-one term mu grad_c grad_c^T on the scale camera's translation.
//
// The Newton steps are damped (H + mu G, G the Gauss-Newton matrix with the solver's IRLS weights,
// mu adapted by the robust cost of the candidate) until the undamped exact-Newton step is accepted;
// near the solution they converge quadratically.
//
// Unknowns are the local coordinates of the solver's own updates: a left rotation omega and a
// translation step v per variable camera (R' = exp(omega) R, t' = exp(omega) t + v) and a point
// step dX.  Point blocks are eliminated (Schur complement) and the camera system is solved by
// block-Jacobi PCG, as in the LM solve; the exact Hessian's cross blocks W_i are stored per
// observation.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace tba {

// Device state words of the adjoint's PCG.
enum AdjWord : int {
  A_RHO = 0, A_ALPHA = 1, A_BETA = 2, A_R0 = 3, A_R2 = 4, A_ACTIVE = 5, A_FAILED = 6, A_STEPS = 7,
  A_POINT_FAILED = 8, A_CAMERA_FAILED = 9, A_GNORM = 10, A_SBAR = 11, A_KBAR = 12, A_DOT = 13,
  A_BASELINE = 14, A_ORIGIN = 15, A_SCALE = 18, A_INVALID = 19, A_COST = 20, A_POINT_SINGULAR = 21,
  A_LOOP_ITERS = 22,  // PCG steps of the current device-side PCG loop
  A_LOOP_LIMIT = 23,  // the steps that loop may take
  A_WORDS = 32
};

struct AdjParams {
  uint32_t C, P, M;
  uint32_t anchor, scale_view, normalize_scale;
  double huber, tol;
  // scene (the evaluation point; updated in place by Newton steps)
  double* poses;   // 12C
  double* points;  // 3P
  const double* cams;    // 6C
  const double* pixels;  // 2M
  const uint32_t* obs_camera;
  const uint32_t* obs_point;
  const uint32_t* point_start;
  const uint32_t* camera_start;
  const uint32_t* camera_obs;
  const uint32_t* active;
  // per observation (point-major): exact Hessian pieces and gradient
  double* Hcp;  // 18M: d2E / d camera d point, row a (camera), column m (point): [a * 3 + m]
  double* Hcc;  // 21M: camera-camera block, lower triangle (sym6 order)
  double* Hpp;  // 6M: point-point block (00, 01, 02, 11, 12, 22)
  double* gc;   // 6M: camera gradient share
  double* gp;   // 3M: point gradient share
  // per point
  double* Vinv;  // 6P
  double* bp;    // 3P: point right-hand side
  double* lp;    // 3P: point solution
  double* yp;    // 3P: product scratch
  // per camera
  double* U;     // 21C: camera blocks (+ the gauge term)
  double* Minv;  // 36C: block-Jacobi preconditioner
  double* bc;    // 6C: camera right-hand side, then the reduced one
  double* x;     // 6C: camera solution
  double* r;
  double* p;
  double* z;
  double* Sp;
  double* cot;   // 6C + 3P: cotangent in local coordinates (cameras, then points)
  double* ybar;  // 2M: cotangent of the observed pixels
  double* state; // A_WORDS
  double* tposes;   // 12C candidate of a Newton step
  double* tpoints;  // 3P
  double mu;        // damping of the Newton steps (H + mu G); 0: exact Newton
  uint32_t rhs_mode;  // 0: Newton (-gradient), 1: adjoint (cot)
  // The one-pass Schur product (when the camera sums fit a block's shared memory): warp tasks of
  // whole points (at most 32 observations, or one longer point), their first observations, and the
  // per-block partial camera rows.
  const uint32_t* task_obs;  // ntasks + 1
  uint32_t ntasks;
  uint32_t prod_blocks;      // 0: the two-pass product
  uint32_t prod_copies;      // copies of the camera sums in a block's shared memory (warp w adds to w % copies)
  double* part;              // prod_blocks x 6C
  // The condition of the CUDA graph's while node that runs the PCG steps on the device (set by
  // k_adj_loop_next inside the loop's body graph; unused outside it).  The step kernels read
  // neither `mu` nor `rhs_mode`.
  cudaGraphConditionalHandle loop;
};

// The largest camera count of the one-pass product (its camera sums in one block's shared memory).
uint32_t adj_one_pass_max_cameras();
// Copies of the camera sums per block of the one-pass product for C cameras, and its blocks per SM.
uint32_t adj_product_copies(uint32_t C);
uint32_t adj_product_blocks_per_sm(uint32_t C);
cudaError_t adj_configure();  // the one-pass product's shared-memory limit

uint32_t adj_launch_init(const AdjParams& a, cudaStream_t s);        // gauge origin and baseline
uint32_t adj_launch_reset(const AdjParams& a, cudaStream_t s);       // zero the per-solve sums and flags
uint32_t adj_launch_assemble(const AdjParams& a, cudaStream_t s);    // per observation, points, cameras
uint32_t adj_launch_pcg_init(const AdjParams& a, cudaStream_t s);
// Product + vector step; with events, the one-pass product's launch is bracketed by them.
uint32_t adj_launch_pcg_step(const AdjParams& a, cudaStream_t s, cudaEvent_t before = nullptr,
                             cudaEvent_t after = nullptr);
// The device-side PCG loop (a CUDA graph with a while node whose body is one PCG step): its step
// budget, set on the stream before the graph's launch, and the body's last kernel, which counts the
// step and keeps the loop going while the PCG is active and within the budget.
uint32_t adj_launch_loop_begin(const AdjParams& a, uint32_t limit, cudaStream_t s);
uint32_t adj_launch_loop_next(const AdjParams& a, cudaStream_t s);
uint32_t adj_launch_back_substitute(const AdjParams& a, cudaStream_t s);
// The candidate theta (+) delta into tposes/tpoints (with the gauge normalisation) and its robust
// cost into A_COST; then, when accepted, its commit.
uint32_t adj_launch_newton_candidate(const AdjParams& a, cudaStream_t s);
uint32_t adj_launch_newton_commit(const AdjParams& a, cudaStream_t s);
// The robust cost of the current point into A_COST.
uint32_t adj_launch_cost(const AdjParams& a, cudaStream_t s);
uint32_t adj_launch_cotangent(const AdjParams& a, const double* cotangent, cudaStream_t s);
uint32_t adj_launch_vjp(const AdjParams& a, cudaStream_t s);

}  // namespace tba
