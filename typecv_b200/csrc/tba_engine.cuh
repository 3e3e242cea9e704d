// The grid engine: one bundle adjustment spread over the whole GPU.
//
// Device layout (all arrays in HBM, resident for the whole solve):
//   * scene: poses 12C, points 3P, cameras 6C, pixels 2M (observations point-major, as the
//     reference packs them), and the trial poses/points of the LM candidate;
//   * index: the reference's packed index array (obsCamera, obsPoint, pointStart, cameraStart,
//     cameraObservations, cameraActive), plus camera-major copies of each observation's point and
//     pixel so that camera passes stream instead of gathering;
//   * per point, a 12-word record: the inverse of the damped point block V_p (6, symmetric), its
//     right-hand side b_p (3) and padding; and y_p = V_p^-1 W^T p of the current product (4);
//   * per camera, the damped block U_c (21, lower triangle), the block-Jacobi preconditioner
//     (S_cc)^-1 (36), the reduced right-hand side (6), the camera/focal coupling H_cf (6) and the
//     radial limit of its lens model;
//   * the PCG vectors x, r, p, Sp, z of length m = 6C (+1 with the shared focal);
//   * the LM/PCG state words of the reference (bundle-shared.ts:362-386) plus the focal scalars.
// Nothing per observation is stored beyond the inputs: the Jacobian factors are recomputed.
//
// Work decomposition: observation-parallel "warp tasks" — runs of whole points of at most 32
// observations, one observation per lane, reduced per point with warp-shuffle segmented scans;
// a point with more than 32 observations is a task of its own, swept in rounds of 32.  Camera
// reductions run over the camera-major observation list in chunks of a fixed schedule.

#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tba_math.cuh"

namespace tba {

// State words.  0..25 are the reference's BUNDLE_STATE layout (gpu/bundle-shared.ts:362-386,
// bundle.shade.ts:68-70): LM [lambda, active, baseline, origin.xyz, cost, SSE, initial cost,
// initial SSE, accepted, rejected, commit, gauge scale, input error, trial valid, CG steps,
// failed solves], PCG [rho, active, failed, initial residual^2, residual^2, steps, converged, -].
enum StateWord : int {
  S_LAMBDA = 0, S_ACTIVE = 1, S_BASELINE = 2, S_ORIGIN = 3, S_COST = 6, S_SSE = 7,
  S_COST0 = 8, S_SSE0 = 9, S_ACCEPTED = 10, S_REJECTED = 11, S_COMMIT = 12, S_SCALE = 13,
  S_INPUT_ERROR = 14, S_TRIAL_VALID = 15, S_CG_STEPS = 16, S_FAILED_SOLVES = 17,
  S_RHO = 18, S_CG_ACTIVE = 19, S_CG_FAILED = 20, S_R0 = 21, S_R2 = 22, S_CG_SOLVE_STEPS = 23,
  S_CG_CONVERGED = 24,
  // Beyond the reference's 26 words:
  S_LOG_FOCAL = 26,        // accepted log focal scale
  S_LOG_FOCAL_TRIAL = 27,  // candidate log focal scale
  S_FOCAL_DIAG = 28,       // damped H_ff
  S_FOCAL_INV = 29,        // 1 / S_ff (preconditioner), -1 when not positive
  S_FOCAL_RHS = 30,        // reduced focal right-hand side
  S_POINT_FAILED = 31,     // a point block failed this LM iteration
  S_ALPHA = 32,            // step length of the current PCG iteration
  S_BETA = 33,             // direction update of the current PCG iteration
  S_REFINE = 34,           // an FP64 refinement of the PCG solution is under way
  S_REFINED = 35,          // refinements that restarted the PCG (this solve)
  S_INNER_R0 = 36,         // residual^2 that the current inner PCG run is measured against
  S_LOOP_ITERS = 37,       // PCG-step launches of the current device-side PCG loop
  S_LOOP_LIMIT = 38,       // the launches that loop may make (its iteration budget)
  S_WORDS = 64
};

constexpr int kTaskObs = 32;        // observations per warp task (one per lane)
constexpr int kFactors = 12;        // stored Jacobian factors per observation
constexpr int kProductThreads = 384;  // two blocks per SM
constexpr int kStagedThreads = 768;   // one block per SM, direction staged in shared memory (FP64 factors)
constexpr int kStagedThreadsWide = 1024;  // the same on large problems (64 registers, a few bytes spilled)
constexpr uint32_t kWideObservations = 2000000;  // observations from which the FP64 product takes 1,024 threads
constexpr int kStagedThreadsF32 = 1024;  // the same with FP32 factors (64 registers a thread)
constexpr int kStagedSmemLimit = 227 * 1024 - 64;  // the dynamic share; the rest is static
// Bytes of a product block's camera sums (6C values of `word` bytes), rounded to 16.
__host__ __device__ inline size_t product_sums_bytes(uint32_t C, size_t word) { return (6 * size_t(C) * word + 15) / 16 * 16; }

constexpr int kPointThreads = 256;  // threads of the task kernels
constexpr int kCameraThreads = 128;
constexpr int kCameraPartials = 60;  // U 21 | b_c 6 | H_cf 6 | (W V^-1 W^T) 21 | W V^-1 b_p 6
constexpr int kScalarPartials = 4;   // H_ff obs | b_f obs | focal diag point terms | focal rhs point terms

struct Params {
  uint32_t C, P, M, D, m;  // cameras, points, observations, directional points, unknowns
  uint32_t anchor, scale_view, normalize_scale, shared;
  double huber, tol, stall;
  double tol_inner;  // PCG tolerance of one inner run (tol in FP64; looser in the mixed form)
  // scene (current) and candidate
  double* poses;    // 12C
  double* points;   // 3P
  const double* cams;    // 6C
  const double* pixels;  // 2M
  double* tposes;   // 12C
  double* tpoints;  // 3P
  // index sections
  const uint32_t* obs_camera;
  const uint32_t* obs_point;
  const uint32_t* point_start;
  const uint32_t* camera_start;
  const uint32_t* camera_obs;
  const uint32_t* active;
  // schedules
  const uint32_t* tasks;     // ntasks + 1 first points
  const uint32_t* task_obs;  // ntasks + 1 first observations
  uint32_t ntasks;
  const uint32_t* chunk_cam;    // nchunks
  const uint32_t* chunk_beg;    // nchunks + 1 positions in camera_obs
  const uint32_t* cam_chunk;    // C + 1 first chunk of each camera
  uint32_t nchunks;
  uint32_t task_blocks;  // grid of the task kernels (point pass, Schur points, update, cost)
  // linearisation
  double* rlim;        // C radial limits
  uint32_t* cm_point;  // M, camera-major
  double* cm_pixel;    // 2M, camera-major
  double* pblk;        // 12P: V^-1 (6), b_p (3), padding
  float* pblk32;       // 6P: V^-1 in FP32 for the FP32 product (mixed form), or null
  double* y;           // 4P: y_p of the current Schur product
  double* chunk_prod;  // 8 per camera chunk: sum W_i y (6), focal share
  // Jacobian factors of each observation (factored engine), component-major [12][Mpad]:
  // q~ = R^T q (3), J_p rows R^T du, R^T dv (6), Huber weight, focal column jf (2).
  double* F;
  float* F32;          // the same factors in FP32 (mixed precision), or null
  uint32_t Mpad;       // stride of a factor component
  uint32_t factored;   // 1: one-pass product over stored factors; 0: two-pass recompute
  uint32_t refine;     // 1: this launch evaluates the FP64 product S x of the refinement
  uint32_t prod_blocks;  // grid of the one-pass product
  double* pw;          // 6C: the PCG direction of each camera in world axes (R^T omega, R^T v)
  double* xw;          // 6C: the PCG solution of each camera in world axes
  double* acc_part;    // prod_blocks x m: per-block camera sums of the one-pass product, in world axes
                       // and in the block sums' type (FP32 values for the FP32 product)
  double* camU;     // 21C
  double* camMinv;  // 36C
  double* camRhs;   // 6C
  double* camHcf;   // 6C
  double* chunk_part;  // kCameraPartials * nchunks
  // PCG
  double* x;
  double* r;
  double* p;
  double* Sp;
  double* z;
  double* blk_part;   // finish partials, 4 per block
  double* scal_part;  // kScalarPartials per block of the task kernels
  double* cost_part;  // 4 per block
  uint32_t* ticket;   // last-block counters
  double* state;      // S_WORDS
  double* output;
  // The condition of the CUDA graph's while node that runs the PCG steps on the device (set by
  // k_pcg_loop_next inside the loop's body graph; unused outside it).
  cudaGraphConditionalHandle pcg_loop;
};

// Launches (tba_kernels.cu), each on stream `s`; grids come from `p`.
void launch_initialize(const Params& p, cudaStream_t s);
void launch_cost(const Params& p, cudaStream_t s);
void launch_finish_metrics(const Params& p, cudaStream_t s);
void launch_point_pass(const Params& p, cudaStream_t s);
void launch_camera_pass(const Params& p, cudaStream_t s);
void launch_camera_finish(const Params& p, cudaStream_t s);
void launch_pcg_init(const Params& p, cudaStream_t s);
void launch_product(const Params& p, cudaStream_t s);
// One PCG step after the product: column reduction of the product partials and alpha, the
// distributed update of x, r, z and beta, then the new direction p.
void launch_product_finish(const Params& p, cudaStream_t s);
// The device-side PCG loop (a CUDA graph with a while node whose body is one PCG step): its
// iteration budget, set on the stream before the graph's launch, and the body's last kernel, which
// counts the step and keeps the loop going while the PCG is active and within the budget.
void launch_pcg_loop_begin(const Params& p, uint32_t limit, cudaStream_t s);
void launch_pcg_loop_next(const Params& p, cudaStream_t s);
// Mixed form: the FP64 residual r = b - S x of the PCG solution (the two-pass recompute product
// on x), and the PCG restarted from it when it is above the tolerance.
void launch_refine(const Params& p, cudaStream_t s);
// Diagnostics: every row of S p after a product launched with `p` (no state is written).
void launch_product_rows(const Params& p, double* out, cudaStream_t s);
void launch_update_cameras(const Params& p, cudaStream_t s);
void launch_update_points(const Params& p, cudaStream_t s);
void launch_accept(const Params& p, cudaStream_t s);
void launch_commit(const Params& p, cudaStream_t s);
void launch_pack(const Params& p, cudaStream_t s);
// Blocks of the widest PCG-step kernel (sizes blk_part).
uint32_t product_finish_blocks(const Params& p);
// The one-pass product keeps m camera sums in shared memory: the largest m it takes, its
// dynamic shared memory, the opt-in of the product kernels, and their blocks per SM.
uint32_t product_max_unknowns();
size_t product_smem_bytes(const Params& p);
bool product_staged(const Params& p);
int product_threads(const Params& p);
cudaError_t configure_kernels();
int product_blocks_per_sm(const Params& p);

}  // namespace tba
