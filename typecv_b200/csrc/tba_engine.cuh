// The grid engine: one bundle adjustment spread over the whole GPU.
//
// Device layout (all arrays in HBM, resident for the whole solve):
//   * scene: poses 12C, points 3P, cameras 6C, pixels 2M (observations point-major, as the
//     reference packs them), and the trial poses/points of the LM candidate;
//   * index: the reference's packed index array (obsCamera, obsPoint, pointStart, cameraStart,
//     cameraObservations, cameraActive);
//   * per observation, the Schur cross blocks W_i = w J_c^T J_p (18 words; 21 with the shared
//     focal, whose 3 words are w J_f^T J_p), stored component-major ([k][M]) so that a warp
//     reading 32 consecutive observations reads 256 contiguous bytes per component;
//   * per point, the inverse of the damped point block V_p (6 words, symmetric) and its
//     right-hand side b_p (3), component-major;
//   * per camera, the damped block U_c (21, lower triangle), the block-Jacobi preconditioner
//     (S_cc)^-1 (36), the reduced right-hand side (6) and the camera/focal coupling H_cf (6);
//   * the PCG vectors x, r, p, Sp, z of length m = 6C (+1 with the shared focal);
//   * the LM/PCG state words of the reference (bundle-shared.ts:362-386) plus the focal scalars.
//
// Work decomposition: observation-parallel "warp tasks" — runs of whole points of at most 32
// observations, one observation per lane, reduced per point with warp-shuffle segmented scans;
// a point with more than 32 observations is a task of its own, swept in rounds of 32.  Camera
// reductions run over the camera-major observation list in chunks.
#pragma once

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
  S_WORDS = 64
};

constexpr int kTaskObs = 32;        // observations per warp task (one per lane)
constexpr int kPointThreads = 256;  // threads of the task kernels
constexpr int kProductThreads = 512;
constexpr int kCameraThreads = 128;
constexpr int kCameraPartials = 60;  // U 21 | b_c 6 | H_cf 6 | (W V^-1 W^T) 21 | W V^-1 b_p 6
constexpr int kScalarPartials = 4;   // H_ff obs | b_f obs | focal diag point terms | focal rhs point terms

struct Params {
  uint32_t C, P, M, D, m;  // cameras, points, observations, directional points, unknowns
  uint32_t anchor, scale_view, normalize_scale, shared;
  double huber, tol, stall;
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
  const uint32_t* tasks;  // ntasks + 1 first points
  uint32_t ntasks;
  const uint32_t* chunk_cam;    // nchunks
  const uint32_t* chunk_beg;    // nchunks + 1 positions in camera_obs
  const uint32_t* cam_chunk;    // C + 1 first chunk of each camera
  uint32_t nchunks;
  uint32_t task_blocks;  // grid of the task kernels (point pass, update, cost)
  uint32_t prod_blocks;  // grid of the Schur product kernel
  // linearisation
  double* W;     // wdim * M, component-major
  uint32_t wdim; // 18 or 21
  float* Wf32;   // mixed precision copy, wdim * M (or null)
  double* vinv;  // 6P
  double* bp;    // 3P
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
  double* acc_part;   // product partials, gridDim * m
  double* blk_part;   // finish partials, 2 per block
  double* scal_part;  // kScalarPartials per block of the task kernels
  double* cost_part;  // 4 per block
  uint32_t* ticket;   // last-block counters
  double* state;      // S_WORDS
  double* output;
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
void launch_update_cameras(const Params& p, cudaStream_t s);
void launch_update_points(const Params& p, cudaStream_t s);
void launch_accept(const Params& p, cudaStream_t s);
void launch_commit(const Params& p, cudaStream_t s);
void launch_pack(const Params& p, cudaStream_t s);
// Blocks of the widest finish kernel (sizes blk_part), and the dynamic shared memory of the
// product kernel.
uint32_t product_finish_blocks(const Params& p);
size_t product_smem_bytes(const Params& p);
// Largest unknown count whose accumulators fit one block's shared memory.
uint32_t product_max_unknowns();
// Opt the product kernel into its shared-memory size; returns the first CUDA error.
cudaError_t configure_kernels();
// Blocks per SM of the product kernel at `smem` bytes (occupancy query).
int product_blocks_per_sm(size_t smem);

}  // namespace tba
