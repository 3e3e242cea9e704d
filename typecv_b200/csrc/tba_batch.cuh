// The batched block solver: many independent bundle adjustments (local windows) in one persistent
// launch.  Each block takes whole problems from a queue (largest first) and runs the complete LM
// loop of one problem with its camera system in shared memory; points and per-observation factors
// stay in HBM.  Same semantics per problem as the grid engine (tba_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace tba {

// One problem of a batch as the block solver sees it; every pointer is device memory.
struct BatchProblem {
  uint32_t C, P, M, ntasks;
  uint32_t anchor, scale_view, normalize_scale, Mpad;
  // The problem's packed scene (packBundleScene) and index (bundleIndexLayout) sections.
  const double* poses0;   // 12C
  const double* points0;  // 3P
  const double* cams;     // 6C
  const double* pixels;   // 2M
  const uint32_t* obs_camera;
  const uint32_t* obs_point;
  const uint32_t* point_start;
  const uint32_t* camera_start;
  const uint32_t* camera_obs;
  const uint32_t* active;
  const uint32_t* tasks;  // ntasks + 1 first points of the warp tasks
  // Workspace.
  double* tpoints;  // 3P candidate points
  double* pblk;     // 12P: V^-1 (6), b_p (3), padding
  void* F;          // 12 x Mpad Jacobian factors (float in the mixed form, else double)
  double* F64;      // the mixed form's FP64 copy of the factors (its FP64 tail and update); else null
  double* output;   // the result record (12C + 3P + 26 [+1])
  double* points;   // output + 12C: the working copy of the points
};

struct BatchArgs {
  const BatchProblem* problems;
  const uint32_t* order;  // solve order (largest first)
  uint32_t* queue;        // next position in `order`
  uint32_t count;
  uint32_t Cmax;          // the shared-memory layout holds this many cameras
  uint32_t iterations, max_cg;
  double huber, tol, tol_inner, stall;
};

// The launch shapes the autotuner chooses among: threads per block and the blocks per SM that the
// register budget is compiled for.
struct BatchShape {
  int threads, min_blocks;
};
constexpr int kBatchShapes = 4;
BatchShape batch_shape(int k);
size_t batch_smem_bytes(uint32_t Cmax);
// The largest camera count whose shared-memory layout fits one block.
uint32_t batch_max_cameras();
cudaError_t batch_configure();
// Blocks per SM of shape k for the given form and dynamic shared memory (0 on error).
int batch_blocks_per_sm(int k, bool shared, bool mixed, size_t smem);
cudaError_t launch_batch(int k, bool shared, bool mixed, const BatchArgs& a, int blocks, size_t smem, cudaStream_t s);

}  // namespace tba
