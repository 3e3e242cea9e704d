// Observation evaluation of a fixed scene (tba_observations.cu): device parameters and launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace tba {

struct ObsParams {
  uint32_t C, P, M;  // camera records, points (= tracks), observations
  uint32_t guarded;  // 1: the depth-sensitivity filter runs (offsets are given)
  double max_error, max_relative_depth, noise;
  const double* cameras;   // 18 per camera record
  const double* points;    // 3P
  const double* pixels;    // 2M
  const uint32_t* indices;  // 2M: camera record, point
  const uint32_t* offsets;  // P + 1 first observations of each track (guarded)
  const uint32_t* tasks;    // ntasks + 1 first tracks of the warp tasks (guarded)
  uint32_t ntasks;
  uint32_t* flags;          // M (+ P with the depth filter: 1 = the track was rejected)
  double* errors;           // M
  double* partials;         // 2 per run of 64 observations
  double* summary;          // inlier error sum, inlier count
};

void launch_observations(const ObsParams& a, cudaStream_t s);
// 34 words in, 23 out per observation (tba_observations.cu).
// Both arrays 16-byte aligned; *error (zeroed by the caller) becomes 1 if a tile's load did not
// complete within `wait_limit` polls, 2 if, after that, the block's loads in flight did not land
// within the full bound either.
constexpr uint32_t kIdWaitPolls = 1u << 22;  // the main-loop bound of a call (TBA_WAIT_LIMIT_DEFAULT)
cudaError_t launch_linearize_inverse_depth(uint32_t count, const double* in, double* out, uint32_t* error,
                                           int sms, cudaStream_t s, uint32_t wait_limit = kIdWaitPolls);

}  // namespace tba
