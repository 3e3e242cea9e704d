// Device-side structural checks of a packed problem; see tba_checks.cuh.  Every kernel records the
// smallest failing position of its check with an atomic minimum, so the host can report the
// failure a serial scan in the same order would meet first.
#include "tba_checks.cuh"

namespace tba {
namespace {

__global__ void __launch_bounds__(256) k_check_points(CheckParams A) {
  const uint32_t* ps = A.index + 2 * size_t(A.M);
  const uint32_t* obs_point = A.index + A.M;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < A.P; p += gridDim.x * blockDim.x) {
    const uint32_t b = ps[p], e = ps[p + 1];
    unsigned long long key = ~0ull;
    if (e > A.M) {
      key = (uint64_t(p) << 2) | 0;
    } else if (uint64_t(e) < uint64_t(b) + 2) {
      key = (uint64_t(p) << 2) | 1;
    } else {
      for (uint32_t i = b; i < e; i++)
        if (obs_point[i] != p) {
          key = (uint64_t(p) << 2) | 2;
          break;
        }
    }
    if (key != ~0ull) atomicMin(A.keys + CK_POINTS, key);
  }
}

__global__ void __launch_bounds__(256) k_check_cameras(CheckParams A) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.M; i += gridDim.x * blockDim.x)
    if (A.index[i] >= A.C) atomicMin(A.keys + CK_CAMERA, (unsigned long long)i);
}

// One block per camera (grid-stride): every entry of the camera's list must be an observation of
// that camera, claimed once.  The camera offsets were checked on the host (monotone, within M).
__global__ void __launch_bounds__(256) k_check_lists(CheckParams A) {
  const uint32_t* obs_camera = A.index;
  const uint32_t* cs = A.index + 2 * size_t(A.M) + A.P + 1;
  const uint32_t* cam_obs = cs + A.C + 1;
  for (uint32_t cam = blockIdx.x; cam < A.C; cam += gridDim.x) {
    bool bad = false;
    for (uint32_t k = cs[cam] + threadIdx.x; k < cs[cam + 1]; k += blockDim.x) {
      const uint32_t i = cam_obs[k];
      if (i >= A.M || obs_camera[i] != cam || atomicAdd(A.claims + i, 1u) != 0) bad = true;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicMin(A.keys + CK_LISTS, (unsigned long long)cam);
  }
}

__global__ void __launch_bounds__(256) k_check_scene(const double* x, uint64_t n, uint64_t base,
                                                      unsigned long long* keys) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const double v = x[i];
    if (!isfinite(v) || fabs(v) > 1e9 || (v != 0 && fabs(v) < 1e-30))
      atomicMin(keys + CK_SCENE, (unsigned long long)(base + i));
  }
}

}  // namespace

cudaError_t launch_checks(const CheckParams& p, int sms, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(p.keys, 0xff, CK_WORDS * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  const uint32_t grid = uint32_t(sms > 0 ? sms : 1) * 8;
  if (p.P) k_check_points<<<grid, 256, 0, s>>>(p);
  if (p.M) k_check_cameras<<<grid, 256, 0, s>>>(p);
  if (p.lists && p.C) {
    if (p.M) {
      e = cudaMemsetAsync(p.claims, 0, sizeof(uint32_t) * p.M, s);
      if (e != cudaSuccess) return e;
    }
    k_check_lists<<<p.C < 4u * uint32_t(sms) ? p.C : 4u * uint32_t(sms), 256, 0, s>>>(p);
  }
  for (int k = 0; k < 4; k++)
    if (p.len[k]) k_check_scene<<<grid, 256, 0, s>>>(p.seg[k], p.len[k], p.base[k], p.keys);
  return cudaGetLastError();
}

}  // namespace tba
