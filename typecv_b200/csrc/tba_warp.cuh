// Warp- and block-level helpers shared by the grid engine (tba_kernels.cu) and the batched block
// solver (tba_batch.cu): vector loads, segmented warp scans, fixed-order block sums, and the
// world-axis Jacobian factors of one observation with the products formed from them.
#pragma once

#include <cstdint>

#include "tba_engine.cuh"

namespace tba {

constexpr unsigned kFull = 0xffffffffu;

__device__ inline void load6(const double* src, double out[6]) {
  const double2* s = reinterpret_cast<const double2*>(src);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double2 v = s[k];
    out[2 * k] = v.x;
    out[2 * k + 1] = v.y;
  }
}

__device__ inline void load_pose(const double* poses, uint32_t c, double out[12]) {
  load6(poses + 12 * size_t(c), out);
  load6(poses + 12 * size_t(c) + 6, out + 6);
}

// Inclusive segmented sum over lanes: lanes with equal `seg` form contiguous runs.
template <int N>
__device__ inline void seg_scan(double (&v)[N], int seg, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int s = __shfl_up_sync(kFull, seg, d);
    double t[N];
#pragma unroll
    for (int n = 0; n < N; n++) t[n] = __shfl_up_sync(kFull, v[n], d);
    if (lane >= d && s == seg) {
#pragma unroll
      for (int n = 0; n < N; n++) v[n] += t[n];
    }
  }
}

// Runs of equal `seg` over the lanes (contiguous): each lane's position in its run, the run heads
// as a lane mask, and the largest position in the warp, which bounds the steps a scan needs.
struct Runs {
  unsigned heads;
  int pos;
  int maxpos;
};

__device__ inline Runs lane_runs(int seg, int lane) {
  const int prev = __shfl_up_sync(kFull, seg, 1);
  const unsigned heads = __ballot_sync(kFull, lane == 0 || prev != seg);
  const int pos = lane - (31 - __clz(heads & (kFull >> (31 - lane))));
  return Runs{heads, pos, int(__reduce_max_sync(kFull, unsigned(pos)))};
}

// Inclusive sum within each run, in as many doubling steps as the longest run needs.
template <typename T, int N>
__device__ inline void run_scan(T (&v)[N], const Runs& r) {
  for (int d = 1; d <= r.maxpos; d <<= 1) {
    T t[N];
#pragma unroll
    for (int n = 0; n < N; n++) t[n] = __shfl_up_sync(kFull, v[n], d);
    if (r.pos >= d) {
#pragma unroll
      for (int n = 0; n < N; n++) v[n] += t[n];
    }
  }
}

// True in the last lane of each run.
__device__ inline bool run_tail(const Runs& r, int lane) { return lane == 31 || ((r.heads >> (lane + 1)) & 1u); }

template <int N>
__device__ inline void warp_allsum(double (&v)[N]) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
#pragma unroll
    for (int n = 0; n < N; n++) v[n] += __shfl_xor_sync(kFull, v[n], d);
  }
}

// Sum N values over the block in a fixed order; the result is valid in thread 0.
template <int N>
__device__ inline void block_sum(double (&v)[N], double* smem) {
  warp_allsum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int n = 0; n < N; n++) smem[warp * N + n] = v[n];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; n++) {
      double s = 0;
      for (int w = 0; w < nwarps; w++) s += smem[w * N + n];
      v[n] = s;
    }
  }
  __syncthreads();
}

// The camera's 6-vector v in world axes: (R^T v_omega, R^T v_t).
__device__ inline void to_world(const double* R, const double v[6], double* out) {
  for (int c = 0; c < 3; c++) {
    out[c] = R[c] * v[0] + R[3 + c] * v[1] + R[6 + c] * v[2];
    out[3 + c] = R[c] * v[3] + R[3 + c] * v[4] + R[6 + c] * v[5];
  }
}

template <typename T>
struct Factors {
  T q[3], ju[3], jv[3], w, jf[2];
};

template <typename T>
__device__ inline void load_factors(const T* F, size_t stride, uint32_t i, Factors<T>& f) {
  const T* p = F + i;
  f.q[0] = __ldg(p); f.q[1] = __ldg(p + stride); f.q[2] = __ldg(p + 2 * stride);
  f.ju[0] = __ldg(p + 3 * stride); f.ju[1] = __ldg(p + 4 * stride); f.ju[2] = __ldg(p + 5 * stride);
  f.jv[0] = __ldg(p + 6 * stride); f.jv[1] = __ldg(p + 7 * stride); f.jv[2] = __ldg(p + 8 * stride);
  f.w = __ldg(p + 9 * stride);
  f.jf[0] = __ldg(p + 10 * stride); f.jf[1] = __ldg(p + 11 * stride);
}

// W_i^T x in world axes, from the factors and the camera's step in world axes (xw).
template <typename T>
__device__ inline void factor_wt(const Factors<T>& f, const double* xw, double xf, bool variable, bool dir, bool shared,
                                 double t[3]) {
  T au = 0, av = 0;
  if (variable) {
    const T o0 = T(xw[0]), o1 = T(xw[1]), o2 = T(xw[2]);
    T m0 = o1 * f.q[2] - o2 * f.q[1], m1 = o2 * f.q[0] - o0 * f.q[2], m2 = o0 * f.q[1] - o1 * f.q[0];
    if (!dir) {
      m0 += T(xw[3]);
      m1 += T(xw[4]);
      m2 += T(xw[5]);
    }
    au = f.ju[0] * m0 + f.ju[1] * m1 + f.ju[2] * m2;
    av = f.jv[0] * m0 + f.jv[1] * m1 + f.jv[2] * m2;
  }
  if (shared) {
    au += f.jf[0] * T(xf);
    av += f.jf[1] * T(xf);
  }
  au *= f.w;
  av *= f.w;
  for (int c = 0; c < 3; c++) t[c] = double(au * f.ju[c] + av * f.jv[c]);
}

}  // namespace tba
