// Device-side structural checks of a packed problem (the bulk of bundleProblem's validation,
// src/sfm/bundle/gpu/bundle-host.ts:31-113 and src/geometry/gpu/bounds.ts:5-26), run on the
// arrays just uploaded, before any solver kernel reads them.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace tba {

// The first failure of each check, as the smallest key; UINT64_MAX where none failed.
enum CheckKey : int {
  CK_POINTS = 0,  // (point << 2) | {0: offsets exceed M, 1: fewer than two observations, 2: point mismatch}
  CK_CAMERA = 1,  // the first observation whose camera is out of range
  CK_LISTS = 2,   // the first camera whose observation list is not exactly its observations
  CK_SCENE = 3,   // the first scene value outside the supported bounds
  CK_WORDS = 4
};

struct CheckParams {
  uint32_t C, P, M;
  const uint32_t* index;  // the packed index on the device
  // The packed scene on the device, in up to four segments (poses, points, cameras, pixels) that
  // follow each other in the packed array: segment k holds values [base[k], base[k] + len[k]).
  const double* seg[4];
  uint64_t base[4], len[4];
  uint32_t* claims;       // M words of scratch (zeroed by the launcher)
  unsigned long long* keys;  // CK_WORDS words (set to all ones by the launcher)
  bool lists;             // run the camera-list check (only when the camera offsets are monotone and within M)
};

// Enqueues the checks on `s` (memsets included).
cudaError_t launch_checks(const CheckParams& p, int sms, cudaStream_t s);

}  // namespace tba
