// The C ABI of libtba.so (include/tba.h) and the host side of one solve: structural checks of
// the packed arrays, the warp-task and camera-chunk schedules, the device workspace, and the LM
// loop that enqueues the grid engine's kernels (tba_kernels.cu).
//
// The loop is the reference's plan (src/sfm/bundle/gpu/bundle.ts:314-772 and
// joint-focal.ts:330-880) with its host round trips reduced to one small read per PCG chunk and
// one per LM iteration: every kernel is guarded by the device state words, so an iteration past
// convergence is a no-op and the reads only end the loops early.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tba.h"
#include "tba_adjoint.cuh"
#include "tba_batch.cuh"
#include "tba_engine.cuh"
#include "tba_checks.cuh"
#include "tba_observations.cuh"

using tba::Params;

// The device-side PCG loop of one product form: a graph of one while node whose body is a PCG
// step (product, column sums and alpha, x/r/z update and beta, new direction) and k_pcg_loop_next,
// which counts the step and ends the loop when the PCG stops or its budget is spent.  The graph
// bakes the launch parameters; `key` holds them, and a solve with the same parameters (the same
// scene shape in the same workspace) launches it again instead of building a new one.
struct PcgLoop {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<char> key;
  uint32_t body_kernels = 0;  // kernels of one body iteration
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key.clear();
  }
};

struct tba_device {
  int ordinal = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t down = nullptr;  // device-to-host copies that overlap the next slice's upload and kernel
  std::mutex mu;
  std::string error;
  char* arena = nullptr;
  size_t capacity = 0;
  double* pinned = nullptr;  // small host buffer for flag reads
  std::vector<cudaEvent_t> events;
  // Polls of each main-loop wait of the inverse-depth linearisation (tba_device_set_wait_limit).
  uint32_t wait_limit = tba::kIdWaitPolls;
  // Batched solves: their own workspace, the cached graph of the last launch and its key, and
  // the autotuner's choices by batch shape.
  char* batch_arena = nullptr;
  size_t batch_capacity = 0;
  cudaGraphExec_t batch_graph = nullptr;
  std::vector<char> batch_key;
  std::map<std::string, int> tuned;
  // The grid engine's device-side PCG loops (the solve's own product and the mixed form's FP64
  // tail) and the adjoint's.
  PcgLoop pcg_loops[2];
  PcgLoop adj_loop;
  // Set when the driver could not build a conditional graph: the PCG steps then run from the host.
  bool host_pcg_only = false;
};

// A scene resident on the device between calls: the packed arrays of one problem and its host
// schedules.
struct tba_scene {
  tba_device* device = nullptr;
  tba_control shape{};
  double* scene = nullptr;     // device, tba_scene_size doubles
  uint32_t* index = nullptr;   // device, tba_index_size words
  void* plan = nullptr;        // HostPlan
  uint32_t* plan_dev = nullptr;  // device copy of the plan's arrays (HostPlan::sections order)
};

namespace {

std::string g_open_error;

struct Fail {
  tba_status status;
  std::string message;
};

#define CUDA_TRY(expr)                                                                     \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess)                                                                 \
      throw Fail{TBA_ERROR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)};      \
  } while (0)

[[noreturn]] void argument(const std::string& m) { throw Fail{TBA_ERROR_ARGUMENT, m}; }

// A bump allocator over the device workspace (256-byte aligned sections).
struct Layout {
  size_t bytes = 0;
  template <typename T>
  size_t take(size_t count) {
    const size_t at = bytes;
    bytes += (count * sizeof(T) + 255) / 256 * 256;
    return at;
  }
};

// bundleProblem's option limits (src/sfm/bundle/gpu/bundle-host.ts:49-65) and the gauge and
// window rules it checks (:66-96), on the packed control block.
void check_control(const tba_control* c) {
  if (!c) argument("Invalid GPU BA scene/options: no control block");
  if (c->cameras < 2 || c->points < 1 || c->directional_points >= c->points + 0u ||
      c->iterations > 100 || !(std::isfinite(c->huber) && c->huber >= 1e-12 && c->huber <= 1e6) ||
      c->max_cg < 1 || c->max_cg > 256 ||
      !(std::isfinite(c->cg_tolerance) && c->cg_tolerance >= 1e-12 && c->cg_tolerance <= 1e-2) ||
      !(std::isfinite(c->stall_tolerance) && c->stall_tolerance >= 0 && c->stall_tolerance < 1) ||
      c->precision > 1 ||
      (c->flags & ~(TBA_FLAG_TIME_PRODUCTS | TBA_FLAG_PRODUCT_ERROR | TBA_FLAG_HOST_PCG_LOOP)) != 0)
    argument("Invalid GPU BA scene/options");
  if (c->anchor >= c->cameras || c->scale_view >= c->cameras || c->anchor == c->scale_view)
    argument("Invalid GPU BA gauge cameras");
}

// The structure of the packed index array (bundleIndexLayout): every section consistent with the
// others, so that no kernel can index out of bounds.
// Runs f(begin, end, worker) over [0, n) split into up to `threads` contiguous ranges on host
// threads (serially below `serial_below`).
template <typename F>
void parallel_ranges(uint64_t n, uint64_t serial_below, F f) {
  unsigned threads = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (n < serial_below || threads == 1) {
    f(uint64_t(0), n, 0u);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; t++)
    pool.emplace_back([&, t] { f(n * t / threads, n * (t + 1) / threads, t); });
  for (auto& th : pool) th.join();
}

// The first failure over parallel ranges: the lowest position that failed, and its message.
struct FirstFailure {
  std::mutex mu;
  uint64_t at = UINT64_MAX;
  const char* message = nullptr;
  void record(uint64_t where, const char* m) {
    std::lock_guard<std::mutex> lock(mu);
    if (where < at) {
      at = where;
      message = m;
    }
  }
  void raise() const {
    if (message) argument(message);
  }
};

// The structure of the packed index array (bundleIndexLayout): every section consistent with the
// others, so that no kernel can index out of bounds.  Large arrays are checked on host threads;
// the failure reported is the one a serial scan in this order would meet first.
void check_index(const tba_control* c, const uint32_t* index) {
  const uint64_t C = c->cameras, P = c->points, M = c->observations;
  const uint32_t* obs_camera = index;
  const uint32_t* obs_point = index + M;
  const uint32_t* ps = index + 2 * M;
  const uint32_t* cs = ps + P + 1;
  const uint32_t* cam_obs = cs + C + 1;
  const uint32_t* active = cam_obs + M;
  if (ps[0] != 0 || ps[P] != M) argument("Invalid GPU BA index: point offsets do not cover the observations");
  {
    FirstFailure ff;
    parallel_ranges(P, 1u << 16, [&](uint64_t b, uint64_t e, unsigned) {
      for (uint64_t p = b; p < e; p++) {
        if (ps[p + 1] > M) return ff.record(p, "Invalid GPU BA index: point offsets exceed the observations");
        if (ps[p + 1] < ps[p] + 2) return ff.record(p, "Landmarks require at least two observations");
        for (uint64_t i = ps[p]; i < ps[p + 1]; i++)
          if (obs_point[i] != p)
            return ff.record(p, "Invalid GPU BA index: observation point does not match the point offsets");
      }
    });
    ff.raise();
  }
  {
    FirstFailure ff;
    parallel_ranges(M, 1u << 18, [&](uint64_t b, uint64_t e, unsigned) {
      for (uint64_t i = b; i < e; i++)
        if (obs_camera[i] >= C) return ff.record(i, "Invalid GPU BA index: observation camera out of range");
    });
    ff.raise();
  }
  if (cs[0] != 0 || cs[C] != M) argument("Invalid GPU BA index: camera offsets do not cover the observations");
  for (uint64_t cam = 0; cam < C; cam++)
    if (cs[cam + 1] < cs[cam] || cs[cam + 1] > M)
      argument("Invalid GPU BA index: camera offsets decrease or exceed the observations");
  {
    // Each observation may be claimed only by its own camera, so a thread owning a range of
    // cameras is the only one to touch `seen` for their observations.
    std::vector<uint8_t> seen(M, 0);
    FirstFailure ff;
    parallel_ranges(C, M < (1u << 18) ? C + 1 : 1, [&](uint64_t b, uint64_t e, unsigned) {
      for (uint64_t cam = b; cam < e; cam++)
        for (uint64_t k = cs[cam]; k < cs[cam + 1]; k++) {
          const uint32_t i = cam_obs[k];
          if (i >= M || obs_camera[i] != cam || seen[i])
            return ff.record(cam, "Invalid GPU BA index: camera observation lists are not the observations of each camera");
          seen[i] = 1;
        }
    });
    ff.raise();
  }
  uint32_t fixed = 0;
  for (uint64_t cam = 0; cam < C; cam++) {
    if (active[cam] > 1) argument("Invalid GPU BA index: camera activity flags must be 0 or 1");
    fixed += active[cam] == 0;
  }
  if (active[c->anchor] != 0) argument("Invalid GPU BA gauge cameras: the anchor must be fixed");
  if (fixed > 1 && active[c->scale_view] != 0) argument("Local GPU BA scale camera must be fixed");
}

// finiteGpuArray and validateGpuCamera (src/geometry/gpu/bounds.ts:5-26) on the scene array.
void check_scene(const tba_control* c, const double* scene, size_t len) {
  FirstFailure ff;
  parallel_ranges(len, 1u << 18, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t i = b; i < e; i++) {
      const double x = scene[i];
      if (!std::isfinite(x) || std::fabs(x) > 1e9 || (x != 0 && std::fabs(x) < 1e-30))
        return ff.record(i, "GPU BA input exceeds supported coordinate bounds");
    }
  });
  ff.raise();
  const double* k = scene + 12 * size_t(c->cameras) + 3 * size_t(c->points);
  for (uint32_t cam = 0; cam < c->cameras; cam++, k += 6)
    if (!(k[0] > 0 && k[1] > 0) || k[0] < 1e-6 || k[1] < 1e-6 || k[0] > 1e6 || k[1] > 1e6 ||
        std::max(std::fabs(k[2]), std::fabs(k[3])) > 1e9 || std::max(std::fabs(k[4]), std::fabs(k[5])) > 1)
      argument("Camera exceeds the supported GPU geometry bounds");
}

// The O(1) and O(C) parts of check_index and check_scene, on the host, with the message each would
// raise (null where it passes); the O(M) and O(P) parts run on the device after the upload
// (tba_checks.cu), and raise_checks reports the failure that check_index then check_scene, in
// their order, would meet first.
struct HostChecks {
  const char* point_ends = nullptr;     // before the per-point checks
  const char* camera_ends = nullptr;    // after the observation cameras
  const char* camera_offsets = nullptr;
  const char* activity = nullptr;       // after the camera lists
  const char* camera_bounds = nullptr;  // after the scene values
};

HostChecks host_checks(const tba_control* c, const uint32_t* index, const double* scene) {
  HostChecks h;
  const uint64_t C = c->cameras, P = c->points, M = c->observations;
  const uint32_t* ps = index + 2 * M;
  const uint32_t* cs = ps + P + 1;
  const uint32_t* active = cs + C + 1 + M;
  if (ps[0] != 0 || ps[P] != M) h.point_ends = "Invalid GPU BA index: point offsets do not cover the observations";
  if (cs[0] != 0 || cs[C] != M) h.camera_ends = "Invalid GPU BA index: camera offsets do not cover the observations";
  for (uint64_t cam = 0; cam < C && !h.camera_offsets; cam++)
    if (cs[cam + 1] < cs[cam] || cs[cam + 1] > M)
      h.camera_offsets = "Invalid GPU BA index: camera offsets decrease or exceed the observations";
  uint32_t fixed = 0;
  for (uint64_t cam = 0; cam < C && !h.activity; cam++) {
    if (active[cam] > 1) h.activity = "Invalid GPU BA index: camera activity flags must be 0 or 1";
    fixed += active[cam] == 0;
  }
  if (!h.activity && active[c->anchor] != 0) h.activity = "Invalid GPU BA gauge cameras: the anchor must be fixed";
  if (!h.activity && fixed > 1 && active[c->scale_view] != 0) h.activity = "Local GPU BA scale camera must be fixed";
  const double* k = scene + 12 * size_t(C) + 3 * size_t(P);
  for (uint64_t cam = 0; cam < C && !h.camera_bounds; cam++, k += 6)
    if (!(k[0] > 0 && k[1] > 0) || k[0] < 1e-6 || k[1] < 1e-6 || k[0] > 1e6 || k[1] > 1e6 ||
        std::max(std::fabs(k[2]), std::fabs(k[3])) > 1e9 || std::max(std::fabs(k[4]), std::fabs(k[5])) > 1)
      h.camera_bounds = "Camera exceeds the supported GPU geometry bounds";
  return h;
}

void raise_checks(const HostChecks& h, const unsigned long long* keys) {
  const unsigned long long none = ~0ull;
  if (h.point_ends) argument(h.point_ends);
  if (keys[tba::CK_POINTS] != none) {
    static const char* const messages[3] = {"Invalid GPU BA index: point offsets exceed the observations",
                                            "Landmarks require at least two observations",
                                            "Invalid GPU BA index: observation point does not match the point offsets"};
    argument(messages[keys[tba::CK_POINTS] & 3]);
  }
  if (keys[tba::CK_CAMERA] != none) argument("Invalid GPU BA index: observation camera out of range");
  if (h.camera_ends) argument(h.camera_ends);
  if (h.camera_offsets) argument(h.camera_offsets);
  if (keys[tba::CK_LISTS] != none)
    argument("Invalid GPU BA index: camera observation lists are not the observations of each camera");
  if (h.activity) argument(h.activity);
  if (keys[tba::CK_SCENE] != none) argument("GPU BA input exceeds supported coordinate bounds");
  if (h.camera_bounds) argument(h.camera_bounds);
}

// Runs of whole points of at most 32 observations; a longer point is a run of its own.
std::vector<uint32_t> build_tasks(const uint32_t* ps, uint32_t P) {
  std::vector<uint32_t> tasks;
  tasks.reserve(P / 4 + 2);
  uint32_t p = 0;
  while (p < P) {
    tasks.push_back(p);
    uint32_t n = ps[p + 1] - ps[p];
    p++;
    if (n > uint32_t(tba::kTaskObs)) continue;
    while (p < P && n + (ps[p + 1] - ps[p]) <= uint32_t(tba::kTaskObs)) {
      n += ps[p + 1] - ps[p];
      p++;
    }
  }
  tasks.push_back(P);
  return tasks;
}

struct Chunks {
  std::vector<uint32_t> cam, beg, cam_first;
};

// Chunks of each camera's observation list, sized so that the camera pass has a few blocks per SM.
Chunks build_chunks(const uint32_t* cs, uint32_t C, uint32_t M, int sms) {
  uint32_t size = M / std::max(1, 8 * sms);
  size = std::min<uint32_t>(2048, std::max<uint32_t>(128, (size + 127) / 128 * 128));
  Chunks ch;
  for (uint32_t c = 0; c < C; c++) {
    ch.cam_first.push_back(uint32_t(ch.cam.size()));
    const uint32_t n = cs[c + 1] - cs[c];
    const uint32_t k = std::max<uint32_t>(1, (n + size - 1) / size);
    for (uint32_t j = 0; j < k; j++) {
      ch.cam.push_back(c);
      ch.beg.push_back(cs[c] + uint32_t(uint64_t(n) * j / k));
    }
  }
  ch.cam_first.push_back(uint32_t(ch.cam.size()));
  ch.beg.push_back(cs[C]);
  return ch;
}

// Reads the first 40 state words into the pinned buffer; returns word `word`.
double read_word(tba_device* d, const double* state, int word) {
  CUDA_TRY(cudaMemcpyAsync(d->pinned, state, 40 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  return d->pinned[word];
}

// Makes `loop` a graph of one while node whose body `capture(handle, stream)` records (returning its
// kernel count): kept when it was built for the same `key` (the launch parameters its kernels bake),
// built again otherwise.
template <class Capture>
cudaError_t build_device_loop(PcgLoop& loop, const void* key, size_t key_len, cudaStream_t s, Capture capture) {
  const char* bytes = static_cast<const char*>(key);
  if (loop.exec && loop.key.size() == key_len && std::memcmp(loop.key.data(), bytes, key_len) == 0)
    return cudaSuccess;
  loop.release();
  cudaError_t e = cudaGraphCreate(&loop.graph, 0);
  if (e != cudaSuccess) return e;
  // The condition starts at 1 at every launch: the body runs at least once (its kernels are no-ops
  // when the PCG is already stopped), then the body's last kernel decides.
  cudaGraphConditionalHandle handle;
  e = cudaGraphConditionalHandleCreate(&handle, loop.graph, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = handle;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, loop.graph, nullptr, 0, &np);
  if (e != cudaSuccess) return e;
  e = cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  loop.body_kernels = capture(handle, s);
  const cudaError_t launched = cudaGetLastError();
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(s, &captured);
  if (launched != cudaSuccess) return launched;
  if (e != cudaSuccess) return e;
  e = cudaGraphInstantiate(&loop.exec, loop.graph, 0);
  if (e != cudaSuccess) {
    loop.exec = nullptr;
    return e;
  }
  loop.key.assign(bytes, bytes + key_len);
  return cudaSuccess;
}

// The grid engine's PCG loop for the launch parameters `q`.
cudaError_t build_pcg_loop(PcgLoop& loop, const tba::Params& q, cudaStream_t s) {
  return build_device_loop(loop, &q, sizeof q, s, [&](cudaGraphConditionalHandle handle, cudaStream_t cs) {
    tba::Params body = q;
    body.pcg_loop = handle;
    tba::launch_product(body, cs);
    tba::launch_product_finish(body, cs);
    tba::launch_pcg_loop_next(body, cs);
    return uint32_t(q.factored ? 4 : 5) + 1;
  });
}

// The adjoint's PCG loop: the step kernels read neither the damping nor the right-hand side's mode,
// so one graph serves every linear solve of a vjp (and of the next call with the same arrays).
cudaError_t build_adjoint_loop(PcgLoop& loop, const tba::AdjParams& a, cudaStream_t s) {
  tba::AdjParams key = a;
  key.mu = 0;
  key.rhs_mode = 0;
  key.loop = 0;
  return build_device_loop(loop, &key, sizeof key, s, [&](cudaGraphConditionalHandle handle, cudaStream_t cs) {
    tba::AdjParams body = key;
    body.loop = handle;
    const uint32_t step = tba::adj_launch_pcg_step(body, cs);
    return step + tba::adj_launch_loop_next(body, cs);
  });
}

// Whether a device-side loop was built.  A driver that cannot build conditional graph nodes makes
// the handle run every later PCG from the host (the same kernels, launched in chunks); any other
// failure is the call's error.
bool device_loop_ready(tba_device* d, PcgLoop& loop, cudaError_t built) {
  if (built == cudaSuccess) return true;
  loop.release();
  if (built == cudaErrorNotSupported || built == cudaErrorStreamCaptureUnsupported) {
    cudaGetLastError();
    d->host_pcg_only = true;
    return false;
  }
  throw Fail{TBA_ERROR_CUDA, std::string("device PCG loop: ") + cudaGetErrorString(built)};
}

cudaEvent_t event(tba_device* d, size_t k) {
  while (d->events.size() <= k) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    d->events.push_back(e);
  }
  return d->events[k];
}

// The host-side schedules of one problem's index: warp tasks (with their first observations),
// camera chunks and the number of fixed cameras.
struct HostPlan {
  std::vector<uint32_t> tasks, task_obs;
  Chunks chunks;
  uint32_t fixed = 0;
  // The arrays a solve uploads, in the order of a resident scene's device copy.
  std::vector<const std::vector<uint32_t>*> sections() const {
    return {&tasks, &task_obs, &chunks.cam, &chunks.beg, &chunks.cam_first};
  }
};

HostPlan make_plan(const tba_control* ctl, const uint32_t* index, int sms) {
  const uint32_t C = ctl->cameras, P = ctl->points, M = ctl->observations;
  const uint32_t* ps = index + 2 * size_t(M);
  const uint32_t* cs = ps + P + 1;
  const uint32_t* active = cs + C + 1 + M;
  HostPlan plan;
  plan.tasks = build_tasks(ps, P);
  plan.task_obs.resize(plan.tasks.size());
  for (size_t t = 0; t < plan.tasks.size(); t++) plan.task_obs[t] = ps[plan.tasks[t]];
  plan.chunks = build_chunks(cs, C, M, sms);
  for (uint32_t c = 0; c < C; c++) plan.fixed += active[c] == 0;
  return plan;
}

// Where a solve reads its problem and where it leaves the solution.  With `device_source` the
// scene and index are device pointers (a resident scene) and `plan` is given; `writeback` (device)
// receives the solved poses and points; `output` may be null and `state` (host) receives the
// result's state words.
struct SolveIO {
  bool device_source = false;
  const HostPlan* plan = nullptr;
  double* writeback = nullptr;
  double* state = nullptr;
  // When set, the O(M) checks run on the device right after the upload and a failure is raised
  // (with these host-side results, in the serial order) before any solver kernel runs.
  const HostChecks* checks = nullptr;
  double* check_ms = nullptr;  // receives the device checks' host wall time
  // With `plan`: a device copy of its arrays (HostPlan::sections, concatenated), copied on the
  // device instead of uploaded.
  const uint32_t* plan_dev = nullptr;
};

void solve(tba_device* d, const tba_control* ctl, const double* scene, const uint32_t* index,
           double* output, tba_report* report, const SolveIO& io = SolveIO()) {
  const auto wall0 = std::chrono::steady_clock::now();
  const uint32_t C = ctl->cameras, P = ctl->points, M = ctl->observations;
  const bool shared = ctl->shared_focal != 0;
  const uint32_t m = 6 * C + (shared ? 1 : 0);
  // The host schedules (warp tasks, camera chunks) are built while the problem arrays upload: the
  // workspace is laid out with bounds of their sizes (at most P + 1 task starts; at most
  // C + M / 128 + 1 chunks, chunks being at least 128 observations long).  A problem whose camera
  // offsets fail the host checks gets no schedule; its checks fail before any kernel runs.
  const bool plannable = !io.checks || (!io.checks->camera_ends && !io.checks->camera_offsets);
  const uint64_t max_tasks = io.plan ? io.plan->tasks.size() : uint64_t(P) + 1;
  const uint64_t max_chunks = io.plan ? io.plan->chunks.cam.size() : uint64_t(C) + M / 128 + 1;

  Params p{};
  p.C = C;
  p.P = P;
  p.M = M;
  p.D = ctl->directional_points;
  p.m = m;
  p.anchor = ctl->anchor;
  p.scale_view = ctl->scale_view;
  p.shared = shared;
  p.huber = ctl->huber;
  p.tol = ctl->cg_tolerance;
  p.stall = ctl->stall_tolerance;
  // The mixed form's inner PCG runs stop at a relative residual the FP32 product can reach; the
  // FP64 refinement then measures the true residual against the caller's tolerance.
  p.tol_inner = ctl->precision == TBA_PRECISION_MIXED ? std::max(ctl->cg_tolerance, 1e-6) : ctl->cg_tolerance;
  const uint32_t max_task_blocks = std::max<uint32_t>(1, 4 * uint32_t(d->sms));
  const uint32_t fblocks = tba::product_finish_blocks(p);
  // The one-pass product over stored factors when its camera sums fit shared memory; the two-pass
  // recompute form otherwise.  The mixed form stores FP32 factors for its PCG and FP64 factors for
  // its refinement residual, its FP64 tail and the back-substitution.
  const bool mixed = ctl->precision == TBA_PRECISION_MIXED;
  p.factored = m <= tba::product_max_unknowns();
  p.Mpad = (M + 31) / 32 * 32;
  const size_t factor_bytes = p.factored ? size_t(tba::kFactors) * p.Mpad * 8 : 0;
  const size_t factor32_bytes = p.factored && mixed ? size_t(tba::kFactors) * p.Mpad * 4 : 0;
  p.F = nullptr;
  p.F32 = mixed && p.factored ? reinterpret_cast<float*>(1) : nullptr;  // set below; selects the occupancy query
  const int per_sm = p.factored ? tba::product_blocks_per_sm(p) : 1;
  const uint32_t max_prod_blocks = std::max<uint32_t>(1, uint32_t(per_sm * d->sms));
  Layout L;
  const size_t o_poses = L.take<double>(12 * size_t(C)), o_points = L.take<double>(3 * size_t(P)),
               o_cams = L.take<double>(6 * size_t(C)), o_pixels = L.take<double>(2 * size_t(M)),
               o_tposes = L.take<double>(12 * size_t(C)), o_tpoints = L.take<double>(3 * size_t(P)),
               o_index = L.take<uint32_t>(3 * size_t(M) + P + 2 * size_t(C) + 2),
               o_pblk32 = L.take<float>(mixed && p.factored ? 6 * size_t(P) : 0),
               o_tasks = L.take<uint32_t>(max_tasks), o_tobs = L.take<uint32_t>(max_tasks),
               o_ccam = L.take<uint32_t>(max_chunks),
               o_cbeg = L.take<uint32_t>(max_chunks + 1), o_cfirst = L.take<uint32_t>(C + 1),
               o_rlim = L.take<double>(C), o_cmp = L.take<uint32_t>(M), o_cmx = L.take<double>(2 * size_t(M)),
               o_pblk = L.take<double>(12 * size_t(P)), o_y = L.take<double>(4 * size_t(P)),
               o_cprod = L.take<double>(8 * max_chunks), o_F = L.take<char>(factor_bytes),
               o_F32 = L.take<char>(factor32_bytes),
               o_pw = L.take<double>(6 * size_t(C)), o_xw = L.take<double>(6 * size_t(C)),
               o_acc = L.take<double>(p.factored ? size_t(max_prod_blocks) * m : 0), o_U = L.take<double>(21 * size_t(C)),
               o_Minv = L.take<double>(36 * size_t(C)), o_rhs = L.take<double>(6 * size_t(C)),
               o_hcf = L.take<double>(6 * size_t(C)),
               o_chunk = L.take<double>(size_t(tba::kCameraPartials) * max_chunks),
               o_vec = L.take<double>(5 * size_t(m)), o_blk = L.take<double>(4 * size_t(fblocks)),
               o_scal = L.take<double>(size_t(tba::kScalarPartials) * max_task_blocks),
               o_cost = L.take<double>(4 * size_t(max_task_blocks)), o_ticket = L.take<uint32_t>(8),
               o_state = L.take<double>(tba::S_WORDS), o_out = L.take<double>(12 * size_t(C) + 3 * size_t(P) + 27),
               o_keys = L.take<unsigned long long>(tba::CK_WORDS),
               o_diag = L.take<double>((ctl->flags & TBA_FLAG_PRODUCT_ERROR) ? 2 * size_t(m) : 0);
  if (d->capacity < L.bytes) {
    if (d->arena) CUDA_TRY(cudaFree(d->arena));
    d->arena = nullptr;
    d->capacity = 0;
    size_t free_bytes = 0, total_bytes = 0;
    CUDA_TRY(cudaMemGetInfo(&free_bytes, &total_bytes));
    if (L.bytes > free_bytes)
      throw Fail{TBA_ERROR_BUDGET, "GPU BA needs " + std::to_string(L.bytes) +
                                       " bytes of device memory, more than the working budget of " +
                                       std::to_string(free_bytes) + " bytes"};
    CUDA_TRY(cudaMalloc(&d->arena, L.bytes));
    d->capacity = L.bytes;
  }
  char* a = d->arena;
  auto D = [&](size_t off) { return reinterpret_cast<double*>(a + off); };
  auto U32 = [&](size_t off) { return reinterpret_cast<uint32_t*>(a + off); };
  p.poses = D(o_poses);
  p.points = D(o_points);
  p.cams = D(o_cams);
  p.pixels = D(o_pixels);
  p.tposes = D(o_tposes);
  p.tpoints = D(o_tpoints);
  uint32_t* dindex = U32(o_index);
  p.obs_camera = dindex;
  p.obs_point = dindex + M;
  p.point_start = dindex + 2 * size_t(M);
  p.camera_start = p.point_start + P + 1;
  p.camera_obs = p.camera_start + C + 1;
  p.active = p.camera_obs + M;
  p.pblk32 = mixed && p.factored ? reinterpret_cast<float*>(a + o_pblk32) : nullptr;
  p.tasks = U32(o_tasks);
  p.task_obs = U32(o_tobs);
  p.chunk_cam = U32(o_ccam);
  p.chunk_beg = U32(o_cbeg);
  p.cam_chunk = U32(o_cfirst);
  p.rlim = D(o_rlim);
  p.cm_point = U32(o_cmp);
  p.cm_pixel = D(o_cmx);
  p.pblk = D(o_pblk);
  p.y = D(o_y);
  p.chunk_prod = D(o_cprod);
  p.F = p.factored ? D(o_F) : nullptr;
  p.F32 = p.factored && mixed ? reinterpret_cast<float*>(a + o_F32) : nullptr;
  p.pw = D(o_pw);
  p.xw = D(o_xw);
  p.acc_part = D(o_acc);
  p.camU = D(o_U);
  p.camMinv = D(o_Minv);
  p.camRhs = D(o_rhs);
  p.camHcf = D(o_hcf);
  p.chunk_part = D(o_chunk);
  double* vec = D(o_vec);
  p.x = vec;
  p.r = vec + m;
  p.p = vec + 2 * size_t(m);
  p.Sp = vec + 3 * size_t(m);
  p.z = vec + 4 * size_t(m);
  p.blk_part = D(o_blk);
  p.scal_part = D(o_scal);
  p.cost_part = D(o_cost);
  p.ticket = U32(o_ticket);
  p.state = D(o_state);
  p.output = D(o_out);

  cudaStream_t s = d->stream;
  size_t ev = 0;
  cudaEvent_t e_start = event(d, ev++), e_up = event(d, ev++), e_solved = event(d, ev++), e_down = event(d, ev++);
  uint64_t h2d = 0;
  // Problem arrays: host-to-device, or device-to-device from a resident scene.
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, io.device_source ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    if (!io.device_source) h2d += bytes;
  };
  auto up_host = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    h2d += bytes;
  };
  CUDA_TRY(cudaEventRecord(e_start, s));
  up(p.poses, scene, 12 * sizeof(double) * C);
  up(p.points, scene + 12 * size_t(C), 3 * sizeof(double) * P);
  up(const_cast<double*>(p.cams), scene + 12 * size_t(C) + 3 * size_t(P), 6 * sizeof(double) * C);
  up(const_cast<double*>(p.pixels), scene + 18 * size_t(C) + 3 * size_t(P), 2 * sizeof(double) * M);
  up(dindex, index, sizeof(uint32_t) * (3 * size_t(M) + P + 2 * size_t(C) + 2));
  // The schedules, built on the host while the copies above run.
  HostPlan own;
  if (!io.plan && plannable) own = make_plan(ctl, index, d->sms);
  const HostPlan& plan = io.plan ? *io.plan : own;
  const std::vector<uint32_t>& tasks = plan.tasks;
  const Chunks& chunks = plan.chunks;
  const uint32_t ntasks = tasks.empty() ? 0 : uint32_t(tasks.size() - 1), nchunks = uint32_t(chunks.cam.size());
  if (plannable) {
    if (tasks.size() > max_tasks || nchunks > max_chunks) throw Fail{TBA_ERROR_INTERNAL, "GPU BA schedule exceeds its bound"};
    // The plan's arrays: from the host, or from a resident scene's device copy.
    const size_t dst[5] = {o_tasks, o_tobs, o_ccam, o_cbeg, o_cfirst};
    size_t at = 0;
    const auto sections = plan.sections();
    for (size_t k = 0; k < sections.size(); k++) {
      const std::vector<uint32_t>& v = *sections[k];
      if (!v.empty()) {
        if (io.plan_dev)
          CUDA_TRY(cudaMemcpyAsync(U32(dst[k]), io.plan_dev + at, sizeof(uint32_t) * v.size(), cudaMemcpyDeviceToDevice, s));
        else
          up_host(U32(dst[k]), v.data(), sizeof(uint32_t) * v.size());
      }
      at += v.size();
    }
  }
  p.normalize_scale = plan.fixed == 1;
  p.ntasks = ntasks;
  p.nchunks = nchunks;
  p.task_blocks = std::max<uint32_t>(1, std::min<uint32_t>(max_task_blocks, (ntasks + 7) / 8));
  p.prod_blocks = std::max<uint32_t>(1, std::min<uint32_t>(max_prod_blocks, (ntasks + 15) / 16));
  CUDA_TRY(cudaEventRecord(e_up, s));
  if (io.checks) {
    const auto c0 = std::chrono::steady_clock::now();
    tba::CheckParams cp{};
    cp.C = C;
    cp.P = P;
    cp.M = M;
    cp.index = dindex;
    cp.seg[0] = p.poses;
    cp.seg[1] = p.points;
    cp.seg[2] = p.cams;
    cp.seg[3] = p.pixels;
    cp.base[0] = 0;
    cp.len[0] = 12 * uint64_t(C);
    cp.base[1] = cp.len[0];
    cp.len[1] = 3 * uint64_t(P);
    cp.base[2] = cp.base[1] + cp.len[1];
    cp.len[2] = 6 * uint64_t(C);
    cp.base[3] = cp.base[2] + cp.len[2];
    cp.len[3] = 2 * uint64_t(M);
    cp.claims = p.cm_point;  // scratch until k_setup writes the camera-major point index
    cp.keys = reinterpret_cast<unsigned long long*>(a + o_keys);
    cp.lists = !io.checks->camera_ends && !io.checks->camera_offsets;
    CUDA_TRY(tba::launch_checks(cp, d->sms, s));
    CUDA_TRY(cudaMemcpyAsync(d->pinned, cp.keys, tba::CK_WORDS * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    unsigned long long keys[tba::CK_WORDS];
    std::memcpy(keys, d->pinned, sizeof keys);
    if (io.check_ms)
      *io.check_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - c0).count();
    raise_checks(*io.checks, keys);
    if (!plannable) throw Fail{TBA_ERROR_INTERNAL, "GPU BA checks passed a problem without a schedule"};
  }

  uint32_t launches = 0, lm_done = 0, refinements = 0, fp64_iterations = 0;
  // Mixed form: once an LM iteration's PCG needed the FP64 tail, the rest of the solve solves on the
  // FP64 product (the FP32 product does not reach the tolerance on such a system, and its restarts
  // would only add PCG runs).
  bool fp64_only = false;
  // Event pairs around the Schur products; after the solve, only the products that ran PCG steps
  // (the first `steps` of each LM iteration; later ones are guarded no-ops) count.
  std::vector<std::pair<size_t, size_t>> product_events;
  std::vector<std::pair<size_t, uint32_t>> product_spans;  // (first event pair, real steps) per LM iteration
  const bool time_products = (ctl->flags & TBA_FLAG_TIME_PRODUCTS) != 0;
  const bool host_loop = time_products || (ctl->flags & TBA_FLAG_HOST_PCG_LOOP) != 0;
  // Kernels per step of the device-side PCG loop launched last, while its step count is unread.
  uint32_t loop_kernels = 0;
  tba::launch_initialize(p, s);
  tba::launch_cost(p, s);
  tba::launch_finish_metrics(p, s);
  launches += 4;
  CUDA_TRY(cudaGetLastError());
  bool lm_active = read_word(d, p.state, tba::S_ACTIVE) != 0;
  // The mixed form's FP64 tail: the one-pass product over the FP64 factors (the two-pass recompute
  // product when the engine keeps no factors).
  tba::Params tail = p;
  tail.F32 = nullptr;
  tail.tol_inner = 0;  // the tail stops at the solve's own tolerance
  double product_error_max = 0, product_error_norm = 0;
  for (uint32_t it = 0; it < ctl->iterations && lm_active; it++) {
    tba::launch_point_pass(p, s);
    tba::launch_camera_pass(p, s);
    tba::launch_camera_finish(p, s);
    tba::launch_pcg_init(p, s);
    launches += 4;
    if (it == 0 && (ctl->flags & TBA_FLAG_PRODUCT_ERROR) && read_word(d, p.state, tba::S_CG_ACTIVE) != 0) {
      // The solve's own product and the FP64 two-pass product on the first PCG direction.
      double* own = D(o_diag);
      double* ref = own + m;
      tba::Params fp64 = p;
      fp64.F32 = nullptr;
      fp64.factored = 0;
      tba::launch_product(p, s);
      tba::launch_product_rows(p, own, s);
      tba::launch_product(fp64, s);
      tba::launch_product_rows(fp64, ref, s);
      launches += p.factored ? 5 : 6;
      CUDA_TRY(cudaGetLastError());
      std::vector<double> a(m), b(m);
      CUDA_TRY(cudaMemcpyAsync(a.data(), own, m * sizeof(double), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaMemcpyAsync(b.data(), ref, m * sizeof(double), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      double dmax = 0, bmax = 0, d2 = 0, b2 = 0;
      for (uint32_t j = 0; j < m; j++) {
        const double e = a[j] - b[j];
        dmax = std::max(dmax, std::fabs(e));
        bmax = std::max(bmax, std::fabs(b[j]));
        d2 += e * e;
        b2 += b[j] * b[j];
      }
      product_error_max = bmax > 0 ? dmax / bmax : dmax;
      product_error_norm = b2 > 0 ? std::sqrt(d2 / b2) : std::sqrt(d2);
    }
    // PCG runs.  By default a run is one launch of the form's device-side PCG loop, which ends on the
    // device; its step count is taken from the next state read (every run is followed by one in the
    // same LM iteration).  With the host loop (timed products, or on request) the steps run in
    // chunks of guarded iterations, events around each product when timed; the read after each
    // chunk only ends the loop early.
    uint32_t done = 0, steps_before = 0;
    // `q` selects the product: the engine's own (FP32 factors in the mixed form), or the FP64
    // product of the mixed form's tail.  Only the engine's own products are timed.
    auto run_pcg = [&](uint32_t budget, const tba::Params& q, bool timed) {
      if (!host_loop && !d->host_pcg_only) {
        if (budget <= done) return;
        PcgLoop& loop = d->pcg_loops[&q == &p ? 0 : 1];
        if (device_loop_ready(d, loop, build_pcg_loop(loop, q, s))) {
          tba::launch_pcg_loop_begin(q, budget - done, s);
          launches++;
          CUDA_TRY(cudaGraphLaunch(loop.exec, s));
          loop_kernels = loop.body_kernels;
          return;
        }
      }
      const size_t first_pair = product_events.size();
      uint32_t chunk = 8;
      while (done < budget) {
        const uint32_t k = std::min(chunk, budget - done);
        for (uint32_t j = 0; j < k; j++) {
          if (time_products && timed) {
            const size_t e0 = ev++, e1 = ev++;
            CUDA_TRY(cudaEventRecord(event(d, e0), s));
            tba::launch_product(q, s);
            CUDA_TRY(cudaEventRecord(event(d, e1), s));
            product_events.emplace_back(e0, e1);
          } else {
            tba::launch_product(q, s);
          }
          tba::launch_product_finish(q, s);
          launches += q.factored ? 4 : 5;
        }
        CUDA_TRY(cudaGetLastError());
        done += k;
        if (done >= budget || read_word(d, p.state, tba::S_CG_ACTIVE) == 0) break;
        chunk = std::min<uint32_t>(2 * chunk, 32);
      }
      // The products of this run that did PCG steps (later launches of a chunk are no-ops).
      const uint32_t steps = uint32_t(read_word(d, p.state, tba::S_CG_SOLVE_STEPS));
      if (time_products && timed) product_spans.emplace_back(first_pair, steps - steps_before);
      steps_before = steps;
    };
    // After a state read: the steps of the device-side PCG loop that ran before it.
    auto account_loop = [&]() {
      if (!loop_kernels) return;
      const uint32_t iters = uint32_t(d->pinned[tba::S_LOOP_ITERS]);
      done += iters;
      launches += iters * loop_kernels;
      loop_kernels = 0;
    };
    if (fp64_only) fp64_iterations++;
    run_pcg(ctl->max_cg, fp64_only ? tail : p, !fp64_only);
    // Mixed form: FP64 iterative refinement.  The true (FP64) residual of the FP32-product solution
    // restarts the PCG from that solution when it is above the tolerance; a restarted run (with an
    // iteration budget of its own) uses the FP32 product again and is checked again.  Only a
    // solution still above the tolerance after kFp32Restarts such runs is finished on the FP64
    // product, which resolves what FP32 factors cannot on badly conditioned systems.
    if (mixed && !fp64_only) {
      constexpr int kFp32Restarts = 2;
      for (int round = 0;; round++) {
        tba::launch_refine(p, s);
        launches += 4;
        CUDA_TRY(cudaGetLastError());
        const bool active = read_word(d, p.state, tba::S_CG_ACTIVE) != 0;
        account_loop();
        if (!active) break;
        refinements++;
        if (round < kFp32Restarts) {
          run_pcg(done + ctl->max_cg, p, true);
          continue;
        }
        run_pcg(done + ctl->max_cg, tail, false);
        fp64_only = true;
        break;
      }
    }
    tba::launch_update_cameras(p, s);
    tba::launch_update_points(p, s);
    tba::launch_accept(p, s);
    tba::launch_commit(p, s);
    launches += 4;
    CUDA_TRY(cudaGetLastError());
    lm_done++;
    CUDA_TRY(cudaMemcpyAsync(d->pinned, p.state, 40 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    account_loop();
    lm_active = d->pinned[tba::S_ACTIVE] != 0;
  }
  tba::launch_pack(p, s);
  launches++;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaEventRecord(e_solved, s));
  const size_t out_len = 12 * size_t(C) + 3 * size_t(P) + 26 + (shared ? 1 : 0);
  const size_t state_len = 26 + (shared ? 1 : 0);
  size_t d2h = 0;
  if (output) {
    CUDA_TRY(cudaMemcpyAsync(output, p.output, out_len * sizeof(double), cudaMemcpyDeviceToHost, s));
    d2h += out_len * sizeof(double);
  }
  if (io.state) {
    CUDA_TRY(cudaMemcpyAsync(io.state, p.output + 12 * size_t(C) + 3 * size_t(P), state_len * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    d2h += state_len * sizeof(double);
  }
  if (io.writeback) {
    CUDA_TRY(cudaMemcpyAsync(io.writeback, p.poses, 12 * sizeof(double) * C, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(io.writeback + 12 * size_t(C), p.points, 3 * sizeof(double) * P, cudaMemcpyDeviceToDevice, s));
  }
  CUDA_TRY(cudaEventRecord(e_down, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    std::memset(report, 0, sizeof *report);
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e_start, e_up));
    report->upload_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e_up, e_solved));
    report->solve_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e_solved, e_down));
    report->download_ms = ms;
    double total = 0;
    uint32_t counted = 0;
    for (size_t k = 0; k < product_spans.size(); k++) {
      const size_t end = k + 1 < product_spans.size() ? product_spans[k + 1].first : product_events.size();
      const size_t last = std::min(end, product_spans[k].first + product_spans[k].second);
      for (size_t j = product_spans[k].first; j < last; j++) {
        CUDA_TRY(cudaEventElapsedTime(&ms, d->events[product_events[j].first], d->events[product_events[j].second]));
        total += ms;
        counted++;
      }
    }
    report->product_ms = total;
    report->product_launches = counted;
    report->h2d_bytes = h2d;
    report->d2h_bytes = d2h;
    report->kernel_launches = launches;
    report->lm_iterations = lm_done;
    const double* st = output ? output + 12 * size_t(C) + 3 * size_t(P) : io.state;
    report->cg_iterations = st ? uint32_t(st[tba::S_CG_STEPS]) : 0;
    report->engine = p.factored ? 0 : 1;
    report->product_blocks = p.factored ? p.prod_blocks : 0;
    report->refinements = uint32_t(refinements);
    report->fp64_iterations = fp64_iterations;
    report->product_error_max = product_error_max;
    report->product_error_norm = product_error_norm;
    report->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
  }
}

// ---- batched local-window solves ------------------------------------------------------------------

// The caller's arrays of one batched problem, checked as tba_bundle_adjust checks a problem.
tba_control batch_problem_control(const tba_batch_control* bc, const tba_batch_problem& q) {
  tba_control c{};
  c.cameras = q.cameras;
  c.points = q.points;
  c.directional_points = 0;
  c.observations = q.observations;
  c.anchor = q.anchor;
  c.scale_view = q.scale_view;
  c.iterations = bc->iterations;
  c.max_cg = bc->max_cg;
  c.shared_focal = bc->shared_focal;
  c.precision = bc->precision;
  c.flags = 0;
  c.huber = bc->huber;
  c.cg_tolerance = bc->cg_tolerance;
  c.stall_tolerance = bc->stall_tolerance;
  return c;
}

void solve_batch(tba_device* d, const tba_batch_control* bc, const tba_batch_problem* probs, uint32_t count,
                 const double* scene, size_t scene_len, const uint32_t* index, size_t index_len, double* output,
                 size_t output_len, tba_batch_report* report) {
  const auto wall0 = std::chrono::steady_clock::now();
  const bool shared = bc->shared_focal != 0, mixed = bc->precision == TBA_PRECISION_MIXED;
  const uint32_t max_cams = tba::batch_max_cameras();
  uint32_t Cmax = 2;
  std::vector<uint32_t> tasks;
  std::vector<uint64_t> task_first(count), task_count(count);
  // Each problem is checked and scheduled on its own; the problems are spread over host threads and
  // the failure reported is the one of the first failing problem, as a loop in order would report.
  std::vector<std::vector<uint32_t>> problem_tasks(count);
  std::mutex fail_mu;
  uint32_t fail_at = UINT32_MAX;
  Fail first_fail{TBA_OK, ""};
  parallel_ranges(count, 2, [&](uint64_t b, uint64_t e, unsigned) {
    for (uint64_t k = b; k < e; k++) {
      try {
        const tba_batch_problem& q = probs[k];
        const tba_control c = batch_problem_control(bc, q);
        check_control(&c);
        if (q.reserved != 0) argument("Invalid GPU BA batch: reserved field must be 0");
        if (q.cameras > max_cams)
          argument("Batched GPU BA problem has " + std::to_string(q.cameras) +
                   " cameras; the block solver takes at most " + std::to_string(max_cams));
        if (uint64_t(3) * q.observations + q.points + 2ull * q.cameras + 2 > 0xffffffffull)
          argument("GPU BA scene dimensions exceed integer index bounds");
        if (q.scene_offset > scene_len || scene_len - q.scene_offset < tba_scene_size(&c))
          argument("Invalid GPU BA batch: a scene lies outside the scene array");
        if (q.index_offset > index_len || index_len - q.index_offset < tba_index_size(&c))
          argument("Invalid GPU BA batch: an index lies outside the index array");
        if (q.output_offset > output_len || output_len - q.output_offset < tba_output_size(&c))
          argument("Invalid GPU BA batch: a result record lies outside the output array");
        check_index(&c, index + q.index_offset);
        check_scene(&c, scene + q.scene_offset, tba_scene_size(&c));
        problem_tasks[k] = build_tasks(index + q.index_offset + 2 * size_t(q.observations), q.points);
      } catch (const Fail& f) {
        std::lock_guard<std::mutex> lock(fail_mu);
        if (k < fail_at) {
          fail_at = uint32_t(k);
          first_fail = f;
        }
        return;
      }
    }
  });
  if (fail_at != UINT32_MAX) throw first_fail;
  for (uint32_t k = 0; k < count; k++) {
    const std::vector<uint32_t>& t = problem_tasks[k];
    task_first[k] = tasks.size();
    task_count[k] = t.size() - 1;
    tasks.insert(tasks.end(), t.begin(), t.end());
    Cmax = std::max(Cmax, probs[k].cameras);
  }
  // Result records must not overlap: the device writes each one whole.
  std::vector<uint32_t> by_out(count);
  std::iota(by_out.begin(), by_out.end(), 0u);
  std::sort(by_out.begin(), by_out.end(), [&](uint32_t a, uint32_t b) { return probs[a].output_offset < probs[b].output_offset; });
  for (uint32_t j = 1; j < count; j++) {
    const tba_batch_problem& prev = probs[by_out[j - 1]];
    const tba_control pc = batch_problem_control(bc, prev);
    if (prev.output_offset + tba_output_size(&pc) > probs[by_out[j]].output_offset)
      argument("Invalid GPU BA batch: result records overlap");
  }
  // Largest problems first (longest-processing-time order for the persistent blocks).
  std::vector<uint32_t> order(count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return uint64_t(probs[a].observations) * probs[a].cameras > uint64_t(probs[b].observations) * probs[b].cameras;
  });

  // Device layout: the caller's arrays as they are, then the schedule and the workspace.
  Layout L;
  const size_t factor_size = mixed ? 4 : 8;
  const size_t o_scene = L.take<double>(scene_len), o_index = L.take<uint32_t>(index_len),
               o_out = L.take<double>(output_len), o_tasks = L.take<uint32_t>(tasks.size()),
               o_desc = L.take<tba::BatchProblem>(count), o_desc64 = L.take<tba::BatchProblem>(mixed ? count : 0),
               o_order = L.take<uint32_t>(count),
               o_queue = L.take<uint32_t>(4);
  std::vector<size_t> o_tp(count), o_pb(count), o_F(count), o_F64(count);
  uint64_t M_total = 0;
  for (uint32_t k = 0; k < count; k++) {
    const tba_batch_problem& q = probs[k];
    const size_t Mpad = (size_t(q.observations) + 31) / 32 * 32;
    o_tp[k] = L.take<double>(3 * size_t(q.points));
    o_pb[k] = L.take<double>(12 * size_t(q.points));
    o_F[k] = L.take<char>(tba::kFactors * Mpad * factor_size);
    o_F64[k] = L.take<char>(mixed ? tba::kFactors * Mpad * sizeof(double) : 0);  // the mixed form's FP64 copy
    M_total += q.observations;
  }
  if (d->batch_capacity < L.bytes) {
    if (d->batch_graph) {
      cudaGraphExecDestroy(d->batch_graph);
      d->batch_graph = nullptr;
      d->batch_key.clear();
    }
    if (d->batch_arena) CUDA_TRY(cudaFree(d->batch_arena));
    d->batch_arena = nullptr;
    d->batch_capacity = 0;
    size_t free_bytes = 0, total_bytes = 0;
    CUDA_TRY(cudaMemGetInfo(&free_bytes, &total_bytes));
    if (L.bytes > free_bytes)
      throw Fail{TBA_ERROR_BUDGET, "GPU BA batch needs " + std::to_string(L.bytes) +
                                       " bytes of device memory, more than the working budget of " +
                                       std::to_string(free_bytes) + " bytes"};
    CUDA_TRY(cudaMalloc(&d->batch_arena, L.bytes));
    d->batch_capacity = L.bytes;
  }
  char* a = d->batch_arena;
  const double* dscene = reinterpret_cast<const double*>(a + o_scene);
  const uint32_t* dindex = reinterpret_cast<const uint32_t*>(a + o_index);
  double* dout = reinterpret_cast<double*>(a + o_out);
  const uint32_t* dtasks = reinterpret_cast<const uint32_t*>(a + o_tasks);
  std::vector<tba::BatchProblem> desc(count);
  for (uint32_t k = 0; k < count; k++) {
    const tba_batch_problem& q = probs[k];
    tba::BatchProblem& b = desc[k];
    const uint32_t C = q.cameras, P = q.points, M = q.observations;
    b.C = C;
    b.P = P;
    b.M = M;
    b.ntasks = uint32_t(task_count[k]);
    b.anchor = q.anchor;
    b.scale_view = q.scale_view;
    const uint32_t* act = index + q.index_offset + 3 * size_t(M) + P + C + 2;
    uint32_t fixed = 0;
    for (uint32_t c = 0; c < C; c++) fixed += act[c] == 0;
    b.normalize_scale = fixed == 1;
    b.Mpad = uint32_t((size_t(M) + 31) / 32 * 32);
    const double* s = dscene + q.scene_offset;
    b.poses0 = s;
    b.points0 = s + 12 * size_t(C);
    b.cams = s + 12 * size_t(C) + 3 * size_t(P);
    b.pixels = s + 18 * size_t(C) + 3 * size_t(P);
    const uint32_t* x = dindex + q.index_offset;
    b.obs_camera = x;
    b.obs_point = x + M;
    b.point_start = x + 2 * size_t(M);
    b.camera_start = b.point_start + P + 1;
    b.camera_obs = b.camera_start + C + 1;
    b.active = b.camera_obs + M;
    b.tasks = dtasks + task_first[k];
    b.tpoints = reinterpret_cast<double*>(a + o_tp[k]);
    b.pblk = reinterpret_cast<double*>(a + o_pb[k]);
    b.F = a + o_F[k];
    b.F64 = mixed ? reinterpret_cast<double*>(a + o_F64[k]) : nullptr;
    b.output = dout + q.output_offset;
    b.points = b.output + 12 * size_t(C);
  }

  tba::BatchArgs args{};
  args.problems = reinterpret_cast<const tba::BatchProblem*>(a + o_desc);
  args.order = reinterpret_cast<const uint32_t*>(a + o_order);
  args.queue = reinterpret_cast<uint32_t*>(a + o_queue);
  args.count = count;
  args.Cmax = Cmax;
  args.iterations = bc->iterations;
  args.max_cg = bc->max_cg;
  args.huber = bc->huber;
  args.tol = bc->cg_tolerance;
  args.tol_inner = mixed ? std::max(bc->cg_tolerance, 1e-6) : bc->cg_tolerance;
  args.stall = bc->stall_tolerance;
  const size_t smem = tba::batch_smem_bytes(Cmax);

  cudaStream_t s = d->stream;
  cudaEvent_t e0 = event(d, 0), e1 = event(d, 1), e2 = event(d, 2), e3 = event(d, 3);
  uint64_t h2d = 0;
  auto up = [&](size_t off, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(a + off, src, bytes, cudaMemcpyHostToDevice, s));
    h2d += bytes;
  };
  CUDA_TRY(cudaEventRecord(e0, s));
  up(o_scene, scene, scene_len * sizeof(double));
  up(o_index, index, index_len * sizeof(uint32_t));
  up(o_tasks, tasks.data(), tasks.size() * sizeof(uint32_t));
  up(o_desc, desc.data(), desc.size() * sizeof(tba::BatchProblem));
  up(o_order, order.data(), order.size() * sizeof(uint32_t));
  // A mixed request may also run as the FP64 form (the tuner's policy choice below): the same
  // problems with their factors in the FP64 region and no FP32 copy.
  tba::BatchArgs args64 = args;
  if (mixed) {
    std::vector<tba::BatchProblem> desc64 = desc;
    for (tba::BatchProblem& b : desc64) {
      b.F = b.F64;
      b.F64 = nullptr;
    }
    up(o_desc64, desc64.data(), desc64.size() * sizeof(tba::BatchProblem));
    args64.problems = reinterpret_cast<const tba::BatchProblem*>(a + o_desc64);
    args64.tol_inner = bc->cg_tolerance;
  }
  CUDA_TRY(cudaEventRecord(e1, s));

  auto blocks_of = [&](int shape, bool form_mixed) {
    const int per_sm = tba::batch_blocks_per_sm(shape, shared, form_mixed, smem);
    return std::min<int>(int(count), per_sm * d->sms);
  };
  // The launch shape, and for a mixed request the form: forced, cached, or tuned now by one timed
  // LM iteration of the whole batch per shape (the trial launches write only the workspace and the
  // device copy of the results).  A mixed request tries the FP64 form too and keeps it when it is
  // faster: on small windows the FP32 product saves less than the FP64 refinement of each PCG
  // solution costs.  The result is the FP64 form's, which the mixed form only approximates.
  double tune_ms = 0;
  int shape = -1;
  bool run_mixed = mixed;
  if (bc->schedule > 0) {
    shape = int(bc->schedule) - 1;
    if (shape >= tba::kBatchShapes) argument("Invalid GPU BA batch schedule");
  } else {
    int lg = 0;
    while ((uint64_t(1) << (lg + 1)) <= std::max<uint64_t>(1, M_total)) lg++;
    const std::string key = std::to_string(shared) + "/" + std::to_string(mixed) + "/" + std::to_string(Cmax) + "/" +
                            std::to_string(lg) + "/" + std::to_string(count);
    auto hit = d->tuned.find(key);
    if (hit != d->tuned.end()) {
      shape = hit->second % tba::kBatchShapes;
      run_mixed = mixed && hit->second < tba::kBatchShapes;
    } else {
      const auto t0 = std::chrono::steady_clock::now();
      cudaEvent_t ta = event(d, 4), tb = event(d, 5);
      // One timed launch of the batch in one form and shape; -1 when the shape does not fit.
      auto trial_ms = [&](int k, bool form_mixed, uint32_t iterations) -> float {
        const int blocks = blocks_of(k, form_mixed);
        if (blocks <= 0) return -1;
        tba::BatchArgs trial = form_mixed || !mixed ? args : args64;
        trial.iterations = iterations;
        CUDA_TRY(cudaMemsetAsync(trial.queue, 0, sizeof(uint32_t), s));
        CUDA_TRY(cudaEventRecord(ta, s));
        CUDA_TRY(tba::launch_batch(k, shared, form_mixed, trial, blocks, smem, s));
        CUDA_TRY(cudaEventRecord(tb, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, ta, tb));
        return ms;
      };
      // Each form's shape by one LM iteration per shape; for a mixed request the two forms' best
      // shapes then run the whole solve once each (one LM iteration does not show the refinement's
      // share), and the faster form is kept.
      int best_shape[2] = {-1, -1};
      for (int form = 0; form < (mixed ? 2 : 1); form++) {
        const bool form_mixed = mixed && form == 0;
        float best = 0;
        for (int k = 0; k < tba::kBatchShapes; k++) {
          const float ms = trial_ms(k, form_mixed, std::min<uint32_t>(args.iterations, 1));
          if (ms >= 0 && (best_shape[form] < 0 || ms < best)) {
            best = ms;
            best_shape[form] = k;
          }
        }
      }
      shape = best_shape[0];
      run_mixed = mixed;
      if (mixed && best_shape[0] >= 0 && best_shape[1] >= 0 && args.iterations > 1) {
        const float ms_mixed = trial_ms(best_shape[0], true, args.iterations);
        const float ms_fp64 = trial_ms(best_shape[1], false, args.iterations);
        if (ms_fp64 < ms_mixed) {
          shape = best_shape[1];
          run_mixed = false;
        }
      } else if (shape < 0) {
        shape = best_shape[1];
        run_mixed = false;
      }
      if (shape < 0) throw Fail{TBA_ERROR_INTERNAL, "no launch shape of the batched solver fits the device"};
      d->tuned[key] = shape + (mixed && !run_mixed ? tba::kBatchShapes : 0);
      tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  }
  if (!run_mixed) args = args64;  // (args64 == args for an FP64 request)
  const int blocks = blocks_of(shape, run_mixed);
  if (blocks <= 0) throw Fail{TBA_ERROR_INTERNAL, "the batched solver's launch shape does not fit the device"};

  // One persistent launch, captured once in a CUDA graph and replayed while its arguments stay.
  std::vector<char> key(sizeof args + 3 * sizeof(int) + sizeof(size_t));
  {
    const int ints[3] = {shape, blocks, int(shared) | (int(run_mixed) << 1)};
    std::memcpy(key.data(), &args, sizeof args);
    std::memcpy(key.data() + sizeof args, ints, sizeof ints);
    std::memcpy(key.data() + sizeof args + sizeof ints, &smem, sizeof smem);
  }
  bool replayed = true;
  if (!d->batch_graph || d->batch_key != key) {
    replayed = false;
    if (d->batch_graph) {
      CUDA_TRY(cudaGraphExecDestroy(d->batch_graph));
      d->batch_graph = nullptr;
    }
    cudaGraph_t graph = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1c = cudaMemsetAsync(args.queue, 0, sizeof(uint32_t), s);
    cudaError_t e2c = e1c == cudaSuccess ? tba::launch_batch(shape, shared, run_mixed, args, blocks, smem, s) : e1c;
    cudaError_t e3c = cudaStreamEndCapture(s, &graph);
    CUDA_TRY(e2c);
    CUDA_TRY(e3c);
    cudaError_t ei = cudaGraphInstantiate(&d->batch_graph, graph, 0);
    cudaGraphDestroy(graph);
    CUDA_TRY(ei);
    d->batch_key = key;
  }
  CUDA_TRY(cudaGraphLaunch(d->batch_graph, s));
  CUDA_TRY(cudaEventRecord(e2, s));
  // Download the result records, merged into contiguous runs.
  uint64_t d2h = 0;
  for (uint32_t j = 0; j < count;) {
    const tba_batch_problem& q0 = probs[by_out[j]];
    const size_t begin = q0.output_offset;
    tba_control c0 = batch_problem_control(bc, q0);
    size_t end = begin + tba_output_size(&c0);
    uint32_t k = j + 1;
    while (k < count && probs[by_out[k]].output_offset == end) {
      const tba_control ck = batch_problem_control(bc, probs[by_out[k]]);
      end += tba_output_size(&ck);
      k++;
    }
    CUDA_TRY(cudaMemcpyAsync(output + begin, dout + begin, (end - begin) * sizeof(double), cudaMemcpyDeviceToHost, s));
    d2h += (end - begin) * sizeof(double);
    j = k;
  }
  CUDA_TRY(cudaEventRecord(e3, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    std::memset(report, 0, sizeof *report);
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    report->upload_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e1, e2));
    report->solve_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e2, e3));
    report->download_ms = ms;
    report->tune_ms = tune_ms;
    report->h2d_bytes = h2d;
    report->d2h_bytes = d2h;
    for (uint32_t k = 0; k < count; k++) {
      const tba_batch_problem& q = probs[k];
      const double* st = output + q.output_offset + 12 * size_t(q.cameras) + 3 * size_t(q.points);
      report->lm_iterations += uint64_t(st[tba::S_ACCEPTED] + st[tba::S_REJECTED]);
      report->cg_iterations += uint64_t(st[tba::S_CG_STEPS]);
    }
    report->problems = count;
    report->schedule = uint32_t(shape);
    report->threads = uint32_t(tba::batch_shape(shape).threads);
    report->blocks = uint32_t(blocks);
    report->graph_replayed = replayed ? 1 : 0;
    report->kernel_launches = 2;
    report->form = run_mixed ? TBA_PRECISION_MIXED : TBA_PRECISION_FP64;
    report->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
  }
}

// ---- the adjoint ---------------------------------------------------------------------------------

void solve_vjp(tba_device* d, const tba_vjp_control* vc, const double* scene, const uint32_t* index,
               const double* cotangent, double* pixels_bar, double* intrinsics_bar, double* solution,
               tba_vjp_report* report) {
  const auto wall0 = std::chrono::steady_clock::now();
  const uint32_t C = vc->cameras, P = vc->points, M = vc->observations;
  const uint32_t* active = index + 3 * size_t(M) + P + C + 2;
  uint32_t fixed = 0;
  for (uint32_t c = 0; c < C; c++) fixed += active[c] == 0;
  tba::AdjParams A{};
  A.C = C;
  A.P = P;
  A.M = M;
  A.anchor = vc->anchor;
  A.scale_view = vc->scale_view;
  A.normalize_scale = fixed == 1;
  A.huber = vc->huber;
  A.tol = vc->cg_tolerance;
  // Warp tasks of the one-pass Schur product (whole points, at most 32 observations each).
  const std::vector<uint32_t> tasks = build_tasks(index + 2 * size_t(M), P);
  std::vector<uint32_t> task_obs(tasks.size());
  for (size_t t = 0; t < tasks.size(); t++) task_obs[t] = index[2 * size_t(M) + tasks[t]];
  A.ntasks = uint32_t(tasks.size() - 1);
  A.prod_blocks = C <= tba::adj_one_pass_max_cameras()
                      ? std::max<uint32_t>(1, std::min<uint32_t>(tba::adj_product_blocks_per_sm(C) * uint32_t(d->sms),
                                                                 (A.ntasks + 7) / 8))
                      : 0;
  A.prod_copies = tba::adj_product_copies(C);
  Layout L;
  const size_t o_poses = L.take<double>(12 * size_t(C)), o_points = L.take<double>(3 * size_t(P)),
               o_cams = L.take<double>(6 * size_t(C)), o_pixels = L.take<double>(2 * size_t(M)),
               o_index = L.take<uint32_t>(3 * size_t(M) + P + 2 * size_t(C) + 2),
               o_hcp = L.take<double>(18 * size_t(M)), o_hcc = L.take<double>(21 * size_t(M)),
               o_hpp = L.take<double>(6 * size_t(M)), o_gc = L.take<double>(6 * size_t(M)),
               o_gp = L.take<double>(3 * size_t(M)), o_vinv = L.take<double>(6 * size_t(P)),
               o_bp = L.take<double>(3 * size_t(P)), o_lp = L.take<double>(3 * size_t(P)),
               o_yp = L.take<double>(3 * size_t(P)), o_U = L.take<double>(21 * size_t(C)),
               o_minv = L.take<double>(36 * size_t(C)), o_bc = L.take<double>(6 * size_t(C)),
               o_vec = L.take<double>(5 * 6 * size_t(C)), o_cot = L.take<double>(6 * size_t(C) + 3 * size_t(P)),
               o_gcot = L.take<double>(12 * size_t(C) + 3 * size_t(P)), o_ybar = L.take<double>(2 * size_t(M)),
               o_state = L.take<double>(tba::A_WORDS), o_tposes = L.take<double>(12 * size_t(C)),
               o_tpoints = L.take<double>(3 * size_t(P)), o_tobs = L.take<uint32_t>(task_obs.size()),
               o_part = L.take<double>(size_t(A.prod_blocks) * 6 * C);
  if (d->capacity < L.bytes) {
    if (d->arena) CUDA_TRY(cudaFree(d->arena));
    d->arena = nullptr;
    d->capacity = 0;
    size_t free_bytes = 0, total_bytes = 0;
    CUDA_TRY(cudaMemGetInfo(&free_bytes, &total_bytes));
    if (L.bytes > free_bytes)
      throw Fail{TBA_ERROR_BUDGET, "GPU BA adjoint needs " + std::to_string(L.bytes) +
                                       " bytes of device memory, more than the working budget of " +
                                       std::to_string(free_bytes) + " bytes"};
    CUDA_TRY(cudaMalloc(&d->arena, L.bytes));
    d->capacity = L.bytes;
  }
  char* a = d->arena;
  auto D = [&](size_t off) { return reinterpret_cast<double*>(a + off); };
  A.poses = D(o_poses);
  A.points = D(o_points);
  A.cams = D(o_cams);
  A.pixels = D(o_pixels);
  uint32_t* dindex = reinterpret_cast<uint32_t*>(a + o_index);
  A.obs_camera = dindex;
  A.obs_point = dindex + M;
  A.point_start = dindex + 2 * size_t(M);
  A.camera_start = A.point_start + P + 1;
  A.camera_obs = A.camera_start + C + 1;
  A.active = A.camera_obs + M;
  A.Hcp = D(o_hcp);
  A.Hcc = D(o_hcc);
  A.Hpp = D(o_hpp);
  A.gc = D(o_gc);
  A.gp = D(o_gp);
  A.Vinv = D(o_vinv);
  A.bp = D(o_bp);
  A.lp = D(o_lp);
  A.yp = D(o_yp);
  A.U = D(o_U);
  A.Minv = D(o_minv);
  A.bc = D(o_bc);
  double* vec = D(o_vec);
  A.x = vec;
  A.r = vec + 6 * size_t(C);
  A.p = vec + 12 * size_t(C);
  A.z = vec + 18 * size_t(C);
  A.Sp = vec + 24 * size_t(C);
  A.cot = D(o_cot);
  A.ybar = D(o_ybar);
  A.state = D(o_state);
  A.tposes = D(o_tposes);
  A.tpoints = D(o_tpoints);
  A.task_obs = reinterpret_cast<const uint32_t*>(a + o_tobs);
  A.part = D(o_part);
  A.mu = 0;

  cudaStream_t s = d->stream;
  cudaEvent_t e0 = event(d, 0), e1 = event(d, 1);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  };
  CUDA_TRY(cudaEventRecord(e0, s));
  up(A.poses, scene, 12 * sizeof(double) * C);
  up(A.points, scene + 12 * size_t(C), 3 * sizeof(double) * P);
  up(const_cast<double*>(A.cams), scene + 12 * size_t(C) + 3 * size_t(P), 6 * sizeof(double) * C);
  up(const_cast<double*>(A.pixels), scene + 18 * size_t(C) + 3 * size_t(P), 2 * sizeof(double) * M);
  up(dindex, index, sizeof(uint32_t) * (3 * size_t(M) + P + 2 * size_t(C) + 2));
  up(const_cast<uint32_t*>(A.task_obs), task_obs.data(), sizeof(uint32_t) * task_obs.size());
  uint32_t launches = 0;
  launches += tba::adj_launch_init(A, s);
  CUDA_TRY(cudaGetLastError());

  auto read_state = [&]() {
    CUDA_TRY(cudaMemcpyAsync(d->pinned, A.state, tba::A_WORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
  };
  uint32_t cg_total = 0, failed = 0, point_failures = 0;
  const bool time_products = (vc->flags & TBA_VJP_FLAG_TIME_PRODUCTS) != 0;
  double product_ms = 0;
  uint32_t product_launches = 0;
  double last_residual = 0, gnorm_initial = -1, gnorm = 0;
  // One linear solve (H + gauge term) z = rhs by Schur complement and PCG; z lands in x (cameras)
  // and lp (points).  The assembly also measures |F|^2 at the current point.
  auto linear_solve = [&](uint32_t mode, bool cotangent_ready) {
    A.rhs_mode = mode;
    if (!cotangent_ready) launches += tba::adj_launch_reset(A, s);
    launches += tba::adj_launch_assemble(A, s);
    launches += tba::adj_launch_pcg_init(A, s);
    CUDA_TRY(cudaGetLastError());
    uint32_t done = 0;
    const bool timed = time_products && A.prod_blocks;
    const bool on_device = !timed && vc->max_cg > 0 && !d->host_pcg_only &&
                           device_loop_ready(d, d->adj_loop, build_adjoint_loop(d->adj_loop, A, s));
    if (on_device) {
      // One launch of the device-side PCG loop, which stops on the device.
      launches += tba::adj_launch_loop_begin(A, vc->max_cg, s);
      CUDA_TRY(cudaGraphLaunch(d->adj_loop.exec, s));
      done = vc->max_cg;
    }
    while (done < vc->max_cg) {
      const uint32_t k = std::min<uint32_t>(16, vc->max_cg - done);
      for (uint32_t j = 0; j < k; j++)
        launches += timed ? tba::adj_launch_pcg_step(A, s, event(d, 8 + 2 * j), event(d, 9 + 2 * j))
                          : tba::adj_launch_pcg_step(A, s);
      CUDA_TRY(cudaGetLastError());
      done += k;
      read_state();
      if (timed) {
        // The chunk's products that ran PCG steps (later launches of a chunk are guarded no-ops).
        const uint32_t steps = uint32_t(d->pinned[tba::A_STEPS]);
        for (uint32_t j = 0; j < k && done - k + j < steps; j++) {
          float ms = 0;
          CUDA_TRY(cudaEventElapsedTime(&ms, event(d, 8 + 2 * j), event(d, 9 + 2 * j)));
          product_ms += ms;
          product_launches++;
        }
      }
      if (d->pinned[tba::A_ACTIVE] == 0) break;
    }
    read_state();
    if (on_device) launches += uint32_t(d->pinned[tba::A_LOOP_ITERS]) * d->adj_loop.body_kernels;
    const double* st = d->pinned;
    cg_total += uint32_t(st[tba::A_STEPS]);
    last_residual = st[tba::A_R0] > 0 ? std::sqrt(st[tba::A_R2] / st[tba::A_R0]) : 0;
    gnorm = std::sqrt(st[tba::A_GNORM]);
    if (gnorm_initial < 0) gnorm_initial = gnorm;
    const bool converged = st[tba::A_R2] <= vc->cg_tolerance * vc->cg_tolerance * st[tba::A_R0] || st[tba::A_R0] == 0;
    if (st[tba::A_POINT_SINGULAR] != 0) failed |= 1;
    point_failures = uint32_t(st[tba::A_POINT_FAILED]);
    if (st[tba::A_CAMERA_FAILED] != 0) failed |= 2;
    if (st[tba::A_FAILED] != 0) failed |= 4;
    if (!converged) failed |= 8;
    launches += tba::adj_launch_back_substitute(A, s);
    CUDA_TRY(cudaGetLastError());
    return st[tba::A_INVALID];
  };
  double invalid = 0;
  // Newton steps on H + mu G (G the IRLS Gauss-Newton matrix): mu shrinks tenfold after a step the
  // robust cost accepts and reaches 0 (exact Newton) below 1e-6, and grows tenfold after a rejected
  // one.  Candidates within a relative 1e-14 of the current cost count as accepted.
  if (vc->newton_steps > 0) {
    launches += tba::adj_launch_cost(A, s);
    read_state();
  }
  double cost = d->pinned[tba::A_COST], mu = 1e-2;
  uint32_t accepted = 0;
  for (uint32_t k = 0; k < vc->newton_steps; k++) {
    A.mu = mu;
    invalid = linear_solve(0, false);
    launches += tba::adj_launch_newton_candidate(A, s);
    CUDA_TRY(cudaGetLastError());
    read_state();
    const double cand = d->pinned[tba::A_COST];
    const bool solved = (failed & 5) == 0;
    failed &= ~uint32_t(13);  // a damped solve that failed is retried with more damping
    if (solved && cand <= cost * (1 + 1e-14)) {
      launches += tba::adj_launch_newton_commit(A, s);
      CUDA_TRY(cudaGetLastError());
      cost = cand;
      accepted++;
      mu = mu < 1e-6 ? 0.0 : mu / 10;
    } else {
      mu = std::max(1e-6, mu * 10);
    }
  }
  A.mu = 0;
  if (cotangent) {
    double* gcot = D(o_gcot);
    up(gcot, cotangent, sizeof(double) * (12 * size_t(C) + 3 * size_t(P)));
    launches += tba::adj_launch_reset(A, s);
    launches += tba::adj_launch_cotangent(A, gcot, s);
    CUDA_TRY(cudaGetLastError());
    invalid = linear_solve(1, true);
    launches += tba::adj_launch_vjp(A, s);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(pixels_bar, A.ybar, 2 * sizeof(double) * M, cudaMemcpyDeviceToHost, s));
    read_state();
    if (intrinsics_bar) {
      intrinsics_bar[0] = d->pinned[tba::A_SBAR];
      intrinsics_bar[1] = d->pinned[tba::A_KBAR];
    }
  } else if (vc->newton_steps > 0) {
    // The gradient at the final point.
    launches += tba::adj_launch_reset(A, s);
    A.rhs_mode = 0;
    launches += tba::adj_launch_assemble(A, s);
    read_state();
    gnorm = std::sqrt(d->pinned[tba::A_GNORM]);
    invalid = d->pinned[tba::A_INVALID];
  }
  if (solution) {
    CUDA_TRY(cudaMemcpyAsync(solution, A.poses, 12 * sizeof(double) * C, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(solution + 12 * size_t(C), A.points, 3 * sizeof(double) * P, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaEventRecord(e1, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    std::memset(report, 0, sizeof *report);
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    report->solve_ms = ms;
    report->gradient_norm_initial = gnorm_initial < 0 ? gnorm : gnorm_initial;
    report->gradient_norm_final = gnorm;
    report->adjoint_residual = cotangent ? last_residual : 0;
    report->cg_iterations = cg_total;
    report->newton_steps = accepted;
    report->failed = failed;
    report->invalid = uint32_t(invalid);
    report->point_failures = point_failures;
    report->product_ms = product_ms;
    report->product_launches = product_launches;
    report->product_blocks = A.prod_blocks;
    report->kernel_launches = launches;
    report->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
  }
}

// ---- observation evaluation ------------------------------------------------------------------------

void evaluate_observations(tba_device* d, const tba_observation_control* oc, const double* cameras,
                           const double* points, const double* pixels, const uint32_t* indices,
                           const uint32_t* offsets, uint32_t* flags, double* summary, tba_observation_report* report) {
  const auto wall0 = std::chrono::steady_clock::now();
  const uint32_t C = oc->cameras, P = oc->points, M = oc->observations;
  const bool guarded = oc->max_relative_depth_std > 0;
  Layout L;
  const size_t o_cam = L.take<double>(18 * size_t(C)), o_pts = L.take<double>(3 * size_t(P)),
               o_pix = L.take<double>(2 * size_t(M)), o_idx = L.take<uint32_t>(2 * size_t(M)),
               o_off = L.take<uint32_t>(guarded ? size_t(P) + 1 : 0),
               o_flags = L.take<uint32_t>(size_t(M) + (guarded ? P : 0)), o_err = L.take<double>(M),
               o_part = L.take<double>(2 * ((size_t(M) + 63) / 64)), o_sum = L.take<double>(2),
               o_tasks = L.take<uint32_t>(guarded ? size_t(P) + 1 : 0);
  if (d->capacity < L.bytes) {
    if (d->arena) CUDA_TRY(cudaFree(d->arena));
    d->arena = nullptr;
    d->capacity = 0;
    size_t free_bytes = 0, total_bytes = 0;
    CUDA_TRY(cudaMemGetInfo(&free_bytes, &total_bytes));
    if (L.bytes > free_bytes)
      throw Fail{TBA_ERROR_BUDGET, "GPU observation evaluation exceeds budget"};
    CUDA_TRY(cudaMalloc(&d->arena, L.bytes));
    d->capacity = L.bytes;
  }
  char* a = d->arena;
  tba::ObsParams p{};
  p.C = C;
  p.P = P;
  p.M = M;
  p.guarded = guarded ? 1 : 0;
  p.max_error = oc->max_error_px;
  p.max_relative_depth = oc->max_relative_depth_std;
  p.noise = oc->pixel_noise_std_px;
  p.cameras = reinterpret_cast<double*>(a + o_cam);
  p.points = reinterpret_cast<double*>(a + o_pts);
  p.pixels = reinterpret_cast<double*>(a + o_pix);
  p.indices = reinterpret_cast<uint32_t*>(a + o_idx);
  p.offsets = guarded ? reinterpret_cast<uint32_t*>(a + o_off) : nullptr;
  p.flags = reinterpret_cast<uint32_t*>(a + o_flags);
  p.errors = reinterpret_cast<double*>(a + o_err);
  p.partials = reinterpret_cast<double*>(a + o_part);
  p.summary = reinterpret_cast<double*>(a + o_sum);
  cudaStream_t s = d->stream;
  cudaEvent_t e0 = event(d, 0), e1 = event(d, 1), e2 = event(d, 2), e3 = event(d, 3);
  uint64_t h2d = 0;
  auto up = [&](size_t off, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(a + off, src, bytes, cudaMemcpyHostToDevice, s));
    h2d += bytes;
  };
  CUDA_TRY(cudaEventRecord(e0, s));
  up(o_cam, cameras, 18 * sizeof(double) * C);
  up(o_pts, points, 3 * sizeof(double) * P);
  up(o_pix, pixels, 2 * sizeof(double) * M);
  up(o_idx, indices, 2 * sizeof(uint32_t) * M);
  if (guarded) {
    up(o_off, offsets, sizeof(uint32_t) * (size_t(P) + 1));
    // Warp tasks of whole tracks, built while the copies above run.
    const std::vector<uint32_t> tasks = build_tasks(offsets, P);
    p.tasks = reinterpret_cast<uint32_t*>(a + o_tasks);
    p.ntasks = uint32_t(tasks.size() - 1);
    up(o_tasks, tasks.data(), sizeof(uint32_t) * tasks.size());
  }
  CUDA_TRY(cudaEventRecord(e1, s));
  tba::launch_observations(p, s);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaEventRecord(e2, s));
  const size_t nflags = size_t(M) + (guarded ? P : 0);
  if (nflags) CUDA_TRY(cudaMemcpyAsync(flags, p.flags, nflags * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(summary, p.summary, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaEventRecord(e3, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    std::memset(report, 0, sizeof *report);
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    report->upload_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e1, e2));
    report->evaluate_ms = ms;
    CUDA_TRY(cudaEventElapsedTime(&ms, e2, e3));
    report->download_ms = ms;
    report->h2d_bytes = h2d;
    report->d2h_bytes = nflags * sizeof(uint32_t) + 2 * sizeof(double);
    report->kernel_launches = (guarded ? (p.ntasks ? 1u : 0u) : (M ? 1u : 0u)) + (M ? 1u : 0u) + 1u;
    report->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
  }
}

}  // namespace

extern "C" {

size_t tba_scene_size(const tba_control* c) {
  return c ? 18 * size_t(c->cameras) + 3 * size_t(c->points) + 2 * size_t(c->observations) : 0;
}
size_t tba_index_size(const tba_control* c) {
  return c ? 3 * size_t(c->observations) + c->points + 2 * size_t(c->cameras) + 2 : 0;
}
size_t tba_output_size(const tba_control* c) {
  return c ? 12 * size_t(c->cameras) + 3 * size_t(c->points) + 26 + (c->shared_focal ? 1 : 0) : 0;
}

tba_status tba_device_open(int ordinal, tba_device** out) {
  if (!out) return TBA_ERROR_ARGUMENT;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    g_open_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return TBA_ERROR_INTERNAL;
  }
  if (ordinal < 0 || ordinal >= count) {
    g_open_error = "CUDA device ordinal out of range";
    return TBA_ERROR_ARGUMENT;
  }
  tba_device* d = new tba_device();
  d->ordinal = ordinal;
  try {
    CUDA_TRY(cudaSetDevice(ordinal));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, ordinal));
    if (prop.major < 10) throw Fail{TBA_ERROR_INTERNAL, "libtba.so is built for sm_100a (B200); device is sm_" +
                                                            std::to_string(prop.major) + std::to_string(prop.minor)};
    d->sms = prop.multiProcessorCount;
    CUDA_TRY(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&d->down, cudaStreamNonBlocking));
    CUDA_TRY(cudaMallocHost(&d->pinned, 64 * sizeof(double)));
    CUDA_TRY(tba::configure_kernels());
    CUDA_TRY(tba::adj_configure());
    CUDA_TRY(tba::batch_configure());
  } catch (const Fail& f) {
    g_open_error = f.message;
    tba_device_close(d);
    return f.status;
  }
  *out = d;
  return TBA_OK;
}

void tba_device_close(tba_device* d) {
  if (!d) return;
  cudaSetDevice(d->ordinal);
  if (d->stream) cudaStreamSynchronize(d->stream);
  if (d->down) cudaStreamSynchronize(d->down);
  for (cudaEvent_t e : d->events) cudaEventDestroy(e);
  if (d->batch_graph) cudaGraphExecDestroy(d->batch_graph);
  for (PcgLoop& loop : d->pcg_loops) loop.release();
  d->adj_loop.release();
  if (d->batch_arena) cudaFree(d->batch_arena);
  if (d->arena) cudaFree(d->arena);
  if (d->pinned) cudaFreeHost(d->pinned);
  if (d->stream) cudaStreamDestroy(d->stream);
  if (d->down) cudaStreamDestroy(d->down);
  delete d;
}

const char* tba_last_error(const tba_device* d) { return d ? d->error.c_str() : g_open_error.c_str(); }

tba_status tba_bundle_adjust(tba_device* d, const tba_control* control, const double* scene, size_t scene_len,
                             const uint32_t* index, size_t index_len, double* output, size_t output_len,
                             tba_report* report) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    check_control(control);
    if (!scene || !index || !output) argument("Invalid GPU BA arrays: null pointer");
    if (scene_len != tba_scene_size(control)) argument("Invalid GPU BA scene array length");
    if (index_len != tba_index_size(control)) argument("Invalid GPU BA index array length");
    if (output_len < tba_output_size(control)) argument("Invalid GPU BA output array length");
    if (uint64_t(3) * control->observations + control->points + 2ull * control->cameras + 2 > 0xffffffffull)
      argument("GPU BA scene dimensions exceed integer index bounds");
    // The O(C) checks here, the O(M) ones on the device after the upload (before any solver kernel).
    const auto t0 = std::chrono::steady_clock::now();
    const HostChecks hc = host_checks(control, index, scene);
    double check_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    CUDA_TRY(cudaSetDevice(d->ordinal));
    SolveIO io;
    io.checks = &hc;
    io.check_ms = &check_ms;
    solve(d, control, scene, index, output, report, io);
    if (report) report->check_ms = check_ms;
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

uint32_t tba_batch_max_cameras(void) { return tba::batch_max_cameras(); }
uint32_t tba_batch_shapes(void) { return uint32_t(tba::kBatchShapes); }

tba_status tba_batch_shape(uint32_t k, uint32_t* threads, uint32_t* min_blocks) {
  if (k >= uint32_t(tba::kBatchShapes)) return TBA_ERROR_ARGUMENT;
  const tba::BatchShape s = tba::batch_shape(int(k));
  if (threads) *threads = uint32_t(s.threads);
  if (min_blocks) *min_blocks = uint32_t(s.min_blocks);
  return TBA_OK;
}

tba_status tba_batch_adjust(tba_device* d, const tba_batch_control* control, const tba_batch_problem* problems,
                            uint32_t count, const double* scene, size_t scene_len, const uint32_t* index,
                            size_t index_len, double* output, size_t output_len, tba_batch_report* report) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (!control) argument("Invalid GPU BA batch: no control block");
    if (count == 0 || !problems) argument("Invalid GPU BA batch: no problems");
    if (!scene || !index || !output) argument("Invalid GPU BA arrays: null pointer");
    CUDA_TRY(cudaSetDevice(d->ordinal));
    solve_batch(d, control, problems, count, scene, scene_len, index, index_len, output, output_len, report);
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

tba_status tba_bundle_vjp(tba_device* d, const tba_vjp_control* vc, const double* scene, size_t scene_len,
                          const uint32_t* index, size_t index_len, const double* cotangent, size_t cotangent_len,
                          double* pixels_bar, size_t pixels_bar_len, double* intrinsics_bar, double* solution,
                          size_t solution_len, tba_vjp_report* report) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (!vc) argument("Invalid GPU BA adjoint: no control block");
    tba_control c{};
    c.cameras = vc->cameras;
    c.points = vc->points;
    c.observations = vc->observations;
    c.anchor = vc->anchor;
    c.scale_view = vc->scale_view;
    c.iterations = 0;
    c.max_cg = 1;
    c.huber = vc->huber;
    c.cg_tolerance = 1e-6;
    c.stall_tolerance = 1e-9;
    check_control(&c);
    if (vc->newton_steps > 50 || vc->max_cg < 1 || vc->max_cg > 100000 || (vc->flags & ~TBA_VJP_FLAG_TIME_PRODUCTS) != 0 ||
        !(std::isfinite(vc->cg_tolerance) && vc->cg_tolerance >= 1e-15 && vc->cg_tolerance <= 1e-2))
      argument("Invalid GPU BA adjoint options");
    if (!scene || !index) argument("Invalid GPU BA arrays: null pointer");
    if (scene_len != tba_scene_size(&c)) argument("Invalid GPU BA scene array length");
    if (index_len != tba_index_size(&c)) argument("Invalid GPU BA index array length");
    const size_t n_theta = 12 * size_t(c.cameras) + 3 * size_t(c.points);
    if (cotangent && (cotangent_len != n_theta || !pixels_bar || pixels_bar_len < 2 * size_t(c.observations)))
      argument("Invalid GPU BA adjoint arrays: the cotangent needs 12C + 3P values and pixels_bar 2M");
    if (solution && solution_len < n_theta) argument("Invalid GPU BA adjoint arrays: solution needs 12C + 3P values");
    if (cotangent)
      for (size_t i = 0; i < n_theta; i++)
        if (!std::isfinite(cotangent[i])) argument("Invalid GPU BA adjoint: the cotangent is not finite");
    if (uint64_t(3) * c.observations + c.points + 2ull * c.cameras + 2 > 0xffffffffull)
      argument("GPU BA scene dimensions exceed integer index bounds");
    check_index(&c, index);
    check_scene(&c, scene, scene_len);
    CUDA_TRY(cudaSetDevice(d->ordinal));
    solve_vjp(d, vc, scene, index, cotangent, pixels_bar, intrinsics_bar, solution, report);
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

tba_status tba_evaluate_observations(tba_device* d, const tba_observation_control* oc, const double* cameras,
                                     size_t cameras_len, const double* points, size_t points_len, const double* pixels,
                                     size_t pixels_len, const uint32_t* indices, size_t indices_len,
                                     const uint32_t* offsets, size_t offsets_len, uint32_t* flags, size_t flags_len,
                                     double* summary, tba_observation_report* report) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (!oc || !summary) argument("Invalid GPU observation request");
    const uint64_t C = oc->cameras, P = oc->points, M = oc->observations;
    const bool guarded = oc->max_relative_depth_std > 0;
    if (!(std::isfinite(oc->max_error_px) && oc->max_error_px >= 1e-12 && oc->max_error_px <= 1e6) ||
        !(std::isfinite(oc->max_relative_depth_std) && oc->max_relative_depth_std >= 0 &&
          oc->max_relative_depth_std <= 1e9) ||
        !(std::isfinite(oc->pixel_noise_std_px) && oc->pixel_noise_std_px > 0 && oc->pixel_noise_std_px <= 1e9))
      argument("Invalid GPU observation threshold");
    if (2 * M + P + 1 > 0xffffffffull || 18 * C > 0xffffffffull || 8 * P > 0xffffffffull)
      argument("GPU observation evaluation exceeds budget");
    if ((C && !cameras) || (P && !points) || (M && (!pixels || !indices)) || ((M || guarded) && !flags))
      argument("Invalid GPU observation arrays: null pointer");
    if (cameras_len < 18 * C || points_len < 3 * P || pixels_len < 2 * M || indices_len < 2 * M ||
        flags_len < M + (guarded ? P : 0))
      argument("Invalid GPU observation arrays: lengths");
    FirstFailure ff;
    parallel_ranges(M, 1u << 18, [&](uint64_t b, uint64_t e, unsigned) {
      for (uint64_t i = b; i < e; i++)
        if (indices[2 * i] >= C || indices[2 * i + 1] >= P)
          return ff.record(i, "Invalid GPU observation indices: a camera or point out of range");
    });
    ff.raise();
    if (guarded) {
      if (!offsets || offsets_len < P + 1) argument("Invalid GPU observation arrays: track offsets");
      if (offsets[0] != 0 || offsets[P] != M) argument("Invalid GPU observation arrays: track offsets");
      FirstFailure tf;
      parallel_ranges(P, 1u << 16, [&](uint64_t b, uint64_t e, unsigned) {
        for (uint64_t h = b; h < e; h++) {
          if (offsets[h + 1] < offsets[h] || offsets[h + 1] > M)
            return tf.record(h, "Invalid GPU observation arrays: track offsets");
          for (uint64_t i = offsets[h]; i < offsets[h + 1]; i++)
            if (indices[2 * i + 1] != h) return tf.record(h, "Invalid GPU observation arrays: track offsets");
        }
      });
      tf.raise();
    }
    FirstFailure bf;
    auto bounded = [&](const double* v, uint64_t n, uint64_t base) {
      parallel_ranges(n, 1u << 18, [&](uint64_t b, uint64_t e, unsigned) {
        for (uint64_t i = b; i < e; i++) {
          const double x = v[i];
          if (!std::isfinite(x) || std::fabs(x) > 1e9 || (x != 0 && std::fabs(x) < 1e-30))
            return bf.record(base + i, "Invalid GPU scene coordinate bounds");
        }
      });
    };
    bounded(cameras, 18 * C, 0);
    bounded(points, 3 * P, 18 * C);
    bounded(pixels, 2 * M, 18 * C + 3 * P);
    bf.raise();
    CUDA_TRY(cudaSetDevice(d->ordinal));
    evaluate_observations(d, oc, cameras, points, pixels, indices, offsets, flags, summary, report);
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

tba_status tba_scene_create(tba_device* d, const tba_control* shape, const double* scene, size_t scene_len,
                            const uint32_t* index, size_t index_len, tba_scene** out) {
  if (!d || !out) return TBA_ERROR_ARGUMENT;
  *out = nullptr;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  tba_scene* r = nullptr;
  try {
    check_control(shape);
    if (!scene || !index) argument("Invalid GPU BA arrays: null pointer");
    if (scene_len != tba_scene_size(shape)) argument("Invalid GPU BA scene array length");
    if (index_len != tba_index_size(shape)) argument("Invalid GPU BA index array length");
    if (uint64_t(3) * shape->observations + shape->points + 2ull * shape->cameras + 2 > 0xffffffffull)
      argument("GPU BA scene dimensions exceed integer index bounds");
    check_index(shape, index);
    check_scene(shape, scene, scene_len);
    CUDA_TRY(cudaSetDevice(d->ordinal));
    r = new tba_scene();
    r->device = d;
    r->shape = *shape;
    r->plan = new HostPlan(make_plan(shape, index, d->sms));
    std::vector<uint32_t> flat;
    for (const std::vector<uint32_t>* v : static_cast<HostPlan*>(r->plan)->sections()) flat.insert(flat.end(), v->begin(), v->end());
    CUDA_TRY(cudaMalloc(&r->scene, scene_len * sizeof(double)));
    CUDA_TRY(cudaMalloc(&r->index, index_len * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&r->plan_dev, std::max<size_t>(1, flat.size()) * sizeof(uint32_t)));
    CUDA_TRY(cudaMemcpyAsync(r->scene, scene, scene_len * sizeof(double), cudaMemcpyHostToDevice, d->stream));
    CUDA_TRY(cudaMemcpyAsync(r->index, index, index_len * sizeof(uint32_t), cudaMemcpyHostToDevice, d->stream));
    CUDA_TRY(cudaMemcpyAsync(r->plan_dev, flat.data(), flat.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  } catch (const Fail& f) {
    d->error = f.message;
    if (r) {
      if (r->scene) cudaFree(r->scene);
      if (r->index) cudaFree(r->index);
      if (r->plan_dev) cudaFree(r->plan_dev);
      delete static_cast<HostPlan*>(r->plan);
      delete r;
    }
    return f.status;
  }
  *out = r;
  return TBA_OK;
}

void tba_scene_destroy(tba_scene* r) {
  if (!r) return;
  {
    std::lock_guard<std::mutex> lock(r->device->mu);
    cudaSetDevice(r->device->ordinal);
    cudaStreamSynchronize(r->device->stream);
    if (r->scene) cudaFree(r->scene);
    if (r->index) cudaFree(r->index);
    if (r->plan_dev) cudaFree(r->plan_dev);
  }
  delete static_cast<HostPlan*>(r->plan);
  delete r;
}

tba_status tba_scene_adjust(tba_device* d, tba_scene* r, const tba_control* control, double* output,
                            size_t output_len, double* state, size_t state_len, tba_report* report) {
  if (!d || !r) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (r->device != d) argument("Invalid GPU BA resident scene: it belongs to another device handle");
    check_control(control);
    const tba_control& s = r->shape;
    if (control->cameras != s.cameras || control->points != s.points || control->observations != s.observations ||
        control->directional_points != s.directional_points || control->anchor != s.anchor ||
        control->scale_view != s.scale_view)
      argument("Invalid GPU BA resident scene: the control's sizes or gauge differ from the scene's");
    if (output && output_len < tba_output_size(control)) argument("Invalid GPU BA output array length");
    if (state && state_len < size_t(26 + (control->shared_focal ? 1 : 0))) argument("Invalid GPU BA state array length");
    CUDA_TRY(cudaSetDevice(d->ordinal));
    SolveIO io;
    io.device_source = true;
    io.plan = static_cast<const HostPlan*>(r->plan);
    io.plan_dev = r->plan_dev;
    io.writeback = r->scene;
    io.state = state;
    solve(d, control, r->scene, r->index, output, report, io);
    if (report) report->check_ms = 0;
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

tba_status tba_scene_write(tba_device* d, tba_scene* r, const double* poses, const double* points) {
  if (!d || !r) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (r->device != d) argument("Invalid GPU BA resident scene: it belongs to another device handle");
    const size_t C = r->shape.cameras, P = r->shape.points;
    auto bounded = [](const double* v, size_t n) {
      for (size_t i = 0; i < n; i++) {
        const double x = v[i];
        if (!std::isfinite(x) || std::fabs(x) > 1e9 || (x != 0 && std::fabs(x) < 1e-30)) return false;
      }
      return true;
    };
    if ((poses && !bounded(poses, 12 * C)) || (points && !bounded(points, 3 * P)))
      argument("GPU BA input exceeds supported coordinate bounds");
    CUDA_TRY(cudaSetDevice(d->ordinal));
    if (poses) CUDA_TRY(cudaMemcpyAsync(r->scene, poses, 12 * C * sizeof(double), cudaMemcpyHostToDevice, d->stream));
    if (points)
      CUDA_TRY(cudaMemcpyAsync(r->scene + 12 * C, points, 3 * P * sizeof(double), cudaMemcpyHostToDevice, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  }
  return TBA_OK;
}

tba_status tba_scene_read(tba_device* d, tba_scene* r, double* poses, double* points) {
  if (!d || !r) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (r->device != d) argument("Invalid GPU BA resident scene: it belongs to another device handle");
    const size_t C = r->shape.cameras, P = r->shape.points;
    CUDA_TRY(cudaSetDevice(d->ordinal));
    if (poses) CUDA_TRY(cudaMemcpyAsync(poses, r->scene, 12 * C * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    if (points)
      CUDA_TRY(cudaMemcpyAsync(points, r->scene + 12 * C, 3 * P * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  }
  return TBA_OK;
}

tba_status tba_device_set_wait_limit(tba_device* d, uint32_t polls) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->wait_limit = polls;
  return TBA_OK;
}

// Rows per slice of an inverse-depth call (2,048 tiles of 128 rows; at most 8 slices a call).
constexpr uint32_t kIdSliceRows = 1u << 18;

tba_status tba_linearize_inverse_depth(tba_device* d, uint32_t count, const double* measurements,
                                       size_t measurements_len, double* linearizations, size_t linearizations_len,
                                       tba_observation_report* report) {
  if (!d) return TBA_ERROR_ARGUMENT;
  std::lock_guard<std::mutex> lock(d->mu);
  d->error.clear();
  try {
    if (count && (!measurements || !linearizations)) argument("Invalid inverse-depth arrays: null pointer");
    if (measurements_len < 34ull * count || linearizations_len < 23ull * count)
      argument("Invalid inverse-depth arrays: lengths");
    if (34ull * count > 0xffffffffull) argument("Inverse-depth measurement budget cannot fit the observations");
    // Values are not checked, as the reference kernel's are not: a row whose projection leaves the
    // camera model's domain comes back with a zero flag.
    CUDA_TRY(cudaSetDevice(d->ordinal));
    const auto wall0 = std::chrono::steady_clock::now();
    Layout L;
    const size_t o_in = L.take<double>(34 * size_t(count)), o_out = L.take<double>(23 * size_t(count));
    const size_t o_err = L.take<uint32_t>(1);
    if (d->capacity < L.bytes) {
      if (d->arena) CUDA_TRY(cudaFree(d->arena));
      d->arena = nullptr;
      d->capacity = 0;
      size_t free_bytes = 0, total_bytes = 0;
      CUDA_TRY(cudaMemGetInfo(&free_bytes, &total_bytes));
      if (L.bytes > free_bytes) throw Fail{TBA_ERROR_BUDGET, "Inverse-depth measurement budget cannot fit the observations"};
      CUDA_TRY(cudaMalloc(&d->arena, L.bytes));
      d->capacity = L.bytes;
    }
    double* din = reinterpret_cast<double*>(d->arena + o_in);
    double* dout = reinterpret_cast<double*>(d->arena + o_out);
    uint32_t* derr = reinterpret_cast<uint32_t*>(d->arena + o_err);
    uint32_t err = 0;
    cudaStream_t s = d->stream, down = d->down;
    // Slices of whole 128-row tiles (so every slice's rows start 16-byte aligned in both arrays):
    // slice j's upload and kernel run on the main stream, its download on the second stream once
    // its kernel is done, so downloads overlap the next slices' uploads (the link is full duplex)
    // and the call takes about one upload plus one slice's kernel and download.
    const uint32_t slices = count <= kIdSliceRows ? 1u : std::min<uint32_t>(8u, (count + kIdSliceRows - 1) / kIdSliceRows);
    const uint32_t per = slices == 1 ? count : ((count + slices - 1) / slices + 127) / 128 * 128;
    // Events: per slice [upload start, upload end = kernel start, kernel end, download start,
    // download end], then the call's end on the second stream.
    CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(uint32_t), s));
    uint32_t launched = 0;
    for (uint32_t j = 0, first = 0; first < count; j++, first += per) {
      const uint32_t n = std::min(per, count - first);
      cudaEvent_t ev[5];
      for (int k = 0; k < 5; k++) ev[k] = event(d, 5 * size_t(j) + k);
      CUDA_TRY(cudaEventRecord(ev[0], s));
      CUDA_TRY(cudaMemcpyAsync(din + 34 * size_t(first), measurements + 34 * size_t(first), 34 * sizeof(double) * n,
                               cudaMemcpyHostToDevice, s));
      CUDA_TRY(cudaEventRecord(ev[1], s));
      CUDA_TRY(tba::launch_linearize_inverse_depth(n, din + 34 * size_t(first), dout + 23 * size_t(first), derr,
                                                   d->sms, s, d->wait_limit));
      launched++;
      CUDA_TRY(cudaEventRecord(ev[2], s));
      CUDA_TRY(cudaStreamWaitEvent(down, ev[2], 0));
      CUDA_TRY(cudaEventRecord(ev[3], down));
      CUDA_TRY(cudaMemcpyAsync(linearizations + 23 * size_t(first), dout + 23 * size_t(first),
                               23 * sizeof(double) * n, cudaMemcpyDeviceToHost, down));
      CUDA_TRY(cudaEventRecord(ev[4], down));
    }
    CUDA_TRY(cudaMemcpyAsync(&err, derr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaStreamSynchronize(down));
    if (err == 1) throw Fail{TBA_ERROR_CUDA, "Inverse-depth linearization: a tile load did not complete"};
    if (err) throw Fail{TBA_ERROR_CUDA, "Inverse-depth linearization: a tile load did not complete, and the loads "
                                        "in flight after it did not land in time"};
    if (report) {
      std::memset(report, 0, sizeof *report);
      // Sums over the slices (the phases of different slices overlap).
      for (uint32_t j = 0; j < launched; j++) {
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, event(d, 5 * size_t(j)), event(d, 5 * size_t(j) + 1)));
        report->upload_ms += ms;
        CUDA_TRY(cudaEventElapsedTime(&ms, event(d, 5 * size_t(j) + 1), event(d, 5 * size_t(j) + 2)));
        report->evaluate_ms += ms;
        CUDA_TRY(cudaEventElapsedTime(&ms, event(d, 5 * size_t(j) + 3), event(d, 5 * size_t(j) + 4)));
        report->download_ms += ms;
      }
      report->h2d_bytes = 34ull * 8 * count;
      report->d2h_bytes = 23ull * 8 * count;
      report->kernel_launches = launched;
      report->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
    }
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  }
  return TBA_OK;
}

}  // extern "C"
