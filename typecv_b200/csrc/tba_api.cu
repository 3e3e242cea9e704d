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
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tba.h"
#include "tba_engine.cuh"

using tba::Params;

struct tba_device {
  int ordinal = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  std::string error;
  char* arena = nullptr;
  size_t capacity = 0;
  double* pinned = nullptr;  // small host buffer for flag reads
  std::vector<cudaEvent_t> events;
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
      c->precision > 1)
    argument("Invalid GPU BA scene/options");
  if (c->anchor >= c->cameras || c->scale_view >= c->cameras || c->anchor == c->scale_view)
    argument("Invalid GPU BA gauge cameras");
}

// The structure of the packed index array (bundleIndexLayout): every section consistent with the
// others, so that no kernel can index out of bounds.
void check_index(const tba_control* c, const uint32_t* index) {
  const uint64_t C = c->cameras, P = c->points, M = c->observations;
  const uint32_t* obs_camera = index;
  const uint32_t* obs_point = index + M;
  const uint32_t* ps = index + 2 * M;
  const uint32_t* cs = ps + P + 1;
  const uint32_t* cam_obs = cs + C + 1;
  const uint32_t* active = cam_obs + M;
  if (ps[0] != 0 || ps[P] != M) argument("Invalid GPU BA index: point offsets do not cover the observations");
  for (uint64_t p = 0; p < P; p++) {
    if (ps[p + 1] > M) argument("Invalid GPU BA index: point offsets exceed the observations");
    if (ps[p + 1] < ps[p] + 2) argument("Landmarks require at least two observations");
    for (uint64_t i = ps[p]; i < ps[p + 1]; i++)
      if (obs_point[i] != p) argument("Invalid GPU BA index: observation point does not match the point offsets");
  }
  for (uint64_t i = 0; i < M; i++)
    if (obs_camera[i] >= C) argument("Invalid GPU BA index: observation camera out of range");
  if (cs[0] != 0 || cs[C] != M) argument("Invalid GPU BA index: camera offsets do not cover the observations");
  std::vector<uint8_t> seen(M, 0);
  for (uint64_t cam = 0; cam < C; cam++) {
    if (cs[cam + 1] < cs[cam] || cs[cam + 1] > M) argument("Invalid GPU BA index: camera offsets decrease or exceed the observations");
    for (uint64_t k = cs[cam]; k < cs[cam + 1]; k++) {
      const uint32_t i = cam_obs[k];
      if (i >= M || seen[i] || obs_camera[i] != cam)
        argument("Invalid GPU BA index: camera observation lists are not the observations of each camera");
      seen[i] = 1;
    }
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
  for (size_t i = 0; i < len; i++) {
    const double x = scene[i];
    if (!std::isfinite(x) || std::fabs(x) > 1e9 || (x != 0 && std::fabs(x) < 1e-30))
      argument("GPU BA input exceeds supported coordinate bounds");
  }
  const double* k = scene + 12 * size_t(c->cameras) + 3 * size_t(c->points);
  for (uint32_t cam = 0; cam < c->cameras; cam++, k += 6)
    if (!(k[0] > 0 && k[1] > 0) || k[0] < 1e-6 || k[1] < 1e-6 || k[0] > 1e6 || k[1] > 1e6 ||
        std::max(std::fabs(k[2]), std::fabs(k[3])) > 1e9 || std::max(std::fabs(k[4]), std::fabs(k[5])) > 1)
      argument("Camera exceeds the supported GPU geometry bounds");
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

cudaEvent_t event(tba_device* d, size_t k) {
  while (d->events.size() <= k) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    d->events.push_back(e);
  }
  return d->events[k];
}

void solve(tba_device* d, const tba_control* ctl, const double* scene, const uint32_t* index,
           double* output, tba_report* report) {
  const auto wall0 = std::chrono::steady_clock::now();
  const uint32_t C = ctl->cameras, P = ctl->points, M = ctl->observations;
  const bool shared = ctl->shared_focal != 0;
  const uint32_t m = 6 * C + (shared ? 1 : 0);
  const uint32_t* ps = index + 2 * size_t(M);
  const uint32_t* cs = ps + P + 1;
  const uint32_t* active = cs + C + 1 + M;
  const std::vector<uint32_t> tasks = build_tasks(ps, P);
  const Chunks chunks = build_chunks(cs, C, M, d->sms);
  const uint32_t ntasks = uint32_t(tasks.size() - 1), nchunks = uint32_t(chunks.cam.size());
  uint32_t fixed = 0;
  for (uint32_t c = 0; c < C; c++) fixed += active[c] == 0;

  Params p{};
  p.C = C;
  p.P = P;
  p.M = M;
  p.D = ctl->directional_points;
  p.m = m;
  p.anchor = ctl->anchor;
  p.scale_view = ctl->scale_view;
  p.normalize_scale = fixed == 1;
  p.shared = shared;
  p.huber = ctl->huber;
  p.tol = ctl->cg_tolerance;
  p.stall = ctl->stall_tolerance;
  // The mixed form's inner PCG runs stop at a relative residual the FP32 product can reach; the
  // FP64 refinement then measures the true residual against the caller's tolerance.
  p.tol_inner = ctl->precision == TBA_PRECISION_MIXED ? std::max(ctl->cg_tolerance, 1e-6) : ctl->cg_tolerance;
  p.ntasks = ntasks;
  p.nchunks = nchunks;
  p.task_blocks = std::max<uint32_t>(1, std::min<uint32_t>(4 * d->sms, (ntasks + 7) / 8));
  const uint32_t fblocks = tba::product_finish_blocks(p);
  // The one-pass product over stored factors when its camera sums fit shared memory; the two-pass
  // recompute form otherwise.  The mixed form stores FP32 factors.
  const bool mixed = ctl->precision == TBA_PRECISION_MIXED;
  p.factored = m <= tba::product_max_unknowns();
  p.Mpad = (M + 31) / 32 * 32;
  const size_t factor_bytes = p.factored ? size_t(tba::kFactors) * p.Mpad * (mixed ? 4 : 8) : 0;
  p.F = nullptr;
  p.F32 = mixed && p.factored ? reinterpret_cast<float*>(1) : nullptr;  // set below; selects the occupancy query
  const int per_sm = p.factored ? tba::product_blocks_per_sm(p) : 1;
  p.prod_blocks = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(per_sm * d->sms), (ntasks + 15) / 16));
  Layout L;
  const size_t o_poses = L.take<double>(12 * size_t(C)), o_points = L.take<double>(3 * size_t(P)),
               o_cams = L.take<double>(6 * size_t(C)), o_pixels = L.take<double>(2 * size_t(M)),
               o_tposes = L.take<double>(12 * size_t(C)), o_tpoints = L.take<double>(3 * size_t(P)),
               o_index = L.take<uint32_t>(3 * size_t(M) + P + 2 * size_t(C) + 2),
               o_tasks = L.take<uint32_t>(tasks.size()), o_ccam = L.take<uint32_t>(nchunks),
               o_cbeg = L.take<uint32_t>(nchunks + 1), o_cfirst = L.take<uint32_t>(C + 1),
               o_rlim = L.take<double>(C), o_cmp = L.take<uint32_t>(M), o_cmx = L.take<double>(2 * size_t(M)),
               o_pblk = L.take<double>(12 * size_t(P)), o_y = L.take<double>(4 * size_t(P)),
               o_cprod = L.take<double>(8 * size_t(nchunks)), o_F = L.take<char>(factor_bytes),
               o_pw = L.take<double>(6 * size_t(C)), o_xw = L.take<double>(6 * size_t(C)),
               o_acc = L.take<double>(p.factored ? size_t(p.prod_blocks) * m : 0), o_U = L.take<double>(21 * size_t(C)),
               o_Minv = L.take<double>(36 * size_t(C)), o_rhs = L.take<double>(6 * size_t(C)),
               o_hcf = L.take<double>(6 * size_t(C)),
               o_chunk = L.take<double>(size_t(tba::kCameraPartials) * nchunks),
               o_vec = L.take<double>(5 * size_t(m)), o_blk = L.take<double>(4 * size_t(fblocks)),
               o_scal = L.take<double>(size_t(tba::kScalarPartials) * p.task_blocks),
               o_cost = L.take<double>(4 * size_t(p.task_blocks)), o_ticket = L.take<uint32_t>(8),
               o_state = L.take<double>(tba::S_WORDS), o_out = L.take<double>(12 * size_t(C) + 3 * size_t(P) + 27);
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
  p.tasks = U32(o_tasks);
  p.chunk_cam = U32(o_ccam);
  p.chunk_beg = U32(o_cbeg);
  p.cam_chunk = U32(o_cfirst);
  p.rlim = D(o_rlim);
  p.cm_point = U32(o_cmp);
  p.cm_pixel = D(o_cmx);
  p.pblk = D(o_pblk);
  p.y = D(o_y);
  p.chunk_prod = D(o_cprod);
  p.F = p.factored && !mixed ? D(o_F) : nullptr;
  p.F32 = p.factored && mixed ? reinterpret_cast<float*>(a + o_F) : nullptr;
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
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    h2d += bytes;
  };
  CUDA_TRY(cudaEventRecord(e_start, s));
  up(p.poses, scene, 12 * sizeof(double) * C);
  up(p.points, scene + 12 * size_t(C), 3 * sizeof(double) * P);
  up(const_cast<double*>(p.cams), scene + 12 * size_t(C) + 3 * size_t(P), 6 * sizeof(double) * C);
  up(const_cast<double*>(p.pixels), scene + 18 * size_t(C) + 3 * size_t(P), 2 * sizeof(double) * M);
  up(dindex, index, sizeof(uint32_t) * (3 * size_t(M) + P + 2 * size_t(C) + 2));
  up(U32(o_tasks), tasks.data(), sizeof(uint32_t) * tasks.size());
  up(U32(o_ccam), chunks.cam.data(), sizeof(uint32_t) * nchunks);
  up(U32(o_cbeg), chunks.beg.data(), sizeof(uint32_t) * (nchunks + 1));
  up(U32(o_cfirst), chunks.cam_first.data(), sizeof(uint32_t) * (C + 1));
  CUDA_TRY(cudaEventRecord(e_up, s));

  uint32_t launches = 0, lm_done = 0;
  // Event pairs around the Schur products; after the solve, only the products that ran PCG steps
  // (the first `steps` of each LM iteration; later ones are guarded no-ops) count.
  std::vector<std::pair<size_t, size_t>> product_events;
  std::vector<std::pair<size_t, uint32_t>> product_spans;  // (first event pair, real steps) per LM iteration
  const bool time_products = (ctl->flags & TBA_FLAG_TIME_PRODUCTS) != 0;
  tba::launch_initialize(p, s);
  tba::launch_cost(p, s);
  tba::launch_finish_metrics(p, s);
  launches += 4;
  CUDA_TRY(cudaGetLastError());
  bool lm_active = read_word(d, p.state, tba::S_ACTIVE) != 0;
  tba::Params tail = p;
  tail.factored = 0;
  tail.F = nullptr;
  tail.F32 = nullptr;
  tail.tol_inner = 0;  // the tail stops at the solve's own tolerance
  for (uint32_t it = 0; it < ctl->iterations && lm_active; it++) {
    tba::launch_point_pass(p, s);
    tba::launch_camera_pass(p, s);
    tba::launch_camera_finish(p, s);
    tba::launch_pcg_init(p, s);
    launches += 4;
    // PCG in chunks of guarded iterations; the read after each chunk only ends the loop early.
    uint32_t done = 0, steps_before = 0;
    // `q` selects the product: the engine's own (FP32 factors in the mixed form), or the FP64
    // two-pass product of the mixed form's tail.  Only the engine's own products are timed.
    auto run_pcg = [&](uint32_t budget, const tba::Params& q, bool timed) {
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
          launches += q.factored ? 5 : 6;
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
    run_pcg(ctl->max_cg, p, true);
    // Mixed form: FP64 iterative refinement.  The true residual of the FP32-product solution
    // restarts the PCG when it is above the tolerance, and the restarted run (with an iteration
    // budget of its own) uses the FP64 two-pass product, which resolves what FP32 factors cannot
    // on badly conditioned systems.
    if (mixed) {
      tba::launch_refine(p, s);
      launches += 4;
      CUDA_TRY(cudaGetLastError());
      if (read_word(d, p.state, tba::S_CG_ACTIVE) != 0) run_pcg(done + ctl->max_cg, tail, false);
    }
    tba::launch_update_cameras(p, s);
    tba::launch_update_points(p, s);
    tba::launch_accept(p, s);
    tba::launch_commit(p, s);
    launches += 4;
    CUDA_TRY(cudaGetLastError());
    lm_done++;
    CUDA_TRY(cudaMemcpyAsync(d->pinned, p.state, 32 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    lm_active = d->pinned[tba::S_ACTIVE] != 0;
  }
  tba::launch_pack(p, s);
  launches++;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaEventRecord(e_solved, s));
  const size_t out_len = 12 * size_t(C) + 3 * size_t(P) + 26 + (shared ? 1 : 0);
  CUDA_TRY(cudaMemcpyAsync(output, p.output, out_len * sizeof(double), cudaMemcpyDeviceToHost, s));
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
    report->d2h_bytes = out_len * sizeof(double);
    report->kernel_launches = launches;
    report->lm_iterations = lm_done;
    report->cg_iterations = uint32_t(output[12 * size_t(C) + 3 * size_t(P) + tba::S_CG_STEPS]);
    report->engine = 0;
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
    CUDA_TRY(cudaMallocHost(&d->pinned, 64 * sizeof(double)));
    CUDA_TRY(tba::configure_kernels());
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
  for (cudaEvent_t e : d->events) cudaEventDestroy(e);
  if (d->arena) cudaFree(d->arena);
  if (d->pinned) cudaFreeHost(d->pinned);
  if (d->stream) cudaStreamDestroy(d->stream);
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
    check_index(control, index);
    check_scene(control, scene, scene_len);
    CUDA_TRY(cudaSetDevice(d->ordinal));
    solve(d, control, scene, index, output, report);
  } catch (const Fail& f) {
    d->error = f.message;
    return f.status;
  } catch (const std::exception& e) {
    d->error = e.what();
    return TBA_ERROR_INTERNAL;
  }
  return TBA_OK;
}

}  // extern "C"
