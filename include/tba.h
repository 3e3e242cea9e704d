/*
 * tba.h — C ABI of the B200-native bundle-adjustment library (libtba.so).
 *
 * The library replaces the GPU half of TypeCV's `bundleAdjustGpu` operator
 * (src/sfm/bundle/gpu/bundle.ts:803-839, exported from src/gpu/index.ts:114-118): everything
 * between the host's packing of the problem and its reading of the result.  The reference host
 * packs the problem into two arrays (packBundleScene, src/sfm/bundle/gpu/bundle-host.ts:177-218),
 * uploads them (bundle.ts:267-271), runs its LM/PCG plan of WebGPU dispatches
 * (bundle.ts:314-772, joint-focal.ts:330-880) and reads one output array back
 * (bundle.ts:773).  `tba_bundle_adjust` takes exactly those two arrays and fills exactly that
 * output array, so the reference's host code before and after the call (bundleProblem,
 * packBundleScene, checkBundleOutput, bundleOutputPose, bundleOutputLandmarks,
 * bundleOutputReport) stays as it is.
 *
 * Conventions: plain pointers and sizes, host memory owned by the caller and only read (inputs)
 * or written (outputs) during the call; no pointer is kept after return.  Every entry point
 * returns a tba_status; on failure `tba_last_error` gives the message.  Calls on one device
 * handle are serialised by the handle; different handles may run concurrently.
 */
#ifndef TBA_H
#define TBA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TBA_ABI_VERSION 1

typedef enum {
  TBA_OK = 0,
  /* The problem or the options are invalid (the reference throws RangeError). */
  TBA_ERROR_ARGUMENT = 1,
  /* The problem does not fit the device (the reference's "budget" RangeError,
   * bundle.ts:235-242). */
  TBA_ERROR_BUDGET = 2,
  /* A CUDA call failed; the device handle should be closed. */
  TBA_ERROR_CUDA = 3,
  /* The library was built without a usable device, or an internal invariant failed. */
  TBA_ERROR_INTERNAL = 4
} tba_status;

/* Arithmetic of the solve.  TBA_PRECISION_FP64 is the drop-in (IEEE binary64 throughout).
 * TBA_PRECISION_MIXED runs the PCG's Schur product over an FP32 copy of the Jacobian factors (and of
 * the point-block inverses), in FP32 with each product block's camera sums in FP32 and the sums
 * across blocks in FP64, inside an FP64 LM loop (cost, gain, right-hand side, the camera/point
 * block inverses and the back-substitution stay FP64; the FP64 factors are kept too, 12 x 4 more
 * bytes per observation of device memory).  Each PCG solution is refined by its FP64 residual (one
 * product over the FP64 factors); when that residual is above the tolerance the PCG restarts from
 * it on the FP32 product, at most twice, and then finishes on the FP64 product, each restart with
 * an iteration budget of its own.  Once an LM iteration needed that FP64 finish, the call's later
 * iterations solve on the FP64 product alone (tba_report.fp64_iterations).  It has no reference
 * counterpart. */
typedef enum { TBA_PRECISION_FP64 = 0, TBA_PRECISION_MIXED = 1 } tba_precision;

/* TBA_FLAG_TIME_PRODUCTS: bracket every Schur product with CUDA events and report their total
 * device time in tba_report.product_ms (a few microseconds of host work per PCG iteration).
 * Without it each PCG run is one launch of a CUDA graph that repeats the PCG step on the device
 * until the PCG stops (or, where the driver cannot build conditional graph nodes, from the host);
 * with it the host launches the steps in chunks, with the same results. */
#define TBA_FLAG_TIME_PRODUCTS 1u
/* TBA_FLAG_PRODUCT_ERROR: once, on the first PCG direction of the first LM iteration, evaluate S p
 * with the solve's own Schur product and with the FP64 two-pass product (Jacobians recomputed from
 * the poses, points and pixels), and report their difference in tba_report.product_error_* (for
 * the mixed form: the FP32 product's error).  Diagnostics only: two more products per call. */
#define TBA_FLAG_PRODUCT_ERROR 2u
/* TBA_FLAG_HOST_PCG_LOOP: launch the PCG steps from the host in chunks, as with
 * TBA_FLAG_TIME_PRODUCTS but without the events, instead of the device-side graph loop (for
 * profilers and tools that do not follow the kernels of conditional graph nodes).  Same results. */
#define TBA_FLAG_HOST_PCG_LOOP 4u

/*
 * The control block of one solve: the reference's `control` uniform
 * (BundleControl, src/sfm/bundle/gpu/bundle.shade.ts:17-48 and joint-focal.shade.ts:14-42) plus
 * the host options that its plan consumes (bundle-host.ts:31-113).  Sizes count the trailing
 * directional points (bearings appended by appendBundleDirections) in `points`.
 */
typedef struct {
  uint32_t cameras;            /* C >= 2 */
  uint32_t points;             /* P >= 1, including `directional_points` */
  uint32_t directional_points; /* trailing points that are world bearings */
  uint32_t observations;       /* M */
  uint32_t anchor;             /* gauge anchor camera index */
  uint32_t scale_view;         /* gauge scale camera index */
  uint32_t iterations;         /* LM iterations, 0..100 (BUNDLE_DEFAULTS.iterations = 20) */
  uint32_t max_cg;             /* PCG iterations per LM iteration, 1..256 */
  uint32_t shared_focal;       /* 1: refineSharedFocal (one log-focal unknown, joint-focal.ts) */
  uint32_t precision;          /* tba_precision */
  uint32_t flags;              /* TBA_FLAG_* */
  double huber;                /* Huber threshold in pixels, 1e-12..1e6 */
  double cg_tolerance;         /* PCG relative residual tolerance, 1e-12..1e-2 */
  double stall_tolerance;      /* LM stall rule, [0, 1); the device rule is max(this, 1e-9) */
} tba_control;

/* Timings and traffic of one call, for the operator's `execution` report
 * (src/geometry/gpu/execution.ts:3-16). */
typedef struct {
  double solve_ms;        /* device time from the first kernel to the last (CUDA events) */
  double upload_ms;       /* device time of the host-to-device copies */
  double download_ms;     /* device time of the device-to-host copy */
  double wall_ms;         /* host wall time of the call, after the structural checks */
  double product_ms;      /* device time of the Schur products alone (sampled by events) */
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint32_t kernel_launches; /* kernels launched by the call, those inside CUDA graphs included */
  uint32_t lm_iterations;  /* LM iterations that ran */
  uint32_t cg_iterations;  /* PCG iterations that ran (state word 16) */
  uint32_t product_launches; /* Schur products timed in product_ms */
  uint32_t engine;         /* 0: grid engine, one-pass product over stored factors;
                              1: grid engine, two-pass recompute product (camera systems beyond
                                 on-chip memory) */
  uint32_t product_blocks; /* blocks of the one-pass product (each writes one partial row) */
  uint32_t refinements;    /* mixed form: PCG restarts from the FP64 residual */
  uint32_t fp64_iterations; /* mixed form: LM iterations solved on the FP64 product alone, after an
                              earlier iteration of the call needed the FP64 tail */
  double check_ms;         /* host wall time of the structural checks of the arrays (before wall_ms) */
  double product_error_max;  /* TBA_FLAG_PRODUCT_ERROR: max |S p - (S p)_64| / max |(S p)_64|, else 0 */
  double product_error_norm; /* TBA_FLAG_PRODUCT_ERROR: ||S p - (S p)_64|| / ||(S p)_64||, else 0 */
} tba_report;

/* Lengths, in elements, of the arrays of one problem (bundleArraySizes, bundle-host.ts:134-143):
 * scene = 18C + 3P + 2M doubles, index = 3M + P + 2C + 2 words, and the output of
 * packBundleResult: 12C + 3P + 26 doubles (+1 with the shared focal: its log scale). */
size_t tba_scene_size(const tba_control* control);
size_t tba_index_size(const tba_control* control);
size_t tba_output_size(const tba_control* control);

typedef struct tba_device tba_device;

/* Open a device handle on CUDA device `ordinal` (replaces ShadeDevice.open,
 * src/device/gpu/device.ts:240-360).  The handle owns a stream and a workspace that grows to the
 * largest problem solved and is reused. */
tba_status tba_device_open(int ordinal, tba_device** device);
void tba_device_close(tba_device* device);
/* The message of the last failed call on `device` (or of tba_device_open when device is NULL). */
const char* tba_last_error(const tba_device* device);

/*
 * One bundle adjustment: the reference's `bundleAdjustGpuFixed` (bundle.ts:89-800) or, with
 * control->shared_focal, `bundleAdjustJointFocalGpu` (joint-focal.ts:78-929), from the upload of
 * the packed arrays to the read of the output array.
 *
 * scene:  [poses 12C (R row-major, t) | points 3P | cameras 6C (fx, fy, cx, cy, k1, k2) |
 *          pixels 2M], observations point-major (packBundleScene).
 * index:  [obsCamera M | obsPoint M | pointStart P+1 | cameraStart C+1 |
 *          cameraObservations M | cameraActive C] (bundleIndexLayout, bundle-host.ts:121-131).
 * output: [poses 12C | points 3P | state 26 (| log focal scale)] (packBundleResult,
 *          bundle.shade.ts:1115-1125; joint-focal.shade.ts:1119-1129): state word 14 is the
 *          input error (1: zero gauge baseline, 2: an observation not in front of its camera).
 * report: may be NULL.
 */
tba_status tba_bundle_adjust(tba_device* device, const tba_control* control, const double* scene,
                             size_t scene_len, const uint32_t* index, size_t index_len,
                             double* output, size_t output_len, tba_report* report);

/*
 * A resident scene: the packed arrays of one problem kept on the device between adjustments, so
 * that repeated adjustments of the same map (the mapper's refinement passes) neither re-check nor
 * re-upload them.  It replaces the reference's per-call packing and upload
 * (packBundleScene, src/sfm/bundle/gpu/bundle-host.ts:177-218; bundle.ts:267-271) for callers that
 * keep the map in the packed layout (the reference's HostScene strides, src/sfm/scene/scene.ts:8-131).
 *
 * tba_scene_create checks and uploads the arrays once (as tba_bundle_adjust does per call);
 * tba_scene_adjust runs a bundle adjustment on them and leaves the solution's poses and points in
 * the scene, so the next adjustment starts from it.  `control` must have the scene's sizes and
 * gauge; its solver options may change between calls.  output (the tba_bundle_adjust record) and
 * state (its 26 [+1] state words) are optional.  tba_scene_write replaces the poses and/or points
 * (NULL: keep), tba_scene_read copies them out.  A scene belongs to the device handle it was created
 * on and is released by tba_scene_destroy.
 */
typedef struct tba_scene tba_scene;
tba_status tba_scene_create(tba_device* device, const tba_control* shape, const double* scene, size_t scene_len,
                            const uint32_t* index, size_t index_len, tba_scene** out);
void tba_scene_destroy(tba_scene* scene);
tba_status tba_scene_adjust(tba_device* device, tba_scene* scene, const tba_control* control, double* output,
                            size_t output_len, double* state, size_t state_len, tba_report* report);
tba_status tba_scene_write(tba_device* device, tba_scene* scene, const double* poses, const double* points);
tba_status tba_scene_read(tba_device* device, tba_scene* scene, double* poses, double* points);

/*
 * The robust cost of a packed scene that is already in device memory, computed without
 * allocating.  No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc — applications whose device memory belongs to their own allocator (a caching pool
 * or an arena reserved at start-up, where a library allocation fails at the limit or fragments
 * it) and code on latency-critical threads (cudaMalloc and cudaFree can synchronise the device).
 *
 * scene, index: device pointers to the packed arrays of tba_bundle_adjust (same layouts; only the
 *   poses, points, cameras, pixels and the obsCamera/obsPoint sections are read).  Indices are not
 *   trusted: an out-of-range one is skipped and counted.
 * scene_len, index_len: their lengths in elements; they must equal tba_scene_size(control) and
 *   tba_index_size(control).
 * result: device pointer to result_len >= 4 doubles: robust cost (Huber, control->huber), sum of
 *   squared errors, observations whose projection failed (behind the camera or outside the lens
 *   model), observations with an out-of-range index.  With the same inputs this equals the initial
 *   cost and squared error of tba_bundle_adjust (state words 8 and 9; word 24 is sqrt(SSE / M)).
 * stream: the cudaStream_t to run on (NULL: the default stream).  The call is asynchronous: the
 *   result is ready when the stream reaches it.
 * message: optional buffer for the error text.
 *
 * Before any launch the call refuses (TBA_ERROR_ARGUMENT, nothing launched) lengths that differ
 * from the control's, and any of scene, index or result that is not device (or managed) memory of
 * the current device or whose allocation holds fewer bytes from the pointer than its length claims
 * (cudaPointerGetAttributes and the driver's cuMemGetAddressRange; neither allocates).
 *
 * Limit: at most 16,777,216 observations (4,096 tiles of 4,096); larger scenes are refused with
 * TBA_ERROR_ARGUMENT.  The tile partials live in one fixed 128 KiB array that every GPU loading
 * the library holds until exit.  The first call on a device (and the first after the caller's
 * current context changes, e.g. after cudaDeviceReset) looks up that array's device address
 * (cudaGetSymbolAddress) with the caller's current device; make that first call before any stream
 * capture.  Every call shares the array: each call writes every tile row it reads, so nothing has
 * to start at zero, but calls that overlap on the GPU (different streams, not ordered) race and
 * must be serialised by the caller.
 */
tba_status tba_scene_cost_noalloc(const tba_control* control, const double* scene, size_t scene_len,
                                  const uint32_t* index, size_t index_len, double* result, size_t result_len,
                                  void* stream, char* message, size_t message_len);

/*
 * Batched local-window bundle adjustment: many independent problems in one persistent launch
 * (captured in a CUDA graph and replayed while the batch keeps its shape).  No counterpart in the
 * reference, whose mapper runs one `bundleAdjustGpu` call per local window
 * (src/sfm/mapper/mapper.ts:859-925 over the windows of src/sfm/bundle/local-bundle.ts:17-208);
 * each problem here gets exactly the result record of tba_bundle_adjust on the same arrays and
 * options (within rounding: the sums run in another order).
 *
 * Each problem is the reference's packed pair (scene, index) of tba_bundle_adjust, stored anywhere
 * in the caller's `scene` and `index` arrays at the offsets its tba_batch_problem gives; its result
 * record goes to `output` at output_offset (tba_output_size elements).  Problems may have at most
 * tba_batch_max_cameras() cameras (their camera system lives in on-chip shared memory); bearings
 * (directional points) are not supported here.
 */
typedef struct {
  uint32_t cameras, points, observations;
  uint32_t anchor, scale_view;
  uint32_t reserved;      /* 0 */
  uint64_t scene_offset;  /* first double of the problem's scene in `scene` */
  uint64_t index_offset;  /* first word of the problem's index in `index` */
  uint64_t output_offset; /* first double of the problem's result record in `output` */
} tba_batch_problem;

/* Options shared by every problem of a batch (tba_control's meaning).  `schedule` picks the
 * launch shape: 0 lets the autotuner choose (timed trial launches the first time a batch shape is
 * seen on the handle, cached afterwards), k >= 1 forces shape k - 1 of tba_batch_shape. */
typedef struct {
  uint32_t iterations;
  uint32_t max_cg;
  uint32_t shared_focal;
  uint32_t precision;
  uint32_t schedule;
  uint32_t flags;
  double huber;
  double cg_tolerance;
  double stall_tolerance;
} tba_batch_control;

typedef struct {
  double solve_ms;     /* device time of the persistent launch (CUDA events) */
  double upload_ms;    /* device time of the host-to-device copies */
  double download_ms;  /* device time of the device-to-host copy */
  double wall_ms;      /* host wall time of the call */
  double tune_ms;      /* host wall time spent in autotuning trial launches (0 when cached) */
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint64_t lm_iterations; /* accepted + rejected steps, summed over the problems */
  uint64_t cg_iterations; /* state word 16, summed over the problems */
  uint32_t problems;
  uint32_t schedule;      /* the launch shape used (0-based) */
  uint32_t threads;       /* threads per block of that shape */
  uint32_t blocks;        /* persistent blocks launched */
  uint32_t graph_replayed; /* 1: the launch replayed a cached CUDA graph */
  uint32_t kernel_launches;
  uint32_t form;           /* the tba_precision that ran: a mixed request runs the FP64 form when the
                              autotuner (schedule 0) timed it faster for this batch shape */
} tba_batch_report;

/* The largest camera count of one batched problem, and the number of launch shapes. */
uint32_t tba_batch_max_cameras(void);
uint32_t tba_batch_shapes(void);
/* Threads per block and compiled blocks per SM of launch shape k (0-based). */
tba_status tba_batch_shape(uint32_t k, uint32_t* threads, uint32_t* min_blocks);

tba_status tba_batch_adjust(tba_device* device, const tba_batch_control* control, const tba_batch_problem* problems,
                            uint32_t count, const double* scene, size_t scene_len, const uint32_t* index,
                            size_t index_len, double* output, size_t output_len, tba_batch_report* report);

/*
 * The adjoint of a converged bundle adjustment: the vector-Jacobian product of the solution
 * (poses and points) with respect to the observed pixels and two shared intrinsics, by implicit
 * differentiation.  No counterpart in the reference.
 *
 * At the solution theta* the robust cost's gradient F vanishes in every free direction, so
 * d theta* = -H^-1 (F_y dy + F_kappa d kappa), H the exact Hessian of the robust cost (second
 * derivatives of the projection and of the Huber loss included).  The gauge is the solver's: the
 * fixed cameras do not move and, with exactly one fixed camera, the anchor-to-scale-camera
 * baseline keeps its value (the cost's scale invariance is removed by that constraint, not by H).
 * The intrinsics are fixed inputs of the solve (refineSharedFocal off): kappa = (s, k1), where s
 * scales every camera's fx and fy by exp(s) and k1 is added to every camera's k1; both
 * derivatives are taken at s = 0 and the given k1.
 *
 * scene, index: the layouts of tba_bundle_adjust; the scene's poses and points are the
 *   evaluation point (normally the output of a converged tba_bundle_adjust).
 * control->newton_steps Newton iterations with the exact Hessian are taken from that point first
 *   (the solver's own update and gauge normalisation; the system H + mu G, G the Gauss-Newton
 *   matrix with the solver's IRLS weights, mu adapted by the robust cost of each candidate and
 *   zero once steps are accepted at mu < 1e-6), to drive
 *   the gradient to zero; with pixels changed slightly from those of a solution, they also re-solve
 *   the perturbed problem (finite-difference checks).
 * cotangent: 12C + 3P doubles on the output poses (R row-major, t) and points, or NULL (Newton
 *   steps only).  pixels_bar: 2M doubles, d<cotangent, theta*>/d pixel.  intrinsics_bar: 2 doubles,
 *   d/ds and d/dk1.  solution: 12C + 3P doubles receiving the evaluation point, or NULL.
 * Bearings (directional points) are not supported here.
 */
typedef struct {
  uint32_t cameras, points, observations;
  uint32_t anchor, scale_view;
  uint32_t newton_steps;  /* Newton iterations, 0..50 */
  uint32_t max_cg;        /* PCG iterations per linear solve, 1..100000 */
  uint32_t flags;         /* 0 or TBA_VJP_FLAG_TIME_PRODUCTS */
  double huber;           /* as tba_control.huber */
  double cg_tolerance;    /* relative PCG residual of every linear solve, 1e-15..1e-2 */
} tba_vjp_control;

typedef struct {
  double solve_ms;              /* device time of the whole call (CUDA events) */
  double wall_ms;
  double gradient_norm_initial; /* |F| at the given point */
  double gradient_norm_final;   /* |F| at the evaluation point (after the Newton steps) */
  double adjoint_residual;      /* relative residual reached by the adjoint's PCG */
  uint32_t cg_iterations;       /* over every linear solve */
  uint32_t newton_steps;        /* Newton iterations accepted */
  uint32_t failed;              /* bits: 1 a point block that no shift made definite, 2 a camera
                                   block not positive definite;
                                   4 a PCG broke down; 8 a PCG did not reach the tolerance */
  uint32_t invalid;             /* observations outside the projection's domain at the evaluation point */
  uint32_t point_failures;      /* point blocks of the last solve that were not positive definite and
                                   were shifted by the smallest power-of-ten multiple of their mean
                                   diagonal that makes them definite (their derivatives are then
                                   approximate: such points have a nearly flat robust cost) */
  uint32_t kernel_launches;     /* kernels launched by the call */
  double product_ms;            /* TBA_VJP_FLAG_TIME_PRODUCTS: device time of the one-pass Schur
                                   products that ran PCG steps (CUDA events), else 0 */
  uint32_t product_launches;    /* the products timed in product_ms */
  uint32_t product_blocks;      /* blocks of the one-pass product (each writes one partial row); 0:
                                   the two-pass product (camera systems beyond shared memory) */
} tba_vjp_report;

/* TBA_VJP_FLAG_TIME_PRODUCTS: bracket every one-pass Schur product of the vjp's linear solves with
 * CUDA events and report their total in tba_vjp_report.product_ms. */
#define TBA_VJP_FLAG_TIME_PRODUCTS 1u

tba_status tba_bundle_vjp(tba_device* device, const tba_vjp_control* control, const double* scene, size_t scene_len,
                          const uint32_t* index, size_t index_len, const double* cotangent, size_t cotangent_len,
                          double* pixels_bar, size_t pixels_bar_len, double* intrinsics_bar, double* solution,
                          size_t solution_len, tba_vjp_report* report);

/*
 * Observation evaluation of a fixed scene: the reference's evaluateObservationsGpu
 * (src/geometry/gpu/observations.ts:34-125), which the mapper runs after a bundle adjustment to
 * measure and filter its observations (src/sfm/mapper/mapper.ts:837-858).  Every observation is
 * projected; it is an inlier when the projection is in the camera model's domain and its error is
 * within max_error_px.  With max_relative_depth_std > 0 every track whose inliers leave its point's
 * linearised depth uncertainty (pixel_noise_std_px of independent pixel noise, poses and
 * intrinsics fixed) above that bound in any inlier camera loses all its inliers.
 *
 * The arrays are the reference's observation layout (observationLayout,
 * src/geometry/gpu/observation-layout.ts): cameras 18 doubles per referenced camera (R row-major,
 * t, fx, fy, cx, cy, k1, k2), points 3 per point (one point per track), pixels 2 per observation,
 * indices 2 per observation (camera record, point), offsets P + 1 first observations of each
 * track (only with the depth bound; observations grouped by track).  flags receives M words (1 =
 * inlier) and, with the depth bound, P more (1 = the track was rejected); summary receives the
 * inliers' error sum and their count.
 */
typedef struct {
  uint32_t cameras, points, observations;
  uint32_t reserved;               /* 0 */
  double max_error_px;             /* 1e-12..1e6 */
  double max_relative_depth_std;   /* 0: no depth filter */
  double pixel_noise_std_px;       /* > 0 (the reference's default is 1) */
} tba_observation_control;

typedef struct {
  double upload_ms, evaluate_ms, download_ms, wall_ms;
  uint64_t h2d_bytes, d2h_bytes;
  uint32_t kernel_launches;
} tba_observation_report;

tba_status tba_evaluate_observations(tba_device* device, const tba_observation_control* control,
                                     const double* cameras, size_t cameras_len, const double* points,
                                     size_t points_len, const double* pixels, size_t pixels_len,
                                     const uint32_t* indices, size_t indices_len, const uint32_t* offsets,
                                     size_t offsets_len, uint32_t* flags, size_t flags_len, double* summary,
                                     tba_observation_report* report);

/*
 * The measurement linearisation of the inverse-depth bundle adjustment: the device half of the
 * reference's linearizeInverseDepthGpu / bundleAdjustInverseDepthGpu
 * (src/sfm/depth/gpu/inverse-depth.ts:15-141, kernel inverse-depth.shade.ts), whose reduced solve
 * stays on the host in FP64.  measurements: 34 doubles per observation (a, b, rho of the anchored
 * point; the reference pose; the observing pose; the observing camera record; its squared radial
 * limit), linearizations: 23 doubles per observation (valid flag, pixel, 2x3 point derivatives,
 * 2x6 pose derivatives, 2 log-focal derivatives), the layouts the reference's host reads.  The
 * report is the observation report's shape (evaluate_ms = the kernel).  A call of more than 262,144
 * rows runs in slices whose downloads overlap the next slices' uploads only when both host arrays
 * are page-locked (cudaHostAlloc / cudaHostRegister); with pageable arrays the copies of each slice
 * complete before the next is issued and the slices run one after another.
 *
 * The kernel streams tiles through shared memory with bulk copies and waits on them with bounded
 * polls: a wait that runs out ends the call with TBA_ERROR_CUDA ("a tile load did not complete")
 * after the block's loads still in flight have landed, and the handle stays usable.
 */
tba_status tba_linearize_inverse_depth(tba_device* device, uint32_t count, const double* measurements,
                                       size_t measurements_len, double* linearizations, size_t linearizations_len,
                                       tba_observation_report* report);

/*
 * Polls of each main-loop tile wait of tba_linearize_inverse_depth on this handle (default
 * TBA_WAIT_LIMIT_DEFAULT).  No counterpart in the reference: it lets a test make the waits run out
 * (0 polls gives up at once) to exercise the failure path; the drain of the loads in flight after
 * such a failure always keeps the full bound.
 */
#define TBA_WAIT_LIMIT_DEFAULT 4194304u
tba_status tba_device_set_wait_limit(tba_device* device, uint32_t polls);

#ifdef __cplusplus
}
#endif

#endif /* TBA_H */
