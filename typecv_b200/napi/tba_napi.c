/*
 * Node N-API addon over libtba.so: the binding TypeCV's TypeScript host would load in place of its
 * WebGPU device plan for `bundleAdjustGpu` (src/sfm/bundle/gpu/bundle.ts:803-839, exported from
 * src/gpu/index.ts:114-118).  UNBUILT HERE: this image and its GPU hosts have no Node toolchain
 * (no node, node-gyp or node_api.h); the same C ABI is exercised from Python by the tests.
 *
 * Exports
 *   openDevice(ordinal: number): External              tba_device_open; closed by the finalizer
 *   closeDevice(device: External): void                tba_device_close (idempotent)
 *   bundleAdjustPacked(device, control, scene: Float64Array, index: Uint32Array)
 *       : Promise<Float64Array>                        tba_bundle_adjust on a worker thread
 *
 * `control` carries the fields of tba_control under the TypeScript names the wrapper uses:
 *   cameras, points, directionalPoints, observations, anchor, scaleView, iterations, maxCg,
 *   sharedFocal (boolean), precision ('fp64' | 'mixed', optional), huber, cgTolerance,
 *   stallTolerance.
 * TBA_ERROR_ARGUMENT and TBA_ERROR_BUDGET reject with a RangeError carrying the library's message
 * (the reference's messages, so its tests' /gauge/, /owned/, /budget/ ... patterns still match);
 * other failures reject with an Error.  The scene and index arrays are held by references until
 * the call completes and are never written; the output is a fresh Float64Array.
 */
#include <node_api.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "tba.h"

#define CHECK(env, call)                                        \
  do {                                                          \
    if ((call) != napi_ok) {                                    \
      napi_throw_error((env), NULL, "tba addon: " #call " failed"); \
      return NULL;                                              \
    }                                                           \
  } while (0)

typedef struct {
  tba_device* device;
} DeviceBox;

typedef struct {
  napi_async_work work;
  napi_deferred deferred;
  DeviceBox* box;
  napi_ref device_ref, scene_ref, index_ref;
  tba_control control;
  const double* scene;
  size_t scene_len;
  const uint32_t* index;
  size_t index_len;
  double* output;
  size_t output_len;
  tba_status status;
  char message[1024];
} Job;

static void finalize_device(napi_env env, void* data, void* hint) {
  (void)env;
  (void)hint;
  DeviceBox* box = (DeviceBox*)data;
  if (box->device) tba_device_close(box->device);
  free(box);
}

static napi_value open_device(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], out;
  int32_t ordinal = 0;
  CHECK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc >= 1) CHECK(env, napi_get_value_int32(env, argv[0], &ordinal));
  DeviceBox* box = (DeviceBox*)calloc(1, sizeof *box);
  if (!box) {
    napi_throw_error(env, NULL, "tba addon: out of host memory");
    return NULL;
  }
  if (tba_device_open(ordinal, &box->device) != TBA_OK) {
    napi_throw_error(env, NULL, tba_last_error(NULL));
    free(box);
    return NULL;
  }
  CHECK(env, napi_create_external(env, box, finalize_device, NULL, &out));
  return out;
}

static DeviceBox* device_of(napi_env env, napi_value v) {
  void* data = NULL;
  if (napi_get_value_external(env, v, &data) != napi_ok || !data) {
    napi_throw_type_error(env, NULL, "expected a device from openDevice()");
    return NULL;
  }
  return (DeviceBox*)data;
}

static napi_value close_device(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  DeviceBox* box = argc >= 1 ? device_of(env, argv[0]) : NULL;
  if (box && box->device) {
    tba_device_close(box->device);
    box->device = NULL;
  }
  return NULL;
}

/* Reads a numeric field of `obj`; `required` fields that are missing throw a TypeError. */
static int field_u32(napi_env env, napi_value obj, const char* name, uint32_t* out, int required) {
  bool has = false;
  napi_value v;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok) return 0;
  if (!has) {
    if (required) napi_throw_type_error(env, NULL, name);
    return !required;
  }
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return 0;
  double d = 0;
  if (napi_get_value_double(env, v, &d) != napi_ok || !(d >= 0 && d <= 4294967295.0) || d != (double)(uint32_t)d) {
    napi_throw_range_error(env, NULL, name);
    return 0;
  }
  *out = (uint32_t)d;
  return 1;
}

static int field_f64(napi_env env, napi_value obj, const char* name, double* out) {
  napi_value v;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok || napi_get_value_double(env, v, out) != napi_ok) {
    napi_throw_type_error(env, NULL, name);
    return 0;
  }
  return 1;
}

static int field_flag(napi_env env, napi_value obj, const char* name, uint32_t* out) {
  bool has = false, b = false;
  napi_value v;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok) return 0;
  if (!has) return 1;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok || napi_get_value_bool(env, v, &b) != napi_ok) return 0;
  *out = b ? 1u : 0u;
  return 1;
}

static int read_control(napi_env env, napi_value obj, tba_control* c) {
  memset(c, 0, sizeof *c);
  char precision[16] = "fp64";
  bool has = false;
  if (!field_u32(env, obj, "cameras", &c->cameras, 1) || !field_u32(env, obj, "points", &c->points, 1) ||
      !field_u32(env, obj, "directionalPoints", &c->directional_points, 0) ||
      !field_u32(env, obj, "observations", &c->observations, 1) || !field_u32(env, obj, "anchor", &c->anchor, 1) ||
      !field_u32(env, obj, "scaleView", &c->scale_view, 1) || !field_u32(env, obj, "iterations", &c->iterations, 1) ||
      !field_u32(env, obj, "maxCg", &c->max_cg, 1) || !field_flag(env, obj, "sharedFocal", &c->shared_focal) ||
      !field_f64(env, obj, "huber", &c->huber) || !field_f64(env, obj, "cgTolerance", &c->cg_tolerance) ||
      !field_f64(env, obj, "stallTolerance", &c->stall_tolerance))
    return 0;
  if (napi_has_named_property(env, obj, "precision", &has) == napi_ok && has) {
    napi_value v;
    size_t n = 0;
    if (napi_get_named_property(env, obj, "precision", &v) != napi_ok ||
        napi_get_value_string_utf8(env, v, precision, sizeof precision, &n) != napi_ok)
      return 0;
  }
  if (strcmp(precision, "mixed") == 0) c->precision = TBA_PRECISION_MIXED;
  else if (strcmp(precision, "fp64") == 0) c->precision = TBA_PRECISION_FP64;
  else {
    napi_throw_range_error(env, NULL, "precision must be 'fp64' or 'mixed'");
    return 0;
  }
  return 1;
}

static void execute(napi_env env, void* data) { /* worker thread: no JavaScript access */
  (void)env;
  Job* j = (Job*)data;
  if (!j->box->device) {
    j->status = TBA_ERROR_ARGUMENT;
    strncpy(j->message, "the device was closed", sizeof j->message - 1);
    return;
  }
  j->status = tba_bundle_adjust(j->box->device, &j->control, j->scene, j->scene_len, j->index, j->index_len,
                                j->output, j->output_len, NULL);
  if (j->status != TBA_OK) strncpy(j->message, tba_last_error(j->box->device), sizeof j->message - 1);
}

static void complete(napi_env env, napi_status status, void* data) {
  Job* j = (Job*)data;
  napi_value result, msg, err;
  if (status == napi_ok && j->status == TBA_OK) {
    void* bytes = NULL;
    napi_value buffer;
    napi_create_arraybuffer(env, j->output_len * sizeof(double), &bytes, &buffer);
    memcpy(bytes, j->output, j->output_len * sizeof(double));
    napi_create_typedarray(env, napi_float64_array, j->output_len, buffer, 0, &result);
    napi_resolve_deferred(env, j->deferred, result);
  } else {
    napi_create_string_utf8(env, status == napi_ok ? j->message : "tba addon: the call was cancelled",
                            NAPI_AUTO_LENGTH, &msg);
    if (j->status == TBA_ERROR_ARGUMENT || j->status == TBA_ERROR_BUDGET) napi_create_range_error(env, NULL, msg, &err);
    else napi_create_error(env, NULL, msg, &err);
    napi_reject_deferred(env, j->deferred, err);
  }
  napi_delete_reference(env, j->device_ref);
  napi_delete_reference(env, j->scene_ref);
  napi_delete_reference(env, j->index_ref);
  napi_delete_async_work(env, j->work);
  free(j->output);
  free(j);
}

static napi_value bundle_adjust_packed(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4], promise, name, ab;
  CHECK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 4) {
    napi_throw_type_error(env, NULL, "bundleAdjustPacked(device, control, scene, index)");
    return NULL;
  }
  DeviceBox* box = device_of(env, argv[0]);
  if (!box) return NULL;
  Job* j = (Job*)calloc(1, sizeof *j);
  if (!j) {
    napi_throw_error(env, NULL, "tba addon: out of host memory");
    return NULL;
  }
  j->box = box;
  napi_typedarray_type t1, t2;
  void* data = NULL;
  size_t offset = 0;
  if (!read_control(env, argv[1], &j->control) ||
      napi_get_typedarray_info(env, argv[2], &t1, &j->scene_len, &data, &ab, &offset) != napi_ok ||
      t1 != napi_float64_array) {
    free(j);
    napi_throw_type_error(env, NULL, "scene must be a Float64Array");
    return NULL;
  }
  j->scene = (const double*)data;
  if (napi_get_typedarray_info(env, argv[3], &t2, &j->index_len, &data, &ab, &offset) != napi_ok ||
      t2 != napi_uint32_array) {
    free(j);
    napi_throw_type_error(env, NULL, "index must be a Uint32Array");
    return NULL;
  }
  j->index = (const uint32_t*)data;
  j->output_len = tba_output_size(&j->control);
  j->output = (double*)malloc(j->output_len * sizeof(double));
  if (!j->output) {
    free(j);
    napi_throw_error(env, NULL, "tba addon: out of host memory");
    return NULL;
  }
  /* The device and both inputs stay alive until `complete` runs. */
  napi_create_reference(env, argv[0], 1, &j->device_ref);
  napi_create_reference(env, argv[2], 1, &j->scene_ref);
  napi_create_reference(env, argv[3], 1, &j->index_ref);
  CHECK(env, napi_create_promise(env, &j->deferred, &promise));
  CHECK(env, napi_create_string_utf8(env, "tba_bundle_adjust", NAPI_AUTO_LENGTH, &name));
  CHECK(env, napi_create_async_work(env, NULL, name, execute, complete, j, &j->work));
  CHECK(env, napi_queue_async_work(env, j->work));
  return promise;
}

static napi_value init(napi_env env, napi_value exports) {
  napi_property_descriptor props[] = {
      {"openDevice", NULL, open_device, NULL, NULL, NULL, napi_default, NULL},
      {"closeDevice", NULL, close_device, NULL, NULL, NULL, napi_default, NULL},
      {"bundleAdjustPacked", NULL, bundle_adjust_packed, NULL, NULL, NULL, napi_default, NULL},
  };
  CHECK(env, napi_define_properties(env, exports, sizeof props / sizeof props[0], props));
  return exports;
}

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)
