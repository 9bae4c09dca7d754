// extern "C" entry points of libever_b200.so (declared in include/ever_b200.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return EVER_OK;
  return fail(EVER_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

EverTune resolve_tune(const EverTune* t) {
  EverTune r{};
  if (t) r = *t;
  if (r.kbuf != 8 && r.kbuf != 16 && r.kbuf != 32) r.kbuf = 16;
  if (r.block != 64 && r.block != 128 && r.block != 256) r.block = 128;
  r.stack_depth = r.stack_depth <= 0 ? ever::kStackDepth : std::min(std::max(r.stack_depth, 8), ever::kStackDepth);
  return r;
}

// sh_degree < 0: the reference's forward colour, the DC term of every ellipsoid whatever
// its SH size (shaders.slang:72-75, eval_sh_col0); 0..3: SH of that degree along rayd.
int resolve_degree(const EverScene* sc, const EverTraceArgs* a, int* deg) {
  int d = a->sh_degree;
  if (d < 0) d = 0;
  if (d > 3) return fail(EVER_ERR_INVALID, "sh_degree %d out of range 0..3", d);
  if ((d + 1) * (d + 1) > sc->sh_coeffs)
    return fail(EVER_ERR_INVALID, "sh_degree %d needs %d SH coefficients, features have %d", d, (d + 1) * (d + 1),
                sc->sh_coeffs);
  if (d > 0 && sc->num_prims > 0 && !sc->features)
    return fail(EVER_ERR_INVALID, "sh_degree %d needs the feature rows; the scene was built with ever_scene_build_dc", d);
  *deg = d;
  return EVER_OK;
}

}  // namespace

int ever::set_last_error(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" {

const char* ever_last_error(void) { return g_last_error.c_str(); }

int ever_abi_version(void) { return EVER_ABI_VERSION; }

size_t ever_scene_workspace_bytes(int64_t num_prims, int32_t sh_coeffs) {
  if (num_prims < 0 || sh_coeffs < 1) return 0;
  return size_t(ever::scene_layout(num_prims, sh_coeffs).total);
}

static int build_scene(const float* mean, const float* scale, const float* quat, const float* density,
                       const float* features, int64_t num_prims, int32_t sh_coeffs, void* workspace,
                       size_t workspace_bytes, EverScene* scene, void* stream, bool dc_only) {
  if (!scene) return fail(EVER_ERR_INVALID, "scene is null");
  if (num_prims < 0 || num_prims >= (int64_t(1) << 30))
    return fail(EVER_ERR_INVALID, "num_prims %lld out of range [0, 2^30)", (long long)num_prims);
  if (sh_coeffs < 1 || sh_coeffs > 16) return fail(EVER_ERR_INVALID, "sh_coeffs %d out of range 1..16", sh_coeffs);
  if (num_prims > 0 && (!mean || !scale || !quat || !density || !features))
    return fail(EVER_ERR_INVALID, "null ellipsoid parameter pointer");
  const ever::SceneLayout L = ever::scene_layout(num_prims, sh_coeffs);
  if (num_prims > 0 && (!workspace || workspace_bytes < size_t(L.total)))
    return fail(EVER_ERR_WORKSPACE, "scene workspace needs %lld bytes, got %zu", (long long)L.total, workspace_bytes);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(EVER_ERR_INVALID, "workspace not 256-byte aligned");
  cudaError_t e = ever::scene_build(mean, scale, quat, density, features, num_prims, sh_coeffs,
                                    static_cast<char*>(workspace), L, scene, static_cast<cudaStream_t>(stream), dc_only);
  return cuda_status(e, dc_only ? "ever_scene_build_dc" : "ever_scene_build");
}

int ever_scene_build(const float* mean, const float* scale, const float* quat, const float* density,
                     const float* features, int64_t num_prims, int32_t sh_coeffs, void* workspace,
                     size_t workspace_bytes, EverScene* scene, void* stream) {
  return build_scene(mean, scale, quat, density, features, num_prims, sh_coeffs, workspace, workspace_bytes, scene,
                     stream, false);
}

int ever_scene_build_dc(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* features, int64_t num_prims, int32_t sh_coeffs, void* workspace,
                        size_t workspace_bytes, EverScene* scene, void* stream) {
  return build_scene(mean, scale, quat, density, features, num_prims, sh_coeffs, workspace, workspace_bytes, scene,
                     stream, true);
}

int ever_scene_set_features(EverScene* scene, const float* features, void* stream) {
  if (!scene) return fail(EVER_ERR_INVALID, "scene is null");
  if (scene->num_prims > 0 && !features) return fail(EVER_ERR_INVALID, "features is null");
  return cuda_status(ever::scene_set_features(scene, features, static_cast<cudaStream_t>(stream)),
                     "ever_scene_set_features");
}

int ever_scene_refit(const float* mean, const float* scale, const float* quat, const float* density,
                     const float* features, void* workspace, size_t workspace_bytes, EverScene* scene, void* stream) {
  if (!scene) return fail(EVER_ERR_INVALID, "scene is null");
  const int64_t N = scene->num_prims;
  if (N == 0) return EVER_OK;
  if (!mean || !scale || !quat || !density) return fail(EVER_ERR_INVALID, "null ellipsoid parameter pointer");
  const ever::SceneLayout L = ever::scene_layout(N, scene->sh_coeffs);
  char* ws = static_cast<char*>(workspace);
  if (!ws || workspace_bytes < size_t(L.total)) return fail(EVER_ERR_WORKSPACE, "scene workspace too small");
  if (scene->nodes != ws + L.nodes || scene->records != ws + L.records)
    return fail(EVER_ERR_INVALID, "scene was not built on this workspace");
  return cuda_status(ever::scene_refit(mean, scale, quat, density, features, ws, L, scene,
                                       static_cast<cudaStream_t>(stream)),
                     "ever_scene_refit");
}

int ever_trace_forward(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                       const EverTraceArgs* args, const int32_t* ray_order, const EverTune* tune,
                       const EverForwardOut* out, void* stream) {
  if (!scene || !args || !out) return fail(EVER_ERR_INVALID, "null scene, args or out");
  if (num_rays < 0 || num_rays >= (int64_t(1) << 40)) return fail(EVER_ERR_INVALID, "num_rays out of range");
  if (num_rays > 0 && (!rayo || !rayd || !out->out || !out->iters))
    return fail(EVER_ERR_INVALID, "null rayo, rayd, out or iters");
  if (out->event_log && out->log_cap < 0) return fail(EVER_ERR_INVALID, "negative log_cap");
  int deg = 0;
  if (int rc = resolve_degree(scene, args, &deg)) return rc;
  ever::FwdParams P{};
  P.nodes = scene->nodes;
  P.records = scene->records;
  P.features = scene->features;
  P.order = scene->order;
  P.N = scene->num_prims;
  P.K = scene->sh_coeffs;
  P.rayo = rayo;
  P.rayd = rayd;
  P.R = num_rays;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.ray_order = ray_order;
  P.out = *out;
  P.depth_hint = args->depth_hint;
  return cuda_status(ever::launch_forward(P, deg, resolve_tune(tune), static_cast<cudaStream_t>(stream)),
                     "ever_trace_forward");
}

size_t ever_trace_forward_workspace_bytes(int64_t num_rays) {
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31)) return 0;
  return size_t(ever::regroup_workspace(num_rays));
}

int ever_trace_forward_regrouped(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                                 const EverTraceArgs* args, const int32_t* ray_order, const EverTune* tune,
                                 const EverForwardOut* out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!scene || !args || !out) return fail(EVER_ERR_INVALID, "null scene, args or out");
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31)) return fail(EVER_ERR_INVALID, "num_rays out of range");
  if (num_rays > 0 && (!rayo || !rayd || !out->out || !out->iters || !out->states || !out->last_dirac))
    return fail(EVER_ERR_INVALID, "null rayo, rayd, out, iters, states or last_dirac");
  if (out->event_log && out->log_cap < 0) return fail(EVER_ERR_INVALID, "negative log_cap");
  const int64_t need = ever::regroup_workspace(num_rays);
  if (num_rays > 0 && (!workspace || workspace_bytes < size_t(need)))
    return fail(EVER_ERR_WORKSPACE, "forward workspace needs %lld bytes, got %zu", (long long)need, workspace_bytes);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(EVER_ERR_INVALID, "workspace not 256-byte aligned");
  int deg = 0;
  if (int rc = resolve_degree(scene, args, &deg)) return rc;
  ever::FwdParams P{};
  P.nodes = scene->nodes;
  P.records = scene->records;
  P.features = scene->features;
  P.order = scene->order;
  P.N = scene->num_prims;
  P.K = scene->sh_coeffs;
  P.rayo = rayo;
  P.rayd = rayd;
  P.R = num_rays;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.ray_order = ray_order;
  P.out = *out;
  P.depth_hint = args->depth_hint;
  if (num_rays == 0) return EVER_OK;
  const ever::RegroupScratch W = ever::regroup_scratch(static_cast<char*>(workspace), num_rays);
  return cuda_status(ever::launch_forward_regrouped(P, W, nullptr, nullptr, deg, resolve_tune(tune),
                                                    static_cast<cudaStream_t>(stream)),
                     "ever_trace_forward_regrouped");
}

size_t ever_backward_workspace_bytes(int64_t num_prims, int32_t sh_coeffs) {
  if (num_prims < 0 || sh_coeffs < 1) return 0;
  ever::WsCursor c;
  c.take(num_prims * 16 * sizeof(float));
  c.take(num_prims * int64_t(ever::feat_stride(sh_coeffs)) * sizeof(float));
  c.take(num_prims * int64_t(sizeof(int32_t)));  // inverse Morton order for the finalize
  return size_t(c.offset);
}

}  // extern "C"

namespace {

int trace_backward(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                   const EverTraceArgs* args, const float* grad_out, const float* states, const int32_t* iters,
                   const int32_t* event_log, int32_t log_cap, const float* wct, int32_t num_wct, const float* mean,
                   const float* scale, const float* quat, void* workspace, size_t workspace_bytes,
                   const int32_t* ray_order, const int32_t* slot_order, const EverTune* tune,
                   const EverBackwardOut* out, void* stream, const ever::CameraParams* cam = nullptr,
                   const float* jitter = nullptr) {
  if (!scene || !args || !out) return fail(EVER_ERR_INVALID, "null scene, args or out");
  const int64_t N = scene->num_prims;
  if (num_rays < 0) return fail(EVER_ERR_INVALID, "num_rays out of range");
  // camera traces make their rays in the kernels and may skip the ray gradients
  const bool need_rays = !cam, need_dray = !cam || out->drayo || out->drayd;
  if (num_rays > 0 && ((need_rays && (!rayo || !rayd)) || !grad_out || !states || !iters || !event_log ||
                       (need_dray && (!out->drayo || !out->drayd))))
    return fail(EVER_ERR_INVALID, "null ray-side pointer");
  if (N > 0 && (!mean || !scale || !quat || !out->dmean || !out->dscale || !out->dquat || !out->ddensity ||
                !out->dfeatures))
    return fail(EVER_ERR_INVALID, "null ellipsoid-side pointer");
  if (log_cap < args->max_iters - 1 && num_rays > 0)
    return fail(EVER_ERR_INVALID, "event log holds %d rows, backward needs max_iters-1 = %d", log_cap,
                args->max_iters - 1);
  if (wct && num_wct < 1) return fail(EVER_ERR_INVALID, "wct given with num_wct < 1");
  int deg = 0;
  if (int rc = resolve_degree(scene, args, &deg)) return rc;
  const size_t need = ever_backward_workspace_bytes(N, scene->sh_coeffs);
  if (N > 0 && (!workspace || workspace_bytes < need))
    return fail(EVER_ERR_WORKSPACE, "backward workspace needs %zu bytes, got %zu", need, workspace_bytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ever::WsCursor c;
  char* ws = static_cast<char*>(workspace);
  float* acc_geo = reinterpret_cast<float*>(ws + c.take(N * 16 * sizeof(float)));
  float* acc_feat = reinterpret_cast<float*>(ws + c.take(N * int64_t(ever::feat_stride(scene->sh_coeffs)) * sizeof(float)));
  int32_t* inv_order = reinterpret_cast<int32_t*>(ws + c.take(N * int64_t(sizeof(int32_t))));
  cudaError_t e = cudaSuccess;
  // degree 0 keeps its DC feature gradients in the geometry rows: only those are cleared
  if (N > 0) e = cudaMemsetAsync(workspace, 0, deg == 0 ? size_t(N) * 16 * sizeof(float) : need, st);
  if (e != cudaSuccess) return cuda_status(e, "ever_trace_backward memset");
  const bool per_ray_wct = wct && num_wct > 1 && out->dmeans2d;
  if (per_ray_wct && N > 0) {
    e = cudaMemsetAsync(out->dmeans2d, 0, N * 2 * sizeof(float), st);
    if (e != cudaSuccess) return cuda_status(e, "ever_trace_backward memset");
  }
  const EverTune tn = resolve_tune(tune);
  if (N > 0) {
    ever::BwdParams P{};
    P.nodes = scene->nodes;
    P.records = scene->records;
    P.features = scene->features;
    P.order = scene->order;
    P.N = N;
    P.K = scene->sh_coeffs;
    P.rayo = rayo;
    P.rayd = rayd;
    P.R = cam ? ever::camera_slots(*cam) : num_rays;  // threads, and the event-log row length
    P.tmin = args->tmin;
    P.tmax = args->tmax;
    P.max_iters = args->max_iters;
    P.ray_order = ray_order;
    P.slot_order = slot_order;
    P.grad_out = grad_out;
    P.states = states;
    P.iters = iters;
    P.event_log = event_log;
    P.log_cap = log_cap;
    P.wct = wct;
    P.num_wct = num_wct;
    P.acc_geo = acc_geo;
    P.acc_feat = acc_feat;
    P.dmeans2d = out->dmeans2d;
    P.drayo = out->drayo;
    P.drayd = out->drayd;
    e = cam ? ever::launch_backward_camera(P, *cam, jitter, deg, tn, st) : ever::launch_backward(P, deg, tn, st);
    if (e != cudaSuccess) return cuda_status(e, "ever_trace_backward");
    ever::FinalizeParams F{};
    F.records = scene->records;
    F.order = scene->order;
    F.N = N;
    F.K = scene->sh_coeffs;
    F.mean = mean;
    F.scale = scale;
    F.quat = quat;
    F.acc_geo = acc_geo;
    F.acc_feat = acc_feat;
    F.inv_order = inv_order;
    F.dc_only = deg == 0;
    F.wct = wct;
    F.num_wct = wct ? num_wct : 0;
    F.out = *out;
    e = ever::launch_finalize(F, st);
    return cuda_status(e, "ever_trace_backward finalize");
  }
  // no ellipsoids: every ray gradient is zero
  if (num_rays > 0 && out->drayo) {
    e = cudaMemsetAsync(out->drayo, 0, num_rays * 3 * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(out->drayd, 0, num_rays * 3 * sizeof(float), st);
  }
  return cuda_status(e, "ever_trace_backward");
}

}  // namespace

extern "C" {

int ever_trace_backward(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                        const EverTraceArgs* args, const float* grad_out, const float* states,
                        const int32_t* iters, const int32_t* event_log, int32_t log_cap, const float* wct,
                        int32_t num_wct, const float* mean, const float* scale, const float* quat, void* workspace,
                        size_t workspace_bytes, const int32_t* ray_order, const EverTune* tune,
                        const EverBackwardOut* out, void* stream) {
  return trace_backward(scene, rayo, rayd, num_rays, args, grad_out, states, iters, event_log, log_cap, wct, num_wct,
                        mean, scale, quat, workspace, workspace_bytes, ray_order, nullptr, tune, out, stream);
}

int ever_trace_backward_ordered(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                                const EverTraceArgs* args, const float* grad_out, const float* states,
                                const int32_t* iters, const int32_t* event_log, int32_t log_cap, const float* wct,
                                int32_t num_wct, const float* mean, const float* scale, const float* quat,
                                void* workspace, size_t workspace_bytes, const int32_t* ray_order,
                                const int32_t* slot_order, const EverTune* tune, const EverBackwardOut* out,
                                void* stream) {
  if (num_rays > 0 && !slot_order) return fail(EVER_ERR_INVALID, "ever_trace_backward_ordered: null slot_order");
  return trace_backward(scene, rayo, rayd, num_rays, args, grad_out, states, iters, event_log, log_cap, wct, num_wct,
                        mean, scale, quat, workspace, workspace_bytes, ray_order, slot_order, tune, out, stream);
}

int ever_backward_slot_order(const int32_t* iters, const int32_t* ray_order, int64_t num_rays, int32_t shift,
                             void* workspace, size_t workspace_bytes, int32_t* slot_order, void* stream) {
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31)) return fail(EVER_ERR_INVALID, "num_rays out of range");
  if (shift < 0 || shift > 16) return fail(EVER_ERR_INVALID, "shift %d out of range 0..16", shift);
  if (num_rays > 0 && (!iters || !slot_order)) return fail(EVER_ERR_INVALID, "null pointer");
  const int64_t need = ever::ray_order_workspace(num_rays);
  if (num_rays > 0 && (!workspace || workspace_bytes < size_t(need)))
    return fail(EVER_ERR_WORKSPACE, "slot order workspace needs %lld bytes, got %zu", (long long)need,
                workspace_bytes);
  return cuda_status(ever::backward_slot_order(iters, ray_order, num_rays, shift, static_cast<char*>(workspace),
                                               slot_order, static_cast<cudaStream_t>(stream)),
                     "ever_backward_slot_order");
}

int ever_event_log_to_reference(const EverScene* scene, const int32_t* event_log, int32_t log_cap,
                                const int32_t* iters, int64_t num_rays, const int32_t* ray_order,
                                int32_t* tri_collection, int32_t max_iters, void* stream) {
  if (!scene || (num_rays > 0 && max_iters > 0 && (!event_log || !iters || !tri_collection)))
    return fail(EVER_ERR_INVALID, "null pointer");
  return cuda_status(ever::launch_log_to_reference(scene->order, event_log, log_cap, iters, num_rays, ray_order,
                                                   tri_collection, max_iters, static_cast<cudaStream_t>(stream)),
                     "ever_event_log_to_reference");
}

size_t ever_ray_order_workspace_bytes(int64_t num_rays) {
  if (num_rays < 0) return 0;
  return size_t(ever::ray_order_workspace(num_rays));
}

int ever_ray_order(const float* rayo, const float* rayd, int64_t num_rays, void* workspace, size_t workspace_bytes,
                   int32_t* ray_order, void* stream) {
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31)) return fail(EVER_ERR_INVALID, "num_rays out of range");
  if (num_rays > 0 && (!rayo || !rayd || !ray_order)) return fail(EVER_ERR_INVALID, "null pointer");
  const int64_t need = ever::ray_order_workspace(num_rays);
  if (num_rays > 0 && (!workspace || workspace_bytes < size_t(need)))
    return fail(EVER_ERR_WORKSPACE, "ray order workspace needs %lld bytes, got %zu", (long long)need, workspace_bytes);
  return cuda_status(ever::ray_order(rayo, rayd, num_rays, static_cast<char*>(workspace), ray_order,
                                     static_cast<cudaStream_t>(stream)),
                     "ever_ray_order");
}

// ---- camera traces: rays made from the camera inside the kernels ----

int64_t ever_camera_slots(const EverCamera* camera) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C)) {
    fail(EVER_ERR_INVALID, "ever_camera_slots: %s", msg);
    return -1;
  }
  return ever::camera_slots(C);
}

int ever_camera_slot_pixels(const EverCamera* camera, int32_t* slot_pixel, void* stream) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_camera_slot_pixels: %s", msg);
  if (ever::camera_slots(C) > 0 && !slot_pixel) return fail(EVER_ERR_INVALID, "ever_camera_slot_pixels: null output");
  return cuda_status(ever::launch_camera_slot_pixels(C, slot_pixel, static_cast<cudaStream_t>(stream)),
                     "ever_camera_slot_pixels");
}

int ever_trace_forward_camera(const EverScene* scene, const EverCamera* camera, const float* jitter,
                              const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                              void* stream) {
  if (!scene || !args || !out) return fail(EVER_ERR_INVALID, "null scene, args or out");
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_trace_forward_camera: %s", msg);
  const int64_t R = int64_t(C.width) * C.height;
  if (R > 0 && (!out->out || !out->iters)) return fail(EVER_ERR_INVALID, "null out or iters");
  if (out->event_log && out->log_cap < 0) return fail(EVER_ERR_INVALID, "negative log_cap");
  int deg = 0;
  if (int rc = resolve_degree(scene, args, &deg)) return rc;
  ever::FwdParams P{};
  P.nodes = scene->nodes;
  P.records = scene->records;
  P.features = scene->features;
  P.order = scene->order;
  P.N = scene->num_prims;
  P.K = scene->sh_coeffs;
  P.R = R;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.out = *out;
  P.depth_hint = args->depth_hint;
  return cuda_status(
      ever::launch_forward_camera(P, C, jitter, deg, resolve_tune(tune), static_cast<cudaStream_t>(stream)),
      "ever_trace_forward_camera");
}

int ever_trace_forward_camera_regrouped(const EverScene* scene, const EverCamera* camera, const float* jitter,
                                        const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                                        void* workspace, size_t workspace_bytes, void* stream) {
  if (!scene || !args || !out) return fail(EVER_ERR_INVALID, "null scene, args or out");
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_trace_forward_camera_regrouped: %s", msg);
  const int64_t R = int64_t(C.width) * C.height, S = ever::camera_slots(C);
  if (R > 0 && (!out->out || !out->iters || !out->states || !out->last_dirac))
    return fail(EVER_ERR_INVALID, "null out, iters, states or last_dirac");
  if (out->event_log && out->log_cap < 0) return fail(EVER_ERR_INVALID, "negative log_cap");
  const int64_t need = ever::regroup_workspace(S);
  if (R > 0 && (!workspace || workspace_bytes < size_t(need)))
    return fail(EVER_ERR_WORKSPACE, "forward workspace needs %lld bytes, got %zu", (long long)need, workspace_bytes);
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(EVER_ERR_INVALID, "workspace not 256-byte aligned");
  int deg = 0;
  if (int rc = resolve_degree(scene, args, &deg)) return rc;
  ever::FwdParams P{};
  P.nodes = scene->nodes;
  P.records = scene->records;
  P.features = scene->features;
  P.order = scene->order;
  P.N = scene->num_prims;
  P.K = scene->sh_coeffs;
  P.R = R;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.out = *out;
  P.depth_hint = args->depth_hint;
  if (R == 0) return EVER_OK;
  const ever::RegroupScratch W = ever::regroup_scratch(static_cast<char*>(workspace), S);
  return cuda_status(ever::launch_forward_regrouped(P, W, &C, jitter, deg, resolve_tune(tune),
                                                    static_cast<cudaStream_t>(stream)),
                     "ever_trace_forward_camera_regrouped");
}

int ever_trace_backward_camera(const EverScene* scene, const EverCamera* camera, const float* jitter,
                               const EverTraceArgs* args, const float* grad_out, const float* states,
                               const int32_t* iters, const int32_t* event_log, int32_t log_cap, const float* wct,
                               int32_t num_wct, const float* mean, const float* scale, const float* quat,
                               void* workspace, size_t workspace_bytes, const int32_t* slot_order,
                               const EverTune* tune, const EverBackwardOut* out, void* stream) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_trace_backward_camera: %s", msg);
  return trace_backward(scene, nullptr, nullptr, int64_t(C.width) * C.height, args, grad_out, states, iters,
                        event_log, log_cap, wct, num_wct, mean, scale, quat, workspace, workspace_bytes, nullptr,
                        slot_order, tune, out, stream, &C, jitter);
}

int ever_camera_backward_slot_order(const EverCamera* camera, const int32_t* iters, int32_t shift, void* workspace,
                                    size_t workspace_bytes, int32_t* slot_order, void* stream) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_camera_backward_slot_order: %s", msg);
  if (shift < 0 || shift > 16) return fail(EVER_ERR_INVALID, "shift %d out of range 0..16", shift);
  const int64_t S = ever::camera_slots(C);
  if (S > 0 && (!iters || !slot_order)) return fail(EVER_ERR_INVALID, "null pointer");
  const int64_t need = ever::ray_order_workspace(S);
  if (S > 0 && (!workspace || workspace_bytes < size_t(need)))
    return fail(EVER_ERR_WORKSPACE, "slot order workspace needs %lld bytes, got %zu", (long long)need,
                workspace_bytes);
  return cuda_status(ever::camera_backward_slot_order(C, iters, shift, static_cast<char*>(workspace), slot_order,
                                                      static_cast<cudaStream_t>(stream)),
                     "ever_camera_backward_slot_order");
}

int ever_camera_event_log_to_reference(const EverScene* scene, const EverCamera* camera, const int32_t* event_log,
                                       int32_t log_cap, const int32_t* iters, int32_t* tri_collection,
                                       int32_t max_iters, void* stream) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return fail(EVER_ERR_INVALID, "ever_camera_event_log_to_reference: %s", msg);
  if (!scene || (int64_t(C.width) * C.height > 0 && max_iters > 0 && (!event_log || !iters || !tri_collection)))
    return fail(EVER_ERR_INVALID, "null pointer");
  return cuda_status(ever::launch_camera_log_to_reference(C, scene->order, event_log, log_cap, iters, tri_collection,
                                                          max_iters, static_cast<cudaStream_t>(stream)),
                     "ever_camera_event_log_to_reference");
}

}  // extern "C"
