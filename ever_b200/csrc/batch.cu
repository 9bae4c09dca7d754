// Batched tracing: C entry points that lay out a batch of views over several scenes and
// drive the persistent forward/backward kernels (trace_fwd.cu, trace_bwd.cu).
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr int kMaxBatch = 64;

struct BatchLayout {
  int64_t scene_table, view_table, slot_ray, counters, order_scratch, total;
  int64_t num_slots;
};

BatchLayout batch_layout(int num_scenes, const EverBatchView* views, int num_views) {
  BatchLayout L{};
  int64_t slots = 0, rays = 0;
  for (int v = 0; v < num_views; ++v) {
    slots += (views[v].ray_count + 31) / 32 * 32;
    rays += views[v].ray_count;
  }
  WsCursor c;
  L.scene_table = c.take(int64_t(num_scenes) * sizeof(BatchScene));
  L.view_table = c.take(int64_t(num_views) * sizeof(BatchView));
  L.slot_ray = c.take(slots * sizeof(int32_t));
  L.counters = c.take(4 * sizeof(uint32_t));
  // sort scratch for the ray order (rays) and the backward's slot order (slots), followed
  // by the backward's slot order itself
  L.order_scratch = c.take(ray_order_workspace(std::max<int64_t>(slots, 1)) + std::max<int64_t>(slots, 1) * 4);
  L.total = c.offset;
  L.num_slots = slots;
  return L;
}

// sh_degree < 0: the reference's DC-only forward colour (as ever_trace_forward)
int degree_of(int K, int sh_degree) {
  (void)K;
  return sh_degree >= 0 ? sh_degree : 0;
}

EverTune tune_of(const EverTune* t) {
  EverTune r{};
  if (t) r = *t;
  if (r.kbuf != 8 && r.kbuf != 16 && r.kbuf != 32) r.kbuf = 16;
  if (r.block != 64 && r.block != 128 && r.block != 256) r.block = 128;
  r.stack_depth = r.stack_depth <= 0 ? kStackDepth : std::min(std::max(r.stack_depth, 8), kStackDepth);
  return r;
}

// Persistent grid: enough resident blocks to fill every SM. Occupancy is bounded by
// registers: 20 warps per SM for the forward with blocks of 64 or 128 threads, 16 warps
// with 256 threads; 24 warps for the degree-0 backward, 16 with SH colour.
int persistent_grid(int block, bool forward, int deg = 0) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int warps_per_sm = forward ? (block <= 128 ? 20 : 16) : (deg == 0 ? 24 : 16);
  return std::max(1, sms * std::max(1, warps_per_sm * 32 / block));
}

}  // namespace
}  // namespace ever

using namespace ever;

extern "C" {

size_t ever_batch_workspace_bytes(int32_t num_scenes, const EverBatchView* views, int32_t num_views,
                                  int64_t* num_slots) {
  if (num_scenes < 1 || num_scenes > kMaxBatch || num_views < 1 || num_views > kMaxBatch || !views) return 0;
  const BatchLayout L = batch_layout(num_scenes, views, num_views);
  if (num_slots) *num_slots = L.num_slots;
  return size_t(L.total);
}

int ever_batch_setup(const EverScene* scenes, void* const* bwd_workspaces, int32_t num_scenes,
                     const EverBatchView* views, int32_t num_views, int64_t num_rays, void* workspace,
                     size_t workspace_bytes, EverBatch* batch) {
  if (!scenes || !views || !batch || !workspace) return set_last_error(EVER_ERR_INVALID, "ever_batch_setup: null pointer");
  if (num_scenes < 1 || num_scenes > kMaxBatch || num_views < 1 || num_views > kMaxBatch)
    return set_last_error(EVER_ERR_INVALID, "ever_batch_setup: 1..64 scenes and 1..64 views");
  int64_t expect = 0;
  for (int v = 0; v < num_views; ++v) {
    const EverBatchView& w = views[v];
    if (w.scene < 0 || w.scene >= num_scenes || w.ray_offset != expect || w.ray_count < 0 ||
        w.ray_count >= (int64_t(1) << 31))
      return set_last_error(EVER_ERR_INVALID, "ever_batch_setup: views must tile the rays in order");
    expect += w.ray_count;
  }
  if (expect != num_rays) return set_last_error(EVER_ERR_INVALID, "ever_batch_setup: views do not cover num_rays");
  const BatchLayout L = batch_layout(num_scenes, views, num_views);
  if (workspace_bytes < size_t(L.total)) return set_last_error(EVER_ERR_WORKSPACE, "ever_batch_setup: workspace too small");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return set_last_error(EVER_ERR_INVALID, "ever_batch_setup: workspace not 256-byte aligned");
  char* ws = static_cast<char*>(workspace);
  std::memset(batch, 0, sizeof(*batch));
  std::vector<BatchScene> st(num_scenes);
  for (int i = 0; i < num_scenes; ++i) {
    const EverScene& sc = scenes[i];
    BatchScene& b = st[i];
    b.nodes = sc.nodes;
    b.records = sc.records;
    b.features = sc.features;
    b.order = sc.order;
    b.N = sc.num_prims;
    b.K = sc.sh_coeffs;
    b.pad = 0;
    b.acc_geo = nullptr;
    b.acc_feat = nullptr;
    if (bwd_workspaces && bwd_workspaces[i]) {
      WsCursor c;
      char* bw = static_cast<char*>(bwd_workspaces[i]);
      b.acc_geo = reinterpret_cast<float*>(bw + c.take(sc.num_prims * 16 * sizeof(float)));
      b.acc_feat =
          reinterpret_cast<float*>(bw + c.take(sc.num_prims * int64_t(feat_stride(sc.sh_coeffs)) * sizeof(float)));
    }
    batch->sh_coeffs[i] = sc.sh_coeffs;
    batch->num_prims[i] = sc.num_prims;
    batch->bwd_workspace[i] = bwd_workspaces ? bwd_workspaces[i] : nullptr;
  }
  std::vector<BatchView> vt(num_views);
  int64_t off = 0;
  for (int v = 0; v < num_views; ++v) {
    vt[v].slot_offset = off;
    vt[v].slot_count = (views[v].ray_count + 31) / 32 * 32;
    vt[v].ray_offset = views[v].ray_offset;
    vt[v].ray_count = views[v].ray_count;
    vt[v].scene = views[v].scene;
    vt[v].pad = 0;
    off += vt[v].slot_count;
  }
  cudaError_t e = cudaMemcpy(ws + L.scene_table, st.data(), st.size() * sizeof(BatchScene), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ws + L.view_table, vt.data(), vt.size() * sizeof(BatchView), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  batch->num_scenes = num_scenes;
  batch->num_views = num_views;
  batch->num_slots = L.num_slots;
  batch->num_rays = num_rays;
  batch->scene_table = ws + L.scene_table;
  batch->view_table = ws + L.view_table;
  batch->slot_ray = reinterpret_cast<int32_t*>(ws + L.slot_ray);
  batch->counters = reinterpret_cast<uint32_t*>(ws + L.counters);
  batch->order_scratch = ws + L.order_scratch;
  return EVER_OK;
}

int ever_batch_order(const EverBatch* batch, const float* rayo, const float* rayd, void* stream) {
  if (!batch || !batch->slot_ray || (batch->num_rays > 0 && (!rayo || !rayd)))
    return set_last_error(EVER_ERR_INVALID, "ever_batch_order: null pointer");
  const cudaError_t e = batch_ray_order(rayo, rayd, batch->num_rays, static_cast<const BatchView*>(batch->view_table),
                                        batch->num_views, static_cast<char*>(batch->order_scratch), batch->slot_ray,
                                        batch->num_slots, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

int ever_trace_forward_batched(const EverBatch* batch, const float* rayo, const float* rayd,
                               const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                               void* stream) {
  if (!batch || !args || !out || !out->out || !out->iters || !rayo || !rayd)
    return set_last_error(EVER_ERR_INVALID, "ever_trace_forward_batched: null pointer");
  const int deg = degree_of(batch->sh_coeffs[0], args->sh_degree);
  for (int i = 0; i < batch->num_scenes; ++i)
    if (deg < 0 || deg > 3 || (deg + 1) * (deg + 1) > batch->sh_coeffs[i])
      return set_last_error(EVER_ERR_INVALID, "ever_trace_forward_batched: scenes do not support the SH degree");
  const EverTune tn = tune_of(tune);
  BatchFwdParams P{};
  P.scenes = static_cast<const BatchScene*>(batch->scene_table);
  P.views = static_cast<const BatchView*>(batch->view_table);
  P.num_views = batch->num_views;
  P.slot_ray = batch->slot_ray;
  P.num_slots = batch->num_slots;
  P.rayo = rayo;
  P.rayd = rayd;
  P.R = batch->num_rays;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.out = *out;
  P.work_counter = batch->counters;
  P.grid = persistent_grid(tn.block, true);
  const cudaError_t e = launch_forward_batched(P, deg, tn, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

int ever_trace_backward_batched(const EverBatch* batch, const float* rayo, const float* rayd,
                                const EverTraceArgs* args, const float* grad_out, const float* states,
                                const int32_t* iters, const int32_t* event_log, int32_t log_cap, float* drayo,
                                float* drayd, const EverTune* tune, void* stream) {
  if (!batch || !args || !rayo || !rayd || !grad_out || !states || !iters || !event_log || !drayo || !drayd)
    return set_last_error(EVER_ERR_INVALID, "ever_trace_backward_batched: null pointer");
  if (log_cap < args->max_iters - 1)
    return set_last_error(EVER_ERR_INVALID, "ever_trace_backward_batched: event log shorter than max_iters-1");
  const int deg = degree_of(batch->sh_coeffs[0], args->sh_degree);
  if (deg < 0 || deg > 3) return set_last_error(EVER_ERR_INVALID, "ever_trace_backward_batched: bad SH degree");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // zero every scene's accumulators (one contiguous workspace per scene)
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < batch->num_scenes; ++i) {
    if (!batch->bwd_workspace[i])
      return set_last_error(EVER_ERR_INVALID, "ever_trace_backward_batched: scene without backward workspace");
    WsCursor c;
    c.take(batch->num_prims[i] * 16 * sizeof(float));
    c.take(batch->num_prims[i] * int64_t(feat_stride(batch->sh_coeffs[i])) * sizeof(float));
    e = cudaMemsetAsync(batch->bwd_workspace[i], 0, size_t(c.offset), st);
    if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  }
  const EverTune tn = tune_of(tune);
  BatchBwdParams P{};
  P.scenes = static_cast<const BatchScene*>(batch->scene_table);
  P.views = static_cast<const BatchView*>(batch->view_table);
  P.num_views = batch->num_views;
  P.slot_ray = batch->slot_ray;
  P.num_slots = batch->num_slots;
  P.rayo = rayo;
  P.rayd = rayd;
  P.R = batch->num_rays;
  P.tmin = args->tmin;
  P.tmax = args->tmax;
  P.max_iters = args->max_iters;
  P.grad_out = grad_out;
  P.states = states;
  P.iters = iters;
  P.event_log = event_log;
  P.log_cap = log_cap;
  P.drayo = drayo;
  P.drayd = drayd;
  P.work_counter = batch->counters + 1;
  P.grid = persistent_grid(tn.block, false, deg);
  // replay order: inside each view, slots grouped by their rays' event counts (longest first)
  char* scratch = static_cast<char*>(batch->order_scratch);
  int32_t* slots = reinterpret_cast<int32_t*>(scratch + ray_order_workspace(std::max<int64_t>(batch->num_slots, 1)));
  e = backward_slot_order(iters, batch->slot_ray, batch->num_slots, 0, scratch, slots, st,
                          static_cast<const BatchView*>(batch->view_table), batch->num_views);
  if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  P.slot_order = slots;
  e = launch_backward_batched(P, deg, tn, st);
  return e == cudaSuccess ? EVER_OK : set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

int ever_scene_finalize_gradients(const EverScene* scene, const float* mean, const float* scale,
                                  const float* quat, void* bwd_workspace, size_t bwd_workspace_bytes,
                                  const EverBackwardOut* out, void* stream) {
  if (!scene || !out) return set_last_error(EVER_ERR_INVALID, "ever_scene_finalize_gradients: null pointer");
  const int64_t N = scene->num_prims;
  if (N == 0) return EVER_OK;
  if (!mean || !scale || !quat || !bwd_workspace || !out->dmean || !out->dscale || !out->dquat || !out->ddensity ||
      !out->dfeatures)
    return set_last_error(EVER_ERR_INVALID, "ever_scene_finalize_gradients: null pointer");
  WsCursor c;
  char* bw = static_cast<char*>(bwd_workspace);
  const int64_t g = c.take(N * 16 * sizeof(float));
  const int64_t f = c.take(N * int64_t(feat_stride(scene->sh_coeffs)) * sizeof(float));
  const int64_t v = c.take(N * int64_t(sizeof(int32_t)));
  if (bwd_workspace_bytes < size_t(c.offset))
    return set_last_error(EVER_ERR_WORKSPACE, "ever_scene_finalize_gradients: workspace too small");
  FinalizeParams F{};
  F.records = scene->records;
  F.order = scene->order;
  F.N = N;
  F.K = scene->sh_coeffs;
  F.mean = mean;
  F.scale = scale;
  F.quat = quat;
  F.acc_geo = reinterpret_cast<const float*>(bw + g);
  F.acc_feat = reinterpret_cast<const float*>(bw + f);
  F.inv_order = reinterpret_cast<int32_t*>(bw + v);
  F.wct = nullptr;
  F.num_wct = 0;
  F.out = *out;
  F.out.dmeans2d = nullptr;
  const cudaError_t e = launch_finalize(F, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
