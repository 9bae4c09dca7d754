// extern "C" entry points of the ray-cost model and the cost-binned ray orders
// (declared in include/ever_b200.h). No counterpart in the reference.
#include <cstdio>

#include "common.cuh"
#include "internal.cuh"

namespace {

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return EVER_OK;
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
  return ever::set_last_error(EVER_ERR_CUDA, buf);
}

bool mlp_valid(const EverMlp* m) { return m && m->params && m->w1 && m->w2 && m->w3; }

ever::MlpParams base_params(const EverMlp* m) {
  ever::MlpParams P{};
  P.w1 = m->w1;
  P.w2 = m->w2;
  P.w3 = m->w3;
  P.params = m->params;
  P.cx = m->centre[0];
  P.cy = m->centre[1];
  P.cz = m->centre[2];
  P.inv_scale = m->inv_scale;
  P.wait_clocks = m->wait_clocks;
  return P;
}

}  // namespace

extern "C" {

size_t ever_mlp_workspace_bytes(void) { return size_t(ever::kMlpMaxGrid) * (ever::kMlpParams + 1) * sizeof(float); }

int ever_mlp_pack(const EverMlp* mlp, void* stream) {
  if (!mlp_valid(mlp)) return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_pack: null pointer");
  return cuda_status(ever::launch_mlp_pack(mlp->params, mlp->w1, mlp->w2, mlp->w3, static_cast<cudaStream_t>(stream)),
                     "ever_mlp_pack");
}

int ever_mlp_predict(const EverMlp* mlp, const float* rayo, const float* rayd, const float* feat, int64_t num_rays,
                     float* pred, uint8_t* bins, const float* thresholds, int32_t* error, void* stream) {
  if (!mlp_valid(mlp)) return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_predict: null model pointer");
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_predict: num_rays out of range");
  if (num_rays > 0 && (!pred || !error || (!feat && (!rayo || !rayd)) || (bins && !thresholds)))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_predict: null pointer");
  ever::MlpParams P = base_params(mlp);
  P.rayo = rayo;
  P.rayd = rayd;
  P.feat = feat;
  P.num_samples = num_rays;
  P.pred = pred;
  P.bins = bins;
  if (bins)
    for (int i = 0; i < 3; ++i) P.thr[i] = thresholds[i];
  P.error = error;
  const int grid = ever::mlp_grid(num_rays, sm_count(), false);
  return cuda_status(ever::launch_mlp(P, false, grid, static_cast<cudaStream_t>(stream)), "ever_mlp_predict");
}

int ever_mlp_gradients(const EverMlp* mlp, const float* rayo, const float* rayd, const float* feat,
                       const int32_t* sample_idx, int64_t num_samples, const float* target, float loss_w0,
                       float loss_w1, float* grads, float* loss, void* workspace, size_t workspace_bytes,
                       int32_t* error, void* stream) {
  if (!mlp_valid(mlp)) return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_gradients: null model pointer");
  if (num_samples <= 0 || num_samples >= (int64_t(1) << 31))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_gradients: num_samples out of range [1, 2^31)");
  if (!target || !grads || !error || (!feat && (!rayo || !rayd)))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_gradients: null pointer");
  if (!workspace || workspace_bytes < ever_mlp_workspace_bytes())
    return ever::set_last_error(EVER_ERR_WORKSPACE, "ever_mlp_gradients: workspace too small");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  ever::MlpParams P = base_params(mlp);
  P.rayo = rayo;
  P.rayd = rayd;
  P.feat = feat;
  P.sample_idx = sample_idx;
  P.num_samples = num_samples;
  P.target = target;
  P.loss_w0 = loss_w0;
  P.loss_w1 = loss_w1;
  P.inv_batch = 1.f / float(num_samples);
  P.partial = static_cast<float*>(workspace);
  P.error = error;
  const int grid = ever::mlp_grid(num_samples, std::min(sm_count(), ever::kMlpMaxGrid), true);
  cudaError_t e = ever::launch_mlp(P, true, grid, st);
  if (e == cudaSuccess) e = ever::launch_mlp_reduce(P.partial, grid, grads, loss, st);
  return cuda_status(e, "ever_mlp_gradients");
}

int ever_mlp_adam(const EverMlp* mlp, const float* grads, float* adam_m, float* adam_v, float lr, float beta1,
                  float beta2, float eps, int32_t step, void* stream) {
  if (!mlp_valid(mlp) || !grads || !adam_m || !adam_v)
    return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_adam: null pointer");
  if (step < 1) return ever::set_last_error(EVER_ERR_INVALID, "ever_mlp_adam: step counts from 1");
  return cuda_status(ever::launch_mlp_adam(mlp->params, grads, adam_m, adam_v, mlp->w1, mlp->w2, mlp->w3, lr, beta1,
                                           beta2, eps, step, static_cast<cudaStream_t>(stream)),
                     "ever_mlp_adam");
}

int ever_ray_order_binned(const float* rayo, const float* rayd, const uint8_t* bins, int64_t num_rays,
                          void* workspace, size_t workspace_bytes, int32_t* ray_order, void* stream) {
  if (num_rays < 0 || num_rays >= (int64_t(1) << 31))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_ray_order_binned: num_rays out of range");
  if (num_rays > 0 && (!rayo || !rayd || !bins || !ray_order))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_ray_order_binned: null pointer");
  if (num_rays > 0 && (!workspace || workspace_bytes < size_t(ever::ray_order_workspace(num_rays))))
    return ever::set_last_error(EVER_ERR_WORKSPACE, "ever_ray_order_binned: workspace too small");
  return cuda_status(ever::ray_order(rayo, rayd, num_rays, static_cast<char*>(workspace), ray_order,
                                     static_cast<cudaStream_t>(stream), bins),
                     "ever_ray_order_binned");
}

int ever_batch_order_binned(const EverBatch* batch, const float* rayo, const float* rayd, const uint8_t* bins,
                            void* stream) {
  if (!batch || !batch->slot_ray || (batch->num_rays > 0 && (!rayo || !rayd || !bins)))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_batch_order_binned: null pointer");
  return cuda_status(ever::batch_ray_order(rayo, rayd, batch->num_rays,
                                           static_cast<const ever::BatchView*>(batch->view_table), batch->num_views,
                                           static_cast<char*>(batch->order_scratch), batch->slot_ray, batch->num_slots,
                                           static_cast<cudaStream_t>(stream), bins),
                     "ever_batch_order_binned");
}

}  // extern "C"
