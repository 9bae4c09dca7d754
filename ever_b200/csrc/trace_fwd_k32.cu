// Forward trace kernels with a 32-event buffer (trace_fwd.cuh).
#include "trace_fwd.cuh"

namespace ever {

template <>
cudaError_t launch_forward_k<32>(const FwdParams& P, int deg, int block, int traversal, cudaStream_t st) {
  return launch_k<32>(P, deg, block, traversal, st);
}

template <>
cudaError_t launch_forward_camera_k<32>(const FwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                         int block, cudaStream_t st) {
  return launch_camera_k<32>(P, cam, jitter, deg, block, st);
}

template <>
cudaError_t launch_forward_regrouped_k<32>(const FwdParams& P, const RegroupScratch& W, const CameraParams* cam,
                                            const float* jitter, int deg, int block, cudaStream_t st) {
  return launch_regrouped_k<32>(P, W, cam, jitter, deg, block, st);
}

template <>
cudaError_t launch_forward_batched_k<32>(const BatchFwdParams& P, int deg, int block, cudaStream_t st) {
  return launch_batched_k<32>(P, deg, block, st);
}

}  // namespace ever
