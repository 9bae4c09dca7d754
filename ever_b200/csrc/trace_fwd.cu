// Forward trace dispatch: k-buffer size -> the instantiations in trace_fwd_k{8,16,32}.cu
// (kernels in trace_fwd.cuh).
#include "common.cuh"
#include "internal.cuh"

namespace ever {

cudaError_t launch_forward_batched(const BatchFwdParams& P, int deg, const EverTune& tune, cudaStream_t st) {
  if (P.num_slots == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_batched_k<8>(P, deg, block, st);
    case 32: return launch_forward_batched_k<32>(P, deg, block, st);
    default: return launch_forward_batched_k<16>(P, deg, block, st);
  }
}

cudaError_t launch_forward(const FwdParams& P, int deg, const EverTune& tune, cudaStream_t st) {
  if (P.R == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_k<8>(P, deg, block, tune.traversal, st);
    case 32: return launch_forward_k<32>(P, deg, block, tune.traversal, st);
    default: return launch_forward_k<16>(P, deg, block, tune.traversal, st);
  }
}

cudaError_t launch_forward_camera(const FwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                  const EverTune& tune, cudaStream_t st) {
  if (int64_t(cam.width) * cam.height == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_camera_k<8>(P, cam, jitter, deg, block, st);
    case 32: return launch_forward_camera_k<32>(P, cam, jitter, deg, block, st);
    default: return launch_forward_camera_k<16>(P, cam, jitter, deg, block, st);
  }
}

}  // namespace ever
