// Per-ellipsoid colour pre-pass of the trainer, and camera ray generation.
//
// Colour pre-pass (reference: splinetracers/slang/sh_kernel.slang:21-99, eval_sh.py:28-82,
// used at integration_utils/gaussian_renderer/ever.py:178-180): for ellipsoid i, the SH of
// degree `sh_degree` is evaluated in the direction normalize(mean_i - cam) from the camera
// centre, colour c = sum_k B_k f_ik + 0.5 (sh.slang:49-100). Mode 0 writes c (N,3), as
// eval_sh does; mode 1 writes the trainer's tracer input RGB2SH(softplus(c, beta = 10)),
// one degree-0 coefficient per channel (N,1,3), in one pass instead of three kernels and
// two (N,3) round trips. The backward returns the feature gradient only, like the
// reference (no gradient reaches the means through the direction), and skips an
// ellipsoid whose colour gradient is below 1e-8 in every channel (sh_kernel.slang:64-67).
//
// Camera rays (reference: integration_utils/gaussian_renderer/ever.py:29-74, 105-118):
// pixel (row, col) -> d = normalize(((col + ox) - cx) / fx, ((row + oy) - cy) / fy, 1),
// rayd = R d, rayo = camera centre, where [R | t] is the camera-to-world matrix; the
// offsets (ox, oy) are 0.5 (pixel centres) or given per pixel (the trainer's random
// jitter). Rays are row-major over the image.
#include <string>

#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

__device__ __forceinline__ float softplus10(float x) {  // torch softplus, beta 10, threshold 20
  return 10.f * x > 20.f ? x : log1pf(expf(10.f * x)) / 10.f;
}
__device__ __forceinline__ float softplus10_grad(float x) {
  if (10.f * x > 20.f) return 1.f;
  const float z = expf(10.f * x);
  return z / (z + 1.f);
}

template <int DEG>
__device__ __forceinline__ void prepass_colour(const float* __restrict__ mean, const float* __restrict__ feat,
                                               int64_t i, int K, float3 cam, float* B, float (&c)[3]) {
  const float vx = mean[3 * i] - cam.x, vy = mean[3 * i + 1] - cam.y, vz = mean[3 * i + 2] - cam.z;
  const float n = sqrtf(vx * vx + vy * vy + vz * vz);
  const float inv = n > 0.f ? 1.f / n : 0.f;  // an ellipsoid at the camera centre: DC term only
  sh_basis<DEG>(make_float3(vx * inv, vy * inv, vz * inv), B);
  constexpr int NB = (DEG + 1) * (DEG + 1);
  const float* f = feat + i * int64_t(3 * K);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < NB; ++k) s = s + B[k] * f[3 * k + ch];
    c[ch] = s + 0.5f;
  }
}

template <int DEG>
__global__ void k_sh_prepass(const float* __restrict__ mean, const float* __restrict__ feat, int64_t N, int K,
                             const float* __restrict__ cam, int mode, float* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float B[16], c[3];
  prepass_colour<DEG>(mean, feat, i, K, make_float3(cam[0], cam[1], cam[2]), B, c);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) out[3 * i + ch] = mode == 1 ? (softplus10(c[ch]) - 0.5f) / kShC0 : c[ch];
}

template <int DEG>
__global__ void k_sh_prepass_bwd(const float* __restrict__ mean, const float* __restrict__ feat, int64_t N, int K,
                                 const float* __restrict__ cam, int mode, const float* __restrict__ grad_out,
                                 float* __restrict__ grad_feat) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float B[16], c[3], g[3];
  prepass_colour<DEG>(mean, feat, i, K, make_float3(cam[0], cam[1], cam[2]), B, c);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float go = grad_out[3 * i + ch];
    g[ch] = mode == 1 ? (go / kShC0) * softplus10_grad(c[ch]) : go;
  }
  const bool skip = fabsf(g[0]) < 1e-8f && fabsf(g[1]) < 1e-8f && fabsf(g[2]) < 1e-8f;
  constexpr int NB = (DEG + 1) * (DEG + 1);
  float* gf = grad_feat + i * int64_t(3 * K);
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) gf[3 * k + ch] = (!skip && k < NB) ? B[k] * g[ch] : 0.f;
}

__global__ void k_camera_rays(CameraParams C, const float* __restrict__ jitter, float* __restrict__ rayo,
                              float* __restrict__ rayd) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t R = int64_t(C.width) * C.height;
  if (p >= R) return;
  float3 o, d;
  camera_ray(C, jitter, p, o, d);
  rayo[3 * p] = o.x;
  rayo[3 * p + 1] = o.y;
  rayo[3 * p + 2] = o.z;
  rayd[3 * p] = d.x;
  rayd[3 * p + 1] = d.y;
  rayd[3 * p + 2] = d.z;
}

template <int DEG>
cudaError_t prepass_t(const float* mean, const float* feat, int64_t N, int K, const float* cam, int mode,
                      const float* grad_out, float* out, cudaStream_t st) {
  const unsigned grid = unsigned((N + 255) / 256);
  if (grad_out) k_sh_prepass_bwd<DEG><<<grid, 256, 0, st>>>(mean, feat, N, K, cam, mode, grad_out, out);
  else k_sh_prepass<DEG><<<grid, 256, 0, st>>>(mean, feat, N, K, cam, mode, out);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sh_prepass(const float* mean, const float* feat, int64_t N, int K, int deg, const float* cam,
                              int mode, const float* grad_out, float* out, cudaStream_t st) {
  if (N == 0) return cudaSuccess;
  switch (deg) {
    case 0: return prepass_t<0>(mean, feat, N, K, cam, mode, grad_out, out, st);
    case 1: return prepass_t<1>(mean, feat, N, K, cam, mode, grad_out, out, st);
    case 2: return prepass_t<2>(mean, feat, N, K, cam, mode, grad_out, out, st);
    default: return prepass_t<3>(mean, feat, N, K, cam, mode, grad_out, out, st);
  }
}

cudaError_t launch_camera_rays(const CameraParams& C, const float* jitter, float* rayo, float* rayd,
                               cudaStream_t st) {
  const int64_t R = int64_t(C.width) * C.height;
  if (R == 0) return cudaSuccess;
  k_camera_rays<<<unsigned((R + 255) / 256), 256, 0, st>>>(C, jitter, rayo, rayd);
  return cudaGetLastError();
}

}  // namespace ever

extern "C" {

int ever_sh_prepass(const float* mean, const float* features, int64_t num_prims, int32_t sh_coeffs,
                    int32_t sh_degree, const float* cam_pos, int32_t mode, float* out, void* stream) {
  if (num_prims < 0) return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass: num_prims < 0");
  if (sh_degree < 0 || sh_degree > 3 || (sh_degree + 1) * (sh_degree + 1) > sh_coeffs || sh_coeffs > 16)
    return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass: sh_degree needs (sh_degree+1)^2 <= sh_coeffs <= 16");
  if (mode != 0 && mode != 1) return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass: mode must be 0 or 1");
  if (num_prims > 0 && (!mean || !features || !cam_pos || !out))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass: null pointer");
  const cudaError_t e = ever::launch_sh_prepass(mean, features, num_prims, sh_coeffs, sh_degree, cam_pos, mode,
                                                nullptr, out, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : ever::set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

int ever_sh_prepass_backward(const float* mean, const float* features, int64_t num_prims, int32_t sh_coeffs,
                             int32_t sh_degree, const float* cam_pos, int32_t mode, const float* grad_out,
                             float* grad_features, void* stream) {
  if (num_prims < 0) return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass_backward: num_prims < 0");
  if (sh_degree < 0 || sh_degree > 3 || (sh_degree + 1) * (sh_degree + 1) > sh_coeffs || sh_coeffs > 16)
    return ever::set_last_error(EVER_ERR_INVALID,
                                "ever_sh_prepass_backward: sh_degree needs (sh_degree+1)^2 <= sh_coeffs <= 16");
  if (mode != 0 && mode != 1)
    return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass_backward: mode must be 0 or 1");
  if (num_prims > 0 && (!mean || !features || !cam_pos || !grad_out || !grad_features))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_sh_prepass_backward: null pointer");
  const cudaError_t e = ever::launch_sh_prepass(mean, features, num_prims, sh_coeffs, sh_degree, cam_pos, mode,
                                                grad_out, grad_features, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : ever::set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

int ever_camera_rays(const EverCamera* camera, const float* jitter, float* rayo, float* rayd, void* stream) {
  ever::CameraParams C{};
  if (const char* msg = ever::camera_params(camera, &C))
    return ever::set_last_error(EVER_ERR_INVALID, (std::string("ever_camera_rays: ") + msg).c_str());
  if (int64_t(C.width) * C.height > 0 && (!rayo || !rayd))
    return ever::set_last_error(EVER_ERR_INVALID, "ever_camera_rays: null output");
  const cudaError_t e = ever::launch_camera_rays(C, jitter, rayo, rayd, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? EVER_OK : ever::set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
