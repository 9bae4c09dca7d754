// ever_ray_order_static: the coherent ray order of ever_ray_order() without any device
// allocation, for callers that cannot allocate. Examples are a frame loop in a viewer
// or render server that must never block on the allocator (cudaFree waits for the
// whole device), and a binding from another language runtime that has no way to hand
// this library a workspace. The scratch lives in one file-scope __device__ array instead.
//
// Limit: at most kStaticOrderMaxRays rays per call (one 1920x1080 view fits). The array
// (about 33 MB) is part of the library image, so every GPU that loads the library holds
// it until the process exits.
//
// Sharing: every call on a device uses the same array and finds the previous call's
// contents in it. Nothing needs clearing: each scratch word the sort reads was written
// earlier in the same call (keys and values by the key kernel, every histogram bucket
// by every histogram block, the scan partials by the scan). Two calls that overlap on
// the GPU (different streams, or work queued from different host threads) race on the
// array, so a caller must order them, e.g. by using one stream.
//
// Set-up: the device address of the array is looked up through cudaGetSymbolAddress on
// every call whose stream is not capturing, and kept per device for the calls made during
// a stream capture (where that lookup could load the module and break the capture). So
// make one call on each device before capturing one; after cudaDeviceReset the next
// uncaptured call looks the address up again.
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr int64_t kStaticOrderMaxRays = int64_t(1) << 21;  // 2,097,152 rays
constexpr int64_t round256(int64_t b) { return (b + 255) / 256 * 256; }
// Same segment layout as ray_order_workspace(): keys, values, keys, values, histogram + scan partials.
constexpr int64_t kStaticOrderBytes =
    4 * round256(kStaticOrderMaxRays * 4) + round256(((kStaticOrderMaxRays + 2047) / 2048 * 256 + 512) * 4);

static __device__ __align__(256) unsigned char g_order_scratch[kStaticOrderBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

}  // namespace
}  // namespace ever

extern "C" int ever_ray_order_static(const float* rayo, const float* rayd, int64_t num_rays, int32_t* ray_order,
                                     void* stream) {
  using namespace ever;
  if (num_rays < 0 || num_rays > kStaticOrderMaxRays)
    return set_last_error(EVER_ERR_INVALID,
                     "ever_ray_order_static: num_rays out of range [0, 2097152]; use ever_ray_order with a workspace");
  if (ever::ray_order_workspace(num_rays) > kStaticOrderBytes)
    return set_last_error(EVER_ERR_INVALID, "ever_ray_order_static: scratch layout larger than the static array");
  if (num_rays > 0 && (!rayo || !rayd || !ray_order)) return set_last_error(EVER_ERR_INVALID, "ever_ray_order_static: null pointer");
  if (num_rays == 0) return EVER_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_last_error(EVER_ERR_INVALID, "ever_ray_order_static: device index too large");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap);
  if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_order_scratch);
      if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
      g_scratch_ptr[dev] = p;
    } else if (!g_scratch_ptr[dev]) {
      return set_last_error(EVER_ERR_INVALID,
                            "ever_ray_order_static: first call on this device made during a stream capture");
    }
    scratch = g_scratch_ptr[dev];
  }
  e = ever::ray_order(rayo, rayd, num_rays, static_cast<char*>(scratch), ray_order, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return set_last_error(EVER_ERR_CUDA, cudaGetErrorString(e));
  return EVER_OK;
}
