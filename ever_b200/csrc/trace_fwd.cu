// Forward trace dispatch: k-buffer size -> the instantiations in trace_fwd_k{8,16,32}.cu
// (kernels in trace_fwd.cuh).
#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

// Exclusive scan of the popcounts of mask[0, ceil(n/32)) into offsets, total into *total.
// One block of 1024 threads; each thread takes 8 consecutive masks per step (two 16-byte
// loads; mask is 256-byte aligned), so a step covers 8192 warps.
__global__ void k_regroup_scan(const uint32_t* __restrict__ mask, const uint32_t* __restrict__ n_dev, int64_t n_max,
                               uint32_t* __restrict__ offsets, uint32_t* __restrict__ total) {
  constexpr int kPer = 8;
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t carry;
  const int64_t n = n_dev ? int64_t(*n_dev) : n_max;
  const int64_t nw = (n + 31) / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nw; base += int64_t(blockDim.x) * kPer) {
    const int64_t w0 = base + int64_t(tid) * kPer;
    uint32_t c[kPer];
    if (w0 + kPer <= nw) {
      const uint4 a = reinterpret_cast<const uint4*>(mask + w0)[0];
      const uint4 b = reinterpret_cast<const uint4*>(mask + w0)[1];
      c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
      c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
    } else {
#pragma unroll
      for (int q = 0; q < kPer; ++q) c[q] = w0 + q < nw ? mask[w0 + q] : 0u;
    }
    uint32_t v = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      c[q] = uint32_t(__popc(c[q]));
      v += c[q];
    }
    uint32_t x = v;  // inclusive scan of the threads' sums inside the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t t = lane < int(blockDim.x / 32) ? warp_sum[lane] : 0u;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, d);
        if (lane >= d) t += y;
      }
      warp_sum[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    uint32_t before = carry + (warp > 0 ? warp_sum[warp - 1] : 0u) + x - v;
    const uint32_t end = before + v;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      if (w0 + q < nw) offsets[w0 + q] = before;
      before += c[q];
    }
    __syncthreads();
    if (tid == blockDim.x - 1) carry = end;
    __syncthreads();
  }
  if (tid == 0) *total = carry;
}

__global__ void k_regroup_scatter(const uint32_t* __restrict__ mask, const uint32_t* __restrict__ offsets,
                                  const uint32_t* __restrict__ n_dev, int64_t n_max, const int32_t* __restrict__ src,
                                  int32_t* __restrict__ dst) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n = n_dev ? int64_t(*n_dev) : n_max;
  if (p >= n) return;
  const uint32_t m = mask[p >> 5];
  const int l = int(p & 31);
  if (!((m >> l) & 1u)) return;
  dst[offsets[p >> 5] + __popc(m & ((1u << l) - 1u))] = src ? src[p] : int32_t(p);
}

}  // namespace

int64_t regroup_workspace(int64_t R) {
  const int64_t nw = (R + 31) / 32;
  WsCursor c;
  c.take(nw * 4);
  c.take(nw * 4);
  c.take((nw + 1) * 4);
  c.take(R * 4);
  c.take(R * 4);
  c.take(4);
  c.take(4);
  return c.offset;
}

RegroupScratch regroup_scratch(char* ws, int64_t R) {
  const int64_t nw = (R + 31) / 32;
  WsCursor c;
  RegroupScratch W;
  W.mask0 = reinterpret_cast<uint32_t*>(ws + c.take(nw * 4));
  W.mask1 = reinterpret_cast<uint32_t*>(ws + c.take(nw * 4));
  W.offsets = reinterpret_cast<uint32_t*>(ws + c.take((nw + 1) * 4));
  W.list1 = reinterpret_cast<int32_t*>(ws + c.take(R * 4));
  W.list2 = reinterpret_cast<int32_t*>(ws + c.take(R * 4));
  W.count1 = reinterpret_cast<uint32_t*>(ws + c.take(4));
  W.count2 = reinterpret_cast<uint32_t*>(ws + c.take(4));
  W.split_min = 0;
  return W;
}

cudaError_t regroup_compact(const uint32_t* mask, const uint32_t* n_dev, int64_t n_max, const int32_t* src,
                            uint32_t* offsets, int32_t* dst, uint32_t* dst_count, cudaStream_t st) {
  k_regroup_scan<<<1, 1024, 0, st>>>(mask, n_dev, n_max, offsets, dst_count);
  k_regroup_scatter<<<unsigned((n_max + 255) / 256), 256, 0, st>>>(mask, offsets, n_dev, n_max, src, dst);
  return cudaGetLastError();
}

// traversal 0: warp packets with the frustum phase; 2: warp packets, rounds only
FwdParams with_mode(const FwdParams& P0, const EverTune& tune) {
  FwdParams P = P0;
  P.frustum = tune.traversal == 0 ? 1 : 0;
  P.stack_depth = tune.stack_depth > 0 ? std::min(tune.stack_depth, kStackDepth) : kStackDepth;
  return P;
}

cudaError_t launch_forward_regrouped(const FwdParams& P0, const RegroupScratch& W, const CameraParams* cam,
                                     const float* jitter, int deg, const EverTune& tune, cudaStream_t st) {
  const FwdParams P = with_mode(P0, tune);
  if (P.R == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  // splitting pays only while the next pass still fills the GPU several times over: four
  // times the resident lanes of the packet kernels (20 warps per SM)
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  RegroupScratch V = W;
  V.split_min = tune.regroup_min > 0 ? int64_t(tune.regroup_min) : int64_t(4) * sms * 20 * 32;
  const int64_t n = cam ? camera_slots(*cam) : P.R;
  if (n < V.split_min) {  // one pass would run every round: the single packet kernel does the same
    EverTune t = tune;
    if (t.traversal == 1) t.traversal = 0;
    return cam ? launch_forward_camera(P, *cam, jitter, deg, t, st) : launch_forward(P, deg, t, st);
  }
  switch (tune.kbuf) {
    case 8: return launch_forward_regrouped_k<8>(P, V, cam, jitter, deg, block, st);
    case 32: return launch_forward_regrouped_k<32>(P, V, cam, jitter, deg, block, st);
    default: return launch_forward_regrouped_k<16>(P, V, cam, jitter, deg, block, st);
  }
}

cudaError_t launch_forward_batched(const BatchFwdParams& P0, int deg, const EverTune& tune, cudaStream_t st) {
  BatchFwdParams P = P0;
  P.frustum = tune.traversal == 2 ? 0 : 1;
  P.stack_depth = tune.stack_depth > 0 ? std::min(tune.stack_depth, kStackDepth) : kStackDepth;
  if (P.num_slots == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_batched_k<8>(P, deg, block, st);
    case 32: return launch_forward_batched_k<32>(P, deg, block, st);
    default: return launch_forward_batched_k<16>(P, deg, block, st);
  }
}

cudaError_t launch_forward(const FwdParams& P0, int deg, const EverTune& tune, cudaStream_t st) {
  const FwdParams P = with_mode(P0, tune);
  if (P.R == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_k<8>(P, deg, block, tune.traversal, st);
    case 32: return launch_forward_k<32>(P, deg, block, tune.traversal, st);
    default: return launch_forward_k<16>(P, deg, block, tune.traversal, st);
  }
}

cudaError_t launch_forward_camera(const FwdParams& P0, const CameraParams& cam, const float* jitter, int deg,
                                  const EverTune& tune, cudaStream_t st) {
  const FwdParams P = with_mode(P0, tune);
  if (int64_t(cam.width) * cam.height == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (tune.kbuf) {
    case 8: return launch_forward_camera_k<8>(P, cam, jitter, deg, block, st);
    case 32: return launch_forward_camera_k<32>(P, cam, jitter, deg, block, st);
    default: return launch_forward_camera_k<16>(P, cam, jitter, deg, block, st);
  }
}

}  // namespace ever
