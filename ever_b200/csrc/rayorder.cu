// Coherent ray order for the packet traversal: rays are sorted by a 30-bit key made of
// a coarse origin cell (6 bits) above the Hilbert index of the octahedral projection of
// the direction (12 bits per axis); a predicted cost bin, when given, goes on top. Thirty-
// two consecutive rays of the result then cover a compact patch of directions (close to a
// screen tile for a pinhole camera: the Hilbert curve has none of the Z-order's jumps, so
// a run of 32 rays rarely splits across distant patches), and a warp's packet walks far
// fewer nodes than a scanline strip would. The order only decides which thread picks up
// which ray; results do not depend on it.
#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

// Index of cell (x, y) of a 4096 x 4096 grid along the Hilbert curve (24 bits): quadrant by
// quadrant from the top bit down, rotating / reflecting the lower bits into the
// quadrant's own frame.
__device__ __forceinline__ uint32_t hilbert12(uint32_t x, uint32_t y) {
  uint32_t d = 0;
#pragma unroll
  for (uint32_t s = 1u << 11; s > 0; s >>= 1) {
    const uint32_t rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
    d += s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx) {
        x ^= s - 1;
        y ^= s - 1;
      }
      const uint32_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

// 24-bit direction key: Hilbert index of the octahedral projection of d.
__device__ __forceinline__ uint32_t direction_key(float dx, float dy, float dz) {
  const float l1 = fabsf(dx) + fabsf(dy) + fabsf(dz);
  float u = 0.f, v = 0.f;
  if (l1 > 0.f && isfinite(l1)) {
    u = dx / l1;
    v = dy / l1;
    if (dz < 0.f) {
      const float uu = (1.f - fabsf(v)) * (u >= 0.f ? 1.f : -1.f);
      const float vv = (1.f - fabsf(u)) * (v >= 0.f ? 1.f : -1.f);
      u = uu;
      v = vv;
    }
  }
  const uint32_t qu = min(uint32_t(fmaxf(u * 0.5f + 0.5f, 0.f) * 4096.f), 4095u);
  const uint32_t qv = min(uint32_t(fmaxf(v * 0.5f + 0.5f, 0.f) * 4096.f), 4095u);
  return hilbert12(qu, qv);
}

// Rank of a cost bin in the sort: costlier bins (larger values) sort first.
__device__ __forceinline__ uint32_t bin_rank(const uint8_t* __restrict__ bins, int64_t r) {
  return 3u - min(uint32_t(bins[r]), 3u);
}

__global__ void k_ray_keys(const float* __restrict__ rayo, const float* __restrict__ rayd, int64_t R,
                           const uint8_t* __restrict__ bins, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const uint32_t dir = direction_key(rayd[3 * r], rayd[3 * r + 1], rayd[3 * r + 2]);
  uint32_t cell = 0;
  for (int a = 0; a < 3; ++a) {
    const float o = rayo[3 * r + a];
    const uint32_t q = o == o ? uint32_t(fminf(fmaxf((o + 4.f) * 0.5f, 0.f), 3.f)) : 0u;  // 4 cells on [-4, 4]
    cell = (cell << 2) | q;
  }
  const uint32_t key = (cell << 24) | dir;
  keys[r] = bins ? (bin_rank(bins, r) << 30) | key : key;
  vals[r] = uint32_t(r);
}

__device__ __forceinline__ int view_of(const BatchView* __restrict__ views, int num_views, int64_t r) {
  int v = 0;
  while (v + 1 < num_views && views[v + 1].ray_offset <= r) ++v;
  return v;
}

// Batched keys: the view index above the direction key, so one sort orders every view at
// once and keeps the views apart. With cost bins the bin's rank sits between the view
// (6 bits) and the direction key.
__global__ void k_batch_ray_keys(const float* __restrict__ rayd, int64_t R, const BatchView* __restrict__ views,
                                 int num_views, const uint8_t* __restrict__ bins, uint32_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const uint32_t view = uint32_t(view_of(views, num_views, r));
  const uint32_t dir = direction_key(rayd[3 * r], rayd[3 * r + 1], rayd[3 * r + 2]);
  keys[r] = bins ? (view << 26) | (bin_rank(bins, r) << 24) | dir : (view << 24) | dir;
  vals[r] = uint32_t(r);
}

// Sorted position p of view v lands in slot slot_offset_v + (p - ray_offset_v).
__global__ void k_batch_fill_slots(const uint32_t* __restrict__ sorted, int64_t R, const BatchView* __restrict__ views,
                                   int num_views, int32_t* __restrict__ slot_ray) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= R) return;
  const int v = view_of(views, num_views, p);  // views tile the rays in order, so p and its ray share a view
  slot_ray[views[v].slot_offset + (p - views[v].ray_offset)] = int32_t(sorted[p]);
}

// Key of forward slot s: its ray's consumed events (coarsened by `shift`), costliest first;
// with views (batched slots), the slot's view above that, so each view's slots stay
// together (a warp's lanes then replay rays of one view and one scene).
__global__ void k_bwd_keys(const int32_t* __restrict__ iters, const int32_t* __restrict__ ray_order, int64_t R,
                           int shift, const BatchView* __restrict__ views, int num_views, uint32_t* __restrict__ keys,
                           uint32_t* __restrict__ vals) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= R) return;
  const int64_t r = ray_order ? int64_t(ray_order[s]) : s;
  const uint32_t n = r >= 0 ? uint32_t(max(iters[r], 0)) >> shift : 0u;  // padding slot: last
  uint32_t key = 255u - min(n, 255u);
  if (views) {
    int lo = 0, hi = num_views - 1;  // last view with slot_offset <= s
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (views[mid].slot_offset <= s) lo = mid;
      else hi = mid - 1;
    }
    key |= uint32_t(lo) << 8;
  }
  keys[s] = key;
  vals[s] = uint32_t(s);
}

// Backward keys of a camera trace: slot -> pixel from the camera's tile order.
__global__ void k_camera_bwd_keys(const CameraParams cam, const int32_t* __restrict__ iters, int64_t num_slots,
                                  int shift, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= num_slots) return;
  const int64_t r = camera_slot_pixel(cam, s);
  const uint32_t n = r >= 0 ? uint32_t(max(iters[r], 0)) >> shift : 0u;  // padding slot: last
  keys[s] = 255u - min(n, 255u);
  vals[s] = uint32_t(s);
}

}  // namespace

cudaError_t camera_backward_slot_order(const CameraParams& cam, const int32_t* iters, int shift, char* ws,
                                       int32_t* slot_order, cudaStream_t st) {
  const int64_t S = camera_slots(cam);
  if (S == 0) return cudaSuccess;
  WsCursor c;
  uint32_t* ka = reinterpret_cast<uint32_t*>(ws + c.take(S * 4));
  uint32_t* va = reinterpret_cast<uint32_t*>(ws + c.take(S * 4));
  uint32_t* kb = reinterpret_cast<uint32_t*>(ws + c.take(S * 4));
  uint32_t* vb = reinterpret_cast<uint32_t*>(ws + c.take(S * 4));
  uint32_t* hist = reinterpret_cast<uint32_t*>(ws + c.take((int64_t(sort_blocks(S)) * 256 + 512) * 4));
  k_camera_bwd_keys<<<unsigned((S + 255) / 256), 256, 0, st>>>(cam, iters, S, shift, ka, va);
  sort_pairs(ka, va, kb, vb, hist, S, 8, st);
  return cudaMemcpyAsync(slot_order, va, S * sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
}

cudaError_t backward_slot_order(const int32_t* iters, const int32_t* ray_order, int64_t R, int shift, char* ws,
                                int32_t* slot_order, cudaStream_t st, const BatchView* views, int num_views) {
  if (R == 0) return cudaSuccess;
  WsCursor c;
  uint32_t* ka = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* va = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* kb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* vb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* hist = reinterpret_cast<uint32_t*>(ws + c.take((int64_t(sort_blocks(R)) * 256 + 512) * 4));
  k_bwd_keys<<<unsigned((R + 255) / 256), 256, 0, st>>>(iters, ray_order, R, shift, views, num_views, ka, va);
  sort_pairs(ka, va, kb, vb, hist, R, views ? 14 : 8, st);
  return cudaMemcpyAsync(slot_order, va, R * sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
}

cudaError_t batch_ray_order(const float* rayo, const float* rayd, int64_t R, const BatchView* views, int num_views,
                            char* ws, int32_t* slot_ray, int64_t num_slots, cudaStream_t st, const uint8_t* bins) {
  (void)rayo;
  cudaError_t e = cudaMemsetAsync(slot_ray, 0xff, num_slots * sizeof(int32_t), st);
  if (e != cudaSuccess || R == 0) return e;
  WsCursor c;
  uint32_t* ka = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* va = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* kb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* vb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* hist = reinterpret_cast<uint32_t*>(ws + c.take((int64_t(sort_blocks(R)) * 256 + 512) * 4));
  k_batch_ray_keys<<<unsigned((R + 255) / 256), 256, 0, st>>>(rayd, R, views, num_views, bins, ka, va);
  sort_pairs(ka, va, kb, vb, hist, R, bins ? 32 : 30, st);
  k_batch_fill_slots<<<unsigned((R + 255) / 256), 256, 0, st>>>(va, R, views, num_views, slot_ray);
  return cudaGetLastError();
}

int64_t ray_order_workspace(int64_t R) {
  WsCursor c;
  c.take(R * 4);
  c.take(R * 4);
  c.take(R * 4);
  c.take(R * 4);
  c.take((int64_t(sort_blocks(R)) * 256 + 512) * 4);
  return c.offset;
}

cudaError_t ray_order(const float* rayo, const float* rayd, int64_t R, char* ws, int32_t* order, cudaStream_t st,
                      const uint8_t* bins) {
  if (R == 0) return cudaSuccess;
  WsCursor c;
  uint32_t* ka = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* va = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* kb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* vb = reinterpret_cast<uint32_t*>(ws + c.take(R * 4));
  uint32_t* hist = reinterpret_cast<uint32_t*>(ws + c.take((int64_t(sort_blocks(R)) * 256 + 512) * 4));
  k_ray_keys<<<unsigned((R + 255) / 256), 256, 0, st>>>(rayo, rayd, R, bins, ka, va);
  sort_pairs(ka, va, kb, vb, hist, R, bins ? 32 : 30, st);
  return cudaMemcpyAsync(order, va, R * sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
}

}  // namespace ever
