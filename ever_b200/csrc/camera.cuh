// Camera rays computed where they are used: the same arithmetic for ever_camera_rays and
// for the fused camera traces (trace_fwd.cuh, trace_bwd.cu), so both see identical rays.
//
// Pixel p (row-major) -> d = normalize(((col + ox) - cx) / fx, ((row + oy) - cy) / fy, 1),
// rayd = R d, rayo = camera centre (integration_utils/gaussian_renderer/ever.py:29-74).
// The camera traces launch in an analytic tile order: slot s belongs to the 8x4 pixel tile
// s / 32, and lane s % 32 to pixel (col, row) = (8 tx + s % 8, 4 ty + (s % 32) / 8) of it.
// Tiles come in supertiles of 8 x 16 tiles (64 x 64 pixels), supertiles row-major, the 128
// tiles of a supertile in Morton order, so that warps running at the same time cover a
// compact patch of the image. Slots outside the image are padding (pixel -1). One warp
// traces one tile.
#pragma once
#include "internal.cuh"

namespace ever {

// supertiles across the image: 64 pixels wide (8 tiles), 64 pixels high (16 tiles)
__host__ __device__ __forceinline__ int64_t camera_supertiles_x(const CameraParams& C) { return (C.width + 63) / 64; }
__host__ __device__ __forceinline__ int64_t camera_slots(const CameraParams& C) {
  return camera_supertiles_x(C) * ((C.height + 63) / 64) * 128 * 32;
}

__device__ __forceinline__ int64_t camera_slot_pixel(const CameraParams& C, int64_t s) {
  const int64_t st = s >> 12;          // supertile
  const int w = int(s >> 5) & 127;     // tile inside it: Morton bits x0 y0 x1 y1 x2 y2 y3
  const int l = int(s & 31);
  const int wx = (w & 1) | ((w >> 1) & 2) | ((w >> 2) & 4);
  const int wy = ((w >> 1) & 1) | ((w >> 2) & 2) | ((w >> 3) & 4) | ((w >> 3) & 8);
  const int64_t sx = st % camera_supertiles_x(C), sy = st / camera_supertiles_x(C);
  const int64_t col = sx * 64 + wx * 8 + (l & 7), row = sy * 64 + wy * 4 + (l >> 3);
  return (col < C.width && row < C.height) ? row * C.width + col : -1;
}

__device__ __forceinline__ void camera_ray(const CameraParams& C, const float* __restrict__ jitter, int64_t p,
                                           float3& ro, float3& rd) {
  const int row = int(p / C.width), col = int(p - int64_t(row) * C.width);
  const float ox = jitter ? jitter[2 * p] : 0.5f, oy = jitter ? jitter[2 * p + 1] : 0.5f;
  const float x = ((float(col) + ox) - C.cx) / C.fx;
  const float y = ((float(row) + oy) - C.cy) / C.fy;
  const float n = sqrtf(x * x + y * y + 1.f);
  const float d[3] = {x / n, y / n, 1.f / n};
  float v[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) v[a] = C.c2w[4 * a] * d[0] + C.c2w[4 * a + 1] * d[1] + C.c2w[4 * a + 2] * d[2];
  rd = make_float3(v[0], v[1], v[2]);
  ro = make_float3(C.c2w[3], C.c2w[7], C.c2w[11]);
}

// Checks a camera of the C API and converts it; returns an error message, or nullptr.
inline const char* camera_params(const EverCamera* c, CameraParams* out) {
  if (!c) return "null camera";
  if (c->width < 0 || c->height < 0 || int64_t(c->width) * c->height >= (int64_t(1) << 31))
    return "image size out of range";
  if (!(c->fx != 0.f) || !(c->fy != 0.f)) return "zero focal length";
  out->width = c->width;
  out->height = c->height;
  out->fx = c->fx;
  out->fy = c->fy;
  out->cx = c->cx;
  out->cy = c->cy;
  for (int i = 0; i < 12; ++i) out->c2w[i] = c->c2w[i];
  if (camera_slots(*out) >= (int64_t(1) << 31)) return "image size out of range";
  return nullptr;
}

}  // namespace ever
