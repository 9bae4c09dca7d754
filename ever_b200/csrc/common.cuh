// Shared device-side definitions of the exact ellipsoid tracer.
//
// The arithmetic below is the float32 specification of the trace: the whole library
// is compiled with --fmad=false, so only the explicit fmaf() calls fuse, and division
// and sqrt are IEEE round-to-nearest. Event times, event order, iteration counts and
// the density sums that drive termination are therefore reproducible bit for bit on
// any IEEE host that follows the same operation order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ever_b200.h"

namespace ever {

constexpr float kTiny = 1.0754944e-20f;  // TINY_VAL, splinetracers/slang/safe-math.slang:16
constexpr float kMaxVal = 1e20f;         // MAX_VAL, safe-math.slang:18
constexpr float kMinVal = -1e20f;        // MIN_VAL, safe-math.slang:17
constexpr float kLogMax = 46.05170185988091f;  // log(MAX_VAL): safe_exp clamp, safe-math.slang:142-144
constexpr float kLogCutoff = 5.54f;      // LOG_CUTOFF, fast_ellipsoid_splinetracer/slang/shaders.slang:17
constexpr int kRefRound = 16;            // BUFFER_SIZE, shaders.slang:18: the reference's k-buffer
constexpr float kSentinel = 1e9f;        // shaders.slang:214: a slot t > 1e9 ends the ray
constexpr int kStackDepth = 64;          // traversal stack (LBVH depth <= 30 code bits + log2 N)

// SH constants, splinetracers/slang/sh.slang:18-27
constexpr float kShC0 = 0.28209479177387814f;
constexpr float kShC1 = 0.4886025119029199f;
__device__ __constant__ static const float kShC2[5] = {1.0925484305920792f, -1.0925484305920792f,
                                                         0.31539156525252005f, -1.0925484305920792f,
                                                         0.5462742152960396f};
__device__ __constant__ static const float kShC3[7] = {-0.5900435899266435f, 2.890611442640554f,
                                                         -0.4570457994644658f, 0.3731763325901154f,
                                                         -0.4570457994644658f, 1.445305721320277f,
                                                         -0.5900435899266435f};

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fmaxf(fminf(v, hi), lo); }

// safe_div, safe-math.slang:84-91
__device__ __forceinline__ float safe_div(float a, float b) {
  if (fabsf(b) < kTiny) return clampf(a / kTiny, kMinVal, kMaxVal);
  return clampf(a / b, kMinVal, kMaxVal);
}
// safe_exp, safe-math.slang:141-144
__device__ __forceinline__ float safe_exp(float v) { return expf(clampf(v, kMinVal, kLogMax)); }
__device__ __forceinline__ float sgnf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// tukey_power_ladder(x, -0.1), safe-math.slang:246-253
__device__ __forceinline__ float tukey(float x) {
  const float p = -0.1f;
  const float pm1 = fabsf(p - 1.f);
  const float xs = fabsf(x) / fmaxf(kTiny, pm1);
  return ((sgnf(x) * pm1) / p) * (powf(xs + 1.f, p) - 1.f);
}
__device__ __forceinline__ float dtukey(float x) {
  const float p = -0.1f;
  const float pm1 = fabsf(p - 1.f);
  const float xs = fabsf(x) / fmaxf(kTiny, pm1);
  return sgnf(x) * sgnf(x) * powf(xs + 1.f, p - 1.f);
}

// rotate_vector(v, q): rotation by the conjugate of q = (r,x,y,z), safe-math.slang:236-244.
__device__ __forceinline__ float3 rotate_vector(float3 v, float4 q) {
  const float w = q.x, ux = -q.y, uy = -q.z, uz = -q.w;
  const float tx = 2.f * (uy * v.z - uz * v.y);
  const float ty = 2.f * (uz * v.x - ux * v.z);
  const float tz = 2.f * (ux * v.y - uy * v.x);
  return make_float3((v.x + w * tx) + (uy * tz - uz * ty), (v.y + w * ty) + (uz * tx - ux * tz),
                     (v.z + w * tz) + (ux * ty - uy * tx));
}

// Intersection record of one ellipsoid, 64 B: rows of W = diag(1/s) A(q) with the mean
// in .w, then (density, DC colour). W (x - mean) are the unit-sphere coordinates of x,
// i.e. rotate_vector(x - mean, q) / s (tri-intersect.slang:164-175). The DC colour is
// C0 * f0 + 0.5 per channel (eval_sh_col0, sh.slang:49-51): the colour the reference's
// forward gives every event (shaders.slang:72-75), so degree-0 traces read no feature row.
// The original index of position j is the scene's order[j].
struct __align__(16) Record {
  float4 r0, r1, r2, r3;
};

// The DC colour held in a record's r3 (the same bits as sh_colour<0> of the feature row).
__device__ __forceinline__ float3 dc_colour(float4 r3) { return make_float3(r3.y, r3.z, r3.w); }
__device__ __forceinline__ float dc_channel(float f0) { return fmaf(kShC0, f0, 0.5f); }

struct __align__(16) Node {
  float4 a;  // child0 lo.xyz, hi.x
  float4 b;  // child0 hi.yz, child1 lo.xy
  float4 c;  // child1 lo.z, hi.xyz
  int4 d;    // child0, child1 (>= 0 internal node, < 0 leaf ~position), pad
};

struct Ray {
  float3 o;   // rayo + tmin * rayd (shaders.slang:179, raw direction)
  float3 d;   // l2_normalize(rayd) (shaders.slang:178)
  float3 rd;  // raw rayd (SH direction)
};

__device__ __forceinline__ Ray make_ray(float3 ro, float3 rd, float tmin) {
  Ray r;
  r.rd = rd;
  r.o = make_float3(fmaf(tmin, rd.x, ro.x), fmaf(tmin, rd.y, ro.y), fmaf(tmin, rd.z, ro.z));
  const float dd = fmaf(rd.z, rd.z, fmaf(rd.y, rd.y, rd.x * rd.x));
  const float nrm = sqrtf(fmaxf(dd, kTiny));
  r.d = make_float3(safe_div(rd.x, nrm), safe_div(rd.y, nrm), safe_div(rd.z, nrm));
  return r;
}

struct HitT {
  float t0, t1;
};

// Ray/ellipsoid roots (eliIntersect, tri-intersect.slang:115-131) in local coordinates.
// Returns false on a miss (h < 0 or NaN).
__device__ __forceinline__ bool intersect(const Record& R, const Ray& ray, HitT& H) {
  const float v0 = ray.o.x - R.r0.w, v1 = ray.o.y - R.r1.w, v2 = ray.o.z - R.r2.w;
  const float oc0 = fmaf(R.r0.z, v2, fmaf(R.r0.y, v1, R.r0.x * v0));
  const float oc1 = fmaf(R.r1.z, v2, fmaf(R.r1.y, v1, R.r1.x * v0));
  const float oc2 = fmaf(R.r2.z, v2, fmaf(R.r2.y, v1, R.r2.x * v0));
  const float rn0 = fmaf(R.r0.z, ray.d.z, fmaf(R.r0.y, ray.d.y, R.r0.x * ray.d.x));
  const float rn1 = fmaf(R.r1.z, ray.d.z, fmaf(R.r1.y, ray.d.y, R.r1.x * ray.d.x));
  const float rn2 = fmaf(R.r2.z, ray.d.z, fmaf(R.r2.y, ray.d.y, R.r2.x * ray.d.x));
  const float a = fmaf(rn2, rn2, fmaf(rn1, rn1, rn0 * rn0));
  const float bp = -fmaf(oc2, rn2, fmaf(oc1, rn1, oc0 * rn0));
  const float ba = bp / a;
  const float l0 = fmaf(ba, rn0, oc0), l1 = fmaf(ba, rn1, oc1), l2 = fmaf(ba, rn2, oc2);
  const float ll = fmaf(l2, l2, fmaf(l1, l1, l0 * l0));
  const float h = a * (1.f - ll);
  const float c = fmaf(oc2, oc2, fmaf(oc1, oc1, oc0 * oc0)) - 1.f;
  if (!(h >= 0.f)) return false;
  const float sq = sqrtf(h);
  const float qq = bp > 0.f ? bp + sq : (bp < 0.f ? bp - sq : bp);
  const float ra = c / qq, rb = qq / a;
  H.t0 = fminf(ra, rb);
  H.t1 = fmaxf(ra, rb);
  return true;
}

// SH basis at the raw ray direction, sh.slang:48-88 (same operation order as the oracle).
template <int DEG>
__device__ __forceinline__ void sh_basis(float3 dir, float* B) {
  const float x = dir.x, y = dir.y, z = dir.z;
  B[0] = kShC0;
  if (DEG < 1) return;
  B[1] = (-kShC1) * y;
  B[2] = kShC1 * z;
  B[3] = (-kShC1) * x;
  if (DEG < 2) return;
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  B[4] = kShC2[0] * xy;
  B[5] = kShC2[1] * yz;
  B[6] = kShC2[2] * ((2.f * zz - xx) - yy);
  B[7] = kShC2[3] * xz;
  B[8] = kShC2[4] * (xx - yy);
  if (DEG < 3) return;
  B[9] = (kShC3[0] * y) * (3.f * xx - yy);
  B[10] = (kShC3[1] * xy) * z;
  B[11] = (kShC3[2] * y) * ((4.f * zz - xx) - yy);
  B[12] = (kShC3[3] * z) * ((2.f * zz - 3.f * xx) - 3.f * yy);
  B[13] = (kShC3[4] * x) * ((4.f * zz - xx) - yy);
  B[14] = (kShC3[5] * z) * (xx - yy);
  B[15] = (kShC3[6] * x) * (xx - 3.f * yy);
}

// Floats per ellipsoid in the device feature rows: 3K rounded up to a multiple of 4 so
// that every row starts on a 16-byte boundary (float4 loads and float4 atomics).
__host__ __device__ __forceinline__ int feat_stride(int K) { return (3 * K + 3) / 4 * 4; }

// Colour of an ellipsoid along the ray: sum_k B_k f_k + 0.5 (eval_color, sh.slang:90-103).
// f: the ellipsoid's 16-byte aligned feature row.
template <int DEG>
__device__ __forceinline__ float3 sh_colour(const float* __restrict__ f, const float* B, int bs = 1) {
  constexpr int NB = (DEG + 1) * (DEG + 1);
  constexpr int NV = (3 * NB + 3) / 4;
  float v[4 * NV];
  const float4* f4 = reinterpret_cast<const float4*>(f);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const float4 x = __ldg(f4 + i);
    v[4 * i] = x.x;
    v[4 * i + 1] = x.y;
    v[4 * i + 2] = x.z;
    v[4 * i + 3] = x.w;
  }
  const float b0 = B[0];
  float3 c = make_float3(fmaf(b0, v[0], 0.5f), fmaf(b0, v[1], 0.5f), fmaf(b0, v[2], 0.5f));
#pragma unroll
  for (int k = 1; k < NB; ++k) {
    const float bk = B[k * bs];
    c.x = fmaf(bk, v[3 * k + 0], c.x);
    c.y = fmaf(bk, v[3 * k + 1], c.y);
    c.z = fmaf(bk, v[3 * k + 2], c.z);
  }
  return c;
}

// SplineState, spline-machine.slang:20-32 (padding dropped in registers).
struct State {
  float dist_x, dist_y, cum_x, cum_y;
  float t;
  float4 drgb;
  float logT;
  float3 C;
};

__device__ __forceinline__ State empty_state() {
  State s;
  s.dist_x = s.dist_y = s.cum_x = s.cum_y = 0.f;
  s.t = 0.f;
  s.drgb = make_float4(0.f, 0.f, 0.f, 0.f);
  s.logT = 0.f;
  s.C = make_float3(0.f, 0.f, 0.f);
  return s;
}

// update(), spline-machine.slang:103-138.
__device__ __forceinline__ void update(State& s, float t, float4 dirac) {
  const float dt = fmaxf(t - s.t, 0.f);
  const float area = fmaxf(s.drgb.x * dt, 0.f);
  const float rgb0 = safe_div(s.drgb.y, s.drgb.x);
  const float rgb1 = safe_div(s.drgb.z, s.drgb.x);
  const float rgb2 = safe_div(s.drgb.w, s.drgb.x);
  const float logT = fmaxf(area + s.logT, 0.f);
  const float w = clampf((1.f - safe_exp(-area)) * safe_exp(-s.logT), 0.f, 1.f);
  s.C.x = fmaf(w, rgb0, s.C.x);
  s.C.y = fmaf(w, rgb1, s.C.y);
  s.C.z = fmaf(w, rgb2, s.C.z);
  const float m = tukey(((t + s.t) * 0.5f) * 1000.f);
  const float w2 = 2.f * w;
  s.dist_x = fmaf(w2 * m, s.cum_x, s.dist_x);
  s.dist_y = fmaf(w2, s.cum_y, s.dist_y);
  s.cum_x = s.cum_x + w;
  s.cum_y = fmaf(w, m, s.cum_y);
  s.drgb.x = s.drgb.x + dirac.x;
  s.drgb.y = s.drgb.y + dirac.y;
  s.drgb.z = s.drgb.z + dirac.z;
  s.drgb.w = s.drgb.w + dirac.w;
  s.logT = logT;
  s.t = t;
}

__device__ __forceinline__ Record load_record(const Record* __restrict__ recs, int j) {
  const float4* p = reinterpret_cast<const float4*>(recs + j);
  Record R;
  R.r0 = __ldg(p + 0);
  R.r1 = __ldg(p + 1);
  R.r2 = __ldg(p + 2);
  R.r3 = __ldg(p + 3);
  return R;
}

// Ordered event key: (t bits << 32) | (2 * position + exit). t > 0, so the float
// bits order like the floats; ties fall back to Morton position, entry before exit.
__device__ __forceinline__ uint64_t event_key(float t, int j, int exitbit) {
  return (uint64_t(__float_as_uint(t)) << 32) | uint32_t(2 * j + exitbit);
}
__device__ __forceinline__ float key_t(uint64_t k) { return __uint_as_float(uint32_t(k >> 32)); }
__device__ __forceinline__ int key_pos(uint64_t k) { return int(uint32_t(k) >> 1); }
__device__ __forceinline__ int key_exit(uint64_t k) { return int(uint32_t(k) & 1u); }
constexpr uint64_t kEmptyKey = ~uint64_t(0);

}  // namespace ever
