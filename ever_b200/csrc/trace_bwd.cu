// Backward trace: one thread per ray replays the ray's events in reverse.
//
// Reference: backwards_kernel (splinetracers/fast_ellipsoid_splinetracer/slang/
// backwards_kernel.slang:259-367), its run_update (:132-222) and the initial-density
// kernel (:374-428). Each step undoes one update() algebraically (inverse_update_dual,
// spline-machine.slang:65-100), recomputes the event's intersection and colour exactly
// as the forward computed them, and applies hand-derived VJPs of update(), of the root
// of |ocn + t rdn|^2 = 1 and of the SH colour. Gradients of the 3x3 local-frame matrix W
// are accumulated per ellipsoid and turned into scale/quaternion gradients once per
// ellipsoid by k_finalize.
#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr int kGeo = 16;  // per-ellipsoid accumulator: W (9), mean (3), density (1), pad (3)
// Resident 256-thread blocks per SM: 24 warps at degree 0 (80 registers; 2.06 ms against
// 2.25 ms with 16 warps at 1M / 1080p), 16 warps with SH colour, which needs more registers.
template <int DEG>
constexpr int kBwdMinBlocks = DEG == 0 ? 3 : 2;

struct Ctrl {
  float t;
  float4 dirac;
  float3 c;
  int j, entry;
};

struct FullHit {
  float t0, t1;
  float ocn[3], rdn[3];
};

__device__ __forceinline__ bool intersect_full(const Record& R, const Ray& ray, FullHit& H) {
  const float v0 = ray.o.x - R.r0.w, v1 = ray.o.y - R.r1.w, v2 = ray.o.z - R.r2.w;
  const float4 rows[3] = {R.r0, R.r1, R.r2};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    H.ocn[i] = fmaf(rows[i].z, v2, fmaf(rows[i].y, v1, rows[i].x * v0));
    H.rdn[i] = fmaf(rows[i].z, ray.d.z, fmaf(rows[i].y, ray.d.y, rows[i].x * ray.d.x));
  }
  HitT h;
  const bool hit = intersect(R, ray, h);
  H.t0 = h.t0;
  H.t1 = h.t1;
  return hit;
}

template <int DEG>
__device__ __forceinline__ Ctrl load_ctrl(const Record* recs, const float* feats, int64_t fstride, const Ray& ray,
                                          const float* B, int id) {
  Ctrl c;
  c.j = id >> 1;
  c.entry = id & 1;
  const Record R = load_record(recs, c.j);
  HitT H;
  intersect(R, ray, H);
  c.t = c.entry ? H.t0 : H.t1;
  c.c = DEG == 0 ? dc_colour(R.r3) : sh_colour<DEG>(feats + c.j * fstride, B);
  const float dh = c.entry ? R.r3.x : -R.r3.x;
  c.dirac = make_float4(dh, dh * c.c.x, dh * c.c.y, dh * c.c.z);
  return c;
}

// inverse_update_dual, spline-machine.slang:65-100.
__device__ __forceinline__ State inverse_update(const State& n, float4 dirac_new, float t_old) {
  State s;
  const float dt = fmaxf(n.t - t_old, 0.f);
  s.drgb = make_float4(n.drgb.x - dirac_new.x, n.drgb.y - dirac_new.y, n.drgb.z - dirac_new.z,
                       n.drgb.w - dirac_new.w);
  s.t = t_old;
  const float area = fmaxf(s.drgb.x * dt, 0.f);
  const float rgb0 = safe_div(s.drgb.y, s.drgb.x), rgb1 = safe_div(s.drgb.z, s.drgb.x),
              rgb2 = safe_div(s.drgb.w, s.drgb.x);
  s.logT = fmaxf(n.logT - area, 0.f);
  const float w = clampf((1.f - safe_exp(-area)) * safe_exp(-s.logT), 0.f, 1.f);
  s.C = make_float3(n.C.x - w * rgb0, n.C.y - w * rgb1, n.C.z - w * rgb2);
  const float m = tukey(((n.t + s.t) * 0.5f) * 1000.f);
  s.cum_x = n.cum_x - w;
  s.cum_y = n.cum_y - w * m;
  s.dist_x = n.dist_x - 2.f * w * m * s.cum_x;
  s.dist_y = n.dist_y - 2.f * w * s.cum_y;
  return s;
}

// safe_div backward, safe-math.slang:68-80.
__device__ __forceinline__ void safe_div_bwd(float a, float b, float R, float& da, float& db) {
  da = fabsf(b) < kTiny ? clampf(R / kTiny, kMinVal, kMaxVal) : clampf(R / b, kMinVal, kMaxVal);
  const float b2 = b * b;
  db = b2 < kTiny ? clampf(-a / kTiny * R, kMinVal, kMaxVal) : clampf(-a / b2 * R, kMinVal, kMaxVal);
}

// VJP of update(s, t, dirac) given the cotangent G of the new state. Clamps pass the
// gradient only strictly inside their range (a zero-density gap gets none).
__device__ __forceinline__ void update_vjp(const State& s, float t, const State& G, State& Gs, float& Gt,
                                           float4& Gdirac) {
  const float dt_raw = t - s.t;
  const float dt = fmaxf(dt_raw, 0.f);
  const float area_raw = s.drgb.x * dt;
  const float area = fmaxf(area_raw, 0.f);
  const float rgb[3] = {safe_div(s.drgb.y, s.drgb.x), safe_div(s.drgb.z, s.drgb.x), safe_div(s.drgb.w, s.drgb.x)};
  const float ea_in = -area, el_in = -s.logT;
  const float e1 = safe_exp(ea_in), e2 = safe_exp(el_in);
  const float wraw = (1.f - e1) * e2;
  const float w = clampf(wraw, 0.f, 1.f);
  const float mid = ((t + s.t) * 0.5f) * 1000.f;
  const float m = tukey(mid);
  Gs.dist_x = G.dist_x;
  Gs.dist_y = G.dist_y;
  Gs.C = G.C;
  Gs.drgb = G.drgb;
  Gdirac = G.drgb;
  Gs.logT = 0.f;
  Gs.t = 0.f;
  Gt = G.t;
  float g_area = 0.f;
  if (area + s.logT > 0.f) {
    g_area += G.logT;
    Gs.logT += G.logT;
  }
  const float Gc[3] = {G.C.x, G.C.y, G.C.z};
  float g_w = Gc[0] * rgb[0] + Gc[1] * rgb[1] + Gc[2] * rgb[2];
  g_w += G.dist_x * 2.f * m * s.cum_x + G.dist_y * 2.f * s.cum_y + G.cum_x + G.cum_y * m;
  const float g_m = G.dist_x * 2.f * w * s.cum_x + G.cum_y * w;
  Gs.cum_x = G.cum_x + G.dist_x * 2.f * w * m;
  Gs.cum_y = G.cum_y + G.dist_y * 2.f * w;
  const float dv[3] = {s.drgb.y, s.drgb.z, s.drgb.w};
  float gd[3], gx = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float da, db;
    safe_div_bwd(dv[i], s.drgb.x, Gc[i] * w, da, db);
    gd[i] = da;
    gx += db;
  }
  Gs.drgb.y += gd[0];
  Gs.drgb.z += gd[1];
  Gs.drgb.w += gd[2];
  Gs.drgb.x += gx;
  if (wraw > 0.f && wraw < 1.f) {
    if (ea_in > kMinVal && ea_in < kLogMax) g_area += g_w * e2 * e1;
    if (el_in > kMinVal && el_in < kLogMax) Gs.logT += -g_w * (1.f - e1) * e2;
  }
  if (area_raw > 0.f) {
    Gs.drgb.x += g_area * dt;
    const float g_dt = g_area * s.drgb.x;
    if (dt_raw > 0.f) {
      Gt += g_dt;
      Gs.t -= g_dt;
    }
  }
  const float g_mid = g_m * dtukey(mid) * 500.f;
  Gt += g_mid;
  Gs.t += g_mid;
}

__device__ __forceinline__ void inverse4(const float* m, float* inv) {
  // cofactor expansion, row-major 4x4
  float a[16];
  a[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  a[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  a[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  a[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  a[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  a[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  a[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  a[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  a[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  a[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  a[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  a[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  a[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  a[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  a[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  a[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  const float det = m[0] * a[0] + m[1] * a[4] + m[2] * a[8] + m[3] * a[12];
  const float idet = 1.f / det;
  for (int i = 0; i < 16; ++i) inv[i] = a[i] * idet;
}

// d B_k / d(x,y,z) contracted with G_B: returns sum_k G_B[k] dB_k/dir.
template <int DEG>
__device__ __forceinline__ float3 sh_basis_vjp(float3 dir, const float* GB) {
  float3 g = make_float3(0.f, 0.f, 0.f);
  if (DEG < 1) return g;
  const float x = dir.x, y = dir.y, z = dir.z;
  g.y += -kShC1 * GB[1];
  g.z += kShC1 * GB[2];
  g.x += -kShC1 * GB[3];
  if (DEG < 2) return g;
  g.x += kShC2[0] * y * GB[4];
  g.y += kShC2[0] * x * GB[4];
  g.y += kShC2[1] * z * GB[5];
  g.z += kShC2[1] * y * GB[5];
  g.x += -2.f * kShC2[2] * x * GB[6];
  g.y += -2.f * kShC2[2] * y * GB[6];
  g.z += 4.f * kShC2[2] * z * GB[6];
  g.x += kShC2[3] * z * GB[7];
  g.z += kShC2[3] * x * GB[7];
  g.x += 2.f * kShC2[4] * x * GB[8];
  g.y += -2.f * kShC2[4] * y * GB[8];
  if (DEG < 3) return g;
  const float xx = x * x, yy = y * y, zz = z * z;
  g.x += 6.f * kShC3[0] * x * y * GB[9];
  g.y += kShC3[0] * (3.f * xx - 3.f * yy) * GB[9];
  g.x += kShC3[1] * y * z * GB[10];
  g.y += kShC3[1] * x * z * GB[10];
  g.z += kShC3[1] * x * y * GB[10];
  g.x += -2.f * kShC3[2] * x * y * GB[11];
  g.y += kShC3[2] * (4.f * zz - xx - 3.f * yy) * GB[11];
  g.z += 8.f * kShC3[2] * y * z * GB[11];
  g.x += -6.f * kShC3[3] * x * z * GB[12];
  g.y += -6.f * kShC3[3] * y * z * GB[12];
  g.z += kShC3[3] * (6.f * zz - 3.f * xx - 3.f * yy) * GB[12];
  g.x += kShC3[4] * (4.f * zz - 3.f * xx - yy) * GB[13];
  g.y += -2.f * kShC3[4] * x * y * GB[13];
  g.z += 8.f * kShC3[4] * x * z * GB[13];
  g.x += 2.f * kShC3[5] * x * z * GB[14];
  g.y += -2.f * kShC3[5] * y * z * GB[14];
  g.z += kShC3[5] * (xx - yy) * GB[14];
  g.x += kShC3[6] * (3.f * xx - 3.f * yy) * GB[15];
  g.y += -6.f * kShC3[6] * x * y * GB[15];
  return g;
}

__device__ __forceinline__ float clip_grad(float v, float lim) { return v != v ? v : fminf(fmaxf(v, -lim), lim); }

// The scene a ray is traced against, with its gradient accumulators.
struct BScene {
  const Node* nodes;
  const Record* recs;
  const float* features;
  const int32_t* order;  // Morton position -> original index
  int K;
  float* acc_geo;
  float* acc_feat;
};

// Per-launch ray-side inputs and outputs of the backward.
struct BRayCtx {
  const float* rayo;
  const float* rayd;
  float tmin;
  int max_iters;
  const float* grad_out;
  const float* states;
  const int32_t* iters;
  const int32_t* event_log;  // ray-major: row `slot` holds the ray's event ids in order
  int64_t log_cap;
  float* drayo;
  float* drayd;
  const float* wct;
  int num_wct;
  float* dmeans2d;
};

// Colour part of one control point's gradient: SH feature gradients (float4 atomics over
// the 16-byte aligned feature row), G_B for the ray direction; returns dL/d density.
template <int DEG>
__device__ __forceinline__ float colour_grads(const BScene& P, int j, float dh, float sign, float3 c, float4 Gd,
                                              const float* B, float* GB) {
  constexpr int NB = (DEG + 1) * (DEG + 1);
  constexpr int NV = (3 * NB + 3) / 4;
  const float g_dh = Gd.x + Gd.y * c.x + Gd.z * c.y + Gd.w * c.z;
  const float gc[3] = {dh * Gd.y, dh * Gd.z, dh * Gd.w};
  const int fst = feat_stride(P.K);
  const float4* f4 = reinterpret_cast<const float4*>(P.features + int64_t(j) * fst);
  float4* a4 = reinterpret_cast<float4*>(P.acc_feat + int64_t(j) * fst);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const float4 f = __ldg(f4 + i);
    const float fv[4] = {f.x, f.y, f.z, f.w};
    float g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = 4 * i + q;  // flat index 3k + ch
      if (e < 3 * NB) {
        const int k = e / 3, ch = e - 3 * (e / 3);
        g[q] = B[k] * gc[ch];
        GB[k] += fv[q] * gc[ch];
      } else {
        g[q] = 0.f;
      }
    }
    atomicAdd(a4 + i, make_float4(g[0], g[1], g[2], g[3]));
  }
  return sign * g_dh;
}

// Colour part of one event's gradient without the atomics: the SH-space colour gradient
// gc (the feature gradient is B_k gc[ch] for every coefficient k), G_B for the ray
// direction; returns dL/d density.
template <int DEG>
__device__ __forceinline__ float colour_coeffs(const BScene& P, int j, float dh, float sign, float3 c, float4 Gd,
                                               float* GB, float (&gc)[3]) {
  constexpr int NB = (DEG + 1) * (DEG + 1);
  constexpr int NV = (3 * NB + 3) / 4;
  const float g_dh = Gd.x + Gd.y * c.x + Gd.z * c.y + Gd.w * c.z;
  gc[0] = dh * Gd.y;
  gc[1] = dh * Gd.z;
  gc[2] = dh * Gd.w;
  const float4* f4 = reinterpret_cast<const float4*>(P.features + int64_t(j) * feat_stride(P.K));
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const float4 f = __ldg(f4 + i);
    const float fv[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = 4 * i + q;  // flat index 3k + ch
      if (e < 3 * NB) GB[e / 3] += fv[q] * gc[e - 3 * (e / 3)];
    }
  }
  return sign * g_dh;
}

// The SH-space colour gradient gc of one ellipsoid on one ray, summed over its events: the
// ellipsoid's feature gradient from this ray is B_k gc[ch] for every coefficient k, since the
// ray's SH basis B is the same at both events. Only this part is held back: it carries 12 of
// the 16 float4 atomics of an event at SH degree 3, in 3 registers per slot.
constexpr int kPendingSlots = 2;  // ellipsoids held open per ray (exit replayed, entry not yet)
constexpr int kGradRow = 3;

template <int DEG>
__device__ __forceinline__ void flush_grads(const BScene& S, const float* B, int j, const float (&v)[kGradRow]) {
  constexpr int NB = (DEG + 1) * (DEG + 1);
  constexpr int NV = (3 * NB + 3) / 4;
  float4* a4 = reinterpret_cast<float4*>(S.acc_feat + int64_t(j) * feat_stride(S.K));
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    float g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = 4 * i + q;
      g[q] = e < 3 * NB ? B[e / 3] * v[e - 3 * (e / 3)] : 0.f;
    }
    atomicAdd(a4 + i, make_float4(g[0], g[1], g[2], g[3]));
  }
}

// Adds one event's colour gradient for ellipsoid j. A convex ellipsoid has one exit and one
// entry per ray, met in that order by the reverse replay, so an exit opens a pending row
// and the entry closes it with one set of feature atomics for both events. An entry without
// a pending row (the exit was not consumed), a row evicted from a full set of slots, and the
// rows left open at the end of the replay are written as they are. On the 1M-ellipsoid
// 1080p view two slots leave 52% of the events' feature atomics (one slot: 59%).
template <int DEG>
__device__ __forceinline__ void pending_add(const BScene& S, const float* B, int (&pj)[kPendingSlots],
                                            float (&acc)[kPendingSlots][kGradRow], int j, bool entry,
                                            const float (&ev)[kGradRow]) {
  int fj = -1;
  float fv[kGradRow];
  bool held = false;
#pragma unroll
  for (int q = 0; q < kPendingSlots; ++q) {
    if (pj[q] == j) {
      held = true;
#pragma unroll
      for (int e = 0; e < kGradRow; ++e) acc[q][e] += ev[e];
      if (entry) {
        fj = j;
#pragma unroll
        for (int e = 0; e < kGradRow; ++e) fv[e] = acc[q][e];
        pj[q] = -1;
      }
    }
  }
  if (!held) {
    if (entry) {
      fj = j;
#pragma unroll
      for (int e = 0; e < kGradRow; ++e) fv[e] = ev[e];
    } else {
      bool placed = false;
#pragma unroll
      for (int q = 0; q < kPendingSlots; ++q) {
        if (!placed && pj[q] < 0) {
          placed = true;
          pj[q] = j;
#pragma unroll
          for (int e = 0; e < kGradRow; ++e) acc[q][e] = ev[e];
        }
      }
      if (!placed) {  // evict slot 0
        fj = pj[0];
#pragma unroll
        for (int e = 0; e < kGradRow; ++e) fv[e] = acc[0][e];
#pragma unroll
        for (int q = 0; q + 1 < kPendingSlots; ++q) {
          pj[q] = pj[q + 1];
#pragma unroll
          for (int e = 0; e < kGradRow; ++e) acc[q][e] = acc[q + 1][e];
        }
        pj[kPendingSlots - 1] = j;
#pragma unroll
        for (int e = 0; e < kGradRow; ++e) acc[kPendingSlots - 1][e] = ev[e];
      }
    }
  }
  if (fj >= 0) flush_grads<DEG>(S, B, fj, fv);
}

__device__ __forceinline__ float3 load3(const float* v, int64_t r) {
  return make_float3(v[3 * r], v[3 * r + 1], v[3 * r + 2]);
}

// Reverse replay of ray r = (ro, rd) (event-log column `slot`) against scene S. Ray
// gradients are written to P.drayo / P.drayd row r unless those are null.
template <int DEG>
__device__ void backward_ray(const BScene& S, const BRayCtx& P, int64_t r, int64_t slot, float3 ro, float3 rd) {
  const int n = P.iters[r];
  if (n >= P.max_iters - 1 || n <= 0) {  // backwards_kernel.slang:304
    if (P.drayo) {
      float* gro = P.drayo + 3 * r;
      float* grd = P.drayd + 3 * r;
      gro[0] = gro[1] = gro[2] = 0.f;
      grd[0] = grd[1] = grd[2] = 0.f;
    }
    return;
  }
  const Node* nodes = S.nodes;
  const Record* recs = S.recs;
  const Ray ray = make_ray(ro, rd, P.tmin);
  float B[16];
  sh_basis<DEG>(ray.rd, B);
  const int64_t fstride = feat_stride(S.K);

  // per-ray camera matrix for dmeans2d (backwards_kernel.slang:313-321)
  const bool per_ray_wct = P.wct && P.num_wct > 1 && P.dmeans2d;
  float wct[16], iwct[16];
  if (per_ray_wct) {
    const int64_t wi = r < P.num_wct ? r : 0;
    for (int i = 0; i < 16; ++i) wct[i] = P.wct[16 * wi + i];
    inverse4(wct, iwct);
  }

  State s;
  {
    const float4* sp = reinterpret_cast<const float4*>(P.states + 16 * r);
    const float4 a = sp[0], b = sp[1], c = sp[2], d = sp[3];
    s.dist_x = a.x;
    s.dist_y = a.y;
    s.cum_x = a.z;
    s.cum_y = a.w;
    s.t = b.w;
    s.drgb = c;
    s.logT = d.x;
    s.C = make_float3(d.y, d.z, d.w);
  }
  const float* go = P.grad_out + 5 * r;
  State G;
  G.C = make_float3(go[0], go[1], go[2]);
  G.logT = go[3] * expf(-s.logT);  // opacity = 1 - exp(-logT)
  G.dist_x = go[4];
  G.dist_y = -go[4];
  G.cum_x = G.cum_y = 0.f;
  G.t = 0.f;
  G.drgb = make_float4(0.f, 0.f, 0.f, 0.f);

  float3 Go = make_float3(0.f, 0.f, 0.f), Gdir = make_float3(0.f, 0.f, 0.f);
  float GB[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) GB[k] = 0.f;

  int pj[kPendingSlots];
  float acc[kPendingSlots][kGradRow];
#pragma unroll
  for (int q = 0; q < kPendingSlots; ++q) pj[q] = -1;
  Ctrl cur = load_ctrl<DEG>(recs, S.features, fstride, ray, B, P.event_log[slot * P.log_cap + (n - 1)]);
  for (int i = n - 1; i >= 0; --i) {
    Ctrl old;
    if (i > 0) {
      old = load_ctrl<DEG>(recs, S.features, fstride, ray, B, P.event_log[slot * P.log_cap + (i - 1)]);
    } else {
      old.t = 0.f;
      old.dirac = make_float4(0.f, 0.f, 0.f, 0.f);
      old.j = -1;
    }
    const State so = inverse_update(s, cur.dirac, old.t);
    State Gs;
    float Gt;
    float4 Gd;
    update_vjp(so, cur.t, G, Gs, Gt, Gd);

    const int j = cur.j;
    const Record R = load_record(recs, j);
    const float sign = cur.entry ? 1.f : -1.f;
    float gc[3];
    float g_sigma;
    if (DEG == 0) {  // the DC colour: no feature row, no direction gradient
      const float dh = sign * R.r3.x;
      g_sigma = sign * (Gd.x + Gd.y * cur.c.x + Gd.z * cur.c.y + Gd.w * cur.c.z);
      gc[0] = dh * Gd.y;
      gc[1] = dh * Gd.z;
      gc[2] = dh * Gd.w;
    } else {
      g_sigma = colour_coeffs<DEG>(S, j, sign * R.r3.x, sign, cur.c, Gd, GB, gc);
    }
    // event time: root of |ocn + t rdn|^2 = 1. dt = -(P.docn + t P.drdn) / (P.rdn) with the
    // hit point in the cancellation-free form P = l +- (sqrt(h)/a) rdn and P.rdn = +-sqrt(h)
    FullHit H;
    intersect_full(R, ray, H);
    const float t = cur.t;
    const float a_ = fmaf(H.rdn[2], H.rdn[2], fmaf(H.rdn[1], H.rdn[1], H.rdn[0] * H.rdn[0]));
    const float ba_ = -fmaf(H.ocn[2], H.rdn[2], fmaf(H.ocn[1], H.rdn[1], H.ocn[0] * H.rdn[0])) / a_;
    const float l_[3] = {fmaf(ba_, H.rdn[0], H.ocn[0]), fmaf(ba_, H.rdn[1], H.ocn[1]), fmaf(ba_, H.rdn[2], H.ocn[2])};
    const float ll_ = fmaf(l_[2], l_[2], fmaf(l_[1], l_[1], l_[0] * l_[0]));
    const float sh = sqrtf(fmaxf(a_ * (1.f - ll_), 0.f));
    const float sg_ = cur.entry ? -1.f : 1.f;
    const float Pv[3] = {fmaf(sg_ * sh / a_, H.rdn[0], l_[0]), fmaf(sg_ * sh / a_, H.rdn[1], l_[1]),
                         fmaf(sg_ * sh / a_, H.rdn[2], l_[2])};
    const float den = sg_ * sh;
    float gW[9], gmu[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 9; ++q) gW[q] = 0.f;
    if (fabsf(den) > kTiny && Gt != 0.f) {
      const float k0 = -Gt / den;
      float g_ocn[3], g_rdn[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        g_ocn[a] = k0 * Pv[a];
        g_rdn[a] = k0 * t * Pv[a];
      }
      const float v[3] = {ray.o.x - R.r0.w, ray.o.y - R.r1.w, ray.o.z - R.r2.w};
      const float dv[3] = {ray.d.x, ray.d.y, ray.d.z};
      const float Wm[9] = {R.r0.x, R.r0.y, R.r0.z, R.r1.x, R.r1.y, R.r1.z, R.r2.x, R.r2.y, R.r2.z};
      float gdd[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          gW[3 * a + b] = g_ocn[a] * v[b] + g_rdn[a] * dv[b];
          gmu[b] += Wm[3 * a + b] * g_ocn[a];
          gdd[b] += Wm[3 * a + b] * g_rdn[a];
        }
      }
      Go.x += gmu[0];
      Go.y += gmu[1];
      Go.z += gmu[2];
      Gdir.x += gdd[0];
      Gdir.y += gdd[1];
      Gdir.z += gdd[2];
      if (per_ray_wct) {
        // project / inv_project, backwards_kernel.slang:213-220, 244-257
        const float mx = R.r0.w, my = R.r1.w, mz = R.r2.w;
        const float z = mx * wct[2] + my * wct[6] + mz * wct[10] + wct[14];
        const float gm[3] = {-gmu[0], -gmu[1], -gmu[2]};
        const int p = __ldg(S.order + j);
        const float dx = z * (iwct[0] * gm[0] + iwct[1] * gm[1] + iwct[2] * gm[2]);
        const float dy = z * (iwct[4] * gm[0] + iwct[5] * gm[1] + iwct[6] * gm[2]);
        atomicAdd(reinterpret_cast<float2*>(P.dmeans2d) + p, make_float2(dx, dy));
      }
    }
    float4* ag = reinterpret_cast<float4*>(S.acc_geo + int64_t(j) * kGeo);
    atomicAdd(ag + 0, make_float4(gW[0], gW[1], gW[2], gW[3]));
    atomicAdd(ag + 1, make_float4(gW[4], gW[5], gW[6], gW[7]));
    atomicAdd(ag + 2, make_float4(gW[8], -gmu[0], -gmu[1], -gmu[2]));
    if (DEG == 0) {
      // degree 0: the DC feature gradient B_0 gc rides in the row's three pad floats
      atomicAdd(ag + 3, make_float4(g_sigma, B[0] * gc[0], B[0] * gc[1], B[0] * gc[2]));
    } else {
      atomicAdd(ag + 3, make_float4(g_sigma, 0.f, 0.f, 0.f));
      const float ev[kGradRow] = {gc[0], gc[1], gc[2]};
      pending_add<DEG>(S, B, pj, acc, j, cur.entry, ev);
    }
    s = so;
    G = Gs;
    G.t = Gs.t;
    cur = old;
  }

#pragma unroll
  for (int q = 0; q < kPendingSlots; ++q)
    if (pj[q] >= 0) flush_grads<DEG>(S, B, pj[q], acc[q]);

  // initial density: backwards_initial_drgb_kernel, backwards_kernel.slang:374-428
  if (G.drgb.x != 0.f || G.drgb.y != 0.f || G.drgb.z != 0.f || G.drgb.w != 0.f) {
    // point-query stack in local memory: only rays that start inside ellipsoids touch it,
    // and the kernels keep all of the SM's on-chip memory as L1 for the scattered loads
    int st_node[kStackDepth];
    int sp = 0, node = 0;
    for (;;) {
      const float4* np = reinterpret_cast<const float4*>(nodes + node);
      const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
      const int4 d = __ldg(reinterpret_cast<const int4*>(np + 3));
      const float3 o = ray.o;
      const bool h0 = o.x >= a.x && o.x <= a.w && o.y >= a.y && o.y <= b.x && o.z >= a.z && o.z <= b.y;
      const bool h1 = o.x >= b.z && o.x <= c.y && o.y >= b.w && o.y <= c.z && o.z >= c.x && o.z <= c.w;
      const int ch[2] = {d.x, d.y};
      const bool hh[2] = {h0, h1};
      for (int k = 0; k < 2; ++k) {
        if (hh[k] && ch[k] < 0) {
          const int j = ~ch[k];
          const Record R = load_record(recs, j);
          HitT H;
          if (intersect(R, ray, H) && H.t0 <= 0.f && H.t1 > 0.f) {
            if (DEG == 0) {
              const float3 col = dc_colour(R.r3);
              const float4 Gd = G.drgb;
              const float dh = R.r3.x;
              const float g_sigma = Gd.x + Gd.y * col.x + Gd.z * col.y + Gd.w * col.z;
              atomicAdd(reinterpret_cast<float4*>(S.acc_geo + int64_t(j) * kGeo) + 3,
                        make_float4(g_sigma, B[0] * (dh * Gd.y), B[0] * (dh * Gd.z), B[0] * (dh * Gd.w)));
            } else {
              const float3 col = sh_colour<DEG>(S.features + j * fstride, B);
              const float g_sigma = colour_grads<DEG>(S, j, R.r3.x, 1.f, col, G.drgb, B, GB);
              atomicAdd(S.acc_geo + int64_t(j) * kGeo + 12, g_sigma);
            }
          }
        }
      }
      const bool i0 = h0 && ch[0] >= 0, i1 = h1 && ch[1] >= 0;
      if (i0 && i1) {
        if (sp < kStackDepth) st_node[sp++] = ch[1];
        node = ch[0];
      } else if (i0) {
        node = ch[0];
      } else if (i1) {
        node = ch[1];
      } else {
        if (sp == 0) break;
        node = st_node[--sp];
      }
    }
  }

  // ray gradients: o = rayo + tmin rayd; d = rayd / |rayd|; SH basis of the raw rayd
  if (!P.drayo) return;
  float* gro = P.drayo + 3 * r;
  float* grd = P.drayd + 3 * r;
  float3 g_rd = sh_basis_vjp<DEG>(ray.rd, GB);
  const float dd = fmaf(rd.z, rd.z, fmaf(rd.y, rd.y, rd.x * rd.x));
  const float nrm = sqrtf(fmaxf(dd, kTiny));
  const float dG = ray.d.x * Gdir.x + ray.d.y * Gdir.y + ray.d.z * Gdir.z;
  g_rd.x += (Gdir.x - ray.d.x * dG) / nrm + P.tmin * Go.x;
  g_rd.y += (Gdir.y - ray.d.y * dG) / nrm + P.tmin * Go.y;
  g_rd.z += (Gdir.z - ray.d.z * dG) / nrm + P.tmin * Go.z;
  gro[0] = clip_grad(Go.x, 1e3f);
  gro[1] = clip_grad(Go.y, 1e3f);
  gro[2] = clip_grad(Go.z, 1e3f);
  grd[0] = clip_grad(g_rd.x, 1e3f);
  grd[1] = clip_grad(g_rd.y, 1e3f);
  grd[2] = clip_grad(g_rd.z, 1e3f);
}

// 128 registers (two 256-thread or four 128-thread blocks per SM): the pending rows cost a
// few spilled bytes, which 16 resident warps hide better than 40 more registers would.
template <int DEG>
__global__ void __launch_bounds__(256, kBwdMinBlocks<DEG>) k_trace_bwd(const BwdParams P) {
  const int tid = threadIdx.x;
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;
  if (gi >= P.R) return;
  const int64_t slot = P.slot_order ? int64_t(P.slot_order[gi]) : gi;  // event-log column
  const int64_t r = P.ray_order ? int64_t(P.ray_order[slot]) : slot;
  const BScene S{reinterpret_cast<const Node*>(P.nodes), reinterpret_cast<const Record*>(P.records), P.features,
                 P.order, P.K, P.acc_geo, P.acc_feat};
  const BRayCtx C{P.rayo, P.rayd, P.tmin, P.max_iters, P.grad_out, P.states, P.iters, P.event_log, P.log_cap,
                  P.drayo, P.drayd, P.wct, P.num_wct, P.dmeans2d};
  backward_ray<DEG>(S, C, r, slot, load3(P.rayo, r), load3(P.rayd, r));
}

// Backward of a camera trace: threads take slots (through the slot order, if any), make
// the slot's pixel ray from the camera as the forward did, and replay it.
template <int DEG>
__global__ void __launch_bounds__(256, kBwdMinBlocks<DEG>)
    k_trace_bwd_camera(const BwdParams P, const CameraParams cam, const float* __restrict__ jitter) {
  const int tid = threadIdx.x;
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;
  if (gi >= P.R) return;
  const int64_t slot = P.slot_order ? int64_t(P.slot_order[gi]) : gi;
  const int64_t p = camera_slot_pixel(cam, slot);
  if (p < 0) return;
  const BScene S{reinterpret_cast<const Node*>(P.nodes), reinterpret_cast<const Record*>(P.records), P.features,
                 P.order, P.K, P.acc_geo, P.acc_feat};
  const BRayCtx C{nullptr, nullptr, P.tmin, P.max_iters, P.grad_out, P.states, P.iters, P.event_log, P.log_cap,
                  P.drayo, P.drayd, P.wct, P.num_wct, P.dmeans2d};
  float3 ro, rd;
  camera_ray(cam, jitter, p, ro, rd);
  backward_ray<DEG>(S, C, p, slot, ro, rd);
}

// Persistent batched backward: warps take 32-slot packets from a device counter. With a
// slot order the lanes of a packet may replay slots of different views and scenes (the
// backward does not traverse, so nothing needs to be warp-uniform): each lane finds its
// own view by binary search over the views' slot ranges.
template <int DEG>
__global__ void __launch_bounds__(256, kBwdMinBlocks<DEG>) k_trace_bwd_batched(const BatchBwdParams P) {
  const int tid = threadIdx.x, lane = tid & 31;
  const BRayCtx C{P.rayo, P.rayd, P.tmin, P.max_iters, P.grad_out, P.states, P.iters, P.event_log, P.log_cap,
                  P.drayo, P.drayd, nullptr, 0, nullptr};
  const int64_t num_packets = P.num_slots / 32;
  for (;;) {
    unsigned int pk = 0;
    if (lane == 0) pk = atomicAdd(P.work_counter, 1u);
    pk = __shfl_sync(0xffffffffu, pk, 0);
    if (int64_t(pk) >= num_packets) break;
    const int64_t pos = int64_t(pk) * 32 + lane;
    const int64_t slot = P.slot_order ? int64_t(P.slot_order[pos]) : pos;
    int lo = 0, hi = P.num_views - 1;  // last view with slot_offset <= slot
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.views[mid].slot_offset <= slot) lo = mid;
      else hi = mid - 1;
    }
    const int v = lo;
    const BatchScene bs_ = P.scenes[P.views[v].scene];
    const BScene S{reinterpret_cast<const Node*>(bs_.nodes), reinterpret_cast<const Record*>(bs_.records),
                   bs_.features, bs_.order, bs_.K, bs_.acc_geo, bs_.acc_feat};
    const int32_t r = P.slot_ray[slot];
    if (r >= 0) backward_ray<DEG>(S, C, r, slot, load3(P.rayo, r), load3(P.rayd, r));
    __syncwarp();
  }
}

// VJP of rotate_vector(v, q) w.r.t. q.
__device__ __forceinline__ void rotate_vector_vjp_q(const float v[3], float4 q, const float g[3], float gq[4]) {
  const float w = q.x, u[3] = {-q.y, -q.z, -q.w};
  const float uxv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  gq[0] += 2.f * (g[0] * uxv[0] + g[1] * uxv[1] + g[2] * uxv[2]);
  const float vxg[3] = {v[1] * g[2] - v[2] * g[1], v[2] * g[0] - v[0] * g[2], v[0] * g[1] - v[1] * g[0]};
  const float uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
  const float gu = g[0] * u[0] + g[1] * u[1] + g[2] * u[2];
  const float gv = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
#pragma unroll
  for (int i = 0; i < 3; ++i) gq[1 + i] -= 2.f * w * vxg[i] + 2.f * (uv * g[i] + gu * v[i] - 2.f * gv * u[i]);
}

// Per ellipsoid: W gradients -> scale / quaternion gradients, dmeans2d, clipping
// (fast_ellipsoid_splinetracer.py:204-219), scatter to original order.
// Morton position of every original index: inv[order[j]] = j.
__global__ void k_inverse_order(const int32_t* __restrict__ order, int64_t N, int32_t* __restrict__ inv) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j < N) inv[order[j]] = int32_t(j);
}

// One thread per ellipsoid in original order (the gradient tensors' order), so the writes
// are coalesced; it reads its Morton-ordered gradient row and record through inv_order.
__global__ void k_finalize(const FinalizeParams P) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  __shared__ float wct[16], iwct[16];
  const bool single_wct = P.wct && P.num_wct == 1 && P.out.dmeans2d;
  if (single_wct && threadIdx.x == 0) {
    for (int i = 0; i < 16; ++i) wct[i] = P.wct[i];
    inverse4(wct, iwct);
  }
  __syncthreads();
  if (p >= P.N) return;
  const int64_t j = P.inv_order[p];
  float g[kGeo];
  {
    const float4* g4 = reinterpret_cast<const float4*>(P.acc_geo + j * kGeo);
#pragma unroll
    for (int i = 0; i < kGeo / 4; ++i) {
      const float4 v = g4[i];
      g[4 * i] = v.x;
      g[4 * i + 1] = v.y;
      g[4 * i + 2] = v.z;
      g[4 * i + 3] = v.w;
    }
  }
  const Record R = load_record(reinterpret_cast<const Record*>(P.records), int(j));
  const float Wm[9] = {R.r0.x, R.r0.y, R.r0.z, R.r1.x, R.r1.y, R.r1.z, R.r2.x, R.r2.y, R.r2.z};
  const float4 q = make_float4(P.quat[4 * p], P.quat[4 * p + 1], P.quat[4 * p + 2], P.quat[4 * p + 3]);
  const float sv[3] = {P.scale[3 * p], P.scale[3 * p + 1], P.scale[3 * p + 2]};
  float gs[3] = {0.f, 0.f, 0.f}, gq[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int b = 0; b < 3; ++b) gs[i] -= g[3 * i + b] * Wm[3 * i + b] / sv[i];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const float e[3] = {b == 0 ? 1.f : 0.f, b == 1 ? 1.f : 0.f, b == 2 ? 1.f : 0.f};
    const float gcol[3] = {g[b] / sv[0], g[3 + b] / sv[1], g[6 + b] / sv[2]};
    rotate_vector_vjp_q(e, q, gcol, gq);
  }
  const float gm[3] = {g[9], g[10], g[11]};
  for (int i = 0; i < 3; ++i) {
    P.out.dmean[3 * p + i] = clip_grad(gm[i], 1e3f);
    P.out.dscale[3 * p + i] = clip_grad(gs[i], 1e3f);
  }
  for (int i = 0; i < 4; ++i) P.out.dquat[4 * p + i] = clip_grad(gq[i], 1e3f);
  P.out.ddensity[p] = clip_grad(g[12], 50.f);

  if (single_wct) {
    const float mx = P.mean[3 * p], my = P.mean[3 * p + 1], mz = P.mean[3 * p + 2];
    const float z = mx * wct[2] + my * wct[6] + mz * wct[10] + wct[14];
    P.out.dmeans2d[2 * p] = z * (iwct[0] * gm[0] + iwct[1] * gm[1] + iwct[2] * gm[2]);
    P.out.dmeans2d[2 * p + 1] = z * (iwct[4] * gm[0] + iwct[5] * gm[1] + iwct[6] * gm[2]);
  }
}

// Feature gradients back to original order and shape (N,K,3), clipped at 1e3: one row per
// threadIdx.y, one float4 column per threadIdx.x (blockDim.x = feat_stride(K) / 4). vec: the
// output rows are whole, 16-byte aligned float4s (3K % 4 == 0, aligned base). The DC
// gradient of degree-0 traces sits in the pad floats 13..15 of the geometry row and is
// added to coefficient 0; dc_only: the feature rows were not used (all zero, not read).
__global__ void k_finalize_features(const int32_t* __restrict__ order, int64_t N, int K,
                                    const float* __restrict__ acc_feat, const float* __restrict__ acc_geo,
                                    bool dc_only, float* __restrict__ dfeat, bool vec) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.y + threadIdx.y;
  if (j >= N) return;
  const int c = threadIdx.x, per = 3 * K;
  float4 a = dc_only ? make_float4(0.f, 0.f, 0.f, 0.f)
                     : reinterpret_cast<const float4*>(acc_feat + j * feat_stride(K))[c];
  if (c == 0) {
    const float* g = acc_geo + j * kGeo;
    a.x += g[13];
    a.y += g[14];
    a.z += g[15];
  }
  const float4 g = make_float4(clip_grad(a.x, 1e3f), clip_grad(a.y, 1e3f), clip_grad(a.z, 1e3f), clip_grad(a.w, 1e3f));
  float* dst = dfeat + int64_t(__ldg(order + j)) * per;
  if (vec) {
    reinterpret_cast<float4*>(dst)[c] = g;
  } else {
    const float t[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (4 * c + q < per) dst[4 * c + q] = t[q];
  }
}

// tri[i * R + ray] from log[slot * log_cap + i], ray = ray_order[slot] (or slot).
__global__ void k_log_to_reference(const int32_t* __restrict__ order, const int32_t* __restrict__ log, int log_cap,
                                   const int32_t* __restrict__ iters, int64_t R, const int32_t* __restrict__ ray_order,
                                   int32_t* __restrict__ tri, int max_iters) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= R * int64_t(max_iters)) return;
  const int64_t i = t / R, slot = t - i * R;
  const int64_t r = ray_order ? int64_t(ray_order[slot]) : slot;
  int32_t v = 0;
  if (i < iters[r] && i < log_cap) {
    const int32_t id = log[slot * log_cap + i];
    v = 2 * order[id >> 1] + (id & 1);
  }
  tri[i * R + r] = v;
}

template <int DEG>
cudaError_t launch_b(const BwdParams& P, int block, cudaStream_t st) {
  k_trace_bwd<DEG><<<unsigned((P.R + block - 1) / block), block, 0, st>>>(P);
  return cudaGetLastError();
}

}  // namespace

template <int DEG>
cudaError_t launch_bc(const BwdParams& P, const CameraParams& cam, const float* jitter, int block, cudaStream_t st) {
  k_trace_bwd_camera<DEG><<<unsigned((P.R + block - 1) / block), block, 0, st>>>(P, cam, jitter);
  return cudaGetLastError();
}

__global__ void k_camera_slot_pixels(const CameraParams cam, int64_t num_slots, int32_t* __restrict__ slot_pixel) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s < num_slots) slot_pixel[s] = int32_t(camera_slot_pixel(cam, s));
}

__global__ void k_camera_log_to_reference(const CameraParams cam, int64_t num_slots, const int32_t* __restrict__ order,
                                          const int32_t* __restrict__ log, int log_cap,
                                          const int32_t* __restrict__ iters, int32_t* __restrict__ tri,
                                          int max_iters) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= num_slots * int64_t(max_iters)) return;
  const int64_t i = t / num_slots, slot = t - i * num_slots;
  const int64_t r = camera_slot_pixel(cam, slot);
  if (r < 0) return;
  int32_t v = 0;
  if (i < iters[r] && i < log_cap) {
    const int32_t id = log[slot * log_cap + i];
    v = 2 * order[id >> 1] + (id & 1);
  }
  tri[i * (int64_t(cam.width) * cam.height) + r] = v;
}

template <int DEG>
cudaError_t launch_bb(const BatchBwdParams& P, int block, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(P.work_counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  k_trace_bwd_batched<DEG><<<P.grid, block, 0, st>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_backward_batched(const BatchBwdParams& P, int deg, const EverTune& tune, cudaStream_t st) {
  if (P.num_slots == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (deg) {
    case 0: return launch_bb<0>(P, block, st);
    case 1: return launch_bb<1>(P, block, st);
    case 2: return launch_bb<2>(P, block, st);
    default: return launch_bb<3>(P, block, st);
  }
}

cudaError_t launch_backward(const BwdParams& P, int deg, const EverTune& tune, cudaStream_t st) {
  if (P.R == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (deg) {
    case 0: return launch_b<0>(P, block, st);
    case 1: return launch_b<1>(P, block, st);
    case 2: return launch_b<2>(P, block, st);
    default: return launch_b<3>(P, block, st);
  }
}

cudaError_t launch_backward_camera(const BwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                   const EverTune& tune, cudaStream_t st) {
  if (P.R == 0) return cudaSuccess;
  const int block = tune.block > 0 ? tune.block : 128;
  switch (deg) {
    case 0: return launch_bc<0>(P, cam, jitter, block, st);
    case 1: return launch_bc<1>(P, cam, jitter, block, st);
    case 2: return launch_bc<2>(P, cam, jitter, block, st);
    default: return launch_bc<3>(P, cam, jitter, block, st);
  }
}

cudaError_t launch_camera_slot_pixels(const CameraParams& cam, int32_t* slot_pixel, cudaStream_t st) {
  const int64_t n = camera_slots(cam);
  if (n == 0) return cudaSuccess;
  k_camera_slot_pixels<<<unsigned((n + 255) / 256), 256, 0, st>>>(cam, n, slot_pixel);
  return cudaGetLastError();
}

cudaError_t launch_camera_log_to_reference(const CameraParams& cam, const int32_t* order, const int32_t* log,
                                           int log_cap, const int32_t* iters, int32_t* tri, int max_iters,
                                           cudaStream_t st) {
  const int64_t n = camera_slots(cam) * int64_t(max_iters);
  if (n == 0) return cudaSuccess;
  k_camera_log_to_reference<<<unsigned((n + 255) / 256), 256, 0, st>>>(cam, camera_slots(cam), order, log, log_cap,
                                                                       iters, tri, max_iters);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeParams& P, cudaStream_t st) {
  if (P.N == 0) return cudaSuccess;
  k_inverse_order<<<unsigned((P.N + 255) / 256), 256, 0, st>>>(P.order, P.N, P.inv_order);
  k_finalize<<<unsigned((P.N + 255) / 256), 256, 0, st>>>(P);
  const int cols = feat_stride(P.K) / 4, rows = 256 / cols > 0 ? 256 / cols : 1;
  const bool vec = (3 * P.K) % 4 == 0 && reinterpret_cast<uintptr_t>(P.out.dfeatures) % 16 == 0;
  k_finalize_features<<<unsigned((P.N + rows - 1) / rows), dim3(cols, rows), 0, st>>>(
      P.order, P.N, P.K, P.acc_feat, P.acc_geo, P.dc_only, P.out.dfeatures, vec);
  return cudaGetLastError();
}

cudaError_t launch_log_to_reference(const int32_t* order, const int32_t* log, int log_cap, const int32_t* iters,
                                    int64_t R, const int32_t* ray_order, int32_t* tri, int max_iters, cudaStream_t st) {
  const int64_t total = R * int64_t(max_iters);
  if (total == 0) return cudaSuccess;
  k_log_to_reference<<<unsigned((total + 255) / 256), 256, 0, st>>>(order, log, log_cap, iters, R, ray_order, tri,
                                                                    max_iters);
  return cudaGetLastError();
}

}  // namespace ever
