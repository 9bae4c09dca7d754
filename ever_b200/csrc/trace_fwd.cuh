// Forward trace kernels (included by trace_fwd_k{8,16,32}.cu, one k-buffer size per
// translation unit so the instantiations compile in parallel).
//
// LBVH traversal that gathers each ray's next KBUF entry/exit events into
// a sorted register buffer, then integrates them in order (update() with SH colour
// evaluated along the ray), round after round.
//
// Two traversals share the same gather/consume semantics:
//  - packet (default): the 32 rays of a warp walk ONE node sequence together. Each
//    lane tests its own ray against the node's two child boxes, __ballot_sync decides
//    where the warp goes, and a per-warp stack lives in shared memory. Node fetches
//    are warp-uniform (one broadcast load) and the control flow never diverges.
//  - per-ray: each thread walks the tree alone (stack in shared memory per thread).
//
// Reference: raygen loop splinetracers/fast_ellipsoid_splinetracer/slang/shaders.slang:171-235,
// intersection program :84-107 and any-hit k-buffer :117-164. Our rounds gather
// events strictly after the last gathered one in the total order (t, Morton position,
// entry-before-exit), so no round boundary of ours drops an event; the reference's own
// 16-event round boundaries are replayed while consuming (s16 below): an event tied with
// the 16th event of a reference round is dropped, and an exit beyond tmax counts only
// inside the reference round that consumed its entry. The result is the reference's
// event sequence for any KBUF.
#pragma once
#include <climits>

#include "camera.cuh"
#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxMembers = 16;

template <int KBUF>
__device__ __forceinline__ void buf_insert(uint64_t (&buf)[KBUF], uint64_t k) {
#pragma unroll
  for (int i = 0; i < KBUF; ++i) {
    const uint64_t b = buf[i];
    const bool lt = k < b;
    buf[i] = lt ? k : b;
    k = lt ? b : k;
  }
}

__device__ __forceinline__ Node load_node(const Node* __restrict__ nodes, int n) {
  const float4* p = reinterpret_cast<const float4*>(nodes + n);
  Node nd;
  nd.a = __ldg(p + 0);
  nd.b = __ldg(p + 1);
  nd.c = __ldg(p + 2);
  nd.d = __ldg(reinterpret_cast<const int4*>(p + 3));
  return nd;
}

struct RaySlab {
  float3 invd, ood;
};

__device__ __forceinline__ RaySlab make_slab(const Ray& r) {
  auto inv = [](float d) { return 1.f / (fabsf(d) > 1e-20f ? d : copysignf(1e-20f, d)); };
  RaySlab s;
  s.invd = make_float3(inv(r.d.x), inv(r.d.y), inv(r.d.z));
  s.ood = make_float3(r.o.x * s.invd.x, r.o.y * s.invd.y, r.o.z * s.invd.z);
  return s;
}

// Slab test of [lo, hi] against [tlo, thi]; returns the entry distance or +inf on a miss.
__device__ __forceinline__ float slab(const RaySlab& s, float lx, float ly, float lz, float hx, float hy, float hz,
                                      float tlo, float thi) {
  const float ax = fmaf(lx, s.invd.x, -s.ood.x), bx = fmaf(hx, s.invd.x, -s.ood.x);
  const float ay = fmaf(ly, s.invd.y, -s.ood.y), by = fmaf(hy, s.invd.y, -s.ood.y);
  const float az = fmaf(lz, s.invd.z, -s.ood.z), bz = fmaf(hz, s.invd.z, -s.ood.z);
  const float tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), tlo));
  const float tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), thi));
  return tn <= tf ? tn : INFINITY;
}

__device__ __forceinline__ bool box_contains(float lx, float ly, float lz, float hx, float hy, float hz, float3 p) {
  return p.x >= lx && p.x <= hx && p.y >= ly && p.y <= hy && p.z >= lz && p.z <= hz;
}

// One leaf: the ellipsoid's entry/exit events that are candidates of this round
// (see the file comment) go into the sorted buffer.
template <int KBUF>
__device__ __forceinline__ void leaf_insert(const Record* __restrict__ recs, int j, const Ray& ray, uint64_t lower,
                                            float s16, float tmax, uint64_t (&buf)[KBUF]) {
  const Record R = load_record(recs, j);
  HitT H;
  if (!intersect(R, ray, H)) return;
  if (H.t0 > s16 && H.t0 <= tmax) {
    const uint64_t e = event_key(H.t0, j, 0);
    if (e > lower && e < buf[KBUF - 1]) buf_insert(buf, e);
  }
  if (H.t1 > s16 && (H.t1 <= tmax || (H.t0 > s16 && H.t0 <= tmax))) {
    const uint64_t e = event_key(H.t1, j, 1);
    if (e > lower && e < buf[KBUF - 1]) buf_insert(buf, e);
  }
}

// ---- per-ray traversal ----
template <int KBUF>
__device__ void gather_ray(const Node* __restrict__ nodes, const Record* __restrict__ recs, const Ray& ray,
                           const RaySlab& sl, uint64_t lower, float s16, float tmax, uint64_t (&buf)[KBUF],
                           int* st_node, float* st_t, int stride, int depth, uint32_t& status) {
  const float lo_t = fmaxf(lower ? key_t(lower) : 0.f, s16);
  const float cap = fminf(tmax, kSentinel);
  int sp = 0;
  int node = 0;
  for (;;) {
    const Node nd = load_node(nodes, node);
    const float hi = fminf(cap, key_t(buf[KBUF - 1]));  // an empty slot is NaN: fminf keeps cap
    const float tc[2] = {slab(sl, nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, lo_t, hi),
                         slab(sl, nd.b.z, nd.b.w, nd.c.x, nd.c.y, nd.c.z, nd.c.w, lo_t, hi)};
    const int c[2] = {nd.d.x, nd.d.y};
#pragma unroll
    for (int k = 0; k < 2; ++k)
      if (tc[k] != INFINITY && c[k] < 0) leaf_insert(recs, ~c[k], ray, lower, s16, tmax, buf);
    const bool i0 = tc[0] != INFINITY && c[0] >= 0;
    const bool i1 = tc[1] != INFINITY && c[1] >= 0;
    if (i0 && i1) {
      const bool first0 = tc[0] <= tc[1];
      if (sp < depth) {
        st_node[sp * stride] = first0 ? c[1] : c[0];
        st_t[sp * stride] = first0 ? tc[1] : tc[0];
        ++sp;
      } else {
        status |= EVER_STATUS_STACK_OVERFLOW;
      }
      node = first0 ? c[0] : c[1];
      continue;
    }
    if (i0 || i1) {
      node = i0 ? c[0] : c[1];
      continue;
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      if (st_t[sp * stride] <= fminf(cap, key_t(buf[KBUF - 1]))) {
        node = st_node[sp * stride];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
}

// ---- packet traversal: the warp walks one node sequence ----
template <int KBUF>
__device__ void gather_packet(const Node* __restrict__ nodes, const Record* __restrict__ recs, const Ray& ray,
                              const RaySlab& sl, bool act, uint64_t lower, float s16, float tmax,
                              uint64_t (&buf)[KBUF], int* wstack, int lane, int depth, uint32_t& status) {
  const float lo_t = fmaxf(lower ? key_t(lower) : 0.f, s16);
  const float cap = fminf(tmax, kSentinel);
  int sp = 0;
  int node = 0;
  for (;;) {
    const Node nd = load_node(nodes, node);
    float t0 = INFINITY, t1 = INFINITY;
    if (act) {
      const float hi = fminf(cap, key_t(buf[KBUF - 1]));
      t0 = slab(sl, nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, lo_t, hi);
      t1 = slab(sl, nd.b.z, nd.b.w, nd.c.x, nd.c.y, nd.c.z, nd.c.w, lo_t, hi);
    }
    const unsigned m0 = __ballot_sync(kFull, t0 != INFINITY);
    const unsigned m1 = __ballot_sync(kFull, t1 != INFINITY);
    const int c0 = nd.d.x, c1 = nd.d.y;
    if (c0 < 0 && t0 != INFINITY) leaf_insert(recs, ~c0, ray, lower, s16, tmax, buf);
    if (c1 < 0 && t1 != INFINITY) leaf_insert(recs, ~c1, ray, lower, s16, tmax, buf);
    const bool g0 = c0 >= 0 && m0 != 0u, g1 = c1 >= 0 && m1 != 0u;
    if (g0 && g1) {
      // nearer child first, by majority of the lanes that hit either
      const unsigned pref0 = __ballot_sync(kFull, t0 <= t1 && t0 != INFINITY);
      const bool first0 = 2 * __popc(pref0) >= __popc(m0 | m1);
      if (sp < depth) {
        if (lane == 0) {
          const int far = first0 ? c1 : c0;
          wstack[sp] = far;
          asm volatile("prefetch.global.L1 [%0];" ::"l"(nodes + far));
        }
        ++sp;
      } else {
        status |= EVER_STATUS_STACK_OVERFLOW;
      }
      __syncwarp();
      node = first0 ? c0 : c1;
    } else if (g0 || g1) {
      node = g0 ? c0 : c1;
    } else {
      if (sp == 0) break;
      --sp;
      node = wstack[sp];
    }
  }
}

__device__ __forceinline__ void member_insert(int p, int j, int& n_mem, int (&mem_p)[kMaxMembers],
                                              int (&mem_j)[kMaxMembers]) {
  int jj = j;
  for (int q = 0; q < n_mem; ++q) {
    if (p < mem_p[q]) {
      const int tp = mem_p[q], tj = mem_j[q];
      mem_p[q] = p;
      mem_j[q] = jj;
      p = tp;
      jj = tj;
    }
  }
  mem_p[n_mem] = p;
  mem_j[n_mem] = jj;
  ++n_mem;
}

// Ellipsoid j contains the ray start (t0 <= 0 < t1): record it (sorted by original index);
// beyond kMaxMembers the rest are summed into `extra` in traversal order (status flag).
template <int DEG>
__device__ __forceinline__ void point_leaf(const Record* __restrict__ recs, const int32_t* __restrict__ order,
                                           const float* __restrict__ feats, int fst, const float* B, int bs,
                                           const Ray& ray, int j, int& n_mem, int (&mem_p)[kMaxMembers],
                                           int (&mem_j)[kMaxMembers], float4& extra, uint32_t& status) {
  const Record R = load_record(recs, j);
  HitT H;
  if (!(intersect(R, ray, H) && H.t0 <= 0.f && H.t1 > 0.f)) return;
  if (n_mem < kMaxMembers) {
    member_insert(__ldg(order + j), j, n_mem, mem_p, mem_j);
  } else {
    status |= EVER_STATUS_INIT_OVERFLOW;
    const float sg = R.r3.x;
    const float3 c = DEG == 0 ? dc_colour(R.r3) : sh_colour<DEG>(feats + int64_t(j) * fst, B, bs);
    extra.x = extra.x + sg;
    extra.y = extra.y + sg * c.x;
    extra.z = extra.z + sg * c.y;
    extra.w = extra.w + sg * c.z;
  }
}

// Point query for the ray start; PACKET: warp-uniform walk.
template <int DEG, bool PACKET>
__device__ int point_members(const Node* __restrict__ nodes, const Record* __restrict__ recs,
                             const int32_t* __restrict__ order, const float* __restrict__ feats, int fst,
                             const float* B, int bs, const Ray& ray, bool act,
                             int* stack, int stride, int depth, int lane, int (&mem_p)[kMaxMembers],
                             int (&mem_j)[kMaxMembers], float4& extra, uint32_t& status) {
  int n_mem = 0;
  int sp = 0;
  int node = 0;
  for (;;) {
    const Node nd = load_node(nodes, node);
    const bool h0 = act && box_contains(nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, ray.o);
    const bool h1 = act && box_contains(nd.b.z, nd.b.w, nd.c.x, nd.c.y, nd.c.z, nd.c.w, ray.o);
    const int c0 = nd.d.x, c1 = nd.d.y;
    if (h0 && c0 < 0) point_leaf<DEG>(recs, order, feats, fst, B, bs, ray, ~c0, n_mem, mem_p, mem_j, extra, status);
    if (h1 && c1 < 0) point_leaf<DEG>(recs, order, feats, fst, B, bs, ray, ~c1, n_mem, mem_p, mem_j, extra, status);
    bool g0 = h0 && c0 >= 0, g1 = h1 && c1 >= 0;
    if (PACKET) {
      g0 = __any_sync(kFull, g0);
      g1 = __any_sync(kFull, g1);
    }
    if (g0 && g1) {
      if (sp < depth) {
        if (!PACKET || lane == 0) stack[sp * stride] = c1;
        ++sp;
      } else {
        status |= EVER_STATUS_STACK_OVERFLOW;
      }
      if (PACKET) __syncwarp();
      node = c0;
    } else if (g0 || g1) {
      node = g0 ? c0 : c1;
    } else {
      if (sp == 0) break;
      --sp;
      node = stack[sp * stride];
    }
  }
  return n_mem;
}

// Which scene a packet traces, and the per-launch constants.
struct SceneRef {
  const Node* nodes;
  const Record* recs;
  const float* features;
  const int32_t* order;  // Morton position -> original index
  int64_t N;
  int K;
};

struct TraceCtx {
  float tmin, tmax;
  int max_iters;
  EverForwardOut out;
  bool frustum;        // packet kernels: run the frustum phase before the rounds
  int depth;           // traversal stack entries in use (<= kStackDepth)
  const float* depth_hint;  // (R) nullable: per-ray guess of the stopping t
};

// One event of a ray's sorted sequence, integrated under the reference's round rules
// (shaders.slang:197-227): an event tied with the 16th event of a reference round is
// dropped, an exit beyond tmax counts only inside the round that consumed its entry, a
// t > 1e9 sentinel ends the ray. Returns true once the ray is finished.
template <int DEG>
__device__ __forceinline__ bool consume_event(const SceneRef& sc, const TraceCtx& C, const Ray& ray, const float* B,
                                              int bs, int64_t slot, uint64_t k, State& s, float4& last_dirac,
                                              int& iters, float& s16, int& cnt16, uint32_t& status) {
  const float t = key_t(k);
  const int j = key_pos(k);
  const int ex = key_exit(k);
  if (!(t > s16)) return false;  // tied with the 16th event of a reference round: dropped
  if (t > kSentinel) return true;
  const float4 r3 = __ldg(&sc.recs[j].r3);
  if (ex && t > C.tmax) {
    HitT H;
    intersect(load_record(sc.recs, j), ray, H);
    if (!(H.t0 > s16 && H.t0 <= C.tmax)) return false;
  }
  const float3 c = DEG == 0 ? dc_colour(r3) : sh_colour<DEG>(sc.features + int64_t(j) * feat_stride(sc.K), B, bs);
  const float dh = ex ? -r3.x : r3.x;
  const float4 dirac = make_float4(dh, dh * c.x, dh * c.y, dh * c.z);
  update(s, t, dirac);
  last_dirac = dirac;
  if (C.out.event_log) {
    if (iters < C.out.log_cap)
      C.out.event_log[slot * int64_t(C.out.log_cap) + iters] = 2 * j + (ex ? 0 : 1);
    else
      status |= EVER_STATUS_LOG_OVERFLOW;
  }
  if (C.out.touch_count) atomicAdd(C.out.touch_count + __ldg(sc.order + j), 1);
  ++iters;
  if (++cnt16 == kRefRound) {
    s16 = t;
    cnt16 = 0;
  }
  return !(s.logT < kLogCutoff && iters < C.max_iters);
}

// Integrates the gathered events in order. Returns true once the ray is finished.
template <int KBUF, int DEG>
__device__ __forceinline__ bool consume(const SceneRef& sc, const TraceCtx& C, const Ray& ray, const float* B,
                                        int bs, int64_t slot, uint64_t (&buf)[KBUF], State& s, float4& last_dirac,
                                        int& iters, float& s16, int& cnt16, uint64_t& lower, uint32_t& status) {
  const uint64_t last = buf[KBUF - 1];
  bool done = false;
  for (int n = 0; n < KBUF && !done; ++n) {
    const uint64_t k = buf[0];
#pragma unroll
    for (int i = 0; i < KBUF - 1; ++i) buf[i] = buf[i + 1];
    buf[KBUF - 1] = kEmptyKey;
    if (k == kEmptyKey) return true;  // nothing left beyond the last gathered event
    done = consume_event<DEG>(sc, C, ray, B, bs, slot, k, s, last_dirac, iters, s16, cnt16, status);
  }
  if (done || last == kEmptyKey) return true;
  lower = last;
  return false;
}

template <int DEG>
__device__ __forceinline__ void init_density(const SceneRef& sc, const float* B, int bs, int n_mem,
                                             const int (&mem_j)[kMaxMembers], float4 extra, uint32_t status,
                                             State& s) {
  const int fst = feat_stride(sc.K);
  for (int q = 0; q < n_mem; ++q) {
    const int j = mem_j[q];
    const float4 r3 = __ldg(&sc.recs[j].r3);
    const float sg = r3.x;
    const float3 c = DEG == 0 ? dc_colour(r3) : sh_colour<DEG>(sc.features + int64_t(j) * fst, B, bs);
    s.drgb.x = s.drgb.x + sg;
    s.drgb.y = s.drgb.y + sg * c.x;
    s.drgb.z = s.drgb.z + sg * c.y;
    s.drgb.w = s.drgb.w + sg * c.z;
  }
  if (status & EVER_STATUS_INIT_OVERFLOW) {
    s.drgb.x = s.drgb.x + extra.x;
    s.drgb.y = s.drgb.y + extra.y;
    s.drgb.z = s.drgb.z + extra.z;
    s.drgb.w = s.drgb.w + extra.w;
  }
}

__device__ __forceinline__ void write_outputs(const EverForwardOut& out, int64_t r, const State& s, float4 last_dirac,
                                              int iters, uint32_t status) {
  float* o = out.out + 5 * r;
  o[0] = s.C.x;
  o[1] = s.C.y;
  o[2] = s.C.z;
  o[3] = 1.f - expf(-s.logT);
  o[4] = s.dist_x - s.dist_y;
  if (out.states) {
    float4* st = reinterpret_cast<float4*>(out.states + 16 * r);
    st[0] = make_float4(s.dist_x, s.dist_y, s.cum_x, s.cum_y);
    st[1] = make_float4(0.f, 0.f, 0.f, s.t);
    st[2] = s.drgb;
    st[3] = make_float4(s.logT, s.C.x, s.C.y, s.C.z);
  }
  if (out.last_dirac) reinterpret_cast<float4*>(out.last_dirac)[r] = last_dirac;
  out.iters[r] = iters;
  if (out.ray_stats) {
    out.ray_stats[2 * r] = float(iters);
    out.ray_stats[2 * r + 1] = s.t;
  }
  if (status && out.status) atomicOr(out.status, int(status));
}

__device__ __forceinline__ Ray load_ray(const float* rayo, const float* rayd, int64_t r, float tmin) {
  const float3 ro = make_float3(rayo[3 * r], rayo[3 * r + 1], rayo[3 * r + 2]);
  const float3 rd = make_float3(rayd[3 * r], rayd[3 * r + 1], rayd[3 * r + 2]);
  return make_ray(ro, rd, tmin);
}

__device__ __forceinline__ SceneRef scene_of(const FwdParams& P) {
  return SceneRef{reinterpret_cast<const Node*>(P.nodes), reinterpret_cast<const Record*>(P.records), P.features,
                  P.order, P.N, P.K};
}

template <int KBUF, int DEG>
__global__ void __launch_bounds__(256) k_trace_fwd_ray(const FwdParams P) {
  extern __shared__ int smem[];
  const int tid = threadIdx.x, stride = blockDim.x;
  int* st_node = smem + tid;
  float* st_t = reinterpret_cast<float*>(smem + kStackDepth * stride) + tid;
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;
  if (gi >= P.R) return;
  const int64_t r = P.ray_order ? int64_t(P.ray_order[gi]) : gi;
  const SceneRef sc = scene_of(P);
  const TraceCtx C{P.tmin, P.tmax, P.max_iters, P.out, P.frustum != 0, P.stack_depth, P.depth_hint};
  const Ray ray = load_ray(P.rayo, P.rayd, r, P.tmin);
  const RaySlab sl = make_slab(ray);
  float B[16];
  sh_basis<DEG>(ray.rd, B);
  uint32_t status = 0;
  State s = empty_state();
  float4 last_dirac = make_float4(0.f, 0.f, 0.f, 0.f);
  int iters = 0;
  if (sc.N > 0) {
    int mem_p[kMaxMembers], mem_j[kMaxMembers];
    float4 extra = make_float4(0.f, 0.f, 0.f, 0.f);
    const int n_mem = point_members<DEG, false>(sc.nodes, sc.recs, sc.order, sc.features, feat_stride(sc.K), B, 1,
                                                ray, true,
                                                st_node, stride, C.depth, 0, mem_p, mem_j, extra, status);
    init_density<DEG>(sc, B, 1, n_mem, mem_j, extra, status, s);
    float s16 = 0.f;
    int cnt16 = 0;
    uint64_t lower = 0;
    bool done = C.max_iters <= 0;
    while (!done) {
      uint64_t buf[KBUF];
#pragma unroll
      for (int i = 0; i < KBUF; ++i) buf[i] = kEmptyKey;
      gather_ray<KBUF>(sc.nodes, sc.recs, ray, sl, lower, s16, C.tmax, buf, st_node, st_t, stride, C.depth,
                       status);
      done = consume<KBUF, DEG>(sc, C, ray, B, 1, gi, buf, s, last_dirac, iters, s16, cnt16, lower, status);
    }
  }
  write_outputs(C.out, r, s, last_dirac, iters, status);
}

// The SH basis of the ray's direction into the block's shared array (B[k * bs]).
template <int DEG>
__device__ __forceinline__ void store_basis(const Ray& ray, float* B, int bs) {
  float Bl[16];
  sh_basis<DEG>(ray.rd, Bl);
#pragma unroll
  for (int k = 0; k < (DEG + 1) * (DEG + 1); ++k) B[k * bs] = Bl[k];
}

// What a ray carries from one gather round to the next. cnt16 is not kept: it always equals
// iters % kRefRound (both count the consumed events from zero).
struct RayLoop {
  State s;
  float4 last_dirac;
  int iters;
  float s16;
  int cnt16;
  uint64_t lower;
  uint32_t status;
};

// Initial state of a ray: empty, plus the density of the ellipsoids its start lies in.
template <int DEG>
__device__ __forceinline__ RayLoop start_ray(const SceneRef& sc, const Ray& ray, bool valid, int* wstack, int depth,
                                             float* B,
                                             int bs, int lane) {
  RayLoop L;
  L.status = 0;
  L.s = empty_state();
  L.last_dirac = make_float4(0.f, 0.f, 0.f, 0.f);
  L.iters = 0;
  L.s16 = 0.f;
  L.cnt16 = 0;
  L.lower = 0;
  if (sc.N > 0) {
    int mem_p[kMaxMembers], mem_j[kMaxMembers];
    float4 extra = make_float4(0.f, 0.f, 0.f, 0.f);
    const int n_mem = point_members<DEG, true>(sc.nodes, sc.recs, sc.order, sc.features, feat_stride(sc.K), B, bs,
                                               ray, valid,
                                               wstack, 1, depth, lane, mem_p, mem_j, extra, L.status);
    init_density<DEG>(sc, B, bs, n_mem, mem_j, extra, L.status, L.s);
  }
  return L;
}

// Gather + consume rounds of a warp's packet until no lane is active or max_rounds rounds
// have run. Returns whether this lane's ray needs another round.
template <int KBUF, int DEG>
__device__ __forceinline__ bool run_rounds(const SceneRef& sc, const TraceCtx& C, const Ray& ray, const float* B, int bs,
                                           int64_t slot, int* wstack, int lane, bool act, RayLoop& L, int max_rounds) {
  const RaySlab sl = make_slab(ray);
  for (int round = 0; round < max_rounds && __any_sync(kFull, act); ++round) {
    uint64_t buf[KBUF];
#pragma unroll
    for (int i = 0; i < KBUF; ++i) buf[i] = kEmptyKey;
    gather_packet<KBUF>(sc.nodes, sc.recs, ray, sl, act, L.lower, L.s16, C.tmax, buf, wstack, lane, C.depth,
                        L.status);
    if (act)
      act = !consume<KBUF, DEG>(sc, C, ray, B, bs, slot, buf, L.s, L.last_dirac, L.iters, L.s16, L.cnt16, L.lower,
                                L.status);
  }
  return act;
}

// ---- packet frustum phase ----
// The warp bounds its active rays by intervals (origins, directions, inverse directions),
// walks the BVH breadth first with one node per lane, keeping every child box some packet
// ray can meet (a conservative interval slab test), and lists the leaves sorted by the
// earliest t at which any packet ray can enter them. Every lane then takes the leaves in
// that order: the leaf's events on its own ray go into its sorted buffer, and before the
// next leaf, whose events all lie at or beyond that leaf's entry bound T, the events
// below T are final and are integrated in order. So each ray integrates exactly its
// sorted event sequence, as the rounds do, with one walk per packet instead of one per
// round, and the box tests spread over the lanes instead of repeating for every ray.
// A lane whose buffer would overflow, and every lane of a packet whose breadth-first
// lists overflow shared memory, stops after its last integrated event; the rounds then
// continue it from there (lower = that event's key), so the results do not depend on it.
// Events a lane holds in the frustum phase. Fewer than the rounds' buffer: the phase's
// buffer lives across the whole leaf loop, and 12 of 16 gave the shortest forward at 1M
// ellipsoids / 1080p (5.90 ms; 16: 6.22, 8: 6.85, 24: 7.13 ms with spills).
constexpr int frustum_buffer(int kbuf) { return kbuf == 16 ? 12 : kbuf; }
constexpr int kFrontierCap = 384;  // nodes per breadth-first level
constexpr int kCandCap = 512;      // leaves per packet (a power of two: the sort's width)
// Shared ints per warp: the traversal stack, two frontier levels, the leaf keys (64-bit).
constexpr int kWarpInts = kStackDepth + 2 * kFrontierCap + 2 * kCandCap;

__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}
__device__ __forceinline__ float warp_min(float v) { return from_ordered(__reduce_min_sync(kFull, ordered_bits(v))); }
__device__ __forceinline__ float warp_max(float v) { return from_ordered(__reduce_max_sync(kFull, ordered_bits(v))); }

struct PacketBounds {
  float omin[3], omax[3];  // origins
  float imin[3], imax[3];  // inverse directions (as the per-ray slab test takes them)
  float dmin[3], dmax[3];  // unit directions
  unsigned free_axes;      // axes whose direction changes sign within the packet
};

// Interval bounds over the lanes with `part` (all lanes take part in the reductions).
__device__ __forceinline__ PacketBounds packet_bounds(const Ray& ray, const RaySlab& sl, bool part) {
  PacketBounds P;
  const float o[3] = {ray.o.x, ray.o.y, ray.o.z}, d[3] = {ray.d.x, ray.d.y, ray.d.z};
  const float iv[3] = {sl.invd.x, sl.invd.y, sl.invd.z};
  P.free_axes = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    P.omin[a] = warp_min(part ? o[a] : INFINITY);
    P.omax[a] = warp_max(part ? o[a] : -INFINITY);
    P.imin[a] = warp_min(part ? iv[a] : INFINITY);
    P.imax[a] = warp_max(part ? iv[a] : -INFINITY);
    P.dmin[a] = warp_min(part ? d[a] : INFINITY);
    P.dmax[a] = warp_max(part ? d[a] : -INFINITY);
    if (P.imin[a] < 0.f && P.imax[a] > 0.f) P.free_axes |= 1u << a;
  }
  return P;
}

__device__ __forceinline__ float min4(float a, float b, float c, float d) { return fminf(fminf(a, b), fminf(c, d)); }
__device__ __forceinline__ float max4(float a, float b, float c, float d) { return fmaxf(fmaxf(a, b), fmaxf(c, d)); }

// A lower bound of the t at which any packet ray enters the box within [0, cap], or +inf
// when no packet ray can meet it there. Interval products bound every ray's plane
// distances; the float rounding of the bound (a few ulps) is covered by widening it by a
// relative 1e-6. Axes whose direction changes sign bound no t: there the positions the
// packet reaches over the t range of the other axes must overlap the box.
__device__ __forceinline__ float packet_entry(const PacketBounds& P, float lx, float ly, float lz, float hx, float hy,
                                              float hz, float cap) {
  const float lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz};
  float tn = 0.f, tf = cap;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (P.free_axes >> a & 1u) continue;
    const float d0 = lo[a] - P.omax[a], d1 = lo[a] - P.omin[a];
    const float e0 = hi[a] - P.omax[a], e1 = hi[a] - P.omin[a];
    const float p0 = d0 * P.imin[a], p1 = d0 * P.imax[a], p2 = d1 * P.imin[a], p3 = d1 * P.imax[a];
    const float q0 = e0 * P.imin[a], q1 = e0 * P.imax[a], q2 = e1 * P.imin[a], q3 = e1 * P.imax[a];
    tn = fmaxf(tn, fminf(min4(p0, p1, p2, p3), min4(q0, q1, q2, q3)));
    tf = fminf(tf, fmaxf(max4(p0, p1, p2, p3), max4(q0, q1, q2, q3)));
  }
  tn = tn - 1e-6f * fabsf(tn);
  tf = tf + 1e-6f * fabsf(tf);
  if (!(tn <= tf)) return INFINITY;
  if (P.free_axes) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (!(P.free_axes >> a & 1u)) continue;
      const float xl = P.omin[a] + min4(tn * P.dmin[a], tn * P.dmax[a], tf * P.dmin[a], tf * P.dmax[a]);
      const float xh = P.omax[a] + max4(tn * P.dmin[a], tn * P.dmax[a], tf * P.dmin[a], tf * P.dmax[a]);
      const float tol = 1e-6f * (fabsf(xl) + fabsf(xh) + fabsf(tf));
      if (xh + tol < lo[a] || xl - tol > hi[a]) return INFINITY;
    }
  }
  return fmaxf(tn, 0.f);
}

// Breadth-first walk: the leaf keys (entry bound bits << 32 | position) of every leaf the
// packet can meet, into cand[0, n). Returns n, or -1 when a level or the leaf list does
// not fit its shared-memory capacity.
__device__ __forceinline__ int packet_leaves(const Node* __restrict__ nodes, const PacketBounds& P, float cap,
                                             int* front, uint64_t* cand, int lane) {
  int* cur = front;
  int* nxt = front + kFrontierCap;
  if (lane == 0) cur[0] = 0;
  __syncwarp();
  int nf = 1, nc = 0;
  const unsigned below = (1u << lane) - 1u;
  for (int level = 0; nf > 0; ++level) {
    if (level >= 4 * kStackDepth) return -1;  // deeper than any tree the build makes
    int nn = 0;
    for (int base = 0; base < nf; base += 32) {
      const int i = base + lane;
      float te0 = INFINITY, te1 = INFINITY;
      int c0 = 0, c1 = 0;
      if (i < nf) {
        const Node nd = load_node(nodes, cur[i]);
        te0 = packet_entry(P, nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, cap);
        te1 = packet_entry(P, nd.b.z, nd.b.w, nd.c.x, nd.c.y, nd.c.z, nd.c.w, cap);
        c0 = nd.d.x;
        c1 = nd.d.y;
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const float te = k ? te1 : te0;
        const int c = k ? c1 : c0;
        const bool hit = te != INFINITY;
        const unsigned mi = __ballot_sync(kFull, hit && c >= 0);
        const unsigned ml = __ballot_sync(kFull, hit && c < 0);
        if (hit && c >= 0) {
          const int q = nn + __popc(mi & below);
          if (q < kFrontierCap) nxt[q] = c;
        }
        if (hit && c < 0) {
          const int q = nc + __popc(ml & below);
          if (q < kCandCap) cand[q] = (uint64_t(__float_as_uint(te)) << 32) | uint32_t(~c);
        }
        nn += __popc(mi);
        nc += __popc(ml);
      }
    }
    __syncwarp();
    if (nn > kFrontierCap || nc > kCandCap) return -1;
    int* t = cur;
    cur = nxt;
    nxt = t;
    nf = nn;
  }
  return nc;
}

// Ascending bitonic sort of cand[0, n) in shared memory by the warp (n <= kCandCap).
__device__ __forceinline__ void sort_keys_smem(uint64_t* cand, int n, int lane) {
  int w = 32;
  while (w < n) w <<= 1;
  for (int i = n + lane; i < w; i += 32) cand[i] = kEmptyKey;
  __syncwarp();
  for (int k = 2; k <= w; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < w; i += 32) {
        const int l = i ^ j;
        if (l > i) {
          const uint64_t a = cand[i], b = cand[l];
          if ((a > b) == ((i & k) == 0)) {
            cand[i] = b;
            cand[l] = a;
          }
        }
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
  const uint32_t lo = __shfl_xor_sync(kFull, uint32_t(v), m), hi = __shfl_xor_sync(kFull, uint32_t(v >> 32), m);
  return (uint64_t(hi) << 32) | lo;
}

// Ascending bitonic sort of 32 * E keys held E per lane (key lane * E + r in k[r]): the
// stages whose partners lie in the same lane compare-swap registers, the others exchange
// with lane ^ (stride / E) by shuffles. No shared memory, no warp barriers.
template <int E>
__device__ __forceinline__ void sort_regs(uint64_t (&k)[E], int lane) {
#pragma unroll
  for (int size = 2; size <= 32 * E; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride < E) {
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const int q = r ^ stride;
          if (q > r) {
            const bool up = ((lane * E + r) & size) == 0;
            const uint64_t a = k[r], b = k[q];
            const bool sw = (a > b) == up;
            k[r] = sw ? b : a;
            k[q] = sw ? a : b;
          }
        }
      } else {
        const int m = stride / E;
        const bool lower = (lane & m) == 0;
#pragma unroll
        for (int r = 0; r < E; ++r) {
          const uint64_t o = shfl_xor64(k[r], m);
          const bool up = ((lane * E + r) & size) == 0;
          const bool take_min = lower == up;
          k[r] = take_min ? (o < k[r] ? o : k[r]) : (o > k[r] ? o : k[r]);
        }
      }
    }
  }
}

// Sorts cand[0, n) ascending (n <= 32 * E) through registers.
template <int E>
__device__ __forceinline__ void sort_keys_r(uint64_t* cand, int n, int lane) {
  uint64_t k[E];
#pragma unroll
  for (int r = 0; r < E; ++r) {
    const int i = lane * E + r;
    k[r] = i < n ? cand[i] : kEmptyKey;
  }
  sort_regs<E>(k, lane);
  __syncwarp();
#pragma unroll
  for (int r = 0; r < E; ++r) cand[lane * E + r] = k[r];
  __syncwarp();
}
// Up to 256 keys sort in registers; longer lists in shared memory.
__device__ __forceinline__ void sort_keys(uint64_t* cand, int n, int lane) {
  if (n <= 32 * 4) sort_keys_r<4>(cand, n, lane);
  else if (n <= 32 * 8) sort_keys_r<8>(cand, n, lane);
  else sort_keys_smem(cand, n, lane);
}

// The frustum phase of a warp's packet. Returns whether this lane's ray still needs rounds
// (L then holds its state after its last integrated event, L.lower that event's key).
template <int KBUF, int DEG>
__device__ __forceinline__ bool frustum_phase(const SceneRef& sc, const TraceCtx& C, const Ray& ray, const float* B,
                                              int bs, int64_t slot, int64_t r, int* wsm, int lane, bool act,
                                              RayLoop& L) {
  constexpr int FBUF = frustum_buffer(KBUF);
  if (!__any_sync(kFull, act)) return act;
  const RaySlab sl = make_slab(ray);
  float cap = fminf(C.tmax, kSentinel);
  // With a depth hint the walk covers t up to the packet's largest guessed stopping t (plus
  // 5%): events up to there are integrated here, the rounds continue any ray that goes on.
  // A poor guess costs time, never correctness.
  float t_final = INFINITY;
  if (C.depth_hint) {
    const float h = warp_max(act ? C.depth_hint[r] : -INFINITY);
    if (h > 0.f && 1.05f * h + 1e-3f < cap) cap = t_final = 1.05f * h + 1e-3f;
  }
  const PacketBounds P = packet_bounds(ray, sl, act);
  int* front = wsm + kStackDepth;
  uint64_t* cand = reinterpret_cast<uint64_t*>(front + 2 * kFrontierCap);
  const int nc = packet_leaves(sc.nodes, P, cap, front, cand, lane);
  if (nc < 0) return act;  // lists too long for shared memory: the rounds trace the packet
  sort_keys(cand, nc, lane);
  uint64_t buf[FBUF];
#pragma unroll
  for (int i = 0; i < FBUF; ++i) buf[i] = kEmptyKey;
  bool live = act;  // still integrating in this phase
  for (int ci = 0;; ++ci) {
    // every 32 leaves, the lanes start the loads of the next 32 records into L1 (one each),
    // so the broadcast record loads of the loop below rarely wait on L2
    if ((ci & 31) == 0 && ci + lane < nc)
      asm volatile("prefetch.global.L1 [%0];" ::"l"(sc.recs + int(uint32_t(cand[ci + lane]))));
    const uint64_t ck = ci < nc ? cand[ci] : kEmptyKey;
    const float T = ci < nc ? key_t(ck) : t_final;
    // events below T are final: no leaf still to come has an event before T
    while (live && buf[0] != kEmptyKey && key_t(buf[0]) < T) {
      const uint64_t k = buf[0];
#pragma unroll
      for (int i = 0; i < FBUF - 1; ++i) buf[i] = buf[i + 1];
      buf[FBUF - 1] = kEmptyKey;
      L.lower = k;
      if (consume_event<DEG>(sc, C, ray, B, bs, slot, k, L.s, L.last_dirac, L.iters, L.s16, L.cnt16, L.status)) {
        live = false;
        act = false;  // finished
      }
    }
    if (ci >= nc) break;
    if (!__any_sync(kFull, live)) break;
    if (live) {
      const int j = int(uint32_t(ck));
      const Record R = load_record(sc.recs, j);
      HitT H;
      if (intersect(R, ray, H)) {
        const bool in0 = H.t0 > L.s16 && H.t0 <= C.tmax;
        const bool in1 = H.t1 > L.s16 && (H.t1 <= C.tmax || in0);
        // a full buffer cannot take another event: stop here, the rounds continue the ray
        if ((in0 || in1) && buf[FBUF - (in0 && in1 ? 2 : 1)] != kEmptyKey) {
          live = false;
        } else {
          if (in0) buf_insert(buf, event_key(H.t0, j, 0));
          if (in1) buf_insert(buf, event_key(H.t1, j, 1));
        }
      }
    }
  }
  // all leaves taken and every event integrated: nothing is left on a lane still active,
  // unless the walk stopped short of the scene (depth hint)
  if (live && t_final == INFINITY) act = false;
  return act;
}

// One warp traces one packet of up to 32 rays against one scene (lanes with valid=false
// only take part in the warp-wide votes).
template <int KBUF, int DEG>
__device__ __forceinline__ void trace_packet(const SceneRef& sc, const TraceCtx& C, const Ray& ray, int64_t r,
                                             bool valid, int64_t slot, int* wstack, float* B, int bs, int lane) {
  store_basis<DEG>(ray, B, bs);
  RayLoop L = start_ray<DEG>(sc, ray, valid, wstack, C.depth, B, bs, lane);
  bool act = valid && C.max_iters > 0 && sc.N > 0;
  if (C.frustum) act = frustum_phase<KBUF, DEG>(sc, C, ray, B, bs, slot, r, wstack, lane, act, L);
  run_rounds<KBUF, DEG>(sc, C, ray, B, bs, slot, wstack, lane, act, L, INT_MAX);
  if (valid) write_outputs(C.out, r, L.s, L.last_dirac, L.iters, L.status);
  __syncwarp();
}

// A ray that needs more rounds parks its loop state in its own output rows: `states` in
// the final layout, with s16 and the 64-bit key bound of the next round in the three
// padding words, `last_dirac` and `iters`. Its status flags are raised now.
__device__ __forceinline__ void park_ray(const EverForwardOut& out, int64_t r, const RayLoop& L) {
  float4* st = reinterpret_cast<float4*>(out.states + 16 * r);
  st[0] = make_float4(L.s.dist_x, L.s.dist_y, L.s.cum_x, L.s.cum_y);
  st[1] = make_float4(L.s16, __uint_as_float(uint32_t(L.lower)), __uint_as_float(uint32_t(L.lower >> 32)), L.s.t);
  st[2] = L.s.drgb;
  st[3] = make_float4(L.s.logT, L.s.C.x, L.s.C.y, L.s.C.z);
  reinterpret_cast<float4*>(out.last_dirac)[r] = L.last_dirac;
  out.iters[r] = L.iters;
  if (L.status && out.status) atomicOr(out.status, int(L.status));
}

__device__ __forceinline__ RayLoop resume_ray(const EverForwardOut& out, int64_t r) {
  const float4* st = reinterpret_cast<const float4*>(out.states + 16 * r);
  const float4 a = st[0], b = st[1], c = st[2], d = st[3];
  RayLoop L;
  L.s.dist_x = a.x;
  L.s.dist_y = a.y;
  L.s.cum_x = a.z;
  L.s.cum_y = a.w;
  L.s.t = b.w;
  L.s.drgb = c;
  L.s.logT = d.x;
  L.s.C = make_float3(d.y, d.z, d.w);
  L.s16 = b.x;
  L.lower = uint64_t(__float_as_uint(b.y)) | (uint64_t(__float_as_uint(b.z)) << 32);
  L.last_dirac = reinterpret_cast<const float4*>(out.last_dirac)[r];
  L.iters = out.iters[r];
  L.cnt16 = L.iters % kRefRound;
  L.status = 0;
  return L;
}

// Resident blocks per SM that the register budget of the packet kernels targets: 20
// warps per SM for blocks of 64 and 128 threads (96 registers; the traversal is
// latency-bound, so the extra warps pay for a few spilled bytes), 16 for 256 threads.
template <int BLOCK>
struct FwdMinBlocks {
  static constexpr int value = BLOCK == 256 ? 2 : 640 / BLOCK;
};

template <int KBUF, int DEG, int BLOCK>
__global__ void __launch_bounds__(BLOCK, FwdMinBlocks<BLOCK>::value) k_trace_fwd_packet(const FwdParams P) {
  extern __shared__ int smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int* wstack = smem + warp * kWarpInts;  // stack, then the frustum phase's lists
  float* B = reinterpret_cast<float*>(smem + (blockDim.x / 32) * kWarpInts) + tid;  // B[k * blockDim.x]
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;
  const bool valid = gi < P.R;  // every lane stays for the warp-wide ballots
  const int64_t r = valid ? (P.ray_order ? int64_t(P.ray_order[gi]) : gi) : 0;
  const TraceCtx C{P.tmin, P.tmax, P.max_iters, P.out, P.frustum != 0, P.stack_depth, P.depth_hint};
  const Ray ray = load_ray(P.rayo, P.rayd, r, P.tmin);
  trace_packet<KBUF, DEG>(scene_of(P), C, ray, r, valid, gi, wstack, B, blockDim.x, lane);
}

// Regrouped forward, one pass. PASS 0 takes every slot in order and runs the first gather
// round; PASS 1 runs one more round and PASS 2 every remaining round, each for the slots in
// `list` (count entries): the rays that the previous pass left active, packed into full
// warps in slot order. A pass 0 or 1 with fewer than `split_min` rays runs every remaining
// round instead (a later pass would hold too few rays to fill the GPU, and its latency-bound
// tail would run alone). Passes 0 and 1 park the rays that still need rounds and write one
// lane mask per warp (mask[position / 32]); the other rays write their outputs.
// Camera passes (CAM): slots are the camera's (camera.cuh); a slot's pixel ray is made in
// the kernel, padding slots take part only in the warp votes, and the event log has one
// column per slot.
struct PassCamera {
  CameraParams cam;
  const float* jitter;
  int64_t num_slots;
};

template <int KBUF, int DEG, int BLOCK, int PASS, bool CAM>
__global__ void __launch_bounds__(BLOCK, FwdMinBlocks<BLOCK>::value)
    k_trace_fwd_pass(const FwdParams P, const int32_t* __restrict__ list, const uint32_t* __restrict__ count,
                     uint32_t* __restrict__ mask, int64_t split_min, const PassCamera Q) {
  extern __shared__ int smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int* wstack = smem + warp * kWarpInts;  // stack, then the frustum phase's lists
  float* B = reinterpret_cast<float*>(smem + (blockDim.x / 32) * kWarpInts) + tid;
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;  // slot (PASS 0) or list position
  const int64_t slots = CAM ? Q.num_slots : P.R;
  const int64_t n = PASS == 0 ? slots : int64_t(*count);
  if ((gi & ~int64_t(31)) >= n) return;  // the whole warp lies beyond the list
  const int64_t slot = gi < n ? (PASS == 0 ? gi : int64_t(list[gi])) : 0;
  int64_t r = 0;
  bool valid = gi < n;
  if (CAM) {
    r = valid ? camera_slot_pixel(Q.cam, slot) : -1;
    valid = r >= 0;
  } else if (valid) {
    r = P.ray_order ? int64_t(P.ray_order[slot]) : slot;
  }
  if (!valid) r = 0;
  const SceneRef sc = scene_of(P);
  const TraceCtx C{P.tmin, P.tmax, P.max_iters, P.out, P.frustum != 0, P.stack_depth, P.depth_hint};
  Ray ray;
  if (CAM) {
    float3 ro, rd;
    camera_ray(Q.cam, Q.jitter, r, ro, rd);
    ray = make_ray(ro, rd, P.tmin);
  } else {
    ray = load_ray(P.rayo, P.rayd, r, P.tmin);
  }
  store_basis<DEG>(ray, B, blockDim.x);
  RayLoop L;
  bool act;
  if (PASS == 0) {
    L = start_ray<DEG>(sc, ray, valid, wstack, C.depth, B, blockDim.x, lane);
    act = valid && C.max_iters > 0 && sc.N > 0;
    if (C.frustum) act = frustum_phase<KBUF, DEG>(sc, C, ray, B, blockDim.x, slot, r, wstack, lane, act, L);
  } else {
    if (valid) L = resume_ray(P.out, r);
    act = valid;
  }
  const bool last = PASS == 2 || n < split_min;
  // after the frustum phase, pass 0 hands its few unfinished rays on without a round
  const int rounds = last ? INT_MAX : (PASS == 0 && C.frustum ? 0 : 1);
  act = run_rounds<KBUF, DEG>(sc, C, ray, B, blockDim.x, slot, wstack, lane, act, L, rounds);
  if (PASS < 2) {
    const unsigned m = __ballot_sync(kFull, act);
    if (lane == 0) mask[gi >> 5] = m;
  }
  if (valid) {
    if (PASS < 2 && act)
      park_ray(P.out, r, L);
    else
      write_outputs(C.out, r, L.s, L.last_dirac, L.iters, L.status);
  }
}

// Camera trace: rays are made from the camera in the kernel (no ray arrays). The launch
// covers the camera's slots, 32 per 8x4 pixel tile, so a warp traces one tile; outputs are
// written by pixel, event-log columns are slots.
template <int KBUF, int DEG, int BLOCK>
__global__ void __launch_bounds__(BLOCK, FwdMinBlocks<BLOCK>::value)
    k_trace_fwd_camera(const FwdParams P, const CameraParams cam, const float* __restrict__ jitter,
                       int64_t num_slots) {
  extern __shared__ int smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int* wstack = smem + warp * kWarpInts;  // stack, then the frustum phase's lists
  float* B = reinterpret_cast<float*>(smem + (blockDim.x / 32) * kWarpInts) + tid;
  const int64_t gi = int64_t(blockIdx.x) * blockDim.x + tid;
  const int64_t p = gi < num_slots ? camera_slot_pixel(cam, gi) : -1;
  const bool valid = p >= 0;
  const TraceCtx C{P.tmin, P.tmax, P.max_iters, P.out, P.frustum != 0, P.stack_depth, P.depth_hint};
  float3 ro, rd;
  camera_ray(cam, jitter, valid ? p : 0, ro, rd);
  const Ray ray = make_ray(ro, rd, P.tmin);
  trace_packet<KBUF, DEG>(scene_of(P), C, ray, valid ? p : 0, valid, gi, wstack, B, blockDim.x, lane);
}

// Persistent batched forward: warps take 32-slot packets from a device counter until
// all views are done. Each packet lies inside one view, hence one scene.
template <int KBUF, int DEG, int BLOCK>
__global__ void __launch_bounds__(BLOCK, FwdMinBlocks<BLOCK>::value) k_trace_fwd_batched(const BatchFwdParams P) {
  extern __shared__ int smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int* wstack = smem + warp * kWarpInts;  // stack, then the frustum phase's lists
  float* B = reinterpret_cast<float*>(smem + (blockDim.x / 32) * kWarpInts) + tid;
  const TraceCtx C{P.tmin, P.tmax, P.max_iters, P.out, P.frustum != 0, P.stack_depth, nullptr};
  const int64_t num_packets = P.num_slots / 32;
  for (;;) {
    unsigned int pk = 0;
    if (lane == 0) pk = atomicAdd(P.work_counter, 1u);
    pk = __shfl_sync(kFull, pk, 0);
    if (int64_t(pk) >= num_packets) break;
    const int64_t slot = int64_t(pk) * 32 + lane;
    int v = 0;  // the view holding this packet (few views: linear scan, warp-uniform)
    while (v + 1 < P.num_views && P.views[v + 1].slot_offset <= int64_t(pk) * 32) ++v;
    const BatchScene bs_ = P.scenes[P.views[v].scene];
    const SceneRef sc{reinterpret_cast<const Node*>(bs_.nodes), reinterpret_cast<const Record*>(bs_.records),
                      bs_.features, bs_.order, bs_.N, bs_.K};
    const int32_t r = P.slot_ray[slot];
    const Ray ray = load_ray(P.rayo, P.rayd, r >= 0 ? r : 0, P.tmin);
    trace_packet<KBUF, DEG>(sc, C, ray, r, r >= 0, slot, wstack, B, blockDim.x, lane);
  }
}

// Dynamic shared memory of a packet kernel: per warp its stack and frustum-phase lists,
// per thread the SH basis of its ray.
template <int DEG>
size_t packet_smem(int block) {
  return size_t(kWarpInts) * (block / 32) * sizeof(int) + size_t((DEG + 1) * (DEG + 1)) * block * sizeof(float);
}

// Dynamic shared memory above the 48 KB default needs the kernel's opt-in.
template <class Kern>
cudaError_t prepare(Kern kern, size_t smem) {
  if (smem <= size_t(48) * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
}

template <int KBUF, int DEG>
cudaError_t launch_t(const FwdParams& P, int block, int traversal, cudaStream_t st) {
  const int64_t grid = (P.R + block - 1) / block;
  if (traversal == 1) {
    const size_t smem = size_t(kStackDepth) * block * (sizeof(int) + sizeof(float));
    auto kern = k_trace_fwd_ray<KBUF, DEG>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    kern<<<unsigned(grid), block, smem, st>>>(P);
  } else {
    const size_t smem = packet_smem<DEG>(block);
    switch (block) {
      case 64: {
        if (cudaError_t e_ = prepare(k_trace_fwd_packet<KBUF, DEG, 64>, smem)) return e_;
        k_trace_fwd_packet<KBUF, DEG, 64><<<unsigned(grid), 64, smem, st>>>(P);
        break;
      }
      case 128: {
        if (cudaError_t e_ = prepare(k_trace_fwd_packet<KBUF, DEG, 128>, smem)) return e_;
        k_trace_fwd_packet<KBUF, DEG, 128><<<unsigned(grid), 128, smem, st>>>(P);
        break;
      }
      default: {
        if (cudaError_t e_ = prepare(k_trace_fwd_packet<KBUF, DEG, 256>, smem)) return e_;
        k_trace_fwd_packet<KBUF, DEG, 256><<<unsigned(grid), 256, smem, st>>>(P);
        break;
      }
    }
  }
  return cudaGetLastError();
}

template <int KBUF>
cudaError_t launch_k(const FwdParams& P, int deg, int block, int traversal, cudaStream_t st) {
  switch (deg) {
    case 0: return launch_t<KBUF, 0>(P, block, traversal, st);
    case 1: return launch_t<KBUF, 1>(P, block, traversal, st);
    case 2: return launch_t<KBUF, 2>(P, block, traversal, st);
    default: return launch_t<KBUF, 3>(P, block, traversal, st);
  }
}

template <int KBUF, int DEG, int BLOCK, bool CAM>
cudaError_t launch_regrouped_b(const FwdParams& P, const RegroupScratch& W, const PassCamera& Q, cudaStream_t st) {
  const int64_t n = CAM ? Q.num_slots : P.R;
  const unsigned grid = unsigned((n + BLOCK - 1) / BLOCK);
  const size_t smem = packet_smem<DEG>(BLOCK);
  if (cudaError_t e_ = prepare(k_trace_fwd_pass<KBUF, DEG, BLOCK, 0, CAM>, smem)) return e_;
  k_trace_fwd_pass<KBUF, DEG, BLOCK, 0, CAM><<<grid, BLOCK, smem, st>>>(P, nullptr, nullptr, W.mask0, W.split_min, Q);
  cudaError_t e = regroup_compact(W.mask0, nullptr, n, nullptr, W.offsets, W.list1, W.count1, st);
  if (e != cudaSuccess) return e;
  if (cudaError_t e_ = prepare(k_trace_fwd_pass<KBUF, DEG, BLOCK, 1, CAM>, smem)) return e_;
  k_trace_fwd_pass<KBUF, DEG, BLOCK, 1, CAM><<<grid, BLOCK, smem, st>>>(P, W.list1, W.count1, W.mask1, W.split_min, Q);
  e = regroup_compact(W.mask1, W.count1, n, W.list1, W.offsets, W.list2, W.count2, st);
  if (e != cudaSuccess) return e;
  if (cudaError_t e_ = prepare(k_trace_fwd_pass<KBUF, DEG, BLOCK, 2, CAM>, smem)) return e_;
  k_trace_fwd_pass<KBUF, DEG, BLOCK, 2, CAM><<<grid, BLOCK, smem, st>>>(P, W.list2, W.count2, nullptr, 0, Q);
  return cudaGetLastError();
}

template <int KBUF, int DEG, bool CAM>
cudaError_t launch_regrouped_t(const FwdParams& P, const RegroupScratch& W, const PassCamera& Q, int block,
                               cudaStream_t st) {
  switch (block) {
    case 64: return launch_regrouped_b<KBUF, DEG, 64, CAM>(P, W, Q, st);
    case 128: return launch_regrouped_b<KBUF, DEG, 128, CAM>(P, W, Q, st);
    default: return launch_regrouped_b<KBUF, DEG, 256, CAM>(P, W, Q, st);
  }
}

template <int KBUF, bool CAM>
cudaError_t launch_regrouped_c(const FwdParams& P, const RegroupScratch& W, const PassCamera& Q, int deg, int block,
                               cudaStream_t st) {
  switch (deg) {
    case 0: return launch_regrouped_t<KBUF, 0, CAM>(P, W, Q, block, st);
    case 1: return launch_regrouped_t<KBUF, 1, CAM>(P, W, Q, block, st);
    case 2: return launch_regrouped_t<KBUF, 2, CAM>(P, W, Q, block, st);
    default: return launch_regrouped_t<KBUF, 3, CAM>(P, W, Q, block, st);
  }
}

// cam: null for ray arrays, else the camera (its slots) and the per-pixel jitter
template <int KBUF>
cudaError_t launch_regrouped_k(const FwdParams& P, const RegroupScratch& W, const CameraParams* cam,
                               const float* jitter, int deg, int block, cudaStream_t st) {
  PassCamera Q{};
  if (!cam) return launch_regrouped_c<KBUF, false>(P, W, Q, deg, block, st);
  Q.cam = *cam;
  Q.jitter = jitter;
  Q.num_slots = camera_slots(*cam);
  return launch_regrouped_c<KBUF, true>(P, W, Q, deg, block, st);
}

template <int KBUF, int DEG>
cudaError_t launch_camera_t(const FwdParams& P, const CameraParams& cam, const float* jitter, int block,
                            cudaStream_t st) {
  const int64_t num_slots = camera_slots(cam);
  const unsigned grid = unsigned((num_slots + block - 1) / block);
  const size_t smem = packet_smem<DEG>(block);
  switch (block) {
    case 64: {
      if (cudaError_t e_ = prepare(k_trace_fwd_camera<KBUF, DEG, 64>, smem)) return e_;
      k_trace_fwd_camera<KBUF, DEG, 64><<<grid, 64, smem, st>>>(P, cam, jitter, num_slots);
      break;
    }
    case 128: {
      if (cudaError_t e_ = prepare(k_trace_fwd_camera<KBUF, DEG, 128>, smem)) return e_;
      k_trace_fwd_camera<KBUF, DEG, 128><<<grid, 128, smem, st>>>(P, cam, jitter, num_slots);
      break;
    }
    default: {
      if (cudaError_t e_ = prepare(k_trace_fwd_camera<KBUF, DEG, 256>, smem)) return e_;
      k_trace_fwd_camera<KBUF, DEG, 256><<<grid, 256, smem, st>>>(P, cam, jitter, num_slots);
      break;
    }
  }
  return cudaGetLastError();
}

template <int KBUF>
cudaError_t launch_camera_k(const FwdParams& P, const CameraParams& cam, const float* jitter, int deg, int block,
                            cudaStream_t st) {
  switch (deg) {
    case 0: return launch_camera_t<KBUF, 0>(P, cam, jitter, block, st);
    case 1: return launch_camera_t<KBUF, 1>(P, cam, jitter, block, st);
    case 2: return launch_camera_t<KBUF, 2>(P, cam, jitter, block, st);
    default: return launch_camera_t<KBUF, 3>(P, cam, jitter, block, st);
  }
}

template <int KBUF, int DEG>
cudaError_t launch_batched_t(const BatchFwdParams& P, int block, cudaStream_t st) {
  const size_t smem = packet_smem<DEG>(block);
  cudaError_t e = cudaMemsetAsync(P.work_counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  switch (block) {
    case 64: {
      if (cudaError_t e_ = prepare(k_trace_fwd_batched<KBUF, DEG, 64>, smem)) return e_;
      k_trace_fwd_batched<KBUF, DEG, 64><<<P.grid, 64, smem, st>>>(P);
      break;
    }
    case 128: {
      if (cudaError_t e_ = prepare(k_trace_fwd_batched<KBUF, DEG, 128>, smem)) return e_;
      k_trace_fwd_batched<KBUF, DEG, 128><<<P.grid, 128, smem, st>>>(P);
      break;
    }
    default: {
      if (cudaError_t e_ = prepare(k_trace_fwd_batched<KBUF, DEG, 256>, smem)) return e_;
      k_trace_fwd_batched<KBUF, DEG, 256><<<P.grid, 256, smem, st>>>(P);
      break;
    }
  }
  return cudaGetLastError();
}

template <int KBUF>
cudaError_t launch_batched_k(const BatchFwdParams& P, int deg, int block, cudaStream_t st) {
  switch (deg) {
    case 0: return launch_batched_t<KBUF, 0>(P, block, st);
    case 1: return launch_batched_t<KBUF, 1>(P, block, st);
    case 2: return launch_batched_t<KBUF, 2>(P, block, st);
    default: return launch_batched_t<KBUF, 3>(P, block, st);
  }
}

}  // namespace
}  // namespace ever
