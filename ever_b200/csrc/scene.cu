// Scene build: per-ellipsoid AABBs and intersection records, 30-bit Morton codes, an
// LSD radix sort, a Karras (2012) LBVH and a bottom-up refit of the child boxes.
//
// Replaces the reference's create_aabbs (splinetracers/fast_ellipsoid_splinetracer/
// create_aabbs.cu:69-132) and its OptiX GAS build (GAS.cpp:56-154). B200 has no RT
// cores, so the hierarchy is built here and traversed by our own kernels.
#include <cstdio>

#include <cuda/atomic>

#include "common.cuh"
#include "internal.cuh"

namespace ever {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ uint32_t float_to_ordered(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// W = diag(1/s) A(q) with A(q) e_j = rotate_vector(e_j, q): same operation order as the oracle.
__device__ __forceinline__ void prim_matrix(float4 q, float3 s, float W[9]) {
  const float sv[3] = {s.x, s.y, s.z};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float3 e = make_float3(j == 0 ? 1.f : 0.f, j == 1 ? 1.f : 0.f, j == 2 ? 1.f : 0.f);
    const float3 col = rotate_vector(e, q);
    W[0 * 3 + j] = col.x / sv[0];
    W[1 * 3 + j] = col.y / sv[1];
    W[2 * 3 + j] = col.z / sv[2];
  }
}

__device__ __forceinline__ float3 ld3(const float* p, int64_t i) {
  return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ float4 ld4(const float* p, int64_t i) {
  return make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
}

// Conservative AABB of {x : |W (x - mean)| <= 1}: half extent i = |row_i(W^-1)|, from the
// same float W the intersection uses. W^-1 = adj(W) / det(W) is evaluated in float next to
// a running bound of its rounding error (each 2x2 minor a*b - c*d is off by at most
// 2u(|ab| + |cd|), u = 2^-24; det by the first row's share of those plus its own sums), and
// the box is padded by that bound twice over, by 2e-3 of the extent (grazing roots in float
// move by ~sqrt(u) of the radius) and by 4e-7 of the magnitudes, then rounded outwards.
// Ill-conditioned W (det not known to 25%) gets an unbounded box. No double precision.
__global__ void k_aabbs(const float* __restrict__ mean, const float* __restrict__ scale,
                        const float* __restrict__ quat, int64_t N, float4* __restrict__ aabb,
                        uint32_t* __restrict__ bounds) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  float3 c = make_float3(0.f, 0.f, 0.f);
  bool valid = false;
  if (p < N) {
    float m[9];
    prim_matrix(ld4(quat, p), ld3(scale, p), m);
    const float3 mu = ld3(mean, p);
    constexpr float u = 5.9604645e-8f;  // 2^-24
    // adjugate (rows of the inverse times det) and the sums of |products| of each minor
    float adj[9], mag[9];
    auto minor = [](float a, float b, float cc, float d, float& v, float& g) {
      const float x = a * b, y = cc * d;
      v = x - y;
      g = fabsf(x) + fabsf(y);
    };
    minor(m[4], m[8], m[5], m[7], adj[0], mag[0]);
    minor(m[2], m[7], m[1], m[8], adj[1], mag[1]);
    minor(m[1], m[5], m[2], m[4], adj[2], mag[2]);
    minor(m[5], m[6], m[3], m[8], adj[3], mag[3]);
    minor(m[0], m[8], m[2], m[6], adj[4], mag[4]);
    minor(m[2], m[3], m[0], m[5], adj[5], mag[5]);
    minor(m[3], m[7], m[4], m[6], adj[6], mag[6]);
    minor(m[1], m[6], m[0], m[7], adj[7], mag[7]);
    minor(m[0], m[4], m[1], m[3], adj[8], mag[8]);
    // det along the first row, with cofactors adj[0], adj[3], adj[6]
    const float d0 = m[0] * adj[0], d1 = m[1] * adj[3], d2 = m[2] * adj[6];
    const float det = (d0 + d1) + d2;
    const float det_err = 3.f * u * (fabsf(m[0]) * mag[0] + fabsf(m[1]) * mag[3] + fabsf(m[2]) * mag[6]) +
                          3.f * u * (fabsf(d0) + fabsf(d1) + fabsf(d2));
    float3 lo, hi;
    bool finite = isfinite(mu.x) && isfinite(mu.y) && isfinite(mu.z);
    for (int i = 0; i < 9; ++i) finite = finite && isfinite(m[i]);
    const float adet = fabsf(det);
    if (!finite) {
      // a degenerate far-away point: the slab test never reports it below tmax (and the
      // intersection of a non-finite ellipsoid yields no events anyway)
      lo = make_float3(3e38f, 3e38f, 3e38f);
      hi = lo;
    } else if (!(adet > 1e-30f) || !isfinite(det) || !(det_err < 0.25f * adet)) {
      lo = make_float3(-3e38f, -3e38f, -3e38f);
      hi = make_float3(3e38f, 3e38f, 3e38f);
    } else {
      const float rel = det_err / (adet - det_err);  // relative error of 1/|det|
      const float mv[3] = {mu.x, mu.y, mu.z};
      float l[3], h[3];
      bool ok = true;
      for (int i = 0; i < 3; ++i) {
        const float a0 = adj[3 * i], a1 = adj[3 * i + 1], a2 = adj[3 * i + 2];
        const float g0 = mag[3 * i], g1 = mag[3 * i + 1], g2 = mag[3 * i + 2];
        const float na = sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
        const float ng = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
        const float e = na / adet;
        const float err = e * (rel + 8.f * u) + 2.f * u * ng / adet * (1.f + rel);
        const float pad = 2e-3f * e + 2.f * err + 4e-7f * (fabsf(mv[i]) + e) + 1e-30f;
        ok = ok && isfinite(e) && isfinite(pad);
        l[i] = __fsub_rd(__fsub_rd(mv[i], e), pad);
        h[i] = __fadd_ru(__fadd_ru(mv[i], e), pad);
      }
      if (ok) {
        lo = make_float3(l[0], l[1], l[2]);
        hi = make_float3(h[0], h[1], h[2]);
        c = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
        valid = isfinite(c.x) && isfinite(c.y) && isfinite(c.z);
      } else {
        lo = make_float3(-3e38f, -3e38f, -3e38f);
        hi = make_float3(3e38f, 3e38f, 3e38f);
      }
    }
    aabb[2 * p] = make_float4(lo.x, lo.y, lo.z, 0.f);
    aabb[2 * p + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
  // block reduction of the centre bounds (ordered-int atomics)
  __shared__ uint32_t smin[3], smax[3];
  if (threadIdx.x < 3) {
    smin[threadIdx.x] = 0xffffffffu;
    smax[threadIdx.x] = 0u;
  }
  __syncthreads();
  if (valid) {
    atomicMin(&smin[0], float_to_ordered(c.x));
    atomicMin(&smin[1], float_to_ordered(c.y));
    atomicMin(&smin[2], float_to_ordered(c.z));
    atomicMax(&smax[0], float_to_ordered(c.x));
    atomicMax(&smax[1], float_to_ordered(c.y));
    atomicMax(&smax[2], float_to_ordered(c.z));
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    if (smin[threadIdx.x] != 0xffffffffu) atomicMin(&bounds[threadIdx.x], smin[threadIdx.x]);
    if (smax[threadIdx.x] != 0u) atomicMax(&bounds[3 + threadIdx.x], smax[threadIdx.x]);
  }
}

__device__ __forceinline__ uint32_t expand_bits10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(const float4* __restrict__ aabb, int64_t N, const uint32_t* __restrict__ bounds,
                         uint32_t* __restrict__ codes, uint32_t* __restrict__ vals) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const float4 lo = aabb[2 * p], hi = aabb[2 * p + 1];
  const float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
  uint32_t q[3];
  for (int i = 0; i < 3; ++i) {
    const float bmin = ordered_to_float(bounds[i]), bmax = ordered_to_float(bounds[3 + i]);
    const float ext = bmax - bmin;
    float u = ext > 0.f ? (c[i] - bmin) / ext : 0.5f;
    if (!(u == u)) u = 0.5f;
    u = fminf(fmaxf(u, 0.f), 1.f);
    q[i] = min(uint32_t(u * 1024.f), 1023u);
  }
  codes[p] = (expand_bits10(q[0]) << 2) | (expand_bits10(q[1]) << 1) | expand_bits10(q[2]);
  vals[p] = uint32_t(p);
}

// ---- LSD radix sort, 8-bit digits, stable ----
__global__ void k_sort_hist(const uint32_t* __restrict__ keys, int64_t N, int shift, uint32_t* __restrict__ hist,
                            int nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * kSortTile;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t i = base + r * kSortThreads + threadIdx.x;
    if (i < N) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[int64_t(threadIdx.x) * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of the digit-major histogram in three coalesced kernels: per-chunk
// sums, a scan of the chunk sums (one block), and a per-chunk scan seeded by it.
constexpr int kScanChunks = 512;
constexpr int kScanThreads = 256;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
  // sh: kScanThreads / 32 words
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? sh[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) sh[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp > 0 ? sh[warp - 1] : 0u;
  total = sh[kScanThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void k_scan_sums(const uint32_t* __restrict__ hist, int64_t len, uint32_t* __restrict__ sums) {
  const int64_t chunk = (len + kScanChunks - 1) / kScanChunks;
  const int64_t b = blockIdx.x * chunk, e = min(len, b + chunk);
  uint32_t s = 0;
  for (int64_t i = b + threadIdx.x; i < e; i += kScanThreads) s += hist[i];
  __shared__ uint32_t sh[kScanThreads / 32];
  uint32_t total;
  block_exclusive_scan(s, sh, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_top(uint32_t* __restrict__ sums) {
  __shared__ uint32_t sh[kScanThreads / 32];
  uint32_t carry = 0;
  for (int base = 0; base < kScanChunks; base += kScanThreads) {
    const uint32_t v = sums[base + threadIdx.x];
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, sh, total);
    sums[base + threadIdx.x] = carry + ex;
    carry += total;
  }
}

__global__ void k_scan_chunks(uint32_t* __restrict__ hist, int64_t len, const uint32_t* __restrict__ sums) {
  const int64_t chunk = (len + kScanChunks - 1) / kScanChunks;
  const int64_t b = blockIdx.x * chunk, e = min(len, b + chunk);
  __shared__ uint32_t sh[kScanThreads / 32];
  uint32_t carry = sums[blockIdx.x];
  for (int64_t base = b; base < e; base += kScanThreads) {
    const int64_t i = base + threadIdx.x;
    const uint32_t v = i < e ? hist[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, sh, total);
    if (i < e) hist[i] = carry + ex;
    carry += total;
  }
}

__global__ void k_sort_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                               uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t N, int shift,
                               const uint32_t* __restrict__ hist, int nblocks) {
  __shared__ uint32_t gofs[256];
  __shared__ uint32_t running[256];
  __shared__ uint32_t wcount[kSortWarps][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  gofs[tid] = hist[int64_t(tid) * nblocks + blockIdx.x];
  running[tid] = 0;
  for (int w = 0; w < kSortWarps; ++w) wcount[w][tid] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * kSortTile;
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t i = base + r * kSortThreads + tid;
    const bool ok = i < N;
    uint32_t key = 0, val = 0, d = 256;  // 256: out of range, never matches a real digit
    if (ok) {
      key = kin[i];
      val = vin[i];
      d = (key >> shift) & 255u;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank_w = __popc(peers & lt_mask);
    if (ok && rank_w == 0) wcount[warp][d] = __popc(peers);
    __syncthreads();
    {
      uint32_t acc = running[tid];
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = wcount[w][tid];
        wcount[w][tid] = acc;
        acc += c;
      }
      running[tid] = acc;
    }
    __syncthreads();
    if (ok) {
      const uint32_t dst = gofs[d] + wcount[warp][d] + rank_w;
      kout[dst] = key;
      vout[dst] = val;
    }
    __syncthreads();
    for (int w = 0; w < kSortWarps; ++w) wcount[w][tid] = 0;
    __syncthreads();
  }
}

// Gathers records, features and leaf boxes into Morton order.
__global__ void k_gather(const uint32_t* __restrict__ sorted_vals, int64_t N, int K,
                         const float* __restrict__ mean, const float* __restrict__ scale,
                         const float* __restrict__ quat, const float* __restrict__ density,
                         const float4* __restrict__ aabb_in,
                         float4* __restrict__ aabb_out, Record* __restrict__ recs, float* __restrict__ feat_out,
                         int32_t* __restrict__ order) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int64_t p = sorted_vals[j];
  order[j] = int32_t(p);
  float W[9];
  prim_matrix(ld4(quat, p), ld3(scale, p), W);
  const float3 mu = ld3(mean, p);
  Record R;
  R.r0 = make_float4(W[0], W[1], W[2], mu.x);
  R.r1 = make_float4(W[3], W[4], W[5], mu.y);
  R.r2 = make_float4(W[6], W[7], W[8], mu.z);
  // r3.yzw (the DC colour) is written by k_gather_features, and kept by a refit without features
  float4* rp = reinterpret_cast<float4*>(recs + j);
  rp[0] = R.r0;
  rp[1] = R.r1;
  rp[2] = R.r2;
  recs[j].r3.x = density[p];
  aabb_out[2 * j] = aabb_in[2 * p];
  aabb_out[2 * j + 1] = aabb_in[2 * p + 1];
}

// Feature rows to Morton order, padded to feat_stride(K): one row per threadIdx.y, one
// float4 column per threadIdx.x (blockDim.x = feat_stride(K) / 4), so no index division per
// element. vec: the source rows are whole, 16-byte aligned float4s (3K % 4 == 0, aligned base).
// Column 0 also writes the record's DC colour C0 * f0 + 0.5 (r3.yzw).
__global__ void k_gather_features(const int32_t* __restrict__ order, int64_t N, int K, const float* __restrict__ feat,
                                  float* __restrict__ feat_out, Record* __restrict__ recs, bool vec) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.y + threadIdx.y;
  if (j >= N) return;
  const int c = threadIdx.x, per = 3 * K;
  const float* src = feat + int64_t(__ldg(order + j)) * per;
  float4 v;
  if (vec) {
    v = __ldg(reinterpret_cast<const float4*>(src) + c);
  } else {
    float t[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) t[q] = 4 * c + q < per ? __ldg(src + 4 * c + q) : 0.f;
    v = make_float4(t[0], t[1], t[2], t[3]);
  }
  reinterpret_cast<float4*>(feat_out + j * feat_stride(K))[c] = v;
  if (c == 0) {
    recs[j].r3.y = dc_channel(v.x);
    recs[j].r3.z = dc_channel(v.y);
    recs[j].r3.w = dc_channel(v.z);
  }
}

// Karras 2012: delta(i, j) = common prefix length of keys i, j (index bits break ties).
__device__ __forceinline__ int delta(const uint32_t* __restrict__ codes, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a == b) return 32 + __clz(uint32_t(i) ^ uint32_t(j));
  return __clz(a ^ b);
}

__global__ void k_lbvh(const uint32_t* __restrict__ codes, int64_t N, Node* __restrict__ nodes,
                       int32_t* __restrict__ parent_node, int32_t* __restrict__ parent_leaf) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= N - 1) return;
  const int d = (delta(codes, N, i, i + 1) - delta(codes, N, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(codes, N, i, i - d);
  int64_t lmax = 2;
  while (delta(codes, N, i, i + lmax * d) > dmin) lmax <<= 1;
  int64_t l = 0;
  for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(codes, N, i, i + (l + t) * d) > dmin) l += t;
  const int64_t j = i + l * d;
  const int dnode = delta(codes, N, i, j);
  int64_t s = 0;
  int64_t t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(codes, N, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int64_t gamma = i + s * d + min(d, 0);
  const int64_t lo = min(i, j), hi = max(i, j);
  int c0, c1;
  if (lo == gamma) {
    c0 = ~int(gamma);
    parent_leaf[gamma] = int(i);
  } else {
    c0 = int(gamma);
    parent_node[gamma] = int(i);
  }
  if (hi == gamma + 1) {
    c1 = ~int(gamma + 1);
    parent_leaf[gamma + 1] = int(i);
  } else {
    c1 = int(gamma + 1);
    parent_node[gamma + 1] = int(i);
  }
  nodes[i].d = make_int4(c0, c1, 0, 0);
  if (i == 0) parent_node[0] = -1;
}

__device__ __forceinline__ void child_box(const Node* nodes, const float4* aabb, int c, float3& lo, float3& hi) {
  if (c < 0) {
    const float4 a = __ldcg(aabb + 2 * int64_t(~c)), b = __ldcg(aabb + 2 * int64_t(~c) + 1);
    lo = make_float3(a.x, a.y, a.z);
    hi = make_float3(b.x, b.y, b.z);
  } else {
    const float4 a = __ldcg(&nodes[c].a), b = __ldcg(&nodes[c].b), cc = __ldcg(&nodes[c].c);
    lo = make_float3(fminf(a.x, b.z), fminf(a.y, b.w), fminf(a.z, cc.x));
    hi = make_float3(fmaxf(a.w, cc.y), fmaxf(b.x, cc.z), fmaxf(b.y, cc.w));
  }
}

__global__ void k_refit(int64_t N, Node* __restrict__ nodes, const float4* __restrict__ aabb,
                        const int32_t* __restrict__ parent_node, const int32_t* __restrict__ parent_leaf,
                        uint32_t* __restrict__ flags) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int n = parent_leaf[j];
  while (n >= 0) {
    // acquire-release at device scope: this thread's box stores above happen before the
    // sibling's loads once it sees the count, and the sibling's stores before this thread's
    // loads below (one instruction instead of two full fences around the atomic)
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> f(flags[n]);
    if (f.fetch_add(1u, cuda::memory_order_acq_rel) == 0u) return;  // the sibling subtree is not done yet
    const int4 ch = __ldcg(&nodes[n].d);
    float3 l0, h0, l1, h1;
    child_box(nodes, aabb, ch.x, l0, h0);
    child_box(nodes, aabb, ch.y, l1, h1);
    __stcg(&nodes[n].a, make_float4(l0.x, l0.y, l0.z, h0.x));
    __stcg(&nodes[n].b, make_float4(h0.y, h0.z, l1.x, l1.y));
    __stcg(&nodes[n].c, make_float4(l1.z, h1.x, h1.y, h1.z));
    n = parent_node[n];
  }
}

__global__ void k_single_leaf(Node* nodes, const float4* aabb) {
  const float4 a = aabb[0], b = aabb[1];
  Node nd;
  nd.a = make_float4(a.x, a.y, a.z, b.x);
  nd.b = make_float4(b.y, b.z, 3e38f, 3e38f);  // child 1: a far-away point box, never hit below tmax
  nd.c = make_float4(3e38f, 3e38f, 3e38f, 3e38f);
  nd.d = make_int4(~0, ~0, 0, 0);
  nodes[0] = nd;
}

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Only the records' DC colour C0 * f0 + 0.5 (r3.yzw), for scenes that keep no feature rows:
// the same bits as k_gather_features' column 0.
__global__ void k_gather_dc(const int32_t* __restrict__ order, int64_t N, int K, const float* __restrict__ feat,
                            Record* __restrict__ recs) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const float* src = feat + int64_t(__ldg(order + j)) * (3 * K);
  recs[j].r3.y = dc_channel(__ldg(src));
  recs[j].r3.z = dc_channel(__ldg(src + 1));
  recs[j].r3.w = dc_channel(__ldg(src + 2));
}

// feat_out null: the scene keeps the DC colour only (ever_scene_build_dc).
void launch_gather_features(const int32_t* order, int64_t N, int K, const float* feat, float* feat_out, void* recs,
                            cudaStream_t st) {
  if (!feat_out) {
    k_gather_dc<<<unsigned(div_up(N, 256)), 256, 0, st>>>(order, N, K, feat, static_cast<Record*>(recs));
    return;
  }
  const int cols = feat_stride(K) / 4, rows = std::max(1, 256 / cols);
  const bool vec = (3 * K) % 4 == 0 && reinterpret_cast<uintptr_t>(feat) % 16 == 0;
  k_gather_features<<<unsigned(div_up(N, rows)), dim3(cols, rows), 0, st>>>(order, N, K, feat, feat_out,
                                                                           static_cast<Record*>(recs), vec);
}

}  // namespace

int sort_blocks(int64_t N) { return int(div_up(std::max<int64_t>(N, 1), kSortTile)); }

// Stable LSD radix sort of (key, value) pairs on the low `bits` key bits, 8 bits per pass.
// On return the sorted pairs are in (ka, va); (kb, vb) are scratch of the same size and
// hist holds sort_blocks(N) * 256 words.
void sort_pairs(uint32_t*& ka, uint32_t*& va, uint32_t*& kb, uint32_t*& vb, uint32_t* hist, int64_t N, int bits,
                cudaStream_t st) {
  const int nblocks = sort_blocks(N);
  const int64_t len = int64_t(nblocks) * 256;
  uint32_t* sums = hist + len;  // kScanChunks words after the histogram
  for (int shift = 0; shift < bits; shift += 8) {
    k_sort_hist<<<nblocks, kSortThreads, 0, st>>>(ka, N, shift, hist, nblocks);
    k_scan_sums<<<kScanChunks, kScanThreads, 0, st>>>(hist, len, sums);
    k_scan_top<<<1, kScanThreads, 0, st>>>(sums);
    k_scan_chunks<<<kScanChunks, kScanThreads, 0, st>>>(hist, len, sums);
    k_sort_scatter<<<nblocks, kSortThreads, 0, st>>>(ka, va, kb, vb, N, shift, hist, nblocks);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
}

SceneLayout scene_layout(int64_t N, int K) {
  SceneLayout L;
  WsCursor c;
  const int64_t n1 = N > 0 ? (N > 1 ? N - 1 : 1) : 0;
  L.nodes = c.take(n1 * sizeof(Node));
  L.records = c.take(N * sizeof(Record));
  L.features = c.take(N * int64_t(feat_stride(K)) * sizeof(float));
  L.order = c.take(N * sizeof(int32_t));
  L.aabb_a = c.take(N * 2 * sizeof(float4));
  L.aabb_b = c.take(N * 2 * sizeof(float4));
  L.keys_a = c.take(N * sizeof(uint32_t));
  L.keys_b = c.take(N * sizeof(uint32_t));
  L.vals_a = c.take(N * sizeof(uint32_t));
  L.vals_b = c.take(N * sizeof(uint32_t));
  L.nblocks = sort_blocks(N);
  L.hist = c.take((int64_t(L.nblocks) * 256 + kScanChunks) * sizeof(uint32_t));
  L.parent_node = c.take(std::max<int64_t>(n1, 1) * sizeof(int32_t));
  L.parent_leaf = c.take(std::max<int64_t>(N, 1) * sizeof(int32_t));
  L.flags = c.take(std::max<int64_t>(n1, 1) * sizeof(uint32_t));
  L.bounds = c.take(8 * sizeof(uint32_t));
  L.total = c.offset;
  return L;
}

cudaError_t scene_build(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* feat, int64_t N, int K, char* ws, const SceneLayout& L, EverScene* sc,
                        cudaStream_t st, bool dc_only) {
  sc->num_prims = N;
  sc->sh_coeffs = K;
  sc->num_nodes = N > 0 ? int32_t(N > 1 ? N - 1 : 1) : 0;
  sc->nodes = ws + L.nodes;
  sc->records = ws + L.records;
  sc->features = dc_only ? nullptr : reinterpret_cast<float*>(ws + L.features);
  sc->order = reinterpret_cast<int32_t*>(ws + L.order);
  sc->scratch = ws + L.aabb_a;
  if (N == 0) return cudaGetLastError();
  Node* nodes = reinterpret_cast<Node*>(ws + L.nodes);
  float4* aabb_a = reinterpret_cast<float4*>(ws + L.aabb_a);
  float4* aabb_b = reinterpret_cast<float4*>(ws + L.aabb_b);
  uint32_t* ka = reinterpret_cast<uint32_t*>(ws + L.keys_a);
  uint32_t* kb = reinterpret_cast<uint32_t*>(ws + L.keys_b);
  uint32_t* va = reinterpret_cast<uint32_t*>(ws + L.vals_a);
  uint32_t* vb = reinterpret_cast<uint32_t*>(ws + L.vals_b);
  uint32_t* hist = reinterpret_cast<uint32_t*>(ws + L.hist);
  uint32_t* bounds = reinterpret_cast<uint32_t*>(ws + L.bounds);
  int32_t* pn = reinterpret_cast<int32_t*>(ws + L.parent_node);
  int32_t* pl = reinterpret_cast<int32_t*>(ws + L.parent_leaf);
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + L.flags);

  cudaError_t e;
  if ((e = cudaMemsetAsync(bounds, 0xff, 3 * sizeof(uint32_t), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(bounds + 3, 0x00, 3 * sizeof(uint32_t), st)) != cudaSuccess) return e;
  const int tb = 256;
  const int64_t gb = div_up(N, tb);
  k_aabbs<<<unsigned(gb), tb, 0, st>>>(mean, scale, quat, N, aabb_a, bounds);
  k_morton<<<unsigned(gb), tb, 0, st>>>(aabb_a, N, bounds, ka, va);
  // 30-bit keys: 4 passes of 8 bits
  sort_pairs(ka, va, kb, vb, hist, N, 30, st);
  k_gather<<<unsigned(gb), tb, 0, st>>>(va, N, K, mean, scale, quat, density, aabb_a, aabb_b,
                                        reinterpret_cast<Record*>(sc->records), sc->features, sc->order);
  launch_gather_features(sc->order, N, K, feat, sc->features, sc->records, st);
  if (N == 1) {
    k_single_leaf<<<1, 1, 0, st>>>(nodes, aabb_b);
    return cudaGetLastError();
  }
  if ((e = cudaMemsetAsync(flags, 0, (N - 1) * sizeof(uint32_t), st)) != cudaSuccess) return e;
  k_lbvh<<<unsigned(div_up(N - 1, tb)), tb, 0, st>>>(ka, N, nodes, pn, pl);
  k_refit<<<unsigned(gb), tb, 0, st>>>(N, nodes, aabb_b, pn, pl, flags);
  return cudaGetLastError();
}

// Refit a built scene to new ellipsoid parameters: same Morton order and tree topology as
// the last build (the parent links stay in the workspace), new records, boxes and, when
// given, features. Tree quality degrades as ellipsoids move far from where they were
// built; a rebuild restores it.
cudaError_t scene_refit(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* feat, char* ws, const SceneLayout& L, EverScene* sc, cudaStream_t st) {
  const int64_t N = sc->num_prims;
  const int K = sc->sh_coeffs;
  if (N == 0) return cudaSuccess;
  Node* nodes = reinterpret_cast<Node*>(ws + L.nodes);
  float4* aabb_a = reinterpret_cast<float4*>(ws + L.aabb_a);
  float4* aabb_b = reinterpret_cast<float4*>(ws + L.aabb_b);
  uint32_t* bounds = reinterpret_cast<uint32_t*>(ws + L.bounds);
  int32_t* pn = reinterpret_cast<int32_t*>(ws + L.parent_node);
  int32_t* pl = reinterpret_cast<int32_t*>(ws + L.parent_leaf);
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + L.flags);
  const int tb = 256;
  const int64_t gb = div_up(N, tb);
  k_aabbs<<<unsigned(gb), tb, 0, st>>>(mean, scale, quat, N, aabb_a, bounds);
  k_gather<<<unsigned(gb), tb, 0, st>>>(reinterpret_cast<const uint32_t*>(sc->order), N, K, mean, scale, quat, density,
                                        aabb_a, aabb_b, reinterpret_cast<Record*>(sc->records), sc->features,
                                        sc->order);
  if (feat)
    launch_gather_features(sc->order, N, K, feat, sc->features, sc->records, st);
  if (N == 1) {
    k_single_leaf<<<1, 1, 0, st>>>(nodes, aabb_b);
    return cudaGetLastError();
  }
  cudaError_t e = cudaMemsetAsync(flags, 0, (N - 1) * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_refit<<<unsigned(gb), tb, 0, st>>>(N, nodes, aabb_b, pn, pl, flags);
  return cudaGetLastError();
}

cudaError_t scene_set_features(EverScene* sc, const float* feat, cudaStream_t st) {
  const int64_t total = sc->num_prims * int64_t(sc->sh_coeffs) * 3;
  if (total == 0) return cudaSuccess;
  launch_gather_features(sc->order, sc->num_prims, sc->sh_coeffs, feat, sc->features, sc->records, st);
  return cudaGetLastError();
}

}  // namespace ever
