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

// Conservative AABB of {x : |W (x - mean)| <= 1}: half extent i = |row_i(W^-1)|, computed
// in double from the same W the intersection uses, then padded so that event times
// computed in float never fall outside the box (grazing roots move by ~sqrt(eps) of the
// radius).
__global__ void k_aabbs(const float* __restrict__ mean, const float* __restrict__ scale,
                        const float* __restrict__ quat, int64_t N, float4* __restrict__ aabb,
                        uint32_t* __restrict__ bounds) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  float3 c = make_float3(0.f, 0.f, 0.f);
  bool valid = false;
  if (p < N) {
    float W[9];
    prim_matrix(ld4(quat, p), ld3(scale, p), W);
    const float3 mu = ld3(mean, p);
    double m[9];
    for (int i = 0; i < 9; ++i) m[i] = W[i];
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    float3 lo, hi;
    bool finite = isfinite(mu.x) && isfinite(mu.y) && isfinite(mu.z);
    for (int i = 0; i < 9; ++i) finite = finite && isfinite(W[i]);
    if (!finite) {
      // a degenerate far-away point: the slab test never reports it below tmax (and the
      // intersection of a non-finite ellipsoid yields no events anyway)
      lo = make_float3(3e38f, 3e38f, 3e38f);
      hi = lo;
    } else if (!(fabs(det) > 1e-30) || !isfinite(det)) {
      lo = make_float3(-3e38f, -3e38f, -3e38f);
      hi = make_float3(3e38f, 3e38f, 3e38f);
    } else {
      // inverse = adj / det, rows of the inverse
      const double inv[9] = {c00 / det, (m[2] * m[7] - m[1] * m[8]) / det, (m[1] * m[5] - m[2] * m[4]) / det,
                             c01 / det, (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                             c02 / det, (m[1] * m[6] - m[0] * m[7]) / det, (m[0] * m[4] - m[1] * m[3]) / det};
      double e[3];
      for (int i = 0; i < 3; ++i)
        e[i] = sqrt(inv[3 * i] * inv[3 * i] + inv[3 * i + 1] * inv[3 * i + 1] + inv[3 * i + 2] * inv[3 * i + 2]);
      const double mv[3] = {mu.x, mu.y, mu.z};
      double l[3], h[3];
      for (int i = 0; i < 3; ++i) {
        const double pad = 2e-3 * e[i] + 4e-7 * (fabs(mv[i]) + e[i]) + 1e-30;
        l[i] = mv[i] - e[i] - pad;
        h[i] = mv[i] + e[i] + pad;
      }
      lo = make_float3(__double2float_rd(l[0]), __double2float_rd(l[1]), __double2float_rd(l[2]));
      hi = make_float3(__double2float_ru(h[0]), __double2float_ru(h[1]), __double2float_ru(h[2]));
      c = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
      valid = isfinite(c.x) && isfinite(c.y) && isfinite(c.z);
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
  R.r3 = make_float4(density[p], __int_as_float(int(p)), 0.f, 0.f);
  recs[j] = R;
  aabb_out[2 * j] = aabb_in[2 * p];
  aabb_out[2 * j + 1] = aabb_in[2 * p + 1];
}

// Feature rows into Morton order, one thread per padded float (coalesced on both sides).
// Feature rows to Morton order, padded to feat_stride(K): one row per threadIdx.y, one
// float4 column per threadIdx.x (blockDim.x = feat_stride(K) / 4), so no index division per
// element. vec: the source rows are whole, 16-byte aligned float4s (3K % 4 == 0, aligned base).
__global__ void k_gather_features(const int32_t* __restrict__ order, int64_t N, int K, const float* __restrict__ feat,
                                  float* __restrict__ feat_out, bool vec) {
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

void launch_gather_features(const int32_t* order, int64_t N, int K, const float* feat, float* feat_out,
                            cudaStream_t st) {
  const int cols = feat_stride(K) / 4, rows = std::max(1, 256 / cols);
  const bool vec = (3 * K) % 4 == 0 && reinterpret_cast<uintptr_t>(feat) % 16 == 0;
  k_gather_features<<<unsigned(div_up(N, rows)), dim3(cols, rows), 0, st>>>(order, N, K, feat, feat_out, vec);
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
                        cudaStream_t st) {
  sc->num_prims = N;
  sc->sh_coeffs = K;
  sc->num_nodes = N > 0 ? int32_t(N > 1 ? N - 1 : 1) : 0;
  sc->nodes = ws + L.nodes;
  sc->records = ws + L.records;
  sc->features = reinterpret_cast<float*>(ws + L.features);
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
  launch_gather_features(sc->order, N, K, feat, sc->features, st);
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
    launch_gather_features(sc->order, N, K, feat, sc->features, st);
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
  launch_gather_features(sc->order, sc->num_prims, sc->sh_coeffs, feat, sc->features, st);
  return cudaGetLastError();
}

}  // namespace ever
