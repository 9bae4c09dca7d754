// Ray-cost model: a 39 -> 64 -> 64 -> 2 ReLU MLP with BF16 weights and activations and
// FP32 accumulation, run on the 5th-generation tensor cores (tcgen05.mma with the
// accumulators in tensor memory), for inference and for training.
//
// Input encoding of a ray (o, d): p = (o - c) - ((o - c).d^) d^, the point of the ray's
// line closest to the scene centre c, times 1/scale; then x, sin(2^k pi x), cos(2^k pi x)
// for k = 0..5 per component: 3 + 36 = 39 features, zero-padded to 64 columns. Outputs:
// the cost the tracer logs per ray, [log(1 + consumed events), depth offset / scale].
//
// One CTA of 128 threads (one warpgroup) loops over tiles of 128 rays (the MMA's M).
// Operands live in shared memory in the canonical no-swizzle layouts: 8 x 8 bf16 core
// matrices of 128 contiguous bytes. Activation tiles [ray][unit] are K-major operands of
// the layer products; the same bytes are the MN-major operands of the weight-gradient
// products, which reduce over rays. Thread 0 issues the MMAs and tcgen05.commit signals
// their completion on an mbarrier; every wait is bounded and reports a timeout through an
// error flag instead of hanging.
#include <cstddef>

#include <cuda_bf16.h>

#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr int kTile = 128;  // rays per tile = MMA M
constexpr int kIn = 64;     // padded encoding width
constexpr int kHid = 64;
constexpr int kOut = 16;    // padded output width (2 used)
// tensor-memory columns: layer accumulators, then (training) weight-gradient accumulators
constexpr uint32_t kColD1 = 0, kColD2 = 64, kColD3 = 128, kColGW1 = 256, kColGW2 = 320, kColGW3 = 384;
// inference: every layer's accumulator reuses D1's columns (each is read out before the next
// MMA is issued), and one activation tile serves all three layers
constexpr uint32_t kColsInfer = 64, kColsTrain = 512;
constexpr size_t kTrainSmem = 120 * 1024;  // keeps one training CTA (512 TMEM columns) per SM
constexpr int kInferCtasPerSm = kMlpInferCtasPerSm;  // 6 x 64 TMEM columns, about 37 KB shared memory each

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, col) of a K-major no-swizzle tile with `rows` rows: core
// matrix (row / 8, col / 8) at ((col / 8) * rows / 8 + row / 8) * 128, 16 bytes per row.
__host__ __device__ constexpr int kmaj(int row, int col, int rows) {
  return ((((col >> 3) * (rows >> 3)) + (row >> 3)) << 7) + ((row & 7) << 4) + ((col & 7) << 1);
}

// Shared-memory matrix descriptor: no swizzle, descriptor version 1, byte offsets >> 4.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
// K-major operand of `rows` rows starting at K chunk pair ks (K = 16 per MMA).
__device__ __forceinline__ uint64_t desc_k(uint32_t base, int rows, int ks) {
  return sdesc(base + ks * 2 * (rows / 8) * 128, (rows / 8) * 128, 128);
}
// MN-major view of a K-major tile whose rows are the MMA's K: MN = the tile's columns.
__device__ __forceinline__ uint64_t desc_mn(uint32_t base, int rows, int ks) {
  return sdesc(base + ks * 2 * 128, 128, (rows / 8) * 128);
}

// Instruction descriptor: BF16 x BF16 -> F32, dense, M x N, operand majors (1 = MN-major).
__device__ __forceinline__ uint32_t idesc(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
         (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

constexpr long long kWaitClocks = 1ll << 31;  // about a second
// Bounded wait for phase `phase` of the barrier; false once `limit` clocks have passed.
// Shorter limits than the default poll with the non-blocking test (a try_wait may itself
// suspend for longer than such a limit), so a test can make a wait run out for certain.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit = kWaitClocks) {
  const long long t0 = clock64();
  if (limit < kWaitClocks) {
    while (!mbar_test(bar, phase))
      if (clock64() - t0 > limit) return false;
    return true;
  }
  while (!mbar_try(bar, phase))
    if (clock64() - t0 > limit) return false;
  return true;
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct Smem {
  float b1[kHid], b2[kHid], b3[kOut];
  float gb1[4][kHid], gb2[4][kHid], gb3[4][kOut], loss[4];  // per-warp sums (fixed order)
  uint64_t bar;
  uint32_t tmem_base;
  __align__(128) __nv_bfloat16 w1[kHid * kIn];  // [h1][in]  K-major, rows = output units
  __nv_bfloat16 w2[kHid * kHid];                 // [h2][h1]
  __nv_bfloat16 w3[kOut * kHid];                 // [out][h2]
  __nv_bfloat16 a0[kTile * kIn];                 // encoding (inference: also hidden 1 and 2) [ray][in]
  // training only: inference launches with the shared memory up to here
  __nv_bfloat16 a1[kTile * kHid];  // hidden 1            [ray][h1]
  __nv_bfloat16 a2[kTile * kHid];  // hidden 2            [ray][h2]
  __nv_bfloat16 g3[kTile * kOut];  // dL/d output         [ray][out]
  __nv_bfloat16 g2[kTile * kHid];  // dL/d pre-act 2      [ray][h2]
  __nv_bfloat16 g1[kTile * kHid];  // dL/d pre-act 1      [ray][h1]
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
// Eight consecutive columns (c0 % 8 == 0) of one row: one 16-byte shared store / load.
__device__ __forceinline__ void st8(__nv_bfloat16* tile, int row, int c0, int rows, const float* v) {
  const uint4 q = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                             pack_bf16x2(v[6], v[7]));
  *reinterpret_cast<uint4*>(reinterpret_cast<char*>(tile) + kmaj(row, c0, rows)) = q;
}
__device__ __forceinline__ void ld8(const __nv_bfloat16* tile, int row, int c0, int rows, float* v) {
  const uint4 q = *reinterpret_cast<const uint4*>(reinterpret_cast<const char*>(tile) + kmaj(row, c0, rows));
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[2 * i] = __uint_as_float(w[i] << 16);
    v[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
  }
}

__device__ __forceinline__ float warp_sum(float t) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

// Encoding of ray r (or its pre-encoded row).
__device__ __forceinline__ void encode(const MlpParams& P, int64_t r, float (&f)[kIn]) {
  if (P.feat) {
#pragma unroll
    for (int c = 0; c < kIn; ++c) f[c] = P.feat[r * kIn + c];
    return;
  }
  const float ox = P.rayo[3 * r] - P.cx, oy = P.rayo[3 * r + 1] - P.cy, oz = P.rayo[3 * r + 2] - P.cz;
  float dx = P.rayd[3 * r], dy = P.rayd[3 * r + 1], dz = P.rayd[3 * r + 2];
  const float n = sqrtf(dx * dx + dy * dy + dz * dz);
  const float inv = n > 0.f ? 1.f / n : 0.f;
  dx *= inv;
  dy *= inv;
  dz *= inv;
  const float od = ox * dx + oy * dy + oz * dz;
  float x[3] = {(ox - od * dx) * P.inv_scale, (oy - od * dy) * P.inv_scale, (oz - od * dz) * P.inv_scale};
#pragma unroll
  for (int i = 0; i < 3; ++i) x[i] = isfinite(x[i]) ? x[i] : 0.f;
  // sin / cos of 2^q pi x from one sincospi per component and the double-angle identities
  // sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a (after five doublings the error is a
  // few 1e-6, far below the bf16 rounding the features go through)
  float sv[3], cv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    f[i] = x[i];
    sincospif(x[i], &sv[i], &cv[i]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      f[3 + 6 * q + i] = sv[i];
      f[6 + 6 * q + i] = cv[i];
      const float s2 = 2.f * sv[i] * cv[i];
      cv[i] = fmaf(-2.f * sv[i], sv[i], 1.f);
      sv[i] = s2;
    }
  }
#pragma unroll
  for (int k = 39; k < kIn; ++k) f[k] = 0.f;
}

// Inference (TRAIN = false: predictions and cost bins) or the gradients of one training
// batch (TRAIN = true: each CTA writes its partial gradient and loss to P.partial).
template <bool TRAIN>
__global__ void __launch_bounds__(128, TRAIN ? 1 : kInferCtasPerSm) k_mlp(const MlpParams P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t kCols = TRAIN ? kColsTrain : kColsInfer;

  // weights into the canonical layouts (8 columns per 16-byte store), biases
  {
    const __nv_bfloat16* w1 = static_cast<const __nv_bfloat16*>(P.w1);
    const __nv_bfloat16* w2 = static_cast<const __nv_bfloat16*>(P.w2);
    const __nv_bfloat16* w3 = static_cast<const __nv_bfloat16*>(P.w3);
    for (int i = tid; i < kHid * kIn / 8; i += 128) {
      const int o = i / (kIn / 8), c0 = (i % (kIn / 8)) * 8;
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(S.w1) + kmaj(o, c0, kHid)) =
          *reinterpret_cast<const uint4*>(w1 + o * kIn + c0);
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(S.w2) + kmaj(o, c0, kHid)) =
          *reinterpret_cast<const uint4*>(w2 + o * kHid + c0);
    }
    for (int i = tid; i < kOut * kHid / 8; i += 128) {
      const int o = i / (kHid / 8), c0 = (i % (kHid / 8)) * 8;
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(S.w3) + kmaj(o, c0, kOut)) =
          *reinterpret_cast<const uint4*>(w3 + o * kHid + c0);
    }
  }
  if (tid < kHid) {
    S.b1[tid] = P.params[kOffB1 + tid];
    S.b2[tid] = P.params[kOffB2 + tid];
    for (int w = 0; w < 4; ++w) S.gb1[w][tid] = S.gb2[w][tid] = 0.f;
  }
  if (tid < kOut) {
    S.b3[tid] = P.params[kOffB3 + tid];
    for (int w = 0; w < 4; ++w) S.gb3[w][tid] = 0.f;
  }
  if (tid < 4) S.loss[tid] = 0.f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  const uint32_t lane_off = uint32_t(warp * 32) << 16;  // TMEM lanes of this warp's quarter
  uint32_t phase = 0, pending = 0;
  bool ok = true;
  int tiles_done = 0;

  // Make the generic shared stores visible to the tensor cores, let thread 0 issue the
  // MMAs and commit them, wait (bounded) for completion. False on timeout.
  auto run = [&](auto issue) -> bool {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      issue();
      mma_commit(&S.bar);
    }
    pending = phase;
    const bool got = mbar_wait(&S.bar, phase, P.wait_clocks > 0 ? P.wait_clocks : kWaitClocks);
    phase ^= 1u;
    tc_fence_after();
    return __syncthreads_and(got) != 0;
  };

  // inference: hidden 1 and 2 overwrite the tile the previous (completed) MMA read
  __nv_bfloat16* const a1 = TRAIN ? S.a1 : S.a0;
  __nv_bfloat16* const a2 = TRAIN ? S.a2 : S.a0;
  constexpr uint32_t kColH2 = TRAIN ? kColD2 : kColD1;  // inference: layers 2 and 3 reuse D1's columns
  constexpr uint32_t kColY = TRAIN ? kColD3 : kColD1;
  const uint32_t sa0 = smem_u32(S.a0), sa1 = smem_u32(a1), sa2 = smem_u32(a2);
  const uint32_t sw1 = smem_u32(S.w1), sw2 = smem_u32(S.w2), sw3 = smem_u32(S.w3);
  const uint32_t sg1 = smem_u32(S.g1), sg2 = smem_u32(S.g2), sg3 = smem_u32(S.g3);
  const int64_t ntiles = (P.num_samples + kTile - 1) / kTile;

  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t s = tile * kTile + tid;
    const bool valid = s < P.num_samples;
    const int64_t r = valid ? (P.sample_idx ? int64_t(P.sample_idx[s]) : s) : 0;
    {
      float f[kIn];
      encode(P, r, f);
      if (!valid)
#pragma unroll
        for (int c = 0; c < kIn; ++c) f[c] = 0.f;
#pragma unroll
      for (int c0 = 0; c0 < kIn; c0 += 8) st8(S.a0, tid, c0, kTile, f + c0);
    }
    // layer 1: D1[128 x 64] = A0 W1^T
    ok = run([&] {
      for (int ks = 0; ks < kIn / 16; ++ks)
        mma(tmem + kColD1, desc_k(sa0, kTile, ks), desc_k(sw1, kHid, ks), idesc(128, kHid, false, false), ks > 0);
    });
    if (!ok) break;
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_off + kColD1 + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + S.b1[c0 + i], 0.f);
      st8(a1, tid, c0, kTile, v);
      st8(a1, tid, c0 + 8, kTile, v + 8);
    }
    // layer 2: D2 = A1 W2^T
    ok = run([&] {
      for (int ks = 0; ks < kHid / 16; ++ks)
        mma(tmem + kColH2, desc_k(sa1, kTile, ks), desc_k(sw2, kHid, ks), idesc(128, kHid, false, false), ks > 0);
    });
    if (!ok) break;
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_off + kColH2 + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + S.b2[c0 + i], 0.f);
      st8(a2, tid, c0, kTile, v);
      st8(a2, tid, c0 + 8, kTile, v + 8);
    }
    // layer 3: D3[128 x 16] = A2 W3^T
    ok = run([&] {
      for (int ks = 0; ks < kHid / 16; ++ks)
        mma(tmem + kColY, desc_k(sa2, kTile, ks), desc_k(sw3, kOut, ks), idesc(128, kOut, false, false), ks > 0);
    });
    if (!ok) break;
    float y[16];
    tmem_ld16(tmem + lane_off + kColY, y);
    const float y0 = y[0] + S.b3[0], y1 = y[1] + S.b3[1];
    ++tiles_done;
    if (!TRAIN) {
      if (valid) {
        P.pred[2 * r] = y0;
        P.pred[2 * r + 1] = y1;
        if (P.bins) P.bins[r] = uint8_t(int(y0 > P.thr[0]) + int(y0 > P.thr[1]) + int(y0 > P.thr[2]));
      }
      continue;
    }
    // ---- training: weighted squared error on the two outputs, mean over the batch
    float g[16] = {};
    float l = 0.f;
    if (valid) {
      const float e0 = y0 - P.target[2 * r], e1 = y1 - P.target[2 * r + 1];
      g[0] = 2.f * P.loss_w0 * e0 * P.inv_batch;
      g[1] = 2.f * P.loss_w1 * e1 * P.inv_batch;
      l = (P.loss_w0 * e0 * e0 + P.loss_w1 * e1 * e1) * P.inv_batch;
    }
    st8(S.g3, tid, 0, kTile, g);
    st8(S.g3, tid, 8, kTile, g + 8);
    {
      const float t0 = warp_sum(g[0]), t1 = warp_sum(g[1]), tl = warp_sum(l);
      if (lane == 0) {
        S.gb3[warp][0] += t0;
        S.gb3[warp][1] += t1;
        S.loss[warp] += tl;
      }
    }
    // dA2[128 x 64] = G3[128 x 16] W3[16 x 64]; W3 read MN-major (MN = h2, K = out)
    ok = run([&] {
      mma(tmem + kColD2, desc_k(sg3, kTile, 0), desc_mn(sw3, kOut, 0), idesc(128, kHid, false, true), 0);
    });
    if (!ok) break;
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16], a[16];
      tmem_ld16(tmem + lane_off + kColD2 + c0, v);
      ld8(S.a2, tid, c0, kTile, a);
      ld8(S.a2, tid, c0 + 8, kTile, a + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = a[i] > 0.f ? v[i] : 0.f;
      st8(S.g2, tid, c0, kTile, v);
      st8(S.g2, tid, c0 + 8, kTile, v + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float t = warp_sum(v[i]);
        if (lane == 0) S.gb2[warp][c0 + i] += t;
      }
    }
    // dA1[128 x 64] = G2[128 x 64] W2[64 x 64]; W2 read MN-major (MN = h1, K = h2)
    ok = run([&] {
      for (int ks = 0; ks < kHid / 16; ++ks)
        mma(tmem + kColD1, desc_k(sg2, kTile, ks), desc_mn(sw2, kHid, ks), idesc(128, kHid, false, true), ks > 0);
    });
    if (!ok) break;
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16], a[16];
      tmem_ld16(tmem + lane_off + kColD1 + c0, v);
      ld8(S.a1, tid, c0, kTile, a);
      ld8(S.a1, tid, c0 + 8, kTile, a + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = a[i] > 0.f ? v[i] : 0.f;
      st8(S.g1, tid, c0, kTile, v);
      st8(S.g1, tid, c0 + 8, kTile, v + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float t = warp_sum(v[i]);
        if (lane == 0) S.gb1[warp][c0 + i] += t;
      }
    }
    // Weight gradients, reduced over the tile's 128 rays (K) and accumulated over this
    // CTA's tiles in TMEM (M = 64). Both operands are tiles read MN-major (K = ray).
    const uint32_t acc = tiles_done > 1 ? 1u : 0u;
    ok = run([&] {
      for (int ks = 0; ks < kTile / 16; ++ks) {
        const uint32_t a = uint32_t(ks > 0) | acc;
        // dW1[h1][in] += G1^T A0
        mma(tmem + kColGW1, desc_mn(sg1, kTile, ks), desc_mn(sa0, kTile, ks), idesc(64, kIn, true, true), a);
        // dW2[h2][h1] += G2^T A1
        mma(tmem + kColGW2, desc_mn(sg2, kTile, ks), desc_mn(sa1, kTile, ks), idesc(64, kHid, true, true), a);
        // dW3^T[h2][out] += A2^T G3
        mma(tmem + kColGW3, desc_mn(sa2, kTile, ks), desc_mn(sg3, kTile, ks), idesc(64, kOut, true, true), a);
      }
    });
    if (!ok) break;
  }

  if (TRAIN && ok && tiles_done > 0) {
    // M = 64 accumulators: row m lives in TMEM lane (m % 16) + 32 (m / 16), so lanes 0..15
    // of warp w hold rows 16 w .. 16 w + 15.
    float* out = P.partial + int64_t(blockIdx.x) * (kMlpParams + 1);
    const int m = warp * 16 + lane;
#pragma unroll
    for (int c0 = 0; c0 < kIn; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_off + kColGW1 + c0, v);
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < 16; ++i) out[kOffW1 + m * kIn + c0 + i] = v[i];
    }
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_off + kColGW2 + c0, v);
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < 16; ++i) out[kOffW2 + m * kHid + c0 + i] = v[i];
    }
    {
      float v[16];
      tmem_ld16(tmem + lane_off + kColGW3, v);  // dW3^T: row m = h2, column = output
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < kOut; ++i) out[kOffW3 + i * kHid + m] = v[i];
    }
    __syncthreads();
    if (tid < kHid) {
      out[kOffB1 + tid] = ((S.gb1[0][tid] + S.gb1[1][tid]) + S.gb1[2][tid]) + S.gb1[3][tid];
      out[kOffB2 + tid] = ((S.gb2[0][tid] + S.gb2[1][tid]) + S.gb2[2][tid]) + S.gb2[3][tid];
    }
    if (tid < kOut) out[kOffB3 + tid] = ((S.gb3[0][tid] + S.gb3[1][tid]) + S.gb3[2][tid]) + S.gb3[3][tid];
    if (tid == 0) out[kMlpParams] = ((S.loss[0] + S.loss[1]) + S.loss[2]) + S.loss[3];
  }
  if (!ok) {
    // let MMAs still in flight finish (bounded, at the full limit) before TMEM is freed
    mbar_wait(&S.bar, pending, kWaitClocks);
    if (tid == 0) atomicExch(P.error, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// Sum of the per-CTA partial gradients (and losses) in CTA order.
__global__ void k_mlp_reduce(const float* __restrict__ partial, int grid, float* __restrict__ grads,
                             float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kMlpParams) return;
  float s = 0.f;
  for (int b = 0; b < grid; ++b) s += partial[int64_t(b) * (kMlpParams + 1) + i];
  if (i < kMlpParams) grads[i] = s;
  else if (loss) *loss = s;
}

// Adam on the fp32 master parameters; refreshes the bf16 weight copies.
__global__ void k_mlp_adam(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                           float* __restrict__ v, __nv_bfloat16* __restrict__ w1, __nv_bfloat16* __restrict__ w2,
                           __nv_bfloat16* __restrict__ w3, float lr, float b1, float b2, float eps, float bc1,
                           float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float g = grads[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float p = params[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  params[i] = p;
  const __nv_bfloat16 pb = __float2bfloat16_rn(p);
  if (i < kOffW2) w1[i - kOffW1] = pb;
  else if (i < kOffW3) w2[i - kOffW2] = pb;
  else if (i < kOffB1) w3[i - kOffW3] = pb;
}

__global__ void k_mlp_pack(const float* __restrict__ params, __nv_bfloat16* __restrict__ w1,
                           __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * kIn) w1[i] = __float2bfloat16_rn(params[kOffW1 + i]);
  if (i < kHid * kHid) w2[i] = __float2bfloat16_rn(params[kOffW2 + i]);
  if (i < kOut * kHid) w3[i] = __float2bfloat16_rn(params[kOffW3 + i]);
}

static_assert(kOffW2 == kOffW1 + kHid * kIn && kOffW3 == kOffW2 + kHid * kHid && kOffB1 == kOffW3 + kOut * kHid &&
                  kOffB2 == kOffB1 + kHid && kOffB3 == kOffB2 + kHid && kMlpParams == kOffB3 + kOut,
              "parameter block layout");
static_assert(sizeof(Smem) + 128 <= kTrainSmem, "training shared memory");
constexpr size_t kInferSmem = offsetof(Smem, a1) + 128;
static_assert(kInferCtasPerSm * (kInferSmem + 1024) <= 228 * 1024, "inference CTAs per SM");
static_assert(kInferCtasPerSm * kColsInfer <= 512, "inference TMEM columns per SM");
static_assert(offsetof(Smem, w1) % 128 == 0 && offsetof(Smem, a0) % 128 == 0 && offsetof(Smem, a1) % 128 == 0,
              "tiles aligned");
static_assert(kmaj(127, 63, 128) + 2 == kTile * kIn * 2, "tile layout covers the tile");

}  // namespace

cudaError_t launch_mlp(const MlpParams& P, bool train, int max_grid, cudaStream_t st) {
  if (P.num_samples == 0) return cudaSuccess;
  const size_t smem = train ? kTrainSmem : kInferSmem;
  auto kern = train ? k_mlp<true> : k_mlp<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int64_t ntiles = (P.num_samples + kTile - 1) / kTile;
  const int g = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, max_grid)));
  kern<<<g, 128, smem, st>>>(P);
  return cudaGetLastError();
}

int mlp_grid(int64_t num_samples, int max_grid) {
  const int64_t ntiles = (num_samples + kTile - 1) / kTile;
  return int(std::max<int64_t>(1, std::min<int64_t>(ntiles, max_grid)));
}

cudaError_t launch_mlp_reduce(const float* partial, int grid, float* grads, float* loss, cudaStream_t st) {
  k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256, 0, st>>>(partial, grid, grads, loss);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* params, const float* grads, float* m, float* v, void* w1, void* w2, void* w3,
                            float lr, float beta1, float beta2, float eps, int step, cudaStream_t st) {
  const float bc1 = 1.f - powf(beta1, float(step)), bc2 = 1.f - powf(beta2, float(step));
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, grads, m, v, static_cast<__nv_bfloat16*>(w1),
                                                       static_cast<__nv_bfloat16*>(w2), static_cast<__nv_bfloat16*>(w3),
                                                       lr, beta1, beta2, eps, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t launch_mlp_pack(const float* params, void* w1, void* w2, void* w3, cudaStream_t st) {
  k_mlp_pack<<<(kHid * kIn + 255) / 256, 256, 0, st>>>(params, static_cast<__nv_bfloat16*>(w1),
                                                      static_cast<__nv_bfloat16*>(w2), static_cast<__nv_bfloat16*>(w3));
  return cudaGetLastError();
}

}  // namespace ever
