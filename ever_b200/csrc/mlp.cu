// Ray-cost model: a 39 -> 64 -> 64 -> 2 ReLU MLP with BF16 weights and activations and
// FP32 accumulation, run on the 5th-generation tensor cores (tcgen05.mma with the
// accumulators in tensor memory), for inference and for training.
//
// Input encoding of a ray (o, d): p = (o - c) - ((o - c).d^) d^, the point of the ray's
// line closest to the scene centre c, times 1/scale; then x, sin(2^k pi x), cos(2^k pi x)
// for k = 0..5 per component: 3 + 36 = 39 features, zero-padded to 48 columns (the first
// layer's K; the parameter block keeps W1 64 wide, its columns 39.. are padding). Outputs:
// the cost the tracer logs per ray, [log(1 + consumed events), depth offset / scale].
//
// One persistent CTA per SM:
// - worker warpgroups (four for training, kInferWorkers for inference). Each takes its own tiles of 128 rays (the MMA's M): it
//   encodes a tile into shared memory, and after each layer's MMAs reads the accumulator
//   from tensor memory (bias, ReLU, bf16) into the next layer's operand tile. The rays of
//   its next tile are loaded into registers while the current tile's MMAs run.
// - inference: one elected thread of each warpgroup issues that warpgroup's MMAs, so the
//   warpgroups run unsynchronised and one's epilogue overlaps another's MMAs.
// - training: one more warp, the MMA warp. Its one thread issues every tcgen05.mma of the
//   CTA, serving the workers' requests (one layer or backward step of one tile each) in a
//   fixed round-robin order, so the gradient sums over the tiles have a fixed order;
//   tcgen05.commit signals the worker's completion barrier.
// The workers' CUDA-core work (encoding, epilogues) overlaps the other workers' MMAs.
// Operands live in shared memory in the canonical no-swizzle layouts: 8 x 8 bf16 core
// matrices of 128 contiguous bytes. Activation tiles [ray][unit] are K-major operands of
// the layer products; the same bytes are the MN-major operands of the weight-gradient
// products, which reduce over rays. Training accumulates the weight and bias gradients of
// all the CTA's tiles in tensor memory; the fixed service order makes the sums
// deterministic. Every wait is bounded and reports a timeout through an error flag.
#include <cstddef>

#include <cuda_bf16.h>

#include "common.cuh"
#include "internal.cuh"

namespace ever {
namespace {

constexpr int kTile = 128;  // rays per tile = MMA M
constexpr int kK0 = 48;     // first layer's K: the 39 features, a constant 1 (column 39), zeros
constexpr int kK1 = 80;     // second layer's K: the 64 hidden units, a constant 1 (column 64), zeros
constexpr int kFeat = 39;
constexpr int kIn = 64;     // row length of W1 in the parameter block
constexpr int kHid = 64;
constexpr int kOut = 16;    // padded output width (2 used)
constexpr int kOnes = 16;   // columns 64..79 of a hidden tile: the constant-1 column, then zeros
constexpr int kTrainWorkers = 4;  // shared memory holds four sets of training tiles
constexpr int kInferWorkers = 5;  // 20 warps: 98.9 us per 2M rays (4: 106.2, 6: 98.1 with spills)
constexpr int kMmaWarp = 4 * kTrainWorkers;  // training: the warp after the workers'
constexpr int kThreads = 32 * (kMmaWarp + 1);
// tensor-memory columns: worker w's layer accumulator at 64 w; training adds the
// weight- and bias-gradient accumulators (M = 64)
constexpr uint32_t kColGW1 = 256, kColGW2 = 320, kColGW3 = 384, kColGB1 = 400, kColGB2 = 416;
constexpr uint32_t kColsInfer = kInferWorkers <= 4 ? 256 : 512, kColsTrain = 512;
constexpr int kInferSteps = 3, kTrainSteps = 6;  // MMA requests per tile

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

// Potentially blocking test: the thread may sleep until the phase completes or about 0.1 ms
// (the suspend-time hint, in ns) has passed, so waiting threads leave the issue slots to
// the others instead of spinning.
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase), "r"(100000u)
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
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Barrier among the 128 threads of one worker warpgroup (ids 1.. ; 0 is __syncthreads).
__device__ __forceinline__ void worker_sync(int w) {
  asm volatile("bar.sync %0, 128;" ::"r"(w + 1) : "memory");
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

// Consecutive fp32 columns of this thread's TMEM lane.
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[N]);
template <>
__device__ __forceinline__ void tmem_ld<2>(uint32_t taddr, float (&v)[2]) {
  uint32_t r[2];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  v[0] = __uint_as_float(r[0]);
  v[1] = __uint_as_float(r[1]);
}
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
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
template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// bf16(relu(a)) of two columns, packed (column 2j in the low half): one converting,
// clamping cvt (the layer's bias is already in the accumulator).
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
// Sixteen consecutive bf16 columns (c0 % 8 == 0) of one row: two 16-byte shared stores.
__device__ __forceinline__ void st16(unsigned char* tile, int row, int c0, int rows, const uint32_t* w) {
  *reinterpret_cast<uint4*>(tile + kmaj(row, c0, rows)) = make_uint4(w[0], w[1], w[2], w[3]);
  *reinterpret_cast<uint4*>(tile + kmaj(row, c0 + 8, rows)) = make_uint4(w[4], w[5], w[6], w[7]);
}
// Eight consecutive bf16 columns as fp32.
__device__ __forceinline__ void ld8(const unsigned char* tile, int row, int c0, int rows, float* v) {
  const uint4 q = *reinterpret_cast<const uint4*>(tile + kmaj(row, c0, rows));
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

// sin(pi x) and cos(pi x): x = n + r with n the nearest integer and |r| <= 1/2 (exact in
// float), the hardware sine and cosine of pi r (|pi r| <= pi/2, absolute error about
// 2^-21), and the sign (-1)^n.
__device__ __forceinline__ void sincospi_reduced(float x, float& s, float& c) {
  const float n = rintf(x);
  const float r = x - n;
  float ps, pc;
  __sincosf(3.14159265358979f * r, &ps, &pc);
  // |x| < 2^24 here (larger inputs are already integers: r = 0); the parity of n flips both
  const uint32_t flip = (uint32_t(int(fminf(fabsf(n), 16777216.f))) & 1u) << 31;
  s = __uint_as_float(__float_as_uint(ps) ^ flip);
  c = __uint_as_float(__float_as_uint(pc) ^ flip);
}

// The 39 features of one ray, packed as bf16 pairs with zero padding to 48 columns.
__device__ __forceinline__ void encode_ray(const MlpParams& P, float ox, float oy, float oz, float dx, float dy,
                                           float dz, uint32_t (&w)[kK0 / 2]) {
  ox -= P.cx;
  oy -= P.cy;
  oz -= P.cz;
  const float n = __fsqrt_rn(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
  const float inv = n > 0.f ? __frcp_rn(n) : 0.f;
  dx *= inv;
  dy *= inv;
  dz *= inv;
  const float od = fmaf(oz, dz, fmaf(oy, dy, ox * dx));
  float x[3] = {fmaf(-od, dx, ox) * P.inv_scale, fmaf(-od, dy, oy) * P.inv_scale, fmaf(-od, dz, oz) * P.inv_scale};
#pragma unroll
  for (int i = 0; i < 3; ++i) x[i] = isfinite(x[i]) ? x[i] : 0.f;
  float f[kK0];
  // sin / cos of 2^q pi x from the reduced sincos at the lowest frequency and the double-angle
  // identities sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a (after five doublings the
  // error is a few 1e-6, far below the bf16 rounding the features go through)
  float sv[3], cv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    f[i] = x[i];
    sincospi_reduced(x[i], sv[i], cv[i]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      f[3 + 6 * q + i] = sv[i];
      f[6 + 6 * q + i] = cv[i];
      const float t = 2.f * sv[i];  // exact
      const float s2 = t * cv[i];
      cv[i] = fmaf(-t, sv[i], 1.f);
      sv[i] = s2;
    }
  }
#pragma unroll
  f[kFeat] = 1.f;  // multiplies the first layer's bias, held in W1's column 39
#pragma unroll
  for (int k = kFeat + 1; k < kK0; ++k) f[k] = 0.f;
#pragma unroll
  for (int j = 0; j < kK0 / 2; ++j) w[j] = pack_bf16x2(f[2 * j], f[2 * j + 1]);
}

// One worker's operand tiles. Inference: a0, then hidden 1 and 2 in h1. Training adds
// h2 and g3; the backward writes G2 over h2 and G1 over h1.
template <bool TRAIN>
struct WorkerTiles {
  __align__(128) unsigned char a0[kTile * kK0 * 2];  // encoding          [ray][48]
  __align__(128) unsigned char h1[kTile * kK1 * 2];  // hidden 1 (and 2)  [ray][80]
};
template <>
struct WorkerTiles<true> {
  __align__(128) unsigned char a0[kTile * kK0 * 2];
  __align__(128) unsigned char h1[kTile * kK1 * 2];  // hidden 1 / G1     [ray][80]
  __align__(128) unsigned char h2[kTile * kHid * 2];  // hidden 2 / G2     [ray][64]
  __align__(128) unsigned char g3[kTile * kOut * 2];  // dL/d output       [ray][16]
};

template <bool TRAIN>
struct Smem {
  float b3[kOut];
  float gb3[kMmaWarp][2], loss[kMmaWarp];  // per worker-warp sums (fixed order)
  uint64_t ready[TRAIN ? kTrainWorkers : kInferWorkers], done[TRAIN ? kTrainWorkers : kInferWorkers];
  int quit[TRAIN ? kTrainWorkers : kInferWorkers];
  int wfail[TRAIN ? kTrainWorkers : kInferWorkers];  // a wait of worker w ran out: it stops at its next barrier
  int abort;   // the MMA warp gave up
  int failed;  // a wait of this CTA ran out
  uint32_t tmem_base;
  __align__(128) unsigned char w1[kHid * kK0 * 2];   // [h1][48]  K-major, rows = output units; b1 in column 39
  __align__(128) unsigned char w2[kHid * kK1 * 2];   // [h2][80]: h1, then b2 in column 64
  __align__(128) unsigned char w3[kOut * kHid * 2];  // [out][h2]
  WorkerTiles<TRAIN> t[TRAIN ? kTrainWorkers : kInferWorkers];
};

struct RayIn {
  float o[3], d[3];
};
__device__ __forceinline__ RayIn load_ray(const MlpParams& P, int64_t s) {
  RayIn x{};
  if (s < P.num_samples && !P.feat) {
    const int64_t r = P.sample_idx ? int64_t(__ldg(P.sample_idx + s)) : s;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      x.o[i] = __ldg(P.rayo + 3 * r + i);
      x.d[i] = __ldg(P.rayd + 3 * r + i);
    }
  }
  return x;
}

// Threads of a CTA: the worker warpgroups, and for training the MMA warp.
template <bool TRAIN>
__host__ __device__ constexpr int threads_of() {
  return TRAIN ? kThreads : 32 * 4 * kInferWorkers;
}

// Which accumulators of the CTA's weight and bias gradients hold a sum already (the first
// MMA into each overwrites).
struct GradStarted {
  bool w3 = false, w2 = false, w1 = false;
};

// The MMAs of step q of worker w's current tile, issued by one thread:
// 0-2 the layers; training 3 dA2 (+ dW3), 4 dA1 (+ dW2, db2), 5 dW1, db1.
template <bool TRAIN>
__device__ __forceinline__ void issue_step(Smem<TRAIN>& S, uint32_t tmem, int w, int q, GradStarted& gs) {
  const uint32_t sw1 = smem_u32(S.w1), sw2 = smem_u32(S.w2), sw3 = smem_u32(S.w3);
  const uint32_t d = tmem + 64u * uint32_t(w);
  const uint32_t sa0 = smem_u32(S.t[w].a0), sh1 = smem_u32(S.t[w].h1);
  if (q == 0) {  // layer 1: D = A0 W1^T
#pragma unroll
    for (int ks = 0; ks < kK0 / 16; ++ks)
      mma(d, desc_k(sa0, kTile, ks), desc_k(sw1, kHid, ks), idesc(128, kHid, false, false), ks > 0);
    return;
  }
  if (q == 1) {  // layer 2: D = [H1 1] [W2 b2]^T
#pragma unroll
    for (int ks = 0; ks < kK1 / 16; ++ks)
      mma(d, desc_k(sh1, kTile, ks), desc_k(sw2, kHid, ks), idesc(128, kHid, false, false), ks > 0);
    return;
  }
  if constexpr (!TRAIN) {  // layer 3: D[., 0:16] = H2 W3^T (inference keeps H2 in h1)
#pragma unroll
    for (int ks = 0; ks < kHid / 16; ++ks)
      mma(d, desc_k(sh1, kTile, ks), desc_k(sw3, kOut, ks), idesc(128, kOut, false, false), ks > 0);
  } else {
    const uint32_t sh2 = smem_u32(S.t[w].h2), sg3 = smem_u32(S.t[w].g3);
    // columns 64..79 of h1 (the constant 1, then zeros), read MN-major: a [ray][16] operand
    const uint32_t sones = sh1 + kmaj(0, kHid, kTile);
    if (q == 2) {  // layer 3
      for (int ks = 0; ks < kHid / 16; ++ks)
        mma(d, desc_k(sh2, kTile, ks), desc_k(sw3, kOut, ks), idesc(128, kOut, false, false), ks > 0);
    } else if (q == 3) {
      // dA2[128 x 64] = G3[128 x 16] W3[16 x 64] (W3 read MN-major: MN = h2, K = out)
      mma(d, desc_k(sg3, kTile, 0), desc_mn(sw3, kOut, 0), idesc(128, kHid, false, true), 0);
      // dW3^T[h2][out] += A2^T G3 (both tiles MN-major, K = ray)
      for (int ks = 0; ks < kTile / 16; ++ks)
        mma(tmem + kColGW3, desc_mn(sh2, kTile, ks), desc_mn(sg3, kTile, ks), idesc(64, kOut, true, true),
            uint32_t(ks > 0 || gs.w3));
      gs.w3 = true;
    } else if (q == 4) {
      // dA1 = G2 W2 (W2 MN-major: MN = h1, K = h2); G2 lives in h2
      for (int ks = 0; ks < kHid / 16; ++ks)
        mma(d, desc_k(sh2, kTile, ks), desc_mn(sw2, kHid, ks), idesc(128, kHid, false, true), ks > 0);
      for (int ks = 0; ks < kTile / 16; ++ks) {
        const uint32_t acc = uint32_t(ks > 0 || gs.w2);
        // dW2[h2][h1] += G2^T A1
        mma(tmem + kColGW2, desc_mn(sh2, kTile, ks), desc_mn(sh1, kTile, ks), idesc(64, kHid, true, true), acc);
        // db2 (every column) += G2^T 1
        mma(tmem + kColGB2, desc_mn(sh2, kTile, ks), desc_mn(sones, kTile, ks), idesc(64, kOnes, true, true), acc);
      }
      gs.w2 = true;
    } else {
      // G1 lives in h1: dW1[h1][0:48] += G1^T A0, db1 += G1^T 1
      for (int ks = 0; ks < kTile / 16; ++ks) {
        const uint32_t acc = uint32_t(ks > 0 || gs.w1);
        mma(tmem + kColGW1, desc_mn(sh1, kTile, ks), desc_mn(sa0, kTile, ks), idesc(64, kK0, true, true), acc);
        mma(tmem + kColGB1, desc_mn(sh1, kTile, ks), desc_mn(sones, kTile, ks), idesc(64, kOnes, true, true), acc);
      }
      gs.w1 = true;
    }
  }
}

// Inference (TRAIN = false: predictions and cost bins) or the gradients of one training
// batch (TRAIN = true: each CTA writes its partial gradient and loss to P.partial).
template <bool TRAIN>
__global__ void __launch_bounds__(threads_of<TRAIN>(), 1) k_mlp(const MlpParams P) {
  constexpr int kThreadsT = threads_of<TRAIN>();
  constexpr int kWorkers = TRAIN ? kTrainWorkers : kInferWorkers;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem<TRAIN>& S = *reinterpret_cast<Smem<TRAIN>*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t kCols = TRAIN ? kColsTrain : kColsInfer;
  constexpr int kSteps = TRAIN ? kTrainSteps : kInferSteps;
  const int64_t ntiles = (P.num_samples + kTile - 1) / kTile;
  const long long wait_limit = P.wait_clocks > 0 ? P.wait_clocks : kWaitClocks;

  // weights into the canonical layouts (8 columns per 16-byte store), biases, barriers
  {
    const __nv_bfloat16* w1 = static_cast<const __nv_bfloat16*>(P.w1);
    const __nv_bfloat16* w2 = static_cast<const __nv_bfloat16*>(P.w2);
    const __nv_bfloat16* w3 = static_cast<const __nv_bfloat16*>(P.w3);
    // the hidden layers' biases go into the weight tiles, as bf16, in the column that meets
    // the operand's constant 1: b1 in W1's column 39, b2 in W2's column 64
    auto bf16_bits = [](float x) { return uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(x))); };
    for (int i = tid; i < kHid * kK0 / 8; i += kThreadsT) {
      const int o = i / (kK0 / 8), c0 = (i % (kK0 / 8)) * 8;
      uint4 q = *reinterpret_cast<const uint4*>(w1 + o * kIn + c0);
      if (c0 == kFeat / 8 * 8) q.w = (q.w & 0xFFFFu) | (bf16_bits(P.params[kOffB1 + o]) << 16);  // column 39
      *reinterpret_cast<uint4*>(S.w1 + kmaj(o, c0, kHid)) = q;
    }
    for (int i = tid; i < kHid * kK1 / 8; i += kThreadsT) {
      const int o = i / (kK1 / 8), c0 = (i % (kK1 / 8)) * 8;
      uint4 q = make_uint4(0u, 0u, 0u, 0u);
      if (c0 < kHid) q = *reinterpret_cast<const uint4*>(w2 + o * kHid + c0);
      else if (c0 == kHid) q.x = bf16_bits(P.params[kOffB2 + o]);  // column 64
      *reinterpret_cast<uint4*>(S.w2 + kmaj(o, c0, kHid)) = q;
    }
    for (int i = tid; i < kOut * kHid / 8; i += kThreadsT) {
      const int o = i / (kHid / 8), c0 = (i % (kHid / 8)) * 8;
      *reinterpret_cast<uint4*>(S.w3 + kmaj(o, c0, kOut)) = *reinterpret_cast<const uint4*>(w3 + o * kHid + c0);
    }
    // columns 64..79 of every worker's hidden tile: the constant 1, then zeros (never rewritten)
    for (int i = tid; i < kWorkers * kTile * 2; i += kThreadsT) {
      const int w = i / (2 * kTile), row = (i / 2) % kTile, c0 = kHid + 8 * (i & 1);
      *reinterpret_cast<uint4*>(S.t[w].h1 + kmaj(row, c0, kTile)) =
          make_uint4(c0 == kHid ? 0x3F80u : 0u, 0u, 0u, 0u);
    }
  }
  if (tid < kOut) S.b3[tid] = P.params[kOffB3 + tid];
  if (tid < kMmaWarp) {
    S.gb3[tid][0] = S.gb3[tid][1] = 0.f;
    S.loss[tid] = 0.f;
  }
  if (tid < kWorkers) S.quit[tid] = S.wfail[tid] = 0;
  if (tid == 0) {
    S.abort = 0;
    S.failed = 0;
    for (int w = 0; w < kWorkers; ++w) {
      mbar_init(&S.ready[w], 1);
      mbar_init(&S.done[w], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // tensor memory: the MMA warp's (training) or the first worker warp's (inference)
  constexpr int kAllocWarp = TRAIN ? kMmaWarp : 0;
  if (warp == kAllocWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  bool ok = true;

  if (TRAIN && warp == kMmaWarp) {
    // ---- MMA warp (training): one thread serves the workers' requests in round-robin
    // order, so the gradient accumulators sum the tiles in a fixed order
    if (lane == 0) {
      int64_t left[kWorkers];
      uint32_t rphase[kWorkers];
      int step[kWorkers];
      int64_t total = 0;
      for (int w = 0; w < kWorkers; ++w) {
        const int64_t first = int64_t(blockIdx.x) * kWorkers + w, stride = int64_t(gridDim.x) * kWorkers;
        left[w] = first < ntiles ? ((ntiles - 1 - first) / stride + 1) * kSteps : 0;
        total += left[w];
        rphase[w] = 0;
        step[w] = 0;
      }
      GradStarted gs;
      while (total > 0 && ok) {
        for (int w = 0; w < kWorkers && ok; ++w) {
          if (left[w] == 0) continue;
          // wait for the worker's operands (bounded; a worker that gave up stops being served)
          const long long t0 = clock64();
          bool got = false;
          while (!(got = mbar_try(&S.ready[w], rphase[w]))) {
            if (*reinterpret_cast<volatile int*>(&S.quit[w])) break;
            if (clock64() - t0 > kWaitClocks) {
              ok = false;
              break;
            }
          }
          if (!got) {
            total -= left[w];
            left[w] = 0;
            continue;
          }
          rphase[w] ^= 1u;
          tc_fence_after();
          issue_step<TRAIN>(S, tmem, w, step[w], gs);
          mma_commit(&S.done[w]);
          step[w] = step[w] + 1 == kSteps ? 0 : step[w] + 1;
          --left[w];
          --total;
        }
      }
      if (!ok) {
        atomicExch(P.error, 1);
        *reinterpret_cast<volatile int*>(&S.abort) = 1;
        *reinterpret_cast<volatile int*>(&S.failed) = 1;
      }
    }
    __syncwarp();
  } else {
    // ---- worker warpgroup g: rows of its tiles = its 128 threads; TMEM lanes = rows
    const int g = warp >> 2, row = tid & 127;
    const uint32_t lanes = uint32_t((warp & 3) * 32) << 16;
    const uint32_t dcol = tmem + lanes + 64u * uint32_t(g);
    WorkerTiles<TRAIN>& T = S.t[g];
    uint32_t dphase = 0;  // phase of the next completion on done[g]
    const int64_t stride = int64_t(gridDim.x) * kWorkers;
    int64_t tile = int64_t(blockIdx.x) * kWorkers + g;
    RayIn next = load_ray(P, tile * kTile + row);
    bool first = true;
    bool stop = false;  // the same on every thread of the warpgroup (read after its barriers)
    GradStarted none;   // inference accumulates no gradients

    // bounded wait for the next completion of this worker's MMAs; a thread whose wait runs
    // out flags the warpgroup, which stops at its next barrier
    auto await_mma = [&]() {
      if (!mbar_wait(&S.done[g], dphase, wait_limit)) *reinterpret_cast<volatile int*>(&S.wfail[g]) = 1;
      dphase ^= 1u;
      tc_fence_after();
    };
    // hand the operand tiles of step q over: inference issues the step's MMAs itself (one
    // thread), training hands them to the MMA warp. False when the warpgroup must stop.
    auto hand_over = [&](int q) -> bool {
      fence_async_smem();
      tc_fence_before();
      worker_sync(g);
      if (*reinterpret_cast<volatile int*>(&S.wfail[g])) {
        stop = true;
        return false;
      }
      if (row == 0) {
        if constexpr (TRAIN) {
          mbar_arrive(&S.ready[g]);
        } else {
          tc_fence_after();
          issue_step<TRAIN>(S, tmem, g, q, none);
          mma_commit(&S.done[g]);
        }
      }
      return true;
    };

    for (; tile < ntiles && !stop; tile += stride) {
      const int64_t s = tile * kTile + row;
      const bool valid = s < P.num_samples;
      const int64_t r = valid ? (P.sample_idx ? int64_t(__ldg(P.sample_idx + s)) : s) : 0;
      // ---- encoding
      uint32_t enc[kK0 / 2];
      if (P.feat) {
        float f[kK0];
#pragma unroll
        for (int c = 0; c < kK0; ++c) f[c] = (valid && c < kFeat) ? __ldg(P.feat + r * kIn + c) : 0.f;
        f[kFeat] = 1.f;
#pragma unroll
        for (int j = 0; j < kK0 / 2; ++j) enc[j] = pack_bf16x2(f[2 * j], f[2 * j + 1]);
      } else {
        encode_ray(P, next.o[0], next.o[1], next.o[2], next.d[0], next.d[1], next.d[2], enc);
        if (!valid)
#pragma unroll
          for (int j = 0; j < kK0 / 2; ++j) enc[j] = 0u;
        next = load_ray(P, (tile + stride) * kTile + row);  // in flight during this tile's MMAs
      }
      // training: the previous tile's weight-gradient MMAs read a0 and h1
      if (TRAIN && !first) await_mma();
      first = false;
#pragma unroll
      for (int c = 0; c < kK0 / 8; ++c)
        *reinterpret_cast<uint4*>(T.a0 + kmaj(row, 8 * c, kTile)) =
            make_uint4(enc[4 * c], enc[4 * c + 1], enc[4 * c + 2], enc[4 * c + 3]);
      // ---- layers 1 and 2 (biases already in the accumulator): ReLU, bf16 into the next operand tile
#pragma unroll 1
      for (int layer = 0; layer < 2; ++layer) {
        if (!hand_over(layer)) break;
        await_mma();
        unsigned char* dst = (TRAIN && layer == 1) ? reinterpret_cast<WorkerTiles<true>&>(T).h2 : T.h1;
#pragma unroll
        for (int half = 0; half < 2; ++half) {  // 32 columns at a time (registers)
          float v[32];
          tmem_ld<32>(dcol + 32 * half, v);
          uint32_t h[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) h[j] = relu_bf16x2(v[2 * j], v[2 * j + 1]);
#pragma unroll
          for (int c = 0; c < 2; ++c) st16(dst, row, 32 * half + 16 * c, kTile, h + 8 * c);
        }
      }
      if (stop) break;
      // ---- layer 3
      if (!hand_over(2)) break;
      await_mma();
      float y2[2];
      tmem_ld<2>(dcol, y2);
      const float y0 = y2[0] + S.b3[0], y1 = y2[1] + S.b3[1];
      if (!TRAIN) {
        if (valid) {
          *reinterpret_cast<float2*>(P.pred + 2 * r) = make_float2(y0, y1);
          if (P.bins) P.bins[r] = uint8_t(int(y0 > P.thr[0]) + int(y0 > P.thr[1]) + int(y0 > P.thr[2]));
        }
        continue;
      }
      // ---- training: weighted squared error on the two outputs, mean over the batch
      WorkerTiles<true>& TT = reinterpret_cast<WorkerTiles<true>&>(T);
      float g0 = 0.f, g1 = 0.f, l = 0.f;
      if (valid) {
        const float e0 = y0 - P.target[2 * r], e1 = y1 - P.target[2 * r + 1];
        g0 = 2.f * P.loss_w0 * e0 * P.inv_batch;
        g1 = 2.f * P.loss_w1 * e1 * P.inv_batch;
        l = (P.loss_w0 * e0 * e0 + P.loss_w1 * e1 * e1) * P.inv_batch;
      }
      {
        const uint32_t gz[8] = {pack_bf16x2(g0, g1), 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        st16(TT.g3, row, 0, kTile, gz);
        const float t0 = warp_sum(g0), t1 = warp_sum(g1), tl = warp_sum(l);
        if (lane == 0) {
          S.gb3[warp][0] += t0;
          S.gb3[warp][1] += t1;
          S.loss[warp] += tl;
        }
      }
      // ---- dA2 = G3 W3 (and dW3): G2 = dA2 masked by A2 > 0, written over A2;
      // then dA1 = G2 W2 (and dW2, db2): G1 = dA1 masked by A1 > 0, written over A1
#pragma unroll 1
      for (int back = 0; back < 2; ++back) {
        if (!hand_over(3 + back)) break;
        await_mma();
        unsigned char* act = back == 0 ? TT.h2 : TT.h1;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          float v[32];
          tmem_ld<32>(dcol + 32 * half, v);
          uint32_t h[16];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float a[8];
            ld8(act, row, 32 * half + 8 * c, kTile, a);
#pragma unroll
            for (int i = 0; i < 4; ++i)
              h[4 * c + i] = pack_bf16x2(a[2 * i] > 0.f ? v[8 * c + 2 * i] : 0.f,
                                         a[2 * i + 1] > 0.f ? v[8 * c + 2 * i + 1] : 0.f);
          }
#pragma unroll
          for (int c = 0; c < 2; ++c) st16(act, row, 32 * half + 16 * c, kTile, h + 8 * c);
        }
      }
      if (stop) break;
      // ---- dW1, db1: handed over now, waited for before a0 / h1 are overwritten
      if (!hand_over(5)) break;
    }
    // training: the last tile's weight-gradient MMAs
    if (TRAIN && !stop && !first) await_mma();
    worker_sync(g);
    if (*reinterpret_cast<volatile int*>(&S.wfail[g])) stop = true;
    if (stop) {
      if (row == 0) atomicExch(P.error, 1);
      *reinterpret_cast<volatile int*>(&S.failed) = 1;
      // let this worker's MMAs in flight finish (bounded, at the full limit) before TMEM is
      // freed, unless the MMA warp itself gave up
      if (!*reinterpret_cast<volatile int*>(&S.abort)) mbar_wait(&S.done[g], dphase ^ 1u, kWaitClocks);
      worker_sync(g);
      if (row == 0) *reinterpret_cast<volatile int*>(&S.quit[g]) = 1;
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const bool cta_ok = *reinterpret_cast<volatile int*>(&S.failed) == 0;
  if (TRAIN && cta_ok && warp < 4) {
    // worker 0's warps read the M = 64 accumulators: row m lives in TMEM lane (m % 16) +
    // 32 (m / 16), so lanes 0..15 of warp w hold rows 16 w .. 16 w + 15
    float* out = P.partial + int64_t(blockIdx.x) * (kMlpParams + 1);
    const uint32_t lanes = uint32_t(warp * 32) << 16;
    const int m = warp * 16 + lane;
    const bool any = int64_t(blockIdx.x) * kWorkers < ntiles;  // this CTA had tiles
#pragma unroll
    for (int c0 = 0; c0 < kIn; c0 += 16) {
      float v[16];
      if (c0 < kK0) tmem_ld<16>(tmem + lanes + kColGW1 + c0, v);
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < 16; ++i) out[kOffW1 + m * kIn + c0 + i] = (any && c0 + i < kFeat) ? v[i] : 0.f;
    }
#pragma unroll
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld<16>(tmem + lanes + kColGW2 + c0, v);
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < 16; ++i) out[kOffW2 + m * kHid + c0 + i] = any ? v[i] : 0.f;
    }
    {
      float v[16];
      tmem_ld<16>(tmem + lanes + kColGW3, v);  // dW3^T: row m = h2, column = output
      if (lane < 16)
#pragma unroll
        for (int i = 0; i < kOut; ++i) out[kOffW3 + i * kHid + m] = any ? v[i] : 0.f;
    }
    {
      float v1[16], v2[16];
      tmem_ld<16>(tmem + lanes + kColGB1, v1);
      tmem_ld<16>(tmem + lanes + kColGB2, v2);
      if (lane < 16) {
        out[kOffB1 + m] = any ? v1[0] : 0.f;
        out[kOffB2 + m] = any ? v2[0] : 0.f;
      }
    }
    if (tid < kOut) {
      float t = 0.f;
      if (tid < 2)
        for (int w = 0; w < kMmaWarp; ++w) t += S.gb3[w][tid];
      out[kOffB3 + tid] = t;
    }
    if (tid == 0) {
      float t = 0.f;
      for (int w = 0; w < kMmaWarp; ++w) t += S.loss[w];
      out[kMlpParams] = t;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kAllocWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
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
constexpr size_t kInferSmem = sizeof(Smem<false>) + 128;
constexpr size_t kTrainSmem = sizeof(Smem<true>) + 128;
static_assert(kTrainSmem <= 227 * 1024, "training shared memory");
static_assert(kInferSmem <= 227 * 1024, "inference shared memory");
static_assert(kInferWorkers * 64 <= int(kColsInfer) && kColGB2 + kOnes <= kColsTrain && kTrainWorkers * 64 <= int(kColGW1),
              "tensor-memory columns");
static_assert(offsetof(Smem<true>, w1) % 128 == 0 && offsetof(Smem<true>, t) % 128 == 0 &&
                  offsetof(Smem<false>, t) % 128 == 0 && sizeof(WorkerTiles<true>) % 128 == 0 &&
                  sizeof(WorkerTiles<false>) % 128 == 0,
              "tiles aligned");
static_assert(kmaj(127, 63, 128) + 2 == kTile * kHid * 2 && kmaj(127, 47, 128) + 2 == kTile * kK0 * 2 &&
                  kmaj(127, 79, 128) + 2 == kTile * kK1 * 2 && kmaj(63, 79, 64) + 2 == kHid * kK1 * 2,
              "tile layout covers the tile");
static_assert(kThreads <= 1024 && 128 * kInferWorkers <= 1024 && kInferWorkers <= 15, "block size and named barriers");

}  // namespace

int mlp_grid(int64_t num_samples, int max_grid, bool train) {
  const int64_t ntiles = (num_samples + kTile - 1) / kTile;
  // training: two tiles per worker, so the warpgroups of a CTA overlap their steps; inference:
  // every SM, as many tiles per worker as it takes
  const int64_t per_cta = train ? 2 * kTrainWorkers : kInferWorkers;
  return int(std::max<int64_t>(1, std::min<int64_t>((ntiles + per_cta - 1) / per_cta, max_grid)));
}

cudaError_t launch_mlp(const MlpParams& P, bool train, int grid, cudaStream_t st) {
  if (P.num_samples == 0) return cudaSuccess;
  const size_t smem = train ? kTrainSmem : kInferSmem;
  auto kern = train ? k_mlp<true> : k_mlp<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  kern<<<grid, train ? threads_of<true>() : threads_of<false>(), smem, st>>>(P);
  return cudaGetLastError();
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
