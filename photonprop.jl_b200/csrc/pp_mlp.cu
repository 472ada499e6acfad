// Learned surrogate: MLP 4 -> 128 -> 128 -> 128 -> 5 with GELU, on sm_100a.
//
// Every CTA owns a tile of 128 rows (queries), one row per thread (4 warps).
// The 128 x 128 layers run on the 5th-generation tensor cores: one thread
// issues eight tcgen05.mma (M = N = 128, K = 16, BF16 inputs, FP32
// accumulation in tensor memory) per layer, commits them to an mbarrier, and
// every warp reads its 32 rows back with tcgen05.ld; bias, GELU and the BF16
// conversion of the next layer's operand are fused into that read-back.  The
// 4-wide input layer and the 5-wide output layer are too narrow for the tensor
// cores and run on the FP32 pipes with BF16-rounded weights.
//
// Operand tiles live in shared memory in the no-swizzle K-major canonical
// layout: 8-row x 16-byte core matrices, core matrices along K 128 bytes apart
// (leading byte offset), 8-row groups 2048 bytes apart (stride byte offset).
//
// Training (one fused kernel per 128-row tile): forward with the activations
// saved, masked-MSE loss, backward through all layers; the weight gradients of
// the 128 x 128 layers are tcgen05 GEMMs over the tile's rows (the transposed
// operands are written transposed into shared memory) accumulated across tiles
// with FP32 atomics; then an Adam kernel updates the FP32 master weights and
// rebuilds the BF16 tensor-core copies.
//
// Every mbarrier wait is bounded (iteration and clock limits); on expiry the
// kernel sets an error flag, stops issuing work and frees its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pp_internal.h"
#include "pp_special.cuh"

namespace mlp {

constexpr int H = 128, IN = 4, OUT = 5, TILE = 128, THREADS = 128;
// flat FP32 parameter vector
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * IN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * H, OFF_W4 = OFF_B3 + H, OFF_B4 = OFF_W4 + OUT * H,
              N_PARAMS = OFF_B4 + OUT;
constexpr int TILE_BYTES = TILE * H * 2;  // one BF16 128 x 128 operand tile

// element offset of (row, k) in a 128-column K-major canonical tile
__host__ __device__ __forceinline__ int tc_offset(int row, int k) {
  return (((row >> 3) * 16 + (k >> 3)) << 6) + ((row & 7) << 3) + (k & 7);
}

__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
  return 0.5f * z * (1.f + tanhf(u));
}
// Twice the inference GELU with the MUFU tanh (tanh.approx.f32, relative
// error below 2^-10, under the BF16 rounding that follows it), in four FP32
// operations: u = z (k + k c z^2), 2 GELU = z (1 + t).  The factor 1/2 is
// folded into the next layer's weights (exact: a power of two commutes with
// the BF16 rounding of both the weights and the activations).
__device__ __forceinline__ float gelu2_fast(float z) {
  const float u = z * fmaf(0.7978845608028654f * 0.044715f, z * z, 0.7978845608028654f);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return fmaf(z, t, z);
}
// The same arithmetic on two activations at once with sm_100's packed FP32
// instructions (round to nearest, so bit for bit the scalar result): half the
// FP32 issue slots of the epilogue.
__device__ __forceinline__ float2 gelu2_fast2(float2 z) {
  constexpr float k0 = 0.7978845608028654f, k1 = 0.7978845608028654f * 0.044715f;
  const float2 k = __ffma2_rn(__fmul2_rn(z, z), make_float2(k1, k1), make_float2(k0, k0));
  const float2 u = __fmul2_rn(z, k);
  float2 t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t.x) : "f"(u.x));
  asm("tanh.approx.f32 %0, %1;" : "=f"(t.y) : "f"(u.y));
  return __ffma2_rn(z, t, z);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
  const float t = tanhf(u);
  const float du = 0.7978845608028654f * fmaf(3.f * 0.044715f, z * z, 1.f);
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * du;
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor: no swizzle, K-major, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: D = F32, A = B = BF16, both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_128x128x16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the given phase parity: about 2^22 polls and ~4e9 cycles.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 4000000000ll) break;
  }
  return false;
}

// 32 FP32 accumulator columns [col, col+32) of this thread's row.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
        "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Tensor-memory allocation of 128 columns by warp 0; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot) {
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(smem_u32(slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
}
__device__ __forceinline__ void tmem_free(uint32_t taddr) {
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(taddr));
}

// Writes 8 consecutive columns [k8*8, k8*8+8) of `row` (FP32 values, rounded
// to BF16) into a canonical tile with one 16-byte store.
__device__ __forceinline__ void store8(__nv_bfloat16* tile, int row, int k8, const float* v) {
  __align__(16) __nv_bfloat162 p[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<int4*>(tile + tc_offset(row, k8 * 8)) = *reinterpret_cast<int4*>(p);
}

// D[128 x 128] (TMEM) = A (tile a, rows x K) * B^T (tile b, N rows x K), issued
// by thread 0 after every thread's shared-memory writes are fenced and synced.
// Returns false if the wait expired.
__device__ __forceinline__ bool tile_gemm(const __nv_bfloat16* a, const __nv_bfloat16* b, uint32_t tmem,
                                          uint32_t mbar, uint32_t& parity) {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    const uint32_t sa = smem_u32(a), sb = smem_u32(b);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      mma_128x128x16(tmem, smem_desc(sa + k * 256, 128, 2048), smem_desc(sb + k * 256, 128, 2048), k > 0);
    mma_commit(mbar);
  }
  const bool ok = mbar_wait(mbar, parity);
  parity ^= 1u;
  tc_fence_after();
  return ok;
}

// element offset of (row, k) in a K-major canonical tile of 16 columns
__host__ __device__ __forceinline__ int tc16_offset(int row, int k) {
  return (((row >> 3) * 2 + (k >> 3)) << 6) + ((row & 7) << 3) + (k & 7);
}
// Instruction descriptor for N = 16 (the padded output layer).
constexpr uint32_t kIdescN16 = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
__device__ __forceinline__ void mma_idesc(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// 16 FP32 accumulator columns [col, col+16) of this thread's row.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t lane_taddr(uint32_t tmem) { return tmem + ((threadIdx.x & ~31u) << 16); }

// ---------------------------------------------------------------------------
// Device parameter block.
struct DevParams {
  const float* p;        // FP32 master parameters (N_PARAMS)
  const float* w1r;      // BF16-rounded W1 [128][4]
  const float* w4r;      // BF16-rounded W4 [5][128]
  const __nv_bfloat16* w2tc;   // W2 as the B operand of h W2^T (canonical tile)
  const __nv_bfloat16* w3tc;
  const __nv_bfloat16* w1tc;   // W1 as the B operand of x W1^T: 128 rows x K 16 (4 used)
  const __nv_bfloat16* w4tc;   // W4 / 2 as the B operand of h W4^T: 16 rows (5 used) x K 128
  const __nv_bfloat16* w2h;    // W2 / 2, W3 / 2: inference B operands (they take 2 GELU)
  const __nv_bfloat16* w3h;
  const __nv_bfloat16* w2ttc;  // W2^T as the B operand of dz W2
  const __nv_bfloat16* w3ttc;
  const float* norm;     // x_mean[4], x_std[4], y_mean[5], y_std[5]
  int* error;
};

// Cooperative copy of a 32 KB canonical tile from global to shared memory.
__device__ __forceinline__ void load_tile(__nv_bfloat16* dst, const __nv_bfloat16* src) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(dst);
  for (int i = threadIdx.x; i < TILE_BYTES / 16; i += blockDim.x) d[i] = s[i];
}

// ---------------------------------------------------------------------------
// Inference: persistent over 128-row tiles.  x [n][4] raw features; out
// [5][n] (structure of arrays): raw = the de-standardised network outputs
// (ln(mu/N), logit w, ln a1, ln a2, ln theta); physical = (mu, w, a1, a2, theta).
//
// One CTA per SM with kGroups independent groups of 128 threads (four
// warps, one query row per thread).  The groups share the BF16 weight tiles
// of layers 2 and 3 in shared memory; each owns an activation tile, an
// mbarrier and 128 of the CTA's TMEM columns, and walks its own sequence of
// row tiles with group-local named barriers.  While one group's MMAs run on
// the tensor cores the others run their GELU epilogues on the FP32 and MUFU
// pipes, and sixteen warps per SM keep those pipes busy.  The biases of the
// hidden layers are added by the tensor cores and the GELU's factor 1/2 sits
// in the next layer's weights, so an activation costs four FP32 operations,
// one tanh and half a BF16 pack.
constexpr int kGroups = 4, INFER_THREADS = kGroups * THREADS;

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(THREADS) : "memory");
}
// Group barrier that also ANDs a flag over the group's threads, so that every
// thread of the group takes the same branch after a bounded wait.
__device__ __forceinline__ bool group_all(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(g + 1), "r"(THREADS)
      : "memory");
  return r != 0;
}

// The group's MMAs of one layer; kind 1: x (128 x 16) W1^T, one MMA (the
// bias rides in K columns 4 and 5: x has ones there, W1 the bias split into
// BF16 hi and lo); kind 2: h (128 x 128) W^T, eight MMAs, then a ninth,
// ones (128 x 16) times the bias tile, that adds the bias in the
// accumulator; kind 4: h W4^T with N = 16.  The epilogues then read z with
// its bias and spend no FP32 add on it.
__device__ __forceinline__ bool group_layer(int kind, const __nv_bfloat16* a, const __nv_bfloat16* b, uint32_t tmem,
                                            uint32_t mbar, uint32_t& parity, int g, int gt,
                                            const __nv_bfloat16* ones = nullptr,
                                            const __nv_bfloat16* bias = nullptr) {
  fence_async_smem();
  tc_fence_before();
  group_sync(g);
  tc_fence_after();
  if (gt == 0) {
    const uint32_t sa = smem_u32(a), sb = smem_u32(b);
    if (kind == 1) {
      mma_idesc(tmem, smem_desc(sa, 128, 256), smem_desc(sb, 128, 256), kIdesc, 0u);
    } else {
      const uint32_t idesc = kind == 4 ? kIdescN16 : kIdesc;
#pragma unroll
      for (int k = 0; k < 8; ++k)
        mma_idesc(tmem, smem_desc(sa + k * 256, 128, 2048), smem_desc(sb + k * 256, 128, 2048), idesc, k > 0);
      if (kind == 2)  // + 1 (bias hi, bias lo): the layer's bias, one more K = 16 step
        mma_idesc(tmem, smem_desc(smem_u32(ones), 128, 256), smem_desc(smem_u32(bias), 128, 256), kIdesc, 1u);
    }
    mma_commit(mbar);
  }
  const bool ok = group_all(g, mbar_wait(mbar, parity));
  parity ^= 1u;
  tc_fence_after();
  return ok;
}

__global__ void __launch_bounds__(INFER_THREADS, 1) infer_kernel(DevParams P, const float* __restrict__ x,
                                                                float* __restrict__ out, int64_t n, int physical) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* w3 = w2 + TILE * H;
  __nv_bfloat16* w1t = w3 + TILE * H;   // 128 x 16: W1 in K 0..3, b1 (hi, lo) in K 4, 5
  __nv_bfloat16* w4t = w1t + H * 16;    // 16 x 128
  __nv_bfloat16* b2t = w4t + 16 * H;    // 128 x 16: b2 (hi, lo) in K 0, 1
  __nv_bfloat16* b3t = b2t + H * 16;
  __nv_bfloat16* ones = b3t + H * 16;   // 128 x 16: 1 in K 0, 1
  __nv_bfloat16* acts = ones + TILE * 16;  // kGroups activation tiles (the x tile is the first 4 KB of one)
  float* b4 = reinterpret_cast<float*>(acts + kGroups * TILE * H);
  float* nrm = b4 + 8;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(nrm + 24);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbars + kGroups);

  const int t = threadIdx.x;
  const int g = t >> 7, gt = t & (THREADS - 1);  // group, thread (= row) within the group
  load_tile(w2, P.w2h);
  load_tile(w3, P.w3h);
  {
    const int4* s1 = reinterpret_cast<const int4*>(P.w1tc);
    int4* d1 = reinterpret_cast<int4*>(w1t);
    for (int i = t; i < 4 * H * 16 * 2 / 16; i += INFER_THREADS) d1[i] = s1[i];  // W1, W4, b2, b3 tiles
  }
  for (int i = t; i < TILE * 16 / 8; i += INFER_THREADS) {  // the ones tile, 8 columns per 16-byte word
    const int row = i >> 1, k8 = i & 1;
    const uint32_t one2 = 0x3F803F80u;  // two BF16 ones
    *reinterpret_cast<int4*>(ones + tc16_offset(row, k8 * 8)) =
        k8 == 0 ? make_int4((int)one2, 0, 0, 0) : make_int4(0, 0, 0, 0);
  }
  if (t < OUT) b4[t] = P.p[OFF_B4 + t];
  if (t < 18) nrm[t] = P.norm[t];
  if (t < IN) nrm[18 + t] = 1.f / P.norm[4 + t];  // feature scales as reciprocals: no division per row
  if (t < kGroups) mbar_init(smem_u32(mbars + t));
  if ((t >> 5) == 0) {  // all 512 columns: 128 per group
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tslot;
  const uint32_t tmem = tmem_base + (uint32_t)(g * 128);           // the group's columns
  const uint32_t taddr = tmem + ((uint32_t)(gt & ~31) << 16);      // this warp's 32 lanes
  __nv_bfloat16* act = acts + g * TILE * H;
  const uint32_t mb = smem_u32(mbars + g);
  uint32_t parity = 0;
  bool ok = true;

  const int64_t tile_step = (int64_t)gridDim.x * kGroups;
  // the row's features, loaded one tile ahead so that the global loads
  // overlap the previous tile's layers
  float xr[IN];
  {
    const int64_t row0 = ((int64_t)blockIdx.x * kGroups + g) * TILE + gt;
#pragma unroll
    for (int j = 0; j < IN; ++j) xr[j] = row0 < n ? x[row0 * IN + j] : nrm[j];
  }
  for (int64_t tile = (int64_t)blockIdx.x * kGroups + g; ok && tile * TILE < n; tile += tile_step) {
    const int64_t row = tile * TILE + gt;
    const bool valid = row < n;
    float xn[8];
    float lnN = 0.f;
#pragma unroll
    for (int j = 0; j < IN; ++j) {
      const float raw = xr[j];
      if (j == 2) lnN = raw * 2.302585092994046f;
      xn[j] = (raw - nrm[j]) * nrm[18 + j];
    }
    {
      const int64_t nrow = row + tile_step * TILE;
#pragma unroll
      for (int j = 0; j < IN; ++j) xr[j] = nrow < n ? x[nrow * IN + j] : nrm[j];
    }
    xn[IN] = 1.f;  // times the bias columns of W1
    xn[IN + 1] = 1.f;
#pragma unroll
    for (int j = IN + 2; j < 8; ++j) xn[j] = 0.f;
    // layer 1 (tensor cores, K = 4 padded to 16): the row's x in the x tile
    {
      __align__(16) __nv_bfloat162 p[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(xn[2 * i], xn[2 * i + 1]);
      *reinterpret_cast<int4*>(act + tc16_offset(gt, 0)) = *reinterpret_cast<int4*>(p);
      *reinterpret_cast<int4*>(act + tc16_offset(gt, 8)) = make_int4(0, 0, 0, 0);
    }
    ok = group_layer(1, act, w1t, tmem, mb, parity, g, gt);
    if (!ok) break;
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(taddr + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; i += 2) {
        const float2 r = gelu2_fast2(make_float2(v[i], v[i + 1]));
        v[i] = r.x;
        v[i + 1] = r.y;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) store8(act, gt, c * 4 + q, v + q * 8);
    }
    // layer 2
    ok = group_layer(2, act, w2, tmem, mb, parity, g, gt, ones, b2t);
    if (!ok) break;
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(taddr + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; i += 2) {
        const float2 r = gelu2_fast2(make_float2(v[i], v[i + 1]));
        v[i] = r.x;
        v[i + 1] = r.y;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) store8(act, gt, c * 4 + q, v + q * 8);
    }
    // layer 3
    ok = group_layer(2, act, w3, tmem, mb, parity, g, gt, ones, b3t);
    if (!ok) break;
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(taddr + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; i += 2) {
        const float2 r = gelu2_fast2(make_float2(v[i], v[i + 1]));
        v[i] = r.x;
        v[i + 1] = r.y;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) store8(act, gt, c * 4 + q, v + q * 8);
    }
    // layer 4 (tensor cores, N = 5 padded to 16)
    ok = group_layer(4, act, w4t, tmem, mb, parity, g, gt);
    if (!ok) break;
    float y[16];
    tmem_ld16(taddr, y);
    if (valid) {
#pragma unroll
      for (int j = 0; j < OUT; ++j) {
        float o = fmaf(y[j] + b4[j], nrm[13 + j], nrm[8 + j]);
        if (physical) {
          if (j == 0) o = expf(o + lnN);
          else if (j == 1) o = 1.f / (1.f + expf(-o));
          else o = expf(o);
        }
        out[(int64_t)j * n + row] = o;
      }
    }
  }
  if (!ok && gt == 0) atomicExch(P.error, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if ((t >> 5) == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem_base));
}

// ---------------------------------------------------------------------------
// Training, one CTA per 128-row tile.  xn [n][4] standardised features,
// yt [n][5] standardised targets, mask [n][5]; grads (N_PARAMS) accumulated
// with atomics; loss_sum += sum of mask * (y - t)^2; inv_count = 1 / sum(mask).
// Scratch: z [3][n][128] FP32 pre-activations, h [3][n][128] BF16 activations.
__global__ void __launch_bounds__(THREADS, 1) train_kernel(DevParams P, const float* __restrict__ xn,
                                                          const float* __restrict__ yt,
                                                          const float* __restrict__ mask, int64_t n,
                                                          float inv_count, float* __restrict__ grad,
                                                          float* __restrict__ loss_sum, float* __restrict__ zs,
                                                          __nv_bfloat16* __restrict__ hs) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __nv_bfloat16* ta = reinterpret_cast<__nv_bfloat16*>(smem_raw);  // A operand
  __nv_bfloat16* tb = ta + TILE * H;                                 // B operand
  __nv_bfloat16* tt = tb + TILE * H;                                 // transposed gradient (A of dW)
  float* w1 = reinterpret_cast<float*>(tt + TILE * H);
  float* w4 = w1 + H * IN;
  float* b4 = w4 + OUT * H;
  float* dys = b4 + 8;            // [128][5]
  float* red = dys + TILE * OUT;  // [4] loss partials
  uint64_t* mbar = reinterpret_cast<uint64_t*>(red + 8);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);

  const int t = threadIdx.x;
  const int64_t row = (int64_t)blockIdx.x * TILE + t;
  const bool valid = row < n;
  for (int i = t; i < H * IN; i += THREADS) w1[i] = P.w1r[i];
  for (int i = t; i < OUT * H; i += THREADS) w4[i] = P.w4r[i];
  if (t < OUT) b4[t] = P.p[OFF_B4 + t];
  if (t == 0) mbar_init(smem_u32(mbar));
  tmem_alloc(tslot);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t mb = smem_u32(mbar);
  uint32_t parity = 0;
  bool ok = true;
  const int64_t rr = valid ? row : 0;  // scratch row (invalid rows compute on zeros, contribute nothing)
  float* z1 = zs + rr * H;
  float* z2 = zs + (n + rr) * H;
  float* z3 = zs + (2 * n + rr) * H;
  __nv_bfloat16* h1 = hs + rr * H;
  __nv_bfloat16* h2 = hs + (n + rr) * H;
  __nv_bfloat16* h3 = hs + (2 * n + rr) * H;

  float x[IN];
#pragma unroll
  for (int j = 0; j < IN; ++j) x[j] = valid ? xn[row * IN + j] : 0.f;
  // ---- forward
  for (int k8 = 0; k8 < H / 8; ++k8) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int f = k8 * 8 + i;
      float z = P.p[OFF_B1 + f];
#pragma unroll
      for (int j = 0; j < IN; ++j) z = fmaf(w1[f * IN + j], bf16r(x[j]), z);
      if (valid) z1[f] = z;
      v[i] = gelu(z);
      if (valid) h1[f] = __float2bfloat16_rn(v[i]);
    }
    store8(ta, t, k8, v);
  }
  load_tile(tb, P.w2tc);
  ok = tile_gemm(ta, tb, tmem, mb, parity);
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int f = c * 32 + i;
        const float z = v[i] + P.p[OFF_B2 + f];
        if (valid) z2[f] = z;
        v[i] = gelu(z);
        if (valid) h2[f] = __float2bfloat16_rn(v[i]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) store8(ta, t, c * 4 + q, v + q * 8);
    }
    tc_fence_before();
    __syncthreads();  // every warp has read the accumulator and the B tile is free
    load_tile(tb, P.w3tc);
    ok = tile_gemm(ta, tb, tmem, mb, parity);
  }
  float y[OUT];
#pragma unroll
  for (int j = 0; j < OUT; ++j) y[j] = b4[j];
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int f = c * 32 + i;
        const float z = v[i] + P.p[OFF_B3 + f];
        if (valid) z3[f] = z;
        const float hb = bf16r(gelu(z));
        if (valid) h3[f] = __float2bfloat16_rn(hb);
#pragma unroll
        for (int j = 0; j < OUT; ++j) y[j] = fmaf(w4[j * H + f], hb, y[j]);
      }
    }
  }
  // ---- loss and output gradient
  float lsum = 0.f;
#pragma unroll
  for (int j = 0; j < OUT; ++j) {
    const float m = valid ? mask[row * OUT + j] : 0.f;
    const float e = valid ? y[j] - yt[row * OUT + j] : 0.f;
    lsum += m * e * e;
    dys[t * OUT + j] = 2.f * m * e * inv_count;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0) red[t >> 5] = lsum;
  tc_fence_before();
  __syncthreads();
  if (t == 0) atomicAdd(loss_sum, red[0] + red[1] + red[2] + red[3]);
  // dW4, db4: thread t owns feature t
  {
    float acc[OUT] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int r = 0; r < TILE; ++r) {
      const int64_t gr = (int64_t)blockIdx.x * TILE + r;
      if (gr >= n) break;
      const float h = __bfloat162float(hs[(2 * n + gr) * H + t]);
#pragma unroll
      for (int j = 0; j < OUT; ++j) acc[j] = fmaf(dys[r * OUT + j], h, acc[j]);
    }
#pragma unroll
    for (int j = 0; j < OUT; ++j) atomicAdd(grad + OFF_W4 + j * H + t, acc[j]);
    if (t < OUT) {
      float s = 0.f;
      for (int r = 0; r < TILE; ++r) s += dys[r * OUT + t];
      atomicAdd(grad + OFF_B4 + t, s);
    }
  }
  // dz3 = (dy W4) * gelu'(z3): natural into ta, transposed into tt
  for (int k8 = 0; k8 < H / 8; ++k8) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int f = k8 * 8 + i;
      float dh = 0.f;
#pragma unroll
      for (int j = 0; j < OUT; ++j) dh = fmaf(dys[t * OUT + j], w4[j * H + f], dh);
      const float dz = valid ? dh * gelu_grad(z3[f]) : 0.f;
      v[i] = dz;
      if (valid) atomicAdd(grad + OFF_B3 + f, dz);
      tt[tc_offset(f, t)] = __float2bfloat16_rn(dz);
    }
    store8(ta, t, k8, v);
  }
  // h2 transposed into tb: dW3 = dz3^T h2 over the tile's rows
  for (int f = 0; f < H; ++f) tb[tc_offset(f, t)] = valid ? h2[f] : __float2bfloat16_rn(0.f);
  if (ok) ok = tile_gemm(tt, tb, tmem, mb, parity);
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) atomicAdd(grad + OFF_W3 + t * H + c * 32 + i, v[i]);
    }
    tc_fence_before();
    __syncthreads();
    load_tile(tb, P.w3ttc);  // dh2 = dz3 W3
    ok = tile_gemm(ta, tb, tmem, mb, parity);
  }
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int f = c * 32 + i;
        const float dz = valid ? v[i] * gelu_grad(z2[f]) : 0.f;
        v[i] = dz;
        if (valid) atomicAdd(grad + OFF_B2 + f, dz);
        tt[tc_offset(f, t)] = __float2bfloat16_rn(dz);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) store8(ta, t, c * 4 + q, v + q * 8);
    }
    tc_fence_before();
    __syncthreads();
    for (int f = 0; f < H; ++f) tb[tc_offset(f, t)] = valid ? h1[f] : __float2bfloat16_rn(0.f);
    ok = tile_gemm(tt, tb, tmem, mb, parity);  // dW2 = dz2^T h1
  }
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) atomicAdd(grad + OFF_W2 + t * H + c * 32 + i, v[i]);
    }
    tc_fence_before();
    __syncthreads();
    load_tile(tb, P.w2ttc);  // dh1 = dz2 W2
    ok = tile_gemm(ta, tb, tmem, mb, parity);
  }
  if (ok) {
    for (int c = 0; c < 4; ++c) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + c * 32, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int f = c * 32 + i;
        const float dz = valid ? v[i] * gelu_grad(z1[f]) : 0.f;
        if (valid) {
          atomicAdd(grad + OFF_B1 + f, dz);
#pragma unroll
          for (int j = 0; j < IN; ++j) atomicAdd(grad + OFF_W1 + f * IN + j, dz * bf16r(x[j]));
        }
      }
    }
  }
  if (!ok && t == 0) atomicExch(P.error, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  tmem_free(tmem);
}

// Adam on the FP32 master parameters (gradients zeroed afterwards).
__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N_PARAMS; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    g[i] = 0.f;
  }
}

// BF16 tensor-core copies and BF16-rounded narrow layers from the masters.
__global__ void prepare_kernel(const float* __restrict__ p, float* __restrict__ w1r, float* __restrict__ w4r,
                               __nv_bfloat16* __restrict__ w2tc, __nv_bfloat16* __restrict__ w3tc,
                               __nv_bfloat16* __restrict__ w2ttc, __nv_bfloat16* __restrict__ w3ttc,
                               __nv_bfloat16* __restrict__ w1tc, __nv_bfloat16* __restrict__ w4tc,
                               __nv_bfloat16* __restrict__ b2t, __nv_bfloat16* __restrict__ b3t,
                               __nv_bfloat16* __restrict__ w2h, __nv_bfloat16* __restrict__ w3h) {
  // a bias as two BF16 columns, hi + lo = b to about 2^-16 relative
  auto split = [](float b, int part) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(b);
    return part == 0 ? hi : __float2bfloat16_rn(b - __bfloat162float(hi));
  };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < H * 16; i += gridDim.x * blockDim.x) {
    const int o = i / 16, k = i % 16;  // layer 1: rows = out (128), K = in (4 of 16), then b1 hi, lo
    w1tc[tc16_offset(o, k)] = k < IN ? __float2bfloat16_rn(p[OFF_W1 + o * IN + k])
                              : k < IN + 2 ? split(p[OFF_B1 + o], k - IN) : __float2bfloat16_rn(0.f);
    b2t[tc16_offset(o, k)] = k < 2 ? split(p[OFF_B2 + o], k) : __float2bfloat16_rn(0.f);
    b3t[tc16_offset(o, k)] = k < 2 ? split(p[OFF_B3 + o], k) : __float2bfloat16_rn(0.f);
    const int r = i / H, kk = i % H;   // layer 4: rows = out (5 of 16), K = in (128); takes 2 GELU
    w4tc[tc_offset(r, kk)] = __float2bfloat16_rn(r < OUT ? 0.5f * p[OFF_W4 + r * H + kk] : 0.f);
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < H * H; i += gridDim.x * blockDim.x) {
    const int o = i / H, k = i % H;
    w2tc[tc_offset(o, k)] = __float2bfloat16_rn(p[OFF_W2 + i]);   // B of h W2^T: rows = out, K = in
    w3tc[tc_offset(o, k)] = __float2bfloat16_rn(p[OFF_W3 + i]);
    w2ttc[tc_offset(k, o)] = __float2bfloat16_rn(p[OFF_W2 + i]);  // B of dz W2: rows = in, K = out
    w3ttc[tc_offset(k, o)] = __float2bfloat16_rn(p[OFF_W3 + i]);
    w2h[tc_offset(o, k)] = __float2bfloat16_rn(0.5f * p[OFF_W2 + i]);
    w3h[tc_offset(o, k)] = __float2bfloat16_rn(0.5f * p[OFF_W3 + i]);
    if (i < H * IN) w1r[i] = bf16r(p[OFF_W1 + i]);
    if (i < OUT * H) w4r[i] = bf16r(p[OFF_W4 + i]);
  }
}

// One 128 x 128 x 128 GEMM through the tensor-core path (descriptor self-test):
// c[i][j] = sum_k a[i][k] b[j][k], a and b BF16 row-major, c FP32.
__global__ void __launch_bounds__(THREADS, 1) gemm_test_kernel(const __nv_bfloat16* __restrict__ a,
                                                              const __nv_bfloat16* __restrict__ b,
                                                              float* __restrict__ c, int* error) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __nv_bfloat16* ta = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* tb = ta + TILE * H;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tb + TILE * H);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int t = threadIdx.x;
  for (int k = 0; k < H; ++k) {
    ta[tc_offset(t, k)] = a[t * H + k];
    tb[tc_offset(t, k)] = b[t * H + k];
  }
  if (t == 0) mbar_init(smem_u32(mbar));
  tmem_alloc(tslot);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  uint32_t parity = 0;
  const bool ok = tile_gemm(ta, tb, tmem, smem_u32(mbar), parity);
  if (ok) {
    for (int q = 0; q < 4; ++q) {
      float v[32];
      tmem_ld32(lane_taddr(tmem) + q * 32, v);
      for (int i = 0; i < 32; ++i) c[t * H + q * 32 + i] = v[i];
    }
  } else if (t == 0) {
    atomicExch(error, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  tmem_free(tmem);
}

// ---------------------------------------------------------------------------
// Two-component Gamma mixture w G(a1, theta) + (1 - w) G(a2, theta) fitted by
// weighted EM to each pair's arrival-time histogram, as a function of the
// time residual t - t_shift (bins with a positive residual only; the reference
// fits a single Gamma to the time residual, src/modelling.jl:52-79).  One warp
// per pair.  M step: theta = sum_k S1_k / sum_k a_k S0_k, then psi(a_k) =
// SL_k / S0_k - ln theta solved by Newton (psi and psi' from their asymptotic
// series after upward recurrence).  Output per pair: w, a1 <= a2, theta,
// mean log-likelihood per weight; NaNs when the histogram is empty.
using ppsf::digamma_d;
using ppsf::trigamma_d;

// a with psi(a) = y (Minka's initialisation, Newton steps).
__device__ double inv_digamma(double y) {
  double a = y >= -2.22 ? exp(y) + 0.5 : -1.0 / (y + 0.5772156649015329);
  for (int i = 0; i < 8; ++i) {
    a -= (digamma_d(a) - y) / trigamma_d(a);
    if (a < 1e-3) a = 1e-3;
  }
  return a;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void gamma_fit_kernel(const double* __restrict__ hist, int64_t n, int bins, float t0, float bw,
                                 const float* __restrict__ tshift, float* __restrict__ out, int iters) {
  const int64_t pair = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (pair >= n) return;  // whole warps exit together
  const double* h = hist + pair * bins;
  const double ts = tshift[pair];
  // moments for the initial guess
  double s0 = 0, s1 = 0, s2 = 0;
  for (int b = lane; b < bins; b += 32) {
    const double t = t0 + (b + 0.5) * bw - ts;
    if (t > 0 && h[b] > 0) {
      s0 += h[b];
      s1 += h[b] * t;
      s2 += h[b] * t * t;
    }
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  float* o = out + pair * 5;
  if (!(s0 > 0)) {
    if (lane < 5) o[lane] = __int_as_float(0x7fc00000);
    return;
  }
  const double m = s1 / s0, v = fmax(s2 / s0 - m * m, 1e-6 * m * m + 1e-12);
  const double a0 = fmax(m * m / v, 0.05);
  double w = 0.5, a1 = fmax(0.5 * a0, 0.02), a2 = 2.0 * a0, th = v / m;
  double ll = 0;
  for (int it = 0; it < iters; ++it) {
    const double lw1 = log(w), lw2 = log1p(-w), lth = log(th);
    const double c1 = lw1 - a1 * lth - lgamma(a1), c2 = lw2 - a2 * lth - lgamma(a2);
    double S0a = 0, S1a = 0, SLa = 0, S0b = 0, S1b = 0, SLb = 0, L = 0;
    for (int b = lane; b < bins; b += 32) {
      const double t = t0 + (b + 0.5) * bw - ts;
      const double hb = h[b];
      if (!(t > 0) || !(hb > 0)) continue;
      const double lt = log(t);
      const double p1 = c1 + (a1 - 1) * lt - t / th, p2 = c2 + (a2 - 1) * lt - t / th;
      const double mx = fmax(p1, p2);
      const double e1 = exp(p1 - mx), e2 = exp(p2 - mx);
      const double r1 = e1 / (e1 + e2);
      L += hb * (mx + log(e1 + e2));
      S0a += hb * r1;
      S1a += hb * r1 * t;
      SLa += hb * r1 * lt;
      S0b += hb * (1 - r1);
      S1b += hb * (1 - r1) * t;
      SLb += hb * (1 - r1) * lt;
    }
    S0a = warp_sum(S0a);
    S1a = warp_sum(S1a);
    SLa = warp_sum(SLa);
    S0b = warp_sum(S0b);
    S1b = warp_sum(S1b);
    SLb = warp_sum(SLb);
    ll = warp_sum(L) / s0;
    w = fmin(fmax(S0a / (S0a + S0b), 1e-4), 1 - 1e-4);
    for (int j = 0; j < 3; ++j) {
      th = (S1a + S1b) / (a1 * S0a + a2 * S0b);
      if (S0a > 0) a1 = inv_digamma(SLa / S0a - log(th));
      if (S0b > 0) a2 = inv_digamma(SLb / S0b - log(th));
    }
  }
  if (a1 > a2) {  // order the components
    const double x = a1;
    a1 = a2;
    a2 = x;
    w = 1 - w;
  }
  if (lane == 0) {
    o[0] = (float)w;
    o[1] = (float)a1;
    o[2] = (float)a2;
    o[3] = (float)th;
    o[4] = (float)ll;
  }
}

constexpr size_t kInferSmem = (2 + kGroups) * TILE_BYTES + 5 * H * 16 * 2 + (8 + 24) * 4 + 8 * kGroups + 16;
constexpr size_t kTrainSmem = 3 * TILE_BYTES + (H * IN + OUT * H + 8 + TILE * OUT + 8) * 4 + 16 + 16;
constexpr size_t kTestSmem = 2 * TILE_BYTES + 32;

}  // namespace mlp

// ---------------------------------------------------------------------------
// Host side.
struct pp_mlp {
  int device = 0;
  int sm_count = 0;
  std::mutex mu;
  float* d_params = nullptr;  // N_PARAMS
  float* d_grad = nullptr;
  float* d_m = nullptr;
  float* d_v = nullptr;
  float* d_w1r = nullptr;
  float* d_w4r = nullptr;
  __nv_bfloat16* d_tc = nullptr;  // 6 tiles of 128 x 128, then 4 of 128 x 16
  float* d_norm = nullptr;        // 18 (+ pad)
  int* d_error = nullptr;
  float* d_loss = nullptr;
  float* d_zs = nullptr;
  __nv_bfloat16* d_hs = nullptr;
  int64_t scratch_rows = 0;
  int64_t step = 0;
  std::string err;
};

namespace {
struct Guard {
  int prev = -1;
  explicit Guard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~Guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

mlp::DevParams dev_params(pp_mlp* m) {
  mlp::DevParams P;
  P.p = m->d_params;
  P.w1r = m->d_w1r;
  P.w4r = m->d_w4r;
  P.w2tc = m->d_tc;
  P.w3tc = m->d_tc + mlp::TILE * mlp::H;
  P.w2ttc = m->d_tc + 2 * mlp::TILE * mlp::H;
  P.w2h = m->d_tc + 4 * mlp::TILE * mlp::H;
  P.w3h = m->d_tc + 5 * mlp::TILE * mlp::H;
  P.w1tc = m->d_tc + 6 * mlp::TILE * mlp::H;
  P.w4tc = P.w1tc + mlp::H * 16;
  P.w3ttc = m->d_tc + 3 * mlp::TILE * mlp::H;
  P.norm = m->d_norm;
  P.error = m->d_error;
  return P;
}

cudaError_t prepare(pp_mlp* m, cudaStream_t s) {
  __nv_bfloat16* t = m->d_tc;
  constexpr int T = mlp::TILE * mlp::H, S = mlp::H * 16;
  mlp::prepare_kernel<<<64, 256, 0, s>>>(m->d_params, m->d_w1r, m->d_w4r, t, t + T, t + 2 * T, t + 3 * T, t + 6 * T,
                                         t + 6 * T + S, t + 6 * T + 2 * S, t + 6 * T + 3 * S, t + 4 * T, t + 5 * T);
  pp::count_launches(1);
  return cudaGetLastError();
}

pp_status fail(pp_mlp* m, pp_status s, const std::string& msg) {
  m->err = msg;
  return s;
}
}  // namespace

extern "C" {

pp_status pp_mlp_create(int device, uint64_t seed, pp_mlp** out) {
  if (!out) return PP_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return PP_ERR_ARG;
  }
  pp_mlp* m = new pp_mlp();
  m->device = device;
  Guard g(device);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  m->sm_count = prop.multiProcessorCount;
  cudaError_t e;
  if ((e = cudaMalloc(&m->d_params, mlp::N_PARAMS * 4)) || (e = cudaMalloc(&m->d_grad, mlp::N_PARAMS * 4)) ||
      (e = cudaMalloc(&m->d_m, mlp::N_PARAMS * 4)) || (e = cudaMalloc(&m->d_v, mlp::N_PARAMS * 4)) ||
      (e = cudaMalloc(&m->d_w1r, mlp::H * mlp::IN * 4)) || (e = cudaMalloc(&m->d_w4r, mlp::OUT * mlp::H * 4)) ||
      (e = cudaMalloc(&m->d_tc, 6 * mlp::TILE_BYTES + 4 * mlp::H * 16 * 2)) || (e = cudaMalloc(&m->d_norm, 32 * 4)) ||
      (e = cudaMalloc(&m->d_error, 16)) || (e = cudaMalloc(&m->d_loss, 16))) {
    cudaGetLastError();
    for (void* b : {(void*)m->d_params, (void*)m->d_grad, (void*)m->d_m, (void*)m->d_v, (void*)m->d_w1r,
                    (void*)m->d_w4r, (void*)m->d_tc, (void*)m->d_norm, (void*)m->d_error, (void*)m->d_loss})
      if (b) cudaFree(b);
    delete m;
    return e == cudaErrorMemoryAllocation ? PP_ERR_OOM : PP_ERR_CUDA;
  }
  // Glorot-uniform weights, zero biases, from a splitmix64 stream of `seed`
  std::vector<float> p(mlp::N_PARAMS, 0.f);
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = (float)((2.0 * next() - 1.0) * a);
  };
  fill(mlp::OFF_W1, mlp::H, mlp::IN);
  fill(mlp::OFF_W2, mlp::H, mlp::H);
  fill(mlp::OFF_W3, mlp::H, mlp::H);
  fill(mlp::OFF_W4, mlp::OUT, mlp::H);
  float norm[32] = {0};
  for (int j = 0; j < 4; ++j) norm[4 + j] = 1.f;
  for (int j = 0; j < 5; ++j) norm[13 + j] = 1.f;
  if ((e = cudaMemcpy(m->d_params, p.data(), mlp::N_PARAMS * 4, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(m->d_grad, 0, mlp::N_PARAMS * 4)) || (e = cudaMemset(m->d_m, 0, mlp::N_PARAMS * 4)) ||
      (e = cudaMemset(m->d_v, 0, mlp::N_PARAMS * 4)) || (e = cudaMemcpy(m->d_norm, norm, 128, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(m->d_error, 0, 16)) || (e = prepare(m, nullptr)) || (e = cudaDeviceSynchronize())) {
    cudaGetLastError();
    pp_mlp_destroy(m);
    return PP_ERR_CUDA;
  }
  cudaFuncSetAttribute(mlp::infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kInferSmem);
  cudaFuncSetAttribute(mlp::train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kTrainSmem);
  cudaFuncSetAttribute(mlp::gemm_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kTestSmem);
  *out = m;
  return PP_OK;
}

void pp_mlp_destroy(pp_mlp* m) {
  if (!m) return;
  Guard g(m->device);
  cudaDeviceSynchronize();
  for (void* p : {(void*)m->d_params, (void*)m->d_grad, (void*)m->d_m, (void*)m->d_v, (void*)m->d_w1r,
                  (void*)m->d_w4r, (void*)m->d_tc, (void*)m->d_norm, (void*)m->d_error, (void*)m->d_loss,
                  (void*)m->d_zs, (void*)m->d_hs})
    if (p) cudaFree(p);
  delete m;
}

const char* pp_mlp_last_error(const pp_mlp* m) { return m ? m->err.c_str() : ""; }

int32_t pp_mlp_num_params(void) { return mlp::N_PARAMS; }

pp_status pp_mlp_get_params(pp_mlp* m, float* out) {
  if (!m || !out) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  return cudaMemcpy(out, m->d_params, mlp::N_PARAMS * 4, cudaMemcpyDeviceToHost) ? PP_ERR_CUDA : PP_OK;
}

pp_status pp_mlp_set_params(pp_mlp* m, const float* in) {
  if (!m || !in) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  if (cudaMemcpy(m->d_params, in, mlp::N_PARAMS * 4, cudaMemcpyHostToDevice) || prepare(m, nullptr) ||
      cudaDeviceSynchronize())
    return fail(m, PP_ERR_CUDA, "pp_mlp_set_params");
  return PP_OK;
}

pp_status pp_mlp_set_normalization(pp_mlp* m, const float* x_mean, const float* x_std, const float* y_mean,
                                   const float* y_std) {
  if (!m || !x_mean || !x_std || !y_mean || !y_std) return PP_ERR_ARG;
  float norm[32] = {0};
  for (int j = 0; j < 4; ++j) {
    norm[j] = x_mean[j];
    norm[4 + j] = x_std[j] > 0.f ? x_std[j] : 1.f;
  }
  for (int j = 0; j < 5; ++j) {
    norm[8 + j] = y_mean[j];
    norm[13 + j] = y_std[j] > 0.f ? y_std[j] : 1.f;
  }
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  return cudaMemcpy(m->d_norm, norm, 128, cudaMemcpyHostToDevice) ? PP_ERR_CUDA : PP_OK;
}

pp_status pp_mlp_get_normalization(pp_mlp* m, float* out18) {
  if (!m || !out18) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  return cudaMemcpy(out18, m->d_norm, 18 * 4, cudaMemcpyDeviceToHost) ? PP_ERR_CUDA : PP_OK;
}

pp_status pp_mlp_forward(pp_mlp* m, const float* d_x, float* d_out, int64_t n, int32_t physical, void* stream) {
  pp::Range range_("pp_mlp_forward");
  if (!m || n < 0 || (n > 0 && (!d_x || !d_out))) return PP_ERR_ARG;
  if (n == 0) return PP_OK;
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  const int64_t tiles = (n + mlp::TILE - 1) / mlp::TILE;
  const int grid = (int)std::min<int64_t>((tiles + mlp::kGroups - 1) / mlp::kGroups, (int64_t)m->sm_count);
  mlp::infer_kernel<<<grid, mlp::INFER_THREADS, mlp::kInferSmem, static_cast<cudaStream_t>(stream)>>>(
      dev_params(m), d_x, d_out, n, physical);
  pp::count_launches(1);
  const cudaError_t e = cudaGetLastError();
  return e ? fail(m, PP_ERR_CUDA, std::string("pp_mlp_forward: ") + cudaGetErrorString(e)) : PP_OK;
}

// One Adam step on a batch (or, with lr = 0 and grad_out, the raw gradients).
pp_status pp_mlp_train_step(pp_mlp* m, const float* d_xn, const float* d_yt, const float* d_mask, int64_t n,
                            float lr, float* loss_out, float* grad_out) {
  pp::Range range_("pp_mlp_train_step");
  if (!m || n <= 0 || !d_xn || !d_yt || !d_mask) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  Guard g(m->device);
  cudaError_t e;
  if (n > m->scratch_rows) {
    if (m->d_zs) cudaFree(m->d_zs);
    if (m->d_hs) cudaFree(m->d_hs);
    m->d_zs = nullptr;
    m->d_hs = nullptr;
    m->scratch_rows = 0;
    if ((e = cudaMalloc(&m->d_zs, (size_t)3 * n * mlp::H * 4)) ||
        (e = cudaMalloc(&m->d_hs, (size_t)3 * n * mlp::H * 2))) {
      cudaGetLastError();
      return fail(m, PP_ERR_OOM, "pp_mlp_train_step: scratch");
    }
    m->scratch_rows = n;
  }
  // mask count for the mean
  std::vector<float> hmask((size_t)n * mlp::OUT);
  if ((e = cudaMemcpy(hmask.data(), d_mask, hmask.size() * 4, cudaMemcpyDeviceToHost)))
    return fail(m, PP_ERR_CUDA, "pp_mlp_train_step: mask");
  double cnt = 0;
  for (float v : hmask) cnt += v;
  const float inv = cnt > 0 ? (float)(1.0 / cnt) : 0.f;
  if ((e = cudaMemset(m->d_loss, 0, 4)) || (e = cudaMemset(m->d_grad, 0, mlp::N_PARAMS * 4)))
    return fail(m, PP_ERR_CUDA, "pp_mlp_train_step: memset");
  const int grid = (int)((n + mlp::TILE - 1) / mlp::TILE);
  mlp::train_kernel<<<grid, mlp::THREADS, mlp::kTrainSmem>>>(dev_params(m), d_xn, d_yt, d_mask, n, inv, m->d_grad,
                                                              m->d_loss, m->d_zs, m->d_hs);
  pp::count_launches(1);
  if ((e = cudaGetLastError())) return fail(m, PP_ERR_CUDA, std::string("train: ") + cudaGetErrorString(e));
  if (grad_out && (e = cudaMemcpy(grad_out, m->d_grad, mlp::N_PARAMS * 4, cudaMemcpyDeviceToHost)))
    return fail(m, PP_ERR_CUDA, "pp_mlp_train_step: grads");
  if (lr > 0.f) {
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)m->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)m->step)));
    mlp::adam_kernel<<<64, 256>>>(m->d_params, m->d_grad, m->d_m, m->d_v, lr, b1, b2, 1e-8f, c1, c2);
    pp::count_launches(1);
    if ((e = prepare(m, nullptr))) return fail(m, PP_ERR_CUDA, "prepare");
  }
  float loss = 0.f;
  int errflag = 0;
  if ((e = cudaMemcpy(&loss, m->d_loss, 4, cudaMemcpyDeviceToHost)) ||
      (e = cudaMemcpy(&errflag, m->d_error, 4, cudaMemcpyDeviceToHost)))
    return fail(m, PP_ERR_CUDA, std::string("train: ") + cudaGetErrorString(e));
  if (errflag) return fail(m, PP_ERR_TIMEOUT, "tensor-core wait expired");
  if (loss_out) *loss_out = (float)(loss * inv);
  return PP_OK;
}

pp_status pp_mlp_gemm_selftest(int device, const uint16_t* a_bf16, const uint16_t* b_bf16, float* c) {
  if (!a_bf16 || !b_bf16 || !c) return PP_ERR_ARG;
  Guard g(device);
  void *da = nullptr, *db = nullptr, *dc = nullptr, *de = nullptr;
  cudaError_t e;
  if ((e = cudaMalloc(&da, 128 * 128 * 2)) || (e = cudaMalloc(&db, 128 * 128 * 2)) ||
      (e = cudaMalloc(&dc, 128 * 128 * 4)) || (e = cudaMalloc(&de, 16))) {
    cudaGetLastError();
    for (void* b : {da, db, dc, de})
      if (b) cudaFree(b);
    return e == cudaErrorMemoryAllocation ? PP_ERR_OOM : PP_ERR_CUDA;
  }
  cudaFuncSetAttribute(mlp::gemm_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::kTestSmem);
  int flag = 0;
  cudaMemcpy(da, a_bf16, 128 * 128 * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(db, b_bf16, 128 * 128 * 2, cudaMemcpyHostToDevice);
  cudaMemset(de, 0, 16);
  mlp::gemm_test_kernel<<<1, mlp::THREADS, mlp::kTestSmem>>>(static_cast<const __nv_bfloat16*>(da),
                                                             static_cast<const __nv_bfloat16*>(db),
                                                             static_cast<float*>(dc), static_cast<int*>(de));
  pp::count_launches(1);
  e = cudaGetLastError();
  if (!e) e = cudaMemcpy(c, dc, 128 * 128 * 4, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(&flag, de, 4, cudaMemcpyDeviceToHost);
  cudaFree(da);
  cudaFree(db);
  cudaFree(dc);
  cudaFree(de);
  if (e) return PP_ERR_CUDA;
  return flag ? PP_ERR_TIMEOUT : PP_OK;
}

}  // extern "C"

extern "C" pp_status pp_gamma_mixture_fit(const double* d_hist, int64_t n, int32_t bins, float t0, float bin_width,
                                          const float* d_tshift, float* d_out, int32_t iters, void* stream) {
  if (n < 0 || bins <= 0 || !(bin_width > 0.f) || iters < 1 || (n > 0 && (!d_hist || !d_tshift || !d_out)))
    return PP_ERR_ARG;
  if (n == 0) return PP_OK;
  const int64_t threads = n * 32;
  const int grid = (int)((threads + 255) / 256);
  mlp::gamma_fit_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_hist, n, bins, t0, bin_width,
                                                                              d_tshift, d_out, iters);
  pp::count_launches(1);
  return cudaGetLastError() ? PP_ERR_CUDA : PP_OK;
}
