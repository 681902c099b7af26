// SPDX-License-Identifier: Apache-2.0
// Per-particle warm-start MLP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Network: 16 features -> 64 -> 64 -> 2 with SiLU, BF16 weights and activations as MMA operands, FP32 accumulation
// in tensor memory (TMEM), FP32 biases and output layer. The two outputs are the warm starts of the two pressure
// solves of a step, in the dt-free form the solver stores them (kappa dt for the divergence solve, kappa dt^2 for the
// density solve), normalised by the training targets' mean and deviation.
//
// One CTA of 128 threads works on tiles of 128 rows (particles or training samples): thread t owns row t. Operand
// tiles live in shared memory in the canonical K-major layout without swizzle (8 x 8 core matrices of 128 bytes);
// one elected thread issues tcgen05.mma (M = 128) and commits to an mbarrier that every thread waits on with an
// iteration limit; the accumulators are read back with tcgen05.ld (32 lanes x 32 bit: thread t reads TMEM lane t,
// which holds row t of the M = 128 accumulator). Every wait is bounded: on expiry the kernel records an error, stops
// issuing work, waits (bounded again) for the MMAs it committed, frees its TMEM and returns.
//
// Training uses the same tiles: forward, loss gradient, dH1 = dZ2 W2 on the tensor cores, and all weight gradients of
// the two hidden layers (and their biases) in ONE accumulating MMA per tile:
//   [dZ2^T ; dZ1^T] (128 x rows) . [H1 | X | 1 | 0]  (rows x 96)  ->  TMEM 128 x 96, accumulated over the CTA's tiles,
// whose blocks are dW2 (rows 0-63, cols 0-63), db2 (col 80), dW1 (rows 64-127, cols 64-79) and db1 (col 80).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace adf {
namespace mlp {

constexpr int NF = 16, NH = 64, NO = 2;
constexpr int TILE = 128;  // rows per MMA (UMMA M)
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NH * NF;
constexpr int OFF_W2 = OFF_B1 + NH;
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;
constexpr int OFF_B3 = OFF_W3 + NO * NH;
constexpr int N_PARAMS = OFF_B3 + NO;  // 5378 FP32 master parameters, this packed order
constexpr int N_WG = 96;               // weight-gradient MMA width: H1 (64) | X (16) | ones (1) | zero (15)
constexpr unsigned WAIT_LIMIT = 1u << 22;  // mbarrier polls before a wait gives up (normal waits need a few)

// Device-side copy of a model: BF16 weight matrices ([out][in] row-major) and the FP32 rest, with the feature and
// target normalisation (x_n = (x - mu) * inv_sigma; y = mu + sigma * y_n).
struct Net {
  const __nv_bfloat16* w1;  // [64][16]
  const __nv_bfloat16* w2;  // [64][64]
  const float* p;           // packed FP32 parameters (N_PARAMS): b1, b2, w3, b3 are read from here
  const float* norm;        // fmu[16], finv[16], tmu[2], tsig[2] (may be null: identity)
  int* error;               // set to 1 when a bounded wait expires
  unsigned wait_limit;      // polls a tensor-core step's wait may take before giving up (WAIT_LIMIT; adf_mlp_set_wait_limit)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) of an R x K BF16 operand tile, canonical K-major layout without swizzle: core
// matrices of 8 rows x 16 bytes, K-adjacent core matrices 128 bytes apart (leading byte offset), row-group-adjacent
// ones K / 8 * 128 bytes apart (stride byte offset).
__host__ __device__ constexpr uint32_t kmaj(int r, int k, int K) {
  return (uint32_t)(((((r >> 3) * (K >> 3)) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor of a K-major tile with K columns (start must be 16-byte aligned).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int K) {
  const uint64_t lbo = 128, sbo = (uint64_t)(K >> 3) * 128;
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (lbo >> 4) << 16;
  d |= (sbo >> 4) << 32;
  d |= 1ull << 46;  // descriptor version of sm_100; base offset 0, relative leading offset, no swizzle
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D FP32, A and B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {  // one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Wait for the phase of `parity` to complete, at most `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane; the load and its completion wait are one asm statement, so
// no register is read before the data has arrived.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 64 consecutive FP32 columns of this thread's TMEM lane: two 32-column loads in flight, one completion wait.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%64];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%65];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr), "r"(taddr + 32u)
      : "memory");
#pragma unroll
  for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of column `col` in the lanes of this thread's warp (warp w may access lanes 32 (w % 4) ...).
__device__ __forceinline__ uint32_t tmem_row(uint32_t base, int col) {
  return base + ((uint32_t)((threadIdx.x >> 5) & 3) * 32u << 16) + (uint32_t)col;
}

// Logistic sigmoid through the identity s(z) = (1 + tanh(z / 2)) / 2 with the hardware tanh approximation (one MUFU
// instruction, relative error about 2^-11, below the BF16 rounding the activations get next): the library is built
// with IEEE division, which would make a 1 / (1 + e^-z) form several times slower.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Eight consecutive K elements of one row (one 16-byte row of a core matrix) in one store.
__device__ __forceinline__ void st_row8(unsigned char* base, uint32_t off, const float* v) {
  uint4 u;
  __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
  __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
  u.x = *reinterpret_cast<uint32_t*>(&h0);
  u.y = *reinterpret_cast<uint32_t*>(&h1);
  u.z = *reinterpret_cast<uint32_t*>(&h2);
  u.w = *reinterpret_cast<uint32_t*>(&h3);
  *reinterpret_cast<uint4*>(base + off) = u;
}

// Copy a [R][K] BF16 row-major matrix from global memory into a K-major operand tile (all threads of the block).
__device__ __forceinline__ void load_operand(unsigned char* dst, const __nv_bfloat16* src, int R, int K) {
  for (int e = threadIdx.x; e < R * K; e += blockDim.x) {
    const int r = e / K, k = e % K;
    *reinterpret_cast<__nv_bfloat16*>(dst + kmaj(r, k, K)) = src[e];
  }
}
// The same matrix transposed: element (r, k) of the tile is src[k][r] (src is [K][R]).
__device__ __forceinline__ void load_operand_t(unsigned char* dst, const __nv_bfloat16* src, int R, int K) {
  for (int e = threadIdx.x; e < R * K; e += blockDim.x) {
    const int k = e / R, r = e % R;
    *reinterpret_cast<__nv_bfloat16*>(dst + kmaj(r, k, K)) = src[e];
  }
}

// Block-wide "did any thread fail", after which every thread takes the same branch.
__device__ __forceinline__ bool any_failed(bool failed) { return __syncthreads_or(failed ? 1 : 0) != 0; }

// ------------------------------------------------------------------------------------------------ forward
// Shared memory of the forward kernels (byte offsets; every operand tile 128-byte aligned).
constexpr int FW_W1 = 0;                           // 64 x 16
constexpr int FW_W2 = FW_W1 + NH * NF * 2;         // 64 x 64
constexpr int FW_X = FW_W2 + NH * NH * 2;          // 128 x 16
constexpr int FW_H = FW_X + TILE * NF * 2;         // 128 x 64
constexpr int FW_F = FW_H + TILE * NH * 2;         // FP32: b1 64, b2 64, w3 128, b3 2 (+2 pad), norm 36
constexpr int FW_BAR = FW_F + (64 + 64 + 128 + 4 + 36) * 4;
constexpr int FW_BYTES = FW_BAR + 16;
// Launched with at least this much dynamic shared memory, at most 4 CTAs fit on an SM: their 4 x 128 TMEM columns
// never exceed the SM's 512, so no allocation waits on another CTA.
constexpr int FW_SMEM = 48 * 1024;
constexpr int FW_TMEM_COLS = 128;  // [0, 64) layer 1, [64, 128) layer 2

// Runs the network on the caller's rows, TILE at a time (persistent CTAs). `Src` provides
//   int rows() const;                          number of rows
//   void features(int row, float (&x)[16]);    features of a valid row (normalised here by net.norm)
//   void output(int row, float y0, float y1);  outputs of a valid row (de-normalised by net.norm)
template <class Src>
__device__ void forward_rows(const Net& net, Src& src) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sW1 = smem + FW_W1;
  unsigned char* sW2 = smem + FW_W2;
  unsigned char* sX = smem + FW_X;
  unsigned char* sH = smem + FW_H;
  float* sF = reinterpret_cast<float*>(smem + FW_F);
  float* b1 = sF;
  float* b2 = sF + 64;
  float* w3 = sF + 128;
  float* b3 = sF + 256;
  float* nrm = sF + 260;  // fmu 16, finv 16, tmu 2, tsig 2
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + FW_BAR);
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x;

  load_operand(sW1, net.w1, NH, NF);
  load_operand(sW2, net.w2, NH, NH);
  for (int e = t; e < 64; e += blockDim.x) {
    b1[e] = net.p[OFF_B1 + e];
    b2[e] = net.p[OFF_B2 + e];
  }
  for (int e = t; e < 128; e += blockDim.x) w3[e] = net.p[OFF_W3 + e];
  if (t < 2) b3[t] = net.p[OFF_B3 + t];
  if (t < 36) nrm[t] = net.norm ? net.norm[t] : (t >= 16 && t < 32) || t >= 34 ? 1.0f : 0.0f;
  if (t == 0) mbar_init(bar, 1);
  if (t < 32) {
    tmem_alloc(&tmem_base, FW_TMEM_COLS);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tm = tmem_base;
  const uint64_t dW1 = sdesc(smem_u32(sW1), NF), dW2 = sdesc(smem_u32(sW2), NH);
  const uint64_t dX = sdesc(smem_u32(sX), NF), dH = sdesc(smem_u32(sH), NH);
  const uint32_t id64 = idesc_bf16(TILE, NH);
  uint32_t phase = 0;
  int committed = 0;  // commits not yet waited for (for the error path)
  bool failed = false;
  const int rows = src.rows();
  const int tiles = (rows + TILE - 1) / TILE;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    if (src.skip_tile(tile * TILE, min(rows, tile * TILE + TILE))) continue;  // the same answer in every thread
    const int row = tile * TILE + t;
    const bool valid = row < rows;
    float x[NF];
    if (valid) src.features(row, x);
#pragma unroll
    for (int k = 0; k < NF; ++k) x[k] = valid ? (x[k] - nrm[k]) * nrm[16 + k] : 0.0f;
    st_row8(sX, kmaj(t, 0, NF), x);
    st_row8(sX, kmaj(t, 8, NF), x + 8);
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    if (t == 0) {
      mma_bf16(tm, dX, dW1, id64, 0);
      mma_commit(bar);
    }
    ++committed;
    failed = !mbar_wait(bar, phase, net.wait_limit);
    if (any_failed(failed)) break;
    phase ^= 1;
    --committed;
    tc_after();
    {
      float v[64];
      tmem_ld64(tmem_row(tm, 0), v);
#pragma unroll
      for (int i = 0; i < 64; ++i) {
        const float z = v[i] + b1[i];
        v[i] = z * sigmoid(z);
      }
#pragma unroll
      for (int c = 0; c < NH; c += 8) st_row8(sH, kmaj(t, c, NH), v + c);
    }
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    if (t == 0) {
#pragma unroll
      for (int s = 0; s < NH / 16; ++s) mma_bf16(tm + 64, dH + (uint64_t)(s * 16), dW2 + (uint64_t)(s * 16), id64, s > 0);
      mma_commit(bar);
    }
    ++committed;
    failed = !mbar_wait(bar, phase, net.wait_limit);
    if (any_failed(failed)) break;
    phase ^= 1;
    --committed;
    tc_after();
    float y0 = b3[0], y1 = b3[1];
    {
      float v[64];
      tmem_ld64(tmem_row(tm, 64), v);
#pragma unroll
      for (int i = 0; i < 64; ++i) {
        const float z = v[i] + b2[i];
        const float h = z * sigmoid(z);
        y0 = fmaf(w3[i], h, y0);
        y1 = fmaf(w3[64 + i], h, y1);
      }
    }
    if (valid) src.output(row, fmaf(y0, nrm[34], nrm[32]), fmaf(y1, nrm[35], nrm[33]));
  }
  if (failed) {
    if (t == 0) atomicExch(net.error, 1);
    // let the MMAs this CTA committed finish before their TMEM is released
    for (int k = 0; k < committed; ++k) {
      mbar_wait(bar, phase, WAIT_LIMIT);
      phase ^= 1;
    }
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (t < 32) tmem_dealloc(tm, FW_TMEM_COLS);
}

// The standalone kernels below are compiled only in the translation unit of the adf_mlp_* entry points.
#ifdef ADF_MLP_STANDALONE

// Standalone inference: x [n][16] features (FP32), y [n][2] outputs; normalised units when net.norm is null.
struct RowsSrc {
  const float* x;
  float* y;
  int n;
  __device__ bool skip_tile(int, int) const { return false; }
  __device__ int rows() const { return n; }
  __device__ void features(int row, float (&f)[16]) const {
    const float4* p = reinterpret_cast<const float4*>(x + (size_t)row * NF);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 v = p[q];
      f[4 * q] = v.x;
      f[4 * q + 1] = v.y;
      f[4 * q + 2] = v.z;
      f[4 * q + 3] = v.w;
    }
  }
  __device__ void output(int row, float y0, float y1) const {
    y[2 * (size_t)row] = y0;
    y[2 * (size_t)row + 1] = y1;
  }
};

__global__ void __launch_bounds__(TILE) k_mlp_forward(Net net, const float* x, float* y, int n) {
  RowsSrc s{x, y, n};
  forward_rows(net, s);
}

// ----------------------------------------------------------------------------------------------- training
constexpr int TR_W1 = 0;                              // B of layer 1: 64 x 16
constexpr int TR_W2 = TR_W1 + NH * NF * 2;            // B of layer 2: 64 x 64
constexpr int TR_W2T = TR_W2 + NH * NH * 2;           // B of dH1 = dZ2 W2: W2^T, 64 x 64
constexpr int TR_X = TR_W2T + NH * NH * 2;            // A of layer 1: 128 x 16
constexpr int TR_H = TR_X + TILE * NF * 2;            // A of layer 2: 128 x 64
constexpr int TR_DZ2 = TR_H + TILE * NH * 2;          // A of dH1: 128 x 64
constexpr int TR_AWG = TR_DZ2 + TILE * NH * 2;        // A of the weight gradients: 128 x 128 ([dZ2^T ; dZ1^T])
constexpr int TR_BWG = TR_AWG + TILE * TILE * 2;      // B of the weight gradients: 96 x 128 ([H1 | X | 1 | 0]^T)
constexpr int TR_F = TR_BWG + N_WG * TILE * 2;        // FP32: b1 64, b2 64, w3 128, b3 2, acc w3 128, acc b3 2, loss
constexpr int TR_BAR = TR_F + (64 + 64 + 128 + 4 + 128 + 4) * 4;
constexpr int TR_SMEM = TR_BAR + 16;  // ~112 KB: at most 2 CTAs per SM, 2 x 256 TMEM columns
constexpr int TR_TMEM_COLS = 256;     // [0, 64) Z1, [64, 128) Z2 then dH1, [128, 224) weight gradients
constexpr int TR_C_WG = 128;

// Per-CTA gradient of the mean squared error over the batch (rows idx[0 .. batch)), written to part[cta][N_PARAMS + 1]
// (the last element: the CTA's summed squared error). x: [N][16] normalised features, y: [N][2] normalised targets.
__global__ void __launch_bounds__(TILE) k_mlp_grad(Net net, const float* __restrict__ x, const float* __restrict__ y,
                                                   const int* __restrict__ idx, int batch, float* part) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sW1 = smem + TR_W1;
  unsigned char* sW2 = smem + TR_W2;
  unsigned char* sW2T = smem + TR_W2T;
  unsigned char* sX = smem + TR_X;
  unsigned char* sH = smem + TR_H;
  unsigned char* sDZ2 = smem + TR_DZ2;
  unsigned char* sAwg = smem + TR_AWG;
  unsigned char* sBwg = smem + TR_BWG;
  float* sF = reinterpret_cast<float*>(smem + TR_F);
  float* b1 = sF;
  float* b2 = sF + 64;
  float* w3 = sF + 128;
  float* b3 = sF + 256;
  float* gw3 = sF + 260;
  float* gb3 = sF + 388;   // [2], then the summed squared error at [2]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + TR_BAR);
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x;
  const int lane = t & 31;

  load_operand(sW1, net.w1, NH, NF);
  load_operand(sW2, net.w2, NH, NH);
  load_operand_t(sW2T, net.w2, NH, NH);
  for (int e = t; e < 64; e += blockDim.x) {
    b1[e] = net.p[OFF_B1 + e];
    b2[e] = net.p[OFF_B2 + e];
  }
  for (int e = t; e < 128; e += blockDim.x) {
    w3[e] = net.p[OFF_W3 + e];
    gw3[e] = 0.0f;
  }
  if (t < 2) b3[t] = net.p[OFF_B3 + t];
  if (t < 4) gb3[t] = 0.0f;
  // constant columns of B_wg: row 80 = ones, rows 81..95 = zero (rows of B are its N index)
  for (int e = t; e < 16 * TILE; e += blockDim.x) {
    const int n = 80 + e / TILE, k = e % TILE;
    st_bf16(sBwg, kmaj(n, k, TILE), n == 80 ? 1.0f : 0.0f);
  }
  if (t == 0) mbar_init(bar, 1);
  if (t < 32) {
    tmem_alloc(&tmem_base, TR_TMEM_COLS);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tm = tmem_base;
  const uint64_t dW1 = sdesc(smem_u32(sW1), NF), dW2 = sdesc(smem_u32(sW2), NH), dW2T = sdesc(smem_u32(sW2T), NH);
  const uint64_t dX = sdesc(smem_u32(sX), NF), dH = sdesc(smem_u32(sH), NH), dDZ2 = sdesc(smem_u32(sDZ2), NH);
  const uint64_t dAwg = sdesc(smem_u32(sAwg), TILE), dBwg = sdesc(smem_u32(sBwg), TILE);
  const uint32_t id64 = idesc_bf16(TILE, NH), idwg = idesc_bf16(TILE, N_WG);
  uint32_t phase = 0;
  int committed = 0;
  bool failed = false;
  int done = 0;  // tiles whose weight gradients are in TMEM
  const float inv_b = 1.0f / (float)max(batch, 1);
  const int tiles = (batch + TILE - 1) / TILE;
  float sq = 0.0f;
  auto wait = [&]() -> bool {
    ++committed;
    failed = !mbar_wait(bar, phase, net.wait_limit);
    if (any_failed(failed)) return false;
    phase ^= 1;
    --committed;
    tc_after();
    return true;
  };
  auto sync_for_mma = [&]() {
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
  };
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int r = tile * TILE + t;
    const bool valid = r < batch;
    const int s = valid ? idx[r] : 0;
    float xr[NF], tg0 = 0.0f, tg1 = 0.0f;
#pragma unroll
    for (int k = 0; k < NF; ++k) xr[k] = valid ? x[(size_t)s * NF + k] : 0.0f;
    if (valid) {
      tg0 = y[2 * (size_t)s];
      tg1 = y[2 * (size_t)s + 1];
    }
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      st_bf16(sX, kmaj(t, k, NF), xr[k]);
      st_bf16(sBwg, kmaj(64 + k, t, TILE), xr[k]);
    }
    sync_for_mma();
    if (t == 0) {
      mma_bf16(tm, dX, dW1, id64, 0);
      mma_commit(bar);
    }
    if (!wait()) break;
    // layer 1 epilogue: H1 as the A operand of layer 2 and as rows 0..63 of B_wg
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tmem_ld16(tmem_row(tm, c), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + b1[c + i];
        const float h = z * sigmoid(z);
        st_bf16(sH, kmaj(t, c + i, NH), h);
        st_bf16(sBwg, kmaj(c + i, t, TILE), h);
      }
    }
    sync_for_mma();
    if (t == 0) {
#pragma unroll
      for (int k = 0; k < NH / 16; ++k)
        mma_bf16(tm + 64, dH + (uint64_t)(k * 16), dW2 + (uint64_t)(k * 16), id64, k > 0);
      mma_commit(bar);
    }
    if (!wait()) break;
    // output and loss gradient (dL/dy = (y - t) / batch for L = sum (y - t)^2 / (2 batch))
    float y0 = b3[0], y1 = b3[1];
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tmem_ld16(tmem_row(tm, 64 + c), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + b2[c + i];
        const float h = z * sigmoid(z);
        y0 = fmaf(w3[c + i], h, y0);
        y1 = fmaf(w3[64 + c + i], h, y1);
      }
    }
    const float e0 = valid ? y0 - tg0 : 0.0f, e1 = valid ? y1 - tg1 : 0.0f;
    sq = fmaf(e0, e0, fmaf(e1, e1, sq));
    const float dy0 = e0 * inv_b, dy1 = e1 * inv_b;
    // dZ2 = (W3^T dy) * silu'(z2); dW3 += dy h2^T (warp sums, then shared atomics)
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tmem_ld16(tmem_row(tm, 64 + c), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = c + i;
        const float z = v[i] + b2[j];
        const float sg = sigmoid(z);
        const float h = z * sg;
        const float dz = fmaf(w3[j], dy0, w3[64 + j] * dy1) * (sg * fmaf(z, 1.0f - sg, 1.0f));
        st_bf16(sDZ2, kmaj(t, j, NH), dz);
        st_bf16(sAwg, kmaj(j, t, TILE), dz);
        float g0 = dy0 * h, g1 = dy1 * h;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
          g0 += __shfl_xor_sync(0xffffffffu, g0, o);
          g1 += __shfl_xor_sync(0xffffffffu, g1, o);
        }
        if (lane == 0) {
          atomicAdd(&gw3[j], g0);
          atomicAdd(&gw3[64 + j], g1);
        }
      }
    }
    {
      float g0 = dy0, g1 = dy1;
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) {
        g0 += __shfl_xor_sync(0xffffffffu, g0, o);
        g1 += __shfl_xor_sync(0xffffffffu, g1, o);
      }
      if (lane == 0) {
        atomicAdd(&gb3[0], g0);
        atomicAdd(&gb3[1], g1);
      }
    }
    sync_for_mma();
    if (t == 0) {  // dH1 = dZ2 W2 into the Z2 columns (Z2 is no longer needed)
#pragma unroll
      for (int k = 0; k < NH / 16; ++k)
        mma_bf16(tm + 64, dDZ2 + (uint64_t)(k * 16), dW2T + (uint64_t)(k * 16), id64, k > 0);
      mma_commit(bar);
    }
    if (!wait()) break;
    // dZ1 = dH1 * silu'(z1) as rows 64..127 of A_wg
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float dh[16], v[16];
      tmem_ld16(tmem_row(tm, 64 + c), dh);
      tmem_ld16(tmem_row(tm, c), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + b1[c + i];
        const float sg = sigmoid(z);
        st_bf16(sAwg, kmaj(64 + c + i, t, TILE), dh[i] * (sg * fmaf(z, 1.0f - sg, 1.0f)));
      }
    }
    sync_for_mma();
    if (t == 0) {  // weight gradients, accumulated in TMEM over this CTA's tiles
#pragma unroll
      for (int k = 0; k < TILE / 16; ++k)
        mma_bf16(tm + TR_C_WG, dAwg + (uint64_t)(k * 16), dBwg + (uint64_t)(k * 16), idwg, (done > 0 || k > 0) ? 1u : 0u);
      mma_commit(bar);
    }
    if (!wait()) break;
    ++done;
  }
  // the CTA's summed squared error
  {
    float g = sq;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
    if (lane == 0) atomicAdd(&gb3[2], g);
  }
  if (failed) {
    if (t == 0) atomicExch(net.error, 1);
    for (int k = 0; k < committed; ++k) {
      mbar_wait(bar, phase, WAIT_LIMIT);
      phase ^= 1;
    }
  }
  tc_before();
  __syncthreads();
  tc_after();
  float* out = part + (size_t)blockIdx.x * (N_PARAMS + 1);
  const bool have = done > 0 && !failed;
  if (t < 64) {  // rows 0..63: dW2 (cols 0..63) and db2 (col 80)
    for (int c = 0; c < 96; c += 16) {
      float v[16];
      tmem_ld16(tmem_row(tm, TR_C_WG + c), v);
      if (c < 64) {
#pragma unroll
        for (int i = 0; i < 16; ++i) out[OFF_W2 + t * NH + c + i] = have ? v[i] : 0.0f;
      } else if (c == 80) {
        out[OFF_B2 + t] = have ? v[0] : 0.0f;
      }
    }
  } else {  // rows 64..127: dW1 (cols 64..79) and db1 (col 80)
    const int m = t - 64;
    float v[16];
    tmem_ld16(tmem_row(tm, TR_C_WG + 64), v);
#pragma unroll
    for (int i = 0; i < 16; ++i) out[OFF_W1 + m * NF + i] = have ? v[i] : 0.0f;
    tmem_ld16(tmem_row(tm, TR_C_WG + 80), v);
    out[OFF_B1 + m] = have ? v[0] : 0.0f;
  }
  for (int e = t; e < 128; e += blockDim.x) out[OFF_W3 + e] = gw3[e];
  if (t < 2) out[OFF_B3 + t] = gb3[t];
  if (t == 0) out[N_PARAMS] = gb3[2];
  tc_before();
  __syncthreads();
  tc_after();
  if (t < 32) tmem_dealloc(tm, TR_TMEM_COLS);
}

// Sum of the CTA partials in CTA order (deterministic), then one Adam step on the FP32 master parameters and their
// BF16 copies. grad_out (optional) receives the summed gradient; loss_out[0] the batch's mean squared error.
__global__ void k_mlp_adam(const float* part, int n_part, int batch, float* w, float* m, float* v,
                           __nv_bfloat16* w1b, __nv_bfloat16* w2b, float lr, float b1, float b2, float eps, int step,
                           int apply, float* grad_out, float* loss_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > N_PARAMS) return;
  float g = 0.0f;
  for (int c = 0; c < n_part; ++c) g += part[(size_t)c * (N_PARAMS + 1) + i];
  if (i == N_PARAMS) {
    if (loss_out) loss_out[0] = g / (float)(2 * max(batch, 1));
    return;
  }
  if (grad_out) grad_out[i] = g;
  if (!apply) return;
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, (float)step));
  const float vh = vi / (1.0f - powf(b2, (float)step));
  const float wi = w[i] - lr * mh / (sqrtf(vh) + eps);
  w[i] = wi;
  if (i < OFF_B1) w1b[i - OFF_W1] = __float2bfloat16_rn(wi);
  else if (i >= OFF_W2 && i < OFF_B2) w2b[i - OFF_W2] = __float2bfloat16_rn(wi);
}

__global__ void k_mlp_to_bf16(const float* w, __nv_bfloat16* w1b, __nv_bfloat16* w2b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NH * NF) w1b[i] = __float2bfloat16_rn(w[OFF_W1 + i]);
  if (i < NH * NH) w2b[i] = __float2bfloat16_rn(w[OFF_W2 + i]);
}

#endif  // ADF_MLP_STANDALONE

}  // namespace mlp
}  // namespace adf

// The network object behind the adf_mlp_* entry points (shared by the solver, which copies a trained network).
struct adf_mlp {
  int device = 0;
  int sms = 148;
  float* w = nullptr;  // FP32 master parameters [N_PARAMS]
  float* m = nullptr;  // Adam first moments
  float* v = nullptr;  // Adam second moments
  __nv_bfloat16* w1b = nullptr;
  __nv_bfloat16* w2b = nullptr;
  float* part = nullptr;  // [sms][N_PARAMS + 1] per-CTA gradients
  float* grad = nullptr;  // [N_PARAMS]
  float* loss = nullptr;  // [1]
  int* error = nullptr;   // bounded-wait expiry flag
  int step = 0;
  unsigned wait_limit = adf::mlp::WAIT_LIMIT;  // the tensor-core waits' poll limit (the drain after an expiry keeps WAIT_LIMIT)
};
