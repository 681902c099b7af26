// SPDX-License-Identifier: Apache-2.0
// adf_world_sum_noalloc: the per-world float64 sum and maximum of a float array (the reduction that decides pressure
// convergence) for callers that cannot allocate device memory: a host loop that must not enter the CUDA allocator
// (cudaMalloc may synchronise the device and has no latency bound), or a process whose device memory is already
// reserved by another framework's memory pool. It needs no solver object and calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// Its scratch (the per-world chunk table and the per-chunk partial sums and maxima) is the file-scope array below,
// of fixed size; every GPU that loads the library holds it until the process exits. Host code never names the array
// as a device address: the first call on a device, with that device current, looks its address up with
// cudaGetSymbolAddress, caches it per device and passes it to the kernels.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/alloy_dfsph.h"
#include "dfsph_reduce.cuh"

namespace adf {
void set_last_error(const std::string& msg);  // dfsph_capi.cu: the message adf_last_error returns
}

namespace {

constexpr int kWcsInts = ((ADF_NOALLOC_MAX_WORLDS + 1) * 4 + 255) / 256 * 64;  // chunk table, 256-byte rounded
constexpr size_t kWcsBytes = (size_t)kWcsInts * 4;
constexpr size_t kSumBytes = (size_t)ADF_NOALLOC_MAX_CHUNKS * 8;
constexpr size_t kMaxBytes = (size_t)ADF_NOALLOC_MAX_CHUNKS * 4;
constexpr size_t kScratchBytes = kWcsBytes + kSumBytes + kMaxBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup;

int fail(int code, const std::string& msg) {
  adf::set_last_error(msg);
  return code;
}

__device__ __forceinline__ void world_range(const int32_t* ws, int w, int n, int& lo, int& hi) {
  lo = min(max(ws[w], 0), n);
  hi = min(max(ws[w + 1], lo), n);
}

// wcs[w] = first chunk of world w (256-particle chunks aligned to each world start), wcs[W] = chunk count.
__global__ void __launch_bounds__(1024) k_na_chunk_table(const int32_t* ws, int W, int n, int* wcs) {
  __shared__ int warp_tot[32];
  const int per = (W + 1023) / 1024;
  const int w0 = threadIdx.x * per;
  int local = 0;
  for (int k = 0; k < per; ++k) {
    int w = w0 + k;
    if (w < W) {
      int lo, hi;
      world_range(ws, w, n, lo, hi);
      local += (hi - lo + 255) / 256;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  int c = x - local + (wid > 0 ? warp_tot[wid - 1] : 0);
  for (int k = 0; k < per; ++k) {
    int w = w0 + k;
    if (w < W) {
      wcs[w] = c;
      int lo, hi;
      world_range(ws, w, n, lo, hi);
      c += (hi - lo + 255) / 256;
    }
  }
  if (threadIdx.x == 1023) wcs[W] = c;
}

__global__ void __launch_bounds__(256) k_na_chunk_sum(const float* __restrict__ v, const int32_t* ws, int W, int n,
                                                      const int* wcs, int max_chunks, double* part_sum,
                                                      float* part_max) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  const int c = blockIdx.x;
  const int total = min(wcs[W], max_chunks);
  if (c >= total) return;
  int a = 0, b = W;  // the world whose chunk range holds c: wcs[w] <= c < wcs[w + 1]
  while (b - a > 1) {
    int m = (a + b) >> 1;
    if (wcs[m] <= c) a = m; else b = m;
  }
  int lo, hi;
  world_range(ws, a, n, lo, hi);
  int i = lo + 256 * (c - wcs[a]) + threadIdx.x;
  bool in = i < hi;
  float x = in ? v[i] : 0.0f;
  double s = adf::fold256(in ? (double)x : 0.0, smd);
  float m = adf::block_max256(in ? x : -3.4e38f, smf);
  if (threadIdx.x == 0) {
    part_sum[c] = s;
    part_max[c] = m;
  }
}

__global__ void __launch_bounds__(256) k_na_world_fold(const int* wcs, int max_chunks, const double* part_sum,
                                                       const float* part_max, double* out_sum, float* out_max) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  const int w = blockIdx.x;
  const int c0 = min(wcs[w], max_chunks), c1 = min(wcs[w + 1], max_chunks);
  double acc = 0.0;
  float m = -3.4e38f;
  for (int c = c0 + threadIdx.x; c < c1; c += 256) {
    acc = acc + part_sum[c];
    m = fmaxf(m, part_max[c]);
  }
  double s = adf::fold256(acc, smd);
  float mx = adf::block_max256(m, smf);
  if (threadIdx.x == 0) {
    out_sum[w] = s;
    out_max[w] = mx > 0.0f ? mx : 0.0f;
  }
}

}  // namespace

extern "C" int adf_world_sum_noalloc(const float* values, int n, const int32_t* world_start, int world_count,
                                     double* out_sum, float* out_max, void* stream) {
  if (n < 0 || world_count < 0) return fail(ADF_ERR_VALUE, "adf_world_sum_noalloc: negative size");
  if (world_count == 0) return ADF_OK;
  if ((n > 0 && !values) || !world_start || !out_sum || !out_max)
    return fail(ADF_ERR_VALUE, "adf_world_sum_noalloc: null argument");
  if (world_count > ADF_NOALLOC_MAX_WORLDS)
    return fail(ADF_ERR_CAPACITY, "adf_world_sum_noalloc: " + std::to_string(world_count) + " worlds exceed the " +
                                      std::to_string(ADF_NOALLOC_MAX_WORLDS) + "-world limit of its static scratch");
  const long long bound = (long long)n / 256 + world_count + 1;  // chunks of W worlds over n values at most
  if (bound > ADF_NOALLOC_MAX_CHUNKS)
    return fail(ADF_ERR_CAPACITY, "adf_world_sum_noalloc: " + std::to_string(n) + " values in " +
                                      std::to_string(world_count) + " worlds need up to " + std::to_string(bound) +
                                      " chunks, above the static scratch limit of " +
                                      std::to_string(ADF_NOALLOC_MAX_CHUNKS) + " (about 12.5 million values)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ADF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(ADF_ERR_VALUE, "adf_world_sum_noalloc: device index too large");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup);
    if (!g_scratch_addr[dev]) {  // set-up, once per device, with that device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(ADF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  unsigned char* b = static_cast<unsigned char*>(base);
  int* wcs = reinterpret_cast<int*>(b);
  double* part_sum = reinterpret_cast<double*>(b + kWcsBytes);
  float* part_max = reinterpret_cast<float*>(b + kWcsBytes + kSumBytes);
  const int max_chunks = (int)bound;
  cudaStream_t st = (cudaStream_t)stream;
  k_na_chunk_table<<<1, 1024, 0, st>>>(world_start, world_count, n, wcs);
  k_na_chunk_sum<<<max_chunks, 256, 0, st>>>(values, world_start, world_count, n, wcs, max_chunks, part_sum, part_max);
  k_na_world_fold<<<world_count, 256, 0, st>>>(wcs, max_chunks, part_sum, part_max, out_sum, out_max);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_ERR_CUDA, std::string("adf_world_sum_noalloc launch: ") + cudaGetErrorString(e));
  return ADF_OK;
}
