// SPDX-License-Identifier: Apache-2.0
// The projected CG pressure solve of small models as ONE persistent launch (krylov.py:254-297 with the iteration loop
// of solve_driver.py:121-186): the start (the product of the warm start, the active set, the first sums and r.z) and
// every iteration of every world run in one cooperative kernel whose blocks are all resident; each phase is the body
// of the multi-launch path's kernel (k_cg_accel_team, k_cg_apply_team, k_sums2_warps / k_sums2_fused, k_cg_step,
// k_cg_apply_finish_team, k_cg_direction, ...) looped over that kernel's own block indices, and a grid-wide barrier
// stands where a kernel boundary was. The arithmetic, the reduction trees and the order of the phases are those of
// the multi-launch path, so the results are the same bits; what goes is ~9 launches per iteration.
//
// The barrier: an arrival counter zeroed before the launch; barrier k is passed once the counter reaches k times the
// blocks of the grid. Every wait polls at most `wait_limit` times; a block whose wait gives up sets the status word
// and leaves, every block leaves at its next barrier once the status is set, and the host reports the solve as
// failed (ADF_ERR_STATE) instead of results. The kernel never waits without a bound.
#pragma once

#include "dfsph_kernels.cuh"

namespace adf {

struct CgPersist {
  int pt_blocks;       // BLOCK-particle blocks of the per-particle phases (k_cg_init, k_cg_step, k_cg_direction)
  int team_blocks;     // blocks of the team products (TL lanes per particle)
  int sum_blocks;      // blocks of the sums (chunks per block: CHECK_WARPS for the warp fold, 1 for the block fold)
  int w_blocks;        // BLOCK-world blocks (k_cg_first_rz)
  int warp_fold;       // the sums by one warp per chunk (worlds of at most WARP_FOLD_MAX_CHUNKS chunks)
  int cap;             // iterations at most (the WHILE node's cap: max_iterations + 2)
  unsigned expect;     // arrivals that pass one barrier: the grid's blocks (more only when a test makes waits expire)
  long long wait_limit;  // polls of one barrier wait before it gives up
  unsigned* arrive;    // [1] arrivals so far (zeroed before the launch)
  int* status;         // [1] set to 1 when a wait gave up (cleared by the host)
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Barrier number `epoch` (counted by the caller): false when the kernel must stop (a wait gave up, here or in another
// block). Thread 0 arrives after a device-scope fence (the phase's writes before the arrival) and, once the count is
// reached, fences again before the block goes on (the next phase reads what the other blocks wrote).
__device__ __forceinline__ bool grid_barrier(const CgPersist& R, unsigned epoch) {
  __shared__ int stop;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(R.arrive, 1u);
    const unsigned target = epoch * R.expect;
    int bad = 0;
    for (long long it = 0;; ++it) {
      if (ld_acquire_gpu(R.arrive) >= target) break;
      if (*(volatile int*)R.status != 0) {
        bad = 1;
        break;
      }
      if (it >= R.wait_limit) {
        atomicExch(R.status, 1);
        bad = 1;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    stop = bad;
  }
  __syncthreads();
  return stop == 0;
}

// One phase: the body for every block index of its launch, this block taking every gridDim.x-th; the block
// synchronises between indices (the sums' bodies keep shared flags that the next index rewrites).
template <class F>
__device__ __forceinline__ void for_blocks(int nvb, F body) {
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
    body(vb);
    __syncthreads();
  }
}

template <bool MS>
__global__ void __launch_bounds__(BLOCK, 4) k_cg_solve(DevP P, CgPersist R) {
  static_assert(32 * CHECK_WARPS == BLOCK, "the warp-fold sums run as BLOCK-thread blocks");
  unsigned epoch = 0;
  auto sums = [&](int with_max, int beta) {
    if (R.warp_fold)
      for_blocks(R.sum_blocks, [&](int vb) { sums2_warps_at(P, with_max, beta, vb); });
    else
      for_blocks(R.sum_blocks, [&](int vb) { sums2_fused_at(P, with_max, beta, vb); });
  };
#define ADF_BARRIER() \
  if (!grid_barrier(R, ++epoch)) return

  // cg_init: cleared restart flags and pairs, w = A k - b from the warm start, the active set, z, p, r.z
  const int stride = gridDim.x * BLOCK;
  for (int w = blockIdx.x * BLOCK + threadIdx.x; w < P.W; w += stride) {
    P.cg_restart[w] = 0;
    P.cg_act_new[w] = 0;
  }
  for (int i = blockIdx.x * BLOCK + threadIdx.x; i < P.n; i += stride) P.cg_pair[i] = make_float2(0.0f, 0.0f);
  for_blocks(R.team_blocks, [&](int vb) { cg_accel_team_at<MS>(P, P.kappa, P.kr, 0, vb); });
  ADF_BARRIER();
  for_blocks(R.team_blocks, [&](int vb) { cg_apply_team_at<MS>(P, P.kappa, P.cg_w, 0, 1, 0, vb); });
  ADF_BARRIER();
  for_blocks(R.pt_blocks, [&](int vb) { cg_init_at(P, vb); });
  ADF_BARRIER();
  sums(0, 0);
  ADF_BARRIER();
  for_blocks(R.w_blocks, [&](int vb) { cg_first_rz_at(P, vb); });
  ADF_BARRIER();
  // the iterations (cg_iteration), while a world is unconverged, at most cap of them
  for (int loop = 0; loop < R.cap; ++loop) {
    if (*(volatile int*)P.n_unconv == 0) break;  // written by the last sums' grid ticket, read by all after a barrier
    for_blocks(R.team_blocks, [&](int vb) { cg_accel_team_at<MS>(P, P.cg_pd, P.cg_pdr, 0, vb); });
    ADF_BARRIER();
    for_blocks(R.team_blocks, [&](int vb) { cg_apply_team_at<MS>(P, P.cg_pd, P.cg_ap, 0, 0, 0, vb); });
    ADF_BARRIER();
    sums(0, 0);
    ADF_BARRIER();
    for_blocks(R.pt_blocks, [&](int vb) { cg_step_at(P, vb); });
    ADF_BARRIER();
    for_blocks(R.team_blocks, [&](int vb) { cg_accel_team_at<MS>(P, P.cg_corr, P.cg_corrr, 1, vb); });
    ADF_BARRIER();
    for_blocks(R.team_blocks, [&](int vb) { cg_apply_finish_team_at<MS>(P, vb); });
    ADF_BARRIER();
    sums(1, 1);
    ADF_BARRIER();
    for_blocks(R.pt_blocks, [&](int vb) { cg_direction_at(P, vb); });
    ADF_BARRIER();
  }
#undef ADF_BARRIER
}

}  // namespace adf
