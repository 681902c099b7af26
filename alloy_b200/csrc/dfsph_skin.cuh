// SPDX-License-Identifier: Apache-2.0
// Verlet-skin reuse of the liquid's neighbour rows (neighbors_skin.py:1-209, Config.reneighbor_skin).
//
// A superset row per liquid particle holds every liquid neighbour of its world within h + s (s = skin) at the row's
// build, in ascending particle id. It stays valid while no particle of the world has moved more than s / 2 since
// then and the world's liquid set is unchanged: every pair now closer than h was closer than h + s at the build.
// Each step: a world is flagged when one of its particles moved more than 0.49 s, became or stopped being liquid, or
// its world was forced by an overfull row last step; the flagged worlds' superset rows are rebuilt from this step's
// cell grid (the grid is re-sorted every step anyway); then a filter writes the rows the step reads: the superset
// entries now closer than h, in row order, the first K of them, by the same distance test as a plain build. Rows,
// counts and overflow counters therefore equal a plain build's bit for bit. A row with more than sup_cap entries
// within h + s is written as a plain radius-h row this step (the filter skips it) and its world rebuilds next step.
//
// Layout: superset rows live in [sup_cap][n] columns indexed by the particle's slot, the rank of its sorted position
// within its world's liquid at the build plus the world's first particle index, so a world's slots stay in its own
// index range whatever other worlds do, and a world whose order has not changed since its build reads its rows
// coalesced. Entries are particle ids (the caller's order), mapped to this step's sorted positions by pos_of.
#pragma once

#include "dfsph_kernels.cuh"

namespace adf {

// neighbors_skin.py:34-40: each world's rebuild flag starts as its force flag, which is cleared.
__global__ void k_skin_seed(DevP P) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  P.skin_flag[w] = P.skin_force[w];
  P.skin_force[w] = 0;
}

// Group of particle i for the skin test: its world when it is liquid, else -1.
__device__ __forceinline__ int skin_group(const DevP& P, int i, int w) { return is_fluid_orig(P, i) ? w : -1; }

// neighbors_skin.py:43-57, over the caller's particles: a world is flagged when a particle's group changed or it
// moved more than 0.49 s since its world's last build (a NaN position moves).
__global__ void k_skin_check(DevP P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int w = P.world[i];
  if (w < 0 || w >= P.W) return;
  const int g = skin_group(P, i, w);
  bool moved = g != P.skin_gref[i];
  if (!moved && g >= 0) {
    const float4 r = P.skin_qref[i];
    const float dx = P.q[3 * (size_t)i] - r.x, dy = P.q[3 * (size_t)i + 1] - r.y, dz = P.q[3 * (size_t)i + 2] - r.z;
    moved = !(dot_plain(dx, dy, dz, dx, dy, dz) <= P.skin_half2);
  }
  if (moved) P.skin_flag[w] = 1;
}

// The flagged worlds' reference positions and groups (neighbors_skin.py:76-78), over the caller's particles.
__global__ void k_skin_ref(DevP P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int w = P.world[i];
  if (w < 0 || w >= P.W || P.skin_flag[w] == 0) return;
  P.skin_qref[i] = make_float4(P.q[3 * (size_t)i], P.q[3 * (size_t)i + 1], P.q[3 * (size_t)i + 2], 0.0f);
  P.skin_gref[i] = skin_group(P, i, w);
}

// Appends particle id `id` to the ascending row at `row` (stride P.n) of m entries, keeping the cap lowest.
__device__ __forceinline__ void skin_insert(int* row, size_t stride, int& m, int cap, int id) {
  if (m == cap && id >= row[(size_t)(cap - 1) * stride]) return;
  int at = m < cap ? m : cap - 1;
  while (at > 0) {
    const int prev = row[(size_t)(at - 1) * stride];
    if (prev <= id) break;
    row[(size_t)at * stride] = prev;
    --at;
  }
  row[(size_t)at * stride] = id;
  if (m < cap) ++m;
}

// neighbors_skin.py:60-110 for the flagged worlds' liquid (sorted order): the superset row within h + s from the
// cells within skin_reach, or, when it holds more than sup_cap entries, this step's plain radius-h row (from the 27
// cells, as the plain build) and a forced rebuild next step. A row is sorted in the thread's column of the block's
// shared buffer (sup_cap x SKIN_THREADS ids, when sup_cap <= SKIN_SMEM_CAP) and then copied out; larger capacities
// sort in place in global memory.
constexpr int SKIN_THREADS = 128;
constexpr int SKIN_SMEM_CAP = 96;

__global__ void __launch_bounds__(SKIN_THREADS) k_skin_build(DevP P) {
  extern __shared__ int sbuf[];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  if (P.skin_flag[w] == 0) return;
  const int i = P.id_of[p];
  const int s = P.skin_ws[w] + (p - P.wrange[w].x);  // the particle's slot: its rank in its world's liquid
  P.skin_slot[i] = s;
  const WorldGrid g = P.grid[w];
  const float4 xi = P.pos[p];
  int cx, cy, cz;
  cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
  const int R = P.skin_reach, cap = P.sup_cap;
  const bool in_smem = cap <= SKIN_SMEM_CAP;
  int* row = in_smem ? sbuf + threadIdx.x : P.sup + s;
  const size_t stride = in_smem ? (size_t)SKIN_THREADS : (size_t)P.n;
  int m = 0, total = 0;
  for (int z = max(cz - R, 0); z <= min(cz + R, g.nz - 1); ++z)
    for (int y = max(cy - R, 0); y <= min(cy + R, g.ny - 1); ++y)
      for_row_ranges(P.cell_start, g, 0, y, z, max(cx - R, 0), min(cx + R, g.nx - 1), [&](int b, int e) {
        for (int j = b; j < e; ++j) {
          if (j == p) continue;
          const float4 xj = P.pos[j];
          const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
          if (dot_plain(dx, dy, dz, dx, dy, dz) < P.skin_r2) {
            ++total;
            skin_insert(row, stride, m, cap, P.id_of[j]);
          }
        }
      });
  if (total <= cap) {
    if (in_smem)
      for (int k = 0; k < m; ++k) P.sup[(size_t)k * P.n + s] = row[(size_t)k * SKIN_THREADS];
    P.sup_cnt[s] = m;
    return;
  }
  // too full for the superset: this step's plain row (ids in the row's own column, then mapped) and a rebuild next step
  int* nrow = P.nbr + p;
  const float h2 = P.kc.h2;
  const int K = P.K;
  m = 0;
  total = 0;
  for (int r = 0; r < 9; ++r) {
    const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
    if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) continue;
    for_row_ranges(P.cell_start, g, 0, y, z, max(cx - 1, 0), min(cx + 1, g.nx - 1), [&](int b, int e) {
      for (int j = b; j < e; ++j) {
        if (j == p) continue;
        const float4 xj = P.pos[j];
        const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        if (dot_plain(dx, dy, dz, dx, dy, dz) < h2) {
          ++total;
          skin_insert(nrow, P.n, m, K, P.id_of[j]);
        }
      }
    });
  }
  for (int k = 0; k < m; ++k) nrow[(size_t)k * P.n] = P.pos_of[nrow[(size_t)k * P.n]];
  P.cnt[p] = m;
  if (total > K) atomicAdd(&P.overflow[w], 1);
  P.sup_cnt[s] = -1;
  P.skin_force[w] = 1;
}

// neighbors_skin.py:113-140 (sorted order): the rows of this step from the superset rows, by the plain build's test
// (d = x_j - x_i, d.d < h^2), in row order, the first K of them; overfull rows count in the world's overflow.
__global__ void __launch_bounds__(BLOCK) k_skin_filter(DevP P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int s = P.skin_slot[P.id_of[p]];
  const int sc = P.sup_cnt[s];
  if (sc < 0) return;  // a plain row written by this step's rebuild
  const float4 xi = P.pos[p];
  const float h2 = P.kc.h2;
  const int K = P.K;
  int m = 0, total = 0;
  constexpr int SB = 8;  // superset entries in flight: their ids, then their sorted positions, then the positions
  for (int k0 = 0; k0 < sc; k0 += SB) {
    int j[SB];
#pragma unroll
    for (int u = 0; u < SB; ++u) j[u] = k0 + u < sc ? P.sup[(size_t)(k0 + u) * P.n + s] : -1;
#pragma unroll
    for (int u = 0; u < SB; ++u) j[u] = j[u] >= 0 ? P.pos_of[j[u]] : p;
    float4 xj[SB];
#pragma unroll
    for (int u = 0; u < SB; ++u) xj[u] = P.pos[j[u]];
#pragma unroll
    for (int u = 0; u < SB; ++u) {
      if (k0 + u >= sc) break;
      const float dx = xj[u].x - xi.x, dy = xj[u].y - xi.y, dz = xj[u].z - xi.z;
      if (dot_plain(dx, dy, dz, dx, dy, dz) < h2) {
        ++total;
        if (m < K) P.nbr[(size_t)m++ * P.n + p] = j[u];
      }
    }
  }
  P.cnt[p] = m;
  if (total > K) atomicAdd(&P.overflow[P.world_s[p]], 1);
}

}  // namespace adf
