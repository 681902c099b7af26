// SPDX-License-Identifier: Apache-2.0
// DFSPH step kernels for sm_100a. One thread per particle; particles of every world are sorted by (class, world,
// cell) at the start of each step so that a warp's neighbour gathers land in a few cells (L1/L2 locality) and every
// array the neighbour loops stream is structure-of-arrays (float4 position+mass, float4 velocity+rest density).
//
// Sorted space: fluid particles occupy [0, nf), boundary (wall) particles [nf, nf + nw); other particles (spares,
// retired, foreign) stay in the caller's arrays only. Results never depend on where a particle lands inside its
// cell: neighbour rows are kept in ascending original particle id (the reference's order), wall-colour sums run in
// ascending wall-particle id, and per-world float64 reductions run over the caller's particle order.
#pragma once

#include <climits>
#include <cstdint>

#include "dfsph_math.cuh"
#include "dfsph_reduce.cuh"

namespace adf {

constexpr int BLOCK = 256;
constexpr int MAXCAP = 128;      // largest neighbor_capacity
constexpr int WT = 4;            // lanes per near-wall particle in k_wall_slots
constexpr int WT_CAP = 48;       // wall particles within h a team sorts in shared memory (more: one lane does it)
constexpr int MAXWALL = 160;     // wall particles within h of one fluid particle (far above any lattice wall)
constexpr int FLAG_ACTIVE = 1;
constexpr int FLAG_PROXY = 2;
constexpr int PROJECT_PASSES = 4;  // integrate.py:50

// A world's cell grid. Cells are numbered tile by tile (4 x 4 x 4 cells per tile, tiles in x-fastest order, cells
// x-fastest inside a tile), so a run of consecutive sorted particles covers a compact brick of space and its
// neighbourhood stays small enough for L1. Cells of one tile row with consecutive x have consecutive keys.
struct WorldGrid {
  float ox, oy, oz, inv_cw;  // origin, 1 / cell width
  int nx, ny, nz, base;      // cells per axis (multiples of 4), first cell of the world in the class-0 key space
  int tnx, tny, pad0, pad1;  // tiles per axis (x, y)
};

__device__ __forceinline__ int cell_key(const WorldGrid& g, int x, int y, int z) {
  return g.base + ((((z >> 2) * g.tny + (y >> 2)) * g.tnx + (x >> 2)) << 6) + (((z & 3) << 4) | ((y & 3) << 2) | (x & 3));
}

// Sorted ranges [b, e) of the cells x = x0..x1 of row (y, z) of key class `cls_off` (0 liquid, total_cells walls):
// one range per tile the row crosses.
template <class F>
__device__ __forceinline__ void for_row_ranges(const int* cell_start, const WorldGrid& g, int cls_off, int y, int z,
                                               int x0, int x1, F&& f) {
  for (int x = x0; x <= x1;) {
    const int xe = min(x1, x | 3);
    f(cell_start[cls_off + cell_key(g, x, y, z)], cell_start[cls_off + cell_key(g, xe, y, z) + 1]);
    x = xe + 1;
  }
}

struct Emit {
  int world, n_layer, pool_begin, pool_size;
  float xform[7];
  float vel[3];
  float interval;
};

struct Sink {
  int world;
  float xform[7];
  float half[3];
};

// Everything a kernel needs, passed by value.
struct DevP {
  KC kc;
  int n;            // particle capacity (caller's n)
  int W;
  int K;            // neighbour capacity
  int total_cells;  // cells of all worlds (one class)
  float dt, n_full, tot_min, wall_offset, wall_amp, taper0, taper1, reach, omega, warm, warm_den, warm_div, min_nb;
  float xsph_c, v_sep, relief, eps;
  int mode;  // 0 divergence, 1 density
  int two_sided;
  float tol, tol_max;
  const float* tol_scale;  // [W] factor of tol and tol_max per world (the resting-jitter rule), null: 1
  int min_it, max_it;
  int has_bounds;
  float blo[3], bhi[3];
  int n_sinks;
  const Sink* sinks;
  // caller model (original order)
  const float* mass;
  const float* rho0;
  int32_t* flags;
  int8_t* phase;
  const int32_t* world;
  const float* wall_vol;
  const float* gravity;
  const float* f_ext;
  // state in/out (original order, [n][3])
  float* q;
  float* qd;
  // persistent warm starts (original order)
  float* kv;
  float* kd;
  // sorting
  const WorldGrid* grid;
  int* key_of;
  int* counts;      // [2 total_cells]
  int* cell_start;  // [2 total_cells + 1]
  int* nfw;         // [2]: nf, nw
  // sorted space
  float4* pos;   // x y z, mass (fluid) or wall volume (walls)
  float4* vel;   // vx vy vz, rest density
  float4* vel2;  // XSPH output
  int* id_of;
  int* pos_of;  // caller order -> sorted position (liquid and walls; written by k_scatter)
  int* world_s;
  float* kv_s;
  float* kd_s;
  int* nbr;     // [K][n] sorted positions, ascending original id
  int2* nbrjf;  // [K][n] (row entry, bits of its gradient factor F(r_ij)), written by k_density_alpha
  float* nbrw;  // [K][n] kernel value W(r_ij) of each row entry, written by k_density_alpha, read by k_xsph
  int* cnt;
  // Item halos of the pressure iterations (k_halo): per 256-particle work item g (world w, first particle b:
  // g = b / 256 + w) the ascending sorted positions its rows address, and the rows as 16-bit indices into that list.
  int* halo_n;              // [G] records of item g; -1: not staged (too many, or too wide a span)
  int* halo_idx;            // [G][HALO_CAP] sorted positions
  unsigned short* halo_row;  // [K][n] row entry as an index into its item's halo
  float* halo_f;            // [K][n] the entry's F(r_ij), as in nbrjf
  // Boundary slots (boundary.py:36): slot b of sorted particle p at b * n + p of each array, nearest wall first.
  float4* slot_g;   // dPsi/dx (3), psi; with slot_cap 1, psi < 0: no slot
  float4* slot_vb;  // wall velocity (3), phi
  float4* slot_n;   // outward normal (3), the wall's id as int bits (the particle wall's is n_shapes)
  float4* slot_xb;  // start-of-step surface point (3; world frame for the particle wall, the box's frame for a box), 0
  int slot_cap;      // 1: the particle wall only; 4: static box walls too (boundary.py:36 NUM_SLOTS)
  int8_t* slot_cnt;  // [n] slots in use (slot_cap 4)
  // the liquid's static axis-aligned box walls (layout.py:207-246), ids into the model's shape table
  int n_shapes;
  const int* sh_start;    // [W + 1]: world w's walls are sh_ids[sh_start[w] .. sh_start[w + 1])
  const int* sh_ids;
  const float4* sh_pos;   // centre (3), bounding radius
  const float4* sh_half;  // the shape's scale (3: box half extents; sphere radius; capsule radius, half height; plane
                          // width, length, 0 for an infinite plane), Coulomb friction mu
  const int* sh_geo;      // newton GeoType per shape (GEO_BOX, GEO_SPHERE, GEO_CAPSULE, GEO_CYLINDER, GEO_PLANE)
  const float4* sh_quat;  // the shape frame's rotation (x, y, z, w); slots hold world normals and world-oriented
                          // offsets of their closest points from the shape's origin
  float sweep_len;        // a step longer than this is swept against the world's boxes (integrate.py:42-49)
  float prad;             // particle radius
  int wall_friction;      // Config.wall_friction
  int* swept;             // [W] particles swept onto a box this step
  // Verlet-skin reuse of the rows (dfsph_skin.cuh; skin_on 0: rows built every step)
  int skin_on;
  int sup_cap;          // superset row capacity
  int skin_reach;       // cells scanned on each side for radius h + s
  float skin_r2;        // (h + s)^2
  float skin_half2;     // (0.49 s)^2
  int* sup;             // [sup_cap][n] superset rows (particle ids, ascending) by slot
  int* sup_cnt;         // [n] by slot: entries, or -1 for a plain row written by this step's rebuild
  int* skin_slot;       // [n] caller order: the particle's slot at its world's last build
  float4* skin_qref;    // [n] caller order: position at its world's last build
  int* skin_gref;       // [n] caller order: group at its world's last build (-2: never built)
  int* skin_flag;       // [W] world rebuilt this step
  int* skin_force;      // [W] world rebuilds next step (an overfull superset row)
  const int* skin_ws;   // [W + 1] first particle index of each world
  float* ratio;
  float* alpha;
  float* neff;
  float* reg;
  float* src;
  float* kappa;
  float* lower;
  float* kr;  // kappa / rho0
  float4* acc;
  float* err_orig;  // original order
  // per world
  int2* wrange;     // [W] sorted liquid range of each world (k_post_scan)
  int* cw;          // [W] worlds still iterating, ascending (k_worklist)
  int* cseg;        // [W + 1] first work item of each listed world; cseg[n_cw] = items
  int* n_cw;        // [1] listed worlds
  unsigned long long* iter_work;  // [1] liquid particles covered by the pressure iterations' work lists so far
  int* converged;
  int* iters;
  float* err_mean;
  int* n_unconv;
  int* wdone;        // [W] chunk blocks of the world finished in the running reduction launch (reset by its last)
  unsigned* gdone;   // worlds of the running reduction launch finished (reset by its last)
  int n_chunk_worlds;  // worlds with at least one chunk
  double* n_active;
  int* overflow;
  int* escaped;
  int* projected;
  int* nonfinite;
  int* wall_overflow;
  int* max_speed_bits;  // float bits of a non-negative max
  long long* mass_out;
  // reductions (original order)
  const int* chunk_begin;
  const int* chunk_end;
  const int* world_chunk_start;
  const int* chunk_world;
  int n_chunks;
  double* part_sum;
  float* part_max;
  float* emax;
  // learned warm start (null when off)
  float* feat;      // [nf][16] features at the step's first solve (sorted), written by k_solve_init when feat_on
  int feat_on;
  float* pred_kv;   // [n] predicted kappa dt (sorted)
  float* pred_kd;   // [n] predicted kappa dt^2 (sorted)
  float* kappa2;    // the learned start's kappa, kappa / rho0, acceleration and residual (first sweep)
  float* kr2;
  float4* acc2;
  float* err2;      // original order
  int* use_l;       // [W] 1: this solve continues from the learned start
  int* learned;     // [2][W] the last step's choice per solve (divergence, density)
  double* sum_c;    // [W] first-sweep residual sums and maxima from the plain and the learned start
  double* sum_l;
  float* max_c;
  float* max_l;
  // evaluation schedule of the learned start under the judge (k_probe_plan)
  int* probe_skip;  // [W] 1: this solve does not evaluate the learned start in the world
  int* probe_gap;   // [2][W] solves between evaluations (per solve kind)
  int* probe_wait;  // [2][W] solves of this kind left before the next evaluation
  const int* warm_need;  // [W] worlds whose learned start is evaluated in one of this step's solves (null: all)
  // projected preconditioned CG (krylov.py; null unless the CG pressure solver is selected)
  float* cg_pd;     // search direction p, and p / rho0 (sorted)
  float* cg_pdr;
  float* cg_z;      // M^-1 r on the active set
  float* cg_w;      // w = A k - b
  float* cg_ap;     // A p
  float* cg_corr;   // clamped part of the step, and / rho0
  float* cg_corrr;
  int* cg_act;      // 1: in the active set F
  float2* cg_pair;  // original order: (dot-product term, error) for the per-world sums
  double* cg_rz;    // [W] r.z
  double* cg_step;  // [W] beta
  double2* cg_sums; // [W] (sum of pair.x, sum of pair.y)
  int* cg_restart;  // [W] variables clamped onto their bound this iteration (k_cg_step)
  int* cg_act_new;  // [W] set when a bound variable was activated this iteration (k_cg_apply_finish)
  double2* part2;   // [chunks] partial sums of pairs
};

// Slots in use by sorted liquid particle p, and the index of its slot b.
__device__ __forceinline__ int slot_count(const DevP& P, int p) {
  return P.slot_cap > 1 ? (int)P.slot_cnt[p] : (P.slot_g[p].w >= 0.0f ? 1 : 0);
}
__device__ __forceinline__ size_t slot_at(const DevP& P, int b, int p) { return (size_t)b * P.n + p; }

// Neighbour-loop kernels take one template integer NBX: the gathers they keep in flight, NB = NBX & NB_MASK, plus
// MS_FLAG when the model has box walls (up to four slots per particle). Without the flag a kernel is compiled for the
// particle-wall build's single slot, one pass of the multi-slot arithmetic, so the common case carries no loop.
constexpr int NB_MASK = 31, MS_FLAG = 32;

// f(b, o) for each wall slot of sorted liquid particle p, nearest first (o: the slot's index in the slot arrays)
template <bool MS, class F>
__device__ __forceinline__ void for_slots(const DevP& P, int p, F f) {
  if constexpr (MS) {
    const int ns = P.slot_cnt[p];
    for (int b = 0; b < ns; ++b) f(b, slot_at(P, b, p));
  } else {
    if (P.slot_g[p].w >= 0.0f) f(0, (size_t)p);
  }
}

__device__ __forceinline__ bool is_fluid_orig(const DevP& P, int i) {
  return (P.flags[i] & FLAG_ACTIVE) != 0 && P.phase[i] >= 1;
}

__device__ __forceinline__ void cell_coords(const WorldGrid& g, float x, float y, float z, int& cx, int& cy, int& cz) {
  float fx = floorf(__fmul_rn(__fsub_rn(x, g.ox), g.inv_cw));
  float fy = floorf(__fmul_rn(__fsub_rn(y, g.oy), g.inv_cw));
  float fz = floorf(__fmul_rn(__fsub_rn(z, g.oz), g.inv_cw));
  fx = fminf(fmaxf(fx, 0.0f), (float)(g.nx - 1));
  fy = fminf(fmaxf(fy, 0.0f), (float)(g.ny - 1));
  fz = fminf(fmaxf(fz, 0.0f), (float)(g.nz - 1));
  cx = (int)fx;
  cy = (int)fy;
  cz = (int)fz;
}

// ------------------------------------------------------------------------------------------------ sorting
// Groups (neighbors.py:36-51): fluid = ACTIVE and phase >= 1; wall = a boundary particle (PROXY at creation),
// ACTIVE, in a world; every other particle stays out of the sorted arrays.
__global__ void k_classify(DevP P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int w = P.world[i];
  int cls = -1;
  if (w >= 0 && w < P.W) {
    if (is_fluid_orig(P, i)) cls = 0;
    else if (P.wall_vol[i] > 0.0f && (P.flags[i] & FLAG_ACTIVE) != 0) cls = 1;
  }
  if (cls < 0) {
    P.key_of[i] = -1;
    return;
  }
  const WorldGrid g = P.grid[w];
  int cx, cy, cz;
  cell_coords(g, P.q[3 * i], P.q[3 * i + 1], P.q[3 * i + 2], cx, cy, cz);
  int key = cls * P.total_cells + cell_key(g, cx, cy, cz);
  P.key_of[i] = key;
  atomicAdd(&P.counts[key], 1);
}

// Exclusive scan of n ints in three passes (per-block sums, a one-block scan of those, per-block scan + offset).
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = (lane < (int)(blockDim.x >> 5)) ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    smem[lane] = s;
  }
  __syncthreads();
  int off = wid > 0 ? smem[wid - 1] : 0;
  total = smem[(blockDim.x >> 5) - 1];
  __syncthreads();
  return off + x - v;
}

__global__ void k_scan_tiles(const int* in, int n, int* tile_sums) {
  __shared__ int smem[32];
  int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) s += (base + k < n) ? in[base + k] : 0;
  int total;
  block_exclusive_scan(s, smem, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_tile_sums(int* tile_sums, int n_tiles) {
  __shared__ int smem[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b = 0; b < n_tiles; b += blockDim.x) {
    int i = b + threadIdx.x;
    int v = i < n_tiles ? tile_sums[i] : 0;
    int total;
    int ex = block_exclusive_scan(v, smem, total);
    int c = carry;
    if (i < n_tiles) tile_sums[i] = c + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry = c + total;
    __syncthreads();
  }
}

__global__ void k_scan_apply(const int* in, int n, const int* tile_off, int* out) {
  __shared__ int smem[32];
  int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  int total;
  int ex = block_exclusive_scan(s, smem, total) + tile_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int idx = base + k;
    if (idx < n) out[idx] = ex;
    ex += v[k];
    if (idx == n - 1) out[n] = ex;
  }
}

// Fluid and wall counts, and each world's liquid count (n_active, an exact integer in float64).
__global__ void k_post_scan(DevP P, const int* world_cells) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w == 0) {
    int nf = P.cell_start[P.total_cells];
    P.nfw[0] = nf;
    P.nfw[1] = P.cell_start[2 * P.total_cells] - nf;
  }
  if (w >= P.W) return;
  int b = P.grid[w].base;
  const int lb = P.cell_start[b], le = P.cell_start[b + world_cells[w]];
  P.wrange[w] = make_int2(lb, le);
  P.n_active[w] = (double)(le - lb);
}

// Place each particle in its cell's range and gather its data into the sorted arrays. The counts go back to zero.
__global__ void k_scatter(DevP P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int key = P.key_of[i];
  if (key < 0) return;
  int p = P.cell_start[key] + atomicSub(&P.counts[key], 1) - 1;
  bool fluid = key < P.total_cells;
  float m = fluid ? P.mass[i] : P.wall_vol[i];
  P.pos[p] = make_float4(P.q[3 * i], P.q[3 * i + 1], P.q[3 * i + 2], m);
  P.vel[p] = make_float4(P.qd[3 * i], P.qd[3 * i + 1], P.qd[3 * i + 2], P.rho0[i]);
  P.id_of[p] = i;
  P.pos_of[i] = p;
  P.world_s[p] = P.world[i];
  if (fluid) {
    P.kv_s[p] = P.kv[i];
    P.kd_s[p] = P.kd[i];
  }
}

// ----------------------------------------------------------------------------------------- neighbour rows
// neighbors.py:160-195: fluid neighbours j != i of the same world with |x_j - x_i|^2 < h^2, ascending original id,
// the lowest K kept; a world's overflow counter counts particles with more than K.

// The same rows, one thread per particle with its row kept in shared memory as ascending original ids (entry k of
// thread t at [k][t]: threads inserting at the same k use distinct banks), mapped back to sorted positions through
// pos_of when written. 32 independent particles per warp keep many candidate loads in flight.
constexpr int LS_THREADS = 128;

__global__ void __launch_bounds__(LS_THREADS) k_lists_smem(DevP P) {
  extern __shared__ int srow[];
  const int p = blockIdx.x * LS_THREADS + threadIdx.x;
  if (p >= P.nfw[0]) return;
  int* buf = srow + threadIdx.x;
  const int K = P.K;
  const int w = P.world_s[p];
  const WorldGrid g = P.grid[w];
  const float4 xi = P.pos[p];
  const float h2 = P.kc.h2;
  int cx, cy, cz;
  cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
  const int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.nx - 1);
  int m = 0, total = 0;
  for (int r = 0; r < 9; ++r) {
    const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
    if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) continue;
    for_row_ranges(P.cell_start, g, 0, y, z, x0, x1, [&](int b, int e) {
      for (int j = b; j < e; ++j) {
        if (j == p) continue;
        float4 xj = P.pos[j];
        float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        if (dot_plain(dx, dy, dz, dx, dy, dz) < h2) {
          ++total;
          const int id = P.id_of[j];
          if (m == K && id >= buf[(K - 1) * LS_THREADS]) continue;
          int at = (m < K) ? m : K - 1;
          while (at > 0) {
            int prev = buf[(at - 1) * LS_THREADS];
            if (prev <= id) break;
            buf[at * LS_THREADS] = prev;
            --at;
          }
          buf[at * LS_THREADS] = id;
          if (m < K) ++m;
        }
      }
    });
  }
  for (int k = 0; k < m; ++k) P.nbr[(size_t)k * P.n + p] = P.pos_of[buf[k * LS_THREADS]];
  P.cnt[p] = m;
  if (total > K) atomicAdd(&P.overflow[w], 1);
}

// Rows of 32 consecutive sorted particles built by one warp in lockstep (capacity K <= 64):
//  1. scan: the union of the 32 particles' 27-cell neighbourhoods is one box of cells; each of its cell rows splits
//     into at most one contiguous candidate range per 4-cell tile. The ranges are flattened into one candidate
//     stream (offsets by a warp scan), 32 candidates at a time are staged in shared memory (the next 32 already in
//     flight in registers) and every lane tests all of them against its own particle as a 32-bit pass mask, then
//     appends the original ids of the passing ones to its row (unsorted). A warp whose particles span a large box
//     (a splash, several worlds) runs the same scan once per compact group of its lanes.
//  2. order: rows of at most 32 entries are sorted in registers by a fully unrolled bitonic network; longer rows by
//     insertion in shared memory; a row with more than 64 candidates selects its K lowest ids by repeated scans.
//  3. write: entry k of the 32 rows is one contiguous 128-byte segment (ids mapped to sorted positions by pos_of).
constexpr int LU_WARPS = 4;
constexpr int LU_ROW = 64;         // row buffer per particle (and the largest capacity this kernel builds)
constexpr int LU_MAX_ROWS = 64;    // cell rows (y, z) of the warp's box scanned in lockstep
constexpr int LU_MAX_SEGS = 160;   // candidate ranges (row x tile) scanned in lockstep

__device__ __forceinline__ void sort32_registers(unsigned (&key)[32]) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned a = key[i], b = key[l];
          const unsigned lo = min(a, b), hi = max(a, b);
          if ((i & k) == 0) {
            key[i] = lo;
            key[l] = hi;
          } else {
            key[i] = hi;
            key[l] = lo;
          }
        }
      }
    }
  }
}

__device__ __forceinline__ void sort16_registers(unsigned (&key)[16]) {
#pragma unroll
  for (int k = 2; k <= 16; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned a = key[i], b = key[l];
          const unsigned lo = min(a, b), hi = max(a, b);
          if ((i & k) == 0) {
            key[i] = lo;
            key[l] = hi;
          } else {
            key[i] = hi;
            key[l] = lo;
          }
        }
      }
    }
  }
}

// G particles per warp: 32 (one lane per particle), or 16 (lanes l and l + 16 share particle l: the warp's union of
// neighbourhoods is about a third smaller and each lane tests every other candidate pair of each staged batch; the
// two lanes' sorted runs are merged on write by lane l). The rows are the same either way.
template <int G>
__global__ void __launch_bounds__(32 * LU_WARPS) k_lists_union(DevP P) {
  __shared__ unsigned rows[LU_WARPS][LU_ROW][32];  // [warp][entry][lane]: lanes of one entry in distinct banks
  __shared__ __align__(8) float cxs[LU_WARPS][32];  // staged candidates, one coordinate per array so that two
  __shared__ __align__(8) float cys[LU_WARPS][32];  // neighbouring candidates are one 8-byte broadcast load
  __shared__ __align__(8) float czs[LU_WARPS][32];
  __shared__ unsigned cid[LU_WARPS][32];
  __shared__ int rbeg[LU_WARPS][LU_MAX_SEGS];     // first sorted index of each candidate range
  __shared__ int roff[LU_WARPS][LU_MAX_SEGS + 1];  // flat offset of each range in the warp's candidate stream
  static_assert(G == 32 || G == 16, "particles per warp");
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int sub = lane % G, half = lane / G;
  const int p0 = (blockIdx.x * LU_WARPS + wq) * G;
  const int nf = P.nfw[0];
  if (p0 >= nf) return;
  const int tend = min(G, nf - p0);
  const bool valid = sub < tend;
  const int p = valid ? p0 + sub : p0;
  const int w = P.world_s[p];
  const WorldGrid g = P.grid[w];
  const float4 xi = P.pos[p];
  const float h2 = P.kc.h2;
  const int K = P.K;
  int cx, cy, cz;
  cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
  const unsigned full = 0xffffffffu;
  unsigned* myrow = &rows[wq][0][lane];
  int cnt = 0, total = 0;
  const unsigned myid = (unsigned)P.id_of[p];
  const f32x2 xi2 = f2_dup(xi.x), yi2 = f2_dup(xi.y), zi2 = f2_dup(xi.z);
  // One lockstep scan of the lanes with `in` set; false (before any candidate is read) when they span more than one
  // world or their box needs more rows or tile segments than the tables hold. The whole warp is scanned at once when
  // it can be; otherwise (a splash, a sparse tile, a world boundary in the sorted order) its lanes are scanned in
  // groups, each the pending lanes of the lowest pending lane's world within 2 cells of its cell per axis: a box of at
  // most 7 x 7 x 7 cells, 49 cell rows of at most 3 tile segments, which the tables always hold.
  auto scan = [&](const bool in) -> bool {
    const int w_lo = __reduce_min_sync(full, in ? (unsigned)w : 0xffffffffu);
    const int w_hi = __reduce_max_sync(full, in ? (unsigned)w : 0u);
    if (w_lo != w_hi) {  // only the whole warp: a group's lanes share the leader's world
      return false;
    }
    const WorldGrid gw = P.grid[w_lo];  // the group's world: every lane computes its cell rows and ranges in it
    const int ylo = max((int)__reduce_min_sync(full, in ? (unsigned)cy : 0xffffffffu) - 1, 0);
    const int yhi = min((int)__reduce_max_sync(full, in ? (unsigned)cy : 0u) + 1, gw.ny - 1);
    const int zlo = max((int)__reduce_min_sync(full, in ? (unsigned)cz : 0xffffffffu) - 1, 0);
    const int zhi = min((int)__reduce_max_sync(full, in ? (unsigned)cz : 0u) + 1, gw.nz - 1);
    const int sy = yhi - ylo + 1, sz = zhi - zlo + 1, nrows = sy * sz;
    if (nrows > LU_MAX_ROWS) {  // likewise: a group spans at most 7 x 7 cell rows
      return false;
    }
    // rows (y, z) of the box, row-major; row j's x range is the union of [cx - 1, cx + 1] over the group's lanes
    // whose cell is within one row of it (empty: x0 > x1). Lane l keeps rows l and l + 32.
    int ax0 = 1, ax1 = 0, bx0 = 1, bx1 = 0;
    for (int j = 0; j < nrows; ++j) {
      const int y = ylo + j % sy, z = zlo + j / sy;
      const bool near = in && abs(cy - y) <= 1 && abs(cz - z) <= 1;
      const unsigned mn = __reduce_min_sync(full, near ? (unsigned)cx : 0xffffffffu);
      const unsigned mx = __reduce_max_sync(full, near ? (unsigned)(cx + 1) : 0u);
      if (lane == (j & 31) && mx != 0u) {
        const int x0 = max((int)mn - 1, 0), x1 = min((int)mx, gw.nx - 1);
        if (j < 32) {
          ax0 = x0;
          ax1 = x1;
        } else {
          bx0 = x0;
          bx1 = x1;
        }
      }
    }
    // one candidate range per tile a row's x range crosses; exclusive scan of the range counts over rows 0..63
    const int sa = ax0 <= ax1 ? (ax1 >> 2) - (ax0 >> 2) + 1 : 0;
    const int sb = bx0 <= bx1 ? (bx1 >> 2) - (bx0 >> 2) + 1 : 0;
    int ia = sa, ib = sb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int va = __shfl_up_sync(full, ia, o), vb = __shfl_up_sync(full, ib, o);
      if (lane >= o) {
        ia += va;
        ib += vb;
      }
    }
    const int ta = __shfl_sync(full, ia, 31);
    const int nseg = ta + __shfl_sync(full, ib, 31);
    if (nseg > LU_MAX_SEGS) {  // only the whole warp: a group has at most 49 rows x 3 segments
      return false;
    }
    // ranges' first sorted index into rbeg; their lengths, prefixed within the row, into roff[r + 1]
    int na = 0, nb = 0;
    for (int hf = 0; hf < 2; ++hf) {
      const int j = lane + 32 * hf;
      const int x0 = hf ? bx0 : ax0, x1 = hf ? bx1 : ax1;
      const int r0 = hf ? ta + ib - sb : ia - sa;
      const int y = ylo + j % sy, z = zlo + j / sy;
      int acc = 0;
      for (int xs = x0, r = r0; xs <= x1; ++r) {
        const int xe = min(x1, xs | 3);
        const int bb = P.cell_start[cell_key(gw, xs, y, z)];
        const int ee = P.cell_start[cell_key(gw, xe, y, z) + 1];
        rbeg[wq][r] = bb;
        acc += ee - bb;
        roff[wq][r + 1] = acc;
        xs = xe + 1;
      }
      (hf ? nb : na) = acc;
    }
    // candidates before each row: scan of the row totals over rows 0..63, then shift each row's ranges by it
    int ca = na, cb = nb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int va = __shfl_up_sync(full, ca, o), vb = __shfl_up_sync(full, cb, o);
      if (lane >= o) {
        ca += va;
        cb += vb;
      }
    }
    const int tca = __shfl_sync(full, ca, 31);
    const int T = tca + __shfl_sync(full, cb, 31);
    for (int r = ia - sa; r < ia; ++r) roff[wq][r + 1] += ca - na;
    for (int r = ta + ib - sb; r < ta + ib; ++r) roff[wq][r + 1] += tca + cb - nb;
    if (lane == 0) roff[wq][0] = 0;
    __syncwarp();
    int rr = 0;  // range of this lane's next candidate; candidates lane, lane + 32, ... only move it forward
    float4 nxt = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    unsigned nid = 0u;
    auto fetch = [&](int c) {
      if (c < T) {
        while (roff[wq][rr + 1] <= c) ++rr;
        const int j = rbeg[wq][rr] + (c - roff[wq][rr]);
        nxt = P.pos[j];
        nid = (unsigned)P.id_of[j];
      }
    };
    fetch(lane);
    for (int c0 = 0; c0 < T; c0 += 32) {
      const int nc = min(32, T - c0);
      cxs[wq][lane] = nxt.x;
      cys[wq][lane] = nxt.y;
      czs[wq][lane] = nxt.z;
      cid[wq][lane] = nid;
      __syncwarp();
      fetch(c0 + 32 + lane);
      unsigned hit = 0u;
      // two candidates per step: the differences in one packed f32x2 subtraction each (exactly rounded per half),
      // squares and sums in scalar dot_plain. Packed multiplies feeding packed adds are not used: the assembler fuses
      // a single-use packed product into the add, which changes the rounding of d^2 at the h^2 boundary.
      auto pair_hits = [&](int t) -> unsigned {
        const f32x2 dx = f2_sub(f2_load(&cxs[wq][t]), xi2);
        const f32x2 dy = f2_sub(f2_load(&cys[wq][t]), yi2);
        const f32x2 dz = f2_sub(f2_load(&czs[wq][t]), zi2);
        const float ax = f2_lo(dx), ay = f2_lo(dy), az = f2_lo(dz);
        const float bx = f2_hi(dx), by = f2_hi(dy), bz = f2_hi(dz);
        return (dot_plain(ax, ay, az, ax, ay, az) < h2 ? 1u : 0u) | (dot_plain(bx, by, bz, bx, by, bz) < h2 ? 2u : 0u);
      };
      // this lane's share of the staged batch: every pair (G = 32), or every other pair (G = 16: pairs 0, 2, 4, ... for
      // the first lane of a particle, 1, 3, 5, ... for the second), so that a particle's hits, which come in runs of
      // the same few cells, split about evenly between its two lanes (halves of the batch did not: on a settled
      // column one lane could get all 37 hits of a row, more than its sorted run holds)
      constexpr int STEP = G == 32 ? 2 : 4;
      const int t0 = G == 32 ? 0 : 2 * half;
      if (nc == 32) {
#pragma unroll
        for (int t = t0; t < 32; t += STEP) hit |= pair_hits(t) << t;
      } else {
        for (int t = t0; t < nc; t += STEP) hit |= pair_hits(t) << t;
        hit &= (1u << nc) - 1u;  // nc < 32: drop the stale slot past the last candidate
      }
      if (!in) hit = 0u;
      while (hit) {
        const int t = __ffs(hit) - 1;
        hit &= hit - 1u;
        const unsigned id = cid[wq][t];
        if (id != myid) {
          if (cnt < LU_ROW) myrow[cnt * 32] = id;
          ++cnt;
        }
      }
      __syncwarp();
    }
    return true;
  };
  if (!scan(true)) {
    unsigned pending = __ballot_sync(full, valid);
    while (pending) {
      const int ld = __ffs(pending) - 1;
      const int lw = __shfl_sync(full, w, ld), lx = __shfl_sync(full, cx, ld), ly = __shfl_sync(full, cy, ld),
                lz = __shfl_sync(full, cz, ld);
      const bool in =
          ((pending >> lane) & 1u) && w == lw && abs(cx - lx) <= 2 && abs(cy - ly) <= 2 && abs(cz - lz) <= 2;
      scan(in);
      pending &= ~__ballot_sync(full, in);
    }
  }
  const int own = valid ? cnt : 0;                                       // this lane's hits
  const int other = G == 16 ? __shfl_xor_sync(full, own, 16) : 0;       // its partner lane's (G = 16)
  total = own + other;
  const bool writer = valid && half == 0;
  cnt = min(own, LU_ROW);
  const int cmax = __reduce_max_sync(full, (unsigned)cnt);
  // G = 32: run A = entries [0, min(cnt, 32)), run B = entries [32, cnt) of this lane's column; G = 16: run A = this
  // lane's column, run B = the partner's; each run sorted in registers
  const bool sel = total > LU_ROW || (G == 16 && (own > 32 || other > 32));
  int a_end = min(cnt, 32), b_end = cnt, b_begin = 32;
  if (G == 16) {
    a_end = min(own, 32);
    b_end = min(other, 32);
    b_begin = 0;
  }
  if (G == 16 && cmax <= 16) {
    unsigned key[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) key[k] = k < cnt ? myrow[k * 32] : 0xffffffffu;
    sort16_registers(key);
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (k < cnt) myrow[k * 32] = key[k];
  } else {
    unsigned key[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) key[k] = k < cnt ? myrow[k * 32] : 0xffffffffu;
    sort32_registers(key);
#pragma unroll
    for (int k = 0; k < 32; ++k)
      if (k < cnt) myrow[k * 32] = key[k];
  }
  if (G == 32 && cmax > 32) {
    unsigned key[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) key[k] = 32 + k < cnt ? myrow[(32 + k) * 32] : 0xffffffffu;
    sort32_registers(key);
#pragma unroll
    for (int k = 0; k < 32; ++k)
      if (32 + k < cnt) myrow[(32 + k) * 32] = key[k];
  }
  __syncwarp();  // the partner's sorted run is read below (G = 16)
  if (sel && writer) {
    // more candidates than the row buffer: the K lowest ids by repeated scans of this particle's 27 cells
    unsigned last = 0;
    const int kk = min(total, K);
    for (int k = 0; k < kk; ++k) {
      unsigned best = 0xffffffffu;
      for (int r = 0; r < 9; ++r) {
        const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
        if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) continue;
        for_row_ranges(P.cell_start, g, 0, y, z, max(cx - 1, 0), min(cx + 1, g.nx - 1), [&](int b, int e) {
          for (int j = b; j < e; ++j) {
            if (j == p) continue;
            const float4 xj = P.pos[j];
            const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            if (dot_plain(dx, dy, dz, dx, dy, dz) < h2) {
              const unsigned id = (unsigned)P.id_of[j];
              if ((k == 0 || id > last) && id < best) best = id;
            }
          }
        });
      }
      myrow[k * 32] = best;
      last = best;
    }
    a_end = kk;
    b_begin = b_end = 0;
  }
  // write the merge of the two runs: entry k of the rows is one contiguous segment
  const unsigned* rowb = G == 16 ? &rows[wq][0][lane ^ 16] : myrow;
  const int m = writer ? min(total, K) : 0;
  const int mmax = __reduce_max_sync(full, (unsigned)m);
  int ia = 0, ib = b_begin;
  unsigned va = ia < a_end ? myrow[ia * 32] : 0xffffffffu;
  unsigned vb = ib < b_end ? rowb[ib * 32] : 0xffffffffu;
  for (int k = 0; k < mmax; ++k) {
    const bool take_a = va < vb;
    const unsigned v = take_a ? va : vb;
    if (k < m) P.nbr[(size_t)k * P.n + p] = P.pos_of[v];
    if (take_a) {
      ++ia;
      va = ia < a_end ? myrow[ia * 32] : 0xffffffffu;
    } else {
      ++ib;
      vb = ib < b_end ? rowb[ib * 32] : 0xffffffffu;
    }
  }
  if (writer) {
    P.cnt[p] = m;
    if (total > K) atomicAdd(&P.overflow[w], 1);
  }
}

// --------------------------------------------------------------------------------------- particle-wall slot
// particle_walls.py:65-119 + boundary.py:241-287: colour c = sum V_j W over the world's wall particles (ascending
// wall id), its gradient and mean velocity; the distance phi with Psi(phi) = c; the slot filled as a flat wall at phi
// with the fitted amplitude, offset and C1 taper. Without box walls this is the particle's one slot; with them
// k_shape_slots merges it with the boxes' (slot_cap 4).

// (Psi, dPsi) of a wall at distance phi: A Psi(phi + delta) with the C1 taper between the first and second lattice
// layer (boundary.py:241-251)
__device__ __forceinline__ void wall_volume(const DevP& P, float phi, float& psi, float& dpsi) {
  halfspace(P.kc, phi + P.wall_offset, psi, dpsi);
  psi = psi * P.wall_amp;
  dpsi = dpsi * P.wall_amp;
  if (phi > P.taper0) {
    float L = P.taper1 - P.taper0;
    float t = minr((phi - P.taper0) / L, 1.0f);
    float sm = 1.0f - (t * t) * (3.0f - 2.0f * t);
    float dsm = ((6.0f * t) * (t - 1.0f)) / L;
    float p0 = psi;
    psi = p0 * sm;
    dpsi = ADF_FMA(p0, dsm, dpsi * sm);
  }
}

__device__ __forceinline__ void wall_slot_fill(const DevP& P, int p, float4 xi, float c, float gx, float gy, float gz,
                                               float mx, float my, float mz, float phi);

// colour_distance (particle_walls.py:87-98, 30 bisection steps) by a team of WT lanes, two steps per round: with
// mid m1 of [lo, hi], lanes 0, 1 and 2 evaluate Psi at m0 = mid(lo, m1), m1 and m2 = mid(m1, hi), the two possible
// midpoints of the second step, so the 15 rounds choose exactly the intervals of the 30 serial steps.
__device__ __forceinline__ float colour_distance_team(const KC& k, float c, int t, int t0, unsigned mask) {
  float lo = -k.h, hi = k.h;
#pragma unroll 1
  for (int r = 0; r < 15; ++r) {
    const float m1 = __fmul_rn(0.5f, __fadd_rn(lo, hi));
    const float m0 = __fmul_rn(0.5f, __fadd_rn(lo, m1)), m2 = __fmul_rn(0.5f, __fadd_rn(m1, hi));
    float psi, dpsi;
    halfspace(k, t == 0 ? m0 : (t == 2 ? m2 : m1), psi, dpsi);
    const int gt = psi > c ? 1 : 0;
    const int g0 = __shfl_sync(mask, gt, t0), g1 = __shfl_sync(mask, gt, t0 + 1), g2 = __shfl_sync(mask, gt, t0 + 2);
    if (g1) {
      lo = m1;
      if (g2) lo = m2;
      else hi = m2;
    } else {
      hi = m1;
      if (g0) lo = m0;
      else hi = m0;
    }
  }
  return __fmul_rn(0.5f, __fadd_rn(lo, hi));
}

// One listed liquid particle's wall slot, by one lane (a cell of its 27 holds boundary particles).
__device__ __forceinline__ void wall_slot_one(const DevP& P, int p) {
  const int w = P.world_s[p];
  const WorldGrid g = P.grid[w];
  const float4 xi = P.pos[p];
  int cx, cy, cz;
  cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
  unsigned buf[MAXWALL];  // original ids of the wall particles within h, kept ascending
  int m = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    int z = cz + dz;
    if (z < 0 || z >= g.nz) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      int y = cy + dy;
      if (y < 0 || y >= g.ny) continue;
      for_row_ranges(P.cell_start, g, P.total_cells, y, z, max(cx - 1, 0), min(cx + 1, g.nx - 1), [&](int b, int e) {
        for (int j = b; j < e; ++j) {
          float4 xj = P.pos[j];
          float dx = xi.x - xj.x, dy2 = xi.y - xj.y, dz2 = xi.z - xj.z;
          float W, F;
          wf(P.kc, dot_plain(dx, dy2, dz2, dx, dy2, dz2), W, F);
          float wj = xj.w * W;
          if (wj > 0.0f) {
            if (m >= MAXWALL) {
              atomicAdd(&P.wall_overflow[w], 1);
              continue;
            }
            const unsigned key = (unsigned)P.id_of[j];
            int at = m;
            while (at > 0 && buf[at - 1] > key) {
              buf[at] = buf[at - 1];
              --at;
            }
            buf[at] = key;
            ++m;
          }
        }
      });
    }
  }
  if (m == 0) return;
  float c = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
  for (int k = 0; k < m; ++k) {
    const int j = P.pos_of[buf[k]];
    float4 xj = P.pos[j];
    float4 vj = P.vel[j];
    float dx = xi.x - xj.x, dy2 = xi.y - xj.y, dz2 = xi.z - xj.z;
    float W, F;
    wf(P.kc, dot_plain(dx, dy2, dz2, dx, dy2, dz2), W, F);
    float vol = xj.w;
    float wj = vol * W;
    c = c + wj;
    gx = ADF_FMA(vol, dx * F, gx);
    gy = ADF_FMA(vol, dy2 * F, gy);
    gz = ADF_FMA(vol, dz2 * F, gz);
    mx = ADF_FMA(wj, vj.x, mx);
    my = ADF_FMA(wj, vj.y, my);
    mz = ADF_FMA(wj, vj.z, mz);
  }
  wall_slot_fill(P, p, xi, c, gx, gy, gz, mx, my, mz, colour_distance(P.kc, minr(c, 1.0f)));
}

// The slot of liquid particle p from its colour sums over the wall particles within h (ascending wall id) and the
// colour distance phi of c (colour_distance): mean wall velocity, amplitude, taper, and the four slot records.
__device__ __forceinline__ void wall_slot_fill(const DevP& P, int p, float4 xi, float c, float gx, float gy, float gz,
                                               float mx, float my, float mz, float phi) {
  mx = mx / c;
  my = my / c;
  mz = mz / c;
  float lg = __fsqrt_rn(dot_plain(gx, gy, gz, gx, gy, gz));
  if (c < (float)(1.0e-4) || lg <= 0.0f) return;
  if (!(phi < P.reach && phi + P.wall_offset < P.kc.h)) return;
  float nx = -gx / lg, ny = -gy / lg, nz = -gz / lg;
  float psi, dpsi;
  wall_volume(P, phi, psi, dpsi);
  P.slot_g[p] = make_float4(dpsi * nx, dpsi * ny, dpsi * nz, psi);
  P.slot_vb[p] = make_float4(mx, my, mz, phi);
  P.slot_n[p] = make_float4(nx, ny, nz, __int_as_float(P.n_shapes));
  P.slot_xb[p] = make_float4(ADF_FMA(-phi, nx, xi.x), ADF_FMA(-phi, ny, xi.y), ADF_FMA(-phi, nz, xi.z), 0.0f);
}


// Every liquid particle's slot starts empty; those whose 27 cells hold boundary particles (tiles checked first, then
// the cells) are compacted within the block, in order (warp ballots, then the warps' counts scanned), and handed to
// teams of the block's lanes: most liquid particles see no wall particle, and the near-wall ones of a block are
// usually a minority of it.
__global__ void __launch_bounds__(BLOCK) k_wall_slots(DevP P) {
  __shared__ int list[BLOCK];
  __shared__ int wcount[BLOCK / 32];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = P.nfw[0];
  bool near = false;
  if (p < nf) {
    P.slot_g[p] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    if (P.nfw[1] > 0) {
      const WorldGrid g = P.grid[P.world_s[p]];
      const float4 xi = P.pos[p];
      int cx, cy, cz;
      cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
      // the 27 cells lie in at most 2 tiles per axis
      const int x0 = max(cx - 1, 0) >> 2, x1 = min(cx + 1, g.nx - 1) >> 2;
      const int y0 = max(cy - 1, 0) >> 2, y1 = min(cy + 1, g.ny - 1) >> 2;
      const int z0 = max(cz - 1, 0) >> 2, z1 = min(cz + 1, g.nz - 1) >> 2;
      int walls = 0;
      for (int tz = z0; tz <= z1; ++tz)
        for (int ty = y0; ty <= y1; ++ty)
          for (int tx = x0; tx <= x1; ++tx) {
            const int t0 = P.total_cells + g.base + (((tz * g.tny + ty) * g.tnx + tx) << 6);
            walls |= P.cell_start[t0 + 64] - P.cell_start[t0];
          }
      if (walls != 0) {  // then the 27 cells themselves (their 9 rows, one range per tile crossed)
        walls = 0;
        for (int r = 0; r < 9 && walls == 0; ++r) {
          const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
          if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) continue;
          for_row_ranges(P.cell_start, g, P.total_cells, y, z, max(cx - 1, 0), min(cx + 1, g.nx - 1),
                         [&](int b, int e) { walls |= e - b; });
        }
      }
      near = walls != 0;
    }
  }
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, near);
  if (lane == 0) wcount[wq] = __popc(m);
  __syncthreads();
  int base = 0, total = 0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
    if (k < wq) base += wcount[k];
    total += wcount[k];
  }
  if (near) list[base + __popc(m & ((1u << lane) - 1u))] = p;
  __syncthreads();
  // WT lanes per listed particle (a team; BLOCK / WT particles per round): the team's lanes take the 9 cell rows in
  // turn, append the wall particles within h (vol W > 0) to the team's buffer, rank them by original id, then compute
  // the terms of the colour sums WT at a time while the team's first lane adds them in ascending id order, exactly as
  // one lane does. A particle with more than WT_CAP such wall particles is done by its first lane alone.
  __shared__ unsigned t_id[BLOCK / WT][WT_CAP];
  __shared__ int t_j[BLOCK / WT][WT_CAP];
  __shared__ int t_sorted[BLOCK / WT][WT_CAP];
  __shared__ int t_cnt[BLOCK / WT];
  const int tm = threadIdx.x / WT, t = threadIdx.x % WT;
  const int t0 = lane - t;  // the team's first lane
  for (int r0 = 0; r0 < total; r0 += BLOCK / WT) {
    const int k = r0 + tm;
    const bool act = k < total;
    const int q = act ? list[k] : 0;
    if (t == 0) t_cnt[tm] = 0;
    __syncwarp();
    float4 xi = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (act) {
      const WorldGrid g = P.grid[P.world_s[q]];
      xi = P.pos[q];
      int cx, cy, cz;
      cell_coords(g, xi.x, xi.y, xi.z, cx, cy, cz);
      for (int r = t; r < 9; r += WT) {
        const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
        if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) continue;
        for_row_ranges(P.cell_start, g, P.total_cells, y, z, max(cx - 1, 0), min(cx + 1, g.nx - 1),
                       [&](int b, int e) {
                         for (int j = b; j < e; ++j) {
                           const float4 xj = P.pos[j];
                           const float dx = xi.x - xj.x, dy2 = xi.y - xj.y, dz2 = xi.z - xj.z;
                           float W, F;
                           wf(P.kc, dot_plain(dx, dy2, dz2, dx, dy2, dz2), W, F);
                           if (xj.w * W > 0.0f) {
                             const int slot = atomicAdd(&t_cnt[tm], 1);
                             if (slot < WT_CAP) {
                               t_id[tm][slot] = (unsigned)P.id_of[j];
                               t_j[tm][slot] = j;
                             }
                           }
                         }
                       });
      }
    }
    __syncwarp();
    const int mt = act ? t_cnt[tm] : 0;
    const bool team = mt <= WT_CAP;  // else the one-lane path below
    if (team) {
      for (int h = t; h < mt; h += WT) {  // rank by original id (ids are distinct)
        const unsigned id = t_id[tm][h];
        int rank = 0;
        for (int u = 0; u < mt; ++u) rank += t_id[tm][u] < id ? 1 : 0;
        t_sorted[tm][rank] = t_j[tm][h];
      }
    }
    __syncwarp();
    const int mrun = __reduce_max_sync(0xffffffffu, team ? (unsigned)mt : 0u);
    float c = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
    for (int k0 = 0; k0 < mrun; k0 += WT) {
      // lane t: the terms of entry k0 + t (the same expressions as the one-lane sum)
      float wj = 0.0f, vol = 0.0f, ax = 0.0f, ay = 0.0f, az = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
      if (team && k0 + t < mt) {
        const int j = t_sorted[tm][k0 + t];
        const float4 xj = P.pos[j];
        const float4 vj = P.vel[j];
        const float dx = xi.x - xj.x, dy2 = xi.y - xj.y, dz2 = xi.z - xj.z;
        float W, F;
        wf(P.kc, dot_plain(dx, dy2, dz2, dx, dy2, dz2), W, F);
        vol = xj.w;
        wj = vol * W;
        ax = dx * F;
        ay = dy2 * F;
        az = dz2 * F;
        vx = vj.x;
        vy = vj.y;
        vz = vj.z;
      }
#pragma unroll
      for (int u = 0; u < WT; ++u) {  // the first lane adds entries k0, k0 + 1, ... in order
        const int src = t0 + u;
        const float swj = __shfl_sync(0xffffffffu, wj, src), svol = __shfl_sync(0xffffffffu, vol, src);
        const float sax = __shfl_sync(0xffffffffu, ax, src), say = __shfl_sync(0xffffffffu, ay, src);
        const float saz = __shfl_sync(0xffffffffu, az, src), svx = __shfl_sync(0xffffffffu, vx, src);
        const float svy = __shfl_sync(0xffffffffu, vy, src), svz = __shfl_sync(0xffffffffu, vz, src);
        if (team && t == 0 && k0 + u < mt) {
          c = c + swj;
          gx = ADF_FMA(svol, sax, gx);
          gy = ADF_FMA(svol, say, gy);
          gz = ADF_FMA(svol, saz, gz);
          mx = ADF_FMA(swj, svx, mx);
          my = ADF_FMA(swj, svy, my);
          mz = ADF_FMA(swj, svz, mz);
        }
      }
    }
    if (act && team && mt > 0) {  // the whole team bisects the colour distance of its first lane's sums
      static_assert(WT >= 3, "the team bisection evaluates three points per round");
      const unsigned tmask = ((1u << WT) - 1u) << t0;
      const float phi = colour_distance_team(P.kc, minr(__shfl_sync(tmask, c, t0), 1.0f), t, t0, tmask);
      if (t == 0) wall_slot_fill(P, q, xi, c, gx, gy, gz, mx, my, mz, phi);
    } else if (act && t == 0 && !team) {
      wall_slot_one(P, q);
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------------- box-shape walls
constexpr float COS_SAME = 0.85f;  // boundary_slots.py:9: walls whose normals agree this much face the same way

// newton geometry/kernels.py:310-370 (sdf_box, sdf_box_grad): signed distance of the axis-aligned box of half extents
// h.xyz at box-frame point (x, y, z), and its outward unit gradient.
__device__ __forceinline__ float box_sdf(float x, float y, float z, const float4& h) {
  const float qx = fabsf(x) - h.x, qy = fabsf(y) - h.y, qz = fabsf(z) - h.z;
  const float ex = maxr(qx, 0.0f), ey = maxr(qy, 0.0f), ez = maxr(qz, 0.0f);
  return __fsqrt_rn(dot_plain(ex, ey, ez, ex, ey, ez)) + minr(maxr(qx, maxr(qy, qz)), 0.0f);
}

__device__ __forceinline__ void normalized3(float& x, float& y, float& z) {
  const float l = __fsqrt_rn(dot_plain(x, y, z, x, y, z));
  if (l > 0.0f) {
    x = x / l;
    y = y / l;
    z = z / l;
  } else {
    x = y = z = 0.0f;
  }
}

__device__ __forceinline__ void box_grad(float x, float y, float z, const float4& h, float& gx, float& gy, float& gz) {
  const float qx = fabsf(x) - h.x, qy = fabsf(y) - h.y, qz = fabsf(z) - h.z;
  if (qx > 0.0f || qy > 0.0f || qz > 0.0f) {  // outside: towards the closest point
    gx = x - minr(maxr(x, -h.x), h.x);
    gy = y - minr(maxr(y, -h.y), h.y);
    gz = z - minr(maxr(z, -h.z), h.z);
    normalized3(gx, gy, gz);
    return;
  }
  const float sx = x < 0.0f ? -1.0f : 1.0f, sy = y < 0.0f ? -1.0f : 1.0f, sz = z < 0.0f ? -1.0f : 1.0f;
  gx = gy = gz = 0.0f;
  if ((qx > qy && qx > qz) || (qy == 0.0f && qz == 0.0f)) gx = sx;
  else if ((qy > qx && qy > qz) || (qx == 0.0f && qz == 0.0f)) gy = sy;
  else gz = sz;
}

// The box's outward unit normal at box-frame point (x, y, z): its SDF gradient, normalised again as the reference's
// slot code does (boundary.py:226-231).
__device__ __forceinline__ void box_normal(float x, float y, float z, const float4& h, float& nx, float& ny, float& nz) {
  box_grad(x, y, z, h, nx, ny, nz);
  normalized3(nx, ny, nz);
}

// newton GeoType ids of the static shapes this path evaluates (geometry/types.py:73-118)
constexpr int GEO_PLANE = 1, GEO_SPHERE = 3, GEO_CAPSULE = 4, GEO_CYLINDER = 6, GEO_BOX = 7;

// A shape's frame: its quaternion q (x, y, z, w); the identity leaves points and directions as they are (the frames of
// unrotated shapes are their translations only, and their arithmetic is exactly the translation's).
__device__ __forceinline__ bool rotated(const float4& q) {
  return !(q.x == 0.0f && q.y == 0.0f && q.z == 0.0f && q.w == 1.0f);
}
__device__ __forceinline__ void to_frame(const float4& q, float& x, float& y, float& z) {  // world direction -> shape
  if (!rotated(q)) return;
  const float c[4] = {-q.x, -q.y, -q.z, q.w};
  float ox, oy, oz;
  quat_rotate(c, x, y, z, ox, oy, oz);
  x = ox;
  y = oy;
  z = oz;
}
__device__ __forceinline__ void from_frame(const float4& q, float& x, float& y, float& z) {  // shape direction -> world
  if (!rotated(q)) return;
  const float c[4] = {q.x, q.y, q.z, q.w};
  float ox, oy, oz;
  quat_rotate(c, x, y, z, ox, oy, oz);
  x = ox;
  y = oy;
  z = oz;
}

// newton geometry/kernels.py:515-546 (sdf_cylinder, straight sides, along z): the radial and axial excesses
__device__ __forceinline__ void cylinder_parts(const float4& s, float x, float y, float z, float& rho, float& dx,
                                               float& dy) {
  rho = __fsqrt_rn(dot_plain(x, y, 0.0f, x, y, 0.0f));
  dx = rho - s.x;
  dy = fabsf(z) - s.y;
}

// The signed distance of shape `geo` (scale s.xyz) at shape-frame point (x, y, z), as newton's eval_shape_sdf evaluates
// the analytic shapes (soft_contacts_sdf.py:249-280, geometry/kernels.py): a box (sdf_box :310-333), a sphere
// (sdf_sphere :277-288), a capsule along the shape's z axis (sdf_capsule :374-393), a plane through the shape's origin
// with normal +z (soft_contacts_sdf.py:73-102 _eval_plane_sdf with depth 0: infinite unless width s.x and length
// s.y are both positive; a finite plane is a two-sided sheet, z over its footprint from above, else the distance to
// its nearest point).
__device__ __forceinline__ bool plane_over(const float4& s, float x, float y, float z) {
  const float hw = 0.5f * s.x, hl = 0.5f * s.y;
  return !(hw > 0.0f && hl > 0.0f) || (fabsf(x) <= hw && fabsf(y) <= hl && z >= 0.0f);
}

__device__ __forceinline__ void plane_delta(const float4& s, float x, float y, float z, float& dx, float& dy, float& dz) {
  const float hw = 0.5f * s.x, hl = 0.5f * s.y;
  dx = x - minr(maxr(x, -hw), hw);
  dy = y - minr(maxr(y, -hl), hl);
  dz = z - 0.0f;
}

__device__ __forceinline__ float shape_phi(int geo, const float4& s, float x, float y, float z) {
  if (geo == GEO_BOX) return box_sdf(x, y, z, s);
  if (geo == GEO_CYLINDER) {
    float rho, dx, dy;
    cylinder_parts(s, x, y, z, rho, dx, dy);
    const float ex = maxr(dx, 0.0f), ey = maxr(dy, 0.0f);
    return minr(maxr(dx, dy), 0.0f) + __fsqrt_rn(ex * ex + ey * ey);
  }
  if (geo == GEO_PLANE) {
    if (plane_over(s, x, y, z)) return z;
    float dx, dy, dz;
    plane_delta(s, x, y, z, dx, dy, dz);
    return __fsqrt_rn(dot_plain(dx, dy, dz, dx, dy, dz));
  }
  float cz = z;
  if (geo == GEO_CAPSULE) cz = z > s.y ? z - s.y : (z < -s.y ? z + s.y : 0.0f);
  return __fsqrt_rn(dot_plain(x, y, cz, x, y, cz)) - s.x;
}

// Its outward unit normal there: the gradient (box: sdf_box_grad; sphere and capsule: the direction from the nearest
// point of the centre or axis segment, +z at it, -z below the lower cap; plane: +z), normalised again as the
// reference's slot code does (boundary.py:226-231).
__device__ __forceinline__ void shape_normal(int geo, const float4& s, float x, float y, float z, float& nx, float& ny,
                                             float& nz) {
  if (geo == GEO_BOX) {
    box_normal(x, y, z, s, nx, ny, nz);
    return;
  }
  if (geo == GEO_CYLINDER) {  // newton geometry/kernels.py:549-600 (sdf_cylinder_grad, straight sides)
    float rho, dx, dy;
    cylinder_parts(s, x, y, z, rho, dx, dy);
    float rx = 0.0f, ry = 0.0f, rz = 1.0f;
    if (rho > 1.0e-8f) {
      rx = x / rho;
      ry = y / rho;
      rz = 0.0f;
    }
    const float az = z < 0.0f ? -1.0f : 1.0f;
    if (dx > 0.0f && dy > 0.0f) {
      const float gx = rx * dx, gy = ry * dx, gz = ADF_FMA(az, dy, rz * dx);
      const float gl = __fsqrt_rn(dot_plain(gx, gy, gz, gx, gy, gz));
      if (gl > 1.0e-8f) {
        nx = gx / gl;
        ny = gy / gl;
        nz = gz / gl;
      } else {
        nx = rx;
        ny = ry;
        nz = rz;
      }
    } else if (dx > dy) {
      nx = rx;
      ny = ry;
      nz = rz;
    } else {
      nx = 0.0f;
      ny = 0.0f;
      nz = az;
    }
    normalized3(nx, ny, nz);
    return;
  }
  if (geo == GEO_PLANE) {
    nx = 0.0f;
    ny = 0.0f;
    nz = 1.0f;
    if (!plane_over(s, x, y, z)) {
      float dx, dy, dz;
      plane_delta(s, x, y, z, dx, dy, dz);
      const float d = __fsqrt_rn(dot_plain(dx, dy, dz, dx, dy, dz));
      if (d > 0.0f) {
        nx = dx / d;
        ny = dy / d;
        nz = dz / d;
      }
    }
    normalized3(nx, ny, nz);
    return;
  }
  float cz = z, dz = 1.0f;
  if (geo == GEO_CAPSULE) {
    if (z > s.y) cz = z - s.y;
    else if (z < -s.y) {
      cz = z + s.y;
      dz = -1.0f;
    } else {
      cz = 0.0f;
    }
  }
  const float l = __fsqrt_rn(dot_plain(x, y, cz, x, y, cz));
  if (l > 1.0e-8f) {
    nx = x / l;
    ny = y / l;
    nz = cz / l;
  } else {
    nx = 0.0f;
    ny = 0.0f;
    nz = dz;
  }
  normalized3(nx, ny, nz);
}

// boundary_slots.py:13-37: (sh, phi) into a phi-ascending row of n_ slots; the slot used, or -1
__device__ __forceinline__ int slot_insert(int (&shp)[4], float (&ph)[4], int n_, int sh, float phi) {
  int pos = n_, k = n_ - 1;
  while (k >= 0) {
    if (ph[k] <= phi) break;
    pos = k;
    --k;
  }
  if (pos >= 4) return -1;
  for (k = n_ >= 4 ? 3 : n_; k > pos; --k) {
    shp[k] = shp[k - 1];
    ph[k] = ph[k - 1];
  }
  shp[pos] = sh;
  ph[pos] = phi;
  return pos;
}

// boundary_slots.py:59-102: a wall (sh, phi, normal nrm) into the row; a full row drops the farthest same-facing
// duplicate (cos > COS_SAME) among its four walls and the new one, never one nearer than `near`, and when there is
// none the farthest of the five. nr holds the slots' normals. 1 if the wall was kept.
__device__ __forceinline__ int shape_insert(int (&shp)[4], float (&ph)[4], float3 (&nr)[4], int n_, int sh, float phi,
                                            float3 nrm, float near) {
  if (n_ < 4) {
    const int r = slot_insert(shp, ph, n_, sh, phi);
    if (r < 0) return 0;
    for (int k = n_; k > r; --k) nr[k] = nr[k - 1];
    nr[r] = nrm;
    return 1;
  }
  auto dot3 = [](const float3& a, const float3& b) { return dot_plain(a.x, a.y, a.z, b.x, b.y, b.z); };
  int ev = -1;
  float ev_phi = -1.0f;
  for (int m = 0; m < 4; ++m)
    if (phi >= near && ph[m] <= phi && dot3(nr[m], nrm) > COS_SAME) {
      ev = 4;
      ev_phi = phi;
    }
  for (int k = 0; k < 4; ++k) {
    const float pk = ph[k];
    int dup = 0;
    for (int m = 0; m < 4; ++m)
      if (m != k && ph[m] <= pk && dot3(nr[m], nr[k]) > COS_SAME) dup = 1;
    if (phi <= pk && dot3(nrm, nr[k]) > COS_SAME) dup = 1;
    if (dup == 1 && pk >= near && pk > ev_phi) {
      ev = k;
      ev_phi = pk;
    }
  }
  if (ev < 0 && phi < ph[3]) ev = 3;
  if (ev < 0 || ev == 4) return 0;
  for (int k = ev; k < 3; ++k) {
    shp[k] = shp[k + 1];
    ph[k] = ph[k + 1];
    nr[k] = nr[k + 1];
  }
  int pos = 3;
  while (pos > 0 && ph[pos - 1] > phi) {
    shp[pos] = shp[pos - 1];
    ph[pos] = ph[pos - 1];
    nr[pos] = nr[pos - 1];
    --pos;
  }
  shp[pos] = sh;
  ph[pos] = phi;
  nr[pos] = nrm;
  return 1;
}

// boundary.py:190-238 (find), 254-334 (fill) and 336-396 (combine), after k_wall_slots, when the model has shape
// walls: every liquid particle's slots from its world's shapes within reach (in the world's shape order, each
// evaluated in its own frame) and the particle wall's slot k_wall_slots left in slot 0, nearest first; each shape's
// slot filled from its SDF (the start-of-step closest point and normal kept, world-oriented, for the projection),
// then overlapping walls combined by inclusion-exclusion (Psi as filled, gradients as rewritten slot by slot). Empty
// slots are zero with wall id -1.
__global__ void __launch_bounds__(BLOCK) k_shape_slots(DevP P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  const float4 xi = P.pos[p];
  const int S = P.n_shapes;
  const float h = P.kc.h, near = 0.1f * h;
  const float4 g0 = P.slot_g[p], vb0 = P.slot_vb[p], n0 = P.slot_n[p], xb0 = P.slot_xb[p];
  int shp[4] = {-1, -1, -1, -1};
  float ph[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  float3 nr[4];
  int ns = 0;
  for (int c = P.sh_start[w]; c < P.sh_start[w + 1]; ++c) {
    const int sh = P.sh_ids[c];
    const float4 cp = P.sh_pos[sh];
    const int geo = P.sh_geo[sh];
    float lx = xi.x - cp.x, ly = xi.y - cp.y, lz = xi.z - cp.z;
    if (geo != GEO_PLANE && __fsqrt_rn(dot_plain(lx, ly, lz, lx, ly, lz)) > cp.w + h) continue;
    const float4 hx = P.sh_half[sh], q = P.sh_quat[sh];
    to_frame(q, lx, ly, lz);
    const float phi = shape_phi(geo, hx, lx, ly, lz);
    if (phi < P.reach && phi + P.wall_offset < h) {
      float nx, ny, nz;
      shape_normal(geo, hx, lx, ly, lz, nx, ny, nz);
      from_frame(q, nx, ny, nz);
      if (shape_insert(shp, ph, nr, ns, sh, phi, make_float3(nx, ny, nz), near) > 0 && ns < 4) ++ns;
    }
  }
  if (g0.w >= 0.0f && slot_insert(shp, ph, ns, S, vb0.w) >= 0 && ns < 4) ++ns;
  float4 sg[4], sv[4], sn[4], sx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    sg[k] = sv[k] = sx[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    sn[k] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
    if (k >= ns) continue;
    const int sh = shp[k];
    if (sh == S) {
      sg[k] = g0;
      sv[k] = vb0;
      sn[k] = n0;
      sx[k] = xb0;
    } else {
      const float4 cp = P.sh_pos[sh], hx = P.sh_half[sh];
      const int geo = P.sh_geo[sh];
      const float4 q = P.sh_quat[sh];
      float lx = xi.x - cp.x, ly = xi.y - cp.y, lz = xi.z - cp.z;
      to_frame(q, lx, ly, lz);
      const float phi = shape_phi(geo, hx, lx, ly, lz);
      float nx, ny, nz, psi, dpsi;
      shape_normal(geo, hx, lx, ly, lz, nx, ny, nz);
      float bx = ADF_FMA(-phi, nx, lx), by = ADF_FMA(-phi, ny, ly), bz = ADF_FMA(-phi, nz, lz);
      from_frame(q, bx, by, bz);
      from_frame(q, nx, ny, nz);
      wall_volume(P, phi, psi, dpsi);
      sg[k] = make_float4(dpsi * nx, dpsi * ny, dpsi * nz, psi);
      sv[k] = make_float4(0.0f, 0.0f, 0.0f, phi);
      sn[k] = make_float4(nx, ny, nz, __int_as_float(sh));
      sx[k] = make_float4(bx, by, bz, 0.0f);
    }
  }
  if (ns > 1) {
    float ps[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) ps[k] = sg[k].w;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (b >= ns) break;
      const float gbx = sg[b].x, gby = sg[b].y, gbz = sg[b].z;
      float ob = 0.0f, sb = 0.0f;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ns) break;
        if (c == b) continue;
        const float gcx = sg[c].x, gcy = sg[c].y, gcz = sg[c].z;
        const float lb = __fsqrt_rn(dot_plain(gbx, gby, gbz, gbx, gby, gbz));
        const float lc = __fsqrt_rn(dot_plain(gcx, gcy, gcz, gcx, gcy, gcz));
        float cbc = 0.0f;
        if (lb > 0.0f && lc > 0.0f) cbc = minr(maxr(dot_plain(gbx, gby, gbz, gcx, gcy, gcz) / (lb * lc), -1.0f), 1.0f);
        ob = ob + (1.0f - fabsf(cbc)) * ps[c];
        if (cbc > 0.0f && (ps[c] > ps[b] || (ps[c] == ps[b] && c < b))) sb = sb + cbc;
      }
      ob = minr(ob, 1.0f);
      sg[b].w = ps[b] * maxr((1.0f - 0.5f * ob) - sb, 0.0f);
      const float f = maxr((1.0f - ob) - sb, 0.0f);
      sg[b].x = gbx * f;
      sg[b].y = gby * f;
      sg[b].z = gbz * f;
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const size_t o = slot_at(P, k, p);
    P.slot_g[o] = sg[k];
    P.slot_vb[o] = sv[k];
    P.slot_n[o] = sn[k];
    P.slot_xb[o] = sx[k];
  }
  P.slot_cnt[p] = (int8_t)ns;
}

// integrate.py:75-95 (box_span) and 98-126 (path_entry) for a static box of half extents h: the last outside parameter
// of the box-frame path o -> e before it first enters the box, by the exact slab test; 2 when the path stays outside or
// starts inside.
__device__ __forceinline__ float box_entry(const float4& h, float ox, float oy, float oz, float ex, float ey, float ez) {
  if (box_sdf(ox, oy, oz, h) < 0.0f) return 2.0f;
  float lo = -1.0e30f, hi = 1.0e30f;
  const float d[3] = {ex - ox, ey - oy, ez - oz}, o[3] = {ox, oy, oz}, hh[3] = {h.x, h.y, h.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (fabsf(d[a]) > 0.0f) {
      const float ta = (-hh[a] - o[a]) / d[a], tb = (hh[a] - o[a]) / d[a];
      lo = maxr(lo, minr(ta, tb));
      hi = minr(hi, maxr(ta, tb));
    } else if (fabsf(o[a]) > hh[a]) {
      lo = 2.0e30f;
    }
  }
  if (lo <= hi && lo <= 1.0f && hi >= 0.0f) return maxr(lo, 0.0f);
  return 2.0f;
}

// integrate.py:48-58 and 98-115 (path_entry) for a static shape other than a box: the path o -> e (shape frame) sampled
// at `samples` evenly spaced parameters; the first sample inside and the last one before it are bisected 8 times, and
// the last outside parameter is returned; 2 when the path stays outside or starts inside.
constexpr int SWEEP_SAMPLES = 64, SWEEP_BISECT = 8;

__device__ __forceinline__ float shape_entry(int geo, const float4& s, float ox, float oy, float oz, float ex, float ey,
                                             float ez, int samples) {
  if (geo == GEO_BOX) return box_entry(s, ox, oy, oz, ex, ey, ez);
  if (shape_phi(geo, s, ox, oy, oz) < 0.0f) return 2.0f;
  const float dx = ex - ox, dy = ey - oy, dz = ez - oz;
  auto inside = [&](float t) {
    return shape_phi(geo, s, ADF_FMA(t, dx, ox), ADF_FMA(t, dy, oy), ADF_FMA(t, dz, oz)) < 0.0f;
  };
  float t_lo = 0.0f, t_hi = 2.0f;
  for (int k = 1; k <= samples && t_hi > 1.0f; ++k) {
    const float t = (float)k / (float)samples;
    if (inside(t)) t_hi = t;
    else t_lo = t;
  }
  if (t_hi > 1.0f) return 2.0f;
  for (int b = 0; b < SWEEP_BISECT; ++b) {
    const float tm = 0.5f * (t_lo + t_hi);
    if (inside(tm)) t_hi = tm;
    else t_lo = tm;
  }
  return t_lo;
}

// integrate.py:192-205: Coulomb friction of a projection onto box sh (Config.wall_friction), after the inward speed
// -vn went: the tangential velocity relative to the wall (velocity b) loses up to mu (-vn), never reversing.
__device__ __forceinline__ void wall_friction(const DevP& P, float& vx, float& vy, float& vz, float bx, float by,
                                              float bz, float nx, float ny, float nz, float vn, int sh) {
  if (!P.wall_friction) return;
  const float mu = P.sh_half[sh].w;
  if (mu <= 0.0f) return;
  const float ux = vx - bx, uy = vy - by, uz = vz - bz;
  const float un = dotf(ux, uy, uz, nx, ny, nz);
  const float tx = ADF_FMA(-un, nx, ux), ty = ADF_FMA(-un, ny, uy), tz = ADF_FMA(-un, nz, uz);
  const float lt = __fsqrt_rn(dot_plain(tx, ty, tz, tx, ty, tz));
  if (lt <= 0.0f) return;
  const float f = minr(1.0f, (mu * (-vn)) / lt);
  vx = ADF_FMA(-f, tx, vx);
  vy = ADF_FMA(-f, ty, vy);
  vz = ADF_FMA(-f, tz, vz);
}

// Neighbour loops read their rows in batches of NB: the NB row entries first, then the NB gathers they address,
// then the arithmetic in ascending row order, so the loads of a batch overlap instead of forming one dependent
// chain per neighbour. Entries past the row's end address the particle itself (a harmless load) and are skipped.
// NB is a template parameter of every neighbour loop (the gathers a thread keeps in flight); the autotuner picks it
// per kernel among NB_CHOICES, NB_DEFAULT otherwise.
constexpr int NB_DEFAULT = 8;

// Rows are streamed once per kernel (evict-first loads) so that the gathered particle arrays keep L1 and L2.
template <int NB>
__device__ __forceinline__ void load_row_batch(const DevP& P, int p, int c, int k, int (&j)[NB]) {
  const int* row = P.nbr + p;
#pragma unroll
  for (int u = 0; u < NB; ++u) j[u] = (k + u < c) ? __ldcs(row + (size_t)(k + u) * P.n) : p;
}

// Row entries with their gradient factor F(r_ij) (the value wf() gives for the pair, stored by k_density_alpha) in
// one 8-byte load: the later loops read F instead of re-evaluating sqrt, branches and a division; the value is the
// same, so every sum is unchanged.
template <int NB>
__device__ __forceinline__ void load_row_batch_f(const DevP& P, int p, int c, int k, int (&j)[NB], float (&f)[NB]) {
  const int2* row = P.nbrjf + p;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    int2 e = (k + u < c) ? __ldcs(row + (size_t)(k + u) * P.n) : make_int2(p, 0);
    j[u] = e.x;
    f[u] = __int_as_float(e.y);
  }
}

// ------------------------------------------------------------------------------------------ density, factor
// pressure.py:144-193
template <int NBX>
__global__ void __launch_bounds__(BLOCK, 5) k_density_alpha(DevP P) {
  constexpr int NB = NBX & NB_MASK;
  constexpr bool MS = (NBX & MS_FLAG) != 0;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  float4 xi = P.pos[p];
  float mi = xi.w;
  float inv_r0 = 1.0f / P.vel[p].w;
  float bi = mi * inv_r0;
  float rho = mi * P.kc.sigma;
  float Gx = 0.0f, Gy = 0.0f, Gz = 0.0f, sq = 0.0f;
  int c = P.cnt[p];
  for (int k = 0; k < c; k += NB) {
    int j[NB];
    load_row_batch(P, p, c, k, j);
    float4 xb[NB];
#pragma unroll
    for (int u = 0; u < NB; ++u) xb[u] = P.pos[j[u]];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      if (k + u >= c) break;
      float4 xj = xb[u];
      float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
      float r2 = dot_plain(rx, ry, rz, rx, ry, rz);
      float W, F;
      wf(P.kc, r2, W, F);
      __stcs(P.nbrjf + (size_t)(k + u) * P.n + p, make_int2(j[u], __float_as_int(F)));
      __stcs(P.nbrw + (size_t)(k + u) * P.n + p, W);
      float mj = xj.w;
      rho = ADF_FMA(mj, W, rho);
      float a = mj * inv_r0;
      float aF = a * F;
      Gx = ADF_FMA(aF, rx, Gx);
      Gy = ADF_FMA(aF, ry, Gy);
      Gz = ADF_FMA(aF, rz, Gz);
      sq = ADF_FMA(bi * a, (F * F) * r2, sq);
    }
  }
  float psi = 0.0f, lam = 0.0f;  // boundary slots, nearest first; lam: the opposing-wall compliance
  for_slots<MS>(P, p, [&](int b, size_t o) {
    const float4 sg = P.slot_g[o];
    psi = psi + sg.w;
    Gx = Gx + sg.x;
    Gy = Gy + sg.y;
    Gz = Gz + sg.z;
    if constexpr (MS) {
      const int ns = P.slot_cnt[p];
      for (int c = b + 1; c < ns; ++c) {
        const float4 gc = P.slot_g[slot_at(P, c, p)];
        lam = lam + maxr(-2.0f * dot_plain(sg.x, sg.y, sg.z, gc.x, gc.y, gc.z), 0.0f);
      }
    }
  });
  float tot = (dotf(Gx, Gy, Gz, Gx, Gy, Gz) + sq) + lam;
  lam = lam + maxr(P.tot_min - tot, 0.0f);
  tot = maxr(tot, P.tot_min);
  P.reg[p] = lam;
  P.ratio[p] = ADF_FMA(rho, inv_r0, psi);
  P.alpha[p] = (tot > (float)(1.0e-12)) ? 1.0f / tot : 0.0f;
  P.neff[p] = ADF_FMA(psi, P.n_full, (float)c);
}

// --------------------------------------------------------------------------------------------- solve start
// pressure.py:196-261
template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_solve_init(DevP P) {
  constexpr int NB = NBX & NB_MASK;
  constexpr bool MS = (NBX & MS_FLAG) != 0;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  float4 xi = P.pos[p];
  float4 vi = P.vel[p];
  float inv_r0 = 1.0f / vi.w;
  float rate = 0.0f;
  int c = P.cnt[p];
  for (int k = 0; k < c; k += NB) {
    int j[NB];
    float fb[NB];
    load_row_batch_f(P, p, c, k, j, fb);
    float4 xb[NB], vb[NB];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      xb[u] = P.pos[j[u]];
      vb[u] = P.vel[j[u]];
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      if (k + u >= c) break;
      float4 xj = xb[u], vj = vb[u];
      float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
      float aF = (xj.w * inv_r0) * fb[u];
      rate = ADF_FMA(aF, dotf(vi.x - vj.x, vi.y - vj.y, vi.z - vj.z, rx, ry, rz), rate);
    }
  }
  for_slots<MS>(P, p, [&](int, size_t o) {
    const float4 sg = P.slot_g[o], vb = P.slot_vb[o];
    rate = rate + dotf(vi.x - vb.x, vi.y - vb.y, vi.z - vb.z, sg.x, sg.y, sg.z);
  });
  const float dt = P.dt;
  float kap, lb, s;
  if (P.mode == 0) {
    float kdv = 0.0f;
    if (P.two_sided) kdv = maxr((P.warm_den * minr(P.kd_s[p], (float)(2.5e-4))) / (dt * dt), 0.0f);
    lb = -kdv;
    float r = rate;
    if (kdv <= 0.0f) {
      r = maxr(rate, 0.0f);
      lb = 0.0f;
    }
    if (P.neff[p] < P.min_nb) {
      r = 0.0f;
      lb = 0.0f;
    }
    s = r;
    kap = maxr((P.warm * minr(P.kv_s[p], 0.5f)) / dt, lb);
  } else {
    float ratio = P.ratio[p];
    float rs = ADF_FMA(dt, rate, ratio);
    if (ratio - 1.0f > P.relief) rs = ADF_FMA(dt, rate, 1.0f + P.relief);
    s = rs;
    lb = 0.0f;
    kap = (P.warm * minr(P.kd_s[p], (float)(2.5e-4))) / (dt * dt);
  }
  P.src[p] = s;
  P.lower[p] = lb;
  P.kappa[p] = kap;
  P.kr[p] = kap / vi.w;
  if (P.feat_on && (!P.warm_need || P.warm_need[P.world_s[p]])) {  // warm-start network features (order: warmstart.py)
    const float ratio = P.ratio[p], al = P.alpha[p], kvp = P.kv_s[p], kdp = P.kd_s[p];
    const float drate = dt * rate;
    const bool on = slot_count(P, p) > 0;  // the nearest wall's slot
    const float4 sg = P.slot_g[p];
    const float phi = on ? P.slot_vb[p].w : P.kc.h;
    const float4 f0 = make_float4(ratio - 1.0f, P.neff[p] / P.n_full, drate, kvp);
    const float4 f1 = make_float4(kdp, al, __fsqrt_rn(dotf(vi.x, vi.y, vi.z, vi.x, vi.y, vi.z)), phi);
    const float4 f2 = make_float4(on ? sg.w : 0.0f, (ratio + drate) - 1.0f, P.warm_div * minr(kvp, 0.5f),
                                  P.warm_den * minr(kdp, (float)(2.5e-4)));
    const float4 f3 = make_float4(vi.z, on ? __fsqrt_rn(dotf(sg.x, sg.y, sg.z, sg.x, sg.y, sg.z)) : 0.0f,
                                  (ratio - 1.0f) * al, drate * al);
    float4* fr = reinterpret_cast<float4*>(P.feat + (size_t)p * 16);
    fr[0] = f0;
    fr[1] = f1;
    fr[2] = f2;
    fr[3] = f3;
  }
}

// The learned start of this solve: the plain start (the previous warm start scaled, in dt-free units) plus the
// network's correction, capped like the stored warm start and kept above the solve's lower bound (a non-finite
// correction ends at the cap). kv_s / kd_s still hold the previous step's values when each solve starts.
__global__ void __launch_bounds__(BLOCK) k_learned_start(DevP P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const float dt = P.dt;
  float kap;
  if (P.mode == 0) {
    const float base = P.warm_div * minr(P.kv_s[p], 0.5f);
    kap = maxr(minr(base + P.pred_kv[p], 0.5f) / dt, P.lower[p]);
  } else {
    const float base = P.warm_den * minr(P.kd_s[p], (float)(2.5e-4));
    kap = maxr(minr(base + P.pred_kd[p], (float)(2.5e-4)) / (dt * dt), P.lower[p]);
  }
  P.kappa2[p] = kap;
  P.kr2[p] = kap / P.vel[p].w;
}

// Without the first-sweep judge every world with liquid takes the learned start.
__global__ void k_mark_learned(DevP P) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  P.learned[P.mode * P.W + w] = P.n_active[w] > 0.0 ? 1 : 0;
}

// The learned start's evaluation schedule under the judge, per world and solve kind: a world whose last evaluated
// learned start lost to the plain start waits gap - 1 solves of this kind before the next evaluation, the gap doubling
// up to PROBE_GAP_MAX; a kept start is evaluated again at the next solve. A world that is not evaluated continues from
// the plain start exactly as when the judge rejects the learned one, so the schedule changes which solves pay for the
// second first sweep, and nothing else. It follows each world's own history only (batch-invariant).
constexpr int PROBE_GAP_MAX = 16;

__global__ void k_probe_plan(DevP P) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  const int o = P.mode * P.W + w;
  const int wait = P.probe_wait[o];
  P.probe_skip[w] = (wait > 0 || !(P.n_active[w] > 0.0)) ? 1 : 0;
  if (wait > 0) P.probe_wait[o] = wait - 1;
}

// After the first sweep from both starts: an evaluated world keeps the learned start unless its residual sum exceeds
// the plain start's (equal liquid counts, so the sums order the mean errors); its schedule is updated.
__global__ void k_choose_start(DevP P) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  const bool probed = P.probe_skip[w] == 0;
  const int use = (probed && P.n_active[w] > 0.0 && !(P.sum_l[w] > P.sum_c[w])) ? 1 : 0;
  P.use_l[w] = use;
  P.learned[P.mode * P.W + w] = use;
  if (probed) {
    const int o = P.mode * P.W + w;
    const int gap = use ? 1 : min(2 * max(P.probe_gap[o], 1), PROBE_GAP_MAX);
    P.probe_gap[o] = gap;
    P.probe_wait[o] = gap - 1;
  }
}

// Worlds that evaluate the learned start in either solve of this step (their schedules wait 0 solves): only their
// particles need features and predictions.
__global__ void k_warm_need(DevP P, int* need) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  need[w] = (P.n_active[w] > 0.0 && (P.probe_wait[w] == 0 || P.probe_wait[P.W + w] == 0)) ? 1 : 0;
}

// The masked worlds' schedules back to "evaluate at the next solve".
__global__ void k_probe_reset(int W, const uint8_t* __restrict__ mask, int* gap, int* wait) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W || !mask[w]) return;
  gap[w] = gap[W + w] = 1;
  wait[w] = wait[W + w] = 0;
}

__global__ void __launch_bounds__(BLOCK) k_select_start(DevP P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  if (!P.use_l[P.world_s[p]]) return;
  P.kappa[p] = P.kappa2[p];
  P.kr[p] = P.kr2[p];
  const int i = P.id_of[p];
  P.err_orig[i] = P.err2[i];
}

// Condition of a solve's WHILE graph node: iterate while any world is unconverged (solve_driver.py:186). runs[0]
// counts the iterations run by WHILE bodies (launch accounting), runs[1] those of the running loop: the call before
// the loop (cap < 0) resets it, and a loop stops after `cap` iterations whatever the unconverged count says (every
// world stops at max_iterations before that, so the cap only guards the loop against a count that never drops).
__global__ void k_set_cond(cudaGraphConditionalHandle h, const int* n_unconv, unsigned long long* runs, int cap) {
  bool more = *n_unconv > 0;
  if (cap < 0) {
    runs[1] = 0ull;
  } else {
    runs[0] += 1ull;
    runs[1] += 1ull;
    more = more && runs[1] < (unsigned long long)cap;
  }
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void k_begin_solve(DevP P) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  P.iters[w] = 0;
  P.err_mean[w] = 0.0f;
  if (P.n_active[w] > 0.0) {
    P.converged[w] = 0;
    atomicAdd(P.n_unconv, 1);
  } else {
    P.converged[w] = 1;
    P.emax[w] = 0.0f;  // no liquid: nothing is iterated or reduced for this world in this solve
  }
}

// Work items of the pressure iterations: 256-particle segments of the sorted liquid range of every world that is still
// iterating. One block lists the worlds (ascending) with the running count of their segments; an iteration kernel's
// block t finds its world by binary search. Converged worlds therefore cost the iteration kernels nothing, which is
// what keeps a batch of uneven worlds cheap once most of them have converged.
constexpr int ITEM = 256;

// The block that builds the list: any multiple of 32 threads. `fresh`: the converged flags were written by other
// blocks of the same launch, so they are read from L2.
__device__ __forceinline__ int build_worklist(const DevP& P, bool fresh) {
  __shared__ int smem[32];
  __shared__ int carry_w, carry_s;
  if (threadIdx.x == 0) {
    carry_w = 0;
    carry_s = 0;
  }
  __syncthreads();
  unsigned long long work = 0;
  for (int w0 = 0; w0 < P.W; w0 += blockDim.x) {
    const int w = w0 + threadIdx.x;
    int segs = 0, parts = 0;
    if (w < P.W && !(fresh ? __ldcg(&P.converged[w]) : P.converged[w])) {
      const int2 r = P.wrange[w];
      segs = (r.y - r.x + ITEM - 1) / ITEM;
      parts = r.y - r.x;
    }
    const int on = segs > 0 ? 1 : 0;
    int tw, ts, tp;
    const int ow = block_exclusive_scan(on, smem, tw);
    const int os = block_exclusive_scan(segs, smem, ts);
    block_exclusive_scan(parts, smem, tp);
    work += (unsigned long long)tp;
    const int cw0 = carry_w, cs0 = carry_s;
    if (on) {
      P.cw[cw0 + ow] = w;
      P.cseg[cw0 + ow] = cs0 + os;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      carry_w = cw0 + tw;
      carry_s = cs0 + ts;
    }
    __syncthreads();
  }
  const int listed = carry_w;
  if (threadIdx.x == 0) {
    P.cseg[carry_w] = carry_s;
    *P.n_cw = carry_w;
    if (P.iter_work && work) atomicAdd(P.iter_work, work);  // the iteration this list drives, if it runs
  }
  return listed;
}

__global__ void __launch_bounds__(1024) k_worklist(DevP P) { build_worklist(P, false); }

// The sorted range [b, e) of this block's work item; false (for the whole block) past the last item.
// The first warp searches the listed worlds 32 probes at a time (cseg rises strictly over listed worlds, so the probes
// at or below t form a prefix of the lanes): about log32 of the worlds rounds of one load per lane.
__device__ __forceinline__ bool work_item(const DevP& P, int& b, int& e, int& w) {
  __shared__ int sb, se, sw;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int n = *P.n_cw;
    const int t = blockIdx.x;
    if (lane == 0) sb = se = sw = 0;
    if (n > 0 && t < P.cseg[n]) {
      int lo = 0, hi = n - 1;  // the last listed world whose first item is <= t lies in [lo, hi]
      while (lo < hi) {
        const int step = (hi - lo + 31) >> 5;
        const int q = lo + (lane + 1) * step;
        const unsigned below = __ballot_sync(0xffffffffu, q <= hi && P.cseg[q] <= t);
        const int k = __popc(below);
        hi = min(hi, lo + (k + 1) * step - 1);
        lo = lo + k * step;
      }
      if (lane == 0) {
        sw = P.cw[lo];
        const int2 r = P.wrange[sw];
        sb = r.x + (t - P.cseg[lo]) * ITEM;
        se = min(sb + ITEM, r.y);
      }
    }
  }
  __syncthreads();
  b = sb;
  e = se;
  w = sw;
  return b < e;
}

__device__ __forceinline__ bool work_item(const DevP& P, int& b, int& e) {
  int w;
  return work_item(P, b, e, w);
}

// ------------------------------------------------------------------------------------------ Jacobi sweep
// Where the pressure loops read a row and the neighbours' records: the rows in HBM and the particle arrays
// (GlobalRows), or the work item's halo staged in shared memory, addressed by 16-bit row entries (HaloRows). Both give
// every entry the same values, so the sums are the same bits.
struct GlobalRows {
  template <int NB>
  __device__ __forceinline__ void row(const DevP& P, int p, int c, int k, int (&j)[NB], float (&f)[NB]) const {
    load_row_batch_f(P, p, c, k, j, f);
  }
  __device__ __forceinline__ float4 pos(const DevP& P, int j) const { return P.pos[j]; }
  __device__ __forceinline__ float4 acc(const DevP& P, int j) const { return P.acc[j]; }
  __device__ __forceinline__ float kr(const DevP& P, int j) const { return P.kr[j]; }
};

struct HaloRows {
  const float4* hpos;  // [H] positions of the item's halo
  const float4* hacc;  // [H] accelerations (Jacobi) or nullptr
  const float* hkr;    // [H] kappa / rho0 (acceleration) or nullptr
  // Entries past the row's end read record 0 (a row with entries implies a halo of at least one) and are skipped.
  template <int NB>
  __device__ __forceinline__ void row(const DevP& P, int p, int c, int k, int (&j)[NB], float (&f)[NB]) const {
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      const size_t o = (size_t)(k + u) * P.n + p;
      j[u] = (k + u < c) ? (int)__ldcs(P.halo_row + o) : 0;
      f[u] = (k + u < c) ? __ldcs(P.halo_f + o) : 0.0f;
    }
  }
  __device__ __forceinline__ float4 pos(const DevP&, int j) const { return hpos[j]; }
  __device__ __forceinline__ float4 acc(const DevP&, int j) const { return hacc[j]; }
  __device__ __forceinline__ float kr(const DevP&, int j) const { return hkr[j]; }
};

// pressure.py:264-291: a_i = -sum_j m_j (k_i/rho0_i + k_j/rho0_j) grad W_ij - k_i sum_b dPsi_b
template <int NBX, class R = GlobalRows>
__device__ __forceinline__ void pressure_accel(const DevP& P, int p, float4 xi, float& ax, float& ay, float& az,
                                               const R& src = R()) {
  constexpr int NB = NBX & NB_MASK;
  constexpr bool MS = (NBX & MS_FLAG) != 0;
  float ki = P.kr[p];
  ax = ay = az = 0.0f;
  int c = P.cnt[p];
  for (int k = 0; k < c; k += NB) {
    int j[NB];
    float fb[NB];
    src.template row<NB>(P, p, c, k, j, fb);
    float4 xb[NB];
    float kb[NB];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      xb[u] = src.pos(P, j[u]);
      kb[u] = src.kr(P, j[u]);
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      if (k + u >= c) break;
      float4 xj = xb[u];
      float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
      float cF = (xj.w * (ki + kb[u])) * fb[u];
      ax = ADF_FMA(-cF, rx, ax);
      ay = ADF_FMA(-cF, ry, ay);
      az = ADF_FMA(-cF, rz, az);
    }
  }
  for_slots<MS>(P, p, [&](int, size_t o) {
    const float4 sg = P.slot_g[o];
    const float kk = P.kappa[p];
    ax = ADF_FMA(-kk, sg.x, ax);
    ay = ADF_FMA(-kk, sg.y, ay);
    az = ADF_FMA(-kk, sg.z, az);
  });
}

template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_accel(DevP P) {
  int b, e;
  if (!work_item(P, b, e)) return;
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
    float ax, ay, az;
    pressure_accel<NBX>(P, p, P.pos[p], ax, ay, az);
    P.acc[p] = make_float4(ax, ay, az, 0.0f);
  }
}

// pressure.py:294-352
// pressure.py:294-310: Ar_i of the accelerations in P.acc (the matrix-free product, before the compliance term)
template <int NBX, class R = GlobalRows>
__device__ __forceinline__ float accel_divergence(const DevP& P, int p, float inv_r0, const R& src = R()) {
  constexpr int NB = NBX & NB_MASK;
  constexpr bool MS = (NBX & MS_FLAG) != 0;
  float4 xi = P.pos[p];
  float4 ai = P.acc[p];
  float ar = 0.0f;
  int c = P.cnt[p];
  for (int k = 0; k < c; k += NB) {
    int j[NB];
    float fb[NB];
    src.template row<NB>(P, p, c, k, j, fb);
    float4 xb[NB], ab[NB];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      xb[u] = src.pos(P, j[u]);
      ab[u] = src.acc(P, j[u]);
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
      if (k + u >= c) break;
      float4 xj = xb[u], aj = ab[u];
      float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
      float aF = (xj.w * inv_r0) * fb[u];
      ar = ADF_FMA(aF, dotf(ai.x - aj.x, ai.y - aj.y, ai.z - aj.z, rx, ry, rz), ar);
    }
  }
  for_slots<MS>(P, p, [&](int, size_t o) {
    const float4 sg = P.slot_g[o];
    ar = ar + dotf(ai.x, ai.y, ai.z, sg.x, sg.y, sg.z);
  });
  return ar;
}

template <int NBX, class R = GlobalRows>
__device__ __forceinline__ void jacobi_one(const DevP& P, int p, const R& src = R()) {
  float r0 = P.vel[p].w;
  float inv_r0 = 1.0f / r0;
  float ar = accel_divergence<NBX>(P, p, inv_r0, src);
  float kap = P.kappa[p];
  ar = ADF_FMA(-P.reg[p], kap, ar);
  const float dt = P.dt;
  const bool div = P.mode == 0;
  float dtn = div ? dt : dt * dt;
  float scale = div ? 1.0f / dt : 1.0f / (dt * dt);
  ar = ar * dtn;
  float s = div ? -P.src[p] : 1.0f - P.src[p];
  float r = s - ar;
  float lb = P.lower[p];
  float knew = maxr(kap - ((P.omega * r) * P.alpha[p]) * scale, lb);
  P.kappa[p] = knew;
  P.kr[p] = knew / r0;
  float e = maxr(-r, 0.0f);
  if (knew > lb) e = fabsf(r);
  if (div) {
    if (P.neff[p] < P.min_nb) e = 0.0f;
    e = e * dt;
  }
  P.err_orig[P.id_of[p]] = e;
}

template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_jacobi(DevP P) {
  int b, e;
  if (!work_item(P, b, e)) return;
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) jacobi_one<NBX>(P, p);
}

// ------------------------------------------------------------------------------------ item halos
// The pressure iterations run one block per 256-particle work item (the item's particles are a compact brick of
// cells in the sorted order). Each row entry gathers two 16-byte records from scattered sorted positions, which is
// what bounds those loops in L1. k_halo, once per step after the rows' F are written, lists per item the distinct
// sorted positions its rows address (ascending: liquid, then walls) and rewrites the rows as 16-bit indices into
// that list with F beside them; the staged kernels then copy the item's records into shared memory with runs of
// consecutive loads and gather from there. Items are numbered g = b / 256 + w for the item of world w starting at
// sorted position b, which is strictly increasing over worlds and items and below nf / 256 + W + 1.
constexpr int HALO_CAP = 1280;    // records an item stages (20 KB of positions + 20 KB of accelerations)
constexpr int HALO_WORDS = 8192;  // bitmap words over the two spans of sorted positions an item addresses

__device__ __forceinline__ int halo_first(const DevP& P, int w) { return P.wrange[w].x / ITEM + w; }

__device__ __forceinline__ void block_min_max(int& lo, int& hi, int* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&red[0], lo);
    atomicMax(&red[1], hi);
  }
}

// One block of 256 threads per item number g (numbers between worlds' items are idle); dynamic shared memory:
// HALO_WORDS bitmap words and HALO_WORDS prefix counts.
__global__ void __launch_bounds__(ITEM) k_halo(DevP P) {
  extern __shared__ unsigned int hsm[];
  unsigned int* bits = hsm;
  unsigned int* pre = hsm + HALO_WORDS;
  __shared__ int sb, se, red[4], scan_smem[32];
  const int g = blockIdx.x;
  if (threadIdx.x == 0) {
    sb = se = 0;
    red[0] = red[2] = INT_MAX;
    red[1] = red[3] = -1;
    int lo = 0, hi = P.W - 1;  // the last world whose first item number is <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (halo_first(P, mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    if (P.W > 0 && halo_first(P, lo) <= g) {
      const int2 r = P.wrange[lo];
      const int t = g - halo_first(P, lo);
      if (r.x + t * ITEM < r.y) {
        sb = r.x + t * ITEM;
        se = min(sb + ITEM, r.y);
      }
    }
  }
  __syncthreads();
  const int b = sb, e = se;
  if (b >= e) return;
  const int nf = P.nfw[0];
  const size_t n = (size_t)P.n;
  // the spans of liquid and wall positions the item's rows address
  int llo = INT_MAX, lhi = -1, wlo = INT_MAX, whi = -1;
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
    const int c = P.cnt[p];
    for (int k = 0; k < c; ++k) {
      const int j = P.nbrjf[k * n + p].x;
      if (j < nf) {
        llo = min(llo, j);
        lhi = max(lhi, j);
      } else {
        wlo = min(wlo, j);
        whi = max(whi, j);
      }
    }
  }
  block_min_max(llo, lhi, red);
  block_min_max(wlo, whi, red + 2);
  __syncthreads();
  const int lwords = red[1] >= 0 ? (red[1] - red[0]) / 32 + 1 : 0;
  const int wwords = red[3] >= 0 ? (red[3] - red[2]) / 32 + 1 : 0;
  const int words = lwords + wwords;
  if (words > HALO_WORDS) {
    if (threadIdx.x == 0) P.halo_n[g] = -1;
    return;
  }
  const int l0 = red[0], w0 = red[2];
  for (int i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0u;
  __syncthreads();
  auto bit_of = [&](int j) { return j < nf ? j - l0 : lwords * 32 + (j - w0); };
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
    const int c = P.cnt[p];
    for (int k = 0; k < c; ++k) {
      const int x = bit_of(P.nbrjf[k * n + p].x);
      atomicOr(&bits[x >> 5], 1u << (x & 31));
    }
  }
  __syncthreads();
  // each thread owns a run of words: their popcounts, the block's exclusive scan, then each word's prefix
  const int per = (words + blockDim.x - 1) / blockDim.x;
  const int w_beg = min(words, (int)threadIdx.x * per), w_end = min(words, w_beg + per);
  int cntw = 0;
  for (int i = w_beg; i < w_end; ++i) cntw += __popc(bits[i]);
  int total;
  int off = block_exclusive_scan(cntw, scan_smem, total);
  if (total > HALO_CAP) {
    if (threadIdx.x == 0) P.halo_n[g] = -1;
    return;
  }
  int* hidx = P.halo_idx + (size_t)g * HALO_CAP;
  for (int i = w_beg; i < w_end; ++i) {
    pre[i] = (unsigned int)off;
    unsigned int m = bits[i];
    const int base = i < lwords ? l0 + i * 32 : w0 + (i - lwords) * 32;
    while (m) {
      const int t = __ffs(m) - 1;
      hidx[off++] = base + t;
      m &= m - 1u;
    }
  }
  __syncthreads();
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
    const int c = P.cnt[p];
    for (int k = 0; k < c; ++k) {
      const int2 jf = P.nbrjf[k * n + p];
      const int x = bit_of(jf.x);
      const unsigned int below = bits[x >> 5] & ((1u << (x & 31)) - 1u);
      P.halo_row[k * n + p] = (unsigned short)(pre[x >> 5] + __popc(below));
      P.halo_f[k * n + p] = __int_as_float(jf.y);
    }
  }
  if (threadIdx.x == 0) P.halo_n[g] = total;
}

// Copies item g's H records into shared memory, four per thread in flight: positions into hpos, src2's records
// (accelerations or kappa / rho0) into h2.
template <class T>
__device__ __forceinline__ void stage_halo(const DevP& P, int g, int H, float4* hpos, const T* src2, T* h2) {
  const int* hidx = P.halo_idx + (size_t)g * HALO_CAP;
  constexpr int U = 4;
  for (int i0 = threadIdx.x; i0 < H; i0 += U * blockDim.x) {
    int j[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      j[u] = i < H ? __ldg(hidx + i) : -1;
    }
    float4 x[U];
    T y[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (j[u] >= 0) {
        x[u] = P.pos[j[u]];
        y[u] = src2[j[u]];
      }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (j[u] >= 0) {
        const int i = i0 + u * (int)blockDim.x;
        hpos[i] = x[u];
        h2[i] = y[u];
      }
  }
  __syncthreads();
}

// The staged pressure iterations (same work items and arithmetic as k_accel and k_jacobi): an item without a halo
// takes the global gathers. Dynamic shared memory: HALO_CAP float4 positions, then HALO_CAP float4 accelerations
// (Jacobi) or HALO_CAP floats of kappa / rho0 (acceleration).
template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_accel_h(DevP P) {
  extern __shared__ float4 hrec[];
  int b, e, w;
  if (!work_item(P, b, e, w)) return;
  const int g = b / ITEM + w;
  const int H = P.halo_n[g];
  if (H < 0) {
    for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
      float ax, ay, az;
      pressure_accel<NBX>(P, p, P.pos[p], ax, ay, az);
      P.acc[p] = make_float4(ax, ay, az, 0.0f);
    }
    return;
  }
  float* hkr = reinterpret_cast<float*>(hrec + HALO_CAP);
  stage_halo(P, g, H, hrec, (const float*)P.kr, hkr);
  const HaloRows src{hrec, nullptr, hkr};
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) {
    float ax, ay, az;
    pressure_accel<NBX>(P, p, P.pos[p], ax, ay, az, src);
    P.acc[p] = make_float4(ax, ay, az, 0.0f);
  }
}

template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_jacobi_h(DevP P) {
  extern __shared__ float4 hrec[];
  int b, e, w;
  if (!work_item(P, b, e, w)) return;
  const int g = b / ITEM + w;
  const int H = P.halo_n[g];
  if (H < 0) {
    for (int p = b + threadIdx.x; p < e; p += blockDim.x) jacobi_one<NBX>(P, p);
    return;
  }
  float4* hacc = hrec + HALO_CAP;
  stage_halo(P, g, H, hrec, (const float4*)P.acc, hacc);
  const HaloRows src{hrec, hacc, nullptr};
  for (int p = b + threadIdx.x; p < e; p += blockDim.x) jacobi_one<NBX>(P, p, src);
}

constexpr size_t HALO_SMEM_BUILD = 2 * HALO_WORDS * sizeof(unsigned int);
constexpr size_t HALO_SMEM_ACCEL = HALO_CAP * (sizeof(float4) + sizeof(float));
constexpr size_t HALO_SMEM_JACOBI = HALO_CAP * 2 * sizeof(float4);

// ------------------------------------------------------------------------------------ projected CG (krylov.py)
// One CG per world on w = A k - b, k >= k_lo (krylov.py:1-17), A k = -dt^n (Ar(k) - reg k). Each kernel follows
// the reference kernel of the same name (krylov.py:71-246); a + b c updates are fused (the oracle fuses the same
// ones), per-world dot products are the float64 sums of k_sums2_fused in the caller's order.
// The stop test of a world at iteration `it` (pressure.py:370-390, krylov.py:236-241): converged after min_it when the
// mean and the maximum are within tol and tol_max, both times the world's tolerance factor, or at max_it.
__device__ __forceinline__ bool stop_test(const DevP& P, int w, int it, float mean, float mx) {
  const float ts = P.tol_scale != nullptr ? P.tol_scale[w] : 1.0f;
  return (it >= P.min_it && mean <= P.tol * ts && mx <= P.tol_max * ts) || it >= P.max_it;
}

__device__ __forceinline__ bool cg_skip(const DevP& P, int w, int gated) {
  return P.converged[w] != 0 || (gated && P.cg_restart[w] == 0);
}

// krylov.py:71-80: acc = pressure acceleration of the field vec (vr = vec / rho0)
template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_cg_accel(DevP P, const float* vec, const float* vr, int gated) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0] || cg_skip(P, P.world_s[p], gated)) return;
  DevP Q = P;
  Q.kappa = const_cast<float*>(vec);
  Q.kr = const_cast<float*>(vr);
  float ax, ay, az;
  pressure_accel<NBX>(Q, p, P.pos[p], ax, ay, az);
  P.acc[p] = make_float4(ax, ay, az, 0.0f);
}

// krylov.py:83-101: out (+)= A vec (- b); pair.x = vec_i (A vec)_i
template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_cg_apply(DevP P, const float* vec, float* out, int gated, int bias,
                                                    int accumulate) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0] || cg_skip(P, P.world_s[p], gated)) return;
  const float dt = P.dt;
  const bool div = P.mode == 0;
  const float scale = div ? dt : dt * dt;
  const float inv_r0 = 1.0f / P.vel[p].w;
  const float t = ADF_FMA(-P.reg[p], vec[p], accel_divergence<NBX>(P, p, inv_r0));
  float v = -(scale * t);
  P.cg_pair[P.id_of[p]] = make_float2(vec[p] * v, 0.0f);
  if (bias) v = v - (div ? P.src[p] : P.src[p] - 1.0f);
  if (accumulate) v = v + out[p];
  out[p] = v;
}

// Team variants of the CG products for worlds too small to fill the GPU with one lane per particle (a 30k-particle
// world is less than one wave, and each lane's row is a chain of dependent gathers): TL lanes share one particle,
// lane t gathers row entries t, t + TL, ... (TB of them per round) and computes their terms, and the team's first
// lane adds the terms in row order with the one-lane loop's own operations, so the results are bit-identical.
constexpr int TL = 4;  // lanes per particle
constexpr int TB = 4;  // row entries per lane per round

struct Team {
  int t, t0;       // this lane's rank in the team, the team's first lane (in the warp)
  unsigned mask;   // the team's lanes
};

// The team of this thread in block `vb` of BLOCK threads (a launch's own block, or a persistent kernel's virtual one).
__device__ __forceinline__ Team team_at(int vb, int& p) {
  const int g = vb * BLOCK + threadIdx.x;
  p = g / TL;
  Team tm;
  tm.t = g % TL;
  tm.t0 = (threadIdx.x & 31) - tm.t;
  tm.mask = ((1u << TL) - 1u) << tm.t0;
  return tm;
}

__device__ __forceinline__ Team team_of(int& p) { return team_at(blockIdx.x, p); }

__device__ __forceinline__ int2 row_entry(const DevP& P, int p, int k) { return __ldcs(P.nbrjf + p + (size_t)k * P.n); }

// pressure_accel with the fields of Q (kappa, kr), valid in the team's first lane
template <bool MS>
__device__ __forceinline__ void pressure_accel_team(const DevP& Q, int p, float4 xi, const Team& tm, float& ax, float& ay,
                                                    float& az) {
  const float ki = Q.kr[p];
  ax = ay = az = 0.0f;
  const int c = Q.cnt[p];
  for (int k0 = 0; k0 < c; k0 += TL * TB) {
    float cf[TB], rx[TB], ry[TB], rz[TB];
#pragma unroll
    for (int u = 0; u < TB; ++u) {
      const int k = k0 + u * TL + tm.t;
      cf[u] = rx[u] = ry[u] = rz[u] = 0.0f;
      if (k < c) {
        const int2 e = row_entry(Q, p, k);
        const float4 xj = Q.pos[e.x];
        const float kj = Q.kr[e.x];
        rx[u] = xi.x - xj.x;
        ry[u] = xi.y - xj.y;
        rz[u] = xi.z - xj.z;
        cf[u] = (xj.w * (ki + kj)) * __int_as_float(e.y);
      }
    }
#pragma unroll
    for (int u = 0; u < TB; ++u) {
#pragma unroll
      for (int s = 0; s < TL; ++s) {
        const float a = __shfl_sync(tm.mask, cf[u], tm.t0 + s), x = __shfl_sync(tm.mask, rx[u], tm.t0 + s);
        const float y = __shfl_sync(tm.mask, ry[u], tm.t0 + s), z = __shfl_sync(tm.mask, rz[u], tm.t0 + s);
        if (tm.t == 0 && k0 + u * TL + s < c) {
          ax = ADF_FMA(-a, x, ax);
          ay = ADF_FMA(-a, y, ay);
          az = ADF_FMA(-a, z, az);
        }
      }
    }
  }
  for_slots<MS>(Q, p, [&](int, size_t o) {
    const float4 sg = Q.slot_g[o];
    const float kk = Q.kappa[p];
    ax = ADF_FMA(-kk, sg.x, ax);
    ay = ADF_FMA(-kk, sg.y, ay);
    az = ADF_FMA(-kk, sg.z, az);
  });
}

// accel_divergence, valid in the team's first lane
template <bool MS>
__device__ __forceinline__ float accel_divergence_team(const DevP& P, int p, float inv_r0, const Team& tm) {
  const float4 xi = P.pos[p];
  const float4 ai = P.acc[p];
  float ar = 0.0f;
  const int c = P.cnt[p];
  for (int k0 = 0; k0 < c; k0 += TL * TB) {
    float af[TB], d[TB];
#pragma unroll
    for (int u = 0; u < TB; ++u) {
      const int k = k0 + u * TL + tm.t;
      af[u] = d[u] = 0.0f;
      if (k < c) {
        const int2 e = row_entry(P, p, k);
        const float4 xj = P.pos[e.x], aj = P.acc[e.x];
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        af[u] = (xj.w * inv_r0) * __int_as_float(e.y);
        d[u] = dotf(ai.x - aj.x, ai.y - aj.y, ai.z - aj.z, rx, ry, rz);
      }
    }
#pragma unroll
    for (int u = 0; u < TB; ++u) {
#pragma unroll
      for (int s = 0; s < TL; ++s) {
        const float a = __shfl_sync(tm.mask, af[u], tm.t0 + s), b = __shfl_sync(tm.mask, d[u], tm.t0 + s);
        if (tm.t == 0 && k0 + u * TL + s < c) ar = ADF_FMA(a, b, ar);
      }
    }
  }
  for_slots<MS>(P, p, [&](int, size_t o) {
    const float4 sg = P.slot_g[o];
    ar = ar + dotf(ai.x, ai.y, ai.z, sg.x, sg.y, sg.z);
  });
  return ar;
}

// k_cg_accel by teams (grid: TL threads per particle). The kernels below are bodies run for one block `vb` of BLOCK
// threads, launched one block each by their __global__ wrappers or looped over by the persistent solve (k_cg_solve).
template <bool MS>
__device__ __forceinline__ void cg_accel_team_at(const DevP& P, const float* vec, const float* vr, int gated, int vb) {
  int p;
  const Team tm = team_at(vb, p);
  if (p >= P.nfw[0] || cg_skip(P, P.world_s[p], gated)) return;
  DevP Q = P;
  Q.kappa = const_cast<float*>(vec);
  Q.kr = const_cast<float*>(vr);
  float ax, ay, az;
  pressure_accel_team<MS>(Q, p, P.pos[p], tm, ax, ay, az);
  if (tm.t == 0) P.acc[p] = make_float4(ax, ay, az, 0.0f);
}

template <bool MS>
__global__ void __launch_bounds__(BLOCK) k_cg_accel_team(DevP P, const float* vec, const float* vr, int gated) {
  cg_accel_team_at<MS>(P, vec, vr, gated, blockIdx.x);
}

// k_cg_apply by teams
template <bool MS>
__device__ __forceinline__ void cg_apply_team_at(const DevP& P, const float* vec, float* out, int gated, int bias,
                                                 int accumulate, int vb) {
  int p;
  const Team tm = team_at(vb, p);
  if (p >= P.nfw[0] || cg_skip(P, P.world_s[p], gated)) return;
  const float inv_r0 = 1.0f / P.vel[p].w;
  const float ar = accel_divergence_team<MS>(P, p, inv_r0, tm);
  if (tm.t != 0) return;
  const float dt = P.dt;
  const bool div = P.mode == 0;
  const float scale = div ? dt : dt * dt;
  const float t = ADF_FMA(-P.reg[p], vec[p], ar);
  float v = -(scale * t);
  P.cg_pair[P.id_of[p]] = make_float2(vec[p] * v, 0.0f);
  if (bias) v = v - (div ? P.src[p] : P.src[p] - 1.0f);
  if (accumulate) v = v + out[p];
  out[p] = v;
}

template <bool MS>
__global__ void __launch_bounds__(BLOCK) k_cg_apply_team(DevP P, const float* vec, float* out, int gated, int bias,
                                                         int accumulate) {
  cg_apply_team_at<MS>(P, vec, out, gated, bias, accumulate, blockIdx.x);
}

// krylov.py:104-133: active set, z = M^-1 r on F (r = -w), first direction p = z; pair.x = r.z
__device__ __forceinline__ void cg_init_at(const DevP& P, int vb) {
  const int p = vb * BLOCK + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const float dt = P.dt;
  const float scale = P.mode == 0 ? dt : dt * dt;
  const float w = P.cg_w[p];
  const bool a = P.kappa[p] > P.lower[p] || w < 0.0f;
  const float zi = a ? ((-w) * P.alpha[p]) / scale : 0.0f;
  P.cg_act[p] = a ? 1 : 0;
  P.cg_z[p] = zi;
  P.cg_pd[p] = zi;
  P.cg_pdr[p] = zi / P.vel[p].w;
  P.cg_pair[P.id_of[p]] = make_float2(-w * zi, 0.0f);
}

__global__ void __launch_bounds__(BLOCK) k_cg_init(DevP P) { cg_init_at(P, blockIdx.x); }

__device__ __forceinline__ void cg_first_rz_at(const DevP& P, int vb) {
  const int w = vb * BLOCK + threadIdx.x;
  if (w >= P.W) return;
  P.cg_rz[w] = P.cg_sums[w].x;
  P.cg_restart[w] = 0;
  P.cg_act_new[w] = 0;
}

__global__ void __launch_bounds__(BLOCK) k_cg_first_rz(DevP P) { cg_first_rz_at(P, blockIdx.x); }

// krylov.py:146-170: k += a p on F, projected onto k >= k_lo (the clamped part into corr); w += a A p
__device__ __forceinline__ void cg_step_at(const DevP& P, int vb) {
  const int p = vb * BLOCK + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  if (P.converged[w]) return;
  const double pap = P.cg_sums[w].x;
  const float a = (float)(pap > 1.0e-30 ? P.cg_rz[w] / pap : 0.0);
  const float r0 = P.vel[p].w;
  float c = 0.0f;
  if (P.cg_act[p]) {
    float k = ADF_FMA(a, P.cg_pd[p], P.kappa[p]);
    const float lb = P.lower[p];
    if (k < lb) {
      c = lb - k;
      k = lb;
      P.cg_act[p] = 0;
      atomicAdd(&P.cg_restart[w], 1);
    }
    P.kappa[p] = k;
    P.kr[p] = k / r0;
  }
  P.cg_corr[p] = c;
  P.cg_corrr[p] = c / r0;
  P.cg_w[p] = ADF_FMA(a, P.cg_ap[p], P.cg_w[p]);
}

__global__ void __launch_bounds__(BLOCK) k_cg_step(DevP P) { cg_step_at(P, blockIdx.x); }

// krylov.py:148-204 after the step: in worlds where k_cg_step clamped a variable, w += A corr (the correction
// product of k_cg_apply: its acceleration field comes from k_cg_accel, launched for the same worlds); then in every
// iterating world the activation of compressed bound variables, z = M^-1 r on F and (r.z, error) per particle. One
// kernel: the finish needs only the particle's own w. Activations are flagged in cg_act_new, not in cg_restart,
// which decides here which worlds take the product.
// The finish of one particle after its w update (activation, z, r.z and error).
__device__ __forceinline__ void cg_finish_one(const DevP& P, int p, int w, float wv, float scale, bool div) {
  int act = P.cg_act[p];
  if (!act && wv < 0.0f) {
    act = 1;
    P.cg_act[p] = 1;
    P.cg_act_new[w] = 1;
  }
  const float zi = act ? ((-wv) * P.alpha[p]) / scale : 0.0f;
  P.cg_z[p] = zi;
  float e = maxr(-wv, 0.0f);
  if (P.kappa[p] > P.lower[p]) e = fabsf(wv);
  if (div) {
    if (P.neff[p] < P.min_nb) e = 0.0f;
    e = e * P.dt;
  }
  const int i = P.id_of[p];
  P.err_orig[i] = e;
  P.cg_pair[i] = make_float2(-wv * zi, e);
}

template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_cg_apply_finish(DevP P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  if (P.converged[w]) return;
  const float dt = P.dt;
  const bool div = P.mode == 0;
  const float scale = div ? dt : dt * dt;
  float wv = P.cg_w[p];
  if (P.cg_restart[w] != 0) {
    const float inv_r0 = 1.0f / P.vel[p].w;
    const float t = ADF_FMA(-P.reg[p], P.cg_corr[p], accel_divergence<NBX>(P, p, inv_r0));
    wv = -(scale * t) + wv;
    P.cg_w[p] = wv;
  }
  cg_finish_one(P, p, w, wv, scale, div);
}

// k_cg_apply_finish by teams
template <bool MS>
__device__ __forceinline__ void cg_apply_finish_team_at(const DevP& P, int vb) {
  int p;
  const Team tm = team_at(vb, p);
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  if (P.converged[w]) return;
  const float dt = P.dt;
  const bool div = P.mode == 0;
  const float scale = div ? dt : dt * dt;
  float wv = P.cg_w[p];
  if (P.cg_restart[w] != 0) {
    const float inv_r0 = 1.0f / P.vel[p].w;
    const float ar = accel_divergence_team<MS>(P, p, inv_r0, tm);
    if (tm.t == 0) {
      const float t = ADF_FMA(-P.reg[p], P.cg_corr[p], ar);
      wv = -(scale * t) + wv;
      P.cg_w[p] = wv;
    }
  }
  if (tm.t == 0) cg_finish_one(P, p, w, wv, scale, div);
}

template <bool MS>
__global__ void __launch_bounds__(BLOCK) k_cg_apply_finish_team(DevP P) { cg_apply_finish_team_at<MS>(P, blockIdx.x); }

// krylov.py:207-233: per world the stop test (as k_world_check), then beta = r.z_new / r.z (0 after a set change)
__device__ __forceinline__ void cg_beta_world(const DevP& P, int w) {
  const int it = P.iters[w] + 1;
  P.iters[w] = it;
  const double2 sm = P.cg_sums[w];
  const double na = P.n_active[w];
  const float mean = (float)(sm.y / (na > 1.0 ? na : 1.0));
  P.err_mean[w] = mean;
  double beta = 0.0;
  if (P.cg_restart[w] == 0 && P.cg_act_new[w] == 0 && P.cg_rz[w] > 1.0e-30) beta = sm.x / P.cg_rz[w];
  P.cg_restart[w] = 0;
  P.cg_act_new[w] = 0;
  P.cg_rz[w] = sm.x;
  P.cg_step[w] = beta;
  if (stop_test(P, w, it, mean, P.emax[w])) P.converged[w] = 1;
}

__global__ void k_cg_beta(DevP P) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W || P.converged[w]) return;
  cg_beta_world(P, w);
  if (!P.converged[w]) atomicAdd(P.n_unconv, 1);
}

// krylov.py:236-246: p = z + beta p on F, 0 elsewhere
__device__ __forceinline__ void cg_direction_at(const DevP& P, int vb) {
  const int p = vb * BLOCK + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int w = P.world_s[p];
  if (P.converged[w]) return;
  const float pd = P.cg_act[p] ? ADF_FMA((float)P.cg_step[w], P.cg_pd[p], P.cg_z[p]) : 0.0f;
  P.cg_pd[p] = pd;
  P.cg_pdr[p] = pd / P.vel[p].w;
}

__global__ void __launch_bounds__(BLOCK) k_cg_direction(DevP P) { cg_direction_at(P, blockIdx.x); }

// Per-world (sum x, sum y, max y) of the CG pairs for models without chunks (no particles): one block per world in
// the fixed tree order of k_world_check; k_sums2_fused does it in one launch otherwise.
__global__ void __launch_bounds__(256) k_world_sum2(DevP P, int with_max) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  const int w = blockIdx.x;
  if (P.converged[w]) return;
  const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
  double ax = 0.0, ay = 0.0;
  float m = -3.4e38f;
  for (int c = c0 + threadIdx.x; c < c1; c += 256) {
    ax = ax + P.part2[c].x;
    ay = ay + P.part2[c].y;
    m = fmaxf(m, P.part_max[c]);
  }
  const double sx = fold256(ax, smd);
  const double sy = fold256(ay, smd);
  const float mx = block_max256(m, smf);
  if (threadIdx.x != 0) return;
  P.cg_sums[w] = make_double2(sx, sy);
  if (with_max) P.emax[w] = maxr(mx, 0.0f);
}

// fold256's tree computed by one warp: value L of the 256 (group L / 32, lane L % 32) comes from value(L); each group
// of 32 folds by the same shuffles (offsets 16..1), then the 8 group sums fold with offsets 4, 2, 1. Valid in lane 0.
template <class F>
__device__ __forceinline__ double fold256_warp(F value) {
  const int lane = threadIdx.x & 31;
  double s[8];
#pragma unroll
  for (int g = 0; g < 8; ++g) {
    double v = value(32 * g + lane);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
    s[g] = v;
  }
#pragma unroll
  for (int o = 4; o >= 1; o >>= 1)
#pragma unroll
    for (int l = 0; l < o; ++l) s[l] = s[l] + s[l + o];
  return s[0];
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return __shfl_sync(0xffffffffu, v, 0);
}

// --------------------------------------------------------------------------- resting-jitter rule (solve_driver.py)
// Per world and step the density solve's tolerance is tol x tol_scale[w] (solve_driver.py:5-21): tol_scale =
// clamp(v dt / (H tol), tol_min / tol, 1) with H = 1.5 S2 / (S1 dt^2 |g|) from the density warm starts kd
// (S1 = sum kd+, S2 = sum kd+^2 over the world's liquid, kd+ = max(kd, 0)) and v = max(speed, ratio |U|), U the mean
// velocity of the liquid in the step's start state. The sums are float64 over the caller's order in the tree order of
// the other per-world sums (chunks of 256 by one warp each, then each world's chunks).
constexpr int JIT_TERMS = 4;

// term k of particle i (caller's order), 0 unless liquid: flow (k: v_z, 1, v_x, v_y; solve_driver.py:40-51, the
// step's start velocity) or head (k: kd+, kd+ kd+; solve_driver.py:27-37)
__device__ __forceinline__ float jitter_term(const DevP& P, int i, int head, int k) {
  if (!is_fluid_orig(P, i)) return 0.0f;
  if (!head) {
    const float* v = P.qd + 3 * (size_t)i;
    return k == 0 ? v[2] : k == 1 ? 1.0f : k == 2 ? v[0] : v[1];
  }
  const float kd = maxr(P.kd[i], 0.0f);
  return k == 0 ? kd : kd * kd;
}

// per chunk (one warp each, 8 per block): the float64 sums of the terms (2 for head, 4 for flow) into part[c][k]
__global__ void __launch_bounds__(256) k_jitter_chunks(DevP P, int head, double* part) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (c >= P.n_chunks) return;
  const int b = P.chunk_begin[c], e = P.chunk_end[c];
  const int K = head ? 2 : JIT_TERMS;
  for (int k = 0; k < K; ++k) {
    const double sum = fold256_warp([&](int L) -> double {
      const int i = b + L;
      return i < e ? (double)jitter_term(P, i, head, k) : 0.0;
    });
    if (lane == 0) part[(size_t)c * JIT_TERMS + k] = sum;
  }
}

// per world (one warp each): its chunks' partials folded into out[w][k]
__global__ void __launch_bounds__(256) k_jitter_worlds(DevP P, int head, const double* part, double* out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (w >= P.W) return;
  const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
  const int K = head ? 2 : JIT_TERMS;
  for (int k = 0; k < K; ++k) {
    const double sum = fold256_warp([&](int L) -> double {
      double a = 0.0;
      for (int c = c0 + L; c < c1; c += 256) a = a + part[(size_t)c * JIT_TERMS + k];
      return a;
    });
    if (lane == 0) out[(size_t)w * JIT_TERMS + k] = sum;
  }
}

// solve_driver.py:54-74 (tol_scale_kernel) and runtime.py:115-116 (the reported tolerance tol x scale); `flow` null
// when the flow ratio is 0
__global__ void k_tol_scale(DevP P, const double* head, const double* flow, float dt, float speed, float ratio,
                            float tol, float tol_min, float* scale, float* den_tol) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.W) return;
  float s = 1.0f;
  const float gx = P.gravity[3 * w], gy = P.gravity[3 * w + 1], gz = P.gravity[3 * w + 2];
  const float g = __fsqrt_rn(dot_plain(gx, gy, gz, gx, gy, gz));
  const float s1 = (float)head[(size_t)w * JIT_TERMS], s2 = (float)head[(size_t)w * JIT_TERMS + 1];
  float v = speed;
  if (flow != nullptr) {
    const double n = flow[(size_t)w * JIT_TERMS + 1];
    if (ratio > 0.0f && n > 0.0) {
      const float ux = (float)(flow[(size_t)w * JIT_TERMS + 2] / n), uy = (float)(flow[(size_t)w * JIT_TERMS + 3] / n);
      const float uz = (float)(flow[(size_t)w * JIT_TERMS] / n);
      v = maxr(v, ratio * __fsqrt_rn(dot_plain(ux, uy, uz, ux, uy, uz)));
    }
  }
  if (g > 0.0f && s1 > 0.0f && s2 > 0.0f) {
    const float depth = (1.5f * s2) / (((s1 * dt) * dt) * g);
    s = minr(maxr((v * dt) / (depth * tol), tol_min / tol), 1.0f);
  }
  scale[w] = s;
  den_tol[w] = tol * s;
}

// Per-chunk float64 sums (fold256's tree) and maxima of v, one warp per 256-value chunk, 8 chunks per block (a block
// per chunk spent most of its time being scheduled on workloads of tens of thousands of chunks).
__global__ void __launch_bounds__(256) k_chunk_sum(const float* __restrict__ v, const int* __restrict__ chunk_begin,
                                                   const int* __restrict__ chunk_end, int n_chunks, double* part_sum,
                                                   float* part_max) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (c >= n_chunks) return;
  const int b = chunk_begin[c], e = chunk_end[c];
  float m = -3.4e38f;
  const double sum = fold256_warp([&](int L) -> double {
    const int i = b + L;
    const float x = i < e ? v[i] : 0.0f;
    if (i < e) m = fmaxf(m, x);
    return i < e ? (double)x : 0.0;
  });
  m = warp_max(m);
  if (lane == 0) {
    part_sum[c] = sum;
    part_max[c] = m;
  }
}

// One block per world: the chunk partials (lane l takes chunks l, l + 256, ...), then the stop test
// (pressure.py:370-390) when `check` is set.
__global__ void __launch_bounds__(256) k_world_check(DevP P, int check, double* out_sum, float* out_max) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  int w = blockIdx.x;
  if (check && P.converged[w]) return;  // its error sums and maximum are those it converged with
  int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
  double a = 0.0;
  float m = -3.4e38f;
  for (int c = c0 + threadIdx.x; c < c1; c += 256) {
    a = a + P.part_sum[c];
    m = fmaxf(m, P.part_max[c]);
  }
  double s = fold256(a, smd);
  float mx = block_max256(m, smf);
  if (threadIdx.x != 0) return;
  mx = maxr(mx, 0.0f);
  if (!check) {
    out_sum[w] = s;
    out_max[w] = mx;
    return;
  }
  P.emax[w] = mx;
  int it = P.iters[w] + 1;
  P.iters[w] = it;
  double na = P.n_active[w];
  float mean = (float)(s / (na > 1.0 ? na : 1.0));
  P.err_mean[w] = mean;
  if (stop_test(P, w, it, mean, mx)) P.converged[w] = 1;
  else atomicAdd(P.n_unconv, 1);
}

// Tickets of the one-launch reductions below: thread 0 of a block that has stored its partials takes a ticket of its
// world (true for the world's last block, which resets the counter for the next launch).
__device__ __forceinline__ bool world_ticket(const DevP& P, int w, int chunks) {
  __threadfence();
  const bool last = atomicAdd(&P.wdone[w], 1) == chunks - 1;
  if (last) P.wdone[w] = 0;
  return last;
}

// The grid's ticket is taken once per world that has chunks: by its last block when the world iterates, by its first
// chunk's block when it had converged before the launch; the last of the n_chunk_worlds tickets is the grid's last.
__device__ __forceinline__ bool grid_ticket(const DevP& P) {
  __threadfence();
  const bool last = atomicAdd(P.gdone, 1u) == (unsigned)P.n_chunk_worlds - 1u;
  if (last) *P.gdone = 0u;
  return last;
}

// The Jacobi iteration's stop test in one launch (k_chunk_sum, k_world_check and k_worklist fused): block c folds
// chunk c (chunks of converged worlds keep their partials); the last block of a world to finish folds the world's
// partials in the same fixed tree order as k_world_check and runs its stop test (pressure.py:370-390); the last block
// of the grid lists the worlds still iterating for the next iteration and stores their count as the unconverged
// count. The sums are those of the separate kernels bit for bit; only the launches are fewer. Used when a world
// has more than WARP_FOLD_MAX_CHUNKS chunks (k_check_warps otherwise), where 256 threads fold its partials in parallel.
__global__ void __launch_bounds__(256) k_check_fused(DevP P) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  __shared__ bool wlast, glast;
  const int c = blockIdx.x;
  const int w = P.chunk_world[c];
  const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
  bool ticket = c == c0;  // the world's grid ticket: its first chunk's block if it had converged, else its last block
  if (!P.converged[w]) {
    const int i = P.chunk_begin[c] + threadIdx.x;
    const bool in = i < P.chunk_end[c];
    const float x = in ? P.err_orig[i] : 0.0f;
    const double s = fold256(in ? (double)x : 0.0, smd);
    const float m = block_max256(in ? x : -3.4e38f, smf);
    if (threadIdx.x == 0) {
      P.part_sum[c] = s;
      P.part_max[c] = m;
      wlast = world_ticket(P, w, c1 - c0);
    }
    __syncthreads();
    if (wlast) {
      __threadfence();
      double a = 0.0;
      float mm = -3.4e38f;
      for (int k = c0 + threadIdx.x; k < c1; k += 256) {
        a = a + __ldcg(&P.part_sum[k]);
        mm = fmaxf(mm, __ldcg(&P.part_max[k]));
      }
      const double sw = fold256(a, smd);
      const float mx = maxr(block_max256(mm, smf), 0.0f);
      if (threadIdx.x == 0) {
        P.emax[w] = mx;
        const int it = P.iters[w] + 1;
        P.iters[w] = it;
        const double na = P.n_active[w];
        const float mean = (float)(sw / (na > 1.0 ? na : 1.0));
        P.err_mean[w] = mean;
        if (stop_test(P, w, it, mean, mx)) P.converged[w] = 1;
      }
    }
    ticket = wlast;
  }
  if (!ticket) return;
  if (threadIdx.x == 0) glast = grid_ticket(P);
  __syncthreads();
  if (glast) {
    __threadfence();
    const int listed = build_worklist(P, true);
    if (threadIdx.x == 0) *P.n_unconv = listed;
  }
}

// k_check_fused with one warp per 256-particle chunk (8 chunks per block), for models whose worlds have at most
// WARP_FOLD_MAX_CHUNKS chunks (many small worlds): the warp folds its chunk in fold256's tree order (chunks of converged
// worlds keep their partials); the last warp of a world to finish folds the world's partials in k_world_check's order
// and runs its stop test (pressure.py:370-390); the block whose tickets complete the grid lists the worlds still
// iterating and stores their count as the unconverged count. The sums are those of the separate kernels bit for bit.
// A block per chunk (80k blocks on the 4,096-world pour) spent most of its time scheduling blocks; a warp folding a
// large world's thousands of partials alone (the 1M dam break's 4,096) waits on them serially. The world's last warp
// folds its
// partials (its 32 lanes stand in for the 256 of k_world_check: value L sums partials L, L + 256, ... serially); a
// block takes one grid ticket for all the worlds its warps completed (or that had converged and start in one of its
// chunks), and the block whose tickets complete the grid lists the worlds still iterating.
constexpr int CHECK_WARPS = 8;
constexpr int WARP_FOLD_MAX_CHUNKS = 256;  // a lane folds at most one partial per group of the 256-lane tree

__global__ void __launch_bounds__(32 * CHECK_WARPS) k_check_warps(DevP P) {
  __shared__ int tickets[CHECK_WARPS];
  __shared__ bool glast;
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int c = blockIdx.x * CHECK_WARPS + wq;
  int ticket = 0;
  if (c < P.n_chunks) {
    const int w = P.chunk_world[c];
    const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
    ticket = c == c0 ? 1 : 0;
    if (!P.converged[w]) {
      const int b = P.chunk_begin[c], e = P.chunk_end[c];
      float m = -3.4e38f;
      const double sum = fold256_warp([&](int L) -> double {
        const int i = b + L;
        const float x = i < e ? P.err_orig[i] : 0.0f;
        if (i < e) m = fmaxf(m, x);
        return i < e ? (double)x : 0.0;
      });
      m = warp_max(m);
      bool last = false;
      if (lane == 0) {
        P.part_sum[c] = sum;
        P.part_max[c] = m;
        last = world_ticket(P, w, c1 - c0);
      }
      last = __shfl_sync(0xffffffffu, last, 0);
      if (last) {
        __threadfence();
        float mm = -3.4e38f;
        const double sw = fold256_warp([&](int L) -> double {
          double a = 0.0;
          for (int k = c0 + L; k < c1; k += 256) {
            a = a + __ldcg(&P.part_sum[k]);
            mm = fmaxf(mm, __ldcg(&P.part_max[k]));
          }
          return a;
        });
        const float mx = maxr(warp_max(mm), 0.0f);
        if (lane == 0) {
          P.emax[w] = mx;
          const int it = P.iters[w] + 1;
          P.iters[w] = it;
          const double na = P.n_active[w];
          const float mean = (float)(sw / (na > 1.0 ? na : 1.0));
          P.err_mean[w] = mean;
          if (stop_test(P, w, it, mean, mx)) P.converged[w] = 1;
        }
      }
      ticket = last ? 1 : 0;
    }
  }
  if (lane == 0) tickets[wq] = ticket;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < CHECK_WARPS; ++k) t += tickets[k];
    glast = false;
    if (t > 0) {
      __threadfence();
      const unsigned before = atomicAdd(P.gdone, (unsigned)t);
      glast = before + (unsigned)t == (unsigned)P.n_chunk_worlds;
      if (glast) *P.gdone = 0u;
    }
  }
  __syncthreads();
  if (glast) {
    __threadfence();
    const int listed = build_worklist(P, true);
    if (threadIdx.x == 0) *P.n_unconv = listed;
  }
}

// The CG reductions in one launch (chunk partials and k_world_sum2's world fold, same tree order); with `beta`
// the world's last block also runs k_cg_beta's stop test and beta for its world, and the grid's last block stores the
// count of worlds still iterating as the unconverged count.
__device__ __forceinline__ void sums2_fused_at(const DevP& P, int with_max, int beta, int vb) {
  __shared__ double smd[8];
  __shared__ float smf[8];
  __shared__ int smi[32];
  __shared__ bool wlast, glast;
  const int c = vb;
  const int w = P.chunk_world[c];
  const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
  bool ticket = c == c0;  // as in k_check_fused
  if (!P.converged[w]) {
    const int i = P.chunk_begin[c] + threadIdx.x;
    const bool in = i < P.chunk_end[c];
    const float2 v = in ? P.cg_pair[i] : make_float2(0.0f, 0.0f);
    const double sx = fold256(in ? (double)v.x : 0.0, smd);
    const double sy = fold256(in ? (double)v.y : 0.0, smd);
    const float m = block_max256(in ? v.y : -3.4e38f, smf);
    if (threadIdx.x == 0) {
      P.part2[c] = make_double2(sx, sy);
      P.part_max[c] = m;
      wlast = world_ticket(P, w, c1 - c0);
    }
    __syncthreads();
    if (wlast) {
      __threadfence();
      double ax = 0.0, ay = 0.0;
      float mm = -3.4e38f;
      for (int k = c0 + threadIdx.x; k < c1; k += 256) {
        const double2 pk = __ldcg(&P.part2[k]);
        ax = ax + pk.x;
        ay = ay + pk.y;
        mm = fmaxf(mm, __ldcg(&P.part_max[k]));
      }
      const double wx = fold256(ax, smd);
      const double wy = fold256(ay, smd);
      const float mx = block_max256(mm, smf);
      if (threadIdx.x == 0) {
        P.cg_sums[w] = make_double2(wx, wy);
        if (with_max) P.emax[w] = maxr(mx, 0.0f);
        if (beta) cg_beta_world(P, w);
      }
    }
    ticket = wlast;
  }
  if (!beta || !ticket) return;
  if (threadIdx.x == 0) glast = grid_ticket(P);
  __syncthreads();
  if (glast) {
    __threadfence();
    int open = 0;
    for (int k = threadIdx.x; k < P.W; k += 256) open += __ldcg(&P.converged[k]) ? 0 : 1;
    int tot;
    block_exclusive_scan(open, smi, tot);
    if (threadIdx.x == 0) *P.n_unconv = tot;
  }
}

__global__ void __launch_bounds__(256) k_sums2_fused(DevP P, int with_max, int beta) {
  sums2_fused_at(P, with_max, beta, blockIdx.x);
}

// fold256_warp for two sums at once (value(L, x, y) gives value L of each)
template <class F>
__device__ __forceinline__ void fold256_warp2(F value, double& rx, double& ry) {
  double sx[8], sy[8];
#pragma unroll
  for (int g = 0; g < 8; ++g) {
    double x, y;
    value(32 * g + (threadIdx.x & 31), x, y);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      x = x + __shfl_down_sync(0xffffffffu, x, o);
      y = y + __shfl_down_sync(0xffffffffu, y, o);
    }
    sx[g] = x;
    sy[g] = y;
  }
#pragma unroll
  for (int o = 4; o >= 1; o >>= 1)
#pragma unroll
    for (int l = 0; l < o; ++l) {
      sx[l] = sx[l] + sx[l + o];
      sy[l] = sy[l] + sy[l + o];
    }
  rx = sx[0];
  ry = sy[0];
}

// k_sums2_fused with one warp per chunk (8 per block), for models whose worlds have at most WARP_FOLD_MAX_CHUNKS
// chunks: the same partials, world folds, stop tests, beta and unconverged count in the same tree orders.
__device__ __forceinline__ void sums2_warps_at(const DevP& P, int with_max, int beta, int vb) {
  __shared__ int tickets[CHECK_WARPS];
  __shared__ int smi[32];
  __shared__ bool glast;
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int c = vb * CHECK_WARPS + wq;
  int ticket = 0;
  if (c < P.n_chunks) {
    const int w = P.chunk_world[c];
    const int c0 = P.world_chunk_start[w], c1 = P.world_chunk_start[w + 1];
    ticket = c == c0 ? 1 : 0;
    if (!P.converged[w]) {
      const int b = P.chunk_begin[c], e = P.chunk_end[c];
      float m = -3.4e38f;
      double sx, sy;
      fold256_warp2([&](int L, double& x, double& y) {
        const int i = b + L;
        const float2 v = i < e ? P.cg_pair[i] : make_float2(0.0f, 0.0f);
        if (i < e) m = fmaxf(m, v.y);
        x = i < e ? (double)v.x : 0.0;
        y = i < e ? (double)v.y : 0.0;
      }, sx, sy);
      m = warp_max(m);
      bool last = false;
      if (lane == 0) {
        P.part2[c] = make_double2(sx, sy);
        P.part_max[c] = m;
        last = world_ticket(P, w, c1 - c0);
      }
      last = __shfl_sync(0xffffffffu, last, 0);
      if (last) {
        __threadfence();
        float mm = -3.4e38f;
        double wx, wy;
        fold256_warp2([&](int L, double& x, double& y) {
          x = 0.0;
          y = 0.0;
          for (int k = c0 + L; k < c1; k += 256) {
            const double2 pk = __ldcg(&P.part2[k]);
            x = x + pk.x;
            y = y + pk.y;
            mm = fmaxf(mm, __ldcg(&P.part_max[k]));
          }
        }, wx, wy);
        const float mx = warp_max(mm);
        if (lane == 0) {
          P.cg_sums[w] = make_double2(wx, wy);
          if (with_max) P.emax[w] = maxr(mx, 0.0f);
          if (beta) cg_beta_world(P, w);
        }
      }
      ticket = last ? 1 : 0;
    }
  }
  if (!beta) return;  // the same for every thread of the launch
  if (lane == 0) tickets[wq] = ticket;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < CHECK_WARPS; ++k) t += tickets[k];
    glast = false;
    if (t > 0) {
      __threadfence();
      const unsigned before = atomicAdd(P.gdone, (unsigned)t);
      glast = before + (unsigned)t == (unsigned)P.n_chunk_worlds;
      if (glast) *P.gdone = 0u;
    }
  }
  __syncthreads();
  if (glast) {
    __threadfence();
    int open = 0;
    for (int k = threadIdx.x; k < P.W; k += blockDim.x) open += __ldcg(&P.converged[k]) ? 0 : 1;
    int tot;
    block_exclusive_scan(open, smi, tot);
    if (threadIdx.x == 0) *P.n_unconv = tot;
  }
}

__global__ void __launch_bounds__(32 * CHECK_WARPS) k_sums2_warps(DevP P, int with_max, int beta) {
  sums2_warps_at(P, with_max, beta, blockIdx.x);
}

// ---------------------------------------------------------------------------------------- apply pressure
// pressure.py:393-414 (lone particles: a push limited like a rigid contact's depenetration) and 461-480
// (v += dt a, warm start stored dt-free). A lone particle has no neighbours, so no other particle reads its kappa.
template <int NBX>
__global__ void __launch_bounds__(BLOCK) k_apply(DevP P) {
  constexpr bool MS = (NBX & MS_FLAG) != 0;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const float dt = P.dt;
  float4 vi = P.vel[p];
  float kap = P.kappa[p];
  const bool lone = P.cnt[p] == 0 && kap > 0.0f && slot_count(P, p) > 0;
  // the walls' summed gradient, the Psi-weighted wall velocity, the Psi sum and the largest-Psi slot
  float Gx = 0.0f, Gy = 0.0f, Gz = 0.0f, vbx = 0.0f, vby = 0.0f, vbz = 0.0f, ps = 0.0f, pbest = 0.0f;
  int best = -1;
  if (lone) {
    for_slots<MS>(P, p, [&](int b, size_t o) {
      const float4 sg = P.slot_g[o], vbs = P.slot_vb[o];
      Gx = Gx + sg.x;
      Gy = Gy + sg.y;
      Gz = Gz + sg.z;
      vbx = ADF_FMA(sg.w, vbs.x, vbx);
      vby = ADF_FMA(sg.w, vbs.y, vby);
      vbz = ADF_FMA(sg.w, vbs.z, vbz);
      ps = ps + sg.w;
      if (sg.w > pbest) {
        pbest = sg.w;
        best = b;
      }
    });
    const float g = __fsqrt_rn(dot_plain(Gx, Gy, Gz, Gx, Gy, Gz));
    if (g > 0.0f) {
      float ux = vbx, uy = vby, uz = vbz;
      if (ps > 0.0f) {
        ux = ux / ps;
        uy = uy / ps;
        uz = uz / ps;
      }
      const float nx = -Gx / g, ny = -Gy / g, nz = -Gz / g;
      const float u = dotf(vi.x - ux, vi.y - uy, vi.z - uz, nx, ny, nz);
      kap = minr(kap, maxr(P.v_sep - u, 0.0f) / (dt * g));
      P.kappa[p] = kap;
      P.kr[p] = kap / vi.w;
    }
  }
  float ax, ay, az;
  pressure_accel<NBX>(P, p, P.pos[p], ax, ay, az);
  P.acc[p] = make_float4(ax, ay, az, 0.0f);
  float vx = ADF_FMA(dt, ax, vi.x), vy = ADF_FMA(dt, ay, vi.y), vz = ADF_FMA(dt, az, vi.z);
  // pressure.py:417-458: Coulomb friction of a lone particle on its walls after the update: the walls' push
  // dv_n = dt k |G| takes up to mu dv_n of its tangential speed relative to them, never reversing it; mu is that of
  // the wall in its largest-Psi slot (a particle wall has none)
  if (MS && lone && P.wall_friction && P.n_shapes > 0 && kap > 0.0f && best >= 0) {  // box walls only
    const float g = __fsqrt_rn(dot_plain(Gx, Gy, Gz, Gx, Gy, Gz));
    const int sh = P.slot_cap > 1 ? __float_as_int(P.slot_n[slot_at(P, best, p)].w) : P.n_shapes;
    if (g > 0.0f && ps > 0.0f && sh >= 0 && sh < P.n_shapes && P.sh_half[sh].w > 0.0f) {
      const float mu = P.sh_half[sh].w;
      const float nx = -Gx / g, ny = -Gy / g, nz = -Gz / g;
      const float ux = vx - vbx / ps, uy = vy - vby / ps, uz = vz - vbz / ps;
      const float un = dotf(ux, uy, uz, nx, ny, nz);
      const float tx = ADF_FMA(-un, nx, ux), ty = ADF_FMA(-un, ny, uy), tz = ADF_FMA(-un, nz, uz);
      const float lt = __fsqrt_rn(dot_plain(tx, ty, tz, tx, ty, tz));
      if (lt > 0.0f) {
        const float f = minr(1.0f, (((mu * dt) * kap) * g) / lt);
        vx = ADF_FMA(-f, tx, vx);
        vy = ADF_FMA(-f, ty, vy);
        vz = ADF_FMA(-f, tz, vz);
      }
    }
  }
  P.vel[p] = make_float4(vx, vy, vz, vi.w);
  if (P.mode == 0) P.kv_s[p] = kap * dt;
  else P.kd_s[p] = (kap * dt) * dt;
}

// ----------------------------------------------------------------------------------------- non-pressure
// integrate.py:150-178: gravity, external force, XSPH with Monaghan's symmetric weight m_j / rho_bar_ij.
// The output array becomes the velocity array for the rest of the step (the host swaps them), so boundary
// particles carry their own velocity across: the wall advance in k_finish reads it.
template <int NBX>
__global__ void __launch_bounds__(BLOCK, 3) k_xsph(DevP P) {
  constexpr int NB = NBX & NB_MASK;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = P.nfw[0];
  if (p >= nf) {
    if (p < nf + P.nfw[1]) P.vel2[p] = P.vel[p];
    return;
  }
  const float dt = P.dt;
  float4 vi = P.vel[p];
  int w = P.world_s[p];
  float gx = P.gravity[3 * w], gy = P.gravity[3 * w + 1], gz = P.gravity[3 * w + 2];
  float4 xi = P.pos[p];
  if (P.f_ext) {
    int i = P.id_of[p];
    gx = gx + P.f_ext[3 * i] / xi.w;
    gy = gy + P.f_ext[3 * i + 1] / xi.w;
    gz = gz + P.f_ext[3 * i + 2] / xi.w;
  }
  float vx = ADF_FMA(dt, gx, vi.x), vy = ADF_FMA(dt, gy, vi.y), vz = ADF_FMA(dt, gz, vi.z);
  const float c = P.xsph_c;
  if (c > 0.0f) {
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    float rho_i = P.ratio[p] * vi.w;
    int cn = P.cnt[p];
    for (int k = 0; k < cn; k += NB) {
      int j[NB];
      float wb[NB];
      load_row_batch(P, p, cn, k, j);
#pragma unroll
      for (int u = 0; u < NB; ++u) wb[u] = (k + u < cn) ? __ldcs(P.nbrw + (size_t)(k + u) * P.n + p) : 0.0f;
      float4 vb[NB];
      float rb[NB], mb[NB];
#pragma unroll
      for (int u = 0; u < NB; ++u) {
        vb[u] = P.vel[j[u]];
        rb[u] = P.ratio[j[u]];
        mb[u] = reinterpret_cast<const float*>(P.pos)[4 * (size_t)j[u] + 3];  // mass (pos.w) only
      }
#pragma unroll
      for (int u = 0; u < NB; ++u) {
        if (k + u >= cn) break;
        float4 vj = vb[u];
        float rho_bar = 0.5f * (rho_i + rb[u] * vj.w);
        if (rho_bar > 0.0f) {
          float cw = (mb[u] / rho_bar) * wb[u];  // W(r_ij) as k_density_alpha evaluated it for this entry
          cx = ADF_FMA(cw, vj.x - vi.x, cx);
          cy = ADF_FMA(cw, vj.y - vi.y, cy);
          cz = ADF_FMA(cw, vj.z - vi.z, cz);
        }
      }
    }
    vx = ADF_FMA(c, cx, vx);
    vy = ADF_FMA(c, cy, vy);
    vz = ADF_FMA(c, cz, vz);
  }
  P.vel2[p] = make_float4(vx, vy, vz, vi.w);
}

// ------------------------------------------------------------------------------------------------ finish
// integrate.py:181-185 advection, particle_walls.py:131-135 wall advance, integrate.py:212-309 sweep and projection
// (finish_walls with box walls; else out of the particle wall's advected slot plane), emitters.py:134-164 sinks and
// escape box, integrate.py:312-326 speed; results written back to the caller's order.
__device__ __forceinline__ bool in_box(const Sink& s, float x, float y, float z) {
  float inv[4] = {-s.xform[3], -s.xform[4], -s.xform[5], s.xform[6]};
  float lx, ly, lz;
  quat_rotate(inv, x - s.xform[0], y - s.xform[1], z - s.xform[2], lx, ly, lz);
  return fabsf(lx) <= s.half[0] && fabsf(ly) <= s.half[1] && fabsf(lz) <= s.half[2];
}

// integrate.py:212-309 with box walls: a liquid particle that moved further than the sweep length is swept along its
// path against its world's boxes (the first box entered, the particle put on its surface plus the skin, the inward
// speed removed with friction); then its slots' walls push it out in up to PROJECT_PASSES passes: the particle wall
// onto its start plane advanced with the wall, a box through its SDF at the new place, onto its start-of-step tangent
// plane when that holds it.
__device__ __forceinline__ void finish_walls(const DevP& P, int p, int w, float dt, float& x, float& y, float& z,
                                             float& vx, float& vy, float& vz) {
  int moved = 0;
  const int c0 = P.sh_start[w], c1 = P.sh_start[w + 1];
  const float stx = dt * vx, sty = dt * vy, stz = dt * vz;
  if (c1 > c0 && __fsqrt_rn(dot_plain(stx, sty, stz, stx, sty, stz)) > P.sweep_len) {
    const float x0 = x - stx, y0 = y - sty, z0 = z - stz;
    const float spx = x - x0, spy = y - y0, spz = z - z0;
    const float len = __fsqrt_rn(dot_plain(spx, spy, spz, spx, spy, spz));
    const float reach = len + P.prad;
    // integrate.py:56-58: samples of a path against a shape other than a box, one per particle radius, 8 to 64
    const int samples = min(max((int)ceilf(len / P.prad) + 1, 8), SWEEP_SAMPLES);
    float best = 2.0f, lhx = 0.0f, lhy = 0.0f, lhz = 0.0f;
    int hit = -1;
    for (int c = c0; c < c1; ++c) {
      const int sh = P.sh_ids[c];
      const float4 cp = P.sh_pos[sh];
      const int geo = P.sh_geo[sh];
      float ox = x0 - cp.x, oy = y0 - cp.y, oz = z0 - cp.z;
      if (geo != GEO_PLANE && !(__fsqrt_rn(dot_plain(ox, oy, oz, ox, oy, oz)) <= cp.w + reach)) continue;
      float ex = x - cp.x, ey = y - cp.y, ez = z - cp.z;
      const float4 q = P.sh_quat[sh];
      to_frame(q, ox, oy, oz);
      to_frame(q, ex, ey, ez);
      const float t = shape_entry(geo, P.sh_half[sh], ox, oy, oz, ex, ey, ez, samples);
      if (t < best) {
        best = t;
        hit = sh;
        lhx = ADF_FMA(t, ex - ox, ox);
        lhy = ADF_FMA(t, ey - oy, oy);
        lhz = ADF_FMA(t, ez - oz, oz);
      }
    }
    if (hit >= 0) {
      const float4 cp = P.sh_pos[hit], hx = P.sh_half[hit];
      const int geo = P.sh_geo[hit];
      const float4 q = P.sh_quat[hit];
      const float phi = shape_phi(geo, hx, lhx, lhy, lhz);
      float nx, ny, nz;
      shape_normal(geo, hx, lhx, lhy, lhz, nx, ny, nz);
      from_frame(q, nx, ny, nz);
      from_frame(q, lhx, lhy, lhz);  // the entry point, world-oriented about the shape's origin
      const float push = maxr(P.eps - phi, 0.0f);
      x = ADF_FMA(push, nx, lhx + cp.x);
      y = ADF_FMA(push, ny, lhy + cp.y);
      z = ADF_FMA(push, nz, lhz + cp.z);
      const float vn = dotf(vx, vy, vz, nx, ny, nz);
      if (vn < 0.0f) {
        vx = ADF_FMA(-vn, nx, vx);
        vy = ADF_FMA(-vn, ny, vy);
        vz = ADF_FMA(-vn, nz, vz);
        wall_friction(P, vx, vy, vz, 0.0f, 0.0f, 0.0f, nx, ny, nz, vn, hit);
      }
      moved = 1;
      atomicAdd(&P.swept[w], 1);
    }
  }
  const int ns = slot_count(P, p);
  int busy = 1;
  for (int pass = 0; pass < PROJECT_PASSES && busy; ++pass) {
    busy = 0;
    for (int b = 0; b < ns; ++b) {
      const size_t o = slot_at(P, b, p);
      const float4 nn = P.slot_n[o], vb = P.slot_vb[o], xb = P.slot_xb[o];
      const int sh = __float_as_int(nn.w);
      if (sh == P.n_shapes) {  // the particle wall's plane at its end-of-step place
        const float px = ADF_FMA(dt, vb.x, xb.x), py = ADF_FMA(dt, vb.y, xb.y), pz = ADF_FMA(dt, vb.z, xb.z);
        const float d = dotf(x - px, y - py, z - pz, nn.x, nn.y, nn.z);
        if (d < P.eps) {
          const float push = P.eps - d;
          x = ADF_FMA(push, nn.x, x);
          y = ADF_FMA(push, nn.y, y);
          z = ADF_FMA(push, nn.z, z);
          const float vn = dotf(vx - vb.x, vy - vb.y, vz - vb.z, nn.x, nn.y, nn.z);
          if (vn < 0.0f) {
            vx = ADF_FMA(-vn, nn.x, vx);
            vy = ADF_FMA(-vn, nn.y, vy);
            vz = ADF_FMA(-vn, nn.z, vz);
          }
          moved = busy = 1;
        }
      } else if (sh >= 0) {  // a static shape: its SDF at the new place, its start plane when that holds it
        const float4 cp = P.sh_pos[sh], hx = P.sh_half[sh];
        const int geo = P.sh_geo[sh];
        const float4 q = P.sh_quat[sh];
        float lx = x - cp.x, ly = y - cp.y, lz = z - cp.z;
        to_frame(q, lx, ly, lz);
        const float phi = shape_phi(geo, hx, lx, ly, lz);
        if (phi < P.eps) {
          float nx, ny, nz;
          shape_normal(geo, hx, lx, ly, lz, nx, ny, nz);
          from_frame(q, nx, ny, nz);
          float push = P.eps - phi;
          if (vb.w >= 0.0f) {
            const float push_s = P.eps - dotf(nn.x, nn.y, nn.z, x - (xb.x + cp.x), y - (xb.y + cp.y), z - (xb.z + cp.z));
            if (push_s > 0.0f) {
              nx = nn.x;
              ny = nn.y;
              nz = nn.z;
              push = push_s;
            }
          }
          if (push > 0.0f) {
            x = ADF_FMA(push, nx, x);
            y = ADF_FMA(push, ny, y);
            z = ADF_FMA(push, nz, z);
            const float vn = dotf(vx, vy, vz, nx, ny, nz);
            if (vn < 0.0f) {
              vx = ADF_FMA(-vn, nx, vx);
              vy = ADF_FMA(-vn, ny, vy);
              vz = ADF_FMA(-vn, nz, vz);
              wall_friction(P, vx, vy, vz, 0.0f, 0.0f, 0.0f, nx, ny, nz, vn, sh);
            }
            moved = busy = 1;
          }
        }
      }
    }
  }
  if (moved) atomicAdd(&P.projected[w], 1);
}

template <bool MS>
__global__ void __launch_bounds__(BLOCK) k_finish(DevP P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int nf = P.nfw[0];
  if (p >= nf + P.nfw[1]) return;
  const float dt = P.dt;
  int i = P.id_of[p];
  float4 xi = P.pos[p];
  float4 vi = P.vel[p];
  float x = ADF_FMA(dt, vi.x, xi.x), y = ADF_FMA(dt, vi.y, xi.y), z = ADF_FMA(dt, vi.z, xi.z);
  if (p >= nf) {  // wall particle
    P.q[3 * i] = x;
    P.q[3 * i + 1] = y;
    P.q[3 * i + 2] = z;
    return;
  }
  int w = P.world_s[p];
  float vx = vi.x, vy = vi.y, vz = vi.z;
  if constexpr (MS) {
    finish_walls(P, p, w, dt, x, y, z, vx, vy, vz);
  } else if (P.slot_g[p].w >= 0.0f) {
    float4 nn = P.slot_n[p], vb = P.slot_vb[p], xb = P.slot_xb[p];
    float px = ADF_FMA(dt, vb.x, xb.x), py = ADF_FMA(dt, vb.y, xb.y), pz = ADF_FMA(dt, vb.z, xb.z);
    int moved = 0;
    for (int pass = 0; pass < PROJECT_PASSES; ++pass) {
      float d = dotf(x - px, y - py, z - pz, nn.x, nn.y, nn.z);
      if (!(d < P.eps)) break;
      float push = P.eps - d;
      x = ADF_FMA(push, nn.x, x);
      y = ADF_FMA(push, nn.y, y);
      z = ADF_FMA(push, nn.z, z);
      float vn = dotf(vx - vb.x, vy - vb.y, vz - vb.z, nn.x, nn.y, nn.z);
      if (vn < 0.0f) {
        vx = ADF_FMA(-vn, nn.x, vx);
        vy = ADF_FMA(-vn, nn.y, vy);
        vz = ADF_FMA(-vn, nn.z, vz);
      }
      moved = 1;
    }
    if (moved) atomicAdd(&P.projected[w], 1);
  }
  int gone = 0;
  for (int s = 0; s < P.n_sinks; ++s)
    if (P.sinks[s].world == w && in_box(P.sinks[s], x, y, z)) gone = 1;
  if (P.has_bounds && gone == 0) {
    bool out = x < P.blo[0] || y < P.blo[1] || z < P.blo[2] || x > P.bhi[0] || y > P.bhi[1] || z > P.bhi[2];
    if (out || !isfinite((x + y) + z)) {
      gone = 2;
      atomicAdd(&P.escaped[w], 1);
    }
  }
  int speed_bits = 0;  // float bits of a non-negative speed (their integer order is the float order)
  if (gone) {
    P.flags[i] = P.flags[i] & ~FLAG_ACTIVE;
    P.phase[i] = (int8_t)-2;
    vx = vy = vz = 0.0f;
    atomicAdd((unsigned long long*)&P.mass_out[w], (unsigned long long)to_fixed(P.mass[i]));
  } else {
    float sp = __fsqrt_rn(dotf(vx, vy, vz, vx, vy, vz));
    if (isfinite(sp) && isfinite((x + y) + z)) speed_bits = __float_as_int(sp);
    else {
      atomicAdd(&P.nonfinite[w], 1);
      speed_bits = __float_as_int(1.0e30f);
    }
  }
  // per-world maximum: one atomic per warp when the warp's liquid lanes share a world (sorted storage groups worlds)
  const unsigned lanes = __activemask();
  const int w0 = __shfl_sync(lanes, w, __ffs(lanes) - 1);
  if (__all_sync(lanes, w == w0)) {
    unsigned m = __reduce_max_sync(lanes, (unsigned)speed_bits);
    if ((threadIdx.x & 31) == __ffs(lanes) - 1 && m) atomicMax(&P.max_speed_bits[w0], (int)m);
  } else if (speed_bits) {
    atomicMax(&P.max_speed_bits[w], speed_bits);
  }
  P.q[3 * i] = x;
  P.q[3 * i + 1] = y;
  P.q[3 * i + 2] = z;
  P.qd[3 * i] = vx;
  P.qd[3 * i + 1] = vy;
  P.qd[3 * i + 2] = vz;
  P.kv[i] = P.kv_s[p];
  P.kd[i] = P.kd_s[p];
}

// ---------------------------------------------------------------------------------------------- emitters
// emitters.py:67-126: per emitter a layer clock; each due layer places its particles (spares of the emitter's
// pool, in pool order) at the region's lattice offsets with the emitter's velocity; the cursor then advances.
__global__ void k_emit_clock(const Emit* em, int n_e, float dt, const int* enabled, float* t_acc, int* emit_now) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_e) return;
  emit_now[e] = 0;
  if (enabled[e] == 0) return;
  float t = t_acc[e] + dt;
  if (t >= em[e].interval) {
    t -= em[e].interval;
    emit_now[e] = 1;
  }
  t_acc[e] = t;
}

__global__ void k_emit(DevP P, const Emit* em, int n_off, const int* off_emitter, const int* off_rank,
                       const float* off_local, const int* emit_now, const int* cursor, const int* pool_ids,
                       long long* mass_in, int* emit_overflow) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_off) return;
  int e = off_emitter[c];
  if (emit_now[e] == 0) return;
  const Emit E = em[e];
  int slot = cursor[e] + off_rank[c];
  int w = E.world;
  if (slot >= E.pool_size) {
    atomicAdd(&emit_overflow[w], 1);
    return;
  }
  int i = pool_ids[E.pool_begin + slot];
  float rx, ry, rz;
  quat_rotate(E.xform + 3, off_local[3 * c], off_local[3 * c + 1], off_local[3 * c + 2], rx, ry, rz);
  float x = rx + E.xform[0], y = ry + E.xform[1], z = rz + E.xform[2];
  P.q[3 * i] = x;
  P.q[3 * i + 1] = y;
  P.q[3 * i + 2] = z;
  P.qd[3 * i] = E.vel[0];
  P.qd[3 * i + 1] = E.vel[1];
  P.qd[3 * i + 2] = E.vel[2];
  P.flags[i] = P.flags[i] | FLAG_ACTIVE;
  P.phase[i] = (int8_t)1;
  atomicAdd((unsigned long long*)&mass_in[w], (unsigned long long)to_fixed(P.mass[i]));
  float sp = __fsqrt_rn(dotf(E.vel[0], E.vel[1], E.vel[2], E.vel[0], E.vel[1], E.vel[2]));
  if (isfinite(sp) && isfinite((x + y) + z)) atomicMax(&P.max_speed_bits[w], __float_as_int(sp));
  else {
    atomicAdd(&P.nonfinite[w], 1);
    atomicMax(&P.max_speed_bits[w], __float_as_int(1.0e30f));
  }
}

__global__ void k_emit_cursor(const Emit* em, int n_e, const int* emit_now, int* cursor) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_e) return;
  if (emit_now[e] != 0) cursor[e] = min(cursor[e] + em[e].n_layer, em[e].pool_size);
}

// prime.py:80-85: the solved divergence warm starts back in the caller's order, then kd = kv dt and kv = 0 for every
// particle (the density solve of the first step starts from the hydrostatic pressure).
__global__ void k_prime_gather(DevP P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  P.kv[P.id_of[p]] = P.kv_s[p];
}

__global__ void k_prime_store(int n, float dt, float* kv, float* kd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  kd[i] = kv[i] * dt;
  kv[i] = 0.0f;
}

// ------------------------------------------------------------------------------------------------- misc
__global__ void k_wall_volume(int n, const int32_t* flags, const float* radius, float* wall_vol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float r = radius[i];
  wall_vol[i] = (flags[i] & FLAG_PROXY) ? (float)(8.0 * (double)r * (double)r * (double)r) : 0.0f;
}

// Exact int64 sum per world; a warp whose particles all belong to one world adds its shuffle-reduced total with one
// atomic (integer addition, so the order does not matter).
__global__ void k_active_mass(DevP P, long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int w = -1;
  long long v = 0;
  if (i < P.n) {
    w = P.world[i];
    if (w < 0 || w >= P.W || !is_fluid_orig(P, i)) w = -1;
    else v = to_fixed(P.mass[i]);
  }
  const unsigned full = 0xffffffffu;
  const int w0 = __shfl_sync(full, w, 0);
  if (__all_sync(full, w == w0)) {
    if (w0 < 0) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)&out[w0], (unsigned long long)v);
  } else if (w >= 0) {
    atomicAdd((unsigned long long*)&out[w], (unsigned long long)v);
  }
}

__global__ void k_unsort_n(int n, const int* nfw, const int* id_of, const float* f, int stride, int comp, float* out,
                           int ncomp) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || p >= nfw[0]) return;
  int i = id_of[p];
  for (int c = 0; c < ncomp; ++c) out[ncomp * i + c] = f[(size_t)stride * p + comp + c];
}

__global__ void k_fill_ones(int n, const int* nfw, const int* id_of, float* out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || p >= nfw[0]) return;
  out[id_of[p]] = 1.0f;
}

__global__ void k_count_entries(int n, const int* nfw, const int* cnt, long long* out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int c = (p < n && p < nfw[0]) ? cnt[p] : 0;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd((unsigned long long*)out, (unsigned long long)c);
}

// Diagnostics: slot k's wall id (-1 empty; the particle wall's id is n_shapes) or, with k < 0, the number of slots in
// use, of each liquid particle, written as floats at its caller index.
__global__ void k_slot_info(DevP P, int k, float* out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.nfw[0]) return;
  const int ns = slot_count(P, p);
  int v = ns;
  if (k >= 0) v = k >= ns ? -1 : (P.slot_cap > 1 ? __float_as_int(P.slot_n[slot_at(P, k, p)].w) : P.n_shapes);
  out[P.id_of[p]] = (float)v;
}

__global__ void k_reset(DevP P, const uint8_t* mask, const int32_t* flags0, const int8_t* phase0) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  int w = P.world[i];
  if (w >= 0 && w < P.W && mask[w]) {
    P.kv[i] = 0.0f;
    P.kd[i] = 0.0f;
    P.flags[i] = flags0[i];
    P.phase[i] = phase0[i];
  }
}

}  // namespace adf
