// SPDX-License-Identifier: Apache-2.0
// C ABI of the B200 DFSPH step (include/alloy_dfsph.h): the solver object, its fixed-capacity device memory and the
// per-step launch sequence (solver.py:218-268 order). Pressure solves run their iterations with a one-ahead host
// check: iteration k+1 is enqueued before the host reads iteration k's unconverged-world count, so the GPU never
// idles on the read; an iteration enqueued after every world converged changes nothing (converged worlds skip every
// kernel, pressure.py:289-290, 326-327).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/alloy_dfsph.h"
#include "dfsph_kernels.cuh"
#include "dfsph_mlp.cuh"
#include "dfsph_persist.cuh"
#include "dfsph_port.cuh"
#include "dfsph_skin.cuh"

using namespace adf;

namespace adf {
// The warm-start network over the liquid particles of a step: raw features from k_solve_init, predictions (kappa dt,
// kappa dt^2) into pred_kv / pred_kd, all in sorted order.
struct WarmSrc {
  const float* feat;
  float* pred_kv;
  float* pred_kd;
  int n;
  const int* world_s;  // world of each sorted liquid particle
  const int* need;     // [W] worlds that need predictions this step (null: all)
  __device__ int rows() const { return n; }
  // a tile of sorted particles [r0, r1) spans worlds world_s[r0] .. world_s[r1 - 1] (worlds are contiguous)
  __device__ bool skip_tile(int r0, int r1) const {
    if (!need || r1 <= r0) return false;
    for (int w = world_s[r0]; w <= world_s[r1 - 1]; ++w)
      if (need[w]) return false;
    return true;
  }
  __device__ void features(int row, float (&f)[16]) const {
    const float4* p = reinterpret_cast<const float4*>(feat + (size_t)row * 16);
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
    pred_kv[row] = y0;
    pred_kd[row] = y1;
  }
};

__global__ void __launch_bounds__(mlp::TILE) k_mlp_warm(DevP P, mlp::Net net) {
  WarmSrc s{P.feat, P.pred_kv, P.pred_kd, P.nfw[0], P.world_s, P.warm_need};
  mlp::forward_rows(net, s);
}

// Kernels the autotuner configures (k_apply runs the acceleration loop and takes TK_ACCEL's choice), and the choices:
// threads per block and the neighbour gathers each thread keeps in flight (NB).
// For the list build the "gathers" field holds the particles per warp (32 or 16) and the block is fixed.
enum TuneKernel { TK_DENSITY = 0, TK_SOLVE_INIT, TK_ACCEL, TK_JACOBI, TK_XSPH, TK_LISTS, TK_COUNT };
struct TuneCfg {
  int block = BLOCK;
  int nb = NB_DEFAULT;
  int halo = 0;  // acceleration and Jacobi: 1 = the item-halo kernels (k_accel_h, k_jacobi_h)
};
constexpr int TUNE_BLOCKS[] = {128, 256};
constexpr int TUNE_NB[] = {4, 8, 16};
constexpr TuneCfg LISTS_DEFAULT{32 * LU_WARPS, 32};
constexpr int TUNE_PPW[] = {32, 16};
inline TuneCfg default_cfg(int id) { return id == TK_LISTS ? LISTS_DEFAULT : TuneCfg{}; }
}  // namespace adf

namespace {
thread_local std::string g_err;
}

namespace adf {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace adf

namespace {

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(x)                                                                               \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) return fail(ADF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CK_NEG(x)                                                                           \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) return -fail(ADF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

inline int blocks(long long n, int b = BLOCK) { return (int)((n + b - 1) / b); }

// Models up to this many particles take the CG products by teams of TL lanes per particle: below it one lane per
// particle fills less than a wave or two of the GPU (148 SMs x 2048 threads) and each lane's row is a chain of gathers.
constexpr int CG_TEAM_MAX = 131072;

template <class T> int dalloc(T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) return fail(ADF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return ADF_OK;
}
}  // namespace

struct adf_solver {
  adf_params prm;
  int n = 0, W = 0, K = 64, device = 0;
  std::vector<int> ws_host;
  std::vector<WorldGrid> grids;
  std::vector<int> world_cells_h;
  int total_cells = 0, n_keys = 0, n_tiles = 0;
  int max_items = 0;  // grid of the pressure iterations: an upper bound of their work items (k_worklist)
  int max_world_chunks = 0;  // the largest world's 256-particle chunks (chooses the stop-test kernel)
  DevP d{};
  std::vector<void*> owned;
  int* world_cells = nullptr;
  int* tile_sums = nullptr;
  // per-world statistics outside DevP
  int *iters_den = nullptr, *iters_div = nullptr, *emit_overflow = nullptr;
  float *den_err = nullptr, *div_err = nullptr, *den_err_max = nullptr, *den_tol = nullptr;
  long long *mass_in = nullptr, *mass0 = nullptr, *tmp_mass = nullptr;
  uint8_t* mask_d = nullptr;
  // emitters and sinks
  std::vector<Emit> em_h;
  std::vector<float> off_local_h;
  std::vector<int> off_emitter_h, off_rank_h, pool_h;
  std::vector<int> enabled_h;
  Emit* em_d = nullptr;
  float* off_local_d = nullptr;
  int *off_emitter_d = nullptr, *off_rank_d = nullptr, *pool_d = nullptr, *enabled_d = nullptr;
  int *cursor_d = nullptr, *emit_now_d = nullptr;
  float* t_acc_d = nullptr;
  int* em_world_d = nullptr;  // [E] world of each emitter (the snapshot keys' item -> world map)
  std::vector<Sink> sinks_h;
  Sink* sinks_d = nullptr;
  // the port (ports.py): world w's held particles are a stack in its own index range [ws[w], ws[w + 1])
  int* ws_d = nullptr;  // [W + 1] world starts
  int *port_stack = nullptr, *port_stack0 = nullptr, *port_top = nullptr, *port_top0 = nullptr;
  int *port_taken = nullptr, *port_granted = nullptr, *port_absorbed = nullptr, *port_emitted = nullptr;
  int* port_retired = nullptr;
  // patch emitters (patch.py): every registration's entries in one table (an entry = one world of one group)
  std::vector<int> pe_world_h, pe_count_h, pe_begin_h, pe_group_h, pg_first_h{0}, pp_pool_h;
  std::vector<float> pp_points_h, pg_vel_h;
  int *pe_world_d = nullptr, *pe_count_d = nullptr, *pe_begin_d = nullptr, *pe_group_d = nullptr;
  int *pe_pending_d = nullptr, *pe_fired_d = nullptr, *pp_pool_d = nullptr;
  float *pp_points_d = nullptr, *pg_vel_d = nullptr;
  // scratch of the between-step calls (adf_energy, adf_stable_dt)
  float* energy_max = nullptr;
  int *cw2 = nullptr, *cseg2 = nullptr, *n_cw2 = nullptr;  // work list of the learned start's first sweep
  int* warm_need = nullptr;  // [W] worlds that evaluate the learned start in this step (k_warm_need)
  int* speed_bits = nullptr;
  // host side of the iteration loop
  int* pinned = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  long long launches = 0;
  bool built = false;  // a step or density_ratio ran (lists exist)
  // live kernel timing (adf_profile_enable)
  bool prof_on = false;
  std::vector<cudaEvent_t> prof_pool;
  std::vector<std::pair<int, int>> prof_marks;  // (kind, first event of the pair)
  size_t prof_used = 0;
  int prof_open = -1;
  long long* list_entries = nullptr;
  // CUDA graphs of whole steps (one per state-pointer set and dt), rebuilt when the emitter or sink tables change
  struct GraphEntry {
    const void* key[5];
    double dt;
    unsigned version;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs;
  unsigned table_version = 0;
  bool use_graphs = true;
  long long graph_kernels = 0;  // kernels a step graph launches outside its WHILE bodies
  long long body_kernels = 0;   // kernels of one WHILE-body iteration
  unsigned long long* body_runs = nullptr;  // device [2]: WHILE-body iterations run so far, those of the running loop
  cudaStream_t cap_stream = nullptr, body_stream = nullptr;
  // learned warm start (adf_set_warm_model) and feature recording (adf_set_feature_recording)
  bool warm_on = false, feat_rec = false, warm_alloc = false, judge = true;
  bool cg = false;  // projected preconditioned CG pressure solve (adf_params.cg)
  bool cg_team = false;  // CG products by teams of TL lanes per particle (models of at most CG_TEAM_MAX particles)
  // the persistent CG solve (k_cg_solve) of team-product models, when adf_set_persistent turned it on
  bool persist_on = false;
  // item halos of the pressure iterations (adf_set_halo): -1 the tuner times both forms, 0 off (the default), 1 always
  int halo_mode = 0;
  int halo_items = 0;  // item numbers k_halo covers: n / 256 + W + 1
  int persist_cap[2] = {0, 0};       // co-resident blocks of k_cg_solve<false/true> on this device
  unsigned persist_extra = 0;        // extra arrivals a barrier waits for (only the wait-expiry test sets it)
  long long persist_wait = 1 << 22;  // polls of one barrier wait (about a second) before it gives up
  unsigned* parrive = nullptr;       // device [1]: barrier arrivals of the running launch
  int* perr = nullptr;               // device [1]: a barrier wait gave up
  // the resting-jitter rule (adf_params.jitter_speed > 0): per-world tolerance factor and its float64 sums
  float* jit_scale = nullptr;                 // [W]
  double *jit_part = nullptr, *jit_flow = nullptr, *jit_head = nullptr;  // [chunks][4], [W][4], [W][4]
  __nv_bfloat16 *mw1 = nullptr, *mw2 = nullptr;
  float *mparams = nullptr, *mnorm = nullptr;
  int* merr = nullptr;
  int mlp_grid = 1;
  // autotuner: block size and gathers in flight per neighbour-loop kernel (adf_set_autotune)
  adf::TuneCfg tune[adf::TK_COUNT];
  float tune_ms[adf::TK_COUNT] = {};
  bool tuned[adf::TK_COUNT] = {};
  bool tune_pending = true, tuning = false;
  float *snap_kappa = nullptr, *snap_kr = nullptr, *snap_err = nullptr;
  int* snap_ovf = nullptr;
  cudaEvent_t tev[2] = {nullptr, nullptr};

  template <class T> int alloc(T** p, size_t count) {
    int rc = dalloc(p, count);
    if (rc == ADF_OK) owned.push_back((void*)*p);
    return rc;
  }
};

namespace {

#define LAUNCH(s, kern, grid, block, stream, ...)          \
  do {                                                     \
    kern<<<(grid), (block), 0, (cudaStream_t)(stream)>>>(__VA_ARGS__); \
    ++(s)->launches;                                       \
  } while (0)

void prof_begin(adf_solver* s, int kind, cudaStream_t st) {
  if (!s->prof_on || s->prof_used + 2 > s->prof_pool.size()) return;
  int e = (int)s->prof_used;
  s->prof_used += 2;
  cudaEventRecord(s->prof_pool[e], st);
  s->prof_marks.push_back({kind, e});
  s->prof_open = e;
}

void prof_end(adf_solver* s, cudaStream_t st) {
  if (s->prof_open < 0) return;
  cudaEventRecord(s->prof_pool[s->prof_open + 1], st);
  s->prof_open = -1;
}

// A neighbour-loop kernel's instance: gathers in flight nb, with MS_FLAG when the model has box walls (solver s in scope)
#define NB_DISPATCH_SM(kern, nb, grid, block, smem, st, ...)                                          \
  do {                                                                                                \
    switch ((nb) | (s->d.slot_cap > 1 ? MS_FLAG : 0)) {                                               \
      case 4: kern<4><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;                           \
      case 16: kern<16><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;                         \
      case 4 | MS_FLAG: kern<4 | MS_FLAG><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;         \
      case 8 | MS_FLAG: kern<8 | MS_FLAG><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;         \
      case 16 | MS_FLAG: kern<16 | MS_FLAG><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;       \
      default: kern<8><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__); break;                          \
    }                                                                                                 \
  } while (0)
#define NB_DISPATCH(kern, nb, grid, block, st, ...) NB_DISPATCH_SM(kern, nb, grid, block, 0, st, __VA_ARGS__)

// A team kernel's instance (box walls or not)
#define MS_DISPATCH(kern, grid, block, st, ...)                                                  \
  do {                                                                                           \
    if (s->d.slot_cap > 1) kern<true><<<(grid), (block), 0, (st)>>>(__VA_ARGS__);                \
    else kern<false><<<(grid), (block), 0, (st)>>>(__VA_ARGS__);                                \
  } while (0)

// One launch of a tuned kernel with configuration c (the pressure iterations' grid is the work-item bound, each block
// covering one 256-particle item whatever its size; the others one particle per thread).
void launch_tk(adf_solver* s, int id, const TuneCfg& c, cudaStream_t st, const DevP& P) {
  const int n = s->n;
  switch (id) {
    case TK_DENSITY: NB_DISPATCH(k_density_alpha, c.nb, blocks(n, c.block), c.block, st, P); break;
    case TK_SOLVE_INIT: NB_DISPATCH(k_solve_init, c.nb, blocks(n, c.block), c.block, st, P); break;
    case TK_ACCEL:
      if (c.halo) NB_DISPATCH_SM(k_accel_h, c.nb, s->max_items, c.block, HALO_SMEM_ACCEL, st, P);
      else NB_DISPATCH(k_accel, c.nb, s->max_items, c.block, st, P);
      break;
    case TK_JACOBI:
      if (c.halo) NB_DISPATCH_SM(k_jacobi_h, c.nb, s->max_items, c.block, HALO_SMEM_JACOBI, st, P);
      else NB_DISPATCH(k_jacobi, c.nb, s->max_items, c.block, st, P);
      break;
    case TK_LISTS:
      if (c.nb == 16) k_lists_union<16><<<blocks(n, 16 * LU_WARPS), 32 * LU_WARPS, 0, st>>>(P);
      else k_lists_union<32><<<blocks(n, 32 * LU_WARPS), 32 * LU_WARPS, 0, st>>>(P);
      break;
    default: NB_DISPATCH(k_xsph, c.nb, blocks(n, c.block), c.block, st, P); break;
  }
  ++s->launches;
}

// Autotuning (the first step after adf_set_autotune, outside any capture): every block size x NB candidate of the
// kernel runs three times on the step's real inputs, timed with CUDA events on the launch stream, and the fastest
// is kept. The tuned kernels are idempotent on their inputs except the Jacobi update, whose kappa, kappa / rho0 and
// residual are restored before every trial and after the last, so the tuning step computes exactly an ordinary step.
void tune_kernel(adf_solver* s, int id, cudaStream_t st, const DevP& P) {
  if (!s->tuning || s->tuned[id]) return;
  const bool restore = id == TK_JACOBI || id == TK_LISTS;
  const size_t nb = sizeof(float) * (size_t)s->n;
  auto copy = [&](bool save) {
    if (!restore) return;
    if (id == TK_LISTS) {  // the rows are rewritten whole; only the overflow counters accumulate
      const size_t wb = sizeof(int) * (size_t)std::max(s->W, 1);
      if (save) cudaMemcpyAsync(s->snap_ovf, P.overflow, wb, cudaMemcpyDeviceToDevice, st);
      else cudaMemcpyAsync(P.overflow, s->snap_ovf, wb, cudaMemcpyDeviceToDevice, st);
      return;
    }
    if (save) {
      cudaMemcpyAsync(s->snap_kappa, P.kappa, nb, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(s->snap_kr, P.kr, nb, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(s->snap_err, P.err_orig, nb, cudaMemcpyDeviceToDevice, st);
    } else {
      cudaMemcpyAsync(P.kappa, s->snap_kappa, nb, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(P.kr, s->snap_kr, nb, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(P.err_orig, s->snap_err, nb, cudaMemcpyDeviceToDevice, st);
    }
  };
  copy(true);
  float best = 3.0e38f;
  TuneCfg pick = s->tune[id];
  std::vector<TuneCfg> cands;
  if (id == TK_LISTS) {
    for (int g : TUNE_PPW) cands.push_back(TuneCfg{32 * LU_WARPS, g});
  } else {
    const bool staged = id == TK_ACCEL || id == TK_JACOBI;
    for (int halo = 0; halo < 2; ++halo) {
      if (halo && !staged) continue;
      if (staged && s->halo_mode >= 0 && halo != s->halo_mode) continue;
      for (int block : TUNE_BLOCKS)
        for (int nbv : TUNE_NB) cands.push_back(TuneCfg{block, nbv, halo});
    }
  }
  {
    for (const TuneCfg& c : cands) {
      float t = 3.0e38f;
      for (int r = 0; r < 3; ++r) {
        copy(false);
        cudaEventRecord(s->tev[0], st);
        launch_tk(s, id, c, st, P);
        cudaEventRecord(s->tev[1], st);
        float ms = 0.0f;
        if (cudaEventSynchronize(s->tev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, s->tev[0], s->tev[1]) ==
            cudaSuccess)
          t = std::min(t, ms);
      }
      if (t < best) {
        best = t;
        pick = c;
      }
    }
  }
  copy(false);
  s->tune[id] = pick;
  s->tune_ms[id] = best;
  s->tuned[id] = true;
}

// Whether this step builds the item halos: always when forced on; with the tuner deciding, in the tuning step (its
// trials time both forms) and whenever the acceleration or Jacobi choice is the staged form.
bool halo_needed(const adf_solver* s) {
  if (s->halo_mode == 0) return false;
  if (s->halo_mode == 1) return true;
  return (s->tuning && !(s->tuned[TK_ACCEL] && s->tuned[TK_JACOBI])) || s->tune[TK_ACCEL].halo ||
         s->tune[TK_JACOBI].halo;
}

// A tuned kernel's launch at its place in the step (tuning it first when this is the tuning step).
void run_tk(adf_solver* s, int id, cudaStream_t st, const DevP& P) {
  tune_kernel(s, id, st, P);
  launch_tk(s, id, s->tune[id], st, P);
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return ADF_OK;
}

// Per-world cell grids over each world's start-state bounding box with a margin; cells are 1.001 h wide (every pair
// closer than h lies in adjacent cells despite float rounding of the cell coordinate) and coarser only where a
// world's box would need more than 2^25 cells. Particles outside a grid are clamped into its border cells, which
// keeps every neighbour query exact.
void size_grids(adf_solver* s, const float* q_host) {
  const double cw0 = 1.001 * s->prm.h;
  s->grids.assign(s->W, WorldGrid{});
  s->world_cells_h.assign(s->W, 0);
  long long base = 0;
  for (int w = 0; w < s->W; ++w) {
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool any = false;
    for (int i = s->ws_host[w]; i < s->ws_host[w + 1] && q_host; ++i) {
      for (int a = 0; a < 3; ++a) {
        double x = q_host[3 * i + a];
        if (!std::isfinite(x)) continue;
        if (!any) { lo[a] = hi[a] = x; }
        lo[a] = std::min(lo[a], x);
        hi[a] = std::max(hi[a], x);
      }
      any = true;
    }
    double cw = cw0;
    int dim[3];
    for (;;) {
      double cells = 1.0;
      for (int a = 0; a < 3; ++a) {
        double margin = 4.0 * cw + 0.1 * (hi[a] - lo[a]);
        dim[a] = (int)std::ceil((hi[a] - lo[a] + 2.0 * margin) / cw) + 1;
        dim[a] = (dim[a] + 3) / 4 * 4;  // whole 4 x 4 x 4 tiles
        cells *= dim[a];
      }
      if (cells <= 33554432.0) break;
      cw *= 1.5;
    }
    WorldGrid g;
    g.inv_cw = (float)(1.0 / cw);
    double m0 = 4.0 * cw + 0.1 * (hi[0] - lo[0]), m1 = 4.0 * cw + 0.1 * (hi[1] - lo[1]),
           m2 = 4.0 * cw + 0.1 * (hi[2] - lo[2]);
    g.ox = (float)(lo[0] - m0);
    g.oy = (float)(lo[1] - m1);
    g.oz = (float)(lo[2] - m2);
    g.nx = dim[0];
    g.ny = dim[1];
    g.nz = dim[2];
    g.tnx = dim[0] / 4;
    g.tny = dim[1] / 4;
    g.pad0 = g.pad1 = 0;
    g.base = (int)base;
    s->grids[w] = g;
    s->world_cells_h[w] = dim[0] * dim[1] * dim[2];
    base += s->world_cells_h[w];
  }
  s->total_cells = (int)base;
}

void set_solve_params(adf_solver* s, DevP& P, int mode, double dt) {
  const adf_params& p = s->prm;
  P.mode = mode;
  P.dt = (float)dt;
  P.warm = (float)(mode == 0 ? p.warm_div : p.warm_den);
  double tol = mode == 0 ? p.tol_div : p.tol_den;
  P.tol = (float)tol;
  P.tol_max = (float)(tol * p.max_error_factor);
  P.tol_scale = (mode == 1 && s->jit_scale) ? s->jit_scale : nullptr;  // the density solve under the rule
  P.relief = (mode == 1 && p.relief_speed > 0.0) ? (float)(p.relief_speed * dt * p.lattice_grad) : (float)(1.0e30);
}

int prepare(adf_solver* s, DevP& P, cudaStream_t st) {
  const int n = s->n;
  prof_begin(s, 0, st);
  if (P.skin_on) {  // which worlds rebuild their superset rows (dfsph_skin.cuh)
    LAUNCH(s, k_skin_seed, blocks(std::max(s->W, 1)), BLOCK, st, P);
    LAUNCH(s, k_skin_check, blocks(n), BLOCK, st, P);
  }
  LAUNCH(s, k_classify, blocks(n), BLOCK, st, P);
  LAUNCH(s, k_scan_tiles, s->n_tiles, SCAN_THREADS, st, P.counts, s->n_keys, s->tile_sums);
  LAUNCH(s, k_scan_tile_sums, 1, SCAN_THREADS, st, s->tile_sums, s->n_tiles);
  LAUNCH(s, k_scan_apply, s->n_tiles, SCAN_THREADS, st, P.counts, s->n_keys, s->tile_sums, P.cell_start);
  LAUNCH(s, k_post_scan, blocks(std::max(s->W, 1)), BLOCK, st, P, s->world_cells);
  LAUNCH(s, k_scatter, blocks(n), BLOCK, st, P);
  prof_end(s, st);
  prof_begin(s, 1, st);
  if (P.skin_on) {
    LAUNCH(s, k_skin_ref, blocks(n), BLOCK, st, P);
    {
      const size_t smem = P.sup_cap <= SKIN_SMEM_CAP ? sizeof(int) * (size_t)P.sup_cap * SKIN_THREADS : 0;
      k_skin_build<<<blocks(n, SKIN_THREADS), SKIN_THREADS, smem, st>>>(P);
      ++s->launches;
    }
    LAUNCH(s, k_skin_filter, blocks(n), BLOCK, st, P);
  } else if (s->K <= LU_ROW) {
    run_tk(s, TK_LISTS, st, P);
  } else {
    const size_t smem = sizeof(int) * (size_t)s->K * LS_THREADS;
    k_lists_smem<<<blocks(n, LS_THREADS), LS_THREADS, smem, st>>>(P);
    ++s->launches;
  }
  prof_end(s, st);
  prof_begin(s, 2, st);
  LAUNCH(s, k_wall_slots, blocks(n), BLOCK, st, P);
  if (P.slot_cap > 1) LAUNCH(s, k_shape_slots, blocks(n), BLOCK, st, P);
  prof_end(s, st);
  prof_begin(s, 3, st);
  run_tk(s, TK_DENSITY, st, P);
  prof_end(s, st);
  if (halo_needed(s)) {
    prof_begin(s, 13, st);
    k_halo<<<s->halo_items, ITEM, HALO_SMEM_BUILD, st>>>(P);
    ++s->launches;
    prof_end(s, st);
  }
  s->built = true;
  return check_launch();
}

// One CG product out (+)= A vec (- b): the pressure acceleration of vec, then its divergence (krylov.py:254-261).
void cg_product(adf_solver* s, DevP& P, cudaStream_t st, const float* vec, const float* vr, float* out, int gated,
                int bias, int accumulate) {
  const int n = s->n;
  const TuneCfg& ca = s->tune[TK_ACCEL];
  const TuneCfg& cj = s->tune[TK_JACOBI];
  prof_begin(s, 5, st);
  if (s->cg_team) MS_DISPATCH(k_cg_accel_team, blocks((long long)n * TL), BLOCK, st, P, vec, vr, gated);
  else NB_DISPATCH(k_cg_accel, ca.nb, blocks(n, ca.block), ca.block, st, P, vec, vr, gated);
  ++s->launches;
  prof_end(s, st);
  prof_begin(s, 6, st);
  if (s->cg_team) MS_DISPATCH(k_cg_apply_team, blocks((long long)n * TL), BLOCK, st, P, vec, out, gated, bias, accumulate);
  else NB_DISPATCH(k_cg_apply, cj.nb, blocks(n, cj.block), cj.block, st, P, vec, out, gated, bias, accumulate);
  ++s->launches;
  prof_end(s, st);
}

void cg_sums(adf_solver* s, DevP& P, cudaStream_t st, int with_max) {
  prof_begin(s, 7, st);
  if (P.n_chunks > 0 && s->max_world_chunks <= WARP_FOLD_MAX_CHUNKS)
    LAUNCH(s, k_sums2_warps, (P.n_chunks + CHECK_WARPS - 1) / CHECK_WARPS, 32 * CHECK_WARPS, st, P, with_max, 0);
  else if (P.n_chunks > 0) LAUNCH(s, k_sums2_fused, P.n_chunks, 256, st, P, with_max, 0);
  else LAUNCH(s, k_world_sum2, s->W, 256, st, P, with_max);
  prof_end(s, st);
}

// krylov.py:278-285: w = A k - b from the warm start, the active set, z, p and r.z
void cg_init(adf_solver* s, DevP& P, cudaStream_t st) {
  const int n = s->n;
  cudaMemsetAsync(P.cg_restart, 0, sizeof(int) * std::max(s->W, 1), st);
  cudaMemsetAsync(P.cg_act_new, 0, sizeof(int) * std::max(s->W, 1), st);
  cudaMemsetAsync(P.cg_pair, 0, sizeof(float2) * std::max(n, 1), st);
  cg_product(s, P, st, P.kappa, P.kr, P.cg_w, 0, 1, 0);
  LAUNCH(s, k_cg_init, blocks(n), BLOCK, st, P);
  cg_sums(s, P, st, 0);
  LAUNCH(s, k_cg_first_rz, blocks(s->W), BLOCK, st, P);
}

// krylov.py:287-297: one projected PCG iteration of every unconverged world, with its stop test
void cg_iteration(adf_solver* s, DevP& P, cudaStream_t st) {
  const int n = s->n;
  cg_product(s, P, st, P.cg_pd, P.cg_pdr, P.cg_ap, 0, 0, 0);
  cg_sums(s, P, st, 0);
  LAUNCH(s, k_cg_step, blocks(n), BLOCK, st, P);
  {  // the correction product (worlds where the step clamped a variable) with the finish of the iteration
    const TuneCfg& ca = s->tune[TK_ACCEL];
    const TuneCfg& cj = s->tune[TK_JACOBI];
    prof_begin(s, 5, st);
    if (s->cg_team)
      MS_DISPATCH(k_cg_accel_team, blocks((long long)n * TL), BLOCK, st, P, (const float*)P.cg_corr,
                  (const float*)P.cg_corrr, 1);
    else
      NB_DISPATCH(k_cg_accel, ca.nb, blocks(n, ca.block), ca.block, st, P, (const float*)P.cg_corr,
                  (const float*)P.cg_corrr, 1);
    ++s->launches;
    prof_end(s, st);
    prof_begin(s, 6, st);
    if (s->cg_team) MS_DISPATCH(k_cg_apply_finish_team, blocks((long long)n * TL), BLOCK, st, P);
    else NB_DISPATCH(k_cg_apply_finish, cj.nb, blocks(n, cj.block), cj.block, st, P);
    ++s->launches;
    prof_end(s, st);
  }
  if (P.n_chunks > 0) {  // sums with the maximum, stop test and beta per world, unconverged count: one launch
    prof_begin(s, 7, st);
    if (s->max_world_chunks <= WARP_FOLD_MAX_CHUNKS)
      LAUNCH(s, k_sums2_warps, (P.n_chunks + CHECK_WARPS - 1) / CHECK_WARPS, 32 * CHECK_WARPS, st, P, 1, 1);
    else
      LAUNCH(s, k_sums2_fused, P.n_chunks, 256, st, P, 1, 1);
    prof_end(s, st);
  } else {
    cg_sums(s, P, st, 1);
    cudaMemsetAsync(P.n_unconv, 0, sizeof(int), st);
    LAUNCH(s, k_cg_beta, blocks(s->W), BLOCK, st, P);
  }
  LAUNCH(s, k_cg_direction, blocks(n), BLOCK, st, P);
}

// The CG solve as one persistent launch (k_cg_solve) for team-product models with chunks, outside profiled runs
// (those time each kernel group of the multi-launch path).
bool persistent_solve(const adf_solver* s, const DevP& P) {
  return s->cg && s->cg_team && s->persist_on && !s->prof_on && P.n_chunks > 0 && s->W > 0;
}

int persistent_cg(adf_solver* s, DevP& P, cudaStream_t st) {
  const bool ms = s->d.slot_cap > 1;
  int& cap = s->persist_cap[ms ? 1 : 0];
  if (cap == 0) {
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms ? k_cg_solve<true> : k_cg_solve<false>, BLOCK, 0));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    cap = per_sm * sms;
    if (cap <= 0) return fail(ADF_ERR_CUDA, "k_cg_solve: no block of it fits on an SM");
  }
  const int n = s->n;
  CgPersist R{};
  R.pt_blocks = blocks(n);
  R.team_blocks = blocks((long long)n * TL);
  R.warp_fold = s->max_world_chunks <= WARP_FOLD_MAX_CHUNKS ? 1 : 0;
  R.sum_blocks = R.warp_fold ? (P.n_chunks + CHECK_WARPS - 1) / CHECK_WARPS : P.n_chunks;
  R.w_blocks = blocks(s->W);
  R.cap = P.max_it + 2;  // as the WHILE node's cap
  const int grid = std::min(cap, std::max(std::max(R.pt_blocks, R.team_blocks), std::max(R.sum_blocks, R.w_blocks)));
  R.expect = (unsigned)grid + s->persist_extra;
  R.wait_limit = s->persist_wait;
  R.arrive = s->parrive;
  R.status = s->perr;
  CK(cudaMemsetAsync(s->parrive, 0, sizeof(unsigned), st));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(BLOCK);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;  // every block resident: the barriers wait on all of them
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  prof_begin(s, 5, st);
  if (ms) CK(cudaLaunchKernelEx(&cfg, k_cg_solve<true>, P, R));
  else CK(cudaLaunchKernelEx(&cfg, k_cg_solve<false>, P, R));
  ++s->launches;
  prof_end(s, st);
  return check_launch();
}

// The stop test of an iteration and the next iteration's work list (one launch: k_check_warps or k_check_fused).
void check_iteration(adf_solver* s, DevP& P, cudaStream_t st) {
  if (P.n_chunks > 0) {
    if (s->max_world_chunks <= WARP_FOLD_MAX_CHUNKS)
      LAUNCH(s, k_check_warps, (P.n_chunks + CHECK_WARPS - 1) / CHECK_WARPS, 32 * CHECK_WARPS, st, P);
    else
      LAUNCH(s, k_check_fused, P.n_chunks, 256, st, P);
  } else {
    cudaMemsetAsync(P.n_unconv, 0, sizeof(int), st);
    if (s->W > 0) LAUNCH(s, k_worklist, 1, 1024, st, P);
  }
}

void enqueue_iteration(adf_solver* s, DevP& P, cudaStream_t st) {
  const int n = s->n;
  (void)n;
  if (s->cg) {
    cg_iteration(s, P, st);
    return;
  }
  prof_begin(s, 5, st);
  run_tk(s, TK_ACCEL, st, P);
  prof_end(s, st);
  prof_begin(s, 6, st);
  run_tk(s, TK_JACOBI, st, P);
  prof_end(s, st);
  prof_begin(s, 7, st);
  check_iteration(s, P, st);
  prof_end(s, st);
}

int host_iterations(adf_solver* s, DevP& P, cudaStream_t st, int done);

// The iteration loop as a WHILE node of the graph being captured on `st` (the body: one iteration plus the
// condition update). Mirrors wp.capture_while (solve_driver.py:186): no host round trip per iteration.
int capture_iterations(adf_solver* s, DevP& P, cudaStream_t st) {
  cudaStreamCaptureStatus cs;
  unsigned long long id;
  cudaGraph_t g;
  const cudaGraphNode_t* deps;
  size_t nd;
  CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) return fail(ADF_ERR_STATE, "capture_iterations: stream not capturing");
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  LAUNCH(s, k_set_cond, 1, 1, st, h, (const int*)P.n_unconv, s->body_runs, -1);
  CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, deps, nd, &cp));
  CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (!s->body_stream) CK(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
  const long long b0 = s->launches;
  CK(cudaStreamBeginCaptureToGraph(s->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  enqueue_iteration(s, P, s->body_stream);
  LAUNCH(s, k_set_cond, 1, 1, s->body_stream, h, (const int*)P.n_unconv, s->body_runs, P.max_it + 2);
  cudaGraph_t out;
  CK(cudaStreamEndCapture(s->body_stream, &out));
  s->body_kernels = s->launches - b0;  // counted per run through body_runs, not per capture
  s->launches = b0;
  return check_launch();
}

// Iteration 1 of a solve with the learned start: one sweep from the plain start and one from the learned start, their
// per-world residual sums, each world's choice (the learned start unless its residual is larger), the chosen state
// copied into the solve's arrays, then the iteration's stop test as in every other iteration.
void dual_iteration(adf_solver* s, DevP& P, cudaStream_t st) {
  DevP L = P;
  L.kappa = P.kappa2;
  L.kr = P.kr2;
  L.acc = P.acc2;
  L.err_orig = P.err2;
  const int W = s->W;
  // the learned start's sweep covers the worlds its schedule evaluates in this solve (their own work list)
  L.converged = P.probe_skip;
  L.cw = s->cw2;
  L.cseg = s->cseg2;
  L.n_cw = s->n_cw2;
  LAUNCH(s, k_probe_plan, blocks(W), BLOCK, st, P);
  LAUNCH(s, k_worklist, 1, 1024, st, L);
  for (int pass = 0; pass < 2; ++pass) {
    DevP& Q = pass == 0 ? P : L;
    prof_begin(s, 5, st);
    run_tk(s, TK_ACCEL, st, Q);
    prof_end(s, st);
    prof_begin(s, 6, st);
    run_tk(s, TK_JACOBI, st, Q);
    prof_end(s, st);
    prof_begin(s, 7, st);
    if (P.n_chunks > 0)
      LAUNCH(s, k_chunk_sum, (P.n_chunks + 7) / 8, 256, st, (const float*)Q.err_orig, P.chunk_begin, P.chunk_end,
             P.n_chunks, P.part_sum, P.part_max);
    LAUNCH(s, k_world_check, W, 256, st, P, 0, pass == 0 ? P.sum_c : P.sum_l, pass == 0 ? P.max_c : P.max_l);
    prof_end(s, st);
  }
  const int n = s->n;
  LAUNCH(s, k_choose_start, blocks(W), BLOCK, st, P);
  LAUNCH(s, k_select_start, blocks(n), BLOCK, st, P);
  prof_begin(s, 7, st);
  check_iteration(s, P, st);
  prof_end(s, st);
}

mlp::Net solver_net(const adf_solver* s) {
  return mlp::Net{s->mw1, s->mw2, s->mparams, s->mnorm, s->merr, mlp::WAIT_LIMIT};
}

// pressure.py:355-390 + solve_driver.py:121-186 (Jacobi branch) + pressure.py:393-480
int solve(adf_solver* s, DevP& P, int mode, double dt, cudaStream_t st, bool graph) {
  set_solve_params(s, P, mode, dt);
  const int n = s->n, W = s->W;
  const bool first = mode == 0 || !s->prm.divergence_solve;  // the step's first solve records the features
  const bool warm = s->warm_on && W > 0;
  CK(cudaMemsetAsync(P.err_orig, 0, sizeof(float) * n, st));
  if (warm) CK(cudaMemsetAsync(P.err2, 0, sizeof(float) * n, st));
  CK(cudaMemsetAsync(P.n_unconv, 0, sizeof(int), st));
  P.feat_on = (first && (s->warm_on || s->feat_rec)) ? 1 : 0;
  // under the judge only the worlds that evaluate the learned start in this step need features and predictions
  const bool subset = warm && first && s->judge && !s->cg && !s->feat_rec;
  P.warm_need = subset ? s->warm_need : nullptr;
  if (subset) LAUNCH(s, k_warm_need, blocks(W), BLOCK, st, P, s->warm_need);
  if (mode == 1 && s->jit_scale && W > 0) {  // this step's density tolerance per world (solve_driver.py:99-110)
    if (P.n_chunks > 0) {
      LAUNCH(s, k_jitter_chunks, (P.n_chunks + 7) / 8, 256, st, P, 1, s->jit_part);
      LAUNCH(s, k_jitter_worlds, (W + 7) / 8, 256, st, P, 1, (const double*)s->jit_part, s->jit_head);
    } else {
      CK(cudaMemsetAsync(s->jit_head, 0, sizeof(double) * JIT_TERMS * W, st));
    }
    const adf_params& p = s->prm;
    LAUNCH(s, k_tol_scale, blocks(W), BLOCK, st, P, (const double*)s->jit_head,
           p.jitter_ratio > 0.0 ? (const double*)s->jit_flow : nullptr, (float)dt, (float)p.jitter_speed,
           (float)p.jitter_ratio, (float)p.tol_den, (float)p.tol_den_min, s->jit_scale, s->den_tol);
  }
  prof_begin(s, 4, st);
  run_tk(s, TK_SOLVE_INIT, st, P);
  prof_end(s, st);
  P.feat_on = 0;
  if (warm) {
    prof_begin(s, 12, st);
    if (first) {
      k_mlp_warm<<<s->mlp_grid, mlp::TILE, mlp::FW_SMEM, st>>>(P, solver_net(s));
      ++s->launches;
    }
    DevP Q = P;
    const bool take = !s->judge || s->cg;
    if (take) {  // the learned start replaces the plain one outright
      Q.kappa2 = P.kappa;
      Q.kr2 = P.kr;
    }
    LAUNCH(s, k_learned_start, blocks(n), BLOCK, st, Q);
    if (take) LAUNCH(s, k_mark_learned, blocks(W), BLOCK, st, P);
    prof_end(s, st);
  }
  if (W > 0) {
    LAUNCH(s, k_begin_solve, blocks(W), BLOCK, st, P);
    LAUNCH(s, k_worklist, 1, 1024, st, P);
  } else {
    CK(cudaMemsetAsync(P.n_cw, 0, sizeof(int), st));
  }
  int rc = check_launch();
  if (rc) return rc;
  const bool dual = warm && s->judge && !s->cg;  // the first-sweep judge is a Jacobi sweep
  if (dual) dual_iteration(s, P, st);
  if (persistent_solve(s, P)) {  // the CG start and its iterations in one launch
    rc = persistent_cg(s, P, st);
    if (rc) return rc;
  } else {
    if (s->cg && W > 0) cg_init(s, P, st);
    rc = graph ? capture_iterations(s, P, st) : host_iterations(s, P, st, dual ? 1 : 0);
    if (rc) return rc;
  }
  prof_begin(s, 8, st);
  {
    const TuneCfg& c = s->tune[TK_ACCEL];
    NB_DISPATCH(k_apply, c.nb, blocks(n, c.block), c.block, st, P);
    ++s->launches;
  }
  prof_end(s, st);
  if (mode == 0) {
    CK(cudaMemcpyAsync(s->iters_div, P.iters, sizeof(int) * W, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->div_err, P.err_mean, sizeof(float) * W, cudaMemcpyDeviceToDevice, st));
  } else {
    CK(cudaMemcpyAsync(s->iters_den, P.iters, sizeof(int) * W, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->den_err, P.err_mean, sizeof(float) * W, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->den_err_max, P.emax, sizeof(float) * W, cudaMemcpyDeviceToDevice, st));
  }
  return check_launch();
}

// The iteration loop driven from the host: iteration k+1 is enqueued before the unconverged count of iteration k
// is read, so the GPU does not idle on the read; iterations before min_iterations cannot stop a world and are not
// checked.
int host_iterations(adf_solver* s, DevP& P, cudaStream_t st, int done) {
  const int limit = s->prm.max_it + 2;  // every world stops at max_iterations
  const bool speculate = !s->prof_on;   // profiled runs time only iterations that do work
  int enq = done;                       // iterations already enqueued (the dual first sweep)
  for (; enq < s->prm.min_it - 1; ++enq) enqueue_iteration(s, P, st);  // these cannot stop a world
  auto push = [&]() -> int {
    const int slot = enq & 1;
    enqueue_iteration(s, P, st);
    CK(cudaMemcpyAsync(&s->pinned[slot], P.n_unconv, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(s->ev[slot], st));
    ++enq;
    return ADF_OK;
  };
  int rc = push();
  if (rc) return rc;
  for (;;) {
    const int last = enq - 1;
    if (speculate && enq < limit && (rc = push())) return rc;
    CK(cudaEventSynchronize(s->ev[last & 1]));
    if (s->pinned[last & 1] == 0 || last + 1 >= limit) break;
    if (!speculate && (rc = push())) return rc;
  }
  return check_launch();
}

// Re-upload the emitter tables; the layer clocks and cursors of the first n_carry emitters are kept.
int upload_emitters(adf_solver* s, int n_carry) {
  int n_old = 0;
  std::vector<float> t_old;
  std::vector<int> c_old;
  if (s->em_d) {
    n_old = n_carry;
    t_old.resize(n_old);
    c_old.resize(n_old);
    if (n_old > 0) {
      CK(cudaMemcpy(t_old.data(), s->t_acc_d, sizeof(float) * n_old, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(c_old.data(), s->cursor_d, sizeof(int) * n_old, cudaMemcpyDeviceToHost));
    }
    void* olds[] = {s->em_d, s->off_local_d, s->off_emitter_d, s->off_rank_d, s->pool_d, s->enabled_d, s->cursor_d,
                    s->emit_now_d, s->t_acc_d, s->em_world_d};
    for (void* p : olds) cudaFree(p);
  }
  int ne = (int)s->em_h.size();
  int no = (int)s->off_emitter_h.size();
  int rc = dalloc(&s->em_d, ne) | dalloc(&s->off_local_d, 3 * (size_t)no) | dalloc(&s->off_emitter_d, no) |
           dalloc(&s->off_rank_d, no) | dalloc(&s->pool_d, s->pool_h.size()) | dalloc(&s->enabled_d, ne) |
           dalloc(&s->cursor_d, ne) | dalloc(&s->emit_now_d, ne) | dalloc(&s->t_acc_d, ne) |
           dalloc(&s->em_world_d, ne);
  if (rc) return fail(ADF_ERR_CUDA, "emitter tables: cudaMalloc failed");
  std::vector<int> em_world(ne);
  for (int e = 0; e < ne; ++e) em_world[e] = s->em_h[e].world;
  if (ne) CK(cudaMemcpy(s->em_world_d, em_world.data(), sizeof(int) * ne, cudaMemcpyHostToDevice));
  std::vector<float> t(ne, 0.0f);
  std::vector<int> c(ne, 0);
  for (int e = 0; e < n_old; ++e) { t[e] = t_old[e]; c[e] = c_old[e]; }
  CK(cudaMemcpy(s->em_d, s->em_h.data(), sizeof(Emit) * ne, cudaMemcpyHostToDevice));
  if (no) {
    CK(cudaMemcpy(s->off_local_d, s->off_local_h.data(), sizeof(float) * 3 * no, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->off_emitter_d, s->off_emitter_h.data(), sizeof(int) * no, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->off_rank_d, s->off_rank_h.data(), sizeof(int) * no, cudaMemcpyHostToDevice));
  }
  if (!s->pool_h.empty())
    CK(cudaMemcpy(s->pool_d, s->pool_h.data(), sizeof(int) * s->pool_h.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->enabled_d, s->enabled_h.data(), sizeof(int) * ne, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->cursor_d, c.data(), sizeof(int) * ne, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->t_acc_d, t.data(), sizeof(float) * ne, cudaMemcpyHostToDevice));
  return ADF_OK;
}

}  // namespace

extern "C" {

const char* adf_last_error(void) { return g_err.c_str(); }

int adf_create(const adf_params* params, const adf_model* m, int device, adf_solver** out) {
  if (!params || !m || !out) return fail(ADF_ERR_VALUE, "adf_create: null argument");
  *out = nullptr;
  const adf_params& p = *params;
  if (m->n < 0 || m->world_count < 0) return fail(ADF_ERR_VALUE, "adf_create: negative sizes");
  if (p.capacity < 8 || p.capacity > MAXCAP)
    return fail(ADF_ERR_VALUE, "neighbor_capacity must be in [8, " + std::to_string(MAXCAP) + "], got " +
                                   std::to_string(p.capacity));
  if (!(p.h > 0.0) || !(p.particle_radius > 0.0)) return fail(ADF_ERR_VALUE, "particle_radius and h must be > 0");
  if (p.kind != 0 && p.kind != 1) return fail(ADF_ERR_VALUE, "kernel must be 0 (cubic) or 1 (wendland_c2)");
  if (!m->world_start) return fail(ADF_ERR_VALUE, "world_start is required");
  for (int w = 0; w < m->world_count; ++w)
    if (m->world_start[w + 1] < m->world_start[w])
      return fail(ADF_ERR_VALUE, "particles must be contiguous per world (Model.particle_world sorted)");
  if (m->world_count > 0 && (m->world_start[0] < 0 || m->world_start[m->world_count] > m->n))
    return fail(ADF_ERR_VALUE, "world_start out of range");
  if (m->n > 0 && (!m->mass || !m->rest_density || !m->radius || !m->flags || !m->phase || !m->world || !m->gravity))
    return fail(ADF_ERR_VALUE, "adf_create: a model array is null");
  if (!(p.skin >= 0.0) || p.skin > p.h) return fail(ADF_ERR_VALUE, "skin must be in [0, h]");
  if (p.skin > 0.0 && (p.skin_cap < 1 || p.skin_cap > 4096))
    return fail(ADF_ERR_VALUE, "skin_cap must be in [1, 4096] when skin > 0");
  if (m->n_shapes < 0) return fail(ADF_ERR_VALUE, "adf_create: negative n_shapes");
  if (m->n_shapes > 0) {
    if (!m->shape_start || !m->shape_box) return fail(ADF_ERR_VALUE, "adf_create: shape_start and shape_box needed");
    if (m->world_count > 0 && m->shape_start[0] != 0) return fail(ADF_ERR_VALUE, "shape_start[0] must be 0");
    for (int w = 0; w < m->world_count; ++w)
      if (m->shape_start[w + 1] < m->shape_start[w]) return fail(ADF_ERR_VALUE, "shape_start must not decrease");
    const int total = m->world_count > 0 ? m->shape_start[m->world_count] : 0;
    if (total > 0 && !m->shape_ids) return fail(ADF_ERR_VALUE, "adf_create: shape_ids needed");
    for (int c = 0; c < total; ++c)
      if (m->shape_ids[c] < 0 || m->shape_ids[c] >= m->n_shapes)
        return fail(ADF_ERR_VALUE, "shape_ids out of range [0, n_shapes)");
    for (int k = 0; k < m->n_shapes; ++k)
      for (int a = 0; a < 8; ++a)
        if (!std::isfinite(m->shape_box[8 * k + a])) return fail(ADF_ERR_VALUE, "shape_box holds a non-finite value");
    if (m->shape_geo)  // the walls a world sees (shapes no world lists are never evaluated)
      for (int c = 0; c < total; ++c) {
        const int g = m->shape_geo[m->shape_ids[c]];
        if (g != GEO_BOX && g != GEO_SPHERE && g != GEO_CAPSULE && g != GEO_CYLINDER && g != GEO_PLANE)
          return fail(ADF_ERR_VALUE, "shape_geo: only boxes (7), spheres (3), capsules (4), cylinders (6), planes (1)");
      }
    if (m->shape_quat)
      for (int k = 0; k < 4 * m->n_shapes; ++k) {
        if (!std::isfinite(m->shape_quat[k])) return fail(ADF_ERR_VALUE, "shape_quat holds a non-finite value");
      }
  }
  CK(cudaSetDevice(device));
  adf_solver* s = new adf_solver();
  s->prm = p;
  s->n = m->n;
  s->W = m->world_count;
  s->K = p.capacity;
  s->device = device;
  s->ws_host.assign(m->world_start, m->world_start + m->world_count + 1);
  if (s->W == 0) s->ws_host.assign(1, 0);
  size_grids(s, m->q_host);
  const int n = std::max(s->n, 1), W = std::max(s->W, 1);
  s->n_keys = 2 * s->total_cells;
  s->n_tiles = std::max((s->n_keys + SCAN_TILE - 1) / SCAN_TILE, 1);

  DevP& d = s->d;
  d.kc = make_kc(p.kind, p.h, p.sigma);
  d.n = s->n;
  d.W = s->W;
  d.K = s->K;
  d.total_cells = s->total_cells;
  d.n_full = (float)p.n_full;
  d.tot_min = (float)p.tot_min;
  d.wall_offset = (float)p.wall_offset;
  d.wall_amp = (float)p.wall_amplitude;
  d.taper0 = (float)p.taper0;
  d.taper1 = (float)p.taper1;
  d.reach = (float)p.reach;
  d.omega = (float)p.omega;
  d.warm_den = (float)p.warm_den;
  d.warm_div = (float)p.warm_div;
  d.min_nb = (float)p.min_nb;
  d.xsph_c = (float)p.xsph_c;
  d.v_sep = (float)p.v_sep;
  d.eps = (float)p.project_eps;
  d.two_sided = p.two_sided;
  d.min_it = p.min_it;
  d.max_it = p.max_it;
  d.has_bounds = p.has_bounds;
  for (int a = 0; a < 3; ++a) {
    d.blo[a] = (float)p.bounds_lo[a];
    d.bhi[a] = (float)p.bounds_hi[a];
  }
  const int n_box_refs = (m->n_shapes > 0 && m->world_count > 0) ? m->shape_start[m->world_count] : 0;
  d.slot_cap = n_box_refs > 0 ? 4 : 1;
  d.n_shapes = m->n_shapes;
  d.sweep_len = (float)m->sweep_len;
  d.prad = (float)p.particle_radius;
  d.wall_friction = p.wall_friction != 0;
  d.mass = m->mass;
  d.rho0 = m->rest_density;
  d.flags = m->flags;
  d.phase = m->phase;
  d.world = m->world;
  d.gravity = m->gravity;

  // chunk table of the per-world reductions (reduce.py:167-182)
  std::vector<int> cb, ce, cs(1, 0), cwld;
  for (int w = 0; w < s->W; ++w) {
    for (int b = s->ws_host[w]; b < s->ws_host[w + 1]; b += 256) {
      cb.push_back(b);
      ce.push_back(std::min(b + 256, s->ws_host[w + 1]));
      cwld.push_back(w);
    }
    cs.push_back((int)cb.size());
  }
  d.n_chunks = (int)cb.size();
  for (size_t k = 0; k + 1 < cs.size(); ++k) s->max_world_chunks = std::max(s->max_world_chunks, cs[k + 1] - cs[k]);
  d.n_chunk_worlds = 0;
  for (size_t k = 0; k + 1 < cs.size(); ++k) d.n_chunk_worlds += cs[k + 1] > cs[k] ? 1 : 0;
  // sum over worlds of ceil(liquid_w / 256) <= n / 256 + W, whatever the worlds' sizes
  s->max_items = (int)std::max<long long>(((long long)s->n + ITEM - 1) / ITEM + s->W, 1);


  int rc = 0;
  float* wall_vol = nullptr;
  WorldGrid* grid = nullptr;
  int *chunk_begin = nullptr, *chunk_end = nullptr, *world_chunk_start = nullptr, *chunk_world = nullptr;
  rc |= s->alloc(&wall_vol, n);
  rc |= s->alloc(&grid, W);
  rc |= s->alloc(&s->world_cells, W);
  rc |= s->alloc(&d.key_of, n);
  rc |= s->alloc(&d.counts, s->n_keys);
  rc |= s->alloc(&d.cell_start, (size_t)s->n_keys + 1);
  rc |= s->alloc(&s->tile_sums, s->n_tiles);
  rc |= s->alloc(&d.nfw, 2);
  rc |= s->alloc(&d.pos, n);
  rc |= s->alloc(&d.vel, n);
  rc |= s->alloc(&d.vel2, n);
  rc |= s->alloc(&d.id_of, n);
  rc |= s->alloc(&d.pos_of, n);
  rc |= s->alloc(&d.world_s, n);
  rc |= s->alloc(&d.kv_s, n);
  rc |= s->alloc(&d.kd_s, n);
  rc |= s->alloc(&d.nbr, (size_t)s->K * n);
  rc |= s->alloc(&d.nbrjf, (size_t)s->K * n);
  rc |= s->alloc(&d.nbrw, (size_t)s->K * n);
  s->halo_items = (int)std::max<long long>((long long)n / ITEM + s->W + 1, 1);  // buffers: adf_set_halo
  rc |= s->alloc(&d.cnt, n);
  rc |= s->alloc(&d.slot_g, (size_t)d.slot_cap * n);
  rc |= s->alloc(&d.slot_vb, (size_t)d.slot_cap * n);
  rc |= s->alloc(&d.slot_n, (size_t)d.slot_cap * n);
  rc |= s->alloc(&d.slot_xb, (size_t)d.slot_cap * n);
  int *sh_start = nullptr, *sh_ids = nullptr;
  float4 *sh_pos = nullptr, *sh_half = nullptr;
  int* sh_geo = nullptr;
  float4* sh_quat = nullptr;
  if (d.slot_cap > 1) {
    rc |= s->alloc(&d.slot_cnt, n);
    rc |= s->alloc(&sh_start, (size_t)W + 1);
    rc |= s->alloc(&sh_ids, (size_t)n_box_refs);
    rc |= s->alloc(&sh_pos, (size_t)m->n_shapes);
    rc |= s->alloc(&sh_half, (size_t)m->n_shapes);
    rc |= s->alloc(&sh_geo, (size_t)m->n_shapes);
    rc |= s->alloc(&sh_quat, (size_t)m->n_shapes);
  }
  rc |= s->alloc(&d.swept, W);
  d.skin_on = p.skin > 0.0;
  if (d.skin_on) {
    d.sup_cap = p.skin_cap;
    const double hs = p.h + p.skin;
    int reach = 1;
    for (const WorldGrid& g : s->grids) reach = std::max(reach, (int)std::floor(hs * (double)g.inv_cw * (1.0 + 1.0e-5)) + 1);
    d.skin_reach = reach;
    d.skin_r2 = (float)hs * (float)hs;
    d.skin_half2 = (float)((0.49 * p.skin) * (0.49 * p.skin));
    rc |= s->alloc(&d.sup, (size_t)d.sup_cap * n);
    rc |= s->alloc(&d.sup_cnt, n);
    rc |= s->alloc(&d.skin_slot, n);
    rc |= s->alloc(&d.skin_qref, n);
    rc |= s->alloc(&d.skin_gref, n);
    rc |= s->alloc(&d.skin_flag, W);
    rc |= s->alloc(&d.skin_force, W);
  }
  rc |= s->alloc(&d.ratio, n);
  rc |= s->alloc(&d.alpha, n);
  rc |= s->alloc(&d.neff, n);
  rc |= s->alloc(&d.reg, n);
  rc |= s->alloc(&d.src, n);
  rc |= s->alloc(&d.kappa, n);
  rc |= s->alloc(&d.lower, n);
  rc |= s->alloc(&d.kr, n);
  rc |= s->alloc(&d.acc, n);
  rc |= s->alloc(&d.err_orig, n);
  rc |= s->alloc(&d.kv, n);
  rc |= s->alloc(&d.kd, n);
  rc |= s->alloc(&d.wrange, W);
  rc |= s->alloc(&d.cw, W);
  rc |= s->alloc(&d.cseg, (size_t)W + 1);
  rc |= s->alloc(&d.n_cw, 1);
  rc |= s->alloc(&d.iter_work, 1);
  rc |= s->alloc(&chunk_world, cb.size());
  s->cg = p.cg != 0;
  s->cg_team = s->cg && n <= CG_TEAM_MAX;
  if (s->cg) {
    rc |= s->alloc(&d.cg_pd, n);
    rc |= s->alloc(&d.cg_pdr, n);
    rc |= s->alloc(&d.cg_z, n);
    rc |= s->alloc(&d.cg_w, n);
    rc |= s->alloc(&d.cg_ap, n);
    rc |= s->alloc(&d.cg_corr, n);
    rc |= s->alloc(&d.cg_corrr, n);
    rc |= s->alloc(&d.cg_act, n);
    rc |= s->alloc(&d.cg_pair, n);
    rc |= s->alloc(&d.cg_rz, W);
    rc |= s->alloc(&d.cg_step, W);
    rc |= s->alloc(&d.cg_sums, W);
    rc |= s->alloc(&d.cg_restart, W);
    rc |= s->alloc(&d.cg_act_new, W);
    rc |= s->alloc(&d.part2, std::max<size_t>(cb.size(), 1));
  }
  rc |= s->alloc(&d.converged, W);
  rc |= s->alloc(&d.iters, W);
  rc |= s->alloc(&d.err_mean, W);
  rc |= s->alloc(&d.n_unconv, 1);
  rc |= s->alloc(&d.wdone, W);
  rc |= s->alloc(&d.gdone, 1);
  rc |= s->alloc(&d.n_active, W);
  rc |= s->alloc(&d.overflow, W);
  rc |= s->alloc(&d.escaped, W);
  rc |= s->alloc(&d.projected, W);
  rc |= s->alloc(&d.nonfinite, W);
  rc |= s->alloc(&d.wall_overflow, W);
  rc |= s->alloc(&d.max_speed_bits, W);
  rc |= s->alloc(&d.mass_out, W);
  rc |= s->alloc(&chunk_begin, cb.size());
  rc |= s->alloc(&chunk_end, ce.size());
  rc |= s->alloc(&world_chunk_start, cs.size());
  rc |= s->alloc(&d.part_sum, cb.size());
  rc |= s->alloc(&d.part_max, cb.size());
  if (p.jitter_speed > 0.0) {
    rc |= s->alloc(&s->jit_scale, W);
    rc |= s->alloc(&s->jit_part, JIT_TERMS * std::max<size_t>(cb.size(), 1));
    rc |= s->alloc(&s->jit_flow, JIT_TERMS * (size_t)W);
    rc |= s->alloc(&s->jit_head, JIT_TERMS * (size_t)W);
  }
  rc |= s->alloc(&d.emax, W);
  rc |= s->alloc(&s->iters_den, W);
  rc |= s->alloc(&s->iters_div, W);
  rc |= s->alloc(&s->emit_overflow, W);
  rc |= s->alloc(&s->den_err, W);
  rc |= s->alloc(&s->div_err, W);
  rc |= s->alloc(&s->den_err_max, W);
  rc |= s->alloc(&s->den_tol, W);
  rc |= s->alloc(&s->mass_in, W);
  rc |= s->alloc(&s->mass0, W);
  rc |= s->alloc(&s->tmp_mass, W);
  rc |= s->alloc(&s->mask_d, W);
  rc |= s->alloc(&s->ws_d, (size_t)W + 1);
  rc |= s->alloc(&s->port_stack, n);
  rc |= s->alloc(&s->port_stack0, n);
  for (int** a : {&s->port_top, &s->port_top0, &s->port_taken, &s->port_granted, &s->port_absorbed,
                  &s->port_emitted, &s->port_retired, &s->speed_bits})
    rc |= s->alloc(a, W);
  rc |= s->alloc(&s->energy_max, W);
  if (rc) {
    std::string msg = g_err;
    adf_destroy(s);
    return fail(ADF_ERR_CUDA, "adf_create: " + msg);
  }
  d.wall_vol = wall_vol;
  d.grid = grid;
  d.skin_ws = s->ws_d;
  d.sh_start = sh_start;
  d.sh_ids = sh_ids;
  d.sh_pos = sh_pos;
  d.sh_half = sh_half;
  d.sh_geo = sh_geo;
  d.sh_quat = sh_quat;
  d.chunk_begin = chunk_begin;
  d.chunk_end = chunk_end;
  d.world_chunk_start = world_chunk_start;
  d.chunk_world = chunk_world;
  auto fin = [&](int code) {
    if (code != ADF_OK) {
      std::string msg = g_err;
      adf_destroy(s);
      return fail(code, msg);
    }
    return ADF_OK;
  };
#define CKC(x)                                                                                       \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) return fin(fail(ADF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_))); \
  } while (0)
  CKC(cudaMemcpy(grid, s->grids.data(), sizeof(WorldGrid) * s->W, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(s->world_cells, s->world_cells_h.data(), sizeof(int) * s->W, cudaMemcpyHostToDevice));
  if (!cb.empty()) {
    CKC(cudaMemcpy(chunk_begin, cb.data(), sizeof(int) * cb.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(chunk_end, ce.data(), sizeof(int) * ce.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(chunk_world, cwld.data(), sizeof(int) * cwld.size(), cudaMemcpyHostToDevice));
  }
  CKC(cudaMemcpy(world_chunk_start, cs.data(), sizeof(int) * cs.size(), cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(s->ws_d, s->ws_host.data(), sizeof(int) * s->ws_host.size(), cudaMemcpyHostToDevice));
  if (d.skin_on) {  // nothing built yet: every world builds its superset rows on the first step
    std::vector<int> never(n, -2);
    CKC(cudaMemcpy(d.skin_gref, never.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CKC(cudaMemset(d.skin_slot, 0, sizeof(int) * n));
    CKC(cudaMemset(d.sup_cnt, 0, sizeof(int) * n));
    CKC(cudaMemset(d.skin_flag, 0, sizeof(int) * W));
    CKC(cudaMemset(d.skin_force, 0, sizeof(int) * W));
  }
  if (d.slot_cap > 1) {  // the box walls: per-world id lists, (centre, radius) and (half extents, mu) per shape
    std::vector<float4> bp(m->n_shapes), bh(m->n_shapes);
    for (int k = 0; k < m->n_shapes; ++k) {
      const float* b = m->shape_box + 8 * (size_t)k;
      bp[k] = make_float4(b[0], b[1], b[2], b[3]);
      bh[k] = make_float4(b[4], b[5], b[6], b[7]);
    }
    CKC(cudaMemcpy(sh_start, m->shape_start, sizeof(int) * (s->W + 1), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(sh_ids, m->shape_ids, sizeof(int) * n_box_refs, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(sh_pos, bp.data(), sizeof(float4) * bp.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(sh_half, bh.data(), sizeof(float4) * bh.size(), cudaMemcpyHostToDevice));
    std::vector<int> geo(m->n_shapes, GEO_BOX);
    if (m->shape_geo) std::copy(m->shape_geo, m->shape_geo + m->n_shapes, geo.begin());
    CKC(cudaMemcpy(sh_geo, geo.data(), sizeof(int) * geo.size(), cudaMemcpyHostToDevice));
    std::vector<float4> quat(m->n_shapes, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
    if (m->shape_quat)
      for (int k = 0; k < m->n_shapes; ++k) {
        const float* r = m->shape_quat + 4 * (size_t)k;
        quat[k] = make_float4(r[0], r[1], r[2], r[3]);
      }
    CKC(cudaMemcpy(sh_quat, quat.data(), sizeof(float4) * quat.size(), cudaMemcpyHostToDevice));
  }
  {  // the port's reservoir: each world's build-time held particles, popped in ascending id order (ports.py:124-133)
    std::vector<int8_t> ph(s->n);
    if (s->n > 0) CKC(cudaMemcpy(ph.data(), m->phase, s->n, cudaMemcpyDeviceToHost));
    std::vector<int> stack0(n, 0), top0(W, 0);
    for (int w = 0; w < s->W; ++w) {
      std::vector<int> ids;
      for (int i = s->ws_host[w]; i < s->ws_host[w + 1]; ++i)
        if (ph[i] == PH_HELD) ids.push_back(i);
      for (size_t j = 0; j < ids.size(); ++j) stack0[s->ws_host[w] + j] = ids[ids.size() - 1 - j];
      top0[w] = (int)ids.size();
    }
    CKC(cudaMemcpy(s->port_stack0, stack0.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->port_stack, stack0.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->port_top0, top0.data(), sizeof(int) * W, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->port_top, top0.data(), sizeof(int) * W, cudaMemcpyHostToDevice));
    for (int* a : {s->port_taken, s->port_granted, s->port_absorbed, s->port_emitted, s->port_retired})
      CKC(cudaMemset(a, 0, sizeof(int) * W));
  }
  CKC(cudaMemset(d.counts, 0, sizeof(int) * std::max(s->n_keys, 1)));
  CKC(cudaMemset(d.nfw, 0, sizeof(int) * 2));
  CKC(cudaMemset(d.kv, 0, sizeof(float) * n));
  CKC(cudaMemset(d.kd, 0, sizeof(float) * n));
  CKC(cudaMemset(d.err_orig, 0, sizeof(float) * n));
  void* zero_w[] = {d.overflow, d.escaped, d.projected, d.swept, d.nonfinite, d.wall_overflow, d.max_speed_bits, d.converged,
                    d.iters, d.err_mean, s->iters_den, s->iters_div, s->emit_overflow, s->den_err, s->div_err,
                    s->den_err_max, d.emax};
  for (void* z : zero_w) CKC(cudaMemset(z, 0, 4 * W));
  CKC(cudaMemset(d.mass_out, 0, 8 * W));
  CKC(cudaMemset(d.wdone, 0, sizeof(int) * std::max(W, 1)));
  CKC(cudaMemset(d.gdone, 0, sizeof(unsigned)));
  CKC(cudaMemset(d.iter_work, 0, sizeof(unsigned long long)));
  CKC(cudaMemset(s->mass_in, 0, 8 * W));
  CKC(cudaMemset(d.n_active, 0, 8 * W));
  std::vector<float> tol(W, (float)p.tol_den);
  CKC(cudaMemcpy(s->den_tol, tol.data(), sizeof(float) * W, cudaMemcpyHostToDevice));
  if (s->jit_scale) {
    const std::vector<float> one(W, 1.0f);
    CKC(cudaMemcpy(s->jit_scale, one.data(), sizeof(float) * W, cudaMemcpyHostToDevice));
    CKC(cudaMemset(s->jit_flow, 0, sizeof(double) * JIT_TERMS * W));
  }
  if (s->n > 0) {
    k_wall_volume<<<blocks(s->n), BLOCK>>>(s->n, m->flags, m->radius, wall_vol);
    ++s->launches;
    // initial liquid mass per world (runtime.py:387-389)
    CKC(cudaMemset(s->mass0, 0, 8 * W));
    k_active_mass<<<blocks(s->n), BLOCK>>>(d, s->mass0);
    ++s->launches;
  } else {
    CKC(cudaMemset(s->mass0, 0, 8 * W));
  }
  CKC(cudaGetLastError());
  CKC(cudaFuncSetAttribute(k_skin_build, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(int) * (size_t)SKIN_SMEM_CAP * SKIN_THREADS)));
  CKC(cudaFuncSetAttribute(k_lists_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(int) * (size_t)s->K * LS_THREADS)));
  CKC(cudaFuncSetAttribute(k_halo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HALO_SMEM_BUILD));
  CKC(cudaFuncSetAttribute(k_jacobi_h<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HALO_SMEM_JACOBI));
  CKC(cudaFuncSetAttribute(k_jacobi_h<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HALO_SMEM_JACOBI));
  CKC(cudaFuncSetAttribute(k_jacobi_h<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HALO_SMEM_JACOBI));
  CKC(cudaFuncSetAttribute(k_jacobi_h<4 | MS_FLAG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)HALO_SMEM_JACOBI));
  CKC(cudaFuncSetAttribute(k_jacobi_h<8 | MS_FLAG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)HALO_SMEM_JACOBI));
  CKC(cudaFuncSetAttribute(k_jacobi_h<16 | MS_FLAG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)HALO_SMEM_JACOBI));
  CKC(cudaHostAlloc((void**)&s->pinned, 2 * sizeof(int), cudaHostAllocDefault));
  CKC(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
  CKC(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
  CKC(cudaMalloc(&s->body_runs, 2 * sizeof(unsigned long long)));
  CKC(cudaMemset(s->body_runs, 0, 2 * sizeof(unsigned long long)));
  CKC(cudaMalloc(&s->parrive, sizeof(unsigned)));
  CKC(cudaMalloc(&s->perr, sizeof(int)));
  CKC(cudaMemset(s->perr, 0, sizeof(int)));
  CKC(cudaEventCreate(&s->tev[0]));
  CKC(cudaEventCreate(&s->tev[1]));
  CKC(cudaMalloc(&s->snap_kappa, sizeof(float) * n));
  CKC(cudaMalloc(&s->snap_kr, sizeof(float) * n));
  CKC(cudaMalloc(&s->snap_err, sizeof(float) * n));
  CKC(cudaMalloc(&s->snap_ovf, sizeof(int) * W));
  s->tune[TK_LISTS] = LISTS_DEFAULT;
  CKC(cudaEventCreateWithFlags(&s->ev[0], cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&s->ev[1], cudaEventDisableTiming));
  CKC(cudaDeviceSynchronize());
#undef CKC
  *out = s;
  return ADF_OK;
}

void adf_destroy(adf_solver* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  for (void* p : s->owned) cudaFree(p);
  void* em[] = {s->em_d, s->off_local_d, s->off_emitter_d, s->off_rank_d, s->pool_d, s->enabled_d, s->cursor_d,
                s->emit_now_d, s->t_acc_d, s->sinks_d, s->em_world_d};
  for (void* p : em)
    if (p) cudaFree(p);
  for (void* p : {(void*)s->pe_world_d, (void*)s->pe_count_d, (void*)s->pe_begin_d, (void*)s->pe_group_d,
                  (void*)s->pe_pending_d, (void*)s->pe_fired_d, (void*)s->pp_pool_d, (void*)s->pp_points_d,
                  (void*)s->pg_vel_d})
    if (p) cudaFree(p);
  if (s->pinned) cudaFreeHost(s->pinned);
  if (s->list_entries) cudaFree(s->list_entries);
  if (s->body_runs) cudaFree(s->body_runs);
  if (s->parrive) cudaFree(s->parrive);
  if (s->perr) cudaFree(s->perr);
  for (auto& g : s->graphs) cudaGraphExecDestroy(g.exec);
  if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
  if (s->body_stream) cudaStreamDestroy(s->body_stream);
  for (auto& e : s->prof_pool) cudaEventDestroy(e);
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : s->tev)
    if (e) cudaEventDestroy(e);
  for (float* p : {s->snap_kappa, s->snap_kr, s->snap_err})
    if (p) cudaFree(p);
  if (s->snap_ovf) cudaFree(s->snap_ovf);
  delete s;
}

}  // extern "C"

namespace {
// One step's work enqueued on `st`; with `graph` the stream is capturing and the solves become WHILE nodes.
int enqueue_step(adf_solver* s, const float* q_in, const float* qd_in, float* q_out, float* qd_out,
                 const float* f_ext, double dt, cudaStream_t st, bool graph) {
  const size_t bytes = sizeof(float) * 3 * (size_t)s->n;
  if (q_out != q_in) CK(cudaMemcpyAsync(q_out, q_in, bytes, cudaMemcpyDeviceToDevice, st));
  if (qd_out != qd_in) CK(cudaMemcpyAsync(qd_out, qd_in, bytes, cudaMemcpyDeviceToDevice, st));
  DevP P = s->d;
  P.q = q_out;
  P.qd = qd_out;
  P.f_ext = f_ext;
  P.dt = (float)dt;
  P.n_sinks = (int)s->sinks_h.size();
  P.sinks = s->sinks_d;
  CK(cudaMemsetAsync(P.max_speed_bits, 0, sizeof(int) * std::max(s->W, 1), st));
  int rc = prepare(s, P, st);
  if (rc) return rc;
  if (s->jit_scale && s->prm.jitter_ratio > 0.0 && P.n_chunks > 0) {  // the liquid's mean start velocity per world
    LAUNCH(s, k_jitter_chunks, (P.n_chunks + 7) / 8, 256, st, P, 0, s->jit_part);
    LAUNCH(s, k_jitter_worlds, (s->W + 7) / 8, 256, st, P, 0, (const double*)s->jit_part, s->jit_flow);
  }
  if (s->prm.divergence_solve) {
    rc = solve(s, P, 0, dt, st, graph);
    if (rc) return rc;
  }
  P.dt = (float)dt;
  prof_begin(s, 9, st);
  run_tk(s, TK_XSPH, st, P);
  prof_end(s, st);
  std::swap(P.vel, P.vel2);
  rc = solve(s, P, 1, dt, st, graph);
  if (rc) return rc;
  prof_begin(s, 10, st);
  MS_DISPATCH(k_finish, blocks(s->n), BLOCK, st, P);
  ++s->launches;
  prof_end(s, st);
  const int ne = (int)s->em_h.size();
  if (ne > 0) {
    prof_begin(s, 11, st);
    LAUNCH(s, k_emit_clock, blocks(ne), BLOCK, st, s->em_d, ne, (float)dt, s->enabled_d, s->t_acc_d, s->emit_now_d);
    int no = (int)s->off_emitter_h.size();
    if (no > 0)
      LAUNCH(s, k_emit, blocks(no), BLOCK, st, P, s->em_d, no, s->off_emitter_d, s->off_rank_d, s->off_local_d,
             s->emit_now_d, s->cursor_d, s->pool_d, s->mass_in, s->emit_overflow);
    LAUNCH(s, k_emit_cursor, blocks(ne), BLOCK, st, s->em_d, ne, s->emit_now_d, s->cursor_d);
    prof_end(s, st);
  }
  const int npe = (int)s->pe_world_h.size();
  if (npe > 0) {  // patch emitters after the box emitters (runtime.py:318-326)
    prof_begin(s, 11, st);
    LAUNCH(s, k_patch_emit, npe, 256, st, P, npe, s->pe_world_d, s->pe_count_d, s->pe_pending_d, s->pe_fired_d,
           s->pe_begin_d, s->pp_pool_d, s->pp_points_d, s->pe_group_d, s->pg_vel_d, s->mass_in);
    LAUNCH(s, k_patch_fire, blocks(npe), BLOCK, st, npe, s->pe_pending_d, s->pe_fired_d);
    prof_end(s, st);
  }
  return check_launch();
}

// A whole step as a CUDA graph (built once per state-pointer set, dt and emitter/sink table version).
int graph_step(adf_solver* s, const float* q_in, const float* qd_in, float* q_out, float* qd_out, const float* f_ext,
               double dt, cudaStream_t st) {
  const void* key[5] = {q_in, qd_in, q_out, qd_out, f_ext};
  for (auto& g : s->graphs) {
    if (g.dt == dt && g.version == s->table_version && std::equal(key, key + 5, g.key)) {
      CK(cudaGraphLaunch(g.exec, st));
      s->launches += s->graph_kernels;
      return ADF_OK;
    }
  }
  if (!s->cap_stream) CK(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
  if (!s->body_stream) CK(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
  const long long before = s->launches;
  CK(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(s, q_in, qd_in, q_out, qd_out, f_ext, dt, s->cap_stream, true);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s->cap_stream, &g);
  s->graph_kernels = s->launches - before;
  s->launches = before;
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc ? rc : fail(ADF_ERR_CUDA, std::string("step graph capture: ") + cudaGetErrorString(e));
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ADF_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  if (s->graphs.size() >= 4) {
    cudaGraphExecDestroy(s->graphs.front().exec);
    s->graphs.erase(s->graphs.begin());
  }
  adf_solver::GraphEntry ge;
  std::copy(key, key + 5, ge.key);
  ge.dt = dt;
  ge.version = s->table_version;
  ge.exec = exec;
  s->graphs.push_back(ge);
  CK(cudaGraphLaunch(exec, st));
  s->launches += s->graph_kernels;
  return ADF_OK;
}
}  // namespace

extern "C" {

int adf_step(adf_solver* s, const float* q_in, const float* qd_in, float* q_out, float* qd_out, const float* f_ext,
             double dt, void* stream) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_step: null solver");
  if (!(dt > 0.0)) return fail(ADF_ERR_VALUE, "SolverDFSPH.step: dt must be > 0, got " + std::to_string(dt));
  if (s->n == 0) return ADF_OK;
  if (!q_in || !qd_in || !q_out || !qd_out) return fail(ADF_ERR_VALUE, "adf_step: null state array");
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(s->device));
  cudaStreamCaptureStatus cs;
  CK(cudaStreamIsCapturing(st, &cs));
  if (cs == cudaStreamCaptureStatusActive)  // the caller is capturing: the step joins its graph
    return enqueue_step(s, q_in, qd_in, q_out, qd_out, f_ext, dt, st, true);
  if (s->tune_pending) {  // the tuning step: kernels one by one, each tuned kernel timed on this step's inputs
    s->tuning = true;
    int rc = enqueue_step(s, q_in, qd_in, q_out, qd_out, f_ext, dt, st, false);
    s->tuning = false;
    s->tune_pending = false;
    ++s->table_version;  // graphs recorded before hold the previous configurations
    return rc;
  }
  if (!s->use_graphs || s->prof_on) return enqueue_step(s, q_in, qd_in, q_out, qd_out, f_ext, dt, st, false);
  return graph_step(s, q_in, qd_in, q_out, qd_out, f_ext, dt, st);
}

int adf_set_graphs(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_graphs: null solver");
  s->use_graphs = enable != 0;
  return ADF_OK;
}

int adf_density_ratio(adf_solver* s, const float* q, const float* qd, float* ratio_out, float* active_out,
                      void* stream) {
  if (!s || !q || !qd) return fail(ADF_ERR_VALUE, "adf_density_ratio: null argument");
  if (s->n == 0) return ADF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(s->device));
  DevP P = s->d;
  P.q = const_cast<float*>(q);
  P.qd = const_cast<float*>(qd);
  int rc = prepare(s, P, st);
  if (rc) return rc;
  if (ratio_out) {
    CK(cudaMemsetAsync(ratio_out, 0, sizeof(float) * s->n, st));
    LAUNCH(s, k_unsort_n, blocks(s->n), BLOCK, st, s->n, P.nfw, P.id_of, P.ratio, 1, 0, ratio_out, 1);
  }
  if (active_out) {
    CK(cudaMemsetAsync(active_out, 0, sizeof(float) * s->n, st));
    LAUNCH(s, k_fill_ones, blocks(s->n), BLOCK, st, s->n, P.nfw, P.id_of, active_out);
  }
  return check_launch();
}

int adf_get_report(adf_solver* s, adf_report* r, void* stream) {
  if (!s || !r) return fail(ADF_ERR_VALUE, "adf_get_report: null argument");
  CK(cudaSetDevice(s->device));
  const cudaStream_t st = (cudaStream_t)stream;
  const int W = s->W;
  if (W == 0) return cudaStreamSynchronize(st) == cudaSuccess ? ADF_OK : fail(ADF_ERR_CUDA, "adf_get_report: sync");
  // every copy is ordered on the caller's stream (never the legacy default stream, which would wait for the work of
  // other streams too); one synchronisation at the end
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (!dst) return ADF_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return ADF_OK;
  };
  int rc = 0;
  rc |= cp(r->density_err, s->den_err, 4 * W);
  rc |= cp(r->divergence_err, s->div_err, 4 * W);
  rc |= cp(r->iters_density, s->iters_den, 4 * W);
  rc |= cp(r->iters_divergence, s->iters_div, 4 * W);
  rc |= cp(r->mass_in, s->mass_in, 8 * W);
  rc |= cp(r->mass_out, s->d.mass_out, 8 * W);
  rc |= cp(r->mass_initial, s->mass0, 8 * W);
  rc |= cp(r->escaped, s->d.escaped, 4 * W);
  rc |= cp(r->neighbor_overflow, s->d.overflow, 4 * W);
  rc |= cp(r->max_speed, s->d.max_speed_bits, 4 * W);
  rc |= cp(r->density_err_max, s->den_err_max, 4 * W);
  rc |= cp(r->projected, s->d.projected, 4 * W);
  rc |= cp(r->nonfinite, s->d.nonfinite, 4 * W);
  rc |= cp(r->emitter_overflow, s->emit_overflow, 4 * W);
  rc |= cp(r->density_tol, s->den_tol, 4 * W);
  rc |= cp(r->swept, s->d.swept, 4 * W);
  if (s->warm_alloc) {
    rc |= cp(r->learned_divergence, s->d.learned, 4 * W);
    rc |= cp(r->learned_density, s->d.learned + W, 4 * W);
  } else {
    if (r->learned_divergence) std::memset(r->learned_divergence, 0, 4 * (size_t)W);
    if (r->learned_density) std::memset(r->learned_density, 0, 4 * (size_t)W);
  }
  if (rc) return ADF_ERR_CUDA;
  int merr = 0, perr = 0;
  if (s->merr) CK(cudaMemcpyAsync(&merr, s->merr, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (s->perr) CK(cudaMemcpyAsync(&perr, s->perr, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (merr) return fail(ADF_ERR_STATE, "warm-start network: a tensor-core wait expired; the learned starts are invalid");
  if (perr)
    return fail(ADF_ERR_STATE, "pressure solve: a grid-barrier wait of the persistent CG solve expired; the step's "
                               "results are invalid");
  return ADF_OK;
}

// Buffers of the learned start and of the feature record, allocated once (outside any step).
static int ensure_warm(adf_solver* s) {
  if (s->warm_alloc) return ADF_OK;
  DevP& d = s->d;
  const size_t n = (size_t)std::max(s->n, 1), W = (size_t)std::max(s->W, 1);
  int rc = 0;
  rc |= s->alloc(&d.feat, 16 * n);
  rc |= s->alloc(&d.pred_kv, n);
  rc |= s->alloc(&d.pred_kd, n);
  rc |= s->alloc(&d.kappa2, n);
  rc |= s->alloc(&d.kr2, n);
  rc |= s->alloc(&d.acc2, n);
  rc |= s->alloc(&d.err2, n);
  rc |= s->alloc(&d.use_l, W);
  rc |= s->alloc(&d.learned, 2 * W);
  rc |= s->alloc(&d.probe_skip, W);
  rc |= s->alloc(&d.probe_gap, 2 * W);
  rc |= s->alloc(&d.probe_wait, 2 * W);
  rc |= s->alloc(&s->cw2, W);
  rc |= s->alloc(&s->cseg2, (size_t)W + 1);
  rc |= s->alloc(&s->n_cw2, 1);
  rc |= s->alloc(&s->warm_need, W);
  rc |= s->alloc(&d.sum_c, W);
  rc |= s->alloc(&d.sum_l, W);
  rc |= s->alloc(&d.max_c, W);
  rc |= s->alloc(&d.max_l, W);
  rc |= s->alloc(&s->mw1, (size_t)mlp::NH * mlp::NF);
  rc |= s->alloc(&s->mw2, (size_t)mlp::NH * mlp::NH);
  rc |= s->alloc(&s->mparams, (size_t)mlp::N_PARAMS);
  rc |= s->alloc(&s->mnorm, (size_t)36);
  rc |= s->alloc(&s->merr, (size_t)1);
  if (rc) return fail(ADF_ERR_CUDA, "learned warm start: " + g_err);
  CK(cudaMemset(d.feat, 0, sizeof(float) * 16 * n));
  CK(cudaMemset(d.learned, 0, sizeof(int) * 2 * W));
  {
    std::vector<int> ones(2 * (size_t)W, 1);
    CK(cudaMemcpy(d.probe_gap, ones.data(), sizeof(int) * 2 * W, cudaMemcpyHostToDevice));
    CK(cudaMemset(d.probe_wait, 0, sizeof(int) * 2 * W));
    CK(cudaMemset(d.probe_skip, 0, sizeof(int) * W));
  }
  CK(cudaMemset(s->merr, 0, sizeof(int)));
  CK(cudaFuncSetAttribute(k_mlp_warm, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::FW_SMEM));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  const long long tiles = ((long long)s->n + mlp::TILE - 1) / mlp::TILE;
  s->mlp_grid = (int)std::max<long long>(1, std::min<long long>(tiles, 4LL * sms));
  s->warm_alloc = true;
  return ADF_OK;
}

int adf_set_warm_model(adf_solver* s, const adf_mlp* m, const float* norm) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_warm_model: null solver");
  CK(cudaSetDevice(s->device));
  ++s->table_version;  // cached step graphs hold the other start
  if (!m) {
    s->warm_on = false;
    return ADF_OK;
  }
  if (!norm) return fail(ADF_ERR_VALUE, "adf_set_warm_model: the feature and target statistics are required");
  if (m->device != s->device) return fail(ADF_ERR_VALUE, "adf_set_warm_model: network and solver on different devices");
  int rc = ensure_warm(s);
  if (rc) return rc;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(s->mw1, m->w1b, sizeof(__nv_bfloat16) * mlp::NH * mlp::NF, cudaMemcpyDeviceToDevice));
  CK(cudaMemcpy(s->mw2, m->w2b, sizeof(__nv_bfloat16) * mlp::NH * mlp::NH, cudaMemcpyDeviceToDevice));
  CK(cudaMemcpy(s->mparams, m->w, sizeof(float) * mlp::N_PARAMS, cudaMemcpyDeviceToDevice));
  CK(cudaMemcpy(s->mnorm, norm, sizeof(float) * 36, cudaMemcpyHostToDevice));
  s->warm_on = true;
  return ADF_OK;
}

int adf_prime(adf_solver* s, const float* q, const float* qd, double dt, double tol, int max_it, int32_t* iters,
              void* stream) {
  if (!s || !q || !qd) return fail(ADF_ERR_VALUE, "adf_prime: null argument");
  if (!(dt > 0.0) || !(tol > 0.0) || max_it < 1) return fail(ADF_ERR_VALUE, "adf_prime: dt, tol and max_it must be > 0");
  if (iters) *iters = 0;
  if (s->n == 0) return ADF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(s->device));
  DevP P = s->d;
  P.q = const_cast<float*>(q);  // read only: the sort gathers from them; nothing is written back
  P.qd = const_cast<float*>(qd);
  P.f_ext = nullptr;
  P.dt = (float)dt;
  P.n_sinks = 0;
  P.min_nb = 0.0f;
  P.max_it = max_it;
  int rc = prepare(s, P, st);
  if (rc) return rc;
  run_tk(s, TK_XSPH, st, P);  // the velocity one gravity step adds (no pressure guess yet)
  std::swap(P.vel, P.vel2);
  const adf_params saved = s->prm;
  const bool warm = s->warm_on, rec = s->feat_rec;
  s->prm.tol_div = tol;
  s->prm.max_it = max_it;
  s->prm.warm_div = 1.0;
  s->prm.max_error_factor = 1.0e9;
  s->warm_on = s->feat_rec = false;
  rc = solve(s, P, 0, dt, st, false);
  s->prm = saved;
  s->warm_on = warm;
  s->feat_rec = rec;
  if (rc) return rc;
  LAUNCH(s, k_prime_gather, blocks(s->n), BLOCK, st, P);
  LAUNCH(s, k_prime_store, blocks(s->n), BLOCK, st, s->n, (float)dt, P.kv, P.kd);
  rc = check_launch();
  if (rc) return rc;
  if (iters) {
    std::vector<int> it(std::max(s->W, 1), 0);
    CK(cudaMemcpyAsync(it.data(), s->iters_div, sizeof(int) * s->W, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int w = 0; w < s->W; ++w) *iters = std::max(*iters, it[w]);
  }
  return ADF_OK;
}

int adf_iteration_work(adf_solver* s, int64_t* particles, void* stream) {
  if (!s || !particles) return fail(ADF_ERR_VALUE, "adf_iteration_work: null argument");
  CK(cudaSetDevice(s->device));
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, s->d.iter_work, sizeof(v), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  *particles = (int64_t)v;
  return ADF_OK;
}

int adf_set_autotune(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_autotune: null solver");
  for (int k = 0; k < TK_COUNT; ++k) {
    s->tune[k] = default_cfg(k);
    s->tuned[k] = false;
    s->tune_ms[k] = 0.0f;
  }
  s->tune_pending = enable != 0;
  ++s->table_version;
  return ADF_OK;
}

int adf_set_tuned_config(adf_solver* s, int kernel, int block, int nb) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_tuned_config: null solver");
  if (kernel < 0 || kernel >= TK_COUNT) return fail(ADF_ERR_VALUE, "adf_set_tuned_config: kernel out of range");
  const bool ok = kernel == TK_LISTS ? (block == 32 * LU_WARPS && (nb == 16 || nb == 32))
                                     : ((block == 128 || block == 256) && (nb == 4 || nb == 8 || nb == 16));
  if (!ok) return fail(ADF_ERR_VALUE, "adf_set_tuned_config: not one of the tuner's candidates");
  s->tune[kernel] = TuneCfg{block, nb};
  s->tuned[kernel] = true;
  s->tune_ms[kernel] = 0.0f;
  ++s->table_version;
  return ADF_OK;
}

int adf_tuned_configs(adf_solver* s, int32_t* block, int32_t* nb, float* ms) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_tuned_configs: null solver");
  for (int k = 0; k < TK_COUNT; ++k) {
    if (block) block[k] = s->tune[k].block;
    if (nb) nb[k] = s->tune[k].nb;
    if (ms) ms[k] = s->tuned[k] ? s->tune_ms[k] : -1.0f;
  }
  return ADF_OK;
}

int adf_set_halo(adf_solver* s, int mode) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_halo: null solver");
  if (mode < -1 || mode > 1) return fail(ADF_ERR_VALUE, "adf_set_halo: mode is -1 (tuned), 0 (off) or 1 (on)");
  if (mode != 0 && s->d.halo_f == nullptr) {  // the halo buffers exist only once halos may run: 6 bytes a row entry
    CK(cudaSetDevice(s->device));
    const size_t n = (size_t)std::max(s->n, 1), items = (size_t)s->halo_items;
    int* hn = nullptr;
    int* hi = nullptr;
    unsigned short* hr = nullptr;
    float* hf = nullptr;
    if (s->alloc(&hn, items) != ADF_OK || s->alloc(&hi, items * HALO_CAP) != ADF_OK ||
        s->alloc(&hr, (size_t)s->K * n) != ADF_OK || s->alloc(&hf, (size_t)s->K * n) != ADF_OK)
      return fail(ADF_ERR_CAPACITY, "adf_set_halo: out of device memory for the item halos");
    s->d.halo_n = hn;  // all four or none (what did get allocated is freed with the solver)
    s->d.halo_idx = hi;
    s->d.halo_row = hr;
    s->d.halo_f = hf;
  }
  s->halo_mode = mode;
  for (int id : {TK_ACCEL, TK_JACOBI}) {
    if (mode >= 0) s->tune[id].halo = mode;
    else if (!s->tuned[id]) s->tune[id].halo = 0;
  }
  ++s->table_version;  // cached step graphs hold the other kernels
  return ADF_OK;
}

int adf_halo_stats(adf_solver* s, int32_t* in_use, int64_t* stats, void* stream) {
  if (!s || !in_use || !stats) return fail(ADF_ERR_VALUE, "adf_halo_stats: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  in_use[0] = s->tune[TK_ACCEL].halo;
  in_use[1] = s->tune[TK_JACOBI].halo;
  for (int k = 0; k < 4; ++k) stats[k] = 0;
  if (!s->built || !halo_needed(s)) return ADF_OK;
  std::vector<int> h((size_t)s->halo_items);
  CK(cudaMemcpyAsync(h.data(), s->d.halo_n, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int v : h) {
    if (v > 0) {
      ++stats[0];
      stats[2] += v;
      stats[3] = std::max<int64_t>(stats[3], v);
    } else if (v < 0) {
      ++stats[1];
    }
  }
  return ADF_OK;
}

int adf_set_persistent(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_persistent: null solver");
  if (s->persist_on != (enable != 0)) ++s->table_version;
  s->persist_on = enable != 0;
  return ADF_OK;
}

int adf_set_barrier_wait(adf_solver* s, long long polls, int extra_arrivals) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_barrier_wait: null solver");
  if (polls < 1 || extra_arrivals < 0) return fail(ADF_ERR_VALUE, "adf_set_barrier_wait: polls >= 1, extra >= 0");
  s->persist_wait = polls;
  s->persist_extra = (unsigned)extra_arrivals;
  ++s->table_version;
  return ADF_OK;
}

int adf_clear_status(adf_solver* s) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_clear_status: null solver");
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  CK(cudaMemset(s->perr, 0, sizeof(int)));
  if (s->merr) CK(cudaMemset(s->merr, 0, sizeof(int)));
  // a launch that left at a barrier may have left the reductions' tickets counted part way
  CK(cudaMemset(s->d.wdone, 0, sizeof(int) * std::max(s->W, 1)));
  CK(cudaMemset(s->d.gdone, 0, sizeof(unsigned)));
  return ADF_OK;
}

int adf_set_warm_judging(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_warm_judging: null solver");
  if (s->judge != (enable != 0)) ++s->table_version;
  s->judge = enable != 0;
  return ADF_OK;
}

int adf_set_feature_recording(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_feature_recording: null solver");
  CK(cudaSetDevice(s->device));
  if (enable) {
    int rc = ensure_warm(s);
    if (rc) return rc;
  }
  if (s->feat_rec != (enable != 0)) ++s->table_version;
  s->feat_rec = enable != 0;
  return ADF_OK;
}

int adf_warm_features(adf_solver* s, float* out, void* stream) {
  if (!s || !out) return fail(ADF_ERR_VALUE, "adf_warm_features: null argument");
  if (!s->warm_alloc || !s->built) return fail(ADF_ERR_STATE, "adf_warm_features: no features recorded yet");
  if (s->n == 0) return ADF_OK;
  CK(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(out, 0, sizeof(float) * 16 * (size_t)s->n, st));
  const DevP& d = s->d;
  LAUNCH(s, k_unsort_n, blocks(s->n), BLOCK, st, s->n, (const int*)d.nfw, (const int*)d.id_of, (const float*)d.feat,
         16, 0, out, 16);
  return check_launch();
}

int adf_active_mass(adf_solver* s, int64_t* out_host, void* stream) {
  if (!s || !out_host) return fail(ADF_ERR_VALUE, "adf_active_mass: null argument");
  CK(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int W = std::max(s->W, 1);
  CK(cudaMemsetAsync(s->tmp_mass, 0, 8 * W, st));
  if (s->n > 0) LAUNCH(s, k_active_mass, blocks(s->n), BLOCK, st, s->d, s->tmp_mass);
  if (s->W) CK(cudaMemcpyAsync(out_host, s->tmp_mass, 8 * s->W, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return check_launch();
}

int adf_get_warm_starts(adf_solver* s, float* kv, float* kd, void* stream) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_get_warm_starts: null solver");
  cudaStream_t st = (cudaStream_t)stream;
  if (kv) CK(cudaMemcpyAsync(kv, s->d.kv, sizeof(float) * s->n, cudaMemcpyDeviceToDevice, st));
  if (kd) CK(cudaMemcpyAsync(kd, s->d.kd, sizeof(float) * s->n, cudaMemcpyDeviceToDevice, st));
  return ADF_OK;
}

int adf_set_warm_starts(adf_solver* s, const float* kv, const float* kd, void* stream) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_warm_starts: null solver");
  cudaStream_t st = (cudaStream_t)stream;
  if (kv) CK(cudaMemcpyAsync(s->d.kv, kv, sizeof(float) * s->n, cudaMemcpyDeviceToDevice, st));
  if (kd) CK(cudaMemcpyAsync(s->d.kd, kd, sizeof(float) * s->n, cudaMemcpyDeviceToDevice, st));
  return ADF_OK;
}

int adf_reset(adf_solver* s, const uint8_t* world_mask, const int32_t* flags0, const int8_t* phase0, void* stream) {
  if (!s || !flags0 || !phase0) return fail(ADF_ERR_VALUE, "adf_reset: null argument");
  const int W = s->W;
  std::vector<uint8_t> mask(std::max(W, 1), 1);
  if (world_mask)
    for (int w = 0; w < W; ++w) mask[w] = world_mask[w] ? 1 : 0;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpy(s->mask_d, mask.data(), std::max(W, 1), cudaMemcpyHostToDevice));
  if (s->n > 0) LAUNCH(s, k_reset, blocks(s->n), BLOCK, st, s->d, s->mask_d, flags0, phase0);
  CK(cudaStreamSynchronize(st));
  auto zero_masked = [&](void* dev, size_t elem) -> int {
    std::vector<unsigned char> h(elem * std::max(W, 1));
    CK(cudaMemcpy(h.data(), dev, elem * W, cudaMemcpyDeviceToHost));
    for (int w = 0; w < W; ++w)
      if (mask[w]) std::memset(h.data() + elem * w, 0, elem);
    CK(cudaMemcpy(dev, h.data(), elem * W, cudaMemcpyHostToDevice));
    return ADF_OK;
  };
  if (W > 0) {
    int rc = 0;
    rc |= zero_masked(s->d.escaped, 4) | zero_masked(s->d.projected, 4) | zero_masked(s->d.overflow, 4);
    rc |= zero_masked(s->d.swept, 4);
    rc |= zero_masked(s->d.nonfinite, 4) | zero_masked(s->emit_overflow, 4) | zero_masked(s->mass_in, 8);
    rc |= zero_masked(s->d.mass_out, 8);
    if (rc) return rc;
    LAUNCH(s, k_port_reset, W, 256, st, W, s->ws_d, s->mask_d, s->port_stack0, s->port_top0, s->port_stack,
           s->port_top, s->port_absorbed, s->port_emitted, s->port_retired, s->port_taken, s->port_granted);
    if (s->warm_alloc)
      LAUNCH(s, k_probe_reset, blocks(W), BLOCK, st, W, s->mask_d, s->d.probe_gap, s->d.probe_wait);
    const int npe = (int)s->pe_world_h.size();
    if (npe > 0)
      LAUNCH(s, k_patch_reset, blocks(npe), BLOCK, st, npe, s->pe_world_d, s->mask_d, s->pe_pending_d, s->pe_fired_d);
    CK(cudaStreamSynchronize(st));
  }
  const int ne = (int)s->em_h.size();
  if (ne > 0) {  // emitters.rewind: layer clock and cursor of the masked worlds' emitters back to 0
    std::vector<float> t(ne);
    std::vector<int> c(ne);
    CK(cudaMemcpy(t.data(), s->t_acc_d, sizeof(float) * ne, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(c.data(), s->cursor_d, sizeof(int) * ne, cudaMemcpyDeviceToHost));
    for (int e = 0; e < ne; ++e)
      if (mask[s->em_h[e].world]) {
        t[e] = 0.0f;
        c[e] = 0;
      }
    CK(cudaMemcpy(s->t_acc_d, t.data(), sizeof(float) * ne, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->cursor_d, c.data(), sizeof(int) * ne, cudaMemcpyHostToDevice));
  }
  return check_launch();
}

static int check_emitter(const adf_solver* s, int world, const float* xform, const float* offsets, int n_off,
                         const float* velocity, float interval, const int32_t* pool, int pool_size) {
  if (!xform || !velocity || (n_off > 0 && !offsets) || (pool_size > 0 && !pool) || n_off < 0 || pool_size < 0)
    return fail(ADF_ERR_VALUE, "adf_add_emitter: null argument or negative size");
  if (world < 0 || world >= s->W) return fail(ADF_ERR_VALUE, "add_emitter: world " + std::to_string(world) +
                                                             " out of range");
  if (!(interval > 0.0f)) return fail(ADF_ERR_VALUE, "add_emitter: interval must be > 0");
  for (int k = 0; k < pool_size; ++k)
    if (pool[k] < s->ws_host[world] || pool[k] >= s->ws_host[world + 1])
      return fail(ADF_ERR_VALUE, "add_emitter: pool particle outside the emitter's world");
  return ADF_OK;
}

static int append_emitter(adf_solver* s, int world, const float* xform, const float* offsets, int n_off,
                          const float* velocity, float interval, const int32_t* pool, int pool_size) {
  Emit e{};
  e.world = world;
  e.n_layer = n_off;
  e.pool_begin = (int)s->pool_h.size();
  e.pool_size = pool_size;
  std::memcpy(e.xform, xform, sizeof(float) * 7);
  std::memcpy(e.vel, velocity, sizeof(float) * 3);
  e.interval = interval;
  int idx = (int)s->em_h.size();
  s->em_h.push_back(e);
  s->enabled_h.push_back(1);
  for (int c = 0; c < n_off; ++c) {
    s->off_emitter_h.push_back(idx);
    s->off_rank_h.push_back(c);
    for (int a = 0; a < 3; ++a) s->off_local_h.push_back(offsets[3 * c + a]);
  }
  s->pool_h.insert(s->pool_h.end(), pool, pool + pool_size);
  return idx;
}

int adf_add_emitter(adf_solver* s, int world, const float* xform, const float* offsets, int n_off,
                    const float* velocity, float interval, const int32_t* pool, int pool_size) {
  if (!s) return -fail(ADF_ERR_VALUE, "adf_add_emitter: null solver");
  int rc = check_emitter(s, world, xform, offsets, n_off, velocity, interval, pool, pool_size);
  if (rc) return -rc;
  const int idx = append_emitter(s, world, xform, offsets, n_off, velocity, interval, pool, pool_size);
  ++s->table_version;
  rc = upload_emitters(s, idx);
  if (rc) return -rc;
  return idx;
}

int adf_add_emitters(adf_solver* s, int count, const int32_t* world, const float* xform, const int32_t* n_off,
                     const float* offsets, const float* velocity, const float* interval, const int32_t* pool_size,
                     const int32_t* pool) {
  if (!s || count < 0 || (count > 0 && (!world || !xform || !n_off || !velocity || !interval || !pool_size)))
    return -fail(ADF_ERR_VALUE, "adf_add_emitters: null argument");
  size_t oo = 0, po = 0;
  for (int k = 0; k < count; ++k) {  // every emitter is checked before any is added
    int rc = check_emitter(s, world[k], xform + 7 * (size_t)k, offsets ? offsets + 3 * oo : nullptr, n_off[k],
                           velocity + 3 * (size_t)k, interval[k], pool ? pool + po : nullptr, pool_size[k]);
    if (rc) return -fail(rc, "add_emitters[" + std::to_string(k) + "]: " + g_err);
    oo += (size_t)std::max(n_off[k], 0);
    po += (size_t)std::max(pool_size[k], 0);
  }
  const int first = (int)s->em_h.size();
  oo = po = 0;
  for (int k = 0; k < count; ++k) {
    append_emitter(s, world[k], xform + 7 * (size_t)k, offsets + 3 * oo, n_off[k], velocity + 3 * (size_t)k,
                   interval[k], pool + po, pool_size[k]);
    oo += (size_t)n_off[k];
    po += (size_t)pool_size[k];
  }
  ++s->table_version;
  int rc = upload_emitters(s, first);
  if (rc) return -rc;
  return first;
}

int adf_state_arrays(adf_solver* s, float** kv, float** kd) {
  if (!s || !kv || !kd) return fail(ADF_ERR_VALUE, "adf_state_arrays: null argument");
  *kv = s->d.kv;
  *kd = s->d.kd;
  return ADF_OK;
}

int adf_set_emitter_pool(adf_solver* s, int e, const int32_t* pool, int pool_size) {
  if (!s || (pool_size > 0 && !pool)) return fail(ADF_ERR_VALUE, "adf_set_emitter_pool: null argument");
  int ne = (int)s->em_h.size();
  if (e < 0 || e >= ne) return fail(ADF_ERR_VALUE, "set_emitter_pool: emitter " + std::to_string(e) + " does not exist");
  const int w = s->em_h[e].world;
  for (int k = 0; k < pool_size; ++k)
    if (pool[k] < s->ws_host[w] || pool[k] >= s->ws_host[w + 1])
      return fail(ADF_ERR_VALUE, "set_emitter_pool: pool particle outside the emitter's world");
  // rebuild the concatenated pool table with emitter e's new pool
  std::vector<int> pools;
  for (int k = 0; k < ne; ++k) {
    int b = (int)pools.size();
    if (k == e) pools.insert(pools.end(), pool, pool + pool_size);
    else pools.insert(pools.end(), s->pool_h.begin() + s->em_h[k].pool_begin,
                      s->pool_h.begin() + s->em_h[k].pool_begin + s->em_h[k].pool_size);
    s->em_h[k].pool_size = (int)pools.size() - b;
    s->em_h[k].pool_begin = b;
  }
  s->pool_h.swap(pools);
  ++s->table_version;
  return upload_emitters(s, ne);
}

int adf_emitter_state(adf_solver* s, float* t_acc, int32_t* cursor) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_emitter_state: null solver");
  int ne = (int)s->em_h.size();
  if (ne == 0) return ADF_OK;
  CK(cudaDeviceSynchronize());
  if (t_acc) CK(cudaMemcpy(t_acc, s->t_acc_d, sizeof(float) * ne, cudaMemcpyDeviceToHost));
  if (cursor) CK(cudaMemcpy(cursor, s->cursor_d, sizeof(int) * ne, cudaMemcpyDeviceToHost));
  return ADF_OK;
}

int adf_set_emitter_enabled(adf_solver* s, int e, int enabled) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_set_emitter_enabled: null solver");
  int ne = (int)s->em_h.size();
  if (e < 0 || e >= ne)
    return fail(ADF_ERR_VALUE, "set_emitter_enabled: emitter " + std::to_string(e) + " does not exist (" +
                                   std::to_string(ne) + " emitters)");
  s->enabled_h[e] = enabled ? 1 : 0;
  int v = s->enabled_h[e];
  CK(cudaMemcpy(s->enabled_d + e, &v, sizeof(int), cudaMemcpyHostToDevice));
  return ADF_OK;
}

int adf_add_sink(adf_solver* s, int world, const float* xform, const float* half) {
  if (!s || !xform || !half) return -fail(ADF_ERR_VALUE, "adf_add_sink: null argument");
  if (world < 0 || world >= s->W) return -fail(ADF_ERR_VALUE, "add_sink: world " + std::to_string(world) +
                                                                 " out of range");
  Sink k{};
  k.world = world;
  std::memcpy(k.xform, xform, sizeof(float) * 7);
  std::memcpy(k.half, half, sizeof(float) * 3);
  s->sinks_h.push_back(k);
  ++s->table_version;
  if (s->sinks_d) cudaFree(s->sinks_d);
  s->sinks_d = nullptr;
  if (dalloc(&s->sinks_d, s->sinks_h.size())) return -ADF_ERR_CUDA;
  cudaError_t e = cudaMemcpy(s->sinks_d, s->sinks_h.data(), sizeof(Sink) * s->sinks_h.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return -fail(ADF_ERR_CUDA, cudaGetErrorString(e));
  return (int)s->sinks_h.size() - 1;
}

int adf_neighbor_rows(adf_solver* s, int32_t* rows, int32_t* count, void* stream) {
  if (!s || !rows || !count) return fail(ADF_ERR_VALUE, "adf_neighbor_rows: null argument");
  if (!s->built) return fail(ADF_ERR_STATE, "adf_neighbor_rows: no lists yet (step or density_ratio first)");
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  const int n = s->n, K = s->K;
  int nfw[2];
  CK(cudaMemcpy(nfw, s->d.nfw, sizeof(nfw), cudaMemcpyDeviceToHost));
  std::vector<int> id(n), cnt(n), nbr((size_t)K * n);
  CK(cudaMemcpy(id.data(), s->d.id_of, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(cnt.data(), s->d.cnt, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nbr.data(), s->d.nbr, sizeof(int) * (size_t)K * n, cudaMemcpyDeviceToHost));
  std::fill(rows, rows + (size_t)n * K, -1);
  std::fill(count, count + n, 0);
  for (int p = 0; p < nfw[0]; ++p) {
    int i = id[p];
    count[i] = cnt[p];
    for (int k = 0; k < cnt[p]; ++k) rows[(size_t)i * K + k] = id[nbr[(size_t)k * n + p]];
  }
  return ADF_OK;
}

int adf_debug_field(adf_solver* s, const char* name, float* out, void* stream) {
  if (!s || !name || !out) return fail(ADF_ERR_VALUE, "adf_debug_field: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const DevP& d = s->d;
  // "name:k" reads slot k of a slot field (k = 0 without a suffix)
  std::string base(name);
  int slot = 0;
  const size_t colon = base.find(':');
  if (colon != std::string::npos) {
    const std::string suffix = base.substr(colon + 1);
    base = base.substr(0, colon);
    if (suffix.empty() || suffix.size() > 1 || suffix[0] < '0' || suffix[0] > '9' || base.rfind("slot_", 0) != 0)
      return fail(ADF_ERR_VALUE, std::string("adf_debug_field: bad slot suffix in ") + name);
    slot = suffix[0] - '0';
    if (slot >= d.slot_cap)
      return fail(ADF_ERR_VALUE, std::string("adf_debug_field: ") + name + ": this model has " +
                                     std::to_string(d.slot_cap) + " slot(s) per particle");
  }
  if (base == "slot_shape" || base == "slot_count") {
    CK(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)s->n, st));
    LAUNCH(s, k_slot_info, blocks(s->n), BLOCK, st, d, base == "slot_count" ? -1 : slot, out);
    return check_launch();
  }
  const size_t so = (size_t)slot * s->n * 4;  // floats to slot k of a float4 slot array
  struct F { const char* nm; const float* ptr; int stride, comp, ncomp; };
  const F fields[] = {
      {"ratio", d.ratio, 1, 0, 1}, {"alpha", d.alpha, 1, 0, 1}, {"neff", d.neff, 1, 0, 1}, {"reg", d.reg, 1, 0, 1},
      {"src", d.src, 1, 0, 1}, {"kappa", d.kappa, 1, 0, 1}, {"lower", d.lower, 1, 0, 1},
      {"slot_psi", (const float*)d.slot_g + so, 4, 3, 1}, {"slot_phi", (const float*)d.slot_vb + so, 4, 3, 1},
      {"acc", (const float*)d.acc, 4, 0, 3}, {"slot_g", (const float*)d.slot_g + so, 4, 0, 3},
      {"slot_vb", (const float*)d.slot_vb + so, 4, 0, 3}, {"slot_n", (const float*)d.slot_n + so, 4, 0, 3},
      {"pred_kv", d.pred_kv, 1, 0, 1}, {"pred_kd", d.pred_kd, 1, 0, 1}};
  for (const F& f : fields) {
    if (base != f.nm) continue;
    if (!f.ptr) return fail(ADF_ERR_STATE, std::string("adf_debug_field: ") + name + " is not recorded");
    CK(cudaMemsetAsync(out, 0, sizeof(float) * f.ncomp * (size_t)s->n, st));
    LAUNCH(s, k_unsort_n, blocks(s->n), BLOCK, st, s->n, d.nfw, d.id_of, f.ptr, f.stride, f.comp, out, f.ncomp);
    return check_launch();
  }
  if (std::strcmp(name, "err") == 0) {
    CK(cudaMemcpyAsync(out, d.err_orig, sizeof(float) * s->n, cudaMemcpyDeviceToDevice, st));
    return ADF_OK;
  }
  return fail(ADF_ERR_VALUE, std::string("adf_debug_field: unknown field ") + name);
}

int adf_skin_flags(adf_solver* s, int32_t* flags, void* stream) {
  if (!s || !flags) return fail(ADF_ERR_VALUE, "adf_skin_flags: null argument");
  if (!s->d.skin_on) return fail(ADF_ERR_STATE, "adf_skin_flags: the solver has no skin (params.skin = 0)");
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  if (s->W > 0) CK(cudaMemcpy(flags, s->d.skin_flag, sizeof(int) * s->W, cudaMemcpyDeviceToHost));
  return ADF_OK;
}

int adf_world_sum(adf_solver* s, const float* values, double* out_sum, float* out_max, void* stream) {
  if (!s || !values || !out_sum || !out_max) return fail(ADF_ERR_VALUE, "adf_world_sum: null argument");
  if (s->W == 0) return ADF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const DevP& P = s->d;
  if (P.n_chunks > 0)
    LAUNCH(s, k_chunk_sum, (P.n_chunks + 7) / 8, 256, st, values, P.chunk_begin, P.chunk_end, P.n_chunks, P.part_sum,
           P.part_max);
  LAUNCH(s, k_world_check, s->W, 256, st, P, 0, out_sum, out_max);
  return check_launch();
}

int64_t adf_kernel_launches(const adf_solver* s) {
  if (!s) return 0;
  unsigned long long runs = 0;
  if (s->body_runs) cudaMemcpy(&runs, s->body_runs, sizeof(runs), cudaMemcpyDeviceToHost);
  return s->launches + s->body_kernels * (long long)runs;
}

int adf_profile_enable(adf_solver* s, int enable) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_profile_enable: null solver");
  if (enable && s->prof_pool.empty()) {
    s->prof_pool.resize(16384);
    for (auto& e : s->prof_pool) CK(cudaEventCreate(&e));
  }
  s->prof_on = enable != 0;
  return ADF_OK;
}

int adf_profile_read(adf_solver* s, double* ms, int64_t* launches) {
  if (!s || !ms || !launches) return fail(ADF_ERR_VALUE, "adf_profile_read: null argument");
  for (int k = 0; k < ADF_PROF_KINDS; ++k) {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  if (!s->prof_marks.empty()) CK(cudaEventSynchronize(s->prof_pool[s->prof_marks.back().second + 1]));
  for (auto& m : s->prof_marks) {
    float t = 0.0f;
    CK(cudaEventElapsedTime(&t, s->prof_pool[m.second], s->prof_pool[m.second + 1]));
    ms[m.first] += t;
    launches[m.first] += 1;
  }
  s->prof_marks.clear();
  s->prof_used = 0;
  return ADF_OK;
}

int adf_list_stats(adf_solver* s, int32_t* fluid, int64_t* entries, void* stream) {
  if (!s || !fluid || !entries) return fail(ADF_ERR_VALUE, "adf_list_stats: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (!s->list_entries) CK(cudaMalloc(&s->list_entries, sizeof(long long)));
  CK(cudaMemsetAsync(s->list_entries, 0, sizeof(long long), st));
  if (s->n > 0) LAUNCH(s, k_count_entries, blocks(s->n), BLOCK, st, s->n, s->d.nfw, s->d.cnt, s->list_entries);
  CK(cudaStreamSynchronize(st));
  int nfw[2];
  CK(cudaMemcpy(nfw, s->d.nfw, sizeof(nfw), cudaMemcpyDeviceToHost));
  long long e = 0;
  CK(cudaMemcpy(&e, s->list_entries, sizeof(e), cudaMemcpyDeviceToHost));
  *fluid = nfw[0];
  *entries = e;
  return check_launch();
}

int adf_add_patch_emitter(adf_solver* s, int entries, const int32_t* world, const int32_t* count,
                          const int32_t* pool_ids, const float* points, const float* velocity) {
  if (!s || entries < 0 || !velocity || (entries > 0 && (!world || !count)))
    return -fail(ADF_ERR_VALUE, "adf_add_patch_emitter: null argument");
  CK_NEG(cudaSetDevice(s->device));
  long long total = 0;
  for (int e = 0; e < entries; ++e) {
    if (world[e] < 0 || world[e] >= s->W) return -fail(ADF_ERR_VALUE, "add_patch_emitter: world out of range");
    if (count[e] < 0) return -fail(ADF_ERR_VALUE, "add_patch_emitter: negative point count");
    total += count[e];
  }
  if (total > 0 && (!pool_ids || !points)) return -fail(ADF_ERR_VALUE, "adf_add_patch_emitter: null argument");
  for (long long k = 0; k < total; ++k)
    if (pool_ids[k] < 0 || pool_ids[k] >= s->n) return -fail(ADF_ERR_VALUE, "add_patch_emitter: pool id out of range");
  const int E0 = (int)s->pe_world_h.size(), gid = (int)s->pg_first_h.size() - 1;
  std::vector<int> pend(E0, 0), fired(E0, 0);
  if (E0 > 0) {  // the earlier groups keep their armed / fired state
    CK_NEG(cudaMemcpy(pend.data(), s->pe_pending_d, sizeof(int) * E0, cudaMemcpyDeviceToHost));
    CK_NEG(cudaMemcpy(fired.data(), s->pe_fired_d, sizeof(int) * E0, cudaMemcpyDeviceToHost));
  }
  for (int e = 0; e < entries; ++e) {
    s->pe_world_h.push_back(world[e]);
    s->pe_count_h.push_back(count[e]);
    s->pe_begin_h.push_back((int)s->pp_pool_h.size());
    s->pe_group_h.push_back(gid);
    for (int k = 0; k < count[e]; ++k) {
      s->pp_pool_h.push_back(pool_ids[0]);
      pool_ids += 1;
      for (int a = 0; a < 3; ++a) s->pp_points_h.push_back(points[a]);
      points += 3;
    }
    pend.push_back(0);
    fired.push_back(0);
  }
  s->pg_first_h.push_back((int)s->pe_world_h.size());
  for (int a = 0; a < 3; ++a) s->pg_vel_h.push_back(velocity[a]);
  for (void* q : {(void*)s->pe_world_d, (void*)s->pe_count_d, (void*)s->pe_begin_d, (void*)s->pe_group_d,
                  (void*)s->pe_pending_d, (void*)s->pe_fired_d, (void*)s->pp_pool_d, (void*)s->pp_points_d,
                  (void*)s->pg_vel_d})
    if (q) cudaFree(q);
  const size_t E = s->pe_world_h.size(), NP = s->pp_pool_h.size(), G = s->pg_first_h.size() - 1;
  int rc = dalloc(&s->pe_world_d, E) | dalloc(&s->pe_count_d, E) | dalloc(&s->pe_begin_d, E) |
           dalloc(&s->pe_group_d, E) | dalloc(&s->pe_pending_d, E) | dalloc(&s->pe_fired_d, E) |
           dalloc(&s->pp_pool_d, NP) | dalloc(&s->pp_points_d, 3 * NP) | dalloc(&s->pg_vel_d, 3 * G);
  if (rc) return -fail(ADF_ERR_CUDA, "patch emitter tables: cudaMalloc failed");
  auto up = [&](void* d, const void* h, size_t bytes) -> int {
    if (bytes) CK(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
    return ADF_OK;
  };
  rc = up(s->pe_world_d, s->pe_world_h.data(), 4 * E) | up(s->pe_count_d, s->pe_count_h.data(), 4 * E) |
       up(s->pe_begin_d, s->pe_begin_h.data(), 4 * E) | up(s->pe_group_d, s->pe_group_h.data(), 4 * E) |
       up(s->pe_pending_d, pend.data(), 4 * E) | up(s->pe_fired_d, fired.data(), 4 * E) |
       up(s->pp_pool_d, s->pp_pool_h.data(), 4 * NP) | up(s->pp_points_d, s->pp_points_h.data(), 12 * NP) |
       up(s->pg_vel_d, s->pg_vel_h.data(), 12 * G);
  if (rc) return -ADF_ERR_CUDA;
  ++s->table_version;  // step graphs recorded before lack the patch launches
  return gid;
}

int adf_trigger(adf_solver* s, int pid, const void* world_flags, int flags_bool, void* stream) {
  if (!s || !world_flags) return fail(ADF_ERR_VALUE, "adf_trigger: null argument");
  if (pid < 0 || pid >= (int)s->pg_first_h.size() - 1)
    return fail(ADF_ERR_VALUE, "trigger: no patch emitter " + std::to_string(pid));
  const int e0 = s->pg_first_h[pid], e1 = s->pg_first_h[pid + 1];
  if (e1 == e0) return ADF_OK;
  LAUNCH(s, k_patch_trigger, blocks(e1 - e0), BLOCK, (cudaStream_t)stream, e0, e1, world_flags, flags_bool ? 1 : 0,
         s->pe_world_d, s->pe_fired_d, s->pe_pending_d);
  return check_launch();
}

int adf_get_state_storage(adf_solver* s, adf_state_storage* out) {
  if (!s || !out) return fail(ADF_ERR_VALUE, "adf_get_state_storage: null argument");
  out->warm_probe_gap = s->warm_alloc ? s->d.probe_gap : nullptr;
  out->warm_probe_wait = s->warm_alloc ? s->d.probe_wait : nullptr;
  out->n_patch_entries = (int)s->pe_world_h.size();
  out->patch_pending = s->pe_pending_d;
  out->patch_fired = s->pe_fired_d;
  out->patch_world = s->pe_world_d;
  out->mass_in = (int64_t*)s->mass_in;
  out->mass_out = (int64_t*)s->d.mass_out;
  out->escaped = s->d.escaped;
  const int ne = (int)s->em_h.size();
  out->n_emitters = ne;
  out->emit_t = ne ? s->t_acc_d : nullptr;
  out->emit_cursor = ne ? s->cursor_d : nullptr;
  out->emit_world = ne ? s->em_world_d : nullptr;
  out->port_stack = s->port_stack;
  out->port_top = s->port_top;
  out->port_absorbed = s->port_absorbed;
  out->port_emitted = s->port_emitted;
  out->port_retired = s->port_retired;
  out->port_taken = s->port_taken;
  out->port_granted = s->port_granted;
  return ADF_OK;
}

int adf_port_take(adf_solver* s, float* qd, const int32_t* mask, int keep, void* stream) {
  if (!s || (s->n > 0 && (!qd || !mask))) return fail(ADF_ERR_VALUE, "adf_port_take: null argument");
  if (s->W == 0 || s->n == 0) return ADF_OK;
  LAUNCH(s, k_port_take, s->W, 256, stream, s->ws_d, mask, keep ? 1 : 0, s->d.flags, s->d.phase, s->d.mass, qd,
         s->port_stack, s->port_top, s->port_taken, keep ? s->port_absorbed : s->port_retired, s->d.mass_out);
  return check_launch();
}

int adf_port_emit(adf_solver* s, float* q, float* qd, const float* pos, const float* vel, int R,
                  const int32_t* n_req, void* stream) {
  if (!s) return fail(ADF_ERR_VALUE, "adf_port_emit: null solver");
  if (R < 0) return fail(ADF_ERR_VALUE, "adf_port_emit: negative request capacity");
  if (s->W == 0 || s->n == 0) return ADF_OK;
  if (!q || !qd || !n_req || (R > 0 && (!pos || !vel))) return fail(ADF_ERR_VALUE, "adf_port_emit: null argument");
  LAUNCH(s, k_port_emit, s->W, 256, stream, s->ws_d, pos, vel, R, n_req, q, qd, s->d.flags, s->d.phase, s->d.mass,
         s->port_stack, s->port_top, s->port_granted, s->port_emitted, s->mass_in);
  return check_launch();
}

int adf_energy(adf_solver* s, const float* q, const float* qd, const double* z_ref, double* out, void* stream) {
  if (!s || !z_ref || !out || (s->n > 0 && (!q || !qd))) return fail(ADF_ERR_VALUE, "adf_energy: null argument");
  if (s->W == 0) return ADF_OK;
  const DevP& P = s->d;
  if (P.n_chunks > 0) LAUNCH(s, k_energy_chunk, P.n_chunks, 256, stream, P, q, qd, z_ref);
  LAUNCH(s, k_world_check, s->W, 256, stream, P, 0, out, s->energy_max);
  return check_launch();
}

int adf_stable_dt(adf_solver* s, const float* qd, double cfl, double dt_min, double dt_max, float* out,
                  void* stream) {
  if (!s || !out || (s->n > 0 && !qd)) return fail(ADF_ERR_VALUE, "adf_stable_dt: null argument");
  if (s->W == 0) return ADF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(s->speed_bits, 0, sizeof(int) * s->W, st));
  if (s->n > 0) LAUNCH(s, k_speed_max, blocks(s->n), BLOCK, st, s->d, qd, s->speed_bits);
  LAUNCH(s, k_stable_dt, blocks(s->W), BLOCK, st, s->W, s->speed_bits, (float)cfl,
         (float)(2.0 * s->prm.particle_radius), (float)dt_min, (float)dt_max, out);
  return check_launch();
}

}  // extern "C"
